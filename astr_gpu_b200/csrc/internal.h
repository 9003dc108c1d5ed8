// Host-side internals shared by the C-ABI implementation and the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "ops.cuh"

namespace astr {

// A line operator as built on the host: the reference's compact_scheme (a, c, ac) plus the
// RHS coefficients, and the device copy of its lane tables for one (S, WPL) layout.
struct HostOp {
  int kind = OP_DERIV;
  int ntype = 3, dim = 0, first_node = 0, last_node = 0;
  bool left_phys = false, right_phys = false, no_note = false;
  std::vector<double> a, c, ac1, ac2, ac3;
  double c10[6] = {0}, ch[3][11] = {{0}}, cb[3][7] = {{0}}, c6[4] = {0}, c8[5] = {0};
  int wind = 1;                 // interface flux: +1 upwind-biased, -1 downwind-biased
  double bfac = 0.0, cfl[4] = {0};
  int nsys() const { return last_node - first_node + 1; }
};

bool build_fd_op(HostOp& op, const char* scheme, int ntype, int dim);
void build_filter_op(HostOp& op, int ntype, int dim, double alfa, double beta_halo, double beta_bound, bool note);
bool build_flux_op(HostOp& op, int scheme, int ntype, int dim, int wind, double bfac);
// Lane tables for S rows per lane and nseg segments (see ops.cuh). Returns host vector.
std::vector<double> lane_tables(const HostOp& op, int S, int nseg);

// Solve layout: S rows per lane, WPL warps per line.
struct Layout { int S, WPL; };
Layout pick_layout(int nsys_max);

// Device-resident line operator for a given layout.
struct DevOp {
  LineOp op{};
  double* dtab = nullptr;
  int S = 0, WPL = 0;
};
cudaError_t make_devop(const HostOp& h, Layout lay, DevOp& out);
// The LineOp fields of a host operator (no lane tables).
void fill_lineop(const HostOp& h, LineOp& o);
void free_devop(DevOp& d);

// Tile line pitch (doubles) for TI lines of dim+1 nodes plus halos, chosen so that line-fastest
// shared-memory accesses of a warp are free of bank conflicts.
// Tile line pitch for lines of dim + 1 nodes, TI lines per tile, S rows per lane (schemes.cu).
int tile_pitch(int dim, int TI, int S);

// Line-level API launch: op along dir over every line of an arbitrary strided array.
struct ArrDesc { int64_t s[3]; int64_t lb[3]; int64_t n[3]; int64_t fs; };
// flags: LINE_ADD accumulates into out (out += result) instead of storing; LINE_DIFF (interface
// flux only) writes scale * (fh(n) - fh(n-1)) at nodes 0..dim instead of fh(-1..dim).
enum { LINE_ADD = 1, LINE_DIFF = 2 };
cudaError_t launch_line_api(const DevOp& op, int dir, const double* f, const ArrDesc& fa, double* out,
                            const ArrDesc& oa, int nfields, double scale, cudaStream_t st, int flags = 0);

// Flow-field checkpoints (checkpoint.cu): q(n, 5) <-> the file's ro, u1, u2, u3, p, t (6 fields of
// n nodes each, contiguous), and the transfers between such a device array and the file.
cudaError_t flowfield_prims_from_q(cudaStream_t st, const double* dq, double* dprims, int64_t n, double mach,
                                   double gamma);
cudaError_t flowfield_q_from_prims(cudaStream_t st, const double* dprims, double* dq, int64_t n, double mach,
                                   double gamma);
int flowfield_write(cudaStream_t st, const double* dprims, const int64_t shape[3], int nstep, double time,
                    const char* filename, std::string& err);
int flowfield_read(cudaStream_t st, double* dprims, const int64_t shape[3], const char* filename, char mode,
                   int* nstep, double* time, std::string& err);

// Host <-> device copies of pageable host memory (checkpoint.cu): host_pageable tells whether a
// host pointer is ordinary (unregistered) memory; staged_copy moves `bytes` between such memory and
// the device through the pinned staging slots with several host threads (to_device: dst is the
// device pointer), on stream st, and returns once the copy has completed. Copies from pinned memory
// need neither: the copy engine reads it directly.
bool host_pageable(const void* p);
// A device-to-host staged copy may be limited to the node rows of a Fortran array: element
// ((m*s2 + k)*s1 + j)*s0 + i is copied only when x_lo <= i <= x_hi, y_lo <= j <= y_hi and
// z_lo <= k <= z_hi, so the caller's halo entries stay as they were.
struct RowMask {
  int64_t s0, s1, s2;
  int64_t x_lo, x_hi, y_lo, y_hi, z_lo, z_hi;
};
int staged_copy(void* dst, const void* src, size_t bytes, bool to_device, cudaStream_t st, std::string& err,
                const RowMask* mask = nullptr);
constexpr size_t STAGED_MIN_BYTES = size_t(32) << 20;   // smaller copies go through cudaMemcpyAsync

}  // namespace astr
