// The fused per-stage passes of the Taylor-Green RK3 step (miniapp ordering,
// miniapps/tgv_solver_3d/tgvsolver.F90:994-1082) and the state they act on.
#pragma once
#include "internal.h"

namespace astr {

// Geometry of one periodic box in HBM: fields are x-fastest with x pitch PX (a multiple of 16
// doubles), nodes 0..N along each axis, no halo storage (halos are index wraps).
struct BoxGeo {
  int N[3];
  int64_t st[3];   // element strides of i, j, k
  int64_t fs;      // elements per field
  double rd[3];    // 1/dx, 1/dy, 1/dz
};

// Thermodynamic constants of tgvsolver.F90:183-195 and miucal (:123-140).
struct Thermo {
  double const2, const5, const6;
  double gm1;       // gamma - 1 (= 1/const6)
  double inv_re;    // 1/Re
  double inv_prc5;  // 1/(Pr const5): heat conductivity per unit viscosity
  double reynolds, prandtl;
  double tc, tc1;   // Sutherland: tempconst = S/ref_tem, 1 + tempconst
  double mach;
};

struct PassArgs {
  BoxGeo g;
  Thermo th;
  LineOp opd, opf;          // compact derivative and filter along this pass's direction
  int dir;                  // physical direction of the lines (0 x, 1 y, 2 z)
  int dA, dB, dC;           // physical directions assigned to passes A, B, C
  int TI, LP;               // lines per CTA, tile line pitch
  int LPW;                  // lines per warp group (y and z streaming passes; 1 elsewhere)
  int FPS;                  // fields per step of A', B' and the filters: 1 (streaming) or 5
  double* q;                // 5 fields
  const double* qsave;      // 5 fields (RK update)
  double* qout;             // 5 fields (RK update output)
  double* R;                // 5 fields: the RHS being accumulated
  double* D;                // 4 fields: du, dv, dw, dT along this direction (A and B passes)
  const double* DA;         // 4 fields read by pass C
  const double* DB;
  double* VF;               // 10 fields written by pass C: G_A = VF_A - F_A (5), then G_B (5)
  int do_filter;
  int mode;                 // pass B': 0 = only R += visc_B, 1 = RK update (+ filter)
  double c1, c2, c3, dt;    // SSP-RK3 stage coefficients (mainloop.F90:350-360)
  double* partials;         // pass C at the first stage: per-CTA (tke, enstrophy, dissipation)
  double* DC;               // pass C, optional: its 4 gradients along C are also stored here
  int* err;                 // device error word: bit 0 = non-finite or non-positive density,
                            // bit 1 = a bulk copy wait ran out of polls
};

cudaError_t launch_pass(int pass, const PassArgs& a, int S, int WPL, cudaStream_t st);
int pass_tiles(int pass);
// One launch of a pass over nbox boxes of one solve layout: dargs[k] are box k's arguments
// (device memory), dcum[k] its first CTA, nctas the total.
cudaError_t launch_pass_batch(int pass, int dir, int S, int WPL, const PassArgs* dargs, const int* dcum, int nbox,
                              int nctas, int threads, size_t smem, cudaStream_t st);
size_t pass_shared_bytes(int pass, int TI, int LP, int WPL, int LPW = 1, int FPS = 5);
// Field tiles of a pass's shared memory for a launch shape (LPW lines per warp group, FPS fields
// per step of the streaming passes).
int shape_tiles(int pass, int LPW, int FPS);

// Batched diagnostics reduce: one CTA per box.
struct DiagArgs {
  const double* partials;
  int nparts;
  double* hist;
  int* counter;
  double norm;
};
cudaError_t launch_diag_reduce_batch(const DiagArgs* dargs, int nbox, cudaStream_t st);

// Final ordered reduction of the pass-C partial sums into the history buffer.
cudaError_t launch_diag_reduce(const double* partials, int nparts, double* hist, int* counter, double norm,
                               cudaStream_t st);
// Taylor-Green initial state (flowfield_init) from per-axis sin/cos tables.
cudaError_t launch_init_tgv(const BoxGeo& g, const Thermo& th, double* q, const double* tabs, cudaStream_t st);
// cflcal partial maxima: per CTA (di, dj, dk).
cudaError_t launch_cfl(const BoxGeo& g, const Thermo& th, const double* q, double* partials, int* nparts,
                       cudaStream_t st);
// Copy between a caller's Fortran array (device) and the state layout.
cudaError_t launch_pack(const BoxGeo& g, double* state, double* user, const int64_t* ushape, const int64_t* ulb,
                        int nfields, int to_state, cudaStream_t st);

enum Pass { PASS_A = 1, PASS_B = 2, PASS_C = 3, PASS_VA = 4, PASS_VB = 5, PASS_F = 6 };

constexpr int SCAN_PER_LINE = 8;   // scan scratch per line in units of WPL doubles (NV <= 4)
constexpr int SP_SOLVES = 13;      // closure tables kept per line (one per pending solve)
constexpr int SP_PER_LINE = SP_SOLVES * 2 * NSP;

// Physical directions of passes A, B, C. C is x: the heaviest pass (13 line solves and the
// stress tensor) runs on contiguous lines, where any number of lines per CTA stays coalesced.
constexpr int DIR_A = 1, DIR_B = 2, DIR_C = 0;

}  // namespace astr
