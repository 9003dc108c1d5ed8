// Line-level operators over arbitrary Fortran-ordered arrays: the drop-in for
//   df = fds%central(asolver, f, dim)      src/derivative.F90:22-41, 171-198
//   ff = compact_filter(afilter, f, dim)   src/filter.F90:112-144
//   fh = flux_compact(asolver, f, dim)     src/flux.F90:125-150 (interfaces -1..dim)
// applied to every line of a 3-D array along one direction; the interface flux can also leave
// its differences fh(i) - fh(i-1) at the nodes (the flux-form derivative of convrsdcmp,
// src/solver.F90:1509-1513, and of the reference's flux test, src/test.F90:755-765).
//
// One CTA takes TI lines of one field. The lines (nodes -HT..dim+HT, the halos read from the
// caller's array, zeros outside it) are staged in shared memory with asynchronous copies, all in
// flight at once: node-fastest for x lines (16-byte copies of node pairs where aligned),
// line-fastest for y/z lines (TI adjacent lines are contiguous in x, so each node of the tile is
// one 8*TI-byte row). Each group of WPL warps solves two lines together with the segmented Thomas
// of ops.cuh (their recurrences and scans interleave); results go back through the tile for
// coalesced stores.
#include "internal.h"

namespace astr {

namespace {

__device__ __forceinline__ void cp8(double* sdst, const double* gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp16(double* sdst, const double* gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// The thread's staging line and its walk over the nodes of that line: x lines give each line
// blockDim/TI consecutive threads; y/z lines give consecutive threads consecutive lines.
struct Slot {
  int l, n0, nst;
};
__device__ __forceinline__ Slot slot_of(int dir, int TI) {
  Slot s;
  if (dir == 0) {
    const int per = blockDim.x / TI;
    s.l = threadIdx.x / per;
    s.n0 = threadIdx.x - s.l * per;
    s.nst = per;
  } else {
    s.l = threadIdx.x % TI;
    s.n0 = threadIdx.x / TI;
    s.nst = blockDim.x / TI;
  }
  return s;
}

}  // namespace

// One-warp-per-line layouts launch 256-thread CTAs: bounding them for three CTAs per SM (four for
// up to 5 rows per lane, which then still need no spills) keeps 24 or 32 warps resident instead
// of the 16 that their register use would otherwise allow.
template <int S, int WPL>
__global__ void __launch_bounds__(WPL == 1 ? 256 : 512, WPL == 1 ? (S <= 5 ? 4 : 3) : 1) k_line_api(LineOp op, int dir, const double* __restrict__ f, ArrDesc fa,
                                                  double* __restrict__ out, ArrDesc oa, int TI, int LP, double scale,
                                                  int flags) {
  extern __shared__ double sm[];
  double* tile = sm;
  double* scan = sm + (size_t)TI * LP;                 // SCAN_LINE doubles per line group
  constexpr int SCAN_LINE = 4 * WPL;                   // two solves at once
  const int ngroups = blockDim.x / (32 * WPL);
  double* sp = scan + (size_t)ngroups * SCAN_LINE;     // closure rows, 2*NSP per line
  const int o1 = (dir == 0) ? 1 : 0;
  const int o2 = (dir == 2) ? 1 : 2;
  const int64_t i1_0 = oa.lb[o1] + (int64_t)blockIdx.x * TI;
  const int64_t i1_end = oa.lb[o1] + oa.n[o1];
  const int64_t i2 = oa.lb[o2] + blockIdx.y;
  const int dim = op.dim;

  // ---- staging: nodes -HT..dim+HT of each line; those outside f along dir are zero
  const Slot sl = slot_of(dir, TI);
  const int64_t i1 = i1_0 + sl.l;
  const bool valid = i1 < i1_end;
  const int nlo = (int)max((int64_t)-HT, fa.lb[dir]);
  const int nhi = (int)min((int64_t)(dim + HT), fa.lb[dir] + fa.n[dir] - 1);
  double* trow = tile + sl.l * LP + HT;   // node 0 of the slot line
  {
    const double* src = f + (int64_t)blockIdx.z * fa.fs + (i2 - fa.lb[o2]) * fa.s[o2] + (i1 - fa.lb[o1]) * fa.s[o1] -
                        fa.lb[dir] * fa.s[dir];   // + n * s[dir] is node n
    const int64_t sd = fa.s[dir];
    int n = -HT + sl.n0;
    if (!valid) {
      for (; n <= dim + HT; n += sl.nst) trow[n] = 0.0;
    } else if (dir == 0 && sd == 1 && (((uintptr_t)(src + nlo) ^ (uintptr_t)(trow + nlo)) & 15u) == 0) {
      // x lines whose array and tile rows share the 16-byte phase: node pairs
      for (; n < nlo; n += sl.nst) trow[n] = 0.0;
      int first = nlo;
      if (((uintptr_t)(trow + nlo) & 15u) != 0) {   // one leading node to reach the phase
        if (sl.n0 == 0) cp8(trow + nlo, src + nlo);
        ++first;
      }
      const int npair = (nhi - first + 1) / 2;
      for (int p = sl.n0; p < npair; p += sl.nst) cp16(trow + first + 2 * p, src + first + 2 * p);
      if (((nhi - first + 1) & 1) && sl.n0 == 0) cp8(trow + nhi, src + nhi);
      for (int m = nhi + 1 + sl.n0; m <= dim + HT; m += sl.nst) trow[m] = 0.0;
    } else {
      for (; n < nlo; n += sl.nst) trow[n] = 0.0;
      for (; n <= nhi; n += sl.nst) cp8(trow + n, src + (int64_t)n * sd);
      for (; n <= dim + HT; n += sl.nst) trow[n] = 0.0;
    }
  }
  cp_wait_all();
  __syncthreads();
  if (op.kind != OP_EXPLICIT) {
    // closure-row RHS values, computed once per line before the solves
    for (int it = threadIdx.x; it < TI * 2 * NSP; it += blockDim.x) {
      const int j = it % (2 * NSP), ll = it / (2 * NSP);
      const bool lo = j < NSP;
      if (lo ? (j >= op.spec_lo) : (j - NSP >= op.spec_hi)) continue;
      const int r = lo ? j : op.nsys - op.spec_hi + (j - NSP);
      const double* li = tile + ll * LP + HT;
      sp[it] = special_value<true>(op, r, [li](int nn) { return li[nn]; });
    }
    __syncthreads();
  }

  // ---- solves: line group g takes lines g and g + ngroups (TI = 2 * ngroups)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = warp / WPL, part = warp - g * WPL;
  const int seg = part * 32 + lane;
  const int ext = (op.kind == OP_EXPLICIT) ? 0 : op.ext_lo;
  double v[2][S];
  if (op.kind == OP_EXPLICIT) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const double* line = tile + (g + i * ngroups) * LP + HT;
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const int r = seg * S + t;
        v[i][t] = (r <= dim) ? explicit_row(op, r, [line](int nn) { return line[nn]; }) : 0.0;
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int l = g + i * ngroups;
      const double* line = tile + l * LP + HT;
      auto get = [line](int nn) { return line[nn]; };
      if (op.kind == OP_DERIV) rhs_deriv<S>(v[i], op, seg, get, sp + l * 2 * NSP);
      else if (op.kind == OP_FLUX) rhs_flux<S>(v[i], op, seg, get, sp + l * 2 * NSP);
      else rhs_filter<S>(v[i], op, seg, get, sp + l * 2 * NSP);
    }
    seg_solve_n<S, WPL, 2>(v, op.tab, seg, lane, part, g, scan + g * SCAN_LINE);
  }
  __syncthreads();
  // outputs: nodes 0..dim, or the interfaces -1..dim of the flux (kept unscaled for differences)
  const bool diff = (op.kind == OP_FLUX) && (flags & LINE_DIFF);
  const int out_lo = (op.kind == OP_FLUX) ? -1 : 0;
  const double sc = diff ? 1.0 : scale;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double* line = tile + (g + i * ngroups) * LP + HT;
#pragma unroll
    for (int t = 0; t < S; ++t) {
      const int n = seg * S + t - ext;
      if (n < out_lo || n > dim) continue;
      // physical-boundary reset ff(0)=f(0), ff(dim)=f(dim) of compact_filter (filter.F90:141-142)
      if (op.kind == OP_FILTER && ((n == 0 && op.left_phys) || (n == dim && op.right_phys))) continue;
      line[n] = (op.kind == OP_FILTER) ? v[i][t] : sc * v[i][t];
    }
  }
  __syncthreads();

  // ---- stores from the tile: nodes 0..dim (interfaces -1..dim for the flux)
  if (!valid) return;
  double* dst = out + (int64_t)blockIdx.z * oa.fs + (i2 - oa.lb[o2]) * oa.s[o2] + (i1 - oa.lb[o1]) * oa.s[o1] -
                oa.lb[dir] * oa.s[dir];
  const int64_t od = oa.s[dir];
  const bool add = flags & LINE_ADD;
  if (diff) {
    for (int n = sl.n0; n <= dim; n += sl.nst) {
      const double d = scale * (trow[n] - trow[n - 1]);
      if (add) dst[(int64_t)n * od] += d;
      else dst[(int64_t)n * od] = d;
    }
  } else {
    if (add) {
      for (int n = out_lo + sl.n0; n <= dim; n += sl.nst) dst[(int64_t)n * od] += trow[n];
    } else {
      for (int n = out_lo + sl.n0; n <= dim; n += sl.nst) dst[(int64_t)n * od] = trow[n];
    }
  }
}

// scan scratch of seg_solve_n: 2 * WPL doubles per solve, two solves per line group
template <int S, int WPL>
static cudaError_t launch_t(const DevOp& op, int dir, const double* f, const ArrDesc& fa, double* out,
                            const ArrDesc& oa, int nfields, double scale, int flags, cudaStream_t st) {
  const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
  // two lines per group of WPL warps, at most 512 threads and 16 lines, one named barrier per
  // group (WPL > 1: at most 15 groups)
  int ngroups = 512 / (32 * WPL);
  if (ngroups > 8) ngroups = 8;
  const int TI = 2 * ngroups;
  const int LP = tile_pitch(op.op.dim, TI, S);
  const size_t smem = ((size_t)TI * LP + (size_t)ngroups * 4 * WPL + (size_t)TI * 2 * NSP) * sizeof(double);
  auto kern = k_line_api<S, WPL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((oa.n[o1] + TI - 1) / TI), (unsigned)oa.n[o2], (unsigned)nfields);
  kern<<<grid, ngroups * WPL * 32, smem, st>>>(op.op, dir, f, fa, out, oa, TI, LP, scale, flags);
  return cudaGetLastError();
}

cudaError_t launch_line_api(const DevOp& op, int dir, const double* f, const ArrDesc& fa, double* out,
                            const ArrDesc& oa, int nfields, double scale, cudaStream_t st, int flags) {
  if (op.S == 3 && op.WPL == 1) return launch_t<3, 1>(op, dir, f, fa, out, oa, nfields, scale, flags, st);
  if (op.S == 5 && op.WPL == 1) return launch_t<5, 1>(op, dir, f, fa, out, oa, nfields, scale, flags, st);
  if (op.S == 5 && op.WPL == 2) return launch_t<5, 2>(op, dir, f, fa, out, oa, nfields, scale, flags, st);
  if (op.S == 5 && op.WPL == 4) return launch_t<5, 4>(op, dir, f, fa, out, oa, nfields, scale, flags, st);
  if (op.S == 9 && op.WPL == 1) return launch_t<9, 1>(op, dir, f, fa, out, oa, nfields, scale, flags, st);
  if (op.S == 9 && op.WPL == 2) return launch_t<9, 2>(op, dir, f, fa, out, oa, nfields, scale, flags, st);
  if (op.S == 9 && op.WPL == 4) return launch_t<9, 4>(op, dir, f, fa, out, oa, nfields, scale, flags, st);
  return cudaErrorInvalidValue;
}

}  // namespace astr
