// Line-level operators over arbitrary Fortran-ordered arrays: the drop-in for
//   df = fds%central(asolver, f, dim)      src/derivative.F90:22-41, 171-198
//   ff = compact_filter(afilter, f, dim)   src/filter.F90:112-144
// applied to every line of a 3-D array along one direction.
//
// One CTA takes TI lines. The lines (nodes -HT..dim+HT, halos read from the caller's array) are
// staged in shared memory with coalesced loads: node-fastest for x lines, line-fastest for
// y/z lines (TI adjacent lines are contiguous in x). WPL warps solve each line with the
// segmented Thomas of ops.cuh; results go back through the tile for coalesced stores.
#include "internal.h"

namespace astr {

template <int S, int WPL>
__global__ void __launch_bounds__(1024) k_line_api(LineOp op, int dir, const double* __restrict__ f, ArrDesc fa,
                                                   double* __restrict__ out, ArrDesc oa, int TI, int LP,
                                                   double scale) {
  extern __shared__ double sm[];
  double* tile = sm;
  double* scan = sm + (size_t)TI * LP;   // 2*WPL per line
  double* sp = scan + (size_t)TI * 2 * WPL;   // closure rows, 2*NSP per line
  const int o1 = (dir == 0) ? 1 : 0;
  const int o2 = (dir == 2) ? 1 : 2;
  const int64_t l1_0 = oa.lb[o1] + (int64_t)blockIdx.x * TI;
  const int64_t l1_end = oa.lb[o1] + oa.n[o1];
  const int64_t i2 = oa.lb[o2] + blockIdx.y;
  const double* fb = f + (int64_t)blockIdx.z * fa.fs;
  double* ob = out + (int64_t)blockIdx.z * oa.fs;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int dim = op.dim;
  const int LPn = dim + 1 + 2 * HT;
  const int64_t fbase2 = (i2 - fa.lb[o2]) * fa.s[o2];
  const int64_t obase2 = (i2 - oa.lb[o2]) * oa.s[o2];

  for (int idx = tid; idx < TI * LPn; idx += nthr) {
    int l, nn;
    if (dir == 0) { l = idx / LPn; nn = idx - l * LPn; }
    else { nn = idx / TI; l = idx - nn * TI; }
    const int n = nn - HT;
    const int64_t i1 = l1_0 + l;
    double val = 0.0;
    if (i1 < l1_end && n >= fa.lb[dir] && n < fa.lb[dir] + fa.n[dir])
      val = fb[fbase2 + (i1 - fa.lb[o1]) * fa.s[o1] + (n - fa.lb[dir]) * fa.s[dir]];
    tile[l * LP + nn] = val;
  }
  __syncthreads();
  if (op.kind != OP_EXPLICIT) {
    // closure-row RHS values, computed once per line before the solves
    for (int it = tid; it < TI * 2 * NSP; it += nthr) {
      const int j = it % (2 * NSP), ll = it / (2 * NSP);
      const bool lo = j < NSP;
      if (lo ? (j >= op.spec_lo) : (j - NSP >= op.spec_hi)) continue;
      const int r = lo ? j : op.nsys - op.spec_hi + (j - NSP);
      const double* li = tile + ll * LP + HT;
      sp[it] = special_value(op, r, [li](int n) { return li[n]; });
    }
    __syncthreads();
  }

  const int warp = tid >> 5, lane = tid & 31;
  const int l = warp / WPL, part = warp - l * WPL;
  const int seg = part * 32 + lane;
  double* line = tile + l * LP + HT;
  auto get = [line](int n) { return line[n]; };
  double v[S];
  if (op.kind == OP_DERIV) {
    rhs_deriv<S>(v, op, seg, get, sp + l * 2 * NSP);
    seg_solve<S, WPL>(v, op.tab, seg, lane, part, l, scan + l * 2 * WPL);
  } else if (op.kind == OP_FILTER) {
    rhs_filter<S>(v, op, seg, get, sp + l * 2 * NSP);
    seg_solve<S, WPL>(v, op.tab, seg, lane, part, l, scan + l * 2 * WPL);
  } else {
#pragma unroll
    for (int t = 0; t < S; ++t) {
      const int r = seg * S + t;
      v[t] = (r <= dim) ? explicit_row(op, r, get) : 0.0;
    }
  }
  __syncthreads();
  const int ext = (op.kind == OP_EXPLICIT) ? 0 : op.ext_lo;
#pragma unroll
  for (int t = 0; t < S; ++t) {
    const int n = seg * S + t - ext;
    if (n < 0 || n > dim) continue;
    // physical-boundary reset ff(0)=f(0), ff(dim)=f(dim) of compact_filter (filter.F90:141-142)
    if (op.kind == OP_FILTER && ((n == 0 && op.left_phys) || (n == dim && op.right_phys))) continue;
    line[n] = (op.kind == OP_FILTER) ? v[t] : scale * v[t];
  }
  __syncthreads();
  const int nout = dim + 1;
  for (int idx = tid; idx < TI * nout; idx += nthr) {
    int l2, n;
    if (dir == 0) { l2 = idx / nout; n = idx - l2 * nout; }
    else { n = idx / TI; l2 = idx - n * TI; }
    const int64_t i1 = l1_0 + l2;
    if (i1 >= l1_end) continue;
    const double val = tile[l2 * LP + HT + n];
    ob[obase2 + (i1 - oa.lb[o1]) * oa.s[o1] + (n - oa.lb[dir]) * oa.s[dir]] = val;
  }
}

template <int S, int WPL>
static cudaError_t launch_t(const DevOp& op, int dir, const double* f, const ArrDesc& fa, double* out,
                            const ArrDesc& oa, int nfields, double scale, cudaStream_t st) {
  const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
  int TI = 512 / (32 * WPL);   // <= 15 lines when WPL > 1 (one named barrier per line)
  if (TI > 16) TI = 16;
  if (TI < 1) TI = 1;
  const int LP = tile_pitch(op.op.dim, TI, S);
  const size_t smem = ((size_t)TI * LP + (size_t)TI * (2 * WPL + 2 * NSP)) * sizeof(double);
  auto kern = k_line_api<S, WPL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((oa.n[o1] + TI - 1) / TI), (unsigned)oa.n[o2], (unsigned)nfields);
  kern<<<grid, TI * WPL * 32, smem, st>>>(op.op, dir, f, fa, out, oa, TI, LP, scale);
  return cudaGetLastError();
}

cudaError_t launch_line_api(const DevOp& op, int dir, const double* f, const ArrDesc& fa, double* out,
                            const ArrDesc& oa, int nfields, double scale, cudaStream_t st) {
  if (op.S == 3 && op.WPL == 1) return launch_t<3, 1>(op, dir, f, fa, out, oa, nfields, scale, st);
  if (op.S == 5 && op.WPL == 1) return launch_t<5, 1>(op, dir, f, fa, out, oa, nfields, scale, st);
  if (op.S == 5 && op.WPL == 2) return launch_t<5, 2>(op, dir, f, fa, out, oa, nfields, scale, st);
  if (op.S == 5 && op.WPL == 4) return launch_t<5, 4>(op, dir, f, fa, out, oa, nfields, scale, st);
  if (op.S == 9 && op.WPL == 1) return launch_t<9, 1>(op, dir, f, fa, out, oa, nfields, scale, st);
  if (op.S == 9 && op.WPL == 2) return launch_t<9, 2>(op, dir, f, fa, out, oa, nfields, scale, st);
  if (op.S == 9 && op.WPL == 4) return launch_t<9, 4>(op, dir, f, fa, out, oa, nfields, scale, st);
  return cudaErrorInvalidValue;
}

}  // namespace astr
