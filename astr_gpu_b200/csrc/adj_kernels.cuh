// Line kernels of the discrete adjoint (included once per solve layout by tgv_l*.cu, after
// tgv_kernels.cuh).
//
// A periodic line operator of the forward step (compact derivative or compact filter along one
// direction) is  L = R A^-1 B E :  E extends nodes 0..N by the periodic halo copy (bchomo /
// bchomovec), B is the RHS stencil with its closure rows, A the tridiagonal system, R keeps the
// rows of nodes 0..N. Its transpose is  L^T = E^T B^T A^-T R^T :
//   * the adjoint input g(0..N) goes into rows e..e+N of the system (zeros in the extra rows),
//   * one tridiagonal solve with A^T (again tridiagonal: sub-diagonal c_{r-1}, super-diagonal
//     a_{r+1}), segmented exactly like the forward solve,
//   * out(m) = sum over rows r of W(m, r) y(r) with W = E^T B^T: a fixed stencil for interior
//     nodes and short explicit lists for the nodes whose column of B has closure rows or periodic
//     images folded into it.
#pragma once
#include "adjoint.cuh"
#include "tgv_kernels.cuh"

namespace astr {

namespace adj_detail {

using namespace pass_detail;

// out(f) = alpha * L^T in(f) (+ out(f) when accumulating) for nf fields along DIR. Up to
// ADJ_MAXF fields are staged together (asynchronous copies, zeros outside nodes 0..dim), solved
// one after the other in place, then gathered through W and stored.
template <int S, int WPL, int DIR, int NB>
__global__ void __launch_bounds__(512) k_adj_lines(AdjLineArgs a) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL> c(a.p, blockIdx.x, blockIdx.y);
  const int dim = c.dim;
  const int tsz = c.TI * c.LP;
  const int nstage = a.nf < ADJ_MAXF ? a.nf : ADJ_MAXF;
  double* T = sm;
  double* scan = sm + (size_t)nstage * tsz;
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  const LineOp& op = a.p.opd;
  const int e = op.ext_lo, nsys = op.nsys;
  const int64_t fs = a.p.g.fs;
  const AdjW& w = a.w;
  for (int f0 = 0; f0 < a.nf; f0 += ADJ_MAXF) {
    const int nfc = (a.nf - f0) < ADJ_MAXF ? (a.nf - f0) : ADJ_MAXF;
    for (int f = 0; f < nfc; ++f) {
      double* Tf = T + f * tsz;
      const double* g = a.in + (f0 + f) * fs + c.sbase;
      c.for_nodes(-HT, dim + HT, [&](int o, int n) {
        if (c.svalid && n >= 0 && n <= dim) cp_async8(Tf + o, g + (int64_t)n * c.sd);
        else Tf[o] = 0.0;
      });
    }
    cp_async_wait_all();
    __syncthreads();
    for (int f = 0; f < nfc; ++f) {
      double* line = T + f * tsz + z.l * c.LP + HT;
      double v[1][S];
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const int r = z.seg * S + t;
        v[0][t] = (r < nsys) ? line[r - e] : 0.0;
      }
      seg_solve_n<S, WPL, 1>(v, op.tab, z.seg, z.lane, z.part, z.l, scl);
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const int r = z.seg * S + t;
        if (r < nsys) line[r - e] = v[0][t];
      }
    }
    __syncthreads();
    if (c.svalid) {
      for (int f = 0; f < nfc; ++f) {
        const double* Tf = T + f * tsz;
        double* dst = a.out + (f0 + f) * fs + c.sbase;
        c.for_nodes(0, dim, [&](int o, int n) {
          double s = 0.0;
          if (n >= w.mlo && n <= w.mhi) {
            const double* y = Tf + o + w.jlo;
#pragma unroll
            for (int j = 0; j < NB; ++j) s = fma(w.wint[j], y[j], s);
          } else {
            const int k = n < w.mlo ? n : w.mlo + (n - w.mhi - 1);
            const double* y = Tf + o - n;
            for (int q = w.sptr[k]; q < w.sptr[k + 1]; ++q) s = fma(w.scoef[q], y[w.snode[q]], s);
          }
          s *= a.alpha;
          const int64_t off = (int64_t)n * c.sd;
          dst[off] = a.accumulate ? dst[off] + s : s;
        });
      }
    }
    __syncthreads();
  }
}

// Velocity and temperature gradients along DIR of the state q (gradcal, tgvsolver.F90:450-537):
// D[k] = d(u, v, w, T)_k / dx_DIR, k = 0..3.
template <int S, int WPL, int DIR>
__global__ void __launch_bounds__(512) k_adj_grad(PassArgs a) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL> c(a, blockIdx.x, blockIdx.y);
  const int tsz = c.TI * c.LP;
  double* T = sm;
  double* O = sm + 5 * tsz;
  double* scan = O + tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;
  const int64_t fs = a.g.fs;
  for (int m = 0; m < 5; ++m) load_tile(c, T + m * tsz, a.q + m * fs);
  cp_async_wait_all();
  __syncthreads();
  to_prims(c, T, tsz, a.th);
  __syncthreads();
  compute_specials<OP_DERIV>(a.opd, c.TI, spb, 4, [&](int l, int k, int n) { return gprim_rt<DIR>(k, T + l * c.LP + HT, tsz, n, a.th); });
  __syncthreads();
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  const double rd = a.g.rd[DIR];
  const double* L0 = T + z.l * c.LP + HT;
  double* oline = O + z.l * c.LP + HT;
  for (int K = 0; K < 4; ++K) {
    double v[1][S];
    dsolve_n<S, WPL, DIR, 1>(v, K, a, z, L0, tsz, scl, rd, spb + (z.l * 4 + K) * 2 * NSP);
    put_lane<S>(oline, v[0], z.seg, a.opd.ext_lo, c.dim, false);
    __syncthreads();
    if (c.svalid) {
      double* dst = a.D + K * fs + c.sbase;
      c.for_nodes(0, c.dim, [&](int o, int n) { dst[(int64_t)n * c.sd] = O[o]; });
    }
    __syncthreads();
  }
}

}  // namespace adj_detail

template <class KernT, class ArgT>
cudaError_t launch_adj_k(KernT kern, dim3 grid, int threads, size_t smem, cudaStream_t st, const ArgT& a) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, threads, smem, st>>>(a);
  return cudaGetLastError();
}

template <int S, int WPL>
cudaError_t launch_adj_lines_t(const AdjLineArgs& a, cudaStream_t st) {
  const int dir = a.p.dir;
  const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
  dim3 grid((unsigned)((a.p.g.N[o1] + 1 + a.p.TI - 1) / a.p.TI), (unsigned)(a.p.g.N[o2] + 1));
  const int threads = a.p.TI * WPL * 32;
  const size_t smem = adj_lines_smem(a.p.TI, a.p.LP, WPL, a.nf < ADJ_MAXF ? a.nf : ADJ_MAXF);
  const int nb = a.w.nint <= 5 ? 5 : (a.w.nint <= 11 ? 11 : ADJ_BAND);
#define ASTR_ADJ_LINES(D, NB) \
  if (dir == D && nb == NB) return launch_adj_k(adj_detail::k_adj_lines<S, WPL, D, NB>, grid, threads, smem, st, a);
  ASTR_ADJ_LINES(0, 5) ASTR_ADJ_LINES(0, 11) ASTR_ADJ_LINES(0, ADJ_BAND)
  ASTR_ADJ_LINES(1, 5) ASTR_ADJ_LINES(1, 11) ASTR_ADJ_LINES(1, ADJ_BAND)
  ASTR_ADJ_LINES(2, 5) ASTR_ADJ_LINES(2, 11) ASTR_ADJ_LINES(2, ADJ_BAND)
#undef ASTR_ADJ_LINES
  return cudaErrorInvalidValue;
}

template <int S, int WPL>
cudaError_t launch_adj_grad_t(const PassArgs& a, cudaStream_t st) {
  const int dir = a.dir;
  const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
  dim3 grid((unsigned)((a.g.N[o1] + 1 + a.TI - 1) / a.TI), (unsigned)(a.g.N[o2] + 1));
  const int threads = a.TI * WPL * 32;
  const size_t smem = adj_grad_smem(a.TI, a.LP, WPL);
  if (dir == 0) return launch_adj_k(adj_detail::k_adj_grad<S, WPL, 0>, grid, threads, smem, st, a);
  if (dir == 1) return launch_adj_k(adj_detail::k_adj_grad<S, WPL, 1>, grid, threads, smem, st, a);
  return launch_adj_k(adj_detail::k_adj_grad<S, WPL, 2>, grid, threads, smem, st, a);
}

}  // namespace astr
