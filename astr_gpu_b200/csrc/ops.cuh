// Device primitives shared by every line kernel: the segmented Thomas solve and the right-hand
// sides of the compact derivative and the compact filter, with all their closure rows.
//
// A line's tridiagonal system (rows r = 0..nsys-1, node = r - ext_lo) is owned by WPL warps:
// lane `lane` of warp `part` owns the S consecutive rows of segment seg = part*32 + lane.
// The reference solves each system with a sequential Thomas sweep on a pre-factored table
// (commfunc.F90:790-813):   y_r = d_r*ac2_r - y_{r-1}*ac3_r ;  x_r = y_r - ac1_r*x_{r+1}.
// Both recurrences are affine in their carry, so each lane runs them over its rows from a zero
// carry, the true carries follow from a scan of the per-segment affine maps (warp shuffles,
// then shared memory across the WPL warps of a line), and each row is corrected by the
// carry times a precomputed product of the table entries. The result equals the sequential
// sweep up to rounding.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace astr {

// Tile halo nodes kept on each side of a line. The real rows of a system read nodes up to
// dim + 8 (filter: 3 extension rows and a half-width of 5); the window of the lane holding the
// last real row reaches S - 1 nodes further for its trailing padding rows: up to dim + 24 for
// 17 rows per lane. Tile lines of layouts with more than 9 rows per lane therefore end with
// WIN_SLACK unstaged slots after the high halo (read only for padding rows, which are zeroed
// before the solve), and only lanes whose rows are all padding reach past that (window_base).
constexpr int HT = 16;
constexpr int WIN_SLACK = 8;
__host__ __device__ constexpr int win_slack(int S) { return S > 9 ? WIN_SLACK : 0; }
constexpr unsigned FULL = 0xffffffffu;

// OP_FLUX: the compact interface flux of flux.F90 (rows are interfaces, outputs fh(-1..dim))
enum OpKind { OP_DERIV = 0, OP_FILTER = 1, OP_EXPLICIT = 2, OP_FLUX = 3 };

// One line operator (a compact_scheme of the reference plus the lane tables of its solve).
// Table layout (doubles), NS = 32*WPL segments of S rows, row t of segment seg:
//   [2*(t*NS + seg)]            (ac2, ac3) pair for the forward sweep
//   [2*S*NS + t*NS + seg]       pf, forward prefix product of -ac3 within the segment
//   [3*S*NS + 2*(t*NS + seg)]   (ac1, qb) pair for the backward sweep (qb: suffix product of -ac1)
//   [5*S*NS + k*NS + seg]       per segment: FS[0..4] forward scan composites for shuffle offsets
//                               1..16, FE forward exclusive product within the warp, BS[0..4], BE
//   [(5*S + 12)*NS + ...]       per warp: MW[WPL], MWB[WPL] (whole-warp products)
//   [(5*S + 12)*NS + 2*WPL]     int per segment: the slot whose row columns (the first three
//                               arrays) it reads; segments with identical columns share a slot
struct LineOp {
  const double* tab;
  int nsys;            // rows of the system (last_node - first_node + 1)
  int ext_lo;          // -first_node: node = r - ext_lo
  int dim;
  int kind;
  int left_phys, right_phys;   // physical closures at node 0 (ntype 1,4) / node dim (ntype 2,4)
  int no_filter_note;          // note='boundary_no_filter'
  int nseg;
  int S;
  int spec_lo, spec_hi;        // closure rows at the start / end of the system (RHS not interior)
  double c10[6], ch[3][11], cb[3][7], c6[4], c8[5];  // filter coefficients (filter.F90:299-432)
  // interface flux: wind +1 ('+', upwind-biased) or -1 ('-'), and the interior RHS weights
  // (1/18 - b/36, 19/18 - 9b/36, 5/9 + 9b/36, b/36) of compact_flux_rhs (flux.F90:241-253)
  int wind;
  double cfl[4];
};

constexpr int NSP = 5;   // closure rows kept per end: sp[0..4] start, sp[5..9] end

enum TabOff { T_FS = 0, T_FE = 5, T_BS = 6, T_BE = 11, T_NSEGTAB = 12 };

// Barrier among the WPL warps of one line (named barrier 1 + line).
template <int WPL>
__device__ __forceinline__ void line_sync(int line) {
  if (WPL > 1) asm volatile("bar.sync %0, %1;" ::"r"(1 + line), "r"(32 * WPL) : "memory");
}

// Segmented Thomas solve of NV right-hand sides at once (the coefficients are shared, the
// chains interleave). v[i] holds the RHS rows of this lane on entry and the solution on exit.
// scan_sm: 2*WPL*NV doubles private to this line (used only when WPL > 1). All warps of the
// line must call it together.
template <int S, int WPL, int NV>
__device__ __forceinline__ void seg_solve_n(double (&v)[NV][S], const double* __restrict__ tab, int seg, int lane,
                                            int part, int line, double* scan_sm) {
  constexpr int NS = 32 * WPL;
  // row coefficients from this segment's slot (shared by segments with identical columns)
  const int rs = __ldg(reinterpret_cast<const int*>(tab + (5 * S + T_NSEGTAB) * NS + 2 * WPL) + seg);
  const double2* fwd = reinterpret_cast<const double2*>(tab) + rs;
  const double* pfp = tab + 2 * S * NS + rs;
  const double2* bwd = reinterpret_cast<const double2*>(tab + 3 * S * NS) + rs;
  const double* sg = tab + 5 * S * NS + seg;
  const double* ws = tab + (5 * S + T_NSEGTAB) * NS;   // per-warp products
  // forward sweeps from a zero carry
  double g[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) g[i] = 0.0;
#pragma unroll
  for (int t = 0; t < S; ++t) {
    const double2 c = __ldg(fwd + t * NS);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      g[i] = v[i][t] * c.x - g[i] * c.y;
      v[i][t] = g[i];
    }
  }
  // inclusive scans of the segment maps c -> G + M c across the warp (composite M precomputed)
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double m = __ldg(sg + (T_FS + k) * NS);
#pragma unroll
    for (int i = 0; i < NV; ++i) g[i] = fma(m, __shfl_up_sync(FULL, g[i], 1 << k), g[i]);
  }
  double cin[NV];
  const double fe = __ldg(sg + T_FE * NS);
  if (WPL > 1) {
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (lane == 31) scan_sm[i * 2 * WPL + part] = g[i];
    line_sync<WPL>(line);
  }
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double ge = __shfl_up_sync(FULL, g[i], 1);
    if (lane == 0) ge = 0.0;
    double cw = 0.0;
    if (WPL > 1)
      for (int p = 0; p < part; ++p) cw = fma(__ldg(ws + p), cw, scan_sm[i * 2 * WPL + p]);
    cin[i] = fma(fe, cw, ge);
  }
#pragma unroll
  for (int t = 0; t < S; ++t) {
    const double pf = __ldg(pfp + t * NS);
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i][t] = fma(pf, cin[i], v[i][t]);
  }

  // backward sweeps from a zero carry
  double qb[S];
#pragma unroll
  for (int i = 0; i < NV; ++i) g[i] = 0.0;
#pragma unroll
  for (int t = S - 1; t >= 0; --t) {
    const double2 c = __ldg(bwd + t * NS);
    qb[t] = c.y;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      g[i] = v[i][t] - c.x * g[i];
      v[i][t] = g[i];
    }
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double m = __ldg(sg + (T_BS + k) * NS);
#pragma unroll
    for (int i = 0; i < NV; ++i) g[i] = fma(m, __shfl_down_sync(FULL, g[i], 1 << k), g[i]);
  }
  const double be = __ldg(sg + T_BE * NS);
  if (WPL > 1) {
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (lane == 0) scan_sm[i * 2 * WPL + WPL + part] = g[i];
    line_sync<WPL>(line);
  }
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double ge = __shfl_down_sync(FULL, g[i], 1);
    if (lane == 31) ge = 0.0;
    double cw = 0.0;
    if (WPL > 1)
      for (int p = WPL - 1; p > part; --p) cw = fma(__ldg(ws + WPL + p), cw, scan_sm[i * 2 * WPL + WPL + p]);
    const double cb = fma(be, cw, ge);
#pragma unroll
    for (int t = 0; t < S; ++t) v[i][t] = fma(qb[t], cb, v[i][t]);
  }
}

template <int S, int WPL>
__device__ __forceinline__ void seg_solve(double (&v)[S], const double* __restrict__ tab, int seg, int lane, int part,
                                          int line, double* scan_sm) {
  seg_solve_n<S, WPL, 1>(reinterpret_cast<double(&)[1][S]>(v), tab, seg, lane, part, line, scan_sm);
}

// ---------------------------------------------------------------- right-hand sides
// Compact derivative closure rows, derivative.F90:230-294. Returns false for interior rows.
template <class Get>
__host__ __device__ __forceinline__ bool deriv_special(const LineOp& op, int r, Get f, double& out) {
  const int j = r - op.ext_lo;
  if (r == 0) {
    if (op.left_phys) { out = -2.5 * f(j) + 2.0 * f(j + 1) + 0.5 * f(j + 2); return true; }
    double var1 = f(j + 1) - f(j - 1), var2 = f(j + 2) - f(j - 2), var3 = f(j + 3) - f(j - 3);
    out = 0.75 * var1 - 0.15 * var2 + (1.0 / 60.0) * var3;
    return true;
  }
  if (r == 1 && op.left_phys) { out = 0.75 * (f(j + 1) - f(j - 1)); return true; }
  if (r == op.nsys - 1) {
    if (op.right_phys) { out = 2.5 * f(j) - 2.0 * f(j - 1) - 0.5 * f(j - 2); return true; }
    double var1 = f(j + 1) - f(j - 1), var2 = f(j + 2) - f(j - 2), var3 = f(j + 3) - f(j - 3);
    out = 0.75 * var1 - 0.15 * var2 + (1.0 / 60.0) * var3;
    return true;
  }
  if (r == op.nsys - 2 && op.right_phys) { out = 0.75 * (f(j + 1) - f(j - 1)); return true; }
  return false;
}

// Interior compact RHS 7/9(f+1 - f-1) + 1/36(f+2 - f-2) (derivative.F90:296-304) on a window
// w[t] = f(n0 - 2 + t), n0 = node of the lane's first row.
template <int S>
__device__ __forceinline__ void stencil_deriv(double (&v)[S], const double (&w)[S + 4]) {
#pragma unroll
  for (int t = 0; t < S; ++t) v[t] = (7.0 / 9.0) * (w[t + 3] - w[t + 1]) + (1.0 / 36.0) * (w[t + 4] - w[t]);
}

// First node of a lane's window of W nodes starting at n0 (layout of S rows per lane). Only
// lanes holding nothing but padding rows run past the tile line (nodes up to dim + HT +
// win_slack(S)); they read its last W slots instead (their rows are zeroed), so every lane loads
// its window without per-node clamps.
template <int W, int S>
__device__ __forceinline__ int window_base(int n0, int dim) {
  constexpr int top = HT + win_slack(S);
  return n0 + W - 1 > dim + top ? dim + top - W + 1 : n0;
}
template <int W, int S, class Get>
__device__ __forceinline__ void fill_window(double (&w)[W], int n0, int dim, Get f) {
  const int b = window_base<W, S>(n0, dim);
#pragma unroll
  for (int t = 0; t < W; ++t) w[t] = f(b + t);
}

template <class Get>
__host__ __device__ __forceinline__ bool filter_special(const LineOp& op, int r, Get f, double& out);

// Compact interface-flux closure rows, compact_flux_rhs (flux.F90:188-230): 3rd-order rows at
// physical ends, the explicit 6th-order central interface value elsewhere. Row r is interface
// j = r - ext_lo (between nodes j and j + 1).
template <class Get>
__host__ __device__ __forceinline__ bool flux_special(const LineOp& op, int r, Get f, double& out) {
  const int j = r - op.ext_lo;
  auto central = [&]() {
    const double var1 = f(j) + f(j + 1), var2 = f(j - 1) + f(j + 2), var3 = f(j - 2) + f(j + 3);
    return (37.0 / 60.0) * var1 - (2.0 / 15.0) * var2 + (1.0 / 60.0) * var3;
  };
  if (r == 0) {
    out = op.left_phys ? 2.5 * f(j + 1) + 0.5 * f(j + 2) : central();
    return true;
  }
  if (r == 1 && op.left_phys) { out = 0.75 * f(j) + 0.75 * f(j + 1); return true; }
  if (r == op.nsys - 1) {
    out = op.right_phys ? 2.5 * f(j) + 0.5 * f(j - 1) : central();
    return true;
  }
  if (r == op.nsys - 2 && op.right_phys) { out = 0.75 * f(j + 1) + 0.75 * f(j); return true; }
  return false;
}

// RHS value of closure row r (derivative or filter; with FLUX also the interface flux, which only
// the line operators take, so that the fused passes compile without its branch), for the
// precomputed closure table.
// KIND >= 0 fixes the operator kind at compile time (a pass that only differentiates then
// carries no filter closure code).
template <bool FLUX = false, int KIND = -1, class Get>
__device__ __forceinline__ double special_value(const LineOp& op, int r, Get f) {
  double s = 0.0;
  if (KIND == OP_DERIV) deriv_special(op, r, f, s);
  else if (KIND == OP_FILTER) filter_special(op, r, f, s);
  else if (op.kind == OP_FILTER) filter_special(op, r, f, s);
  else if (FLUX && op.kind == OP_FLUX) flux_special(op, r, f, s);
  else deriv_special(op, r, f, s);
  return s;
}
// Replace the closure rows of this lane by their precomputed values and zero its padding rows.
// Only the first lanes of a line (start rows) and the lanes at or past the end rows branch in.
template <int S>
__device__ __forceinline__ void apply_specials(double (&v)[S], const LineOp& op, int r0, const double* sp) {
  if (r0 < op.spec_lo) {
#pragma unroll
    for (int t = 0; t < S; ++t)
      if (r0 + t < op.spec_lo) v[t] = sp[r0 + t];
  }
  const int e0 = op.nsys - op.spec_hi;   // first closure row at the end
  if (r0 + S > e0) {
#pragma unroll
    for (int t = 0; t < S; ++t) {
      const int k = r0 + t - e0;
      if (k >= op.spec_hi) v[t] = 0.0;
      else if (k >= 0) v[t] = sp[NSP + k];
    }
  }
}

template <int S, class Get>
__device__ __forceinline__ void rhs_deriv(double (&v)[S], const LineOp& op, int seg, Get f, const double* sp) {
  const int r0 = seg * S;
  double w[S + 4];
  fill_window<S + 4, S>(w, r0 - op.ext_lo - 2, op.dim, f);
  stencil_deriv<S>(v, w);
  apply_specials<S>(v, op, r0, sp);
}

// Interior rows of the compact interface flux (flux.F90:241-253), in the reference's order of
// the four products for each wind; window w[t] = f(n0 - 1 + t), n0 = interface of the first row.
template <int S, class Get>
__device__ __forceinline__ void rhs_flux(double (&v)[S], const LineOp& op, int seg, Get f, const double* sp) {
  const int r0 = seg * S;
  double w[S + 3];
  fill_window<S + 3, S>(w, r0 - op.ext_lo - 1, op.dim, f);
  if (op.wind > 0) {
#pragma unroll
    for (int t = 0; t < S; ++t)
      v[t] = op.cfl[0] * w[t] + op.cfl[1] * w[t + 1] + op.cfl[2] * w[t + 2] + op.cfl[3] * w[t + 3];
  } else {
#pragma unroll
    for (int t = 0; t < S; ++t)
      v[t] = op.cfl[0] * w[t + 3] + op.cfl[1] * w[t + 2] + op.cfl[2] * w[t + 1] + op.cfl[3] * w[t];
  }
  apply_specials<S>(v, op, r0, sp);
}

// Explicit 6th-order derivative with its closures (diff6ec, derivative.F90:350-413); rows are
// nodes 0..dim (no solve).
template <class Get>
__device__ __forceinline__ double explicit_row(const LineOp& op, int i, Get v) {
  const int dim = op.dim;
  if (op.left_phys) {
    if (i == 0) return -0.5 * v(2) + 2.0 * v(1) - 1.5 * v(0);
    if (i == 1) return 0.5 * (v(2) - v(0));
    if (i == 2) return (2.0 / 3.0) * (v(3) - v(1)) - (1.0 / 12.0) * (v(4) - v(0));
  }
  if (op.right_phys) {
    if (i == dim - 2) return (2.0 / 3.0) * (v(dim - 1) - v(dim - 3)) - (1.0 / 12.0) * (v(dim) - v(dim - 4));
    if (i == dim - 1) return 0.5 * (v(dim) - v(dim - 2));
    if (i == dim) return 0.5 * v(dim - 2) - 2.0 * v(dim - 1) + 1.5 * v(dim);
  }
  return 0.75 * (v(i + 1) - v(i - 1)) - 0.15 * (v(i + 2) - v(i - 2)) + (1.0 / 60.0) * (v(i + 3) - v(i - 3));
}

// Compact filter closure rows, filter.F90:176-269. Returns false for interior rows.
template <class Get>
__host__ __device__ __forceinline__ bool filter_special(const LineOp& op, int r, Get f, double& out) {
  const int i0 = -op.ext_lo;
  const int im = op.nsys - 1 - op.ext_lo;
  const int j = r - op.ext_lo;
  if (op.no_filter_note && (r == 0 || r == op.nsys - 1)) { out = f(j); return true; }
  if (op.left_phys) {
    if (r <= 2) {
      double var0 = 0.0;
      for (int jj = 0; jj <= 6; ++jj) var0 = var0 + op.cb[r][jj] * f(i0 + jj);
      out = var0; return true;
    }
    if (r == 3) {
      out = op.c6[0] * (f(j) + f(j)) + op.c6[1] * (f(j + 1) + f(j - 1)) + op.c6[2] * (f(j + 2) + f(j - 2)) +
            op.c6[3] * (f(j + 3) + f(j - 3));
      return true;
    }
    if (r == 4) {
      out = op.c8[0] * (f(j) + f(j)) + op.c8[1] * (f(j + 1) + f(j - 1)) + op.c8[2] * (f(j + 2) + f(j - 2)) +
            op.c8[3] * (f(j + 3) + f(j - 3)) + op.c8[4] * (f(j + 4) + f(j - 4));
      return true;
    }
  } else if (r <= 2) {
    double var0 = 0.0;
    for (int jj = 0; jj <= 10; ++jj) var0 = var0 + op.ch[r][jj] * f(i0 - 2 + jj);
    out = var0; return true;
  }
  const int k = op.nsys - 1 - r;   // distance from the last row
  if (op.right_phys) {
    if (k <= 2) {
      double var0 = 0.0;
      for (int jj = 0; jj <= 6; ++jj) var0 = var0 + op.cb[k][jj] * f(im - jj);
      out = var0; return true;
    }
    if (k == 3) {
      out = op.c6[0] * (f(j) + f(j)) + op.c6[1] * (f(j + 1) + f(j - 1)) + op.c6[2] * (f(j + 2) + f(j - 2)) +
            op.c6[3] * (f(j + 3) + f(j - 3));
      return true;
    }
    if (k == 4) {
      out = op.c8[0] * (f(j) + f(j)) + op.c8[1] * (f(j + 1) + f(j - 1)) + op.c8[2] * (f(j + 2) + f(j - 2)) +
            op.c8[3] * (f(j + 3) + f(j - 3)) + op.c8[4] * (f(j + 4) + f(j - 4));
      return true;
    }
  } else if (k <= 2) {
    double var0 = 0.0;
    for (int jj = 0; jj <= 10; ++jj) var0 = var0 + op.ch[k][jj] * f(im + 2 - jj);
    out = var0; return true;
  }
  return false;
}

// Interior 11-point filter RHS (filter.F90:271-283) over a window, then closure rows.
template <int S, class Get>
__device__ __forceinline__ void rhs_filter(double (&v)[S], const LineOp& op, int seg, Get f, const double* sp) {
  const int r0 = seg * S;
  double w[S + 10];
  fill_window<S + 10, S>(w, r0 - op.ext_lo - 5, op.dim, f);
#pragma unroll
  for (int t = 0; t < S; ++t) {
    double var0 = w[t + 5] + w[t + 5];
    double var1 = w[t + 6] + w[t + 4];
    double var2 = w[t + 7] + w[t + 3];
    double var3 = w[t + 8] + w[t + 2];
    double var4 = w[t + 9] + w[t + 1];
    double var5 = w[t + 10] + w[t];
    v[t] = op.c10[0] * var0 + op.c10[1] * var1 + op.c10[2] * var2 + op.c10[3] * var3 + op.c10[4] * var4 +
           op.c10[5] * var5;
  }
  apply_specials<S>(v, op, r0, sp);
}

// Periodic node wrap of the reference's halo copy: f(-k) = f(dim-k), f(dim+k) = f(k).
__device__ __forceinline__ int wrap_node(int n, int dim) {
  return n < 0 ? n + dim : (n > dim ? n - dim : n);
}

}  // namespace astr
