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

constexpr int HT = 8;             // tile halo nodes kept on each side of a line
constexpr unsigned FULL = 0xffffffffu;

enum OpKind { OP_DERIV = 0, OP_FILTER = 1, OP_EXPLICIT = 2 };

// One line operator (a compact_scheme of the reference plus the lane tables of its solve).
// Table layout (doubles), nseg = 32*WPL segments of S rows:
//   [(f*S + t)*nseg + seg]  f = 0 ac1, 1 ac2, 2 ac3, 3 pf (forward prefix product within the
//                           segment), 4 qb (backward suffix product within the segment)
//   then per segment (nseg each): FS[0..4] forward scan composites for shuffle offsets 1..16,
//   FE forward exclusive product within the warp, BS[0..4], BE (backward), and per warp
//   MW[WPL], MWB[WPL] (whole-warp products).
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
  double c10[6], ch[3][11], cb[3][7], c6[4], c8[5];  // filter coefficients (filter.F90:299-432)
};

enum TabOff { T_FS = 0, T_FE = 5, T_BS = 6, T_BE = 11, T_NSEGTAB = 12 };

// Barrier among the WPL warps of one line (named barrier 1 + line).
template <int WPL>
__device__ __forceinline__ void line_sync(int line) {
  if (WPL > 1) asm volatile("bar.sync %0, %1;" ::"r"(1 + line), "r"(32 * WPL) : "memory");
}

// Segmented Thomas solve. v holds the RHS rows of this lane on entry and the solution on exit.
// tab is the operator's lane table laid out for this (S, WPL); all offsets are compile-time.
// scan_sm: 2*WPL doubles private to this line (used only when WPL > 1). All warps of the line
// must call it together.
template <int S, int WPL>
__device__ __forceinline__ void seg_solve(double (&v)[S], const double* __restrict__ tab, int seg, int lane, int part,
                                          int line, double* scan_sm) {
  constexpr int NS = 32 * WPL;
  const double* tb = tab + seg;
  const double* ws = tab + (5 * S + T_NSEGTAB) * NS;   // per-warp products
  // forward sweep from a zero carry
  double g = 0.0;
#pragma unroll
  for (int t = 0; t < S; ++t) {
    g = v[t] * __ldg(tb + (S + t) * NS) - g * __ldg(tb + (2 * S + t) * NS);
    v[t] = g;
  }
  // inclusive scan of the segment maps c -> G + M c across the warp (composite M precomputed)
  double G = g;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double Go = __shfl_up_sync(FULL, G, 1 << k);
    G = fma(__ldg(tb + (5 * S + T_FS + k) * NS), Go, G);
  }
  double Ge = __shfl_up_sync(FULL, G, 1);
  if (lane == 0) Ge = 0.0;
  double cw = 0.0;
  if (WPL > 1) {
    if (lane == 31) scan_sm[part] = G;
    line_sync<WPL>(line);
    for (int p = 0; p < part; ++p) cw = fma(__ldg(ws + p), cw, scan_sm[p]);
  }
  const double cin = fma(__ldg(tb + (5 * S + T_FE) * NS), cw, Ge);
#pragma unroll
  for (int t = 0; t < S; ++t) v[t] = fma(__ldg(tb + (3 * S + t) * NS), cin, v[t]);

  // backward sweep from a zero carry
  double h = 0.0;
#pragma unroll
  for (int t = S - 1; t >= 0; --t) {
    h = v[t] - __ldg(tb + t * NS) * h;
    v[t] = h;
  }
  G = h;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double Go = __shfl_down_sync(FULL, G, 1 << k);
    G = fma(__ldg(tb + (5 * S + T_BS + k) * NS), Go, G);
  }
  Ge = __shfl_down_sync(FULL, G, 1);
  if (lane == 31) Ge = 0.0;
  cw = 0.0;
  if (WPL > 1) {
    if (lane == 0) scan_sm[WPL + part] = G;
    line_sync<WPL>(line);
    for (int p = WPL - 1; p > part; --p) cw = fma(__ldg(ws + WPL + p), cw, scan_sm[WPL + p]);
  }
  const double cb = fma(__ldg(tb + (5 * S + T_BE) * NS), cw, Ge);
#pragma unroll
  for (int t = 0; t < S; ++t) v[t] = fma(__ldg(tb + (4 * S + t) * NS), cb, v[t]);
}

// ---------------------------------------------------------------- right-hand sides
// Compact derivative closure rows, derivative.F90:230-294. Returns false for interior rows.
template <class Get>
__device__ __forceinline__ bool deriv_special(const LineOp& op, int r, Get f, double& out) {
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
// Closure rows of the compact derivative and zero padding rows; only lanes that hold them call
// this (deriv_edge_lane).
template <int S, class Get>
__device__ __forceinline__ void fix_deriv_rows(double (&v)[S], const LineOp& op, int r0, Get f) {
#pragma unroll
  for (int t = 0; t < S; ++t) {
    const int r = r0 + t;
    double s;
    if (r >= op.nsys) v[t] = 0.0;
    else if (deriv_special(op, r, f, s)) v[t] = s;
  }
}
template <int S>
__device__ __forceinline__ bool deriv_edge_lane(const LineOp& op, int r0) { return r0 < 2 || r0 + S > op.nsys - 2; }

// Fill w[t] = f(n0 + t), t < W, clamping to the staged range only for lanes near the ends.
template <int W, class Get>
__device__ __forceinline__ void fill_window(double (&w)[W], int n0, int dim, Get f) {
  if (n0 >= -HT && n0 + W - 1 <= dim + HT) {
#pragma unroll
    for (int t = 0; t < W; ++t) w[t] = f(n0 + t);
  } else {
#pragma unroll
    for (int t = 0; t < W; ++t) {
      int n = n0 + t;
      n = n < -HT ? -HT : (n > dim + HT ? dim + HT : n);
      w[t] = f(n);
    }
  }
}

template <int S, class Get>
__device__ __forceinline__ void rhs_deriv(double (&v)[S], const LineOp& op, int seg, Get f) {
  const int r0 = seg * S;
  double w[S + 4];
  fill_window<S + 4>(w, r0 - op.ext_lo - 2, op.dim, f);
  stencil_deriv<S>(v, w);
  if (deriv_edge_lane<S>(op, r0)) fix_deriv_rows<S>(v, op, r0, f);
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
__device__ __forceinline__ bool filter_special(const LineOp& op, int r, Get f, double& out) {
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

// Interior 11-point filter RHS (filter.F90:271-283) over a sliding window, then closure rows.
template <int S, class Get>
__device__ __forceinline__ void rhs_filter(double (&v)[S], const LineOp& op, int seg, Get f) {
  const int r0 = seg * S;
  double w[S + 10];
  fill_window<S + 10>(w, r0 - op.ext_lo - 5, op.dim, f);
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
  const int nspec = op.left_phys || op.right_phys ? 5 : 3;
  if (r0 < nspec || r0 + S > op.nsys - nspec) {
#pragma unroll
    for (int t = 0; t < S; ++t) {
      const int r = r0 + t;
      double s;
      if (r >= op.nsys) v[t] = 0.0;
      else if (filter_special(op, r, f, s)) v[t] = s;
    }
  }
}

// Periodic node wrap of the reference's halo copy: f(-k) = f(dim-k), f(dim+k) = f(k).
__device__ __forceinline__ int wrap_node(int n, int dim) {
  return n < 0 ? n + dim : (n > dim ? n - dim : n);
}

}  // namespace astr
