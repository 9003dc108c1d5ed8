// Host construction of the line operators: the reference's scheme set-up restated in C++, and
// the lane tables the segmented solve reads.
//   fd_scheme_initiate          src/derivative.F90:63-158
//   compact_filter_initiate     src/filter.F90:31-100
//   filter_coefficient_cal      src/filter.F90:299-432
//   compact_flux_initiate       src/flux.F90:32-112
//   tridiagonal_thomas_proprocess src/commfunc.F90:752-774
#include <cmath>
#include <cstring>

#include "internal.h"

namespace astr {

static void thomas_factor(HostOp& op) {
  const int n = op.nsys();
  op.ac1.assign(n, 0.0); op.ac2.assign(n, 0.0); op.ac3.assign(n, 0.0);
  op.ac1[0] = op.c[0];
  for (int i = 1; i < n; ++i) {
    const double piv = 1.0 - op.a[i] * op.ac1[i - 1];
    op.ac1[i] = op.c[i] / piv;
    op.ac2[i] = 1.0 / piv;
    op.ac3[i] = op.a[i] / piv;
  }
}

static void set_range(HostOp& op, int ntype, int dim, int ext) {
  op.ntype = ntype;
  op.dim = dim;
  op.left_phys = (ntype == 1 || ntype == 4);
  op.right_phys = (ntype == 2 || ntype == 4);
  op.first_node = op.left_phys ? 0 : -ext;
  op.last_node = op.right_phys ? dim : dim + ext;
}

bool build_fd_op(HostOp& op, const char* scheme, int ntype, int dim) {
  if (ntype < 1 || ntype > 4 || dim < 8) return false;
  const int nscheme = (scheme[0] - '0') * 100 + (scheme[1] - '0') * 10 + (scheme[2] - '0');
  if (scheme[3] == 'e' && nscheme / 100 == 6) {
    // explicit central scheme: diff6ec has no system; rows are nodes 0..dim
    op.kind = OP_EXPLICIT;
    op.ntype = ntype; op.dim = dim;
    op.left_phys = (ntype == 1 || ntype == 4);
    op.right_phys = (ntype == 2 || ntype == 4);
    op.first_node = 0; op.last_node = dim;
    const int n = op.nsys();
    op.a.assign(n, 0.0); op.c.assign(n, 0.0);
    thomas_factor(op);
    return true;
  }
  if (scheme[3] != 'c' || nscheme != 643) return false;
  op.kind = OP_DERIV;
  set_range(op, ntype, dim, 1);
  const int n = op.nsys();
  op.a.assign(n, 1.0 / 3.0);
  op.c.assign(n, 1.0 / 3.0);
  // explicit 6th-order rows at interfaces
  op.a[0] = op.c[0] = 0.0;
  op.a[n - 1] = op.c[n - 1] = 0.0;
  if (op.left_phys) {
    op.a[0] = op.c[0] = 2.0;      // 3rd-order biased compact closure
    op.a[1] = op.c[1] = 0.25;     // 4th-order compact
  }
  if (op.right_phys) {
    op.a[n - 1] = op.c[n - 1] = 2.0;
    op.a[n - 2] = op.c[n - 2] = 0.25;
  }
  thomas_factor(op);
  return true;
}

void build_filter_op(HostOp& op, int ntype, int dim, double alfa, double bh, double bb, bool note) {
  op.kind = OP_FILTER;
  set_range(op, ntype, dim, 3);
  op.no_note = note;
  const int n = op.nsys();
  // end-row LHS coefficients are fixed by ntype (filter.F90:44-68)
  const double b0 = op.left_phys ? 0.98 : 1.11;
  const double bm = op.right_phys ? 0.98 : 1.11;
  op.a.assign(n, alfa);
  op.c.assign(n, alfa);
  if (note) {
    op.a[0] = op.c[0] = 0.0;
    op.a[n - 1] = op.c[n - 1] = 0.0;
  } else {
    op.a[0] = op.c[0] = b0;
    op.a[n - 1] = op.c[n - 1] = bm;
  }
  thomas_factor(op);
  // RHS coefficients
  op.c6[0] = (11.0 + 10.0 * alfa) / 32.0;
  op.c6[1] = (15.0 + 34.0 * alfa) / 64.0;
  op.c6[2] = (-3.0 + 6.0 * alfa) / 32.0;
  op.c6[3] = (1.0 - 2.0 * alfa) / 64.0;
  op.c8[0] = (93.0 + 70.0 * alfa) / 256.0;
  op.c8[1] = (7.0 + 18.0 * alfa) / 32.0;
  op.c8[2] = (-7.0 + 14.0 * alfa) / 64.0;
  op.c8[3] = (1.0 - 2.0 * alfa) / 32.0;
  op.c8[4] = (-1.0 + 2.0 * alfa) / 256.0;
  op.c10[0] = (193.0 + 126.0 * alfa) / 512.0;
  op.c10[1] = (105.0 + 302.0 * alfa) / 512.0;
  op.c10[2] = (-15.0 + 30.0 * alfa) / 128.0;
  op.c10[3] = (45.0 - 90.0 * alfa) / 1024.0;
  op.c10[4] = (-5.0 + 10.0 * alfa) / 512.0;
  op.c10[5] = (1.0 - 2.0 * alfa) / 1024.0;
  // one-sided rows 0..2 (row 0 carries beta_bound)
  const double b[3][7] = {
      {(63.0 + 1.0 * bb) / 64.0, (3.0 + 29.0 * bb) / 32.0, (-15.0 + 15.0 * bb) / 64.0, (5.0 - 5.0 * bb) / 16.0,
       (-15.0 + 15.0 * bb) / 64.0, (3.0 - 3.0 * bb) / 32.0, (-1.0 + 1.0 * bb) / 64.0},
      {(1.0 + 62.0 * alfa) / 64.0, (29.0 + 6.0 * alfa) / 32.0, (15.0 + 34.0 * alfa) / 64.0, (-5.0 + 10.0 * alfa) / 16.0,
       (15.0 - 30.0 * alfa) / 64.0, (-3.0 + 6.0 * alfa) / 32.0, (1.0 - 2.0 * alfa) / 64.0},
      {(-1.0 + 2.0 * alfa) / 64.0, (3.0 + 26.0 * alfa) / 32.0, (49.0 + 30.0 * alfa) / 64.0, (5.0 + 6.0 * alfa) / 16.0,
       (-15.0 + 30.0 * alfa) / 64.0, (3.0 - 6.0 * alfa) / 32.0, (-1.0 + 2.0 * alfa) / 64.0}};
  std::memcpy(op.cb, b, sizeof(b));
  // halo-closure rows 0..2 (row 0 carries beta_halo)
  const double h[3][11] = {
      {(-1.0 + 1.0 * bh) / 1024.0, (5.0 - 5.0 * bh) / 512.0, (979.0 + 45.0 * bh) / 1024.0, (15.0 + 113.0 * bh) / 128.0,
       (-105.0 + 105.0 * bh) / 512.0, (63.0 - 63.0 * bh) / 256.0, (-105.0 + 105.0 * bh) / 512.0,
       (15.0 - 15.0 * bh) / 128.0, (-45.0 + 45.0 * bh) / 1024.0, (5.0 - 5.0 * bh) / 512.0, (-1.0 + 1.0 * bh) / 1024.0},
      {(1.0 - 2.0 * alfa) / 1024.0, (-5.0 + 10.0 * alfa) / 512.0, (45.0 + 934.0 * alfa) / 1024.0,
       (113.0 + 30.0 * alfa) / 128.0, (105.0 + 302.0 * alfa) / 512.0, (-63.0 + 126.0 * alfa) / 256.0,
       (105.0 - 210.0 * alfa) / 512.0, (-15.0 + 30.0 * alfa) / 128.0, (45.0 - 90.0 * alfa) / 1024.0,
       (-5.0 + 10.0 * alfa) / 512.0, (1.0 - 2.0 * alfa) / 1024.0},
      {(-1.0 + 2.0 * alfa) / 1024.0, (5.0 - 10.0 * alfa) / 512.0, (-45.0 + 90.0 * alfa) / 1024.0,
       (15.0 + 98.0 * alfa) / 128.0, (407.0 + 210.0 * alfa) / 512.0, (63.0 + 130.0 * alfa) / 256.0,
       (-105.0 + 210.0 * alfa) / 512.0, (15.0 - 30.0 * alfa) / 128.0, (-45.0 + 90.0 * alfa) / 1024.0,
       (5.0 - 10.0 * alfa) / 512.0, (-1.0 + 2.0 * alfa) / 1024.0}};
  std::memcpy(op.ch, h, sizeof(h));
}

// The '543' compact interface-flux scheme: interfaces i_0..i_m with i_0 = -1 at a physical left
// end (ntype 1, 4) else -2, i_m = dim at a physical right end (ntype 2, 4) else dim + 1. Interior
// LHS a, c biased by the wind and blended by bfac (the MP-LD b factor, bfacmpld of commvar);
// explicit central rows (a = c = 0) at interfaces; at physical ends the 3rd-order rows with
// a = c = 2 and a = c = 1/4 next to them.
bool build_flux_op(HostOp& op, int scheme, int ntype, int dim, int wind, double bfac) {
  if (ntype < 1 || ntype > 4 || dim < 8 || scheme != 543 || (wind != 1 && wind != -1)) return false;
  op.kind = OP_FLUX;
  op.ntype = ntype;
  op.dim = dim;
  op.left_phys = (ntype == 1 || ntype == 4);
  op.right_phys = (ntype == 2 || ntype == 4);
  op.first_node = op.left_phys ? -1 : -2;
  op.last_node = op.right_phys ? dim : dim + 1;
  op.wind = wind;
  op.bfac = bfac;
  const int n = op.nsys();
  const double a = (wind == 1) ? 0.5 - (1.0 / 6.0) * bfac : (1.0 / 6.0) + (1.0 / 6.0) * bfac;
  const double c = (wind == 1) ? (1.0 / 6.0) + (1.0 / 6.0) * bfac : 0.5 - (1.0 / 6.0) * bfac;
  op.a.assign(n, a);
  op.c.assign(n, c);
  op.a[0] = op.c[0] = 0.0;
  op.a[n - 1] = op.c[n - 1] = 0.0;
  if (op.left_phys) {
    op.a[0] = op.c[0] = 2.0;
    op.a[1] = op.c[1] = 0.25;
  }
  if (op.right_phys) {
    op.a[n - 1] = op.c[n - 1] = 2.0;
    op.a[n - 2] = op.c[n - 2] = 0.25;
  }
  thomas_factor(op);
  op.cfl[0] = 1.0 / 18.0 - (1.0 / 36.0) * bfac;
  op.cfl[1] = 19.0 / 18.0 - (9.0 / 36.0) * bfac;
  op.cfl[2] = 5.0 / 9.0 + (9.0 / 36.0) * bfac;
  op.cfl[3] = (1.0 / 36.0) * bfac;
  return true;
}

std::vector<double> lane_tables(const HostOp& op, int S, int nseg) {
  const int nsys = op.nsys();
  const int WPL = nseg / 32;
  const size_t base = (size_t)5 * S * nseg;
  const size_t slot_off = base + (size_t)T_NSEGTAB * nseg + 2 * (size_t)WPL;
  std::vector<double> t(slot_off + (size_t)(nseg + 1) / 2, 0.0);
  // f: 0 ac1, 1 ac2, 2 ac3, 3 pf, 4 qb (see the layout in ops.cuh)
  auto at = [&](int f, int tt, int seg) -> double& {
    const size_t rs = (size_t)tt * nseg + seg;
    switch (f) {
      case 1: return t[2 * rs];
      case 2: return t[2 * rs + 1];
      case 3: return t[(size_t)2 * S * nseg + rs];
      case 0: return t[(size_t)3 * S * nseg + 2 * rs];
      default: return t[(size_t)3 * S * nseg + 2 * rs + 1];
    }
  };
  auto sg = [&](int k, int seg) -> double& { return t[base + (size_t)k * nseg + seg]; };
  std::vector<double> mf(nseg), mb(nseg);
  for (int seg = 0; seg < nseg; ++seg) {
    double e1[64], e2[64], e3[64];
    for (int tt = 0; tt < S; ++tt) {
      const int r = seg * S + tt;
      if (r < nsys) {
        e1[tt] = (r == nsys - 1) ? 0.0 : op.ac1[r];  // back substitution starts at x_n = d_n
        e2[tt] = (r == 0) ? 1.0 : op.ac2[r];         // row 1 of the forward sweep is untouched
        e3[tt] = (r == 0) ? 0.0 : op.ac3[r];
      } else {
        e1[tt] = e2[tt] = e3[tt] = 0.0;              // padding rows solve to zero
      }
      at(0, tt, seg) = e1[tt];
      at(1, tt, seg) = e2[tt];
      at(2, tt, seg) = e3[tt];
    }
    double p = 1.0;
    for (int tt = 0; tt < S; ++tt) { p *= -e3[tt]; at(3, tt, seg) = p; }
    mf[seg] = p;
    double q = 1.0;
    for (int tt = S - 1; tt >= 0; --tt) { q *= -e1[tt]; at(4, tt, seg) = q; }
    mb[seg] = q;
  }
  // scan composites within each warp (see seg_solve)
  for (int w = 0; w < WPL; ++w) {
    const int s0 = 32 * w;
    for (int l = 0; l < 32; ++l) {
      for (int k = 0; k < 5; ++k) {
        const int off = 1 << k;
        double pf = 0.0, pb = 0.0;
        if (l >= off) { pf = 1.0; for (int j = l - off + 1; j <= l; ++j) pf *= mf[s0 + j]; }
        if (l + off <= 31) { pb = 1.0; for (int j = l; j <= l + off - 1; ++j) pb *= mb[s0 + j]; }
        sg(T_FS + k, s0 + l) = pf;
        sg(T_BS + k, s0 + l) = pb;
      }
      double fe = 1.0, be = 1.0;
      for (int j = 0; j < l; ++j) fe *= mf[s0 + j];
      for (int j = l + 1; j < 32; ++j) be *= mb[s0 + j];
      sg(T_FE, s0 + l) = fe;
      sg(T_BE, s0 + l) = be;
    }
    double mw = 1.0, mwb = 1.0;
    for (int j = 0; j < 32; ++j) { mw *= mf[s0 + j]; mwb *= mb[s0 + j]; }
    t[base + (size_t)T_NSEGTAB * nseg + w] = mw;
    t[base + (size_t)T_NSEGTAB * nseg + WPL + w] = mwb;
  }
  // Row-coefficient slot of every segment: the first segment whose (ac2, ac3, pf, ac1, qb)
  // column is bitwise the same. Interior segments (converged factors) share one slot, so the
  // lanes of a warp read the same addresses and the loads are broadcasts.
  int* slot = reinterpret_cast<int*>(t.data() + slot_off);
  for (int seg = 0; seg < nseg; ++seg) {
    slot[seg] = seg;
    for (int o = 0; o < seg; ++o) {
      bool same = true;
      for (int f = 0; f < 5 && same; ++f)
        for (int tt = 0; tt < S && same; ++tt) same = at(f, tt, o) == at(f, tt, seg);
      if (same) { slot[seg] = o; break; }
    }
  }
  return t;
}

Layout pick_layout(int nsys_max) {
  if (nsys_max <= 96) return {3, 1};
  if (nsys_max <= 160) return {5, 1};
  if (nsys_max <= 288) return {9, 1};
  if (nsys_max <= 576) return {9, 2};
  if (nsys_max <= 1152) return {9, 4};
  return {0, 0};
}

void fill_lineop(const HostOp& h, LineOp& o) {
  o.tab = nullptr;
  o.nsys = h.nsys();
  o.ext_lo = -h.first_node;
  o.dim = h.dim;
  o.kind = h.kind;
  o.left_phys = h.left_phys;
  o.right_phys = h.right_phys;
  o.no_filter_note = h.no_note;
  o.nseg = 0;
  o.S = 0;
  // closure rows with their own RHS formulas (derivative.F90:230-294, filter.F90:176-269)
  if (h.kind == OP_FILTER) {
    o.spec_lo = h.left_phys ? 5 : 3;
    o.spec_hi = h.right_phys ? 5 : 3;
  } else {   // derivative and interface flux: two closure rows at a physical end, else one
    o.spec_lo = h.left_phys ? 2 : 1;
    o.spec_hi = h.right_phys ? 2 : 1;
  }
  std::memcpy(o.c10, h.c10, sizeof(o.c10));
  std::memcpy(o.ch, h.ch, sizeof(o.ch));
  std::memcpy(o.cb, h.cb, sizeof(o.cb));
  std::memcpy(o.c6, h.c6, sizeof(o.c6));
  std::memcpy(o.c8, h.c8, sizeof(o.c8));
  o.wind = h.wind;
  std::memcpy(o.cfl, h.cfl, sizeof(o.cfl));
}

cudaError_t make_devop(const HostOp& h, Layout lay, DevOp& out) {
  out.S = lay.S;
  out.WPL = lay.WPL;
  const int nseg = 32 * lay.WPL;
  std::vector<double> tab = lane_tables(h, lay.S, nseg);
  cudaError_t e = cudaMalloc(&out.dtab, tab.size() * sizeof(double));
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(out.dtab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  LineOp& o = out.op;
  fill_lineop(h, o);
  o.tab = out.dtab;
  o.nseg = nseg;
  o.S = lay.S;
  return cudaSuccess;
}

void free_devop(DevOp& d) {
  if (d.dtab) cudaFree(d.dtab);
  d.dtab = nullptr;
}

int tile_pitch(int dim, int TI, int S) {
  const int need = dim + 1 + 2 * HT + win_slack(S);   // halos and the window slack (ops.cuh)
  const int want = TI >= 16 ? 1 : 16 / TI;   // residue mod 16 for conflict-free line-fastest access
  int lp = need;
  while ((lp % 16) != (want % 16)) ++lp;
  return lp;
}

}  // namespace astr
