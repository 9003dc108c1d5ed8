// ORACLE — test infrastructure only. Nothing in the product path links or calls this file.
//
// A CPU restatement, in C++17, of the reference ASTR (Perrbit/astr_gpu) CPU algorithm for the
// per-step RHS hot path. Each routine follows the reference routine it names, in the same
// operation order, so that with -ffp-contract=off it reproduces the reference's arithmetic:
//
//   commfunc.F90:752-813        tridiagonal_thomas_proprocess / tridiagonal_thomas_solver
//   derivative.F90:63-306       fd_scheme_initiate, df_compact, compact_fd_rhs
//   derivative.F90:350-413      diff6ec (explicit 6th-order, the '643e' scheme)
//   filter.F90:31-285, 299-432  compact_filter_initiate, compact_filter, compact_filter_rhs,
//                               filter_coefficient_cal
//   miniapps/tgv_solver_3d/tgvsolver.F90:48-1082
//                               the Taylor-Green miniapp: fvar2q, thermal_scar, q2fvar, miucal,
//                               flowfield_init, bchomo/bchomovec, gradcal, convection,
//                               diffusion, filterq, stacal, rhscal, rk3
//   commcal.F90:27-87           cflcal (only to fix dt once at t=0)
//   statistic.F90:993-1040      diss_rate_cal (dissipation diagnostic)
//
// Parity is pinned by the reference's golden history miniapps/tgv_solver_3d/state.ref_128
// (kinetic energy and enstrophy, 100 steps at 128^3), checked in tests/test_oracle_golden.py.
//
// OpenMP splits only independent line loops; every reduction keeps the reference's
// sequential i-fastest order.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <string>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int HM = 5;                      // halo width, commvar.F90:190
constexpr double num1d3 = 1.0 / 3.0;       // constdef.F90:13-27
constexpr double num2d3 = 2.0 / 3.0;
constexpr double num7d9 = 7.0 / 9.0;
constexpr double num1d36 = 1.0 / 36.0;
constexpr double num1d60 = 1.0 / 60.0;
constexpr double num1d12 = 1.0 / 12.0;
constexpr double num1d6 = 1.0 / 6.0;
constexpr double num1d18 = 1.0 / 18.0;
constexpr double num19d18 = 19.0 / 18.0;
constexpr double num5d9 = 5.0 / 9.0;
constexpr double num9d36 = 9.0 / 36.0;
constexpr double num2d15 = 2.0 / 15.0;
constexpr double num37d60 = 37.0 / 60.0;

// ---------------------------------------------------------------- compact_scheme (commtype.F90:13-23)
struct Scheme {
  int first_node = 0, last_node = 0, dimension = 0, nbctype = 3;
  bool compact = true;       // '643c' (compact) or '643e' (explicit)
  bool is_filter = false;
  bool no_filter_note = false;
  std::vector<double> a, c;  // index 0 <-> first_node
  std::vector<double> ac1, ac2, ac3;
  // filter coefficients carried by the scheme (filter.F90:17-20 keeps them module-global)
  double coef6i[4], coef8i[5], coef10i[6], coefb[5][9], coefh[5][11];
  int n() const { return last_node - first_node + 1; }
  // compact interface flux (flux.F90): wind '+' (upwind-biased) or '-', and the MP-LD b factor
  bool is_flux = false;
  int wind = 1;
  double bfac = 0.0;
};

// tridiagonal_thomas_proprocess, commfunc.F90:752-774
void thomas_proprocess(Scheme& s) {
  const int n = s.n();
  s.ac1.assign(n, 0.0); s.ac2.assign(n, 0.0); s.ac3.assign(n, 0.0);
  s.ac1[0] = s.c[0];
  for (int i = 1; i < n; ++i) {
    s.ac1[i] = s.c[i] / (1.0 - s.a[i] * s.ac1[i - 1]);
    s.ac2[i] = 1.0 / (1.0 - s.a[i] * s.ac1[i - 1]);
    s.ac3[i] = s.a[i] / (1.0 - s.a[i] * s.ac1[i - 1]);
  }
}

// tridiagonal_thomas_solver, commfunc.F90:790-813 (d is overwritten, x returned)
void thomas_solve(const Scheme& s, double* d, double* x) {
  const int n = s.n();
  for (int i = 1; i < n; ++i) d[i] = d[i] * s.ac2[i] - d[i - 1] * s.ac3[i];
  x[n - 1] = d[n - 1];
  for (int i = n - 2; i >= 0; --i) x[i] = d[i] - s.ac1[i] * x[i + 1];
}

void node_range(int ntype, int dim, int ext, int& i0, int& im_) {
  switch (ntype) {
    case 1: i0 = 0;    im_ = dim + ext; break;
    case 2: i0 = -ext; im_ = dim;       break;
    case 3: i0 = -ext; im_ = dim + ext; break;
    default: i0 = 0;   im_ = dim;       break;  // 4
  }
}

// fd_scheme_initiate, derivative.F90:63-158 ('643c' and '643e' are the only schemes it defines)
bool fd_scheme_initiate(Scheme& s, const char* scheme, int ntype, int dim) {
  int i0, imx;
  node_range(ntype, dim, 1, i0, imx);
  s.first_node = i0; s.last_node = imx; s.dimension = dim; s.nbctype = ntype;
  const int n = s.n();
  s.a.assign(n, 0.0); s.c.assign(n, 0.0);
  int nscheme = (scheme[0] - '0') * 100 + (scheme[1] - '0') * 10 + (scheme[2] - '0');
  if (scheme[3] == 'e') { s.compact = false; return nscheme == 643 || nscheme / 100 == 6; }
  if (scheme[3] != 'c' || nscheme != 643) return false;
  s.compact = true;
  for (int i = 0; i < n; ++i) { s.a[i] = num1d3; s.c[i] = num1d3; }
  s.a[0] = 0.0; s.c[0] = 0.0;
  s.a[n - 1] = 0.0; s.c[n - 1] = 0.0;
  if (ntype == 1 || ntype == 4) {
    s.a[0] = 2.0; s.c[0] = 2.0;
    s.a[1] = 0.25; s.c[1] = 0.25;
  }
  if (ntype == 2 || ntype == 4) {
    s.a[n - 1] = 2.0; s.c[n - 1] = 2.0;
    s.a[n - 2] = 0.25; s.c[n - 2] = 0.25;
  }
  thomas_proprocess(s);
  return true;
}

// compact_fd_rhs, derivative.F90:210-306. f points at f(0); valid f(-HM..dim+HM).
void compact_fd_rhs(const Scheme& s, const double* f, double* d) {
  const int i0 = s.first_node, im_ = s.last_node, nt = s.nbctype;
  auto D = [&](int j) -> double& { return d[j - i0]; };
  int is, ie;
  if (nt == 1 || nt == 4) {
    is = i0 + 2;
    int j = i0 + 1;
    double var1 = f[j + 1] - f[j - 1];
    D(j) = 0.75 * var1;
    j = i0;
    D(j) = -2.5 * f[j] + 2.0 * f[j + 1] + 0.5 * f[j + 2];
  } else {
    is = i0 + 1;
    int j = i0;
    double var1 = f[j + 1] - f[j - 1];
    double var2 = f[j + 2] - f[j - 2];
    double var3 = f[j + 3] - f[j - 3];
    D(j) = 0.75 * var1 - 0.15 * var2 + num1d60 * var3;
  }
  if (nt == 2 || nt == 4) {
    ie = im_ - 2;
    int j = im_ - 1;
    double var1 = f[j + 1] - f[j - 1];
    D(j) = 0.75 * var1;
    j = im_;
    D(j) = 2.5 * f[j] - 2.0 * f[j - 1] - 0.5 * f[j - 2];
  } else {
    ie = im_ - 1;
    int j = im_;
    double var1 = f[j + 1] - f[j - 1];
    double var2 = f[j + 2] - f[j - 2];
    double var3 = f[j + 3] - f[j - 3];
    D(j) = 0.75 * var1 - 0.15 * var2 + num1d60 * var3;
  }
  for (int j = is; j <= ie; ++j) {
    double var1 = f[j + 1] - f[j - 1];
    double var2 = f[j + 2] - f[j - 2];
    D(j) = num7d9 * var1 + num1d36 * var2;
  }
}

// diff6ec, derivative.F90:350-413
void diff6ec(const double* v, int dim, int ntype, double* out) {
  auto e6 = [&](int i) {
    return 0.75 * (v[i + 1] - v[i - 1]) - 0.15 * (v[i + 2] - v[i - 2]) + num1d60 * (v[i + 3] - v[i - 3]);
  };
  switch (ntype) {
    case 1:
      out[0] = -0.5 * v[2] + 2.0 * v[1] - 1.5 * v[0];
      out[1] = 0.5 * (v[2] - v[0]);
      out[2] = num2d3 * (v[3] - v[1]) - num1d12 * (v[4] - v[0]);
      for (int i = 3; i <= dim; ++i) out[i] = e6(i);
      break;
    case 2:
      for (int i = 0; i <= dim - 3; ++i) out[i] = e6(i);
      out[dim - 2] = num2d3 * (v[dim - 1] - v[dim - 3]) - num1d12 * (v[dim] - v[dim - 4]);
      out[dim - 1] = 0.5 * (v[dim] - v[dim - 2]);
      out[dim] = 0.5 * v[dim - 2] - 2.0 * v[dim - 1] + 1.5 * v[dim];
      break;
    case 3:
      for (int i = 0; i <= dim; ++i) out[i] = e6(i);
      break;
    default:
      out[0] = -0.5 * v[2] + 2.0 * v[1] - 1.5 * v[0];
      out[1] = 0.5 * (v[2] - v[0]);
      out[2] = num2d3 * (v[3] - v[1]) - num1d12 * (v[4] - v[0]);
      for (int i = 3; i <= dim - 3; ++i) out[i] = e6(i);
      out[dim - 2] = num2d3 * (v[dim - 1] - v[dim - 3]) - num1d12 * (v[dim] - v[dim - 4]);
      out[dim - 1] = 0.5 * (v[dim] - v[dim - 2]);
      out[dim] = 0.5 * v[dim - 2] - 2.0 * v[dim - 1] + 1.5 * v[dim];
      break;
  }
}

// df_compact / df_explicit, derivative.F90:171-198 and :319-336. scratch >= 2*(dim+3)
void df_line(const Scheme& s, const double* f, double* df, double* scratch) {
  if (!s.compact) { diff6ec(f, s.dimension, s.nbctype, df); return; }
  const int n = s.n();
  double* d = scratch;
  double* xx = scratch + n;
  compact_fd_rhs(s, f, d);
  thomas_solve(s, d, xx);
  for (int i = 0; i <= s.dimension; ++i) df[i] = xx[i - s.first_node];
}

// ---------------------------------------------------------------- compact interface flux
// compact_flux_initiate, flux.F90:32-112: the '543' compact interface scheme, rows i_0..i_m with
// i_0 = -1 (ntype 1, 4) or -2 (2, 3) and i_m = dim+1 (1, 3) or dim (2, 4); interior a, c biased
// by the wind and blended by bfac; explicit central rows at interfaces, 3rd-order rows at
// physical ends.
bool compact_flux_initiate(Scheme& s, int scheme, int ntype, int dim, int wind, double bfac) {
  int i0, imx;
  switch (ntype) {
    case 1: i0 = -1; imx = dim + 1; break;
    case 2: i0 = -2; imx = dim;     break;
    case 3: i0 = -2; imx = dim + 1; break;
    case 4: i0 = -1; imx = dim;     break;
    default: return false;
  }
  s.first_node = i0; s.last_node = imx; s.dimension = dim; s.nbctype = ntype;
  s.is_flux = true; s.wind = wind; s.bfac = bfac;
  const int n = s.n();
  s.a.assign(n, 0.0); s.c.assign(n, 0.0);
  if (scheme / 100 != 5 || (wind != 1 && wind != -1)) return false;
  for (int i = 0; i < n; ++i) {
    if (wind == 1) { s.a[i] = 0.5 - num1d6 * bfac; s.c[i] = num1d6 + num1d6 * bfac; }
    else { s.a[i] = num1d6 + num1d6 * bfac; s.c[i] = 0.5 - num1d6 * bfac; }
  }
  s.a[0] = 0.0; s.c[0] = 0.0;
  s.a[n - 1] = 0.0; s.c[n - 1] = 0.0;
  if (scheme != 543) return false;
  if (ntype == 1 || ntype == 4) { s.a[0] = 2.0; s.c[0] = 2.0; s.a[1] = 0.25; s.c[1] = 0.25; }
  if (ntype == 2 || ntype == 4) { s.a[n - 1] = 2.0; s.c[n - 1] = 2.0; s.a[n - 2] = 0.25; s.c[n - 2] = 0.25; }
  thomas_proprocess(s);
  return true;
}

// compact_flux_rhs, flux.F90:163-256 (f points at node 0 of f(-hm..dim+hm))
void compact_flux_rhs(const Scheme& s, const double* f, double* d) {
  const int i0 = s.first_node, imx = s.last_node, ntype = s.nbctype;
  const double b = s.bfac;
  auto D = [&](int j) -> double& { return d[j - i0]; };
  int is = i0 + 1, ie = imx - 1;
  if (ntype == 1 || ntype == 4) {
    int j = i0;
    D(j) = 2.5 * f[j + 1] + 0.5 * f[j + 2];
    j = i0 + 1;
    D(j) = 0.75 * f[j] + 0.75 * f[j + 1];
    is = i0 + 2;
  } else {
    const int j = i0;
    const double var1 = f[j] + f[j + 1], var2 = f[j - 1] + f[j + 2], var3 = f[j - 2] + f[j + 3];
    D(j) = num37d60 * var1 - num2d15 * var2 + num1d60 * var3;
  }
  if (ntype == 2 || ntype == 4) {
    int j = imx - 1;
    D(j) = 0.75 * f[j + 1] + 0.75 * f[j];
    j = imx;
    D(j) = 2.5 * f[j] + 0.5 * f[j - 1];
    ie = imx - 2;
  } else {
    const int j = imx;
    const double var1 = f[j] + f[j + 1], var2 = f[j - 1] + f[j + 2], var3 = f[j - 2] + f[j + 3];
    D(j) = num37d60 * var1 - num2d15 * var2 + num1d60 * var3;
  }
  if (s.wind == 1) {
    for (int j = is; j <= ie; ++j)
      D(j) = (num1d18 - num1d36 * b) * f[j - 1] + (num19d18 - num9d36 * b) * f[j] + (num5d9 + num9d36 * b) * f[j + 1] +
             num1d36 * b * f[j + 2];
  } else {
    for (int j = is; j <= ie; ++j)
      D(j) = (num1d18 - num1d36 * b) * f[j + 2] + (num19d18 - num9d36 * b) * f[j + 1] + (num5d9 + num9d36 * b) * f[j] +
             num1d36 * b * f[j - 1];
  }
}

// flux_compact, flux.F90:125-150: interface values fh(-1:dim) -> fh[0..dim+1]. scratch >= 2*(dim+4)
void flux_line(const Scheme& s, const double* f, double* fh, double* scratch) {
  const int n = s.n();
  double* d = scratch;
  double* xx = scratch + n;
  compact_flux_rhs(s, f, d);
  thomas_solve(s, d, xx);
  for (int i = -1; i <= s.dimension; ++i) fh[i + 1] = xx[i - s.first_node];
}

// filter_coefficient_cal, filter.F90:299-432
void filter_coefficient_cal(Scheme& s, double alfa, double beter_halo, double beter_bouond) {
  s.coef6i[0] = (11.0 + 10.0 * alfa) / 32.0;
  s.coef6i[1] = (15.0 + 34.0 * alfa) / 64.0;
  s.coef6i[2] = (-3.0 + 6.0 * alfa) / 32.0;
  s.coef6i[3] = (1.0 - 2.0 * alfa) / 64.0;
  s.coef8i[0] = (93.0 + 70.0 * alfa) / 256.0;
  s.coef8i[1] = (7.0 + 18.0 * alfa) / 32.0;
  s.coef8i[2] = (-7.0 + 14.0 * alfa) / 64.0;
  s.coef8i[3] = (1.0 - 2.0 * alfa) / 32.0;
  s.coef8i[4] = (-1.0 + 2.0 * alfa) / 256.0;
  s.coef10i[0] = (193.0 + 126.0 * alfa) / 512.0;
  s.coef10i[1] = (105.0 + 302.0 * alfa) / 512.0;
  s.coef10i[2] = (-15.0 + 30.0 * alfa) / 128.0;
  s.coef10i[3] = (45.0 - 90.0 * alfa) / 1024.0;
  s.coef10i[4] = (-5.0 + 10.0 * alfa) / 512.0;
  s.coef10i[5] = (1.0 - 2.0 * alfa) / 1024.0;
  for (auto& r : s.coefb) for (double& v : r) v = 0.0;
  for (auto& r : s.coefh) for (double& v : r) v = 0.0;
  s.coefb[3][0] = (1.0 - 2.0 * alfa) / 256.0;
  s.coefb[3][1] = (-1.0 + 2.0 * alfa) / 32.0;
  s.coefb[3][2] = (7.0 + 50.0 * alfa) / 64.0;
  s.coefb[3][3] = (25.0 + 14.0 * alfa) / 32.0;
  s.coefb[3][4] = (35.0 + 58.0 * alfa) / 128.0;
  s.coefb[3][5] = (-7.0 + 14.0 * alfa) / 32.0;
  s.coefb[3][6] = (7.0 - 14.0 * alfa) / 64.0;
  s.coefb[3][7] = (-1.0 + 2.0 * alfa) / 32.0;
  s.coefb[3][8] = (1.0 - 2.0 * alfa) / 256.0;
  s.coefb[2][0] = (-1.0 + 2.0 * alfa) / 64.0;
  s.coefb[2][1] = (3.0 + 26.0 * alfa) / 32.0;
  s.coefb[2][2] = (49.0 + 30.0 * alfa) / 64.0;
  s.coefb[2][3] = (5.0 + 6.0 * alfa) / 16.0;
  s.coefb[2][4] = (-15.0 + 30.0 * alfa) / 64.0;
  s.coefb[2][5] = (3.0 - 6.0 * alfa) / 32.0;
  s.coefb[2][6] = (-1.0 + 2.0 * alfa) / 64.0;
  s.coefb[1][0] = (1.0 + 62.0 * alfa) / 64.0;
  s.coefb[1][1] = (29.0 + 6.0 * alfa) / 32.0;
  s.coefb[1][2] = (15.0 + 34.0 * alfa) / 64.0;
  s.coefb[1][3] = (-5.0 + 10.0 * alfa) / 16.0;
  s.coefb[1][4] = (15.0 - 30.0 * alfa) / 64.0;
  s.coefb[1][5] = (-3.0 + 6.0 * alfa) / 32.0;
  s.coefb[1][6] = (1.0 - 2.0 * alfa) / 64.0;
  s.coefb[0][0] = (63.0 + 1.0 * beter_bouond) / 64.0;
  s.coefb[0][1] = (3.0 + 29.0 * beter_bouond) / 32.0;
  s.coefb[0][2] = (-15.0 + 15.0 * beter_bouond) / 64.0;
  s.coefb[0][3] = (5.0 - 5.0 * beter_bouond) / 16.0;
  s.coefb[0][4] = (-15.0 + 15.0 * beter_bouond) / 64.0;
  s.coefb[0][5] = (3.0 - 3.0 * beter_bouond) / 32.0;
  s.coefb[0][6] = (-1.0 + 1.0 * beter_bouond) / 64.0;
  s.coefh[0][0] = (-1.0 + 1.0 * beter_halo) / 1024.0;
  s.coefh[0][1] = (5.0 - 5.0 * beter_halo) / 512.0;
  s.coefh[0][2] = (979.0 + 45.0 * beter_halo) / 1024.0;
  s.coefh[0][3] = (15.0 + 113.0 * beter_halo) / 128.0;
  s.coefh[0][4] = (-105.0 + 105.0 * beter_halo) / 512.0;
  s.coefh[0][5] = (63.0 - 63.0 * beter_halo) / 256.0;
  s.coefh[0][6] = (-105.0 + 105.0 * beter_halo) / 512.0;
  s.coefh[0][7] = (15.0 - 15.0 * beter_halo) / 128.0;
  s.coefh[0][8] = (-45.0 + 45.0 * beter_halo) / 1024.0;
  s.coefh[0][9] = (5.0 - 5.0 * beter_halo) / 512.0;
  s.coefh[0][10] = (-1.0 + 1.0 * beter_halo) / 1024.0;
  s.coefh[1][0] = (1.0 - 2.0 * alfa) / 1024.0;
  s.coefh[1][1] = (-5.0 + 10.0 * alfa) / 512.0;
  s.coefh[1][2] = (45.0 + 934.0 * alfa) / 1024.0;
  s.coefh[1][3] = (113.0 + 30.0 * alfa) / 128.0;
  s.coefh[1][4] = (105.0 + 302.0 * alfa) / 512.0;
  s.coefh[1][5] = (-63.0 + 126.0 * alfa) / 256.0;
  s.coefh[1][6] = (105.0 - 210.0 * alfa) / 512.0;
  s.coefh[1][7] = (-15.0 + 30.0 * alfa) / 128.0;
  s.coefh[1][8] = (45.0 - 90.0 * alfa) / 1024.0;
  s.coefh[1][9] = (-5.0 + 10.0 * alfa) / 512.0;
  s.coefh[1][10] = (1.0 - 2.0 * alfa) / 1024.0;
  s.coefh[2][0] = (-1.0 + 2.0 * alfa) / 1024.0;
  s.coefh[2][1] = (5.0 - 10.0 * alfa) / 512.0;
  s.coefh[2][2] = (-45.0 + 90.0 * alfa) / 1024.0;
  s.coefh[2][3] = (15.0 + 98.0 * alfa) / 128.0;
  s.coefh[2][4] = (407.0 + 210.0 * alfa) / 512.0;
  s.coefh[2][5] = (63.0 + 130.0 * alfa) / 256.0;
  s.coefh[2][6] = (-105.0 + 210.0 * alfa) / 512.0;
  s.coefh[2][7] = (15.0 - 30.0 * alfa) / 128.0;
  s.coefh[2][8] = (-45.0 + 90.0 * alfa) / 1024.0;
  s.coefh[2][9] = (5.0 - 10.0 * alfa) / 512.0;
  s.coefh[2][10] = (-1.0 + 2.0 * alfa) / 1024.0;
}

// compact_filter_initiate, filter.F90:31-100 (alfa plays the role of commvar's alfa_filter)
void compact_filter_initiate(Scheme& s, int ntype, int dim, double alfa, bool no_filter_note) {
  int i0, imx;
  double b0, bm;
  switch (ntype) {
    case 1: i0 = 0;  imx = dim + 3; b0 = 0.98; bm = 1.11; break;
    case 2: i0 = -3; imx = dim;     b0 = 1.11; bm = 0.98; break;
    case 3: i0 = -3; imx = dim + 3; b0 = 1.11; bm = 1.11; break;
    default: i0 = 0; imx = dim;     b0 = 0.98; bm = 0.98; break;
  }
  s.first_node = i0; s.last_node = imx; s.dimension = dim; s.nbctype = ntype;
  s.is_filter = true; s.no_filter_note = no_filter_note;
  const int n = s.n();
  s.a.assign(n, alfa); s.c.assign(n, alfa);
  if (no_filter_note) {
    s.a[0] = 0.0; s.c[0] = 0.0; s.a[n - 1] = 0.0; s.c[n - 1] = 0.0;
  } else {
    s.a[0] = b0; s.c[0] = b0; s.a[n - 1] = bm; s.c[n - 1] = bm;
  }
  thomas_proprocess(s);
}

// compact_filter_rhs, filter.F90:156-285. f points at f(0).
void compact_filter_rhs(const Scheme& s, const double* f, double* d) {
  const int i0 = s.first_node, im_ = s.last_node, nt = s.nbctype;
  auto D = [&](int j) -> double& { return d[j - i0]; };
  int is, ie;
  if (nt == 1 || nt == 4) {
    is = i0 + 5;
    for (int k = i0; k <= i0 + 2; ++k) {
      double var0 = 0.0;
      for (int j = 0; j <= 6; ++j) var0 = var0 + s.coefb[k - i0][j] * f[i0 + j];
      D(k) = var0;
    }
    int j = i0 + 3;
    double var0 = f[j] + f[j], var1 = f[j + 1] + f[j - 1], var2 = f[j + 2] + f[j - 2],
           var3 = f[j + 3] + f[j - 3];
    D(j) = s.coef6i[0] * var0 + s.coef6i[1] * var1 + s.coef6i[2] * var2 + s.coef6i[3] * var3;
    j = i0 + 4;
    var0 = f[j] + f[j]; var1 = f[j + 1] + f[j - 1]; var2 = f[j + 2] + f[j - 2];
    var3 = f[j + 3] + f[j - 3];
    double var4 = f[j + 4] + f[j - 4];
    D(j) = s.coef8i[0] * var0 + s.coef8i[1] * var1 + s.coef8i[2] * var2 + s.coef8i[3] * var3 +
           s.coef8i[4] * var4;
  } else {
    is = i0 + 3;
    for (int k = i0; k <= i0 + 2; ++k) {
      double var0 = 0.0;
      for (int j = 0; j <= 10; ++j) var0 = var0 + s.coefh[k - i0][j] * f[i0 - 2 + j];
      D(k) = var0;
    }
  }
  if (nt == 2 || nt == 4) {
    ie = im_ - 5;
    for (int k = im_ - 2; k <= im_; ++k) {
      double var0 = 0.0;
      for (int j = 0; j <= 6; ++j) var0 = var0 + s.coefb[im_ - k][j] * f[im_ - j];
      D(k) = var0;
    }
    int j = im_ - 3;
    double var0 = f[j] + f[j], var1 = f[j + 1] + f[j - 1], var2 = f[j + 2] + f[j - 2],
           var3 = f[j + 3] + f[j - 3];
    D(j) = s.coef6i[0] * var0 + s.coef6i[1] * var1 + s.coef6i[2] * var2 + s.coef6i[3] * var3;
    j = im_ - 4;
    var0 = f[j] + f[j]; var1 = f[j + 1] + f[j - 1]; var2 = f[j + 2] + f[j - 2];
    var3 = f[j + 3] + f[j - 3];
    double var4 = f[j + 4] + f[j - 4];
    D(j) = s.coef8i[0] * var0 + s.coef8i[1] * var1 + s.coef8i[2] * var2 + s.coef8i[3] * var3 +
           s.coef8i[4] * var4;
  } else {
    ie = im_ - 3;
    for (int k = im_ - 2; k <= im_; ++k) {
      double var0 = 0.0;
      for (int j = 0; j <= 10; ++j) var0 = var0 + s.coefh[im_ - k][j] * f[im_ + 2 - j];
      D(k) = var0;
    }
  }
  if (s.no_filter_note) { D(i0) = f[i0]; D(im_) = f[im_]; }
  for (int j = is; j <= ie; ++j) {
    double var0 = f[j] + f[j];
    double var1 = f[j + 1] + f[j - 1];
    double var2 = f[j + 2] + f[j - 2];
    double var3 = f[j + 3] + f[j - 3];
    double var4 = f[j + 4] + f[j - 4];
    double var5 = f[j + 5] + f[j - 5];
    D(j) = s.coef10i[0] * var0 + s.coef10i[1] * var1 + s.coef10i[2] * var2 + s.coef10i[3] * var3 +
           s.coef10i[4] * var4 + s.coef10i[5] * var5;
  }
}

// compact_filter, filter.F90:112-144. scratch >= 2*(dim+7)
void filter_line(const Scheme& s, const double* f, double* ff, double* scratch) {
  const int n = s.n();
  double* d = scratch;
  double* xx = scratch + n;
  compact_filter_rhs(s, f, d);
  thomas_solve(s, d, xx);
  for (int i = 0; i <= s.dimension; ++i) ff[i] = xx[i - s.first_node];
  if (s.nbctype == 1 || s.nbctype == 4) ff[0] = f[0];
  if (s.nbctype == 2 || s.nbctype == 4) ff[s.dimension] = f[s.dimension];
}

// ---------------------------------------------------------------- 3-D helpers
// Fortran-ordered array a(l0:l0+n0-1, l1:l1+n1-1, l2:l2+n2-1, 1:nf), first index fastest.
struct Box {
  int64_t n[3], l[3];
  int64_t idx(int64_t i, int64_t j, int64_t k) const {
    return ((k - l[2]) * n[1] + (j - l[1])) * n[0] + (i - l[0]);
  }
  int64_t size() const { return n[0] * n[1] * n[2]; }
};

// Apply a line operator along `dir` (0,1,2) to every line of every field. Input lines must
// carry f(-HM..dim+HM) along dir (ntype 3) or f(0..dim) (ntype 4); output spans 0..dim.
template <class LineFn>
void apply_lines(const Scheme& s, int dir, const double* f, const Box& bf, int nfields, double* out,
                 LineFn fn) {
  Box bo = bf;
  bo.n[dir] = s.dimension + 1;
  bo.l[dir] = 0;
  const int o1 = (dir == 0) ? 1 : 0;
  const int o2 = (dir == 2) ? 1 : 2;
  const int64_t n1 = bf.n[o1], n2 = bf.n[o2];
  const int L = s.dimension + 1 + 2 * HM;
#pragma omp parallel
  {
    std::vector<double> lin(L, 0.0), lout(s.dimension + 1), scr(2 * (s.dimension + 8));
#pragma omp for collapse(2) schedule(static)
    for (int64_t b = 0; b < n2; ++b)
      for (int64_t a = 0; a < n1; ++a) {
        int64_t ijk[3];
        ijk[o1] = bf.l[o1] + a;
        ijk[o2] = bf.l[o2] + b;
        for (int m = 0; m < nfields; ++m) {
          const double* fm = f + m * bf.size();
          double* om = out + m * bo.size();
          for (int t = -HM; t <= s.dimension + HM; ++t) {
            int64_t p[3] = {ijk[0], ijk[1], ijk[2]};
            p[dir] = t;
            lin[t + HM] = (t >= bf.l[dir] && t < bf.l[dir] + bf.n[dir]) ? fm[bf.idx(p[0], p[1], p[2])] : 0.0;
          }
          fn(s, lin.data() + HM, lout.data(), scr.data());
          for (int t = 0; t <= s.dimension; ++t) {
            int64_t p[3] = {ijk[0], ijk[1], ijk[2]};
            p[dir] = t;
            om[bo.idx(p[0], p[1], p[2])] = lout[t];
          }
        }
      }
  }
}

// ---------------------------------------------------------------- TGV miniapp (tgvsolver.F90)
struct Field3 {
  int64_t ni, nj, nk, li, lj, lk;
  std::vector<double> v;
  void init(int im, int jm, int km, int h, int ncomp) {
    ni = im + 1 + 2 * h; nj = jm + 1 + 2 * h; nk = km + 1 + 2 * h;
    li = lj = lk = -h;
    v.assign((size_t)(ni * nj * nk * ncomp), 0.0);
  }
  double& operator()(int64_t i, int64_t j, int64_t k, int m = 0) {
    return v[(size_t)((((int64_t)m * nk + (k - lk)) * nj + (j - lj)) * ni + (i - li))];
  }
};

struct TGV {
  int im, jm, km;
  double gamma, mach, reynolds, prandtl, ref_tem, suth;
  double const1, const2, const3, const4, const5, const6, const7;
  double dx, dy, dz, deltat, time;
  int nstep;
  bool lfilter;
  Scheme fds[3], flt[3];
  // boundary type per direction (fd_scheme_initiate's ntype: 3 periodic, 1/2/4 physical ends) and
  // the temperature of the isothermal no-slip walls at the physical ends (bctype 41)
  int ntype[3] = {3, 3, 3};
  double twall = 1.0;
  double alfa_f = 0.49, beta_h = 1.11, beta_b = 0.98;
  bool periodic(int d) const { return ntype[d] == 3; }
  // convection scheme of the full-solver mode: 643 central compact (convrsdcal6) or 543 the
  // upwind compact flux (convrsdcmp without characteristic decomposition), with its b factor
  int conschm = 643;
  double bfacmpld = 0.0;
  // characteristic decomposition of convrsdcmp (lchardecomp) with the Ducros sensor's threshold
  bool lchardecomp = false;
  double shkcrt = 0.0;
  Field3 ssf;                  // Ducros sensor (allocated with the decomposition)
  std::vector<char> lshock;    // shock flag on nodes 0..N
  Scheme fuw[3], fdw[3];
  Field3 q, rho, prs, tmp, vel, qrhs, dvel, dtmp, sigma, qflux, qsave;
  std::vector<double> hist;   // rows of (nstep, time, tke, enst, diss)
  std::vector<double> hist_c; // the same rows with compensated sums

  void setup(int im_, int jm_, int km_, double mach_, double re_, double pr_, double gam_,
             double ref_tem_, double suth_, double alfa_filter, double beta_halo, double beta_bound,
             int filter_on) {
    im = im_; jm = jm_; km = km_;
    mach = mach_; reynolds = re_; prandtl = pr_; gamma = gam_; ref_tem = ref_tem_; suth = suth_;
    lfilter = filter_on != 0;
    const int dims[3] = {im, jm, km};
    alfa_f = alfa_filter; beta_h = beta_halo; beta_b = beta_bound;
    for (int d = 0; d < 3; ++d) {
      ntype[d] = 3;
      fd_scheme_initiate(fds[d], "643c", 3, dims[d]);
      compact_filter_initiate(flt[d], 3, dims[d], alfa_filter, false);
      filter_coefficient_cal(flt[d], alfa_filter, beta_halo, beta_bound);
    }
    q.init(im, jm, km, HM, 5); rho.init(im, jm, km, HM, 1); prs.init(im, jm, km, HM, 1);
    tmp.init(im, jm, km, HM, 1); vel.init(im, jm, km, HM, 3);
    qrhs.init(im, jm, km, 0, 5); dvel.init(im, jm, km, 0, 9); dtmp.init(im, jm, km, 0, 3);
    sigma.init(im, jm, km, HM, 6); qflux.init(im, jm, km, HM, 3); qsave.init(im, jm, km, 0, 5);
    // flowfield_init constants, tgvsolver.F90:189-195
    const1 = 1.0 / (gamma * (gamma - 1.0) * (mach * mach));
    const2 = gamma * (mach * mach);
    const3 = (gamma - 1.0) / 3.0 * prandtl * (mach * mach);
    const4 = (gamma - 1.0) * (mach * mach) * reynolds * prandtl;
    const5 = (gamma - 1.0) * (mach * mach);
    const6 = 1.0 / (gamma - 1.0);
    const7 = (gamma - 1.0) * (mach * mach) * reynolds * prandtl;
    const double pi = 4.0 * std::atan(1.0);
    dx = 2.0 * pi / double(im); dy = 2.0 * pi / double(jm); dz = 2.0 * pi / double(km);
    nstep = 0; time = 0.0; deltat = 1e-3;
    hist.clear();
    hist_c.clear();
  }

  // fvar2q with pressure, tgvsolver.F90:48-71
  void fvar2q(double* qq, double density, const double* u, double pressure) const {
    qq[0] = density;
    qq[1] = density * u[0];
    qq[2] = density * u[1];
    qq[3] = density * u[2];
    double var1 = 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    qq[4] = pressure * const6 + density * var1;
  }
  // q2fvar with temperature, tgvsolver.F90:92-121
  void q2fvar(const double* qq, double& density, double* u, double& pressure, double& temperature) const {
    density = qq[0];
    u[0] = qq[1] / density; u[1] = qq[2] / density; u[2] = qq[3] / density;
    pressure = (qq[4] - 0.5 * density * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2])) / const6;
    temperature = pressure / density * const2;
  }
  double miucal(double t) const {  // tgvsolver.F90:123-140
    double tc = suth / ref_tem;
    double tc1 = 1.0 + tc;
    return t * std::sqrt(t) * tc1 / (t + tc);
  }

  // flowfield_init, tgvsolver.F90:172-234
  void init_tgv() {
    const double pi = 4.0 * std::atan(1.0);
    const double pinf = 1.0 / const2;
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          double x1 = 2.0 * pi / double(im) * double(i);
          double x2 = 2.0 * pi / double(jm) * double(j);
          double x3 = 2.0 * pi / double(km) * double(k);
          rho(i, j, k) = 1.0;
          vel(i, j, k, 0) = std::sin(x1) * std::cos(x2) * std::cos(x3);
          vel(i, j, k, 1) = -std::cos(x1) * std::sin(x2) * std::cos(x3);
          vel(i, j, k, 2) = 0.0;
          prs(i, j, k) = pinf + 1.0 / 16.0 * (std::cos(2.0 * x1) + std::cos(2.0 * x2)) * (std::cos(2.0 * x3) + 2.0);
          tmp(i, j, k) = prs(i, j, k) / rho(i, j, k) * const2;
          double u[3] = {vel(i, j, k, 0), vel(i, j, k, 1), vel(i, j, k, 2)};
          double qq[5];
          fvar2q(qq, rho(i, j, k), u, prs(i, j, k));
          for (int m = 0; m < 5; ++m) q(i, j, k, m) = qq[m];
        }
    nstep = 0; time = 0.0;
  }

  // Start from user conserved variables on nodes 0..N (Fortran order, 5 fields); prims by q2fvar.
  void set_q(const double* qin) {
    const int64_t n0 = im + 1, n1 = jm + 1, n2 = km + 1, nn = n0 * n1 * n2;
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          double qq[5];
          for (int m = 0; m < 5; ++m) { qq[m] = qin[m * nn + ((int64_t)k * n1 + j) * n0 + i]; q(i, j, k, m) = qq[m]; }
          double u[3], r, p, t;
          q2fvar(qq, r, u, p, t);
          rho(i, j, k) = r; prs(i, j, k) = p; tmp(i, j, k) = t;
          for (int c = 0; c < 3; ++c) vel(i, j, k, c) = u[c];
        }
  }
  void get_q(double* out) {
    const int64_t n0 = im + 1, n1 = jm + 1, n2 = km + 1, nn = n0 * n1 * n2;
    for (int m = 0; m < 5; ++m)
      for (int k = 0; k <= km; ++k)
        for (int j = 0; j <= jm; ++j)
          for (int i = 0; i <= im; ++i) out[m * nn + ((int64_t)k * n1 + j) * n0 + i] = q(i, j, k, m);
  }

  // bchomo, tgvsolver.F90:271-369
  void bchomo() {
    auto setq = [&](int i, int j, int k) {
      double u[3] = {vel(i, j, k, 0), vel(i, j, k, 1), vel(i, j, k, 2)};
      double qq[5];
      fvar2q(qq, rho(i, j, k), u, prs(i, j, k));
      for (int m = 0; m < 5; ++m) q(i, j, k, m) = qq[m];
    };
    auto cp = [&](int i, int j, int k, int si, int sj, int sk) {
      rho(i, j, k) = rho(si, sj, sk);
      for (int c = 0; c < 3; ++c) vel(i, j, k, c) = vel(si, sj, sk, c);
      tmp(i, j, k) = tmp(si, sj, sk);
      prs(i, j, k) = prs(si, sj, sk);
      setq(i, j, k);
    };
#pragma omp parallel for collapse(2)
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j) {
        for (int i = -HM; i <= -1; ++i) cp(i, j, k, im + i, j, k);
        for (int i = im + 1; i <= im + HM; ++i) cp(i, j, k, i - im, j, k);
      }
#pragma omp parallel for collapse(2)
    for (int k = 0; k <= km; ++k)
      for (int i = 0; i <= im; ++i) {
        for (int j = -HM; j <= -1; ++j) cp(i, j, k, i, jm + j, k);
        for (int j = jm + 1; j <= jm + HM; ++j) cp(i, j, k, i, j - jm, k);
      }
#pragma omp parallel for collapse(2)
    for (int j = 0; j <= jm; ++j)
      for (int i = 0; i <= im; ++i) {
        for (int k = -HM; k <= -1; ++k) cp(i, j, k, i, j, km + k);
        for (int k = km + 1; k <= km + HM; ++k) cp(i, j, k, i, j, k - km);
      }
  }

  // bchomovec, tgvsolver.F90:371-440 (ndir: 0 = all, 1..3 one direction)
  void bchomovec(Field3& var, int ncomp, int ndir) {
    if (ndir == 1 || ndir == 0) {
#pragma omp parallel for collapse(2)
      for (int k = 0; k <= km; ++k)
        for (int j = 0; j <= jm; ++j)
          for (int m = 0; m < ncomp; ++m) {
            for (int i = -HM; i <= -1; ++i) var(i, j, k, m) = var(im + i, j, k, m);
            for (int i = im + 1; i <= im + HM; ++i) var(i, j, k, m) = var(i - im, j, k, m);
          }
    }
    if (ndir == 2 || ndir == 0) {
#pragma omp parallel for collapse(2)
      for (int k = 0; k <= km; ++k)
        for (int i = 0; i <= im; ++i)
          for (int m = 0; m < ncomp; ++m) {
            for (int j = -HM; j <= -1; ++j) var(i, j, k, m) = var(i, jm + j, k, m);
            for (int j = jm + 1; j <= jm + HM; ++j) var(i, j, k, m) = var(i, j - jm, k, m);
          }
    }
    if (ndir == 3 || ndir == 0) {
#pragma omp parallel for collapse(2)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i)
          for (int m = 0; m < ncomp; ++m) {
            for (int k = -HM; k <= -1; ++k) var(i, j, k, m) = var(i, j, km + k, m);
            for (int k = km + 1; k <= km + HM; ++k) var(i, j, k, m) = var(i, j, k - km, m);
          }
    }
  }

  // Generic line loop: for each line along dir, gather ncolm inputs f(-HM..dim+HM) via `gather`,
  // take the compact derivative, hand the result to `scatter`.
  template <class Gather, class Scatter>
  void line_loop(int dir, int ncolm, Gather gather, Scatter scatter) {
    const int dims[3] = {im, jm, km};
    const int dim = dims[dir];
    const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
#pragma omp parallel
    {
      std::vector<double> ff((size_t)ncolm * (dim + 1 + 2 * HM)), df((size_t)ncolm * (dim + 1)),
          scr(2 * (dim + 8));
#pragma omp for collapse(2) schedule(static)
      for (int b = 0; b <= dims[o2]; ++b)
        for (int a = 0; a <= dims[o1]; ++a) {
          int ijk[3];
          ijk[o1] = a; ijk[o2] = b; ijk[dir] = 0;
          for (int n = 0; n < ncolm; ++n) {
            double* fn = ff.data() + (size_t)n * (dim + 1 + 2 * HM) + HM;
            for (int t = -HM; t <= dim + HM; ++t) {
              int p[3] = {ijk[0], ijk[1], ijk[2]};
              p[dir] = t;
              fn[t] = gather(n, p[0], p[1], p[2]);
            }
          }
          for (int n = 0; n < ncolm; ++n)
            df_line(fds[dir], ff.data() + (size_t)n * (dim + 1 + 2 * HM) + HM, df.data() + (size_t)n * (dim + 1), scr.data());
          for (int t = 0; t <= dim; ++t) {
            int p[3] = {ijk[0], ijk[1], ijk[2]};
            p[dir] = t;
            for (int n = 0; n < ncolm; ++n) scatter(n, p[0], p[1], p[2], df[(size_t)n * (dim + 1) + t]);
          }
        }
    }
  }

  double dstep(int dir) const { return dir == 0 ? dx : (dir == 1 ? dy : dz); }

  // gradcal, tgvsolver.F90:450-537
  void gradcal() {
    for (int dir = 0; dir < 3; ++dir) {
      const double h = dstep(dir);
      line_loop(dir, 4,
                [&](int n, int i, int j, int k) { return n < 3 ? vel(i, j, k, n) : tmp(i, j, k); },
                [&](int n, int i, int j, int k, double v) {
                  if (n < 3) dvel(i, j, k, n + 3 * dir) = v / h;  // dvel(:,:,:,n,dir)
                  else dtmp(i, j, k, dir) = v / h;
                });
    }
  }

  // convection, tgvsolver.F90:539-633
  void convection() {
    for (int dir = 0; dir < 3; ++dir) {
      const double h = dstep(dir);
      line_loop(dir, 5,
                [&](int n, int i, int j, int k) {
                  double uu = vel(i, j, k, dir);
                  if (n == 4) return (q(i, j, k, 4) + prs(i, j, k)) * uu;
                  if (n == dir + 1) return q(i, j, k, n) * uu + prs(i, j, k);
                  return q(i, j, k, n) * uu;
                },
                [&](int n, int i, int j, int k, double v) { qrhs(i, j, k, n) = qrhs(i, j, k, n) + v / h; });
    }
  }

  // diffusion, tgvsolver.F90:635-789
  void diffusion() {
#pragma omp parallel for collapse(2)
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          double s11 = dvel(i, j, k, 0);
          double s12 = 0.5 * (dvel(i, j, k, 3) + dvel(i, j, k, 1));
          double s13 = 0.5 * (dvel(i, j, k, 6) + dvel(i, j, k, 2));
          double s22 = dvel(i, j, k, 4);
          double s23 = 0.5 * (dvel(i, j, k, 7) + dvel(i, j, k, 5));
          double s33 = dvel(i, j, k, 8);
          double skk = num1d3 * (s11 + s22 + s33);
          double miu = miucal(tmp(i, j, k)) / reynolds;
          double miu2 = 2.0 * miu;
          double hcc = (miu / prandtl) / const5;
          sigma(i, j, k, 0) = miu2 * (s11 - skk);
          sigma(i, j, k, 1) = miu2 * s12;
          sigma(i, j, k, 2) = miu2 * s13;
          sigma(i, j, k, 3) = miu2 * (s22 - skk);
          sigma(i, j, k, 4) = miu2 * s23;
          sigma(i, j, k, 5) = miu2 * (s33 - skk);
          qflux(i, j, k, 0) = hcc * dtmp(i, j, k, 0) + sigma(i, j, k, 0) * vel(i, j, k, 0) +
                              sigma(i, j, k, 1) * vel(i, j, k, 1) + sigma(i, j, k, 2) * vel(i, j, k, 2);
          qflux(i, j, k, 1) = hcc * dtmp(i, j, k, 1) + sigma(i, j, k, 1) * vel(i, j, k, 0) +
                              sigma(i, j, k, 3) * vel(i, j, k, 1) + sigma(i, j, k, 4) * vel(i, j, k, 2);
          qflux(i, j, k, 2) = hcc * dtmp(i, j, k, 2) + sigma(i, j, k, 2) * vel(i, j, k, 0) +
                              sigma(i, j, k, 4) * vel(i, j, k, 1) + sigma(i, j, k, 5) * vel(i, j, k, 2);
        }
    bchomovec(sigma, 6, 0);
    bchomovec(qflux, 3, 0);
    // (sigma component, qflux component) per direction: x: s1 s2 s3 q1; y: s2 s4 s5 q2; z: s3 s5 s6 q3
    static const int sg[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (int dir = 0; dir < 3; ++dir) {
      const double h = dstep(dir);
      line_loop(dir, 4,
                [&](int n, int i, int j, int k) { return n < 3 ? sigma(i, j, k, sg[dir][n]) : qflux(i, j, k, dir); },
                [&](int n, int i, int j, int k, double v) { qrhs(i, j, k, n + 1) = qrhs(i, j, k, n + 1) + v / h; });
    }
  }

  // filterq, tgvsolver.F90:791-883
  void filterq() {
    const int dims[3] = {im, jm, km};
    for (int dir = 0; dir < 3; ++dir) {
      if (periodic(dir)) bchomovec(q, 5, dir + 1);
      const int dim = dims[dir];
      const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
#pragma omp parallel
      {
        std::vector<double> phi(dim + 1 + 2 * HM), fph((size_t)5 * (dim + 1)), scr(2 * (dim + 8));
#pragma omp for collapse(2) schedule(static)
        for (int b = 0; b <= dims[o2]; ++b)
          for (int a = 0; a <= dims[o1]; ++a) {
            int ijk[3];
            ijk[o1] = a; ijk[o2] = b; ijk[dir] = 0;
            for (int n = 0; n < 5; ++n) {
              for (int t = -HM; t <= dim + HM; ++t) {
                int p[3] = {ijk[0], ijk[1], ijk[2]};
                p[dir] = t;
                phi[t + HM] = q(p[0], p[1], p[2], n);
              }
              filter_line(flt[dir], phi.data() + HM, fph.data() + (size_t)n * (dim + 1), scr.data());
            }
            for (int t = 0; t <= dim; ++t) {
              int p[3] = {ijk[0], ijk[1], ijk[2]};
              p[dir] = t;
              for (int n = 0; n < 5; ++n) q(p[0], p[1], p[2], n) = fph[(size_t)n * (dim + 1) + t];
            }
          }
      }
    }
  }

  // Neumaier's compensated summation: s + c carries the sum of the added terms to about one
  // rounding of the final value, independent of their number and order.
  struct CSum {
    double s = 0.0, c = 0.0;
    void add(double x) {
      const double t = s + x;
      c += (std::fabs(s) >= std::fabs(x)) ? (s - t) + x : (x - t) + s;
      s = t;
    }
    double value() const { return s + c; }
  };

  // stacal, tgvsolver.F90:893-942, plus diss_rate_cal (statistic.F90:993-1040); sequential sums
  // in the reference's order. The same per-node terms are also summed with compensation (hist_c),
  // a reference value for the sums whose rounding does not grow with the number of nodes: a
  // sequential sum of N terms carries an error of order sqrt(N) ulps (about 1e-12 relative at
  // 512^3), which an implementation that sums in another order cannot reproduce.
  void stacal() {
    double tke = 0.0, enst = 0.0, diss = 0.0;
    CSum ctke, censt, cdiss;
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          double var1 = vel(i, j, k, 0) * vel(i, j, k, 0) + vel(i, j, k, 1) * vel(i, j, k, 1) +
                        vel(i, j, k, 2) * vel(i, j, k, 2);
          tke = tke + rho(i, j, k) * var1;
          ctke.add(rho(i, j, k) * var1);
          double om1 = dvel(i, j, k, 2 + 3) - dvel(i, j, k, 1 + 6);
          double om2 = dvel(i, j, k, 0 + 6) - dvel(i, j, k, 2 + 0);
          double om3 = dvel(i, j, k, 1 + 0) - dvel(i, j, k, 0 + 3);
          enst = enst + rho(i, j, k) * (om1 * om1 + om2 * om2 + om3 * om3);
          censt.add(rho(i, j, k) * (om1 * om1 + om2 * om2 + om3 * om3));
          double miu = miucal(tmp(i, j, k)) / reynolds;
          double du11 = dvel(i, j, k, 0), du12 = dvel(i, j, k, 3), du13 = dvel(i, j, k, 6);
          double du21 = dvel(i, j, k, 1), du22 = dvel(i, j, k, 4), du23 = dvel(i, j, k, 7);
          double du31 = dvel(i, j, k, 2), du32 = dvel(i, j, k, 5), du33 = dvel(i, j, k, 8);
          double s11 = du11, s12 = 0.5 * (du12 + du21), s13 = 0.5 * (du13 + du31);
          double s22 = du22, s23 = 0.5 * (du23 + du32), s33 = du33;
          double div = s11 + s22 + s33;
          double v = 2.0 * miu * (s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23) -
                                  num1d3 * (div * div));
          diss = diss + v;
          cdiss.add(v);
        }
    const double nn = double((int64_t)im * jm * km);
    tke = 0.5 * tke / nn;
    enst = 0.5 * enst / nn;
    diss = diss / nn;
    hist.push_back(nstep); hist.push_back(time); hist.push_back(tke); hist.push_back(enst); hist.push_back(diss);
    hist_c.push_back(nstep); hist_c.push_back(time); hist_c.push_back(0.5 * ctke.value() / nn);
    hist_c.push_back(0.5 * censt.value() / nn); hist_c.push_back(cdiss.value() / nn);
  }

  // rhscal, tgvsolver.F90:962-992
  void rhscal() {
    std::fill(qrhs.v.begin(), qrhs.v.end(), 0.0);
    gradcal();
    convection();
    for (double& v : qrhs.v) v = -v;
    diffusion();
  }

  // readcheckpoint + updateq (src/readwrite.F90:1378-1528, src/fludyna.F90:254-300): the
  // primitive arrays take the file's ro, u1, u2, u3, p, t on nodes 0..N (6 Fortran fields) and q
  // is fvar2q's temperature branch (src/fludyna.F90:449-533):
  // q5 = rho (t const1 + 0.5 (u1^2 + u2^2 + u3^2)).
  void set_flowfield(const double* f) {
    const int64_t n0 = im + 1, n1 = jm + 1, n2 = km + 1, nn = n0 * n1 * n2;
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          const int64_t o = ((int64_t)k * n1 + j) * n0 + i;
          const double r = f[o], u[3] = {f[nn + o], f[2 * nn + o], f[3 * nn + o]};
          rho(i, j, k) = r;
          for (int c = 0; c < 3; ++c) vel(i, j, k, c) = u[c];
          prs(i, j, k) = f[4 * nn + o];
          tmp(i, j, k) = f[5 * nn + o];
          q(i, j, k, 0) = r;
          for (int c = 0; c < 3; ++c) q(i, j, k, 1 + c) = r * u[c];
          q(i, j, k, 4) = r * (tmp(i, j, k) * const1 + 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
        }
  }
  // The primitive arrays on nodes 0..N as writeflfed writes them (ro, u1, u2, u3, p, t).
  void get_flowfield(double* f) {
    const int64_t n0 = im + 1, n1 = jm + 1, n2 = km + 1, nn = n0 * n1 * n2;
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          const int64_t o = ((int64_t)k * n1 + j) * n0 + i;
          f[o] = rho(i, j, k);
          for (int c = 0; c < 3; ++c) f[(1 + c) * nn + o] = vel(i, j, k, c);
          f[4 * nn + o] = prs(i, j, k);
          f[5 * nn + o] = tmp(i, j, k);
        }
  }

  void update_prims() {
#pragma omp parallel for collapse(2)
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          double qq[5] = {q(i, j, k, 0), q(i, j, k, 1), q(i, j, k, 2), q(i, j, k, 3), q(i, j, k, 4)};
          double u[3], r, p, t;
          q2fvar(qq, r, u, p, t);
          rho(i, j, k) = r; prs(i, j, k) = p; tmp(i, j, k) = t;
          for (int c = 0; c < 3; ++c) vel(i, j, k, c) = u[c];
        }
  }

  // ---------------------------------------------------------------- full-solver mode
  // The stage of the full solver's time_integration_rk (src/mainloop.F90:392-476) on a periodic
  // box of one rank with a uniform Cartesian grid: filterq first (src/comsolver.F90:514-632), then
  // qswap (src/parallel.F90:4877-5060: per direction the periodic halo copy of q, the average of
  // nodes 0 and N, and q2fvar on the planes -hm..0 and N..N+hm only), rhscal (src/solver.F90:
  // 184-283) in its metric form -- gradcal (src/comsolver.F90:244-497) multiplies by dxi,
  // convrsdcal6 (src/solver.F90:2174-2342) and diffrsdcal6 (src/solver.F90:2355-2874) carry the
  // Jacobian -- then the update of q*jacob (src/mainloop.F90:438-446) and updatefvar
  // (src/fludyna.F90:191-242). The primitive variables of the interior nodes used by rhscal are
  // those of the last updatefvar, i.e. of the unfiltered state: qswap recomputes them only on the
  // boundary planes and halos. The metrics of a uniform grid are taken in closed form: dxi =
  // diag(1/dx, 1/dy, 1/dz), jacob = dx*dy*dz (src/geom.F90:350-385 computes them numerically from
  // the grid; for a uniform grid those equal these to rounding). The off-diagonal metric terms
  // are zero and add exactly zero, so they are left out.
  double jac() const { return dx * dy * dz; }

  // qswap on one rank with every direction periodic (parallel.F90:4877-5060)
  void fs_qswap() {
    const int dims[3] = {im, jm, km};
    for (int dir = 0; dir < 3; ++dir) {
      if (!periodic(dir)) continue;   // one rank, non-periodic: nothing to exchange
      bchomovec(q, 5, dir + 1);
      const int dim = dims[dir];
      const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
#pragma omp parallel for collapse(2)
      for (int b = 0; b <= dims[o2]; ++b)
        for (int a = 0; a <= dims[o1]; ++a) {
          int p0[3], pn[3];
          p0[o1] = pn[o1] = a; p0[o2] = pn[o2] = b; p0[dir] = 0; pn[dir] = dim;
          for (int m = 0; m < 5; ++m) {
            q(p0[0], p0[1], p0[2], m) = 0.5 * (q(p0[0], p0[1], p0[2], m) + q(pn[0], pn[1], pn[2], m));
            q(pn[0], pn[1], pn[2], m) = q(p0[0], p0[1], p0[2], m);
          }
          // q2fvar on the planes -hm..0 and dim..dim+hm of this line
          for (int t = -HM; t <= dim + HM; ++t) {
            if (t > 0 && t < dim) continue;
            int p[3] = {p0[0], p0[1], p0[2]};
            p[dir] = t;
            double qq[5], u[3], r, pr, tt;
            for (int m = 0; m < 5; ++m) qq[m] = q(p[0], p[1], p[2], m);
            q2fvar(qq, r, u, pr, tt);
            rho(p[0], p[1], p[2]) = r; prs(p[0], p[1], p[2]) = pr; tmp(p[0], p[1], p[2]) = tt;
            for (int c = 0; c < 3; ++c) vel(p[0], p[1], p[2], c) = u[c];
          }
        }
    }
  }

  // gradcal in the metric form: dvel(:,:,:,n,d) = df * dxi(d,d)
  void fs_gradcal() {
    for (int dir = 0; dir < 3; ++dir) {
      const double dxi = 1.0 / dstep(dir);
      line_loop(dir, 4,
                [&](int n, int i, int j, int k) { return n < 3 ? vel(i, j, k, n) : tmp(i, j, k); },
                [&](int n, int i, int j, int k, double v) {
                  if (n < 3) dvel(i, j, k, n + 3 * dir) = v * dxi;
                  else dtmp(i, j, k, dir) = v * dxi;
                });
    }
  }

  // convrsdcal6: fcs = jacob * (q uu + dxi p e_d), uu = dxi(d,d) u_d; qrhs += D(fcs)
  void fs_convection() {
    const double jb = jac();
    for (int dir = 0; dir < 3; ++dir) {
      const double dxi = 1.0 / dstep(dir);
      line_loop(dir, 5,
                [&](int n, int i, int j, int k) {
                  const double uu = dxi * vel(i, j, k, dir);
                  if (n == 0) return jb * q(i, j, k, 0) * uu;
                  if (n == 4) return jb * (q(i, j, k, 4) + prs(i, j, k)) * uu;
                  if (n == dir + 1) return jb * (q(i, j, k, n) * uu + dxi * prs(i, j, k));
                  return jb * (q(i, j, k, n) * uu);
                },
                [&](int n, int i, int j, int k, double v) { qrhs(i, j, k, n) = qrhs(i, j, k, n) + v; });
    }
  }

  // diffrsdcal6: sigma and qflux as in the miniapp, then ff = (sigma . dxi(d,:)) * jacob
  void fs_diffusion() {
#pragma omp parallel for collapse(2)
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          double s11 = dvel(i, j, k, 0);
          double s12 = 0.5 * (dvel(i, j, k, 3) + dvel(i, j, k, 1));
          double s13 = 0.5 * (dvel(i, j, k, 6) + dvel(i, j, k, 2));
          double s22 = dvel(i, j, k, 4);
          double s23 = 0.5 * (dvel(i, j, k, 7) + dvel(i, j, k, 5));
          double s33 = dvel(i, j, k, 8);
          double skk = num1d3 * (s11 + s22 + s33);
          double miu = miucal(tmp(i, j, k)) / reynolds;
          double miu2 = 2.0 * miu;
          double hcc = (miu / prandtl) / const5;
          sigma(i, j, k, 0) = miu2 * (s11 - skk);
          sigma(i, j, k, 1) = miu2 * s12;
          sigma(i, j, k, 2) = miu2 * s13;
          sigma(i, j, k, 3) = miu2 * (s22 - skk);
          sigma(i, j, k, 4) = miu2 * s23;
          sigma(i, j, k, 5) = miu2 * (s33 - skk);
          qflux(i, j, k, 0) = hcc * dtmp(i, j, k, 0) + sigma(i, j, k, 0) * vel(i, j, k, 0) +
                              sigma(i, j, k, 1) * vel(i, j, k, 1) + sigma(i, j, k, 2) * vel(i, j, k, 2);
          qflux(i, j, k, 1) = hcc * dtmp(i, j, k, 1) + sigma(i, j, k, 1) * vel(i, j, k, 0) +
                              sigma(i, j, k, 3) * vel(i, j, k, 1) + sigma(i, j, k, 4) * vel(i, j, k, 2);
          qflux(i, j, k, 2) = hcc * dtmp(i, j, k, 2) + sigma(i, j, k, 2) * vel(i, j, k, 0) +
                              sigma(i, j, k, 4) * vel(i, j, k, 1) + sigma(i, j, k, 5) * vel(i, j, k, 2);
        }
    for (int d = 0; d < 3; ++d)
      if (periodic(d)) {
        bchomovec(sigma, 6, d + 1);
        bchomovec(qflux, 3, d + 1);
      }
    static const int sg[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    const double jb = jac();
    for (int dir = 0; dir < 3; ++dir) {
      const double dxi = 1.0 / dstep(dir);
      line_loop(dir, 4,
                [&](int n, int i, int j, int k) {
                  return (n < 3 ? sigma(i, j, k, sg[dir][n]) : qflux(i, j, k, dir)) * dxi * jb;
                },
                [&](int n, int i, int j, int k, double v) { qrhs(i, j, k, n + 1) = qrhs(i, j, k, n + 1) + v; });
    }
  }

  // ---- upwind compact convection: convrsdcmp (src/solver.F90:1272-1938) with lchardecomp off.
  // Without the characteristic decomposition no Ducros sensor runs, so lshock stays unallocated
  // (shock = .true. at every interface, solver.F90:1440-1455); crinod is .false. everywhere
  // (mainloop.F90:80), so every interface goes through the MP limiter.

  // flux_steger_warming of one node (riemann.F90:23-161, the non-reacting branch) with the metric
  // row m = dxi(dir, :) and sos = sqrt(T)/M (fludyna.F90:832-859, nondimensional).
  void sw_split(double r, const double* u, double p, double t, const double* qq, const double* m, double jb,
                double* fp, double* fm) const {
    const double eps = 0.04;
    const double uu = m[0] * u[0] + m[1] * u[1] + m[2] * u[2];
    const double var0 = 1.0 / std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const double gpd[3] = {m[0] * var0, m[1] * var0, m[2] * var0};
    const double gm2 = 0.5 / gamma;
    const double css = std::sqrt(t) / mach;
    const double csa = css / var0;
    const double lmach = uu / csa;
    const double lmda[5] = {uu, uu, uu, uu + csa, uu - csa};
    double lp[5], lm[5];
    for (int k = 0; k < 5; ++k) {
      lp[k] = 0.5 * (lmda[k] + std::sqrt(lmda[k] * lmda[k] + eps * eps));
      lm[k] = lmda[k] - lp[k];
    }
    if (lmach >= 1.0 || lmach <= -1.0) {
      double* f = lmach >= 1.0 ? fp : fm;
      double* z = lmach >= 1.0 ? fm : fp;
      f[0] = jb * qq[0] * uu;
      f[1] = jb * (qq[1] * uu + m[0] * p);
      f[2] = jb * (qq[2] * uu + m[1] * p);
      f[3] = jb * (qq[3] * uu + m[2] * p);
      f[4] = jb * (qq[4] + p) * uu;
      for (int k = 0; k < 5; ++k) z[k] = 0.0;
      return;
    }
    const double fhi = 0.5 * (gamma - 1.0) * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double jro = jb * r;
    for (int side = 0; side < 2; ++side) {
      const double* l = side == 0 ? lp : lm;
      double* f = side == 0 ? fp : fm;
      const double var1 = l[0];
      const double var2 = l[3] - l[4];
      const double var3 = 2.0 * l[0] - l[3] - l[4];
      const double var4 = var1 - var3 * gm2;
      f[0] = jro * var4;
      f[1] = jro * (var4 * u[0] + var2 * css * gpd[0] * gm2);
      f[2] = jro * (var4 * u[1] + var2 * css * gpd[1] * gm2);
      f[3] = jro * (var4 * u[2] + var2 * css * gpd[2] * gm2);
      f[4] = jb * (var1 * qq[4] + r * (var2 * uu * var0 * css * gm2 - var3 * (fhi + css * css) * gm2 / (gamma - 1.0)));
    }
  }

  static double minmod2(double a, double b) {   // commfunc.F90:699-714
    if (a > 0.0 && b > 0.0) return std::min(std::fabs(a), std::fabs(b));
    if (a < 0.0 && b < 0.0) return -1.0 * std::min(std::fabs(a), std::fabs(b));
    return 0.0;
  }
  static double minmod4(double a, double b, double c, double d) {   // commfunc.F90:722-738
    if (a > 0.0 && b > 0.0 && c > 0.0 && d > 0.0)
      return std::min(std::min(std::min(std::fabs(a), std::fabs(b)), std::fabs(c)), std::fabs(d));
    if (a < 0.0 && b < 0.0 && c < 0.0 && d < 0.0)
      return -1.0 * std::min(std::min(std::min(std::fabs(a), std::fabs(b)), std::fabs(c)), std::fabs(d));
    return 0.0;
  }
  // MP5 with the compact value as the linear value (flux.F90:434-496); no limiting unless
  // discont (the shock flag) is set
  static double mp5(const double* u, double ul, bool discont) {
    double var1 = u[3] - u[2];
    double var2 = 4.0 * (u[2] - u[1]);
    const double ump = u[2] + minmod2(var1, var2);
    var1 = (ul - u[2]) * (ul - ump);
    if (!(discont && var1 >= 1.0e-10)) return ul;
    const double dm1 = u[0] - 2.0 * u[1] + u[2];
    const double d0 = u[1] - 2.0 * u[2] + u[3];
    const double d1 = u[2] - 2.0 * u[3] + u[4];
    const double dhm1 = minmod4(4.0 * dm1 - d0, 4.0 * d0 - dm1, dm1, d0);
    const double dh0 = minmod4(4.0 * d0 - d1, 4.0 * d1 - d0, d0, d1);
    const double uul = u[2] + 4.0 * (u[2] - u[1]);
    const double uav = 0.5 * (u[2] + u[3]);
    const double umd = uav - 0.5 * dh0;
    const double ulc = u[2] + 0.5 * (u[2] - u[1]) + 1.333333333333333 * dhm1;
    const double umin = std::max(std::min(std::min(u[2], u[3]), umd), std::min(std::min(u[2], uul), ulc));
    const double umax = std::min(std::max(std::max(u[2], u[3]), umd), std::max(std::max(u[2], uul), ulc));
    return ul + minmod2(umin - ul, umax - ul);
  }
  // mplimiter, flux.F90:363-379: the compact value itself at the two interfaces next to a block's
  // physical end (ntype 1 or 2 only), MP5 elsewhere
  static double mplimiter(const double* f, double fl, bool shock, int inode, int dim, int nt) {
    if ((nt == 1 && inode == 0) || (nt == 2 && inode == dim - 1) || (nt == 1 && inode == 1) ||
        (nt == 2 && inode == dim - 2))
      return fl;
    return mp5(f, fl, shock);
  }

  // chardecomp (solver.F90:1959-2163, non-reacting): Roe-averaged right and left eigenvectors of
  // the interface between two nodes for the metric direction ddi (the same at both nodes here).
  void chardecomp(double tl, double rl, double pl, double el, const double* vl, double tr, double rr, double pr,
                  double er, const double* vr, const double* ddi, double (&REV)[5][5], double (&LEV)[5][5]) const {
    (void)tl; (void)tr;
    const double rero = 1.0e-12;
    const double wroe = std::sqrt(rl) / (std::sqrt(rl) + std::sqrt(rr));
    const double wroe1 = 1.0 - wroe;
    const double u1 = wroe * vl[0] + wroe1 * vr[0];
    const double u2 = wroe * vl[1] + wroe1 * vr[1];
    const double u3 = wroe * vl[2] + wroe1 * vr[2];
    const double kroe = 0.5 * (u1 * u1 + u2 * u2 + u3 * u3);
    const double hl = (el + pl) / rl;
    const double hr = (er + pr) / rr;
    const double hroe = wroe * hl + wroe1 * hr;
    const double css = std::sqrt((gamma - 1.0) * (hroe - kroe));
    const double rcs = 1.0 / css;
    const double var1 = 0.5 * (ddi[0] + ddi[0]);
    const double var2 = 0.5 * (ddi[1] + ddi[1]);
    const double var3 = 0.5 * (ddi[2] + ddi[2]);
    const double var4 = 1.0 / std::sqrt(var1 * var1 + var2 * var2 + var3 * var3);
    const double g1 = var1 * var4, g2 = var2 * var4, g3 = var3 * var4;
    const double ugp = u1 * g1 + u2 * g2 + u3 * g3;
    const double b1 = (gamma - 1.0) / (css * css);
    const double b2 = 1.0 + 2.0 * b1 * kroe - b1 * hroe;
    LEV[0][0] = 0.5 * (b2 + ugp * rcs);
    LEV[0][1] = -0.5 * (b1 * u1 + g1 * rcs);
    LEV[0][2] = -0.5 * (b1 * u2 + g2 * rcs);
    LEV[0][3] = -0.5 * (b1 * u3 + g3 * rcs);
    LEV[0][4] = 0.5 * b1;
    REV[0][0] = 1.0;
    REV[1][0] = u1 - css * g1;
    REV[2][0] = u2 - css * g2;
    REV[3][0] = u3 - css * g3;
    REV[4][0] = hroe - ugp * css;
    LEV[1][0] = 1.0 - b2;
    LEV[1][1] = b1 * u1;
    LEV[1][2] = b1 * u2;
    LEV[1][3] = b1 * u3;
    LEV[1][4] = -b1;
    REV[0][1] = 1.0;
    REV[1][1] = u1;
    REV[2][1] = u2;
    REV[3][1] = u3;
    REV[4][1] = hroe - 1.0 / b1;
    if (std::fabs(var1) > rero) {
      const double rgp = 1.0 / g1;
      LEV[2][0] = (ugp * g2 - u2) * rgp; LEV[2][1] = -g2; LEV[2][2] = (1.0 - g2 * g2) * rgp;
      LEV[2][3] = -g2 * g3 * rgp; LEV[2][4] = 0.0;
      LEV[3][0] = (ugp * g3 - u3) * rgp; LEV[3][1] = -g3; LEV[3][2] = -g2 * g3 * rgp;
      LEV[3][3] = (1.0 - g3 * g3) * rgp; LEV[3][4] = 0.0;
      REV[0][2] = 0.0; REV[1][2] = -g2; REV[2][2] = g1; REV[3][2] = 0.0; REV[4][2] = u2 * g1 - u1 * g2;
      REV[0][3] = 0.0; REV[1][3] = -g3; REV[2][3] = 0.0; REV[3][3] = g1; REV[4][3] = u3 * g1 - u1 * g3;
    } else if (std::fabs(var2) > rero) {
      const double rgp = 1.0 / g2;
      LEV[2][0] = (ugp * g1 - u1) * rgp; LEV[2][1] = (1.0 - g1 * g1) * rgp; LEV[2][2] = -g1;
      LEV[2][3] = -g1 * g3 * rgp; LEV[2][4] = 0.0;
      LEV[3][0] = (ugp * g3 - u3) * rgp; LEV[3][1] = -g1 * g3 * rgp; LEV[3][2] = -g3;
      LEV[3][3] = (1.0 - g3 * g3) * rgp; LEV[3][4] = 0.0;
      REV[0][2] = 0.0; REV[1][2] = g2; REV[2][2] = -g1; REV[3][2] = 0.0; REV[4][2] = u1 * g2 - u2 * g1;
      REV[0][3] = 0.0; REV[1][3] = 0.0; REV[2][3] = -g3; REV[3][3] = g2; REV[4][3] = u3 * g2 - u2 * g3;
    } else {
      const double rgp = 1.0 / g3;
      LEV[2][0] = (ugp * g1 - u1) * rgp; LEV[2][1] = (1.0 - g1 * g1) * rgp; LEV[2][2] = -g1 * g2 * rgp;
      LEV[2][3] = -g1; LEV[2][4] = 0.0;
      LEV[3][0] = (ugp * g2 - u2) * rgp; LEV[3][1] = -g1 * g2 * rgp; LEV[3][2] = (1.0 - g2 * g2) * rgp;
      LEV[3][3] = -g2; LEV[3][4] = 0.0;
      REV[0][2] = 0.0; REV[1][2] = g3; REV[2][2] = 0.0; REV[3][2] = -g1; REV[4][2] = u1 * g3 - u3 * g1;
      REV[0][3] = 0.0; REV[1][3] = 0.0; REV[2][3] = g3; REV[3][3] = -g2; REV[4][3] = u2 * g3 - u3 * g2;
    }
    LEV[4][0] = 0.5 * (b2 - ugp * rcs);
    LEV[4][1] = -0.5 * (b1 * u1 - g1 * rcs);
    LEV[4][2] = -0.5 * (b1 * u2 - g2 * rcs);
    LEV[4][3] = -0.5 * (b1 * u3 - g3 * rcs);
    LEV[4][4] = 0.5 * b1;
    REV[0][4] = 1.0;
    REV[1][4] = u1 + css * g1;
    REV[2][4] = u2 + css * g2;
    REV[3][4] = u3 + css * g3;
    REV[4][4] = hroe + ugp * css;
  }

  // ducrossensor (commcal.F90:196-353): ssf = div^2/(div^2 + |omega|^2 + 1e-30) times the largest
  // normalised second difference of p, the periodic halo swap of ssf, then lshock = the maximum
  // of ssf over the 10-node stencils i-4..i+5 along each axis exceeds shkcrt. Neighbours are
  // clamped at physical ends only for ntype 1 (low) and 2 (high), as the reference does.
  void ducros_sensor() {
    const int dims[3] = {im, jm, km};
#pragma omp parallel for collapse(2)
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          const double div = dvel(i, j, k, 0) + dvel(i, j, k, 4) + dvel(i, j, k, 8);
          const double div2 = div * div;
          // dvel(i,j,k,n,d) is field n + 3 d here
          const double vx = dvel(i, j, k, 2 + 3) - dvel(i, j, k, 1 + 6);
          const double vy = dvel(i, j, k, 0 + 6) - dvel(i, j, k, 2 + 0);
          const double vz = dvel(i, j, k, 1 + 0) - dvel(i, j, k, 0 + 3);
          const double vort = vx * vx + vy * vy + vz * vz;
          int ip = i + 1, imn = i - 1, jp = j + 1, jmn = j - 1, kp = k + 1, kmn = k - 1;
          if (ntype[0] == 1 && imn < 0) imn = 0;
          if (ntype[1] == 1 && jmn < 0) jmn = 0;
          if (ntype[2] == 1 && kmn < 0) kmn = 0;
          if (ntype[0] == 2 && ip > im) ip = im;
          if (ntype[1] == 2 && jp > jm) jp = jm;
          if (ntype[2] == 2 && kp > km) kp = km;
          const double p0 = prs(i, j, k);
          const double di = std::fabs(prs(ip, j, k) - 2.0 * p0 + prs(imn, j, k)) / (prs(ip, j, k) + 2.0 * p0 + prs(imn, j, k));
          const double dj = std::fabs(prs(i, jp, k) - 2.0 * p0 + prs(i, jmn, k)) / (prs(i, jp, k) + 2.0 * p0 + prs(i, jmn, k));
          const double dk = std::fabs(prs(i, j, kp) - 2.0 * p0 + prs(i, j, kmn)) / (prs(i, j, kp) + 2.0 * p0 + prs(i, j, kmn));
          ssf(i, j, k) = div2 / (div2 + vort + 1.0e-30) * std::max(std::max(di, dj), dk);
        }
    for (int d = 0; d < 3; ++d)
      if (periodic(d)) bchomovec(ssf, 1, d + 1);
#pragma omp parallel for collapse(2)
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          double mx = 0.0;
          for (int o = -HM + 1; o <= HM; ++o) {
            int ii = i + o;
            if (ntype[0] == 1 && ii < 0) ii = 0;
            if (ntype[0] == 2 && ii > im) ii = im;
            mx = std::max(mx, ssf(ii, j, k));
          }
          for (int o = -HM + 1; o <= HM; ++o) {
            int jj = j + o;
            if (ntype[1] == 1 && jj < 0) jj = 0;
            if (ntype[1] == 2 && jj > jm) jj = jm;
            mx = std::max(mx, ssf(i, jj, k));
          }
          for (int o = -HM + 1; o <= HM; ++o) {
            int kk = k + o;
            if (ntype[2] == 1 && kk < 0) kk = 0;
            if (ntype[2] == 2 && kk > km) kk = km;
            mx = std::max(mx, ssf(i, j, kk));
          }
          lshock[((size_t)k * (jm + 1) + j) * (im + 1) + i] = mx > shkcrt;
        }
    (void)dims;
  }
  bool shock_at(int i, int j, int k) const { return lshock[((size_t)k * (jm + 1) + j) * (im + 1) + i] != 0; }

  void build_flux_schemes() {
    const int dims[3] = {im, jm, km};
    for (int d = 0; d < 3; ++d) {
      fuw[d] = Scheme();
      fdw[d] = Scheme();
      if (conschm != 543) continue;
      compact_flux_initiate(fuw[d], 543, ntype[d], dims[d], 1, bfacmpld);
      compact_flux_initiate(fdw[d], 543, ntype[d], dims[d], -1, bfacmpld);
    }
  }

  void fs_convection_upwind() {
    const int dims[3] = {im, jm, km};
    const double jb = jac();
    for (int dir = 0; dir < 3; ++dir) {
      const int dim = dims[dir], nt = ntype[dir];
      const int iss = (nt == 1 || nt == 4) ? 0 : -HM;
      const int iee = (nt == 2 || nt == 4) ? dim : dim + HM;
      double mrow[3] = {0.0, 0.0, 0.0};
      mrow[dir] = 1.0 / dstep(dir);
      const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
      const int L = dim + 1 + 2 * HM;
#pragma omp parallel
      {
        std::vector<double> fsp(5 * L), fsm(5 * L), fhp(5 * (dim + 2)), fhm(5 * (dim + 2)), fh(5 * (dim + 2)),
            scr(2 * (dim + 8));
#pragma omp for collapse(2) schedule(static)
        for (int b = 0; b <= dims[o2]; ++b)
          for (int a = 0; a <= dims[o1]; ++a) {
            int p[3];
            p[o1] = a; p[o2] = b;
            std::fill(fsp.begin(), fsp.end(), 0.0);
            std::fill(fsm.begin(), fsm.end(), 0.0);
            for (int t = iss; t <= iee; ++t) {
              p[dir] = t;
              const double u[3] = {vel(p[0], p[1], p[2], 0), vel(p[0], p[1], p[2], 1), vel(p[0], p[1], p[2], 2)};
              double qq[5], fp[5], fm[5];
              for (int m = 0; m < 5; ++m) qq[m] = q(p[0], p[1], p[2], m);
              sw_split(rho(p[0], p[1], p[2]), u, prs(p[0], p[1], p[2]), tmp(p[0], p[1], p[2]), qq, mrow, jb, fp, fm);
              for (int m = 0; m < 5; ++m) { fsp[m * L + t + HM] = fp[m]; fsm[m * L + t + HM] = fm[m]; }
            }
            for (int m = 0; m < 5; ++m) {
              flux_line(fuw[dir], fsp.data() + m * L + HM, fhp.data() + m * (dim + 2), scr.data());
              flux_line(fdw[dir], fsm.data() + m * L + HM, fhm.data() + m * (dim + 2), scr.data());
            }
            for (int i = -1; i <= dim; ++i) {
              int jp[5], jn[5];
              for (int n = 1; n <= 5; ++n) {   // iwind6 (solver.F90:1237-1258)
                jp[n - 1] = std::min(std::max(i + n - 3, iss), iee);
                jn[n - 1] = std::min(std::max(i + 4 - n, iss), iee);
              }
              // the shock flag of the interface (solver.F90:1440-1455): both nodes' flags, or the
              // one node inside 0..dim
              bool lsh = true;
              if (lchardecomp) {
                int pa[3] = {p[0], p[1], p[2]}, pb[3] = {p[0], p[1], p[2]};
                pa[dir] = i; pb[dir] = i + 1;
                if (i < 0) lsh = shock_at(pb[0], pb[1], pb[2]);
                else if (i + 1 > dim) lsh = shock_at(pa[0], pa[1], pa[2]);
                else lsh = shock_at(pa[0], pa[1], pa[2]) || shock_at(pb[0], pb[1], pb[2]);
              }
              if (lchardecomp) {
                int pa[3] = {p[0], p[1], p[2]}, pb[3] = {p[0], p[1], p[2]};
                pa[dir] = i; pb[dir] = i + 1;
                const double vl[3] = {vel(pa[0], pa[1], pa[2], 0), vel(pa[0], pa[1], pa[2], 1), vel(pa[0], pa[1], pa[2], 2)};
                const double vr[3] = {vel(pb[0], pb[1], pb[2], 0), vel(pb[0], pb[1], pb[2], 1), vel(pb[0], pb[1], pb[2], 2)};
                double REV[5][5], LEV[5][5];
                chardecomp(tmp(pa[0], pa[1], pa[2]), rho(pa[0], pa[1], pa[2]), prs(pa[0], pa[1], pa[2]),
                           q(pa[0], pa[1], pa[2], 4), vl, tmp(pb[0], pb[1], pb[2]), rho(pb[0], pb[1], pb[2]),
                           prs(pb[0], pb[1], pb[2]), q(pb[0], pb[1], pb[2], 4), vr, mrow, REV, LEV);
                double fhc[5];
                for (int m = 0; m < 5; ++m) {
                  double up[5], um[5];
                  for (int n = 0; n < 5; ++n) {
                    double sp = 0.0, sm = 0.0;
                    sp = LEV[m][0] * fsp[0 * L + jp[n] + HM] + LEV[m][1] * fsp[1 * L + jp[n] + HM] +
                         LEV[m][2] * fsp[2 * L + jp[n] + HM] + LEV[m][3] * fsp[3 * L + jp[n] + HM] +
                         LEV[m][4] * fsp[4 * L + jp[n] + HM];
                    sm = LEV[m][0] * fsm[0 * L + jn[n] + HM] + LEV[m][1] * fsm[1 * L + jn[n] + HM] +
                         LEV[m][2] * fsm[2 * L + jn[n] + HM] + LEV[m][3] * fsm[3 * L + jn[n] + HM] +
                         LEV[m][4] * fsm[4 * L + jn[n] + HM];
                    up[n] = sp;
                    um[n] = sm;
                  }
                  const int c = i + 1;
                  const double hp = LEV[m][0] * fhp[0 * (dim + 2) + c] + LEV[m][1] * fhp[1 * (dim + 2) + c] +
                                    LEV[m][2] * fhp[2 * (dim + 2) + c] + LEV[m][3] * fhp[3 * (dim + 2) + c] +
                                    LEV[m][4] * fhp[4 * (dim + 2) + c];
                  const double hm = LEV[m][0] * fhm[0 * (dim + 2) + c] + LEV[m][1] * fhm[1 * (dim + 2) + c] +
                                    LEV[m][2] * fhm[2 * (dim + 2) + c] + LEV[m][3] * fhm[3 * (dim + 2) + c] +
                                    LEV[m][4] * fhm[4 * (dim + 2) + c];
                  fhc[m] = mplimiter(up, hp, lsh, i, dim, nt) + mplimiter(um, hm, lsh, i, dim, nt);
                }
                for (int m = 0; m < 5; ++m)
                  fh[m * (dim + 2) + i + 1] = REV[m][0] * fhc[0] + REV[m][1] * fhc[1] + REV[m][2] * fhc[2] +
                                              REV[m][3] * fhc[3] + REV[m][4] * fhc[4];
                continue;
              }
              for (int m = 0; m < 5; ++m) {
                double up[5], um[5];
                for (int n = 0; n < 5; ++n) {
                  up[n] = fsp[m * L + jp[n] + HM];
                  um[n] = fsm[m * L + jn[n] + HM];
                }
                const double v1 = mplimiter(up, fhp[m * (dim + 2) + i + 1], lsh, i, dim, nt);
                const double v2 = mplimiter(um, fhm[m * (dim + 2) + i + 1], lsh, i, dim, nt);
                fh[m * (dim + 2) + i + 1] = v1 + v2;
              }
            }
            for (int i = 0; i <= dim; ++i) {
              p[dir] = i;
              for (int m = 0; m < 5; ++m)
                qrhs(p[0], p[1], p[2], m) = qrhs(p[0], p[1], p[2], m) + fh[m * (dim + 2) + i + 1] - fh[m * (dim + 2) + i];
            }
          }
      }
    }
  }

  void fs_rhscal() {
    std::fill(qrhs.v.begin(), qrhs.v.end(), 0.0);
    fs_gradcal();
    if (conschm == 543) {
      if (lchardecomp) ducros_sensor();
      fs_convection_upwind();
    } else {
      fs_convection();
    }
    for (double& v : qrhs.v) v = -v;
    fs_diffusion();
  }

  // boucon with isothermal no-slip walls (bctype 41, noslip, src/bc.F90:6281-6595) at every
  // physical end: u = v = w = 0, T = twall, the pressure extrapolated from the two nodes next to
  // the wall, p_w = (4 p_1 - p_2)/3, rho = p/T gamma M^2 (thermal), q by fvar2q. The ends are
  // visited in boucon's order (i-min, i-max, j-min, j-max, k-min, k-max).
  void fs_boucon() {
    const int dims[3] = {im, jm, km};
    for (int dir = 0; dir < 3; ++dir) {
      const bool lo = ntype[dir] == 1 || ntype[dir] == 4, hi = ntype[dir] == 2 || ntype[dir] == 4;
      const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
      for (int side = 0; side < 2; ++side) {
        if (!(side == 0 ? lo : hi)) continue;
        const int w = side == 0 ? 0 : dims[dir], s1 = side == 0 ? 1 : -1;
        for (int b = 0; b <= dims[o2]; ++b)
          for (int a = 0; a <= dims[o1]; ++a) {
            int p[3], p1[3], p2[3];
            p[o1] = p1[o1] = p2[o1] = a;
            p[o2] = p1[o2] = p2[o2] = b;
            p[dir] = w; p1[dir] = w + s1; p2[dir] = w + 2 * s1;
            const double pe = num1d3 * (4.0 * prs(p1[0], p1[1], p1[2]) - prs(p2[0], p2[1], p2[2]));
            for (int c = 0; c < 3; ++c) vel(p[0], p[1], p[2], c) = 0.0;
            prs(p[0], p[1], p[2]) = pe;
            tmp(p[0], p[1], p[2]) = twall;
            rho(p[0], p[1], p[2]) = pe / twall * const2;
            const double u[3] = {0.0, 0.0, 0.0};
            double qq[5];
            fvar2q(qq, rho(p[0], p[1], p[2]), u, pe);
            for (int m = 0; m < 5; ++m) q(p[0], p[1], p[2], m) = qq[m];
          }
      }
    }
  }

  // One step of time_integration_rk (rk3), mainloop.F90:392-476; history row at stage 1 after
  // gradcal, as in the miniapp.
  void rk3_full() {
    static const double rkcoe[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {num1d3, num2d3, num2d3}};
    const double jb = jac();
    for (int rk = 0; rk < 3; ++rk) {
      if (lfilter) filterq();
      fs_boucon();
      fs_qswap();
      fs_rhscal();
      if (rk == 0) {
        stacal();
#pragma omp parallel for collapse(2)
        for (int k = 0; k <= km; ++k)
          for (int j = 0; j <= jm; ++j)
            for (int i = 0; i <= im; ++i)
              for (int m = 0; m < 5; ++m) qsave(i, j, k, m) = q(i, j, k, m) * jb;
      }
      const double c1 = rkcoe[rk][0], c2 = rkcoe[rk][1], c3 = rkcoe[rk][2];
#pragma omp parallel for collapse(2)
      for (int k = 0; k <= km; ++k)
        for (int j = 0; j <= jm; ++j)
          for (int i = 0; i <= im; ++i)
            for (int m = 0; m < 5; ++m) {
              double v = c1 * qsave(i, j, k, m) + c2 * q(i, j, k, m) * jb + c3 * qrhs(i, j, k, m) * deltat;
              q(i, j, k, m) = v / jb;
            }
      update_prims();
    }
    nstep += 1;
    time = time + deltat;
  }

  // One rhscal of the full solver on the current state (filterq and qswap first, as a stage does)
  void rhs_full() {
    if (lfilter) filterq();
    fs_boucon();
    fs_qswap();
    fs_rhscal();
  }

  // Boundary types per direction (ntype of fd_scheme_initiate / compact_filter_initiate) and
  // the wall temperature of the physical ends.
  void set_boundaries(const int* nt, double tw) {
    const int dims[3] = {im, jm, km};
    twall = tw;
    for (int d = 0; d < 3; ++d) {
      ntype[d] = nt[d];
      fds[d] = Scheme();
      flt[d] = Scheme();
      fd_scheme_initiate(fds[d], "643c", nt[d], dims[d]);
      compact_filter_initiate(flt[d], nt[d], dims[d], alfa_f, false);
      filter_coefficient_cal(flt[d], alfa_f, beta_h, beta_b);
    }
    build_flux_schemes();
  }

  // Convection scheme of the full-solver mode: 643 (central) or 543 (upwind compact flux).
  bool set_convection(int scheme, double bfac, int chardecomp_on, double shock_threshold) {
    if (scheme != 643 && scheme != 543) return false;
    conschm = scheme;
    bfacmpld = bfac;
    lchardecomp = scheme == 543 && chardecomp_on != 0;
    shkcrt = shock_threshold;
    if (lchardecomp) {
      ssf.init(im, jm, km, HM, 1);
      lshock.assign((size_t)(im + 1) * (jm + 1) * (km + 1), 0);
    }
    build_flux_schemes();
    return true;
  }

  // rk3, tgvsolver.F90:994-1082, and the step counter of steploop (:944-960)
  void rk3() {
    static const double rkcoe[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {num1d3, num2d3, num2d3}};
    for (int rk = 0; rk < 3; ++rk) {
      bchomo();
      rhscal();
      if (rk == 0) {
        stacal();
#pragma omp parallel for collapse(2)
        for (int k = 0; k <= km; ++k)
          for (int j = 0; j <= jm; ++j)
            for (int i = 0; i <= im; ++i)
              for (int m = 0; m < 5; ++m) qsave(i, j, k, m) = q(i, j, k, m);
      }
      const double c1 = rkcoe[rk][0], c2 = rkcoe[rk][1], c3 = rkcoe[rk][2];
#pragma omp parallel for collapse(2)
      for (int k = 0; k <= km; ++k)
        for (int j = 0; j <= jm; ++j)
          for (int i = 0; i <= im; ++i)
            for (int m = 0; m < 5; ++m)
              q(i, j, k, m) = c1 * qsave(i, j, k, m) + c2 * q(i, j, k, m) + c3 * qrhs(i, j, k, m) * deltat;
      if (lfilter) filterq();
      update_prims();
    }
    nstep += 1;
    time = time + deltat;
  }

  // cflcal's spectral-radius sum (commcal.F90:46-77) on a uniform grid, dxi = diag(1/dx,1/dy,1/dz)
  double cfl_dt(double cfl) {
    double di = 0.0, dj = 0.0, dk = 0.0;
    const double dxi[3] = {1.0 / dx, 1.0 / dy, 1.0 / dz};
    for (int k = 0; k <= km; ++k)
      for (int j = 0; j <= jm; ++j)
        for (int i = 0; i <= im; ++i) {
          double ubar = dxi[0] * vel(i, j, k, 0), vbar = dxi[1] * vel(i, j, k, 1), wbar = dxi[2] * vel(i, j, k, 2);
          double css = std::sqrt(tmp(i, j, k)) / mach;
          double csi = css * std::sqrt(dxi[0] * dxi[0]), csj = css * std::sqrt(dxi[1] * dxi[1]),
                 csk = css * std::sqrt(dxi[2] * dxi[2]);
          di = std::max({di, ubar, ubar - csi, ubar + csi});
          dj = std::max({dj, vbar, vbar - csj, vbar + csj});
          dk = std::max({dk, wbar, wbar - csk, wbar + csk});
        }
    return cfl / (di + dj + dk);
  }
};

}  // namespace

// ================================================================ C entry points (ctypes)
extern "C" {

void* orc_fd_scheme_create(const char* scheme, int ntype, int dim) {
  Scheme* s = new Scheme();
  if (!fd_scheme_initiate(*s, scheme, ntype, dim)) { delete s; return nullptr; }
  return s;
}
void* orc_filter_create(int ntype, int dim, double alfa, double beta_halo, double beta_bound, int no_filter_note) {
  Scheme* s = new Scheme();
  compact_filter_initiate(*s, ntype, dim, alfa, no_filter_note != 0);
  filter_coefficient_cal(*s, alfa, beta_halo, beta_bound);
  return s;
}
void orc_scheme_free(void* h) { delete static_cast<Scheme*>(h); }
int orc_scheme_info(void* h, int* first_node, int* last_node) {
  Scheme* s = static_cast<Scheme*>(h);
  *first_node = s->first_node; *last_node = s->last_node;
  return s->n();
}
void orc_scheme_ac(void* h, double* ac1, double* ac2, double* ac3) {
  Scheme* s = static_cast<Scheme*>(h);
  for (int i = 0; i < s->n(); ++i) { ac1[i] = s->ac1[i]; ac2[i] = s->ac2[i]; ac3[i] = s->ac3[i]; }
}

// One line: f holds f(-5..dim+5), out holds dim+1 values.
void orc_deriv_line(void* h, const double* f, double* out) {
  Scheme* s = static_cast<Scheme*>(h);
  std::vector<double> scr(2 * (s->dimension + 8));
  df_line(*s, f + HM, out, scr.data());
}
void orc_filter_line(void* h, const double* f, double* out) {
  Scheme* s = static_cast<Scheme*>(h);
  std::vector<double> scr(2 * (s->dimension + 8));
  filter_line(*s, f + HM, out, scr.data());
}

// Every line of a Fortran-ordered multi-field array; output extent along dir is 0..dim.
void orc_deriv3d(void* h, int dir, const double* f, const int64_t* shape, const int64_t* lbound, int nfields, double* out) {
  Scheme* s = static_cast<Scheme*>(h);
  Box b{{shape[0], shape[1], shape[2]}, {lbound[0], lbound[1], lbound[2]}};
  apply_lines(*s, dir, f, b, nfields, out, [](const Scheme& sc, const double* fi, double* o, double* scr) { df_line(sc, fi, o, scr); });
}
void* orc_flux_create(int scheme, int ntype, int dim, int wind, double bfac) {
  Scheme* s = new Scheme();
  if (!compact_flux_initiate(*s, scheme, ntype, dim, wind, bfac)) { delete s; return nullptr; }
  return s;
}
// One line: f holds f(-5..dim+5), out holds the dim+2 interface values fh(-1..dim).
void orc_flux_line(void* h, const double* f, double* out) {
  Scheme* s = static_cast<Scheme*>(h);
  std::vector<double> scr(2 * (s->dimension + 8));
  flux_line(*s, f + HM, out, scr.data());
}
// Every line of a Fortran-ordered multi-field array; output extent along dir is -1..dim.
void orc_flux3d(void* h, int dir, const double* f, const int64_t* shape, const int64_t* lbound, int nfields, double* out) {
  Scheme* s = static_cast<Scheme*>(h);
  Box bf{{shape[0], shape[1], shape[2]}, {lbound[0], lbound[1], lbound[2]}};
  Box bo = bf;
  bo.n[dir] = s->dimension + 2;
  bo.l[dir] = -1;
  const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
  const int dim = s->dimension;
#pragma omp parallel
  {
    std::vector<double> lin(dim + 1 + 2 * HM, 0.0), lout(dim + 2), scr(2 * (dim + 8));
#pragma omp for collapse(2) schedule(static)
    for (int64_t b = 0; b < bf.n[o2]; ++b)
      for (int64_t a = 0; a < bf.n[o1]; ++a) {
        int64_t ijk[3];
        ijk[o1] = bf.l[o1] + a;
        ijk[o2] = bf.l[o2] + b;
        for (int m = 0; m < nfields; ++m) {
          for (int t = -HM; t <= dim + HM; ++t) {
            int64_t p[3] = {ijk[0], ijk[1], ijk[2]};
            p[dir] = t;
            lin[t + HM] = (t >= bf.l[dir] && t < bf.l[dir] + bf.n[dir]) ? f[m * bf.size() + bf.idx(p[0], p[1], p[2])] : 0.0;
          }
          flux_line(*s, lin.data() + HM, lout.data(), scr.data());
          for (int t = -1; t <= dim; ++t) {
            int64_t p[3] = {ijk[0], ijk[1], ijk[2]};
            p[dir] = t;
            out[m * bo.size() + bo.idx(p[0], p[1], p[2])] = lout[t + 1];
          }
        }
      }
  }
}
void orc_filter3d(void* h, int dir, const double* f, const int64_t* shape, const int64_t* lbound, int nfields, double* out) {
  Scheme* s = static_cast<Scheme*>(h);
  Box b{{shape[0], shape[1], shape[2]}, {lbound[0], lbound[1], lbound[2]}};
  apply_lines(*s, dir, f, b, nfields, out, [](const Scheme& sc, const double* fi, double* o, double* scr) { filter_line(sc, fi, o, scr); });
}

void* orc_tgv_create(int im, int jm, int km, double mach, double re, double pr, double gamma, double ref_tem,
                     double suth, double alfa_filter, double beta_halo, double beta_bound, int filter_on) {
  TGV* t = new TGV();
  t->setup(im, jm, km, mach, re, pr, gamma, ref_tem, suth, alfa_filter, beta_halo, beta_bound, filter_on);
  return t;
}
void orc_tgv_free(void* h) { delete static_cast<TGV*>(h); }
void orc_tgv_init_tgv(void* h) { static_cast<TGV*>(h)->init_tgv(); }
void orc_tgv_set_q(void* h, const double* q) { static_cast<TGV*>(h)->set_q(q); }
void orc_tgv_get_q(void* h, double* q) { static_cast<TGV*>(h)->get_q(q); }
void orc_tgv_set_flowfield(void* h, const double* f) { static_cast<TGV*>(h)->set_flowfield(f); }
void orc_tgv_get_flowfield(void* h, double* f) { static_cast<TGV*>(h)->get_flowfield(f); }
void orc_tgv_set_dt(void* h, double dt) { static_cast<TGV*>(h)->deltat = dt; }
double orc_tgv_cfl_dt(void* h, double cfl) { return static_cast<TGV*>(h)->cfl_dt(cfl); }
void orc_tgv_steps(void* h, int n) { TGV* t = static_cast<TGV*>(h); for (int s = 0; s < n; ++s) t->rk3(); }
void orc_tgv_set_boundaries(void* h, int n0, int n1, int n2, double twall) {
  const int nt[3] = {n0, n1, n2};
  static_cast<TGV*>(h)->set_boundaries(nt, twall);
}
int orc_tgv_set_convection(void* h, int scheme, double bfac, int lchardecomp, double shkcrt) {
  return static_cast<TGV*>(h)->set_convection(scheme, bfac, lchardecomp, shkcrt) ? 0 : -1;
}
// flux_steger_warming of one node for a gas (gamma, mach): fp[5], fm[5].
void orc_sw_split(double gamma, double mach, double r, const double* u, double p, double t, const double* qq,
                  const double* metric, double jb, double* fp, double* fm) {
  TGV tg;
  tg.gamma = gamma;
  tg.mach = mach;
  tg.sw_split(r, u, p, t, qq, metric, jb, fp, fm);
}
// MP5 of one stencil u[5] with the linear value ul (flux.F90:434-496).
double orc_mp5(const double* u, double ul, int discont) { return TGV::mp5(u, ul, discont != 0); }
// chardecomp of one interface (row-major R[5][5], L[5][5]) for a gas with ratio of specific heats gamma.
void orc_chardecomp(double gamma, double rl, double pl, double el, const double* vl, double rr, double pr, double er,
                    const double* vr, const double* ddi, double* R, double* L) {
  TGV t;
  t.gamma = gamma;
  double RR[5][5], LL[5][5];
  t.chardecomp(1.0, rl, pl, el, vl, 1.0, rr, pr, er, vr, ddi, RR, LL);
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 5; ++b) { R[5 * a + b] = RR[a][b]; L[5 * a + b] = LL[a][b]; }
}
// The shock flags of the last rhscal with the characteristic decomposition (nodes 0..N, x fastest).
int orc_tgv_shock_flags(void* h, unsigned char* out) {
  TGV* t = static_cast<TGV*>(h);
  if (!t->lchardecomp) return -1;
  for (size_t n = 0; n < t->lshock.size(); ++n) out[n] = (unsigned char)t->lshock[n];
  return 0;
}
// Full-solver mode (time_integration_rk of the full solver, see rk3_full).
void orc_tgv_steps_full(void* h, int n) { TGV* t = static_cast<TGV*>(h); for (int s = 0; s < n; ++s) t->rk3_full(); }
// One full-solver rhscal (after the stage's filterq and qswap) into qrhs on nodes 0..N; the state
// keeps the filtered, averaged q.
void orc_tgv_rhs_full(void* h, double* out) {
  TGV* t = static_cast<TGV*>(h);
  t->rhs_full();
  const int64_t n0 = t->im + 1, n1 = t->jm + 1, n2 = t->km + 1, nn = n0 * n1 * n2;
  for (int m = 0; m < 5; ++m)
    for (int k = 0; k <= t->km; ++k)
      for (int j = 0; j <= t->jm; ++j)
        for (int i = 0; i <= t->im; ++i) out[m * nn + ((int64_t)k * n1 + j) * n0 + i] = t->qrhs(i, j, k, m);
}
int orc_tgv_history(void* h, double* out, int maxrows) {
  TGV* t = static_cast<TGV*>(h);
  int rows = (int)(t->hist.size() / 5);
  int nr = std::min(rows, maxrows);
  std::memcpy(out, t->hist.data(), sizeof(double) * 5 * nr);
  return rows;
}
int orc_tgv_history_compensated(void* h, double* out, int maxrows) {
  TGV* t = static_cast<TGV*>(h);
  int rows = (int)(t->hist_c.size() / 5);
  int nr = std::min(rows, maxrows);
  std::memcpy(out, t->hist_c.data(), sizeof(double) * 5 * nr);
  return rows;
}
// One rhscal on the current state (after the halo fill): qrhs on nodes 0..N, Fortran order.
void orc_tgv_rhs(void* h, double* out) {
  TGV* t = static_cast<TGV*>(h);
  t->bchomo();
  t->rhscal();
  const int64_t n0 = t->im + 1, n1 = t->jm + 1, n2 = t->km + 1, nn = n0 * n1 * n2;
  for (int m = 0; m < 5; ++m)
    for (int k = 0; k <= t->km; ++k)
      for (int j = 0; j <= t->jm; ++j)
        for (int i = 0; i <= t->im; ++i) out[m * nn + ((int64_t)k * n1 + j) * n0 + i] = t->qrhs(i, j, k, m);
}
// Diagnostics of the current state computed the way stacal does (needs one gradcal).
void orc_tgv_diagnostics(void* h, double* out3) {
  TGV* t = static_cast<TGV*>(h);
  t->bchomo();
  t->gradcal();
  t->stacal();
  size_t n = t->hist.size();
  out3[0] = t->hist[n - 3]; out3[1] = t->hist[n - 2]; out3[2] = t->hist[n - 1];
  t->hist.resize(n - 5);
  t->hist_c.resize(t->hist_c.size() - 5);
}
int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // extern "C"
