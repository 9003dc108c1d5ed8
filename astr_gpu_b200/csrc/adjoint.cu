// Discrete adjoint of the periodic RK3 step: transposed line operators (host construction),
// the pointwise vector-Jacobian products of the right-hand side, and the objective.
//
// The forward right-hand side of one stage (rhscal, tgvsolver.F90:962-992) is
//   rhs = -sum_d D_d F_d(q) + sum_d D_d VF_d(G, T, u),   G_kd = D_d(u_k, T),
// with D_d = (compact derivative along d)/dx_d, F_d the Euler fluxes (convection,
// tgvsolver.F90:539-633), VF_d = (sigma_d1, sigma_d2, sigma_d3, qflux_d) (diffusion,
// tgvsolver.F90:635-789); the stage update is q' = Fz Fy Fx (c1 qsave + c2 q + c3 dt rhs)
// (rk3, tgvsolver.F90:1037-1074, filterq :791-883). The adjoint of a stage, given lam' = dJ/dq':
//   lam_new = Fx^T Fy^T Fz^T lam'
//   lam_qsave += c1 lam_new,  lam_q = c2 lam_new + (d rhs/d q)^T (c3 dt lam_new)
// where (d rhs/dq)^T y is assembled from Y_d = D_d^T y: the flux products with lam_F_d = -Y_d, the
// viscous products with lam_VF_d = Y_d(1..4), the gradient transposes D_d^T of lam_G, and the
// products of the primitive-variable map q -> (u, p, T).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "adjoint.cuh"
#include "internal.h"

namespace astr {

// ------------------------------------------------------------------ transposed operators (host)
namespace {

// Value of RHS row r of `op` for the line f (the forward kernels' formulas, host copy).
template <class Get>
double row_value(const LineOp& op, int r, Get f) {
  double s = 0.0;
  const int j = r - op.ext_lo;
  if (op.kind == OP_FILTER) {
    if (filter_special(op, r, f, s)) return s;
    return op.c10[0] * (f(j) + f(j)) + op.c10[1] * (f(j + 1) + f(j - 1)) + op.c10[2] * (f(j + 2) + f(j - 2)) +
           op.c10[3] * (f(j + 3) + f(j - 3)) + op.c10[4] * (f(j + 4) + f(j - 4)) + op.c10[5] * (f(j + 5) + f(j - 5));
  }
  if (deriv_special(op, r, f, s)) return s;
  return (7.0 / 9.0) * (f(j + 1) - f(j - 1)) + (1.0 / 36.0) * (f(j + 2) - f(j - 2));
}

}  // namespace

bool build_adjoint_op(const HostOp& fwd, AdjHostOp& out, std::string& err) {
  if (fwd.ntype != 3 || fwd.kind == OP_EXPLICIT) {
    err = "the adjoint covers periodic (ntype 3) compact operators only";
    return false;
  }
  const int n = fwd.nsys(), dim = fwd.dim, e = -fwd.first_node;
  // A^T: sub-diagonal c_{r-1}, super-diagonal a_{r+1} (A's a_0 and c_{n-1} are never used)
  HostOp t = fwd;
  for (int r = 0; r < n; ++r) {
    t.a[r] = (r >= 1) ? fwd.c[r - 1] : 0.0;
    t.c[r] = (r <= n - 2) ? fwd.a[r + 1] : 0.0;
  }
  t.ac1.assign(n, 0.0); t.ac2.assign(n, 0.0); t.ac3.assign(n, 0.0);
  t.ac1[0] = t.c[0];
  for (int r = 1; r < n; ++r) {
    const double piv = 1.0 - t.a[r] * t.ac1[r - 1];
    t.ac1[r] = t.c[r] / piv;
    t.ac2[r] = 1.0 / piv;
    t.ac3[r] = t.a[r] / piv;
  }
  out.tri = t;
  // W(m, r) = sum over extended nodes x with wrap(x) = m of B(r, x)
  LineOp op{};
  fill_lineop(fwd, op);
  std::vector<double> W((size_t)(dim + 1) * n, 0.0);
  const int reach = 12;
  for (int r = 0; r < n; ++r) {
    const int node = r - e;
    for (int x = node - reach; x <= node + reach; ++x) {
      const double b = row_value(op, r, [x](int k) { return k == x ? 1.0 : 0.0; });
      if (b == 0.0) continue;
      if (x < -dim || x > 2 * dim) { err = "operator reaches past one periodic image"; return false; }
      const int m = x < 0 ? x + dim : (x > dim ? x - dim : x);
      W[(size_t)m * n + r] += b;
    }
  }
  AdjW& w = out.w;
  std::memset(&w, 0, sizeof(w));
  w.jlo = -(ADJ_BAND / 2);
  auto band_ok = [&](int m, const double* pat) {
    for (int r = 0; r < n; ++r) {
      const int j = r - e - m - w.jlo;
      const double v = W[(size_t)m * n + r];
      if (j < 0 || j >= ADJ_BAND) { if (v != 0.0) return false; }
      else if (pat && v != pat[j]) return false;
    }
    return true;
  };
  const int mid = dim / 2;
  for (int j = 0; j < ADJ_BAND; ++j) {
    const int r = mid + w.jlo + j + e;
    w.wint[j] = (r >= 0 && r < n) ? W[(size_t)mid * n + r] : 0.0;
  }
  if (!band_ok(mid, w.wint)) { err = "interior column of the operator is wider than the adjoint band"; return false; }
  w.mlo = mid;
  while (w.mlo > 0 && band_ok(w.mlo - 1, w.wint)) --w.mlo;
  w.mhi = mid;
  while (w.mhi < dim && band_ok(w.mhi + 1, w.wint)) ++w.mhi;
  // trim the interior stencil to its nonzero span (5 points for the derivative, 11 for the filter)
  int j0 = 0, j1 = ADJ_BAND - 1;
  while (j0 < j1 && w.wint[j0] == 0.0) ++j0;
  while (j1 > j0 && w.wint[j1] == 0.0) --j1;
  double trimmed[ADJ_BAND] = {0.0};
  for (int j = j0; j <= j1; ++j) trimmed[j - j0] = w.wint[j];
  std::memcpy(w.wint, trimmed, sizeof(trimmed));
  w.jlo += j0;
  w.nint = j1 - j0 + 1;
  out.sptr.assign(1, 0);
  out.snode.clear();
  out.scoef.clear();
  auto add_list = [&](int m) {
    for (int r = 0; r < n; ++r) {
      const double v = W[(size_t)m * n + r];
      if (v == 0.0) continue;
      out.snode.push_back(r - e);
      out.scoef.push_back(v);
    }
    out.sptr.push_back((int)out.snode.size());
  };
  for (int m = 0; m < w.mlo; ++m) add_list(m);
  for (int m = w.mhi + 1; m <= dim; ++m) add_list(m);
  return true;
}

cudaError_t make_adj_devop(const AdjHostOp& h, Layout lay, AdjDevOp& out) {
  cudaError_t e = make_devop(h.tri, lay, out.tri);
  if (e != cudaSuccess) return e;
  out.w = h.w;
  const size_t ni = h.sptr.size(), ns = h.snode.size();
  e = cudaMalloc(&out.dmem, ni * sizeof(int) + ns * sizeof(int) + ns * sizeof(double) + 16);
  if (e != cudaSuccess) return e;
  char* base = static_cast<char*>(out.dmem);
  double* scoef = reinterpret_cast<double*>(base);
  int* sptr = reinterpret_cast<int*>(base + ns * sizeof(double));
  int* snode = sptr + ni;
  if (ns) e = cudaMemcpy(scoef, h.scoef.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(sptr, h.sptr.data(), ni * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && ns) e = cudaMemcpy(snode, h.snode.data(), ns * sizeof(int), cudaMemcpyHostToDevice);
  out.w.sptr = sptr;
  out.w.snode = snode;
  out.w.scoef = scoef;
  return e;
}

void free_adj_devop(AdjDevOp& d) {
  free_devop(d.tri);
  if (d.dmem) cudaFree(d.dmem);
  d.dmem = nullptr;
}

// ------------------------------------------------------------------ pointwise products
namespace {

// Nodes of a state array: n0 x n1 x n2, x rows padded to px elements; fs elements per field.
struct PtGeo {
  int n0, n1, n2;
  int64_t px, fs;
};

// Element index of this thread; false for the x padding and past the end.
__device__ __forceinline__ bool pt_index(const PtGeo& g, int64_t& idx) {
  idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  return idx < g.fs && (idx % g.px) < g.n0;
}

// Flux, viscous and RK-combination products of one stage at every node (see the file header).
__global__ void k_adj_point1(PtGeo g, Thermo th, const double* __restrict__ q, const double* __restrict__ G,
                             const double* __restrict__ Y, const double* __restrict__ lnew, double c1, double c2,
                             double* __restrict__ lsave, double* __restrict__ lq, double* __restrict__ U,
                             double* __restrict__ lp_out, double* __restrict__ LG) {
  int64_t i;
  if (!pt_index(g, i)) return;
  const int64_t fs = g.fs;
  const double rho = q[i];
  double m[3], u[3];
  for (int a = 0; a < 3; ++a) { m[a] = q[(a + 1) * fs + i]; u[a] = m[a] / rho; }
  const double q4 = q[4 * fs + i];
  const double p = (q4 - 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2])) / th.const6;
  const double T = p / rho * th.const2;
  double Gab[3][3], GT[3];
  for (int b = 0; b < 3; ++b) {
    for (int a = 0; a < 3; ++a) Gab[a][b] = G[(b * 4 + a) * fs + i];
    GT[b] = G[(b * 4 + 3) * fs + i];
  }
  double Sab[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Sab[a][b] = 0.5 * (Gab[a][b] + Gab[b][a]);
  const double skk = (1.0 / 3.0) * (Sab[0][0] + Sab[1][1] + Sab[2][2]);
  const double sq = sqrt(T);
  const double miu = T * sq * th.tc1 / (T + th.tc) / th.reynolds;
  const double hcc = (miu / th.prandtl) / th.const5;
  double sig[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) sig[a][b] = 2.0 * miu * (Sab[a][b] - (a == b ? skk : 0.0));
  double Yd[3][5];
  for (int d = 0; d < 3; ++d)
    for (int n = 0; n < 5; ++n) Yd[d][n] = Y[(d * 5 + n) * fs + i];
  double ln[5], lqv[5];
  for (int n = 0; n < 5; ++n) {
    ln[n] = lnew[n * fs + i];
    lsave[n * fs + i] += c1 * ln[n];
    lqv[n] = c2 * ln[n];
  }
  // Euler fluxes F_d = (q_n u_d + p delta_{n,d+1}, (q4 + p) u_d), lam_F_d = -Y_d
  double lu[3] = {0.0, 0.0, 0.0}, lp = 0.0;
  const double qn[5] = {rho, m[0], m[1], m[2], q4};
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int n = 0; n < 4; ++n) {
      const double lf = -Yd[d][n];
      lqv[n] += lf * u[d];
      s += lf * qn[n];
    }
    const double lf4 = -Yd[d][4];
    lqv[4] += lf4 * u[d];
    s += lf4 * (q4 + p);
    lu[d] += s;
    lp += -Yd[d][d + 1] + lf4 * u[d];
  }
  // viscous fluxes VF_d = (sigma_d0, sigma_d1, sigma_d2, Q_d), lam_VF_d = Y_d(1..4)
  double Lam[3][3], lQ[3];
  for (int a = 0; a < 3; ++a) lQ[a] = Yd[a][4];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Lam[a][b] = Yd[a][b + 1] + lQ[a] * u[b];
  double lhcc = 0.0;
  for (int a = 0; a < 3; ++a) {
    for (int b = 0; b < 3; ++b) lu[b] += lQ[a] * sig[a][b];
    lhcc += lQ[a] * GT[a];
  }
  const double trL = Lam[0][0] + Lam[1][1] + Lam[2][2];
  double lmiu = 0.0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) lmiu += Lam[a][b] * Sab[a][b];
  lmiu = 2.0 * (lmiu - skk * trL) + lhcc / (th.prandtl * th.const5);
  // miucal'(T) = tc1 sqrt(T) (T + 3 tc) / (2 (T + tc)^2)
  const double tp = T + th.tc;
  const double lT = lmiu * th.tc1 * sq * (T + 3.0 * th.tc) / (2.0 * tp * tp) / th.reynolds;
  for (int b = 0; b < 3; ++b) {
    for (int a = 0; a < 3; ++a)
      LG[(b * 4 + a) * fs + i] = 2.0 * miu * (0.5 * (Lam[a][b] + Lam[b][a]) - (a == b ? trL / 3.0 : 0.0));
    LG[(b * 4 + 3) * fs + i] = lQ[b] * hcc;
  }
  for (int n = 0; n < 5; ++n) lq[n * fs + i] = lqv[n];
  for (int a = 0; a < 3; ++a) U[a * fs + i] = lu[a];
  U[3 * fs + i] = lT;
  lp_out[i] = lp;
}

// lam_q += products of the primitive map q -> (u, p, T) with (lam_u, lam_T) = U, lam_p.
__global__ void k_adj_point2(PtGeo g, Thermo th, const double* __restrict__ q, const double* __restrict__ U,
                             const double* __restrict__ lp_in, double* __restrict__ lq, const double* __restrict__ lsum,
                             int add_sum) {
  int64_t i;
  if (!pt_index(g, i)) return;
  const int64_t fs = g.fs;
  const double rho = q[i];
  double u[3];
  for (int a = 0; a < 3; ++a) u[a] = q[(a + 1) * fs + i] / rho;
  const double u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const double p = (q[4 * fs + i] - 0.5 * rho * u2) / th.const6;
  const double lT = U[3 * fs + i];
  const double lpt = lp_in[i] + lT * th.const2 / rho;
  double l0 = -lT * p * th.const2 / (rho * rho) + lpt * 0.5 * u2 / th.const6;
  double out[5];
  for (int a = 0; a < 3; ++a) {
    const double lu = U[a * fs + i];
    l0 -= lu * u[a] / rho;
    out[a + 1] = lu / rho - lpt * u[a] / th.const6;
  }
  out[0] = l0;
  out[4] = lpt / th.const6;
  for (int n = 0; n < 5; ++n) {
    double v = lq[n * fs + i] + out[n];
    if (add_sum) v += lsum[n * fs + i];
    lq[n * fs + i] = v;
  }
}

// dJ/dq of J = (1 / (2 im jm km)) sum over nodes 1..N of |rho u|^2 / rho.
__global__ void k_adj_objective(PtGeo g, const double* __restrict__ q, double scale, double* __restrict__ lam) {
  int64_t i;
  if (!pt_index(g, i)) return;
  const int64_t fs = g.fs;
  const int ii = (int)(i % g.px), jj = (int)((i / g.px) % g.n1), kk = (int)(i / (g.px * g.n1));
  const bool in = ii >= 1 && jj >= 1 && kk >= 1;
  const double rho = q[i];
  double m2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double mv = q[(a + 1) * fs + i];
    lam[(a + 1) * fs + i] = in ? scale * mv / rho : 0.0;
    m2 += mv * mv;
  }
  lam[i] = in ? -0.5 * scale * m2 / (rho * rho) : 0.0;
  lam[4 * fs + i] = 0.0;
}

// Per-plane sums of |rho u|^2 / rho over nodes i, j >= 1 of plane k (in node order).
__global__ void k_ke_planes(PtGeo g, const double* __restrict__ q, double* __restrict__ part) {
  __shared__ double s[256];
  const int k = blockIdx.x;
  const int64_t fs = g.fs;
  double acc = 0.0;
  if (k >= 1) {
    for (int idx = threadIdx.x; idx < (g.n0 - 1) * (g.n1 - 1); idx += blockDim.x) {
      const int ii = 1 + idx % (g.n0 - 1), jj = 1 + idx / (g.n0 - 1);
      const int64_t i = ((int64_t)k * g.n1 + jj) * g.px + ii;
      const double rho = q[i], a = q[fs + i], b = q[2 * fs + i], c = q[3 * fs + i];
      acc += (a * a + b * b + c * c) / rho;
    }
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[k] = s[0];
}

__global__ void k_ke_final(const double* __restrict__ part, int n, double scale, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += part[k];
    *out = 0.5 * scale * s;
  }
}

PtGeo pt_geo(const BoxGeo& g) {
  PtGeo p;
  p.n0 = g.N[0] + 1; p.n1 = g.N[1] + 1; p.n2 = g.N[2] + 1;
  p.px = g.st[1];
  p.fs = g.fs;
  return p;
}

unsigned pt_blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t launch_adj_point1(const BoxGeo& g, const Thermo& th, const double* q, const double* G, const double* Y,
                              const double* lnew, double c1, double c2, double* lsave, double* lq, double* U,
                              double* lp, double* LG, cudaStream_t st) {
  const PtGeo p = pt_geo(g);
  k_adj_point1<<<pt_blocks(p.fs), 256, 0, st>>>(p, th, q, G, Y, lnew, c1, c2, lsave, lq, U, lp, LG);
  return cudaGetLastError();
}

cudaError_t launch_adj_point2(const BoxGeo& g, const Thermo& th, const double* q, const double* U, const double* lp,
                              double* lq, const double* lsum, cudaStream_t st) {
  const PtGeo p = pt_geo(g);
  k_adj_point2<<<pt_blocks(p.fs), 256, 0, st>>>(p, th, q, U, lp, lq, lsum, lsum != nullptr);
  return cudaGetLastError();
}

cudaError_t launch_adj_objective(const BoxGeo& g, const double* q, double* lam, cudaStream_t st) {
  const PtGeo p = pt_geo(g);
  const double scale = 1.0 / ((double)g.N[0] * (double)g.N[1] * (double)g.N[2]);
  k_adj_objective<<<pt_blocks(p.fs), 256, 0, st>>>(p, q, scale, lam);
  return cudaGetLastError();
}

cudaError_t launch_kinetic_energy(const BoxGeo& g, const double* q, double* part, double* out, cudaStream_t st) {
  const PtGeo p = pt_geo(g);
  const double scale = 1.0 / ((double)g.N[0] * (double)g.N[1] * (double)g.N[2]);
  k_ke_planes<<<p.n2, 256, 0, st>>>(p, q, part);
  k_ke_final<<<1, 32, 0, st>>>(part, p.n2, scale, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ layout dispatch
template <int S, int WPL>
cudaError_t launch_adj_lines_t(const AdjLineArgs& a, cudaStream_t st);
template <int S, int WPL>
cudaError_t launch_adj_grad_t(const PassArgs& a, cudaStream_t st);

#define ASTR_ADJ_DISPATCH(FN, ARG)                                          \
  if (S == 3 && WPL == 1) return FN<3, 1>(ARG, st);                         \
  if (S == 5 && WPL == 1) return FN<5, 1>(ARG, st);                         \
  if (S == 9 && WPL == 1) return FN<9, 1>(ARG, st);                         \
  if (S == 5 && WPL == 2) return FN<5, 2>(ARG, st);                         \
  if (S == 9 && WPL == 2) return FN<9, 2>(ARG, st);                         \
  if (S == 5 && WPL == 4) return FN<5, 4>(ARG, st);                         \
  if (S == 9 && WPL == 4) return FN<9, 4>(ARG, st);                         \
  return cudaErrorInvalidValue;

cudaError_t launch_adj_lines(const AdjLineArgs& a, int S, int WPL, cudaStream_t st) {
  ASTR_ADJ_DISPATCH(launch_adj_lines_t, a)
}
cudaError_t launch_adj_grad(const PassArgs& a, int S, int WPL, cudaStream_t st) {
  ASTR_ADJ_DISPATCH(launch_adj_grad_t, a)
}
#undef ASTR_ADJ_DISPATCH

}  // namespace astr
