// The full solver's time integration on a box of one rank, on the reference's own array layout:
// periodic directions, or physical ends with the compact closures and isothermal no-slip walls.
//
// ASTR's production stage (time_integration_rk with rk3, src/mainloop.F90:392-476) differs from
// the miniapp's (tgvsolver.F90:994-1082) in four ways that change results: the filter runs
// before rhscal at every stage (filterq, src/comsolver.F90:514-632); qswap
// (src/parallel.F90:4877-5060) copies the periodic halos of q, averages nodes 0 and N per
// direction and recomputes the primitive variables only on the planes -hm..0 and N..N+hm, so the
// interior primitives used by rhscal stay those of the unfiltered state of the last updatefvar
// (src/fludyna.F90:191-242); rhscal takes the metric form (gradcal multiplies by dxi,
// src/comsolver.F90:244-497; convrsdcal6 and diffrsdcal6 carry the Jacobian,
// src/solver.F90:2174-2874); the update advances q*jacob (src/mainloop.F90:438-446).
//
// Because halo values differ from the periodic images of the interior (stale copies taken before
// the averaging, primitives of the filtered state), this mode keeps every field on the reference's
// layout: Fortran order, nodes -hm..N+hm on every axis (hm = 5), halos stored. Each stage is a
// sequence of small pointwise kernels and line-operator launches (lines.cu) over those arrays,
// one operation of the reference at a time. The metrics of the uniform grid are taken in closed
// form: dxi = diag(1/dx, 1/dy, 1/dz), jacob = dx*dy*dz; the off-diagonal terms add zeros.
//
// Convection is the central compact scheme (convrsdcal6) or, with conschm 543, the upwind
// compact interface flux of convrsdcmp (src/solver.F90:1272-1938) without the characteristic
// decomposition: Steger-Warming splitting (src/riemann.F90:23-161) on the line's range, the
// compact flux of each split part (flux_uw/flux_dw, src/flux.F90:125-150), the MP limiter at
// every interface (shock = .true. with no Ducros sensor, crinod .false.), and the flux
// difference added to qrhs.
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "../../include/astr_b200.h"
#include "internal.h"
#include "tgv.cuh"

using namespace astr;

// Defined in capi.cu.
cudaStream_t astr_ctx_stream(astr_ctx* ctx);
int astr_ctx_device(astr_ctx* ctx);
void astr_ctx_set_error(astr_ctx* ctx, const char* msg);

namespace {

constexpr int HMW = 5;   // halo width of the reference's arrays (commvar.F90:190)

struct FsGeo {
  int N[3];
  int ntype[3];    // 3 periodic; 1, 2, 4 physical ends
  int64_t s[3];    // element strides of i, j, k (s[0] = 1)
  int64_t fs;      // elements per field
  double rd[3];    // dxi: 1/dx, 1/dy, 1/dz
  double jac;      // dx*dy*dz
  // element offset of node (i, j, k) from node (-hm, -hm, -hm)
  __host__ __device__ int64_t at(int i, int j, int k) const {
    return (int64_t)(i + HMW) + (int64_t)(j + HMW) * s[1] + (int64_t)(k + HMW) * s[2];
  }
  // Per-direction members by a runtime direction, as selects (an indexed read of a kernel
  // parameter's array would move the whole parameter into local memory).
  __host__ __device__ int n_(int d) const { return d == 0 ? N[0] : (d == 1 ? N[1] : N[2]); }
  __host__ __device__ int64_t s_(int d) const { return d == 0 ? s[0] : (d == 1 ? s[1] : s[2]); }
  __host__ __device__ double rd_(int d) const { return d == 0 ? rd[0] : (d == 1 ? rd[1] : rd[2]); }
};

// Coordinate d of node (i, j, k), as a select.
__host__ __device__ __forceinline__ int coord(int d, int i, int j, int k) { return d == 0 ? i : (d == 1 ? j : k); }

struct FsThermo {
  double const2, const5, const6, reynolds, prandtl, tc, tc1;
  double twall;    // isothermal no-slip walls at the physical ends
  double mach, gamma;
};

// Node (i, j, k) of the flat index p over the box [lo[a], hi[a]] on each axis.
struct Box3 {
  int lo[3], n[3];
  __host__ __device__ int64_t size() const { return (int64_t)n[0] * n[1] * n[2]; }
  __device__ void node(int64_t p, int& i, int& j, int& k) const {
    i = lo[0] + (int)(p % n[0]);
    const int64_t r = p / n[0];
    j = lo[1] + (int)(r % n[1]);
    k = lo[2] + (int)(r / n[1]);
  }
};

// The box of nodes 0..N on every axis except `dir`, where it spans [a, b] (dir < 0: none).
__host__ __device__ Box3 box_line(const FsGeo& g, int dir, int a, int b) {
  Box3 x;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    x.lo[d] = (d == dir) ? a : 0;
    x.n[d] = (d == dir) ? b - a + 1 : g.N[d] + 1;
  }
  return x;
}

#define GRID_STRIDE(p, total) \
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < (total); p += (int64_t)gridDim.x * blockDim.x)

// q2fvar (fludyna.F90:545-634, tgvsolver.F90:92-121) of one node
__device__ __forceinline__ void fs_q2fvar(const FsThermo& th, double q0, double q1, double q2, double q3, double q4,
                                          double& rho, double& u, double& v, double& w, double& p, double& t) {
  rho = q0;
  u = q1 / rho;
  v = q2 / rho;
  w = q3 / rho;
  p = (q4 - 0.5 * rho * (u * u + v * v + w * w)) / th.const6;
  t = p / rho * th.const2;
}

// Periodic halo copy along dir of nf fields (dataswap / bchomovec): F(-k) = F(N-k), F(N+k) = F(k),
// k = 1..hm, on the lines whose other indices lie in 0..N.
__global__ void k_fs_halo(double* F, int nf, int dir, FsGeo g) {
  const Box3 b = box_line(g, dir, 1, HMW);
  const int64_t total = b.size() * nf;
  const int N = g.n_(dir);
  const int64_t sd = g.s_(dir);
  GRID_STRIDE(p, total) {
    const int m = (int)(p / b.size());
    int i, j, k;
    b.node(p - (int64_t)m * b.size(), i, j, k);
    const int kk = coord(dir, i, j, k);   // 1..hm
    double* f = F + m * g.fs + g.at(i, j, k) - (int64_t)kk * sd;   // node 0 of the line
    f[-(int64_t)kk * sd] = f[(int64_t)(N - kk) * sd];
    f[(int64_t)(N + kk) * sd] = f[(int64_t)kk * sd];
  }
}

// qswap along dir (parallel.F90:4877-5060), first part: per line and field, the halo copy of q
// (thread kk = 1..hm: q(-kk) = q(N-kk), q(N+kk) = q(kk)) and the average of nodes 0 and N (thread
// kk = 0). The copies read nodes 1..hm and N-hm..N-1 only, which no thread writes.
__global__ void k_fs_qswap(double* q, int dir, FsGeo g) {
  const Box3 b = box_line(g, dir, 0, 0);
  const int N = g.n_(dir);
  const int64_t sd = g.s_(dir);
  const int64_t per_line = 5 * (HMW + 1);
  GRID_STRIDE(p, b.size() * per_line) {
    const int64_t line = p / per_line;
    const int r = (int)(p - line * per_line);
    const int m = r / (HMW + 1), kk = r - m * (HMW + 1);
    int i, j, k;
    b.node(line, i, j, k);
    double* f = q + m * g.fs + g.at(i, j, k);   // node 0 of the line
    if (kk == 0) {
      const double avg = 0.5 * (f[0] + f[(int64_t)N * sd]);
      f[0] = avg;
      f[(int64_t)N * sd] = avg;
    } else {
      f[-kk * sd] = f[(int64_t)(N - kk) * sd];
      f[(int64_t)(N + kk) * sd] = f[(int64_t)kk * sd];
    }
  }
}

// qswap, second part: q2fvar on the nodes -hm..0 and N..N+hm of every line along dir.
__global__ void k_fs_qswap_prims(const double* q, double* rho, double* vel, double* prs, double* tmp, int dir,
                                 FsGeo g, FsThermo th) {
  const Box3 b = box_line(g, dir, 0, 0);
  const int N = g.n_(dir);
  const int64_t sd = g.s_(dir);
  const int per_line = 2 * (HMW + 1);
  GRID_STRIDE(p, b.size() * per_line) {
    const int64_t line = p / per_line;
    const int r = (int)(p - line * per_line);
    const int t = r <= HMW ? r - HMW : N + (r - HMW - 1);   // -hm..0, then N..N+hm
    int i, j, k;
    b.node(line, i, j, k);
    const int64_t o = g.at(i, j, k) + (int64_t)t * sd;
    double rr, u, v, w, pr, tt;
    fs_q2fvar(th, q[o], q[g.fs + o], q[2 * g.fs + o], q[3 * g.fs + o], q[4 * g.fs + o], rr, u, v, w, pr, tt);
    rho[o] = rr; vel[o] = u; vel[g.fs + o] = v; vel[2 * g.fs + o] = w; prs[o] = pr; tmp[o] = tt;
  }
}

// boucon with isothermal no-slip walls (bctype 41, noslip, src/bc.F90:6281-6595) on the end
// `side` (0: node 0, 1: node N) along dir: u = v = w = 0, T = twall, p = (4 p_1 - p_2)/3 from the
// two nodes next to the wall, rho = p/T gamma M^2 (thermal), q by fvar2q.
__global__ void k_fs_noslip(double* q, double* rho, double* vel, double* prs, double* tmp, int dir, int side, FsGeo g,
                            FsThermo th) {
  const int N = g.n_(dir);
  const Box3 b = box_line(g, dir, side ? N : 0, side ? N : 0);
  const int64_t sd = g.s_(dir) * (side ? -1 : 1);   // towards the interior
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    const double pe = (1.0 / 3.0) * (4.0 * prs[o + sd] - prs[o + 2 * sd]);
    vel[o] = 0.0; vel[g.fs + o] = 0.0; vel[2 * g.fs + o] = 0.0;
    prs[o] = pe;
    tmp[o] = th.twall;
    const double r = pe / th.twall * th.const2;
    rho[o] = r;
    q[o] = r;
    q[g.fs + o] = r * 0.0; q[2 * g.fs + o] = r * 0.0; q[3 * g.fs + o] = r * 0.0;
    q[4 * g.fs + o] = pe * th.const6 + r * 0.0;   // fvar2q with |u|^2 = 0
  }
}

// convrsdcal6's fluxes along dir at nodes -hm..N+hm (solver.F90:2201-2207): uu = dxi u_dir,
// fcs1 = jacob q1 uu, fcs(1+m) = jacob (q(1+m) uu + dxi p delta(m,dir)), fcs5 = jacob (q5 + p) uu.
__global__ void k_fs_conv_flux(double* F, const double* q, const double* vel, const double* prs, int dir, FsGeo g) {
  const Box3 b = box_line(g, dir, -HMW, g.n_(dir) + HMW);
  const double dxi = g.rd_(dir), jb = g.jac;
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    const double uu = dxi * vel[dir * g.fs + o];
    const double pr = prs[o];
    F[o] = jb * q[o] * uu;
#pragma unroll
    for (int m = 1; m <= 3; ++m) {
      const double qm = q[m * g.fs + o];
      F[m * g.fs + o] = (m - 1 == dir) ? jb * (qm * uu + dxi * pr) : jb * (qm * uu);
    }
    F[4 * g.fs + o] = jb * (q[4 * g.fs + o] + pr) * uu;
  }
}

// The full flux jacob (q uu + dxi p e_dir, (E + p) uu) of a supersonic node (one side of the split).
__device__ __forceinline__ void fs_sw_full(double (&f)[5], int dir, double dxi, double jb, double uu, double p,
                                           const double (&qq)[5]) {
  f[0] = jb * qq[0] * uu;
#pragma unroll
  for (int c = 0; c < 3; ++c) f[1 + c] = (c == dir) ? jb * (qq[1 + c] * uu + dxi * p) : jb * (qq[1 + c] * uu);
  f[4] = jb * (qq[4] + p) * uu;
}
// One side of the subsonic split from its eigenvalue weights l1 (= l2 = l3), l4, l5.
__device__ __forceinline__ void fs_sw_side(double (&f)[5], const FsThermo& th, int dir, double jb, double jro, double r,
                                           double l1, double l4, double l5, const double (&u)[3], double uu,
                                           double var0, double css, double gpd, double gm2, double fhi, double q4) {
  const double var1 = l1;
  const double var2 = l4 - l5;
  const double var3 = 2.0 * l1 - l4 - l5;
  const double var4 = var1 - var3 * gm2;
  f[0] = jro * var4;
#pragma unroll
  for (int c = 0; c < 3; ++c) f[1 + c] = (c == dir) ? jro * (var4 * u[c] + var2 * css * gpd * gm2) : jro * (var4 * u[c]);
  f[4] = jb * (var1 * q4 + r * (var2 * uu * var0 * css * gm2 - var3 * (fhi + css * css) * gm2 / (th.gamma - 1.0)));
}

// flux_steger_warming of one node (riemann.F90:23-161, non-reacting) for the metric row
// dxi e_dir: uu = dxi u_dir, the sound speed sqrt(T)/M (sos, fludyna.F90:832-859), eigenvalues
// (uu, uu, uu, uu + c dxi, uu - c dxi) split with the entropy fix eps = 0.04. The operations
// follow the reference's order with the zero metric components left out (they add zeros).
__device__ __forceinline__ void fs_sw_split(const FsThermo& th, int dir, double dxi, double jb, double r,
                                            const double (&u)[3], double p, double t, const double (&qq)[5],
                                            double (&fp)[5], double (&fm)[5]) {
  const double eps = 0.04;
  const double ud = dir == 0 ? u[0] : (dir == 1 ? u[1] : u[2]);
  const double uu = dxi * ud;
  const double var0 = 1.0 / sqrt(dxi * dxi);
  const double gpd = dxi * var0;                 // the dir component; the others are zero
  const double gm2 = 0.5 / th.gamma;
  const double css = sqrt(t) / th.mach;
  const double csa = css / var0;
  const double lmach = uu / csa;
  if (lmach >= 1.0) {
    fs_sw_full(fp, dir, dxi, jb, uu, p, qq);
#pragma unroll
    for (int k = 0; k < 5; ++k) fm[k] = 0.0;
    return;
  }
  if (lmach <= -1.0) {
    fs_sw_full(fm, dir, dxi, jb, uu, p, qq);
#pragma unroll
    for (int k = 0; k < 5; ++k) fp[k] = 0.0;
    return;
  }
  const double l4 = uu + csa, l5 = uu - csa;
  const double p1 = 0.5 * (uu + sqrt(uu * uu + eps * eps));
  const double p4 = 0.5 * (l4 + sqrt(l4 * l4 + eps * eps));
  const double p5 = 0.5 * (l5 + sqrt(l5 * l5 + eps * eps));
  const double fhi = 0.5 * (th.gamma - 1.0) * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  const double jro = jb * r;
  fs_sw_side(fp, th, dir, jb, jro, r, p1, p4, p5, u, uu, var0, css, gpd, gm2, fhi, qq[4]);
  fs_sw_side(fm, th, dir, jb, jro, r, uu - p1, l4 - p4, l5 - p5, u, uu, var0, css, gpd, gm2, fhi, qq[4]);
}

// The split fluxes along dir on the nodes iss..iee of every line (solver.F90:1333-1345); the
// rest of the line stays zero (never read).
__global__ void k_fs_sw_split(double* fsp, double* fsm, const double* q, const double* rho, const double* vel,
                              const double* prs, const double* tmp, int dir, int iss, int iee, FsGeo g, FsThermo th) {
  const Box3 b = box_line(g, dir, iss, iee);
  const double dxi = g.rd_(dir), jb = g.jac;
  const int64_t fs = g.fs;
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    const double u[3] = {vel[o], vel[fs + o], vel[2 * fs + o]};
    const double qq[5] = {q[o], q[fs + o], q[2 * fs + o], q[3 * fs + o], q[4 * fs + o]};
    double fp[5], fm[5];
    fs_sw_split(th, dir, dxi, jb, rho[o], u, prs[o], tmp[o], qq, fp, fm);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      fsp[m * fs + o] = fp[m];
      fsm[m * fs + o] = fm[m];
    }
  }
}

__device__ __forceinline__ double fs_minmod2(double a, double b) {   // commfunc.F90:699-714
  if (a > 0.0 && b > 0.0) return fmin(fabs(a), fabs(b));
  if (a < 0.0 && b < 0.0) return -1.0 * fmin(fabs(a), fabs(b));
  return 0.0;
}
__device__ __forceinline__ double fs_minmod4(double a, double b, double c, double d) {   // commfunc.F90:722-738
  if (a > 0.0 && b > 0.0 && c > 0.0 && d > 0.0) return fmin(fmin(fmin(fabs(a), fabs(b)), fabs(c)), fabs(d));
  if (a < 0.0 && b < 0.0 && c < 0.0 && d < 0.0) return -1.0 * fmin(fmin(fmin(fabs(a), fabs(b)), fabs(c)), fabs(d));
  return 0.0;
}
// MP5 with the compact value as the linear value (flux.F90:434-496); no limiting unless
// discont (the shock flag) is set
__device__ __forceinline__ double fs_mp5(const double* u, double ul, bool discont) {
  double var1 = u[3] - u[2];
  double var2 = 4.0 * (u[2] - u[1]);
  const double ump = u[2] + fs_minmod2(var1, var2);
  var1 = (ul - u[2]) * (ul - ump);
  if (!(discont && var1 >= 1.0e-10)) return ul;
  const double dm1 = u[0] - 2.0 * u[1] + u[2];
  const double d0 = u[1] - 2.0 * u[2] + u[3];
  const double d1 = u[2] - 2.0 * u[3] + u[4];
  const double dhm1 = fs_minmod4(4.0 * dm1 - d0, 4.0 * d0 - dm1, dm1, d0);
  const double dh0 = fs_minmod4(4.0 * d0 - d1, 4.0 * d1 - d0, d0, d1);
  const double uul = u[2] + 4.0 * (u[2] - u[1]);
  const double uav = 0.5 * (u[2] + u[3]);
  const double umd = uav - 0.5 * dh0;
  const double ulc = u[2] + 0.5 * (u[2] - u[1]) + 1.333333333333333 * dhm1;
  const double umin = fmax(fmin(fmin(u[2], u[3]), umd), fmin(fmin(u[2], uul), ulc));
  const double umax = fmin(fmax(fmax(u[2], u[3]), umd), fmax(fmax(u[2], uul), ulc));
  return ul + fs_minmod2(umin - ul, umax - ul);
}
// mplimiter (flux.F90:363-379): the compact value at the two interfaces next to a block's
// physical end for ntype 1 or 2 only, MP5 elsewhere.
__device__ __forceinline__ double fs_mplimiter(const double* f, double fl, bool shock, int inode, int dim, int nt) {
  if ((nt == 1 && (inode == 0 || inode == 1)) || (nt == 2 && (inode == dim - 1 || inode == dim - 2))) return fl;
  return fs_mp5(f, fl, shock);
}

// Interface flux Fh(i) = mplimiter(+) + mplimiter(-) of field m at interface i of the line whose
// node 0 is at o0 (solver.F90:1423-1478 with no characteristic decomposition): the stencils of
// iwind6 (solver.F90:1237-1258), clamped to iss..iee.
__device__ __forceinline__ double fs_interface(const double* fsp, const double* fsm, const double* fhp,
                                               const double* fhm, int64_t o0, int64_t sd, int i, int dim, int nt,
                                               int iss, int iee) {
  double up[5], um[5];
#pragma unroll
  for (int n = 1; n <= 5; ++n) {
    const int jp = min(max(i + n - 3, iss), iee);
    const int jm = min(max(i + 4 - n, iss), iee);
    up[n - 1] = fsp[o0 + (int64_t)jp * sd];
    um[n - 1] = fsm[o0 + (int64_t)jm * sd];
  }
  const double v1 = fs_mplimiter(up, fhp[o0 + (int64_t)i * sd], true, i, dim, nt);
  const double v2 = fs_mplimiter(um, fhm[o0 + (int64_t)i * sd], true, i, dim, nt);
  return v1 + v2;
}

// chardecomp (solver.F90:1959-2163, non-reacting) of the interface between nodes a and b along
// the metric row m: the Roe-averaged right (R) and left (L) eigenvectors, R[row][col].
__device__ __forceinline__ void fs_chardecomp(const FsThermo& th, double rl, double pl, double el, const double* vl,
                                              double rr, double pr, double er, const double* vr, const double* m,
                                              double (&R)[5][5], double (&L)[5][5]) {
  const double gamma = th.gamma;
  const double wroe = sqrt(rl) / (sqrt(rl) + sqrt(rr));
  const double wroe1 = 1.0 - wroe;
  const double u1 = wroe * vl[0] + wroe1 * vr[0];
  const double u2 = wroe * vl[1] + wroe1 * vr[1];
  const double u3 = wroe * vl[2] + wroe1 * vr[2];
  const double kroe = 0.5 * (u1 * u1 + u2 * u2 + u3 * u3);
  const double hl = (el + pl) / rl;
  const double hr = (er + pr) / rr;
  const double hroe = wroe * hl + wroe1 * hr;
  const double css = sqrt((gamma - 1.0) * (hroe - kroe));
  const double rcs = 1.0 / css;
  const double var1 = 0.5 * (m[0] + m[0]), var2 = 0.5 * (m[1] + m[1]), var3 = 0.5 * (m[2] + m[2]);
  const double var4 = 1.0 / sqrt(var1 * var1 + var2 * var2 + var3 * var3);
  const double g1 = var1 * var4, g2 = var2 * var4, g3 = var3 * var4;
  const double ugp = u1 * g1 + u2 * g2 + u3 * g3;
  const double b1 = (gamma - 1.0) / (css * css);
  const double b2 = 1.0 + 2.0 * b1 * kroe - b1 * hroe;
  L[0][0] = 0.5 * (b2 + ugp * rcs);
  L[0][1] = -0.5 * (b1 * u1 + g1 * rcs);
  L[0][2] = -0.5 * (b1 * u2 + g2 * rcs);
  L[0][3] = -0.5 * (b1 * u3 + g3 * rcs);
  L[0][4] = 0.5 * b1;
  R[0][0] = 1.0; R[1][0] = u1 - css * g1; R[2][0] = u2 - css * g2; R[3][0] = u3 - css * g3; R[4][0] = hroe - ugp * css;
  L[1][0] = 1.0 - b2; L[1][1] = b1 * u1; L[1][2] = b1 * u2; L[1][3] = b1 * u3; L[1][4] = -b1;
  R[0][1] = 1.0; R[1][1] = u1; R[2][1] = u2; R[3][1] = u3; R[4][1] = hroe - 1.0 / b1;
  if (fabs(var1) > 1.0e-12) {
    const double rgp = 1.0 / g1;
    L[2][0] = (ugp * g2 - u2) * rgp; L[2][1] = -g2; L[2][2] = (1.0 - g2 * g2) * rgp; L[2][3] = -g2 * g3 * rgp; L[2][4] = 0.0;
    L[3][0] = (ugp * g3 - u3) * rgp; L[3][1] = -g3; L[3][2] = -g2 * g3 * rgp; L[3][3] = (1.0 - g3 * g3) * rgp; L[3][4] = 0.0;
    R[0][2] = 0.0; R[1][2] = -g2; R[2][2] = g1; R[3][2] = 0.0; R[4][2] = u2 * g1 - u1 * g2;
    R[0][3] = 0.0; R[1][3] = -g3; R[2][3] = 0.0; R[3][3] = g1; R[4][3] = u3 * g1 - u1 * g3;
  } else if (fabs(var2) > 1.0e-12) {
    const double rgp = 1.0 / g2;
    L[2][0] = (ugp * g1 - u1) * rgp; L[2][1] = (1.0 - g1 * g1) * rgp; L[2][2] = -g1; L[2][3] = -g1 * g3 * rgp; L[2][4] = 0.0;
    L[3][0] = (ugp * g3 - u3) * rgp; L[3][1] = -g1 * g3 * rgp; L[3][2] = -g3; L[3][3] = (1.0 - g3 * g3) * rgp; L[3][4] = 0.0;
    R[0][2] = 0.0; R[1][2] = g2; R[2][2] = -g1; R[3][2] = 0.0; R[4][2] = u1 * g2 - u2 * g1;
    R[0][3] = 0.0; R[1][3] = 0.0; R[2][3] = -g3; R[3][3] = g2; R[4][3] = u3 * g2 - u2 * g3;
  } else {
    const double rgp = 1.0 / g3;
    L[2][0] = (ugp * g1 - u1) * rgp; L[2][1] = (1.0 - g1 * g1) * rgp; L[2][2] = -g1 * g2 * rgp; L[2][3] = -g1; L[2][4] = 0.0;
    L[3][0] = (ugp * g2 - u2) * rgp; L[3][1] = -g1 * g2 * rgp; L[3][2] = (1.0 - g2 * g2) * rgp; L[3][3] = -g2; L[3][4] = 0.0;
    R[0][2] = 0.0; R[1][2] = g3; R[2][2] = 0.0; R[3][2] = -g1; R[4][2] = u1 * g3 - u3 * g1;
    R[0][3] = 0.0; R[1][3] = 0.0; R[2][3] = g3; R[3][3] = -g2; R[4][3] = u2 * g3 - u3 * g2;
  }
  L[4][0] = 0.5 * (b2 - ugp * rcs);
  L[4][1] = -0.5 * (b1 * u1 - g1 * rcs);
  L[4][2] = -0.5 * (b1 * u2 - g2 * rcs);
  L[4][3] = -0.5 * (b1 * u3 - g3 * rcs);
  L[4][4] = 0.5 * b1;
  R[0][4] = 1.0; R[1][4] = u1 + css * g1; R[2][4] = u2 + css * g2; R[3][4] = u3 + css * g3; R[4][4] = hroe + ugp * css;
}

// ducrossensor, first part (commcal.F90:224-269): ssf on nodes 0..N from the velocity gradients
// (dvel field n + 3d = du_n/dx_d) and the normalised second differences of p; neighbours clamped
// at physical ends for ntype 1 (low) and 2 (high) only, as the reference does.
__global__ void k_fs_ssf(double* ssf, const double* dvel, const double* prs, FsGeo g) {
  const Box3 b = box_line(g, -1, 0, 0);
  const int64_t fs = g.fs;
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    const double div = dvel[o] + dvel[4 * fs + o] + dvel[8 * fs + o];
    const double div2 = div * div;
    const double vx = dvel[5 * fs + o] - dvel[7 * fs + o];
    const double vy = dvel[6 * fs + o] - dvel[2 * fs + o];
    const double vz = dvel[1 * fs + o] - dvel[3 * fs + o];
    const double vort = vx * vx + vy * vy + vz * vz;
    const int idx[3] = {i, j, k};
    double dmax = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int lo = -1, hi = 1;
      if (g.ntype[d] == 1 && idx[d] - 1 < 0) lo = 0;
      if (g.ntype[d] == 2 && idx[d] + 1 > g.N[d]) hi = 0;
      const double p0 = prs[o], pp = prs[o + hi * g.s[d]], pm = prs[o + lo * g.s[d]];
      const double dd = fabs(pp - 2.0 * p0 + pm) / (pp + 2.0 * p0 + pm);
      dmax = d == 0 ? dd : fmax(dmax, dd);
    }
    ssf[o] = div2 / (div2 + vort + 1.0e-30) * dmax;
  }
}

// ducrossensor, second part (commcal.F90:273-318): lshock (1 or 0) on nodes 0..N, the largest ssf
// over the 10-node stencils i-4..i+5 along each axis above shkcrt.
__global__ void k_fs_lshock(double* lsh, const double* ssf, double shkcrt, FsGeo g) {
  const Box3 b = box_line(g, -1, 0, 0);
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    const int idx[3] = {i, j, k};
    double mx = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      for (int off = -HMW + 1; off <= HMW; ++off) {
        int t = idx[d] + off;
        if (g.ntype[d] == 1 && t < 0) t = 0;
        if (g.ntype[d] == 2 && t > g.N[d]) t = g.N[d];
        mx = fmax(mx, ssf[o + (int64_t)(t - idx[d]) * g.s[d]]);
      }
    lsh[o] = mx > shkcrt ? 1.0 : 0.0;
  }
}

// Interface fluxes of convrsdcmp with the characteristic decomposition (solver.F90:1359-1495):
// one thread per interface i = -1..N of a line, all five components: the split fluxes of the
// iwind6 stencils and the compact fluxes projected on the left eigenvectors, the MP limiter in
// characteristic variables with the interface's shock flag, back by the right eigenvectors.
// Fh(i) is stored at node i of the layout (work fields).
__global__ void k_fs_char_flux(double* Fh, const double* fsp, const double* fsm, const double* fhp, const double* fhm,
                               const double* q, const double* rho, const double* vel, const double* prs,
                               const double* lsh, int dir, int nt, int iss, int iee, FsGeo g, FsThermo th) {
  const int N = g.n_(dir);
  const Box3 b = box_line(g, dir, -1, N);
  const int64_t sd = g.s_(dir), fs = g.fs;
  const double mrow[3] = {dir == 0 ? g.rd[0] : 0.0, dir == 1 ? g.rd[1] : 0.0, dir == 2 ? g.rd[2] : 0.0};
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int t = dir == 0 ? i : (dir == 1 ? j : k);
    const int64_t oa = g.at(i, j, k), ob = oa + sd;
    const int64_t o0 = oa - (int64_t)t * sd;
    bool shock;
    if (t < 0) shock = lsh[ob] != 0.0;
    else if (t + 1 > N) shock = lsh[oa] != 0.0;
    else shock = lsh[oa] != 0.0 || lsh[ob] != 0.0;
    const double vl[3] = {vel[oa], vel[fs + oa], vel[2 * fs + oa]};
    const double vr[3] = {vel[ob], vel[fs + ob], vel[2 * fs + ob]};
    double R[5][5], L[5][5];
    fs_chardecomp(th, rho[oa], prs[oa], q[4 * fs + oa], vl, rho[ob], prs[ob], q[4 * fs + ob], vr, mrow, R, L);
    int64_t jp[5], jn[5];
#pragma unroll
    for (int n = 1; n <= 5; ++n) {
      jp[n - 1] = o0 + (int64_t)min(max(t + n - 3, iss), iee) * sd;
      jn[n - 1] = o0 + (int64_t)min(max(t + 4 - n, iss), iee) * sd;
    }
    double fhc[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      double up[5], um[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        up[n] = L[m][0] * fsp[jp[n]] + L[m][1] * fsp[fs + jp[n]] + L[m][2] * fsp[2 * fs + jp[n]] +
                L[m][3] * fsp[3 * fs + jp[n]] + L[m][4] * fsp[4 * fs + jp[n]];
        um[n] = L[m][0] * fsm[jn[n]] + L[m][1] * fsm[fs + jn[n]] + L[m][2] * fsm[2 * fs + jn[n]] +
                L[m][3] * fsm[3 * fs + jn[n]] + L[m][4] * fsm[4 * fs + jn[n]];
      }
      const double hp = L[m][0] * fhp[oa] + L[m][1] * fhp[fs + oa] + L[m][2] * fhp[2 * fs + oa] +
                        L[m][3] * fhp[3 * fs + oa] + L[m][4] * fhp[4 * fs + oa];
      const double hm = L[m][0] * fhm[oa] + L[m][1] * fhm[fs + oa] + L[m][2] * fhm[2 * fs + oa] +
                        L[m][3] * fhm[3 * fs + oa] + L[m][4] * fhm[4 * fs + oa];
      fhc[m] = fs_mplimiter(up, hp, shock, t, N, nt) + fs_mplimiter(um, hm, shock, t, N, nt);
    }
#pragma unroll
    for (int m = 0; m < 5; ++m)
      Fh[m * fs + oa] = R[m][0] * fhc[0] + R[m][1] * fhc[1] + R[m][2] * fhc[2] + R[m][3] * fhc[3] + R[m][4] * fhc[4];
  }
}

// qrhs(i) = qrhs(i) + Fh(i) - Fh(i-1) at nodes 0..N, Fh stored per interface (solver.F90:1509-1513),
// kept negated: rhscal negates qrhs after the convection (qrhs = -qrhs, solver.F90:243), and with
// q holding -qrhs, (q - Fh(i)) + Fh(i-1) is -((qrhs + Fh(i)) - Fh(i-1)) exactly.
__global__ void k_fs_flux_diff(double* qrhs, const double* Fh, int dir, FsGeo g) {
  const Box3 b = box_line(g, -1, 0, 0);
  const int64_t sd = g.s_(dir);
  GRID_STRIDE(p, b.size() * 5) {
    const int m = (int)(p / b.size());
    int i, j, k;
    b.node(p - (int64_t)m * b.size(), i, j, k);
    const int64_t o = m * g.fs + g.at(i, j, k);
    qrhs[o] = (qrhs[o] - Fh[o]) + Fh[o - sd];
  }
}

// Interface fluxes without the characteristic decomposition (solver.F90:1423-1478): one thread
// per interface i = -1..N of a line and field, Fh(i) = mplimiter(+) + mplimiter(-) with shock =
// .true., stored at node i of the layout (work fields).
__global__ void k_fs_mp_flux(double* Fh, const double* fsp, const double* fsm, const double* fhp, const double* fhm,
                             int dir, int nt, int iss, int iee, FsGeo g) {
  const int N = g.n_(dir);
  const Box3 b = box_line(g, dir, -1, N);
  const int64_t sd = g.s_(dir);
  GRID_STRIDE(p, b.size() * 5) {
    const int m = (int)(p / b.size());
    int i, j, k;
    b.node(p - (int64_t)m * b.size(), i, j, k);
    const int t = dir == 0 ? i : (dir == 1 ? j : k);
    const int64_t o = m * g.fs + g.at(i, j, k);
    Fh[o] = fs_interface(fsp, fsm, fhp, fhm, o - (int64_t)t * sd, sd, t, N, nt, iss, iee);
  }
}

// diffrsdcal6's pointwise part at nodes 0..N (solver.F90:2458-2546): Sutherland viscosity, the
// viscous stress and the heat flux.
__global__ void k_fs_stress(double* sigma, double* qflux, const double* dvel, const double* dtmp, const double* vel,
                            const double* tmp, FsGeo g, FsThermo th) {
  const Box3 b = box_line(g, -1, 0, 0);
  const int64_t fs = g.fs;
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    // dvel(:,:,:,n,d) is field 3d + n
    const double s11 = dvel[0 * fs + o];
    const double s12 = 0.5 * (dvel[3 * fs + o] + dvel[1 * fs + o]);
    const double s13 = 0.5 * (dvel[6 * fs + o] + dvel[2 * fs + o]);
    const double s22 = dvel[4 * fs + o];
    const double s23 = 0.5 * (dvel[7 * fs + o] + dvel[5 * fs + o]);
    const double s33 = dvel[8 * fs + o];
    const double skk = (1.0 / 3.0) * (s11 + s22 + s33);
    const double t = tmp[o];
    const double miu = t * sqrt(t) * th.tc1 / (t + th.tc) / th.reynolds;
    const double miu2 = 2.0 * miu;
    const double hcc = (miu / th.prandtl) / th.const5;
    const double sg0 = miu2 * (s11 - skk), sg1 = miu2 * s12, sg2 = miu2 * s13;
    const double sg3 = miu2 * (s22 - skk), sg4 = miu2 * s23, sg5 = miu2 * (s33 - skk);
    sigma[o] = sg0; sigma[fs + o] = sg1; sigma[2 * fs + o] = sg2;
    sigma[3 * fs + o] = sg3; sigma[4 * fs + o] = sg4; sigma[5 * fs + o] = sg5;
    const double u = vel[o], v = vel[fs + o], w = vel[2 * fs + o];
    qflux[o] = hcc * dtmp[o] + sg0 * u + sg1 * v + sg2 * w;
    qflux[fs + o] = hcc * dtmp[fs + o] + sg1 * u + sg3 * v + sg4 * w;
    qflux[2 * fs + o] = hcc * dtmp[2 * fs + o] + sg2 * u + sg4 * v + sg5 * w;
  }
}

// diffrsdcal6's fluxes along dir at nodes -hm..N+hm (solver.F90:2622-2640):
// ff = (sigma(row dir) . dxi) * jacob for the momenta, (qflux . dxi) * jacob for the energy.
__global__ void k_fs_visc_flux(double* F, const double* sigma, const double* qflux, int dir, FsGeo g) {
  const Box3 b = box_line(g, dir, -HMW, g.n_(dir) + HMW);
  const double dxi = g.rd_(dir), jb = g.jac;
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      // sigma(dir, n) in the symmetric storage 11 12 13 22 23 33
      const int lo = min(dir, n), hi = max(dir, n);
      const int sg = lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
      F[n * g.fs + o] = sigma[sg * g.fs + o] * dxi * jb;
    }
    F[3 * g.fs + o] = qflux[dir * g.fs + o] * dxi * jb;
  }
}

// The rk3 update of q*jacob (mainloop.F90:426-446); at the first stage qsave = q*jacob first.
__global__ void k_fs_update(double* q, double* qsave, const double* qrhs, double c1, double c2, double c3, double dt,
                            int first, FsGeo g) {
  const Box3 b = box_line(g, -1, 0, 0);
  const double jb = g.jac;
  GRID_STRIDE(p, b.size() * 5) {
    const int m = (int)(p / b.size());
    int i, j, k;
    b.node(p - (int64_t)m * b.size(), i, j, k);
    const int64_t o = m * g.fs + g.at(i, j, k);
    if (first) qsave[o] = q[o] * jb;
    const double v = c1 * qsave[o] + c2 * q[o] * jb + c3 * qrhs[o] * dt;
    q[o] = v / jb;
  }
}

// updatefvar on nodes 0..N (fludyna.F90:191-242)
__global__ void k_fs_prims(const double* q, double* rho, double* vel, double* prs, double* tmp, FsGeo g, FsThermo th) {
  const Box3 b = box_line(g, -1, 0, 0);
  const int64_t fs = g.fs;
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    double r, u, v, w, pr, t;
    fs_q2fvar(th, q[o], q[fs + o], q[2 * fs + o], q[3 * fs + o], q[4 * fs + o], r, u, v, w, pr, t);
    rho[o] = r; vel[o] = u; vel[fs + o] = v; vel[2 * fs + o] = w; prs[o] = pr; tmp[o] = t;
  }
}

// stacal / diss_rate_cal terms summed over nodes 1..N, per CTA (tgvsolver.F90:913-931,
// statistic.F90:1009-1034); the ordered final reduction is k_diag_reduce.
__global__ void k_fs_diag(double* partials, const double* rho, const double* vel, const double* dvel,
                          const double* tmp, FsGeo g, FsThermo th) {
  Box3 b;
  for (int d = 0; d < 3; ++d) { b.lo[d] = 1; b.n[d] = g.N[d]; }
  const int64_t fs = g.fs;
  double ke = 0.0, en = 0.0, di = 0.0;
  GRID_STRIDE(p, b.size()) {
    int i, j, k;
    b.node(p, i, j, k);
    const int64_t o = g.at(i, j, k);
    const double u = vel[o], v = vel[fs + o], w = vel[2 * fs + o], r = rho[o];
    ke += r * (u * u + v * v + w * w);
    const double om1 = dvel[5 * fs + o] - dvel[7 * fs + o];
    const double om2 = dvel[6 * fs + o] - dvel[2 * fs + o];
    const double om3 = dvel[1 * fs + o] - dvel[3 * fs + o];
    en += r * (om1 * om1 + om2 * om2 + om3 * om3);
    const double t = tmp[o];
    const double miu = t * sqrt(t) * th.tc1 / (t + th.tc) / th.reynolds;
    const double s11 = dvel[o], s12 = 0.5 * (dvel[3 * fs + o] + dvel[1 * fs + o]);
    const double s13 = 0.5 * (dvel[6 * fs + o] + dvel[2 * fs + o]);
    const double s22 = dvel[4 * fs + o], s23 = 0.5 * (dvel[7 * fs + o] + dvel[5 * fs + o]), s33 = dvel[8 * fs + o];
    const double div = s11 + s22 + s33;
    di += 2.0 * miu * (s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23) -
                       (1.0 / 3.0) * (div * div));
  }
  __shared__ double s[3][256];
  s[0][threadIdx.x] = ke; s[1][threadIdx.x] = en; s[2][threadIdx.x] = di;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int c = 0; c < 3; ++c) s[c][threadIdx.x] += s[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) partials[3 * blockIdx.x + c] = s[c][0];
}

// Copy between the caller's Fortran array (nodes 0..N inside it) and nodes 0..N of the layout,
// nf fields.
__global__ void k_fs_pack(double* state, double* user, FsGeo g, int64_t u0, int64_t u1, int64_t u2, int64_t ufs,
                          int64_t uoff, int to_state, int nf) {
  const Box3 b = box_line(g, -1, 0, 0);
  GRID_STRIDE(p, b.size() * nf) {
    const int m = (int)(p / b.size());
    int i, j, k;
    b.node(p - (int64_t)m * b.size(), i, j, k);
    const int64_t os = m * g.fs + g.at(i, j, k);
    const int64_t ou = uoff + m * ufs + i * u0 + j * u1 + k * u2;
    if (to_state) state[os] = user[ou];
    else user[ou] = state[os];
  }
}

unsigned blocks_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = 148 * 16;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

struct astr_full {
  astr_ctx* ctx = nullptr;
  astr_params p{};
  FsGeo g{};
  FsThermo th{};
  double* buf = nullptr;
  double *q = nullptr, *qt = nullptr, *rho = nullptr, *vel = nullptr, *prs = nullptr, *tmp = nullptr;
  double *qsave = nullptr, *qrhs = nullptr, *dvel = nullptr, *dtmp = nullptr, *sigma = nullptr, *qflux = nullptr;
  double* work = nullptr;   // flux lines of one direction (5 fields)
  double* up = nullptr;     // upwind convection: split fluxes f+ f-, their compact fluxes, ssf, lshock (22)
  double* partials = nullptr;
  int nparts = 0;
  double* hist = nullptr;
  int* counter = nullptr;
  int hist_cap = 1 << 16;
  HostOp hd[3], hf[3], hfu[3], hfd[3];
  DevOp dd[3], df[3], dfu[3], dfd[3];
  int nstep = 0;
  double time = 0.0;
  std::vector<double> row_key;
};

namespace {

int ffail(astr_full* f, int code, const std::string& msg) {
  if (f && f->ctx) astr_ctx_set_error(f->ctx, msg.c_str());
  return code;
}
#define FCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return ffail(fs, ASTR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct OnDev {
  int prev = -1;
  explicit OnDev(int dev) {
    int cur = -1;
    if (dev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
  }
  ~OnDev() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Line-operator view of a field of the layout: the full range -hm..N+hm along `full` (or none
// when full < 0), nodes 0..N on the other axes. Returns the pointer the descriptor is relative to.
double* view(const astr_full* fs, double* base, int full, ArrDesc& a) {
  int64_t off = 0;
  for (int d = 0; d < 3; ++d) {
    a.s[d] = fs->g.s[d];
    if (d == full) { a.lb[d] = -HMW; a.n[d] = fs->g.N[d] + 1 + 2 * HMW; }
    else { a.lb[d] = 0; a.n[d] = fs->g.N[d] + 1; off += HMW * fs->g.s[d]; }
  }
  a.fs = fs->g.fs;
  return base + off;
}

// out (nodes 0..N) [+]= scale * op(in) along dir for nf fields
cudaError_t line_op(astr_full* fs, const DevOp& op, int dir, double* in, double* out, int nf, double scale, int add) {
  ArrDesc fa, oa;
  double* fp = view(fs, in, dir, fa);
  double* op_ = view(fs, out, -1, oa);
  return launch_line_api(op, dir, fp, fa, op_, oa, nf, scale, astr_ctx_stream(fs->ctx), add);
}

// fh (interfaces -1..N along dir, nodes 0..N elsewhere) = the compact flux of in along dir
cudaError_t flux_op(astr_full* fs, const DevOp& op, int dir, double* in, double* out, int nf) {
  ArrDesc fa, oa;
  double* fp = view(fs, in, dir, fa);
  double* op_ = view(fs, out, -1, oa);
  oa.lb[dir] = -1;
  oa.n[dir] = fs->g.n_(dir) + 2;
  op_ -= fs->g.s_(dir);   // the descriptor is relative to node -1 along dir
  return launch_line_api(op, dir, fp, fa, op_, oa, nf, 1.0, astr_ctx_stream(fs->ctx), 0);
}

cudaError_t fs_halo(astr_full* fs, double* F, int nf, int dir);

// convrsdcmp, every direction (see the file header); with the characteristic decomposition the
// Ducros sensor runs first (ducrossensor, called by rhscal before convrsdcmp, solver.F90:228-231)
cudaError_t fs_convection_upwind(astr_full* fs) {
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  const FsGeo& g = fs->g;
  const int64_t nn = (int64_t)(g.N[0] + 1) * (g.N[1] + 1) * (g.N[2] + 1);
  double *fsp = fs->up, *fsm = fs->up + 5 * g.fs, *fhp = fs->up + 10 * g.fs, *fhm = fs->up + 15 * g.fs;
  double *ssf = fs->up + 20 * g.fs, *lsh = fs->up + 21 * g.fs;
  cudaError_t e;
  if (fs->p.lchardecomp) {
    k_fs_ssf<<<blocks_for(nn), 256, 0, st>>>(ssf, fs->dvel, fs->prs, g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    for (int d = 0; d < 3; ++d)
      if (g.ntype[d] == 3 && (e = fs_halo(fs, ssf, 1, d)) != cudaSuccess) return e;
    k_fs_lshock<<<blocks_for(nn), 256, 0, st>>>(lsh, ssf, fs->p.shkcrt, g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  for (int d = 0; d < 3; ++d) {
    const int nt = g.ntype[d];
    const int iss = (nt == 1 || nt == 4) ? 0 : -HMW;
    const int iee = (nt == 2 || nt == 4) ? g.N[d] : g.N[d] + HMW;
    const int64_t nl = nn / (g.N[d] + 1) * (iee - iss + 1);
    k_fs_sw_split<<<blocks_for(nl), 256, 0, st>>>(fsp, fsm, fs->q, fs->rho, fs->vel, fs->prs, fs->tmp, d, iss, iee, g,
                                                  fs->th);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = flux_op(fs, fs->dfu[d], d, fsp, fhp, 5)) != cudaSuccess) return e;
    if ((e = flux_op(fs, fs->dfd[d], d, fsm, fhm, 5)) != cudaSuccess) return e;
    if (fs->p.lchardecomp) {
      const int64_t ni = nn / (g.N[d] + 1) * (g.N[d] + 2);
      k_fs_char_flux<<<blocks_for(ni), 256, 0, st>>>(fs->work, fsp, fsm, fhp, fhm, fs->q, fs->rho, fs->vel, fs->prs,
                                                     lsh, d, nt, iss, iee, g, fs->th);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      k_fs_flux_diff<<<blocks_for(5 * nn), 256, 0, st>>>(fs->qrhs, fs->work, d, g);
    } else {
      const int64_t ni = nn / (g.N[d] + 1) * (g.N[d] + 2);
      k_fs_mp_flux<<<blocks_for(5 * ni), 256, 0, st>>>(fs->work, fsp, fsm, fhp, fhm, d, nt, iss, iee, g);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      k_fs_flux_diff<<<blocks_for(5 * nn), 256, 0, st>>>(fs->qrhs, fs->work, d, g);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t fs_halo(astr_full* fs, double* F, int nf, int dir) {
  const int64_t n = (int64_t)nf * HMW * (fs->g.N[0] + 1) * (fs->g.N[1] + 1) * (fs->g.N[2] + 1) / (fs->g.n_(dir) + 1);
  k_fs_halo<<<blocks_for(n), 256, 0, astr_ctx_stream(fs->ctx)>>>(F, nf, dir, fs->g);
  return cudaGetLastError();
}

int64_t nodes(const astr_full* fs) { return (int64_t)(fs->g.N[0] + 1) * (fs->g.N[1] + 1) * (fs->g.N[2] + 1); }

// filterq, then qswap, then rhscal into qrhs; diagnostics of the stage when `diag`
cudaError_t fs_stage_rhs(astr_full* fs, bool diag) {
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  cudaError_t e;
  const FsGeo& g = fs->g;
  const int64_t nn = nodes(fs);
  if (fs->p.filter_on) {
    for (int d = 0; d < 3; ++d) {
      if (g.ntype[d] == 3 && (e = fs_halo(fs, fs->q, 5, d)) != cudaSuccess) return e;
      if ((e = line_op(fs, fs->df[d], d, fs->q, fs->qt, 5, 1.0, 0)) != cudaSuccess) return e;
      std::swap(fs->q, fs->qt);
    }
  }
  if ((e = cudaMemsetAsync(fs->qrhs, 0, 5 * (size_t)g.fs * sizeof(double), st)) != cudaSuccess) return e;
  // boucon: no-slip walls at the physical ends, in boucon's order (i-min, i-max, j-min, ...)
  for (int d = 0; d < 3; ++d)
    for (int side = 0; side < 2; ++side) {
      const int t = g.ntype[d];
      if (!(side == 0 ? (t == 1 || t == 4) : (t == 2 || t == 4))) continue;
      const int64_t nw = nn / (g.N[d] + 1);
      k_fs_noslip<<<blocks_for(nw), 256, 0, st>>>(fs->q, fs->rho, fs->vel, fs->prs, fs->tmp, d, side, g, fs->th);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
  for (int d = 0; d < 3; ++d) {
    if (g.ntype[d] != 3) continue;   // one rank, non-periodic: nothing to exchange
    const int64_t nl = nn / (g.N[d] + 1);
    k_fs_qswap<<<blocks_for(nl * 5 * (HMW + 1)), 256, 0, st>>>(fs->q, d, g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_fs_qswap_prims<<<blocks_for(nl * 2 * (HMW + 1)), 256, 0, st>>>(fs->q, fs->rho, fs->vel, fs->prs, fs->tmp, d, g,
                                                                     fs->th);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  // gradcal
  for (int d = 0; d < 3; ++d) {
    if ((e = line_op(fs, fs->dd[d], d, fs->vel, fs->dvel + 3 * d * g.fs, 3, g.rd[d], 0)) != cudaSuccess) return e;
    if ((e = line_op(fs, fs->dd[d], d, fs->tmp, fs->dtmp + d * g.fs, 1, g.rd[d], 0)) != cudaSuccess) return e;
  }
  if (fs->up) {
    if ((e = fs_convection_upwind(fs)) != cudaSuccess) return e;
  } else {
    // convrsdcal6, accumulated negated (scale -1: qrhs holds -qrhs, which is what rhscal's
    // qrhs = -qrhs leaves; negation is exact, so the sums are the reference's bit for bit)
    for (int d = 0; d < 3; ++d) {
      const int64_t nl = nn / (g.N[d] + 1) * (g.N[d] + 1 + 2 * HMW);
      k_fs_conv_flux<<<blocks_for(nl), 256, 0, st>>>(fs->work, fs->q, fs->vel, fs->prs, d, g);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if ((e = line_op(fs, fs->dd[d], d, fs->work, fs->qrhs, 5, -1.0, 1)) != cudaSuccess) return e;
    }
  }
  // diffrsdcal6
  k_fs_stress<<<blocks_for(nn), 256, 0, st>>>(fs->sigma, fs->qflux, fs->dvel, fs->dtmp, fs->vel, fs->tmp, g, fs->th);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  for (int d = 0; d < 3; ++d) {
    if (g.ntype[d] != 3) continue;
    if ((e = fs_halo(fs, fs->sigma, 6, d)) != cudaSuccess) return e;
    if ((e = fs_halo(fs, fs->qflux, 3, d)) != cudaSuccess) return e;
  }
  for (int d = 0; d < 3; ++d) {
    const int64_t nl = nn / (g.N[d] + 1) * (g.N[d] + 1 + 2 * HMW);
    k_fs_visc_flux<<<blocks_for(nl), 256, 0, st>>>(fs->work, fs->sigma, fs->qflux, d, g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = line_op(fs, fs->dd[d], d, fs->work, fs->qrhs + g.fs, 4, 1.0, 1)) != cudaSuccess) return e;
  }
  if (diag) {
    k_fs_diag<<<fs->nparts, 256, 0, st>>>(fs->partials, fs->rho, fs->vel, fs->dvel, fs->tmp, g, fs->th);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const double norm = (double)fs->p.im * (double)fs->p.jm * (double)fs->p.km;
    if ((e = launch_diag_reduce(fs->partials, fs->nparts, fs->hist, fs->counter, norm, st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t fs_step(astr_full* fs, double dt) {
  static const double rk[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  const int64_t nn = nodes(fs);
  cudaError_t e;
  for (int s = 0; s < 3; ++s) {
    if ((e = fs_stage_rhs(fs, s == 0)) != cudaSuccess) return e;
    k_fs_update<<<blocks_for(5 * nn), 256, 0, st>>>(fs->q, fs->qsave, fs->qrhs, rk[s][0], rk[s][1], rk[s][2], dt,
                                                   s == 0, fs->g);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_fs_prims<<<blocks_for(nn), 256, 0, st>>>(fs->q, fs->rho, fs->vel, fs->prs, fs->tmp, fs->g, fs->th);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int fs_copy(astr_full* fs, double* user, const int64_t* shape, const int64_t* lb, int to_state, int where) {
  const int N[3] = {fs->p.im, fs->p.jm, fs->p.km};
  for (int d = 0; d < 3; ++d)
    if (lb[d] > 0 || lb[d] + shape[d] - 1 < N[d]) return ffail(fs, ASTR_ERR_ARG, "array must cover nodes 0..N on every axis");
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  const int64_t u1 = shape[0], u2 = shape[0] * shape[1], ufs = shape[0] * shape[1] * shape[2];
  const int64_t uoff = -lb[0] - lb[1] * u1 - lb[2] * u2;
  double* dev = user;
  if (where == ASTR_HOST) {
    // through the filter's second buffer (free between calls)
    if ((size_t)(5 * ufs) > 5 * (size_t)fs->g.fs) return ffail(fs, ASTR_ERR_ARG, "host array larger than the staging buffer");
    dev = fs->qt;
  }
  // large pageable arrays move through pinned staging slots with several host threads
  const size_t bytes = 5 * (size_t)ufs * sizeof(double);
  const bool staged = where == ASTR_HOST && bytes >= STAGED_MIN_BYTES && host_pageable(user);
  std::string err;
  if (where == ASTR_HOST && to_state) {
    if (staged) {
      const int rc = staged_copy(dev, user, bytes, true, st, err);
      if (rc != ASTR_OK) return ffail(fs, rc, err);
    } else {
      FCK(cudaMemcpyAsync(dev, user, bytes, cudaMemcpyHostToDevice, st));
    }
  }
  k_fs_pack<<<blocks_for(5 * nodes(fs)), 256, 0, st>>>(fs->q, dev, fs->g, 1, u1, u2, ufs, uoff, to_state, 5);
  FCK(cudaGetLastError());
  if (where == ASTR_HOST && !to_state) {
    // the staging buffer holds the caller's layout with only nodes 0..N written: an array with
    // halos gets its node rows back and keeps its own halo entries
    const bool exact = lb[0] == 0 && lb[1] == 0 && lb[2] == 0 && shape[0] == N[0] + 1 && shape[1] == N[1] + 1 &&
                       shape[2] == N[2] + 1;
    if (staged) {
      const RowMask m{shape[0], shape[1], shape[2], -lb[0], N[0] - lb[0], -lb[1], N[1] - lb[1], -lb[2], N[2] - lb[2]};
      const int rc = staged_copy(user, dev, bytes, false, st, err, exact ? nullptr : &m);
      if (rc != ASTR_OK) return ffail(fs, rc, err);
    } else if (exact) {
      FCK(cudaMemcpyAsync(user, dev, bytes, cudaMemcpyDeviceToHost, st));
    } else {
      for (int m = 0; m < 5; ++m) {
        cudaMemcpy3DParms prm{};
        prm.srcPtr = make_cudaPitchedPtr(dev + m * ufs, (size_t)shape[0] * 8, (size_t)shape[0], (size_t)shape[1]);
        prm.dstPtr = make_cudaPitchedPtr(user + m * ufs, (size_t)shape[0] * 8, (size_t)shape[0], (size_t)shape[1]);
        prm.srcPos = prm.dstPos = make_cudaPos((size_t)(-lb[0]) * 8, (size_t)(-lb[1]), (size_t)(-lb[2]));
        prm.extent = make_cudaExtent((size_t)(N[0] + 1) * 8, (size_t)N[1] + 1, (size_t)N[2] + 1);
        prm.kind = cudaMemcpyDeviceToHost;
        FCK(cudaMemcpy3DAsync(&prm, st));
      }
    }
  }
  FCK(cudaStreamSynchronize(st));
  return ASTR_OK;
}

}  // namespace

extern "C" {

int astr_full_create(astr_ctx* ctx, const astr_params* p, astr_full** out) {
  if (!ctx || !p || !out) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(ctx));
  const int N[3] = {p->im, p->jm, p->km};
  for (int d = 0; d < 3; ++d)
    if (N[d] < 16) {
      astr_ctx_set_error(ctx, "each dimension must be >= 16");
      return ASTR_ERR_ARG;
    }
  astr_full* fs = new (std::nothrow) astr_full();
  if (!fs) return ASTR_ERR_NOMEM;
  fs->ctx = ctx;
  fs->p = *p;
  FsGeo& g = fs->g;
  const double pi = 4.0 * std::atan(1.0);
  for (int d = 0; d < 3; ++d) {
    g.N[d] = N[d];
    g.ntype[d] = p->ntype[d] == 0 ? 3 : p->ntype[d];
    if (g.ntype[d] < 1 || g.ntype[d] > 4 || (g.ntype[d] != 3 && !(p->twall > 0.0))) {
      delete fs;
      astr_ctx_set_error(ctx, "ntype must be 0 or 3 (periodic), 1, 2 or 4, and a wall needs twall > 0");
      return ASTR_ERR_ARG;
    }
  }
  g.s[0] = 1;
  g.s[1] = N[0] + 1 + 2 * HMW;
  g.s[2] = g.s[1] * (N[1] + 1 + 2 * HMW);
  g.fs = g.s[2] * (N[2] + 1 + 2 * HMW);
  const double h[3] = {2.0 * pi / double(N[0]), 2.0 * pi / double(N[1]), 2.0 * pi / double(N[2])};
  for (int d = 0; d < 3; ++d) g.rd[d] = 1.0 / h[d];
  g.jac = h[0] * h[1] * h[2];
  const double gm = p->gamma, m = p->mach;
  fs->th.const2 = gm * (m * m);
  fs->th.const5 = (gm - 1.0) * (m * m);
  fs->th.const6 = 1.0 / (gm - 1.0);
  fs->th.reynolds = p->reynolds;
  fs->th.prandtl = p->prandtl;
  fs->th.tc = p->sutherland / p->ref_tem;
  fs->th.tc1 = 1.0 + fs->th.tc;
  fs->th.twall = p->twall;
  fs->th.mach = p->mach;
  fs->th.gamma = p->gamma;
  const bool upwind = p->conschm == 543;
  if (p->conschm != 0 && p->conschm != 643 && !upwind) {
    delete fs;
    astr_ctx_set_error(ctx, "conschm must be 0 or 643 (central compact) or 543 (upwind compact flux)");
    return ASTR_ERR_ARG;
  }
  if (upwind && !(std::isfinite(p->bfacmpld) && (!p->lchardecomp || std::isfinite(p->shkcrt)))) {
    delete fs;
    astr_ctx_set_error(ctx, "bfacmpld (and shkcrt with the characteristic decomposition) must be finite");
    return ASTR_ERR_ARG;
  }
  if (!(p->mach > 0.0 && p->gamma > 1.0 && p->reynolds > 0.0 && p->prandtl > 0.0)) {
    delete fs;
    astr_ctx_set_error(ctx, "mach, reynolds and prandtl must be positive and gamma above 1");
    return ASTR_ERR_ARG;
  }
  if (p->lchardecomp && !upwind) fs->p.lchardecomp = 0;   // the decomposition belongs to convrsdcmp
  if (fs->p.lchardecomp && (g.ntype[0] != 3 || g.ntype[1] != 3 || g.ntype[2] != 3)) {
    delete fs;
    astr_ctx_set_error(ctx, "the characteristic decomposition reads the primitives of the halo node beyond each end: "
                            "periodic directions only on one rank");
    return ASTR_ERR_UNSUPPORTED;
  }
  for (int d = 0; d < 3; ++d) {
    build_fd_op(fs->hd[d], "643c", g.ntype[d], N[d]);
    build_filter_op(fs->hf[d], g.ntype[d], N[d], p->alfa_filter, p->beta_halo, p->beta_bound, false);
    const Layout L = pick_layout(fs->hf[d].nsys());
    if (L.S == 0) { delete fs; astr_ctx_set_error(ctx, "dimension too large (max 1145)"); return ASTR_ERR_UNSUPPORTED; }
    if (make_devop(fs->hd[d], pick_layout(fs->hd[d].nsys()), fs->dd[d]) != cudaSuccess ||
        make_devop(fs->hf[d], L, fs->df[d]) != cudaSuccess) {
      astr_full_destroy(fs);
      astr_ctx_set_error(ctx, "scheme tables");
      return ASTR_ERR_CUDA;
    }
    if (upwind) {
      build_flux_op(fs->hfu[d], 543, g.ntype[d], N[d], 1, p->bfacmpld);
      build_flux_op(fs->hfd[d], 543, g.ntype[d], N[d], -1, p->bfacmpld);
      const Layout Lf = pick_layout(fs->hfu[d].nsys());
      if (make_devop(fs->hfu[d], Lf, fs->dfu[d]) != cudaSuccess || make_devop(fs->hfd[d], Lf, fs->dfd[d]) != cudaSuccess) {
        astr_full_destroy(fs);
        astr_ctx_set_error(ctx, "scheme tables");
        return ASTR_ERR_CUDA;
      }
    }
  }
  // q(5) qt(5) rho vel(3) prs tmp qsave(5) qrhs(5) dvel(9) dtmp(3) sigma(6) qflux(3) work(5)
  // [+ f+ f- fh+ fh- (20), ssf and lshock (2) for the upwind convection]
  const size_t nf = upwind ? 74 : 52;
  if (cudaMalloc(&fs->buf, nf * (size_t)g.fs * sizeof(double)) != cudaSuccess) {
    astr_full_destroy(fs);
    astr_ctx_set_error(ctx, "full-solver state allocation");
    return ASTR_ERR_NOMEM;
  }
  cudaStream_t st = astr_ctx_stream(ctx);
  cudaMemsetAsync(fs->buf, 0, nf * (size_t)g.fs * sizeof(double), st);
  double* b = fs->buf;
  auto take = [&](int n) { double* r = b; b += (size_t)n * g.fs; return r; };
  fs->q = take(5); fs->qt = take(5); fs->rho = take(1); fs->vel = take(3); fs->prs = take(1); fs->tmp = take(1);
  fs->qsave = take(5); fs->qrhs = take(5); fs->dvel = take(9); fs->dtmp = take(3); fs->sigma = take(6);
  fs->qflux = take(3); fs->work = take(5);
  if (upwind) fs->up = take(22);
  fs->nparts = 148 * 4;
  if (cudaMalloc(&fs->partials, (size_t)fs->nparts * 3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&fs->hist, (size_t)fs->hist_cap * 3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&fs->counter, sizeof(int)) != cudaSuccess) {
    astr_full_destroy(fs);
    astr_ctx_set_error(ctx, "full-solver state allocation");
    return ASTR_ERR_NOMEM;
  }
  cudaMemsetAsync(fs->counter, 0, sizeof(int), st);
  if (cudaStreamSynchronize(st) != cudaSuccess) { astr_full_destroy(fs); return ASTR_ERR_CUDA; }
  *out = fs;
  return ASTR_OK;
}

int astr_full_destroy(astr_full* fs) {
  if (!fs) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  cudaStreamSynchronize(astr_ctx_stream(fs->ctx));
  for (int d = 0; d < 3; ++d) {
    free_devop(fs->dd[d]); free_devop(fs->df[d]); free_devop(fs->dfu[d]); free_devop(fs->dfd[d]);
  }
  if (fs->buf) cudaFree(fs->buf);
  if (fs->partials) cudaFree(fs->partials);
  if (fs->hist) cudaFree(fs->hist);
  if (fs->counter) cudaFree(fs->counter);
  delete fs;
  return ASTR_OK;
}

int astr_full_upload(astr_full* fs, const double* q, const int64_t shape[3], const int64_t lbound[3], int where) {
  if (!fs || !q || !shape || !lbound) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  int rc = fs_copy(fs, const_cast<double*>(q), shape, lbound, 1, where);
  if (rc) return rc;
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  k_fs_prims<<<blocks_for(nodes(fs)), 256, 0, st>>>(fs->q, fs->rho, fs->vel, fs->prs, fs->tmp, fs->g, fs->th);
  FCK(cudaGetLastError());
  FCK(cudaStreamSynchronize(st));
  return ASTR_OK;
}

// The file's fields are the primitive arrays rho, vel(1:3), prs, tmp, which the layout holds as six
// consecutive fields from fs->rho in the file's order (ro, u1, u2, u3, p, t).
int astr_full_write_flowfield(astr_full* fs, const char* filename) {
  if (!fs || !filename) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  const int64_t shape[3] = {fs->p.im + 1, fs->p.jm + 1, fs->p.km + 1};
  const int64_t n = shape[0] * shape[1] * shape[2];
  double* dprims = fs->dvel;   // 9 layout fields, free between steps
  k_fs_pack<<<blocks_for(6 * n), 256, 0, st>>>(fs->rho, dprims, fs->g, 1, shape[0], shape[0] * shape[1], n, 0, 0, 6);
  cudaError_t e = cudaGetLastError();
  std::string err;
  int rc = e != cudaSuccess ? ASTR_ERR_CUDA : flowfield_write(st, dprims, shape, fs->nstep, fs->time, filename, err);
  if (e != cudaSuccess) err = std::string("k_fs_pack: ") + cudaGetErrorString(e);
  return rc == ASTR_OK ? rc : ffail(fs, rc, err);
}

// readcheckpoint + updateq: q = fvar2q(ro, u, t) on nodes 0..N, the primitives of the layout
// recomputed from q (upload), then the interior primitives replaced by the file's, which the
// reference's first stage after a restart uses as read.
int astr_full_read_flowfield(astr_full* fs, const char* filename, char mode, int* nstep, double* time) {
  if (!fs || !filename) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  const int64_t shape[3] = {fs->p.im + 1, fs->p.jm + 1, fs->p.km + 1}, lb[3] = {0, 0, 0};
  const int64_t n = shape[0] * shape[1] * shape[2];
  // q (5 x n) in qsave and the file's primitives (6 x n) in dvel: stage buffers, free between steps
  double* dq = fs->qsave;
  double* dprims = fs->dvel;
  std::string err;
  int ns = 0;
  double t = 0.0;
  int rc = flowfield_read(st, dprims, shape, filename, mode, &ns, &t, err);
  cudaError_t e = cudaSuccess;
  if (rc == ASTR_OK && (e = flowfield_q_from_prims(st, dprims, dq, n, fs->p.mach, fs->p.gamma)) != cudaSuccess) {
    rc = ASTR_ERR_CUDA;
    err = std::string("fvar2q: ") + cudaGetErrorString(e);
  }
  if (rc == ASTR_OK) {
    rc = astr_full_upload(fs, dq, shape, lb, ASTR_DEVICE);   // sets the context's message on failure
    if (rc == ASTR_OK) {
      k_fs_pack<<<blocks_for(6 * n), 256, 0, st>>>(fs->rho, dprims, fs->g, 1, shape[0], shape[0] * shape[1], n, 0, 1, 6);
      if ((e = cudaGetLastError()) == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) {
        rc = ASTR_ERR_CUDA;
        err = std::string("k_fs_pack: ") + cudaGetErrorString(e);
      }
    }
  }
  if (rc != ASTR_OK) return err.empty() ? rc : ffail(fs, rc, err);
  fs->nstep = ns;
  fs->time = t;
  if (nstep) *nstep = ns;
  if (time) *time = t;
  return ASTR_OK;
}

int astr_full_download(astr_full* fs, double* q, const int64_t shape[3], const int64_t lbound[3], int where) {
  if (!fs || !q || !shape || !lbound) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  return fs_copy(fs, q, shape, lbound, 0, where);
}

int astr_full_rhs(astr_full* fs, double* qrhs, const int64_t shape[3], const int64_t lbound[3], int where) {
  if (!fs || !qrhs || !shape || !lbound) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  FCK(fs_stage_rhs(fs, false));
  // qrhs goes out through the pack kernel: swap it in for q for the copy
  std::swap(fs->q, fs->qrhs);
  int rc = fs_copy(fs, qrhs, shape, lbound, 0, where);
  std::swap(fs->q, fs->qrhs);
  return rc;
}

int astr_full_step(astr_full* fs, double dt, int nsteps) {
  if (!fs || !(dt > 0.0) || nsteps < 0) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  if ((int)(fs->row_key.size() / 2) + nsteps > fs->hist_cap) return ffail(fs, ASTR_ERR_UNSUPPORTED, "history buffer full (65536 steps)");
  for (int s = 0; s < nsteps; ++s) {
    fs->row_key.push_back((double)fs->nstep);
    fs->row_key.push_back(fs->time);
    FCK(fs_step(fs, dt));
    fs->nstep += 1;
    fs->time = fs->time + dt;
  }
  FCK(cudaStreamSynchronize(astr_ctx_stream(fs->ctx)));
  return ASTR_OK;
}

int astr_full_history(astr_full* fs, double* rows, int maxrows, int* nrows) {
  if (!fs || !nrows) return ASTR_ERR_ARG;
  const OnDev on(astr_ctx_device(fs->ctx));
  const int n = (int)(fs->row_key.size() / 2);   // rows written (nstep may start elsewhere after a restart)
  *nrows = n;
  if (!rows || maxrows <= 0 || n == 0) return ASTR_OK;
  const int k = n < maxrows ? n : maxrows;
  std::vector<double> h((size_t)3 * k);
  cudaStream_t st = astr_ctx_stream(fs->ctx);
  FCK(cudaMemcpyAsync(h.data(), fs->hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  FCK(cudaStreamSynchronize(st));
  for (int r = 0; r < k; ++r) {
    rows[5 * r] = fs->row_key[2 * r];
    rows[5 * r + 1] = fs->row_key[2 * r + 1];
    rows[5 * r + 2] = h[3 * r];
    rows[5 * r + 3] = h[3 * r + 1];
    rows[5 * r + 4] = h[3 * r + 2];
  }
  return ASTR_OK;
}

}  // extern "C"
