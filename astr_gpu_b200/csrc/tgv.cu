// Fused per-stage passes of the Taylor-Green RK3 step.
//
// The reference stage (tgvsolver.F90:1037-1074) is: bchomo; rhscal = gradcal (12 line solves),
// convection (15), qrhs=-qrhs, diffusion (pointwise sigma/qflux + 12 line solves); RK update;
// filterq (15 line solves, x then y then z). Here one stage is six directional passes over
// lines of directions A, B, C (a permutation of x, y, z); each pass stages TI lines of its
// inputs in shared memory once and does every line solve that the stage needs along that
// direction:
//   A : filter-A of the previous stage (in place on q), dA(u,v,w,T), R  = -conv_A
//   B : dB(u,v,w,T), R -= conv_B
//   C : dC(u,v,w,T); sigma/qflux at every node from dA,dB (HBM) and dC (smem); writes the
//       A and B viscous fluxes (7 fields) and keeps the C ones in smem; R += visc_C - conv_C
//   A': R += visc_A
//   B': R += visc_B, RK update, filter-B
//   C'(F): filter-C
// Separable line filters commute, so filtering B, C then A (instead of x, y, z) changes only
// rounding. Periodic halos are index wraps (tile loads read node dim-k for -k and k for dim+k,
// the copies bchomo/bchomovec make); q at halo nodes of the convective flux is rebuilt from the
// primitive variables as bchomo does (fvar2q of q2fvar).
#include "tgv.cuh"

namespace astr {

namespace {

// ------------------------------------------------------------------ small kernels
__global__ void k_diag_reduce(const double* __restrict__ partials, int nparts, double* hist, int* counter,
                              double norm) {
  __shared__ double s[3][1024];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    a0 += partials[3 * i];
    a1 += partials[3 * i + 1];
    a2 += partials[3 * i + 2];
  }
  s[0][threadIdx.x] = a0;
  s[1][threadIdx.x] = a1;
  s[2][threadIdx.x] = a2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s[0][threadIdx.x] += s[0][threadIdx.x + w];
      s[1][threadIdx.x] += s[1][threadIdx.x + w];
      s[2][threadIdx.x] += s[2][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int row = *counter;
    hist[3 * row] = 0.5 * s[0][0] / norm;
    hist[3 * row + 1] = 0.5 * s[1][0] / norm;
    hist[3 * row + 2] = s[2][0] / norm;
    *counter = row + 1;
  }
}

__global__ void k_diag_reduce_batch(const DiagArgs* __restrict__ args) {
  const DiagArgs a = args[blockIdx.x];
  __shared__ double s[3][256];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = threadIdx.x; i < a.nparts; i += blockDim.x) {
    a0 += a.partials[3 * i];
    a1 += a.partials[3 * i + 1];
    a2 += a.partials[3 * i + 2];
  }
  s[0][threadIdx.x] = a0;
  s[1][threadIdx.x] = a1;
  s[2][threadIdx.x] = a2;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s[0][threadIdx.x] += s[0][threadIdx.x + w];
      s[1][threadIdx.x] += s[1][threadIdx.x + w];
      s[2][threadIdx.x] += s[2][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int row = *a.counter;
    a.hist[3 * row] = 0.5 * s[0][0] / a.norm;
    a.hist[3 * row + 1] = 0.5 * s[1][0] / a.norm;
    a.hist[3 * row + 2] = s[2][0] / a.norm;
    *a.counter = row + 1;
  }
}

// flowfield_init (tgvsolver.F90:203-224). Arithmetic is spelled with explicit _rn intrinsics so
// that no multiply-add is contracted: the state matches the reference's bit for bit.
__global__ void k_init_tgv(BoxGeo g, double const6, double pinf, double* q, const double* __restrict__ tabs) {
  const int64_t n0 = g.N[0] + 1, n1 = g.N[1] + 1, n2 = g.N[2] + 1;
  const double* sx = tabs;
  const double* cx = sx + n0;
  const double* c2x = cx + n0;
  const double* sy = c2x + n0;
  const double* cy = sy + n1;
  const double* c2y = cy + n1;
  const double* sz = c2y + n1;
  const double* cz = sz + n2;
  const double* c2z = cz + n2;
  const int64_t total = n0 * n1 * n2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = p % n0, j = (p / n0) % n1, k = p / (n0 * n1);
    const double rho = 1.0;
    const double u = __dmul_rn(__dmul_rn(sx[i], cy[j]), cz[k]);
    const double v = -__dmul_rn(__dmul_rn(cx[i], sy[j]), cz[k]);
    const double w = 0.0;
    const double pr = __dadd_rn(pinf, __dmul_rn(__dmul_rn(1.0 / 16.0, __dadd_rn(c2x[i], c2y[j])), __dadd_rn(c2z[k], 2.0)));
    const double var1 = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w)));
    const int64_t off = i + j * g.st[1] + k * g.st[2];
    q[off] = rho;
    q[g.fs + off] = __dmul_rn(rho, u);
    q[2 * g.fs + off] = __dmul_rn(rho, v);
    q[3 * g.fs + off] = __dmul_rn(rho, w);
    q[4 * g.fs + off] = __dadd_rn(__dmul_rn(pr, const6), __dmul_rn(rho, var1));
  }
}

// cflcal (commcal.F90:46-77) on a uniform grid: per-CTA maxima of the three spectral radii.
__global__ void k_cfl(BoxGeo g, Thermo th, const double* __restrict__ q, double* partials) {
  __shared__ double s[3][256];
  const int64_t n0 = g.N[0] + 1, n1 = g.N[1] + 1, n2 = g.N[2] + 1, total = n0 * n1 * n2;
  double m[3] = {0.0, 0.0, 0.0};
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = p % n0, j = (p / n0) % n1, k = p / (n0 * n1);
    const int64_t off = i + j * g.st[1] + k * g.st[2];
    const double q0 = q[off], q1 = q[g.fs + off], q2 = q[2 * g.fs + off], q3 = q[3 * g.fs + off], q4 = q[4 * g.fs + off];
    const double vel[3] = {q1 / q0, q2 / q0, q3 / q0};
    const double pr = (q4 - 0.5 * q0 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) / th.const6;
    const double tmp = pr / q0 * th.const2;
    const double css = sqrt(tmp) / th.mach;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double ub = g.rd[d] * vel[d];
      const double cs = css * sqrt(g.rd[d] * g.rd[d]);
      m[d] = fmax(m[d], fmax(ub, fmax(ub - cs, ub + cs)));
    }
  }
  for (int d = 0; d < 3; ++d) s[d][threadIdx.x] = m[d];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int d = 0; d < 3; ++d) s[d][threadIdx.x] = fmax(s[d][threadIdx.x], s[d][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) partials[3 * blockIdx.x + d] = s[d][0];
}

__global__ void k_pack(BoxGeo g, double* state, double* user, int64_t us0, int64_t us1, int64_t us2, int64_t ul0,
                       int64_t ul1, int64_t ul2, int nfields, int to_state) {
  const int64_t n0 = g.N[0] + 1, n1 = g.N[1] + 1, n2 = g.N[2] + 1, total = n0 * n1 * n2 * nfields;
  const int64_t ufs = us0 * us1 * us2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = p % n0, j = (p / n0) % n1, k = (p / (n0 * n1)) % n2, m = p / (n0 * n1 * n2);
    const int64_t so = m * g.fs + i + j * g.st[1] + k * g.st[2];
    const int64_t uo = m * ufs + ((k - ul2) * us1 + (j - ul1)) * us0 + (i - ul0);
    if (to_state) state[so] = user[uo];
    else user[uo] = state[so];
  }
}

}  // namespace

int pass_tiles(int pass) {
  switch (pass) {
    case PASS_A: case PASS_B: return 5;
    case PASS_C: return 10;
    case PASS_VA: case PASS_VB: case PASS_F: return 5;   // all fields at once (see shape_tiles)
  }
  return 0;
}

template <int S, int WPL>
cudaError_t launch_pass_t(int pass, const PassArgs& a, cudaStream_t st);
template <int S, int WPL>
cudaError_t launch_pass_batch_t(int pass, int dir, const PassArgs* dargs, const int* dcum, int nbox, int nctas,
                                int threads, size_t smem, cudaStream_t st);

cudaError_t launch_pass_batch(int pass, int dir, int S, int WPL, const PassArgs* dargs, const int* dcum, int nbox,
                              int nctas, int threads, size_t smem, cudaStream_t st) {
#define ASTR_B(s_, w_) \
  if (S == s_ && WPL == w_) return launch_pass_batch_t<s_, w_>(pass, dir, dargs, dcum, nbox, nctas, threads, smem, st);
  ASTR_B(3, 1) ASTR_B(5, 1) ASTR_B(5, 2) ASTR_B(5, 4) ASTR_B(9, 1) ASTR_B(9, 2) ASTR_B(9, 4) ASTR_B(17, 1)
#undef ASTR_B
  return cudaErrorInvalidValue;
}

int shape_tiles(int pass, int LPW, int FPS) {
  // A', B' and the filters (stream_fields): all five fields in one buffer, or one field at a time
  // through one buffer (warps looping over lines) or two
  if (pass == PASS_VA || pass == PASS_VB || pass == PASS_F) return FPS > 1 ? 5 : (LPW > 1 ? 1 : 2);
  return pass_tiles(pass);
}

size_t pass_shared_bytes(int pass, int TI, int LP, int WPL, int LPW, int FPS) {
  const size_t tiles = shape_tiles(pass, LPW, FPS);
  size_t smem = (tiles * TI * LP + (size_t)TI * (SCAN_PER_LINE * WPL + SP_PER_LINE)) * sizeof(double);
  if (pass == PASS_C) smem += 32 * 3 * sizeof(double);
  return smem;
}

cudaError_t launch_pass(int pass, const PassArgs& a, int S, int WPL, cudaStream_t st) {
  if (S == 3 && WPL == 1) return launch_pass_t<3, 1>(pass, a, st);
  if (S == 5 && WPL == 1) return launch_pass_t<5, 1>(pass, a, st);
  if (S == 5 && WPL == 2) return launch_pass_t<5, 2>(pass, a, st);
  if (S == 5 && WPL == 4) return launch_pass_t<5, 4>(pass, a, st);
  if (S == 9 && WPL == 1) return launch_pass_t<9, 1>(pass, a, st);
  if (S == 9 && WPL == 2) return launch_pass_t<9, 2>(pass, a, st);

  if (S == 9 && WPL == 4) return launch_pass_t<9, 4>(pass, a, st);
  if (S == 17 && WPL == 1) return launch_pass_t<17, 1>(pass, a, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_diag_reduce(const double* partials, int nparts, double* hist, int* counter, double norm,
                               cudaStream_t st) {
  k_diag_reduce<<<1, 1024, 0, st>>>(partials, nparts, hist, counter, norm);
  return cudaGetLastError();
}

cudaError_t launch_diag_reduce_batch(const DiagArgs* dargs, int nbox, cudaStream_t st) {
  k_diag_reduce_batch<<<nbox, 256, 0, st>>>(dargs);
  return cudaGetLastError();
}

cudaError_t launch_init_tgv(const BoxGeo& g, const Thermo& th, double* q, const double* tabs, cudaStream_t st) {
  k_init_tgv<<<148 * 8, 256, 0, st>>>(g, th.const6, 1.0 / th.const2, q, tabs);
  return cudaGetLastError();
}

cudaError_t launch_cfl(const BoxGeo& g, const Thermo& th, const double* q, double* partials, int* nparts,
                       cudaStream_t st) {
  *nparts = 148 * 4;
  k_cfl<<<*nparts, 256, 0, st>>>(g, th, q, partials);
  return cudaGetLastError();
}

cudaError_t launch_pack(const BoxGeo& g, double* state, double* user, const int64_t* us, const int64_t* ul,
                        int nfields, int to_state, cudaStream_t st) {
  k_pack<<<148 * 8, 256, 0, st>>>(g, state, user, us[0], us[1], us[2], ul[0], ul[1], ul[2], nfields, to_state);
  return cudaGetLastError();
}

}  // namespace astr
