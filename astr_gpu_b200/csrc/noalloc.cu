// The CFL time step of a conserved-variable field without any device allocation.
//
// Some callers cannot let a library allocate device memory: codes that size one device pool
// at start-up and run the whole time loop inside it (a CUDA-Fortran or OpenACC solver, or a
// framework with a capped caching allocator), where a cudaMalloc either fails against the cap
// or, because cudaMalloc/cudaFree synchronise the device, stalls every other stream mid-step.
// For them, astr_cfl_dt_noalloc does the work of astr_cfl_dt with its scratch (one triple of
// partial maxima per CTA, plus the final triple) in a file-scope __device__ array: every GPU
// that loads this library holds kScratchDoubles doubles (1.5 MB) of it until exit.
#include <mutex>

#include "../../include/astr_b200.h"
#include "internal.h"

namespace {

constexpr int kLinesPerCta = 8;                      // x lines per CTA
constexpr int kMaxCtas = 65536;                      // partial maxima kept
constexpr int kScratchDoubles = 3 * kMaxCtas + 3;    // + the final triple

static __device__ __align__(256) double g_cfl_scratch[kScratchDoubles];

// Device address of g_cfl_scratch per device, looked up once per device with that device
// current (the call's device, made current by the caller of scratch_address).
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

cudaError_t scratch_address(int dev, double** out) {
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

// The device of the call current for its duration; the caller's device restored afterwards.
struct OnDevice {
  int prev = -1;
  explicit OnDevice(int dev) {
    int cur = -1;
    if (dev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
  }
  ~OnDevice() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

struct FieldDesc {
  const double* q;
  int64_t s1, s2, fs;       // element strides of j, k and of the field index
  int64_t off0;             // element offset of node (0,0,0) of field 1
  int n0, n1, n2;           // nodes per axis (im+1, jm+1, km+1)
};

// cflcal (src/commcal.F90:46-77) on a uniform grid: per-CTA maxima of the three spectral radii
// over kLinesPerCta x lines. Same arithmetic as k_cfl in tgv.cu.
__global__ void k_cfl_lines(FieldDesc f, double rd0, double rd1, double rd2, double const2, double const6, double mach,
                            double* partials) {
  __shared__ double s[3][256];
  const double rd[3] = {rd0, rd1, rd2};
  double m[3] = {0.0, 0.0, 0.0};
  const int64_t nlines = (int64_t)f.n1 * f.n2;
  for (int l = 0; l < kLinesPerCta; ++l) {
    const int64_t line = (int64_t)blockIdx.x * kLinesPerCta + l;
    if (line >= nlines) break;
    const int64_t j = line % f.n1, k = line / f.n1;
    const double* base = f.q + f.off0 + j * f.s1 + k * f.s2;
    for (int i = threadIdx.x; i < f.n0; i += blockDim.x) {
      const double q0 = base[i], q1 = base[f.fs + i], q2 = base[2 * f.fs + i], q3 = base[3 * f.fs + i],
                   q4 = base[4 * f.fs + i];
      const double vel[3] = {q1 / q0, q2 / q0, q3 / q0};
      const double pr = (q4 - 0.5 * q0 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) / const6;
      const double tmp = pr / q0 * const2;
      const double css = sqrt(tmp) / mach;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double ub = rd[d] * vel[d];
        const double cs = css * sqrt(rd[d] * rd[d]);
        m[d] = fmax(m[d], fmax(ub, fmax(ub - cs, ub + cs)));
      }
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

// Maximum over the nctas partial triples into out[0..2] (all of them written by this call).
__global__ void k_cfl_final(const double* partials, int nctas, double* out) {
  __shared__ double s[3][256];
  double m[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nctas; b += blockDim.x)
    for (int d = 0; d < 3; ++d) m[d] = fmax(m[d], partials[3 * b + d]);
  for (int d = 0; d < 3; ++d) s[d][threadIdx.x] = m[d];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int d = 0; d < 3; ++d) s[d][threadIdx.x] = fmax(s[d][threadIdx.x], s[d][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) out[d] = s[d][0];
}

}  // namespace

// Defined in capi.cu: stream and device of a context, and its error slot.
cudaStream_t astr_ctx_stream(astr_ctx* ctx);
int astr_ctx_device(astr_ctx* ctx);
void astr_ctx_set_error(astr_ctx* ctx, const char* msg);

extern "C" int astr_cfl_dt_noalloc(astr_ctx* ctx, const double* q, const int64_t shape[3], const int64_t lbound[3],
                                   int im, int jm, int km, double mach, double gamma, double cfl, double* dt) {
  if (!q || !shape || !lbound || !dt || im < 1 || jm < 1 || km < 1 || !(mach > 0.0) || !(gamma > 1.0)) {
    if (ctx) astr_ctx_set_error(ctx, "astr_cfl_dt_noalloc: null pointer or bad size/parameter");
    return ASTR_ERR_ARG;
  }
  const int N[3] = {im, jm, km};
  for (int d = 0; d < 3; ++d) {
    if (lbound[d] > 0 || lbound[d] + shape[d] - 1 < N[d]) {
      if (ctx) astr_ctx_set_error(ctx, "astr_cfl_dt_noalloc: q must cover nodes 0..N on every axis");
      return ASTR_ERR_ARG;
    }
  }
  const int64_t nlines = (int64_t)(jm + 1) * (km + 1);
  const int64_t nctas = (nlines + kLinesPerCta - 1) / kLinesPerCta;
  if (nctas > kMaxCtas) {
    if (ctx)
      astr_ctx_set_error(ctx, "astr_cfl_dt_noalloc: (jm+1)*(km+1) exceeds the 524288 x lines its static scratch holds");
    return ASTR_ERR_UNSUPPORTED;
  }
  // the context's device (else the caller's current one) for the whole call
  int dev = 0;
  if (ctx) dev = astr_ctx_device(ctx);
  else if (cudaGetDevice(&dev) != cudaSuccess) return ASTR_ERR_CUDA;
  const OnDevice on(dev);
  cudaStream_t st = ctx ? astr_ctx_stream(ctx) : nullptr;
  // dt comes back to the host, so the call synchronises its stream: not allowed under capture
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(st, &cap);
  if (e == cudaSuccess && cap != cudaStreamCaptureStatusNone) {
    if (ctx) astr_ctx_set_error(ctx, "astr_cfl_dt_noalloc: called during stream capture (it returns dt to the host)");
    return ASTR_ERR_ARG;
  }
  double* scratch = nullptr;
  if (e == cudaSuccess) e = scratch_address(dev, &scratch);
  if (e != cudaSuccess) {
    if (ctx) astr_ctx_set_error(ctx, cudaGetErrorString(e));
    return ASTR_ERR_CUDA;
  }
  FieldDesc f;
  f.q = q;
  f.s1 = shape[0];
  f.s2 = shape[0] * shape[1];
  f.fs = shape[0] * shape[1] * shape[2];
  f.off0 = -lbound[0] - lbound[1] * f.s1 - lbound[2] * f.s2;
  f.n0 = im + 1;
  f.n1 = jm + 1;
  f.n2 = km + 1;
  const double pi = 4.0 * atan(1.0);
  const double const2 = gamma * (mach * mach), const6 = 1.0 / (gamma - 1.0);
  double rd0 = 1.0 / (2.0 * pi / im), rd1 = 1.0 / (2.0 * pi / jm), rd2 = 1.0 / (2.0 * pi / km);
  double* partials = scratch;
  double* final3 = scratch + 3 * kMaxCtas;
  int nc = (int)nctas;
  // launch errors are taken from each launch itself, so an error left by unrelated earlier work
  // is neither reported as this call's nor cleared
  void* a1[] = {&f, &rd0, &rd1, &rd2, (void*)&const2, (void*)&const6, &mach, &partials};
  e = cudaLaunchKernel((const void*)k_cfl_lines, dim3((unsigned)nctas), dim3(256), a1, 0, st);
  void* a2[] = {&partials, &nc, &final3};
  if (e == cudaSuccess) e = cudaLaunchKernel((const void*)k_cfl_final, dim3(1), dim3(256), a2, 0, st);
  double m[3] = {0.0, 0.0, 0.0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(m, final3, sizeof(m), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    if (ctx) astr_ctx_set_error(ctx, cudaGetErrorString(e));
    return ASTR_ERR_CUDA;
  }
  *dt = cfl / (m[0] + m[1] + m[2]);
  return ASTR_OK;
}
