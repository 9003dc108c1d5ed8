// Flow-field checkpoints of the solver states (the flow-field part of writeflfed and of
// readcheckpoint + updateq): conversions between the conserved variables and the file's primitive
// fields on the GPU, and the transfers between HBM and the file (h5file.cpp).
//
// File: datasets ro, u1, u2, u3, p, t of Fortran shape (im+1, jm+1, km+1) (write_io_tree,
// src/readwrite.F90:1920-1979), nstep (integer) and time (real(8)) of one element each (h5srite,
// src/readwrite.F90:1834-1835). Conversions, evaluated in the reference's order with every
// operation rounded separately (no multiply-add contraction), so that they equal the reference's
// gfortran build bit for bit:
//   q2fvar (src/fludyna.F90:545-634): u = q_m / rho, p = (q5 - 0.5 rho (u1^2 + u2^2 + u3^2)) / const6,
//           t = p / rho * const2 (thermal_3d, src/fludyna.F90:136-153);
//   fvar2q with temperature (src/fludyna.F90:449-533, the branch updateq takes,
//           src/fludyna.F90:254-300): q_m = rho u_m, q5 = rho (t const1 + 0.5 (u1^2 + u2^2 + u3^2)).
// const1 = 1/(gamma (gamma-1) M^2), const2 = gamma M^2, const6 = 1/(gamma-1) (nondimensional run).

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/astr_b200.h"
#include "internal.h"

namespace astr {

namespace {

__global__ void k_ckpt_prims(const double* __restrict__ q, int64_t n, double const2, double const6,
                             double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double r = q[i];
    const double u = __ddiv_rn(q[n + i], r), v = __ddiv_rn(q[2 * n + i], r), w = __ddiv_rn(q[3 * n + i], r);
    const double ke = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    const double p = __ddiv_rn(__dsub_rn(q[4 * n + i], __dmul_rn(__dmul_rn(0.5, r), ke)), const6);
    out[i] = r;
    out[n + i] = u;
    out[2 * n + i] = v;
    out[3 * n + i] = w;
    out[4 * n + i] = p;
    out[5 * n + i] = __dmul_rn(__ddiv_rn(p, r), const2);
  }
}

__global__ void k_ckpt_q(const double* __restrict__ f, int64_t n, double const1, double* __restrict__ q) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double r = f[i], u = f[n + i], v = f[2 * n + i], w = f[3 * n + i], t = f[5 * n + i];
    const double ke = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
    q[i] = r;
    q[n + i] = __dmul_rn(r, u);
    q[2 * n + i] = __dmul_rn(r, v);
    q[3 * n + i] = __dmul_rn(r, w);
    q[4 * n + i] = __dmul_rn(r, __dadd_rn(__dmul_rn(t, const1), __dmul_rn(0.5, ke)));
  }
}

unsigned grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (unsigned)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

const char* const NAMES[6] = {"ro", "u1", "u2", "u3", "p", "t"};

// Two pinned host buffers of one field each: field f moves through buf[f % 2] while the other
// buffer's file I/O or copy proceeds.
struct Pinned {
  double* buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  ~Pinned() {
    for (int b = 0; b < 2; ++b) {
      if (done[b]) cudaEventDestroy(done[b]);
      if (buf[b]) cudaFreeHost(buf[b]);
    }
  }
  cudaError_t init(size_t bytes) {
    cudaError_t e;
    for (int b = 0; b < 2; ++b) {
      if ((e = cudaMallocHost(&buf[b], bytes)) != cudaSuccess) return e;
      if ((e = cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
};

int cuda_err(std::string& err, cudaError_t e, const char* what) {
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return ASTR_ERR_CUDA;
}
int h5_err(std::string& err, astr_h5* h, int rc) {
  err = astr_h5_last_error(h);
  return rc;
}

}  // namespace

void thermo_constants(double mach, double gamma, double& const1, double& const2, double& const6) {
  const1 = 1.0 / (gamma * (gamma - 1.0) * (mach * mach));
  const2 = gamma * (mach * mach);
  const6 = 1.0 / (gamma - 1.0);
}

cudaError_t flowfield_prims_from_q(cudaStream_t st, const double* dq, double* dprims, int64_t n, double mach,
                                   double gamma) {
  double c1, c2, c6;
  thermo_constants(mach, gamma, c1, c2, c6);
  k_ckpt_prims<<<grid_for(n), 256, 0, st>>>(dq, n, c2, c6, dprims);
  return cudaGetLastError();
}

cudaError_t flowfield_q_from_prims(cudaStream_t st, const double* dprims, double* dq, int64_t n, double mach,
                                   double gamma) {
  double c1, c2, c6;
  thermo_constants(mach, gamma, c1, c2, c6);
  k_ckpt_q<<<grid_for(n), 256, 0, st>>>(dprims, n, c1, dq);
  return cudaGetLastError();
}

int flowfield_write(cudaStream_t st, const double* dprims, const int64_t shape[3], int nstep, double time,
                    const char* filename, std::string& err) {
  const int64_t n = shape[0] * shape[1] * shape[2];
  Pinned pin;
  cudaError_t e;
  if ((e = pin.init((size_t)n * sizeof(double))) != cudaSuccess) return cuda_err(err, e, "pinned host buffers");
  astr_h5* h = nullptr;
  int rc = astr_h5io_init(filename, "write", &h);
  if (rc != ASTR_OK) return h5_err(err, nullptr, rc);
  // field f: copied into buf[f % 2] while field f - 1 is written from the other buffer
  if ((e = cudaMemcpyAsync(pin.buf[0], dprims, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaEventRecord(pin.done[0], st)) != cudaSuccess) {
    astr_h5io_end(h);
    return cuda_err(err, e, "flow-field download");
  }
  for (int f = 0; f < 6 && rc == ASTR_OK; ++f) {
    if ((e = cudaEventSynchronize(pin.done[f % 2])) != cudaSuccess) { rc = cuda_err(err, e, "flow-field download"); break; }
    if (f + 1 < 6 &&
        ((e = cudaMemcpyAsync(pin.buf[(f + 1) % 2], dprims + (size_t)(f + 1) * n, (size_t)n * sizeof(double),
                              cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
         (e = cudaEventRecord(pin.done[(f + 1) % 2], st)) != cudaSuccess)) {
      rc = cuda_err(err, e, "flow-field download");
      break;
    }
    if ((rc = astr_h5write_r8(h, NAMES[f], 3, shape, pin.buf[f % 2])) != ASTR_OK) h5_err(err, h, rc);
  }
  cudaStreamSynchronize(st);
  const int64_t one = 1;
  const int32_t ns = nstep;
  if (rc == ASTR_OK && (rc = astr_h5write_i4(h, "nstep", 1, &one, &ns)) != ASTR_OK) h5_err(err, h, rc);
  if (rc == ASTR_OK && (rc = astr_h5write_r8(h, "time", 1, &one, &time)) != ASTR_OK) h5_err(err, h, rc);
  const int rc_end = astr_h5io_end(h);
  if (rc == ASTR_OK && rc_end != ASTR_OK) rc = h5_err(err, nullptr, rc_end);
  return rc;
}

int flowfield_read(cudaStream_t st, double* dprims, const int64_t shape[3], const char* filename, char mode,
                   int* nstep, double* time, std::string& err) {
  if (mode != 'h' && mode != 's') {
    err = "mode must be 'h' (3-D datasets) or 's' (1-D stream datasets)";
    return ASTR_ERR_ARG;
  }
  const int64_t n = shape[0] * shape[1] * shape[2];
  astr_h5* h = nullptr;
  int rc = astr_h5io_init(filename, "read", &h);
  if (rc != ASTR_OK) return h5_err(err, nullptr, rc);
  const int64_t one = 1;
  int32_t ns = 0;
  double t = 0.0;
  if ((rc = astr_h5read_i4(h, "nstep", 1, &one, nullptr, 'h', &ns)) != ASTR_OK ||
      (rc = astr_h5read_r8(h, "time", 1, &one, nullptr, 'h', &t)) != ASTR_OK) {
    h5_err(err, h, rc);
    astr_h5io_end(h);
    return rc;
  }
  Pinned pin;
  cudaError_t e;
  if ((e = pin.init((size_t)n * sizeof(double))) != cudaSuccess) {
    astr_h5io_end(h);
    return cuda_err(err, e, "pinned host buffers");
  }
  // field f is read into buf[f % 2] once the upload of field f - 2 from it has finished
  const int64_t flat = n;
  for (int f = 0; f < 6; ++f) {
    if (f >= 2 && (e = cudaEventSynchronize(pin.done[f % 2])) != cudaSuccess) { rc = cuda_err(err, e, "flow-field upload"); break; }
    rc = mode == 'h' ? astr_h5read_r8(h, NAMES[f], 3, shape, nullptr, 'h', pin.buf[f % 2])
                     : astr_h5read_r8(h, NAMES[f], 1, &flat, nullptr, 's', pin.buf[f % 2]);
    if (rc != ASTR_OK) { h5_err(err, h, rc); break; }
    if ((e = cudaMemcpyAsync(dprims + (size_t)f * n, pin.buf[f % 2], (size_t)n * sizeof(double), cudaMemcpyHostToDevice,
                             st)) != cudaSuccess ||
        (e = cudaEventRecord(pin.done[f % 2], st)) != cudaSuccess) {
      rc = cuda_err(err, e, "flow-field upload");
      break;
    }
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess && rc == ASTR_OK) rc = cuda_err(err, e, "flow-field upload");
  astr_h5io_end(h);
  if (rc == ASTR_OK) {
    *nstep = ns;
    *time = t;
  }
  return rc;
}

}  // namespace astr
