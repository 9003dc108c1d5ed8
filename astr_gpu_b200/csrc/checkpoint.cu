// Flow-field checkpoints of the solver states (the flow-field part of writeflfed and of
// readcheckpoint + updateq): conversions between the conserved variables and the file's primitive
// fields on the GPU, and chunked transfers between HBM and the file through pinned slots and host
// I/O threads (the file format itself is h5file.cpp).
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
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/astr_b200.h"
#include "h5file.h"
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

int cuda_err(std::string& err, cudaError_t e, const char* what) {
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return ASTR_ERR_CUDA;
}
int h5_err(std::string& err, astr_h5* h, int rc) {
  err = astr_h5_last_error(h);
  return rc;
}

// One contiguous run of doubles between device memory and a file.
struct Piece {
  int fd;
  uint64_t off;          // absolute file offset
  const double* dsrc;    // device source (to the file)
  double* ddst;          // device destination (from the file)
  size_t bytes;
};

// Pinned staging slots, allocated on first use and kept for the process (portable, so any
// device's transfers may use them); one transfer at a time holds them.
struct SlotPool {
  std::mutex m;
  std::vector<char*> buf;
};
SlotPool& slot_pool() {
  static SlotPool p;
  return p;
}
constexpr size_t SLOT_BYTES = size_t(8) << 20;

int io_threads() { return (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency())); }

// Grows the pool to nslots slots (the caller holds P.m).
int ensure_slots(SlotPool& P, int nslots, std::string& err) {
  while ((int)P.buf.size() < nslots) {
    void* b = nullptr;
    cudaError_t e = cudaHostAlloc(&b, SLOT_BYTES, cudaHostAllocPortable);
    if (e != cudaSuccess) return cuda_err(err, e, "pinned staging slots");
    P.buf.push_back(static_cast<char*>(b));
  }
  return ASTR_OK;
}

bool file_io(int fd, char* p, size_t n, uint64_t off, bool write) {
  while (n) {
    ssize_t r = write ? ::pwrite(fd, p, n, off_t(off)) : ::pread(fd, p, n, off_t(off));
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    p += r; n -= size_t(r); off += uint64_t(r);
  }
  return true;
}

// Moves every piece between HBM and its file range in chunks of SLOT_BYTES: to the file, the
// calling thread queues device-to-host copies into free slots on the stream and host threads write
// each slot once its copy has completed; from the file, host threads read into free slots and
// queue the host-to-device copy of each. The copy engine, the file I/O of several chunks and the
// page cache work concurrently.
int transfer(const std::vector<Piece>& pieces, bool to_file, cudaStream_t st, std::string& err) {
  int dev = 0;
  cudaGetDevice(&dev);
  SlotPool& P = slot_pool();
  std::lock_guard<std::mutex> hold(P.m);
  const int nthreads = io_threads();
  const int nslots = 2 * nthreads;
  if (ensure_slots(P, nslots, err) != ASTR_OK) return ASTR_ERR_CUDA;
  std::vector<cudaEvent_t> ev(nslots, nullptr);
  for (cudaEvent_t& e : ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      for (cudaEvent_t& x : ev)
        if (x) cudaEventDestroy(x);
      return cuda_err(err, cudaGetLastError(), "transfer events");
    }
  struct Job { int slot; const Piece* pc; size_t at, bytes; };
  std::mutex qm;
  std::condition_variable qcv, freecv;
  std::deque<Job> queue;
  std::vector<int> free_slots;
  for (int k = 0; k < nslots; ++k) free_slots.push_back(k);
  bool closing = false;
  int code = ASTR_OK;
  std::string msg;
  auto failure = [&](int c, const std::string& m) {
    std::lock_guard<std::mutex> lk(qm);
    if (code == ASTR_OK) { code = c; msg = m; }
  };
  auto worker = [&]() {
    cudaSetDevice(dev);
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lk(qm);
        qcv.wait(lk, [&] { return closing || !queue.empty(); });
        if (queue.empty()) return;
        j = queue.front();
        queue.pop_front();
      }
      char* hb = P.buf[j.slot];
      if (to_file) {
        cudaError_t e = cudaEventSynchronize(ev[j.slot]);
        if (e != cudaSuccess) failure(ASTR_ERR_CUDA, std::string("flow-field download: ") + cudaGetErrorString(e));
        else if (!file_io(j.pc->fd, hb, j.bytes, j.pc->off + j.at, true))
          failure(ASTR_ERR_STATE, std::string("file write failed: ") + std::strerror(errno));
      } else if (!file_io(j.pc->fd, hb, j.bytes, j.pc->off + j.at, false)) {
        failure(ASTR_ERR_STATE, "file read failed (truncated file?)");
      } else {
        cudaError_t e = cudaMemcpyAsync(reinterpret_cast<char*>(j.pc->ddst) + j.at, hb, j.bytes,
                                        cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(ev[j.slot], st);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[j.slot]);
        if (e != cudaSuccess) failure(ASTR_ERR_CUDA, std::string("flow-field upload: ") + cudaGetErrorString(e));
      }
      {
        std::lock_guard<std::mutex> lk(qm);
        free_slots.push_back(j.slot);
      }
      freecv.notify_one();
    }
  };
  std::vector<std::thread> threads;
  for (int t = 0; t < nthreads; ++t) threads.emplace_back(worker);
  bool stop = false;
  for (const Piece& pc : pieces) {
    for (size_t at = 0; at < pc.bytes && !stop; at += SLOT_BYTES) {
      const size_t bytes = std::min(SLOT_BYTES, pc.bytes - at);
      int slot;
      {
        std::unique_lock<std::mutex> lk(qm);
        freecv.wait(lk, [&] { return !free_slots.empty(); });
        slot = free_slots.back();
        free_slots.pop_back();
        stop = code != ASTR_OK;
      }
      if (!stop && to_file) {
        cudaError_t e = cudaMemcpyAsync(P.buf[slot], reinterpret_cast<const char*>(pc.dsrc) + at, bytes,
                                        cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(ev[slot], st);
        if (e != cudaSuccess) {
          failure(ASTR_ERR_CUDA, std::string("flow-field download: ") + cudaGetErrorString(e));
          stop = true;
        }
      }
      std::lock_guard<std::mutex> lk(qm);
      if (stop) free_slots.push_back(slot);
      else queue.push_back({slot, &pc, at, bytes});
      qcv.notify_one();
    }
  }
  {
    std::lock_guard<std::mutex> lk(qm);
    closing = true;
  }
  qcv.notify_all();
  for (std::thread& t : threads) t.join();
  cudaStreamSynchronize(st);
  for (cudaEvent_t& e : ev) cudaEventDestroy(e);
  if (code != ASTR_OK) err = msg;
  return code;
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
  astr_h5* h = nullptr;
  int rc = astr_h5io_init(filename, "write", &h);
  if (rc != ASTR_OK) return h5_err(err, nullptr, rc);
  std::vector<Piece> pieces;
  for (int f = 0; f < 6 && rc == ASTR_OK; ++f) {
    Piece pc{-1, 0, dprims + (size_t)f * n, nullptr, (size_t)n * sizeof(double)};
    if ((rc = h5_reserve_r8(h, NAMES[f], 3, shape, &pc.fd, &pc.off)) != ASTR_OK) h5_err(err, h, rc);
    else pieces.push_back(pc);
  }
  if (rc == ASTR_OK) rc = transfer(pieces, true, st, err);
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
  const int rank = mode == 'h' ? 3 : 1;
  const int64_t* dims = mode == 'h' ? shape : &n;
  std::vector<Piece> pieces;
  std::vector<int> elementwise;
  if ((rc = astr_h5read_i4(h, "nstep", 1, &one, nullptr, 'h', &ns)) != ASTR_OK ||
      (rc = astr_h5read_r8(h, "time", 1, &one, nullptr, 'h', &t)) != ASTR_OK) {
    h5_err(err, h, rc);
  } else {
    for (int f = 0; f < 6; ++f) {
      // every field must be there with the state's shape before anything reaches the device
      int64_t fdims[32];
      int r = 0, cls = 0, size = 0;
      if ((rc = astr_h5_dataset_info(h, NAMES[f], &r, fdims, &cls, &size)) != ASTR_OK) { h5_err(err, h, rc); break; }
      Piece pc{-1, 0, nullptr, dprims + (size_t)f * n, (size_t)n * sizeof(double)};
      if (h5_locate_r8(h, NAMES[f], rank, dims, mode, &pc.fd, &pc.off) == ASTR_OK) pieces.push_back(pc);
      else elementwise.push_back(f);
    }
  }
  // datasets stored otherwise (other element type or byte order, compact storage): read through
  // the converting reader first, which also rejects a wrong shape before any transfer
  std::vector<double> tmp;
  for (size_t k = 0; k < elementwise.size() && rc == ASTR_OK; ++k) {
    const int f = elementwise[k];
    tmp.resize((size_t)n);
    if ((rc = astr_h5read_r8(h, NAMES[f], rank, dims, nullptr, mode, tmp.data())) != ASTR_OK) { h5_err(err, h, rc); break; }
    cudaError_t e = cudaMemcpyAsync(dprims + (size_t)f * n, tmp.data(), (size_t)n * sizeof(double),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_err(err, e, "flow-field upload");
  }
  if (rc == ASTR_OK) rc = transfer(pieces, false, st, err);
  astr_h5io_end(h);
  if (rc == ASTR_OK) {
    *nstep = ns;
    *time = t;
  }
  return rc;
}

bool host_pageable(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// Pageable host memory <-> device through the pinned slots: host thread t takes chunks t, t + T,
// ... and alternates between its two slots. To the device it copies a chunk into a slot and queues
// that slot's host-to-device copy, waiting for the slot's previous copy first; from the device it
// queues the device-to-host copy of a chunk into a slot, waits for it and copies the slot out. The
// threads' host copies overlap each other and the copy engine's transfers.
// Copies the node-row segments of elements [e0, e0 + n) from the slot to the caller's array.
void masked_out(char* dst, const char* slot, uint64_t e0, uint64_t n, const RowMask& m) {
  const uint64_t s0 = (uint64_t)m.s0, e1 = e0 + n;
  for (uint64_t r = e0 / s0; r * s0 < e1; ++r) {
    const int64_t j = (int64_t)(r % (uint64_t)m.s1), k = (int64_t)((r / (uint64_t)m.s1) % (uint64_t)m.s2);
    if (j < m.y_lo || j > m.y_hi || k < m.z_lo || k > m.z_hi) continue;
    const uint64_t a = std::max(e0, r * s0 + (uint64_t)m.x_lo), b = std::min(e1, r * s0 + (uint64_t)m.x_hi + 1);
    if (a < b) std::memcpy(dst + 8 * a, slot + 8 * (a - e0), 8 * (b - a));
  }
}

int staged_copy(void* dst, const void* src, size_t bytes, bool to_device, cudaStream_t st, std::string& err,
                const RowMask* mask) {
  int dev = 0;
  cudaGetDevice(&dev);
  SlotPool& P = slot_pool();
  std::lock_guard<std::mutex> hold(P.m);
  const int nthreads = io_threads();
  if (ensure_slots(P, 2 * nthreads, err) != ASTR_OK) return ASTR_ERR_CUDA;
  const size_t nchunks = (bytes + SLOT_BYTES - 1) / SLOT_BYTES;
  std::mutex em;
  int code = ASTR_OK;
  auto failure = [&](cudaError_t e, const char* what) {
    std::lock_guard<std::mutex> lk(em);
    if (code == ASTR_OK) code = cuda_err(err, e, what);
  };
  auto failed = [&]() {
    std::lock_guard<std::mutex> lk(em);
    return code != ASTR_OK;
  };
  auto worker = [&](int t) {
    cudaSetDevice(dev);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool busy[2] = {false, false};
    for (int k = 0; k < 2; ++k)
      if (cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess) {
        failure(cudaGetLastError(), "staging events");
        return;
      }
    int k = 0;
    for (size_t c = (size_t)t; c < nchunks && !failed(); c += (size_t)nthreads, k ^= 1) {
      char* slot = P.buf[2 * t + k];
      const size_t at = c * SLOT_BYTES, n = std::min(SLOT_BYTES, bytes - at);
      cudaError_t e = cudaSuccess;
      if (busy[k] && (e = cudaEventSynchronize(ev[k])) != cudaSuccess) { failure(e, "staged copy"); break; }
      busy[k] = false;
      if (to_device) {
        std::memcpy(slot, static_cast<const char*>(src) + at, n);
        e = cudaMemcpyAsync(static_cast<char*>(dst) + at, slot, n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k], st);
        busy[k] = e == cudaSuccess;
      } else {
        e = cudaMemcpyAsync(slot, static_cast<const char*>(src) + at, n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k], st);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[k]);
        if (e == cudaSuccess) {
          if (mask) masked_out(static_cast<char*>(dst), slot, at / 8, n / 8, *mask);
          else std::memcpy(static_cast<char*>(dst) + at, slot, n);
        }
      }
      if (e != cudaSuccess) { failure(e, "staged copy"); break; }
    }
    for (int j = 0; j < 2; ++j) {
      if (busy[j]) {
        cudaError_t e = cudaEventSynchronize(ev[j]);
        if (e != cudaSuccess) failure(e, "staged copy");
      }
      if (ev[j]) cudaEventDestroy(ev[j]);
    }
  };
  std::vector<std::thread> threads;
  for (int t = 0; t < nthreads; ++t) threads.emplace_back(worker, t);
  for (std::thread& th : threads) th.join();
  return code;
}

}  // namespace astr
