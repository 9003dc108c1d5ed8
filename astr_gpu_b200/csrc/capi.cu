// C-ABI implementation (include/astr_b200.h): contexts, schemes, the solver state, and the
// orchestration of the RK3 step as fused passes (one CUDA graph per step).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <array>
#include <vector>

#include "../../include/astr_b200.h"
#include "internal.h"
#include "tgv.cuh"
#include "adjoint.cuh"

using namespace astr;

struct astr_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  double* stage = nullptr;     // device staging of the line calls on host arrays (grows, kept)
  size_t stage_bytes = 0;
};

struct astr_scheme {
  astr_ctx* ctx = nullptr;
  HostOp h;
  DevOp d;
};

// Launch shape of one pass: solve layout (S rows per lane, WPL warps per line) and TI lines
// per CTA with tile pitch LP.
// FPS: fields per step of A', B' and the filters: 5 (all at once) or 1 (streamed one at a time)
struct PassCfg { int S = 0, WPL = 0, TI = 0, LP = 0, LPW = 1, FPS = 5; };
enum { CFG_A = 0, CFG_B, CFG_C, CFG_VA, CFG_VB, CFG_FC, CFG_FA, NCFG };
static const int CFG_PASS[NCFG] = {PASS_A, PASS_B, PASS_C, PASS_VA, PASS_VB, PASS_F, PASS_F};
static const int CFG_DIR[NCFG] = {DIR_A, DIR_B, DIR_C, DIR_A, DIR_B, DIR_C, DIR_A};

struct astr_state {
  astr_ctx* ctx = nullptr;
  astr_params p{};
  BoxGeo g{};
  Thermo th{};
  double* buf = nullptr;
  double *Q0 = nullptr, *Q1 = nullptr, *R = nullptr, *DA = nullptr, *DB = nullptr, *VF = nullptr;
  double* partials = nullptr;
  int nparts = 0;
  double* hist = nullptr;
  int* counter = nullptr;
  int* err = nullptr;
  int hist_cap = 1 << 16;
  HostOp hd[3], hf[3];                     // derivative and filter operators per direction
  std::map<int, std::pair<DevOp, DevOp>> ops;   // lane tables per (direction, layout)
  PassCfg cfg[NCFG];                       // launch shape of every pass
  bool autotune = true, tuned = false;
  bool pending = false;       // filter along DIR_A of the last stage not yet applied
  bool split_fa = false;      // that filter as its own streaming pass (else fused into pass A)
  int nstep = 0;
  double time = 0.0;
  std::vector<double> row_key;  // (nstep, time) per history row
  bool use_graph = true;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  double gdt[2] = {0.0, 0.0};
};

// One launch of the batched step: a pass over the boxes of one solve layout, or the batched
// diagnostics reduce (pass == 0).
struct EnsLaunch {
  int pass = 0, dir = 0, S = 0, WPL = 0, nbox = 0, nctas = 0, threads = 0;
  size_t smem = 0, args_off = 0, cum_off = 0;
};

struct astr_ensemble {
  astr_ctx* ctx = nullptr;
  std::vector<astr_state*> boxes;
  struct Group {
    int S = 0, WPL = 0;
    std::vector<int> members;
    int TI[NCFG] = {0};
  };
  std::vector<Group> groups;
  PassArgs* dargs = nullptr;
  int* dcum = nullptr;
  DiagArgs* ddiag = nullptr;
  std::vector<EnsLaunch> plan[2];   // per variant: filter along A owed at the start of the step or not
  std::vector<double> dt;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool pending = false;
  bool tuned = false;
};

namespace {

int fail(astr_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
int cuda_fail(astr_ctx* c, cudaError_t e, const char* where) {
  return fail(c, ASTR_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
// Makes a context's device current for the duration of one C-ABI call and restores the caller's
// device afterwards, so that allocations, launches and graph captures of a context whose device is
// not the caller's current one land on the right GPU. dev < 0 (a null handle) does nothing.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    int cur = -1;
    if (dev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// History rows written so far (the step counter may start elsewhere after a restart).
int hist_rows(const astr_state* st) { return (int)(st->row_key.size() / 2); }

#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

// Lines per CTA of a launch shape with `ntile` field tiles (shape_tiles) along a direction of dim
// + 1 nodes, solve layout (S, WPL): at most 512 threads and ~110 KB of tiles, so that two CTAs fit
// on an SM.
int pick_ti(int ntile, int dim, int WPL, int S, size_t budget = 110 * 1024) {
  int ti_thr = 512 / (WPL * 32);
  if (ti_thr < 1) ti_thr = 1;
  int ti = ti_thr > 16 ? 16 : ti_thr;
  if (WPL > 1 && ti > 8) ti = 8;   // one named barrier per line: at most 15 lines
  while (ti > 1) {
    const size_t bytes = (size_t)ntile * ti * tile_pitch(dim, ti, S) * 8;
    if (bytes <= budget) break;
    ti >>= 1;
  }
  return ti;
}

// Solve layouts compiled into the library (tgv_l*.cu, lines.cu).
const Layout kLayouts[] = {{3, 1}, {5, 1}, {9, 1}, {5, 2}, {9, 2}, {5, 4}, {9, 4}, {17, 1}};

bool covers(const int64_t* shape, const int64_t* lb, int d, int64_t lo, int64_t hi) {
  return lb[d] <= lo && lb[d] + shape[d] - 1 >= hi;
}

ArrDesc fortran_desc(const int64_t* shape, const int64_t* lb) {
  ArrDesc a;
  for (int d = 0; d < 3; ++d) { a.n[d] = shape[d]; a.lb[d] = lb[d]; }
  a.s[0] = 1;
  a.s[1] = shape[0];
  a.s[2] = shape[0] * shape[1];
  a.fs = shape[0] * shape[1] * shape[2];
  return a;
}

// A host array to device memory: large pageable arrays through the pinned staging slots.
int host_to_device(astr_ctx* ctx, double* dst, const double* src, size_t bytes) {
  if (bytes >= STAGED_MIN_BYTES && host_pageable(src)) return staged_copy(dst, src, bytes, true, ctx->stream, ctx->err);
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return ASTR_OK;
}

int line_call(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f, const int64_t* fsh, const int64_t* flb,
              double* out, const int64_t* osh, const int64_t* olb, int nfields, double scale, int where,
              int flags = 0) {
  if (!ctx || !s || !f || !out || !fsh || !flb || !osh || !olb) return fail(ctx, ASTR_ERR_ARG, "null argument");
  if (dir < 0 || dir > 2 || nfields < 1) return fail(ctx, ASTR_ERR_ARG, "bad dir or nfields");
  const int dim = s->h.dim;
  for (int d = 0; d < 3; ++d)
    if (fsh[d] < 1 || osh[d] < 1) return fail(ctx, ASTR_ERR_ARG, "empty extent");
  const bool interfaces = s->h.kind == OP_FLUX && !(flags & LINE_DIFF);
  if (interfaces) {
    if (!covers(osh, olb, dir, -1, dim)) return fail(ctx, ASTR_ERR_ARG, "output must cover interfaces -1..dim along dir");
  } else if (!covers(osh, olb, dir, 0, dim)) {
    return fail(ctx, ASTR_ERR_ARG, "output must cover nodes 0..dim along dir");
  }
  const int64_t lo = s->h.left_phys ? 0 : -5, hi = s->h.right_phys ? dim : dim + 5;
  if (s->h.kind != OP_EXPLICIT || s->h.ntype != 4)
    if (!covers(fsh, flb, dir, lo, hi)) return fail(ctx, ASTR_ERR_ARG, "input line must hold nodes -5..dim+5 (halo) along dir");
  for (int d = 0; d < 3; ++d) {
    if (d == dir) continue;
    if (!covers(fsh, flb, d, olb[d], olb[d] + osh[d] - 1)) return fail(ctx, ASTR_ERR_ARG, "output lines must lie inside the input");
  }
  ArrDesc fa = fortran_desc(fsh, flb), oa = fortran_desc(osh, olb);
  const double* df_ = f;
  double* dout = out;
  double *tf = nullptr, *to = nullptr;
  const size_t fb = (size_t)fa.fs * nfields * sizeof(double), ob = (size_t)oa.fs * nfields * sizeof(double);
  if (where == ASTR_HOST) {
    // the context's staging buffer holds the input and the output; it grows when a call needs
    // more and is kept for the next call (freed by astr_destroy)
    const size_t fpad = (fb + 255) / 256 * 256;
    if (ctx->stage_bytes < fpad + ob) {
      CK(cudaStreamSynchronize(ctx->stream));
      if (ctx->stage) cudaFree(ctx->stage);
      ctx->stage = nullptr;
      ctx->stage_bytes = 0;
      if (cudaMalloc(&ctx->stage, fpad + ob) != cudaSuccess) return fail(ctx, ASTR_ERR_NOMEM, "line call staging");
      ctx->stage_bytes = fpad + ob;
    }
    tf = ctx->stage;
    to = ctx->stage + fpad / sizeof(double);
    int rc = host_to_device(ctx, tf, f, fb);
    if (rc != ASTR_OK) return rc;
    // an output whose range along dir reaches past the entries the kernel writes (nodes 0..dim,
    // interfaces -1..dim) starts from the caller's values, so those entries come back unchanged
    const int64_t wlo = interfaces ? -1 : 0;
    if (olb[dir] < wlo || olb[dir] + osh[dir] - 1 > dim) {
      rc = host_to_device(ctx, to, out, ob);
      if (rc != ASTR_OK) return rc;
    }
    df_ = tf;
    dout = to;
  }
  cudaError_t e = launch_line_api(s->d, dir, df_, fa, dout, oa, nfields, scale, ctx->stream, flags);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "line kernel");
  if (where == ASTR_HOST) {
    if (ob >= STAGED_MIN_BYTES && host_pageable(out)) {
      const int rc = staged_copy(out, to, ob, false, ctx->stream, ctx->err);
      if (rc != ASTR_OK) return rc;
    } else {
      CK(cudaMemcpyAsync(out, to, ob, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return ASTR_OK;
}

std::pair<DevOp, DevOp>& get_ops(astr_state* st, int dir, int S, int WPL) {
  const int key = dir * 10000 + S * 100 + WPL;
  auto it = st->ops.find(key);
  if (it != st->ops.end()) return it->second;
  std::pair<DevOp, DevOp> o;
  make_devop(st->hd[dir], Layout{S, WPL}, o.first);
  make_devop(st->hf[dir], Layout{S, WPL}, o.second);
  return st->ops.emplace(key, o).first->second;
}

// Number of pass-C CTAs, i.e. of partial sums the diagnostics reduce.
int diag_parts(astr_state* st) {
  const int o1 = (DIR_C == 0) ? 1 : 0, o2 = (DIR_C == 2) ? 1 : 2;
  const int ti = st->cfg[CFG_C].TI;
  return (int)(((st->g.N[o1] + 1 + ti - 1) / ti) * (int64_t)(st->g.N[o2] + 1));
}

PassArgs base_args(astr_state* st, int id) {
  const PassCfg& pc = st->cfg[id];
  const int dir = CFG_DIR[id];
  auto& o = get_ops(st, dir, pc.S, pc.WPL);
  PassArgs a{};
  a.g = st->g;
  a.th = st->th;
  a.opd = o.first.op;
  a.opf = o.second.op;
  a.dir = dir;
  a.dA = DIR_A; a.dB = DIR_B; a.dC = DIR_C;
  a.TI = pc.TI;
  a.LP = pc.LP;
  a.LPW = pc.LPW;
  a.FPS = pc.FPS;
  a.R = st->R;
  a.VF = st->VF;
  a.err = st->err;
  return a;
}

// Optional per-pass event timing (astr_pass_timings); null in normal runs.
struct PassTimer {
  std::vector<cudaEvent_t> ev;   // pairs
  std::vector<int> kind;
};
thread_local PassTimer* g_timer = nullptr;

cudaError_t run_pass(astr_state* st, int id, PassArgs& a) {
  const int pass = CFG_PASS[id];
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (g_timer) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st->ctx->stream);
  }
  cudaError_t e = launch_pass(pass, a, st->cfg[id].S, st->cfg[id].WPL, st->ctx->stream);
  if (g_timer) {
    cudaEventRecord(e1, st->ctx->stream);
    g_timer->ev.push_back(e0);
    g_timer->ev.push_back(e1);
    g_timer->kind.push_back(id == CFG_FA ? 7 : (pass == PASS_F ? 5 : pass - 1));
  }
  return e;
}

// Filter along DIR_A still owed by the last stage.
cudaError_t finalize_filter(astr_state* st) {
  if (!st->pending) return cudaSuccess;
  PassArgs a = base_args(st, CFG_FA);
  a.q = st->Q0;
  cudaError_t e = run_pass(st, CFG_FA, a);
  if (e == cudaSuccess) st->pending = false;
  return e;
}

// rhscal of the state in q into R (no filter, no update).
cudaError_t run_rhs(astr_state* st, double* q) {
  PassArgs a = base_args(st, CFG_A);
  a.q = q; a.D = st->DA; a.do_filter = 0;
  cudaError_t e = run_pass(st, CFG_A, a);
  if (e != cudaSuccess) return e;
  a = base_args(st, CFG_B);
  a.q = q; a.D = st->DB;
  if ((e = run_pass(st, CFG_B, a)) != cudaSuccess) return e;
  a = base_args(st, CFG_C);
  a.q = q; a.DA = st->DA; a.DB = st->DB;
  if ((e = run_pass(st, CFG_C, a)) != cudaSuccess) return e;
  a = base_args(st, CFG_VA);
  a.q = q;
  if ((e = run_pass(st, CFG_VA, a)) != cudaSuccess) return e;
  a = base_args(st, CFG_VB);
  a.q = q;
  a.mode = 0;
  return run_pass(st, CFG_VB, a);
}

// One SSP-RK3 step (tgvsolver.F90:1037-1074): 6 passes per stage, diagnostics at stage 1.
cudaError_t run_step(astr_state* st, double dt, bool pending_at_start) {
  static const double rk[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  const int filt = st->p.filter_on;
  cudaError_t e;
  for (int s = 0; s < 3; ++s) {
    double* qin = (s == 0) ? st->Q0 : st->Q1;
    double* qout = (s == 2) ? st->Q0 : st->Q1;
    const bool owed = filt && (s > 0 || pending_at_start);   // the filter along A of the last stage
    if (owed && st->split_fa) {
      PassArgs f = base_args(st, CFG_FA);
      f.q = qin;
      if ((e = run_pass(st, CFG_FA, f)) != cudaSuccess) return e;
    }
    PassArgs a = base_args(st, CFG_A);
    a.q = qin; a.D = st->DA;
    a.do_filter = owed && !st->split_fa;
    if ((e = run_pass(st, CFG_A, a)) != cudaSuccess) return e;
    a = base_args(st, CFG_B);
    a.q = qin; a.D = st->DB;
    if ((e = run_pass(st, CFG_B, a)) != cudaSuccess) return e;
    a = base_args(st, CFG_C);
    a.q = qin; a.DA = st->DA; a.DB = st->DB;
    a.partials = (s == 0) ? st->partials : nullptr;
    if ((e = run_pass(st, CFG_C, a)) != cudaSuccess) return e;
    if (s == 0) {
      const double norm = (double)st->p.im * (double)st->p.jm * (double)st->p.km;
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (g_timer) { cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventRecord(e0, st->ctx->stream); }
      if ((e = launch_diag_reduce(st->partials, diag_parts(st), st->hist, st->counter, norm, st->ctx->stream)) != cudaSuccess)
        return e;
      if (g_timer) {
        cudaEventRecord(e1, st->ctx->stream);
        g_timer->ev.push_back(e0); g_timer->ev.push_back(e1); g_timer->kind.push_back(6);
      }
    }
    a = base_args(st, CFG_VA);
    a.q = qin;
    if ((e = run_pass(st, CFG_VA, a)) != cudaSuccess) return e;
    a = base_args(st, CFG_VB);
    a.q = qin; a.qsave = st->Q0; a.qout = qout;
    a.mode = 1; a.do_filter = filt;
    a.c1 = rk[s][0]; a.c2 = rk[s][1]; a.c3 = rk[s][2]; a.dt = dt;
    if ((e = run_pass(st, CFG_VB, a)) != cudaSuccess) return e;
    if (filt) {
      a = base_args(st, CFG_FC);
      a.q = qout;
      if ((e = run_pass(st, CFG_FC, a)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

int check_err(astr_state* st) {
  astr_ctx* ctx = st->ctx;
  int h = 0;
  CK(cudaMemcpyAsync(&h, st->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (h & 2) return fail(ctx, ASTR_ERR_CUDA, "a bulk copy into a tile did not complete within its wait limit");
  if (h) return fail(ctx, ASTR_ERR_STATE, "invalid state: non-finite or non-positive density (crashcheck)");
  return ASTR_OK;
}

int copy_fields(astr_state* st, double* dev, double* user, const int64_t* shape, const int64_t* lb, int to_state,
                int where) {
  astr_ctx* ctx = st->ctx;
  const int N[3] = {st->p.im, st->p.jm, st->p.km};
  for (int d = 0; d < 3; ++d)
    if (!covers(shape, lb, d, 0, N[d])) return fail(ctx, ASTR_ERR_ARG, "array must cover nodes 0..N on every axis");
  if (where == ASTR_DEVICE) {
    CK(launch_pack(st->g, dev, user, shape, lb, 5, to_state, ctx->stream));
    return ASTR_OK;
  }
  const size_t ufs = (size_t)(shape[0] * shape[1] * shape[2]);
  // A host array of exactly nodes 0..N moves as one contiguous copy through the stage buffer Q1
  // (free between steps), repacked to the padded state layout on the device: one large DMA instead
  // of 5 (N+1)^2 short rows.
  const bool exact = lb[0] == 0 && lb[1] == 0 && lb[2] == 0 && shape[0] == N[0] + 1 && shape[1] == N[1] + 1 &&
                     shape[2] == N[2] + 1;
  if (exact && dev != st->Q1) {
    const size_t bytes = 5 * ufs * sizeof(double);
    // large pageable arrays move through pinned staging slots with several host threads
    // (several times the rate of the driver's own staging of pageable memory)
    const bool staged = bytes >= STAGED_MIN_BYTES && host_pageable(user);
    if (to_state) {
      if (staged) {
        const int rc = staged_copy(st->Q1, user, bytes, true, ctx->stream, ctx->err);
        if (rc != ASTR_OK) return rc;
      } else {
        CK(cudaMemcpyAsync(st->Q1, user, bytes, cudaMemcpyHostToDevice, ctx->stream));
      }
      CK(launch_pack(st->g, dev, st->Q1, shape, lb, 5, 1, ctx->stream));
    } else {
      CK(launch_pack(st->g, dev, st->Q1, shape, lb, 5, 0, ctx->stream));
      if (staged) {
        const int rc = staged_copy(user, st->Q1, bytes, false, ctx->stream, ctx->err);
        if (rc != ASTR_OK) return rc;
      } else {
        CK(cudaMemcpyAsync(user, st->Q1, bytes, cudaMemcpyDeviceToHost, ctx->stream));
      }
    }
    return ASTR_OK;
  }
  // Other bounds (halos in the caller's array): a large pageable array moves whole through the
  // pinned staging slots into the stage buffers DA.. (18 fields, free between steps; never the
  // source or target, which is Q0, R or an adjoint buffer) and is repacked on the device; on the way
  // back only its node rows are written, so its halo entries stay as they were.
  const size_t ubytes = 5 * ufs * sizeof(double);
  if (ubytes >= STAGED_MIN_BYTES && 5 * ufs <= 18 * (size_t)st->g.fs && host_pageable(user)) {
    double* stage = st->DA;
    if (to_state) {
      const int rc = staged_copy(stage, user, ubytes, true, ctx->stream, ctx->err);
      if (rc != ASTR_OK) return rc;
      CK(launch_pack(st->g, dev, stage, shape, lb, 5, 1, ctx->stream));
    } else {
      CK(launch_pack(st->g, dev, stage, shape, lb, 5, 0, ctx->stream));
      const RowMask m{shape[0], shape[1], shape[2], -lb[0], N[0] - lb[0], -lb[1], N[1] - lb[1], -lb[2], N[2] - lb[2]};
      const int rc = staged_copy(user, stage, ubytes, false, ctx->stream, ctx->err, &m);
      if (rc != ASTR_OK) return rc;
    }
    return ASTR_OK;
  }
  for (int m = 0; m < 5; ++m) {
    cudaMemcpy3DParms prm{};
    cudaPitchedPtr hp = make_cudaPitchedPtr(user + m * ufs, (size_t)shape[0] * 8, (size_t)shape[0], (size_t)shape[1]);
    cudaPitchedPtr dp = make_cudaPitchedPtr(dev + m * st->g.fs, (size_t)st->g.st[1] * 8, (size_t)st->g.st[1], (size_t)N[1] + 1);
    cudaPos hpos = make_cudaPos((size_t)(-lb[0]) * 8, (size_t)(-lb[1]), (size_t)(-lb[2]));
    cudaPos dpos = make_cudaPos(0, 0, 0);
    prm.extent = make_cudaExtent((size_t)(N[0] + 1) * 8, (size_t)N[1] + 1, (size_t)N[2] + 1);
    if (to_state) { prm.srcPtr = hp; prm.srcPos = hpos; prm.dstPtr = dp; prm.dstPos = dpos; prm.kind = cudaMemcpyHostToDevice; }
    else { prm.srcPtr = dp; prm.srcPos = dpos; prm.dstPtr = hp; prm.dstPos = hpos; prm.kind = cudaMemcpyDeviceToHost; }
    CK(cudaMemcpy3DAsync(&prm, ctx->stream));
  }
  return ASTR_OK;
}

// Per-pass autotuner: every compiled solve layout that covers the longest system of the pass
// direction with at least half of its rows used, and two or three tile widths each, timed on
// scratch copies of the live state (the solution is not touched). Picks the fastest.
cudaError_t autotune(astr_state* st) {
  cudaStream_t sm = st->ctx->stream;
  cudaError_t e = cudaMemcpyAsync(st->Q1, st->Q0, 5 * (size_t)st->g.fs * sizeof(double), cudaMemcpyDeviceToDevice, sm);
  if (e != cudaSuccess) return e;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  // pass A is timed without and with the owed filter along A fused in; the filter goes into its
  // own pass F_A only where A + F_A beat the fused pass
  const bool filt = st->p.filter_on != 0;
  float tbest[NCFG], tfused = 1e30f;
  PassCfg fusedc = st->cfg[CFG_A];
  for (int id = 0; id < NCFG; ++id) {
    const int dir = CFG_DIR[id], pass = CFG_PASS[id];
    const int nsys = st->hf[dir].nsys();
    const int dim = st->g.N[dir];
    float best = 1e30f;
    PassCfg bestc = st->cfg[id];
    for (const Layout& L : kLayouts) {
      const int rows = 32 * L.WPL * L.S;
      if (rows < nsys || 2 * nsys < rows) continue;
      // (lines per CTA, lines per warp group, fields per step): A', B' and the filters also try
      // streaming one field at a time, and along y and z warps that loop over 2 lines of a wider
      // tile (rows of 8*TI contiguous bytes in each load)
      const bool streaming = pass == PASS_VA || pass == PASS_VB || pass == PASS_F;
      struct Shape { int ti, lpw, fps; };
      std::vector<Shape> shapes;
      for (int fps : {5, 1}) {
        if (fps == 1 && !streaming) continue;
        const int nt = shape_tiles(pass, 1, fps);
        for (int ti : {pick_ti(nt, dim, L.WPL, L.S), pick_ti(nt, dim, L.WPL, L.S) / 2, pick_ti(nt, dim, L.WPL, L.S, 220 * 1024)})
          if (ti >= 1) shapes.push_back({ti, 1, fps});
      }
      if (streaming && dir != 0)
        for (int ti : {8, 16})
          if (ti * L.WPL * 32 / 2 <= 512 && (L.WPL == 1 || ti / 2 <= 8)) shapes.push_back({ti, 2, 1});
      for (const Shape& sh : shapes) {
        const int ti = sh.ti;
        PassCfg c;
        c.S = L.S; c.WPL = L.WPL; c.TI = ti; c.LP = tile_pitch(dim, ti, L.S); c.LPW = sh.lpw; c.FPS = sh.fps;
        const PassCfg saved = st->cfg[id];
        st->cfg[id] = c;
        for (int fused = 0; fused < ((id == CFG_A && filt) ? 2 : 1); ++fused) {
          PassArgs a = base_args(st, id);
          a.q = st->Q1; a.D = st->DA; a.DA = st->DA; a.DB = st->DB;
          // stage 2-3 form of the update, reading q (the scratch copy) and qsave (the live state,
          // only read) from distinct arrays as the step does; values stay bounded: q <- (q + q) / 2
          a.qsave = st->Q0; a.qout = st->Q1; a.mode = 1; a.do_filter = (id == CFG_A) ? fused : st->p.filter_on;
          a.c1 = 0.5; a.c2 = 0.5; a.c3 = 0.0; a.dt = 0.0;
          float ms = 1e30f;
          if ((e = launch_pass(pass, a, c.S, c.WPL, sm)) == cudaSuccess) {
            cudaEventRecord(t0, sm);
            for (int r = 0; r < 4 && e == cudaSuccess; ++r) e = launch_pass(pass, a, c.S, c.WPL, sm);
            cudaEventRecord(t1, sm);
            cudaEventSynchronize(t1);
            cudaEventElapsedTime(&ms, t0, t1);
          }
          if (e != cudaSuccess) {   // a shape the device cannot launch (e.g. too much shared memory)
            cudaGetLastError();
            e = cudaSuccess;
            ms = 1e30f;
          }
          if (fused) {
            if (ms < tfused) { tfused = ms; fusedc = c; }
          } else if (ms < best) {
            best = ms; bestc = c;
          }
        }
        st->cfg[id] = saved;
      }
    }
    st->cfg[id] = bestc;
    tbest[id] = best;
  }
  st->split_fa = filt && tbest[CFG_A] + tbest[CFG_FA] < tfused;
  if (filt && !st->split_fa) st->cfg[CFG_A] = fusedc;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  e = cudaMemsetAsync(st->err, 0, sizeof(int), sm);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sm);
  st->tuned = true;
  return e;
}

void drop_graphs(astr_state* st) {
  for (auto& g : st->gexec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

}  // namespace

// Used by noalloc.cu.
cudaStream_t astr_ctx_stream(astr_ctx* ctx) { return ctx->stream; }
int astr_ctx_device(astr_ctx* ctx) { return ctx->device; }
void astr_ctx_set_error(astr_ctx* ctx, const char* msg) { ctx->err = msg; }

extern "C" {

int astr_init(int device, astr_ctx** out) {
  if (!out) return ASTR_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return ASTR_ERR_CUDA;
  if (device < 0 || device >= n) return ASTR_ERR_ARG;
  const DeviceGuard dg_(device);   // the stream belongs to `device`; the caller's device is restored
  astr_ctx* c = new (std::nothrow) astr_ctx();
  if (!c) return ASTR_ERR_NOMEM;
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return ASTR_ERR_CUDA; }
  c->own_stream = true;
  *out = c;
  return ASTR_OK;
}

int astr_destroy(astr_ctx* c) {
  const DeviceGuard dg_(c ? c->device : -1);
  if (!c) return ASTR_ERR_ARG;
  if (c->stage) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->stage);
  }
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return ASTR_OK;
}

const char* astr_last_error(astr_ctx* c) { return c ? c->err.c_str() : "null context"; }

int astr_set_stream(astr_ctx* ctx, void* s) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx) return ASTR_ERR_ARG;
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = (cudaStream_t)s;
  ctx->own_stream = false;
  return ASTR_OK;
}

int astr_synchronize(astr_ctx* ctx) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx) return ASTR_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_fd_scheme_create(astr_ctx* ctx, const char scheme[4], int ntype, int dim, astr_scheme** out) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx || !scheme || !out) return fail(ctx, ASTR_ERR_ARG, "null argument");
  astr_scheme* s = new astr_scheme();
  s->ctx = ctx;
  if (!build_fd_op(s->h, scheme, ntype, dim)) {
    delete s;
    return fail(ctx, ASTR_ERR_ARG, "scheme not defined (only 643c and 643e) or bad ntype/dim");
  }
  Layout lay = pick_layout(s->h.nsys());
  if (lay.S == 0) { delete s; return fail(ctx, ASTR_ERR_UNSUPPORTED, "line longer than 1152 rows"); }
  cudaError_t e = make_devop(s->h, lay, s->d);
  if (e != cudaSuccess) { free_devop(s->d); delete s; return cuda_fail(ctx, e, "scheme tables"); }
  *out = s;
  return ASTR_OK;
}

int astr_filter_create(astr_ctx* ctx, int ntype, int dim, double alpha_f, double beta_halo, double beta_bound,
                       int boundary_no_filter, astr_scheme** out) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx || !out) return fail(ctx, ASTR_ERR_ARG, "null argument");
  if (ntype < 1 || ntype > 4 || dim < 16) return fail(ctx, ASTR_ERR_ARG, "bad ntype or dim < 16");
  astr_scheme* s = new astr_scheme();
  s->ctx = ctx;
  build_filter_op(s->h, ntype, dim, alpha_f, beta_halo, beta_bound, boundary_no_filter != 0);
  Layout lay = pick_layout(s->h.nsys());
  if (lay.S == 0) { delete s; return fail(ctx, ASTR_ERR_UNSUPPORTED, "line longer than 1152 rows"); }
  cudaError_t e = make_devop(s->h, lay, s->d);
  if (e != cudaSuccess) { free_devop(s->d); delete s; return cuda_fail(ctx, e, "scheme tables"); }
  *out = s;
  return ASTR_OK;
}

int astr_flux_create(astr_ctx* ctx, int scheme, int ntype, int dim, char wind, double bfac, astr_scheme** out) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx || !out) return fail(ctx, ASTR_ERR_ARG, "null argument");
  if (wind != '+' && wind != '-') return fail(ctx, ASTR_ERR_ARG, "wind must be '+' or '-'");
  if (!std::isfinite(bfac)) return fail(ctx, ASTR_ERR_ARG, "bfac must be finite");
  astr_scheme* s = new astr_scheme();
  s->ctx = ctx;
  if (!build_flux_op(s->h, scheme, ntype, dim, wind == '+' ? 1 : -1, bfac)) {
    delete s;
    return fail(ctx, ASTR_ERR_ARG, "flux scheme not defined (only 543) or bad ntype/dim");
  }
  Layout lay = pick_layout(s->h.nsys());
  if (lay.S == 0) { delete s; return fail(ctx, ASTR_ERR_UNSUPPORTED, "line longer than 1152 rows"); }
  cudaError_t e = make_devop(s->h, lay, s->d);
  if (e != cudaSuccess) { free_devop(s->d); delete s; return cuda_fail(ctx, e, "scheme tables"); }
  *out = s;
  return ASTR_OK;
}

int astr_scheme_destroy(astr_scheme* s) {
  const DeviceGuard dg_(s && s->ctx ? s->ctx->device : -1);
  if (!s) return ASTR_ERR_ARG;
  free_devop(s->d);
  delete s;
  return ASTR_OK;
}

int astr_scheme_ac(const astr_scheme* s, double* ac, int* first_node, int* last_node) {
  if (!s || !ac) return ASTR_ERR_ARG;
  const int n = s->h.nsys();
  for (int r = 0; r < n; ++r) {
    ac[3 * r] = s->h.ac1[r];
    ac[3 * r + 1] = s->h.ac2[r];
    ac[3 * r + 2] = s->h.ac3[r];
  }
  if (first_node) *first_node = s->h.first_node;
  if (last_node) *last_node = s->h.last_node;
  return ASTR_OK;
}

int astr_deriv_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f, const int64_t f_shape[3],
                     const int64_t f_lbound[3], double* df, const int64_t df_shape[3], const int64_t df_lbound[3],
                     int nfields, double scale, int where) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (s && s->h.kind == OP_FILTER) return fail(ctx, ASTR_ERR_ARG, "scheme is a filter");
  return line_call(ctx, s, dir, f, f_shape, f_lbound, df, df_shape, df_lbound, nfields, scale, where);
}

int astr_filter_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f, const int64_t f_shape[3],
                      const int64_t f_lbound[3], double* ff, const int64_t ff_shape[3], const int64_t ff_lbound[3],
                      int nfields, int where) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (s && s->h.kind != OP_FILTER) return fail(ctx, ASTR_ERR_ARG, "scheme is not a filter");
  return line_call(ctx, s, dir, f, f_shape, f_lbound, ff, ff_shape, ff_lbound, nfields, 1.0, where);
}

int astr_flux_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f, const int64_t f_shape[3],
                    const int64_t f_lbound[3], double* fh, const int64_t fh_shape[3], const int64_t fh_lbound[3],
                    int nfields, int where) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (s && s->h.kind != OP_FLUX) return fail(ctx, ASTR_ERR_ARG, "scheme is not an interface flux");
  return line_call(ctx, s, dir, f, f_shape, f_lbound, fh, fh_shape, fh_lbound, nfields, 1.0, where);
}

int astr_flux_diff_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f, const int64_t f_shape[3],
                         const int64_t f_lbound[3], double* df, const int64_t df_shape[3], const int64_t df_lbound[3],
                         int nfields, double scale, int accumulate, int where) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (s && s->h.kind != OP_FLUX) return fail(ctx, ASTR_ERR_ARG, "scheme is not an interface flux");
  if (accumulate && where == ASTR_HOST) return fail(ctx, ASTR_ERR_ARG, "accumulate needs device arrays");
  return line_call(ctx, s, dir, f, f_shape, f_lbound, df, df_shape, df_lbound, nfields, scale, where,
                   LINE_DIFF | (accumulate ? LINE_ADD : 0));
}

int astr_state_create(astr_ctx* ctx, const astr_params* p, astr_state** out) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx || !p || !out) return fail(ctx, ASTR_ERR_ARG, "null argument");
  const int N[3] = {p->im, p->jm, p->km};
  for (int d = 0; d < 3; ++d)
    if (N[d] < 16) return fail(ctx, ASTR_ERR_ARG, "each dimension must be >= 16");
  for (int d = 0; d < 3; ++d)
    if (p->ntype[d] != 0 && p->ntype[d] != 3)
      return fail(ctx, ASTR_ERR_UNSUPPORTED, "the miniapp step is periodic: non-periodic boxes run in the full-solver mode (astr_full_create)");
  if (p->conschm != 0 && p->conschm != 643)
    return fail(ctx, ASTR_ERR_UNSUPPORTED, "the miniapp step is central (643): the upwind compact flux runs in the full-solver mode (astr_full_create)");
  astr_state* st = new astr_state();
  st->ctx = ctx;
  st->p = *p;
  const int64_t PX = ((int64_t)(N[0] + 1) + 15) / 16 * 16;
  st->g.N[0] = N[0]; st->g.N[1] = N[1]; st->g.N[2] = N[2];
  st->g.st[0] = 1;
  st->g.st[1] = PX;
  st->g.st[2] = PX * (N[1] + 1);
  st->g.fs = PX * (N[1] + 1) * (N[2] + 1);
  const double pi = 4.0 * std::atan(1.0);
  for (int d = 0; d < 3; ++d) st->g.rd[d] = 1.0 / (2.0 * pi / double(N[d]));
  const double g = p->gamma, m = p->mach;
  st->th.const2 = g * (m * m);
  st->th.const5 = (g - 1.0) * (m * m);
  st->th.const6 = 1.0 / (g - 1.0);
  st->th.gm1 = g - 1.0;
  st->th.inv_re = 1.0 / st->p.reynolds;
  st->th.inv_prc5 = 1.0 / (st->p.prandtl * st->th.const5);
  st->th.reynolds = p->reynolds;
  st->th.prandtl = p->prandtl;
  st->th.tc = p->sutherland / p->ref_tem;
  st->th.tc1 = 1.0 + st->th.tc;
  st->th.mach = m;
  // operators per direction and default launch shapes
  for (int d = 0; d < 3; ++d) {
    build_fd_op(st->hd[d], "643c", 3, N[d]);
    build_filter_op(st->hf[d], 3, N[d], p->alfa_filter, p->beta_halo, p->beta_bound, false);
    if (pick_layout(st->hf[d].nsys()).S == 0) { delete st; return fail(ctx, ASTR_ERR_UNSUPPORTED, "dimension too large (max 1145)"); }
  }
  for (int id = 0; id < NCFG; ++id) {
    const int d = CFG_DIR[id];
    const Layout L = pick_layout(st->hf[d].nsys());
    PassCfg& c = st->cfg[id];
    c.S = L.S; c.WPL = L.WPL;
    c.TI = pick_ti(pass_tiles(CFG_PASS[id]), N[d], L.WPL, L.S);
    c.LP = tile_pitch(N[d], c.TI, c.S);
  }
  // a small box gains nothing from tuning
  st->autotune = (N[0] + 1) * (int64_t)(N[1] + 1) * (N[2] + 1) >= 100 * 100 * 100;
  // 33 fields: Q0(5) Q1(5) R(5) DA(4) DB(4) VF(10: the combined fluxes along A and along B)
  const size_t nf = 33;
  cudaError_t e = cudaMalloc(&st->buf, nf * (size_t)st->g.fs * sizeof(double));
  if (e != cudaSuccess) { delete st; return fail(ctx, ASTR_ERR_NOMEM, "state allocation"); }
  cudaMemsetAsync(st->buf, 0, nf * (size_t)st->g.fs * sizeof(double), ctx->stream);
  st->Q0 = st->buf;
  st->Q1 = st->Q0 + 5 * st->g.fs;
  st->R = st->Q1 + 5 * st->g.fs;
  st->DA = st->R + 5 * st->g.fs;
  st->DB = st->DA + 4 * st->g.fs;
  st->VF = st->DB + 4 * st->g.fs;
  // partial sums of pass C: one per CTA
  const int o1 = (DIR_C == 0) ? 1 : 0, o2 = (DIR_C == 2) ? 1 : 2;
  st->nparts = (int)((N[o1] + 1) * (int64_t)(N[o2] + 1));   // one per CTA; at least one line per CTA
  if (cudaMalloc(&st->partials, (size_t)st->nparts * 3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&st->hist, (size_t)st->hist_cap * 3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&st->counter, 2 * sizeof(int)) != cudaSuccess) {
    astr_state_destroy(st);
    return fail(ctx, ASTR_ERR_NOMEM, "state allocation");
  }
  st->err = st->counter + 1;
  cudaMemsetAsync(st->counter, 0, 2 * sizeof(int), ctx->stream);
  *out = st;
  return ASTR_OK;
}

int astr_state_destroy(astr_state* st) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st) return ASTR_ERR_ARG;
  drop_graphs(st);
  for (auto& kv : st->ops) { free_devop(kv.second.first); free_devop(kv.second.second); }
  if (st->buf) cudaFree(st->buf);
  if (st->partials) cudaFree(st->partials);
  if (st->hist) cudaFree(st->hist);
  if (st->counter) cudaFree(st->counter);
  delete st;
  return ASTR_OK;
}

int astr_state_init_tgv(astr_state* st) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  const int N[3] = {st->p.im, st->p.jm, st->p.km};
  const double pi = 4.0 * std::atan(1.0);
  std::vector<double> tabs;
  for (int d = 0; d < 3; ++d) {
    std::vector<double> sv(N[d] + 1), cv(N[d] + 1), c2(N[d] + 1);
    for (int i = 0; i <= N[d]; ++i) {
      const double x = 2.0 * pi / double(N[d]) * double(i);   // tgvsolver.F90:208-210
      sv[i] = std::sin(x);
      cv[i] = std::cos(x);
      c2[i] = std::cos(2.0 * x);
    }
    tabs.insert(tabs.end(), sv.begin(), sv.end());
    tabs.insert(tabs.end(), cv.begin(), cv.end());
    tabs.insert(tabs.end(), c2.begin(), c2.end());
  }
  double* dt = nullptr;
  CK(cudaMalloc(&dt, tabs.size() * sizeof(double)));
  CK(cudaMemcpyAsync(dt, tabs.data(), tabs.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(launch_init_tgv(st->g, st->th, st->Q0, dt, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(dt);
  st->pending = false;
  st->nstep = 0;
  st->time = 0.0;
  st->row_key.clear();
  CK(cudaMemsetAsync(st->counter, 0, 2 * sizeof(int), ctx->stream));
  return ASTR_OK;
}

int astr_state_upload(astr_state* st, const double* q, const int64_t shape[3], const int64_t lbound[3], int where) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !q || !shape || !lbound) return ASTR_ERR_ARG;
  int rc = copy_fields(st, st->Q0, const_cast<double*>(q), shape, lbound, 1, where);
  if (rc) return rc;
  st->pending = false;
  astr_ctx* ctx = st->ctx;
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_state_download(astr_state* st, double* q, const int64_t shape[3], const int64_t lbound[3], int where) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !q || !shape || !lbound) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  CK(finalize_filter(st));
  int rc = copy_fields(st, st->Q0, q, shape, lbound, 0, where);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_state_write_flowfield(astr_state* st, const char* filename) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !filename) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  const int64_t shape[3] = {st->p.im + 1, st->p.jm + 1, st->p.km + 1}, lb[3] = {0, 0, 0};
  const int64_t n = shape[0] * shape[1] * shape[2];
  // q (5 x n) in R and the file's 6 primitive fields (6 x n) from DA on: stage buffers, free
  // between steps (R..VF hold 23 padded fields)
  double* dq = st->R;
  double* dprims = st->DA;
  int rc = astr_state_download(st, dq, shape, lb, ASTR_DEVICE);
  if (rc == ASTR_OK) {
    cudaError_t e = flowfield_prims_from_q(ctx->stream, dq, dprims, n, st->p.mach, st->p.gamma);
    rc = e != cudaSuccess ? cuda_fail(ctx, e, "q2fvar") : flowfield_write(ctx->stream, dprims, shape, st->nstep,
                                                                          st->time, filename, ctx->err);
  }
  return rc;
}

int astr_state_read_flowfield(astr_state* st, const char* filename, char mode, int* nstep, double* time) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !filename) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  const int64_t shape[3] = {st->p.im + 1, st->p.jm + 1, st->p.km + 1}, lb[3] = {0, 0, 0};
  const int64_t n = shape[0] * shape[1] * shape[2];
  double* dq = st->R;          // as in astr_state_write_flowfield
  double* dprims = st->DA;
  int ns = 0;
  double t = 0.0;
  int rc = flowfield_read(ctx->stream, dprims, shape, filename, mode, &ns, &t, ctx->err);
  if (rc == ASTR_OK) {
    cudaError_t e = flowfield_q_from_prims(ctx->stream, dprims, dq, n, st->p.mach, st->p.gamma);
    rc = e != cudaSuccess ? cuda_fail(ctx, e, "fvar2q") : astr_state_upload(st, dq, shape, lb, ASTR_DEVICE);
  }
  if (rc != ASTR_OK) return rc;
  st->nstep = ns;
  st->time = t;
  if (nstep) *nstep = ns;
  if (time) *time = t;
  return ASTR_OK;
}

int astr_cfl_dt(astr_state* st, double cfl, double* dt) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !dt) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  CK(finalize_filter(st));
  int np = 0;
  double* part = nullptr;
  CK(cudaMalloc(&part, 148 * 4 * 3 * sizeof(double)));
  CK(launch_cfl(st->g, st->th, st->Q0, part, &np, ctx->stream));
  std::vector<double> h((size_t)np * 3);
  CK(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(part);
  double m[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < np; ++b)
    for (int d = 0; d < 3; ++d) m[d] = std::max(m[d], h[3 * b + d]);
  *dt = cfl / (m[0] + m[1] + m[2]);
  return ASTR_OK;
}

int astr_rhs(astr_state* st, double* qrhs, const int64_t shape[3], const int64_t lbound[3], int where) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !qrhs) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  CK(finalize_filter(st));
  CK(run_rhs(st, st->Q0));
  int rc = copy_fields(st, st->R, qrhs, shape, lbound, 0, where);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return check_err(st);
}

int astr_state_autotune(astr_state* st, int on) {
  if (!st) return ASTR_ERR_ARG;
  st->autotune = on != 0;
  return ASTR_OK;
}

int astr_state_launch_shapes(astr_state* st, int shapes[42]) {
  if (!st || !shapes) return ASTR_ERR_ARG;
  for (int id = 0; id < NCFG; ++id) {
    shapes[6 * id] = st->cfg[id].S;
    shapes[6 * id + 1] = st->cfg[id].WPL;
    shapes[6 * id + 2] = st->cfg[id].TI;
    shapes[6 * id + 3] = st->cfg[id].LP;
    shapes[6 * id + 4] = st->cfg[id].LPW;
    shapes[6 * id + 5] = st->cfg[id].FPS;
  }
  return ASTR_OK;
}

int astr_state_set_launch_shape(astr_state* st, int pass, int S, int WPL, int TI, int LPW, int FPS) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || pass < 0 || pass >= NCFG) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  bool known = false;
  for (const Layout& L : kLayouts) known |= (L.S == S && L.WPL == WPL);
  const int dir = CFG_DIR[pass];
  if (!known || 32 * WPL * S < st->hf[dir].nsys()) return fail(ctx, ASTR_ERR_ARG, "layout not compiled or too short");
  if (TI < 1 || (TI & (TI - 1))) return fail(ctx, ASTR_ERR_ARG, "TI must be a power of 2");
  const int pk = CFG_PASS[pass];
  const bool loop_ok = dir != 0 && (pk == PASS_VA || pk == PASS_VB || pk == PASS_F);
  if (LPW < 1 || (LPW > 1 && (!loop_ok || TI % LPW != 0)))
    return fail(ctx, ASTR_ERR_ARG, "lines per warp: 1, or a divisor of TI for the y/z passes A', B' and filter-A");
  // a CTA runs (TI / LPW) line groups of WPL warps: at most 512 threads (the kernels' launch
  // bound), and with WPL > 1 one named barrier per group (ids 1..15)
  if ((TI / LPW) * WPL * 32 > 512 || (WPL > 1 && TI / LPW > 15))
    return fail(ctx, ASTR_ERR_ARG, "(TI / LPW) * WPL * 32 must be <= 512, and TI / LPW <= 15 when WPL > 1");
  const bool streaming = pk == PASS_VA || pk == PASS_VB || pk == PASS_F;
  if (FPS != 5 && !(FPS == 1 && streaming))
    return fail(ctx, ASTR_ERR_ARG, "fields per step: 5, or 1 for the passes A', B' and the filters");
  if (LPW > 1 && FPS != 1) return fail(ctx, ASTR_ERR_ARG, "lines per warp 2 streams one field per step");
  PassCfg c;
  c.S = S; c.WPL = WPL; c.TI = TI; c.LP = tile_pitch(st->g.N[dir], TI, S); c.LPW = LPW; c.FPS = FPS;
  st->cfg[pass] = c;
  st->autotune = false;
  drop_graphs(st);
  return ASTR_OK;
}

int astr_state_split_filter(astr_state* st, int on) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st) return ASTR_ERR_ARG;
  st->split_fa = on != 0;
  st->autotune = false;
  drop_graphs(st);
  return ASTR_OK;
}

int astr_state_use_graph(astr_state* st, int on) {
  if (!st) return ASTR_ERR_ARG;
  st->use_graph = on != 0;
  return ASTR_OK;
}

int astr_rk3_step(astr_state* st, double dt, int nsteps) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || nsteps < 0 || !(dt > 0.0)) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  if (hist_rows(st) + nsteps > st->hist_cap) return fail(ctx, ASTR_ERR_UNSUPPORTED, "history buffer full (65536 steps)");
  if (st->autotune && !st->tuned && nsteps > 0) {
    drop_graphs(st);
    CK(autotune(st));
  }
  for (int s = 0; s < nsteps; ++s) {
    const int variant = st->pending ? 1 : 0;
    st->row_key.push_back((double)st->nstep);
    st->row_key.push_back(st->time);
    if (st->use_graph) {
      if (!st->gexec[variant] || st->gdt[variant] != dt) {
        if (st->gexec[variant]) { cudaGraphExecDestroy(st->gexec[variant]); st->gexec[variant] = nullptr; }
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
        cudaError_t e = run_step(st, dt, variant == 1);
        cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "step capture");
        if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "cudaStreamEndCapture");
        CK(cudaGraphInstantiate(&st->gexec[variant], graph, 0));
        cudaGraphDestroy(graph);
        st->gdt[variant] = dt;
      }
      CK(cudaGraphLaunch(st->gexec[variant], ctx->stream));
    } else {
      CK(run_step(st, dt, variant == 1));
    }
    st->pending = st->p.filter_on != 0;
    st->nstep += 1;
    st->time = st->time + dt;
  }
  return check_err(st);
}

int astr_rk3_step_host(astr_state* st, double* q, const int64_t shape[3], const int64_t lbound[3], double dt,
                       int nsteps, double diag_out[3]) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !q) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  int rc = copy_fields(st, st->Q0, q, shape, lbound, 1, ASTR_HOST);
  if (rc) return rc;
  st->pending = false;
  rc = astr_rk3_step(st, dt, nsteps);
  if (rc) return rc;
  CK(finalize_filter(st));
  rc = copy_fields(st, st->Q0, q, shape, lbound, 0, ASTR_HOST);
  if (rc) return rc;
  if (diag_out && hist_rows(st) > 0) {
    CK(cudaMemcpyAsync(diag_out, st->hist + 3 * (size_t)(hist_rows(st) - 1), 3 * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_pass_timings(astr_state* st, double dt, int nsteps, double ms[8]) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !ms || nsteps < 1) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  if (hist_rows(st) + nsteps > st->hist_cap) return fail(ctx, ASTR_ERR_UNSUPPORTED, "history buffer full");
  PassTimer timer;
  g_timer = &timer;
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < nsteps && e == cudaSuccess; ++s) {
    st->row_key.push_back((double)st->nstep);
    st->row_key.push_back(st->time);
    e = run_step(st, dt, st->pending);
    st->pending = st->p.filter_on != 0;
    st->nstep += 1;
    st->time = st->time + dt;
  }
  g_timer = nullptr;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "timed step");
  CK(cudaStreamSynchronize(ctx->stream));
  double sum[8] = {0}, cnt[8] = {0};
  for (size_t i = 0; i < timer.kind.size(); ++i) {
    float t = 0.f;
    cudaEventElapsedTime(&t, timer.ev[2 * i], timer.ev[2 * i + 1]);
    sum[timer.kind[i]] += t;
    cnt[timer.kind[i]] += 1;
  }
  for (cudaEvent_t ev : timer.ev) cudaEventDestroy(ev);
  for (int k = 0; k < 8; ++k) ms[k] = cnt[k] > 0 ? sum[k] / cnt[k] : 0.0;
  return check_err(st);
}

int astr_history(astr_state* st, double* rows, int maxrows, int* nrows) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !nrows) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  const int n = hist_rows(st);
  *nrows = n;
  if (!rows || maxrows <= 0 || n == 0) return ASTR_OK;
  const int k = n < maxrows ? n : maxrows;
  std::vector<double> h((size_t)3 * k);
  CK(cudaMemcpyAsync(h.data(), st->hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int r = 0; r < k; ++r) {
    rows[5 * r] = st->row_key[2 * r];
    rows[5 * r + 1] = st->row_key[2 * r + 1];
    rows[5 * r + 2] = h[3 * r];
    rows[5 * r + 3] = h[3 * r + 1];
    rows[5 * r + 4] = h[3 * r + 2];
  }
  return ASTR_OK;
}

int astr_diagnostics(astr_state* st, double out[3]) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !out) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  CK(finalize_filter(st));
  // one gradient evaluation of the current state, reduced like stacal
  PassArgs a = base_args(st, CFG_A);
  a.q = st->Q0; a.D = st->DA; a.do_filter = 0;
  CK(run_pass(st, CFG_A, a));
  a = base_args(st, CFG_B);
  a.q = st->Q0; a.D = st->DB;
  CK(run_pass(st, CFG_B, a));
  a = base_args(st, CFG_C);
  a.q = st->Q0; a.DA = st->DA; a.DB = st->DB; a.partials = st->partials;
  CK(run_pass(st, CFG_C, a));
  int* cnt = nullptr;
  double* h = nullptr;
  CK(cudaMalloc(&cnt, sizeof(int)));
  CK(cudaMalloc(&h, 3 * sizeof(double)));
  CK(cudaMemsetAsync(cnt, 0, sizeof(int), ctx->stream));
  const double norm = (double)st->p.im * (double)st->p.jm * (double)st->p.km;
  CK(launch_diag_reduce(st->partials, diag_parts(st), h, cnt, norm, ctx->stream));
  CK(cudaMemcpyAsync(out, h, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(cnt);
  cudaFree(h);
  return check_err(st);
}

}  // extern "C"

// ====================================================================== batched ensemble
// Many independent periodic boxes of uneven sizes advanced together: boxes are grouped by the
// solve layout their size selects, and every pass of a stage is one launch per group whose
// CTAs walk the concatenated tile grids of the group's boxes (launch_pass_batch); the stage's
// diagnostics reduce is one launch for all boxes. Each ensemble step is one CUDA graph.
namespace {

void ens_drop_graphs(astr_ensemble* e) {
  for (auto& g : e->gexec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

void ens_free_plan(astr_ensemble* e) {
  if (e->dargs) cudaFree(e->dargs);
  if (e->dcum) cudaFree(e->dcum);
  if (e->ddiag) cudaFree(e->ddiag);
  e->dargs = nullptr; e->dcum = nullptr; e->ddiag = nullptr;
}

// Build the launch plans of both variants for the current dt and upload their arguments.
int ens_build(astr_ensemble* e) {
  astr_ctx* ctx = e->ctx;
  static const double rk[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  std::vector<PassArgs> hargs;
  std::vector<int> hcum;
  std::vector<DiagArgs> hdiag;
  for (astr_state* st : e->boxes) {
    DiagArgs d;
    d.partials = st->partials; d.nparts = 0; d.hist = st->hist; d.counter = st->counter;
    d.norm = (double)st->p.im * (double)st->p.jm * (double)st->p.km;
    hdiag.push_back(d);
  }
  const int slots[6] = {CFG_A, CFG_B, CFG_C, CFG_VA, CFG_VB, CFG_FC};
  // base_args reads a box's launch configuration: lend it the group's for the build only.
  std::vector<std::array<PassCfg, NCFG>> saved(e->boxes.size());
  for (size_t b = 0; b < e->boxes.size(); ++b)
    for (int id = 0; id < NCFG; ++id) saved[b][id] = e->boxes[b]->cfg[id];
  for (int variant = 0; variant < 2; ++variant) {
    e->plan[variant].clear();
    for (int s = 0; s < 3; ++s) {
      for (int si = 0; si < 6; ++si) {
        const int id = slots[si];
        for (auto& g : e->groups) {
          EnsLaunch L;
          L.pass = CFG_PASS[id]; L.dir = CFG_DIR[id]; L.S = g.S; L.WPL = g.WPL;
          L.nbox = (int)g.members.size();
          L.threads = g.TI[id] * g.WPL * 32;
          L.args_off = hargs.size();
          L.cum_off = hcum.size();
          int ctas = 0;
          for (int b : g.members) {
            astr_state* st = e->boxes[b];
            const int dir = CFG_DIR[id];
            PassCfg c;
            c.S = g.S; c.WPL = g.WPL; c.TI = g.TI[id]; c.LP = tile_pitch(st->g.N[dir], c.TI, g.S);
            st->cfg[id] = c;
            PassArgs a = base_args(st, id);
            double* qin = (s == 0) ? st->Q0 : st->Q1;
            double* qout = (s == 2) ? st->Q0 : st->Q1;
            const int filt = st->p.filter_on;
            switch (id) {
              case CFG_A: a.q = qin; a.D = st->DA; a.do_filter = filt && (s > 0 || variant == 1); break;
              case CFG_B: a.q = qin; a.D = st->DB; break;
              case CFG_C: a.q = qin; a.DA = st->DA; a.DB = st->DB; a.partials = (s == 0) ? st->partials : nullptr; break;
              case CFG_VA: a.q = qin; break;
              case CFG_VB:
                a.q = qin; a.qsave = st->Q0; a.qout = qout; a.mode = 1; a.do_filter = filt;
                a.c1 = rk[s][0]; a.c2 = rk[s][1]; a.c3 = rk[s][2]; a.dt = e->dt[b];
                break;
              case CFG_FC: a.q = qout; break;
              default: break;
            }
            hargs.push_back(a);
            hcum.push_back(ctas);
            const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
            ctas += ((st->g.N[o1] + 1 + c.TI - 1) / c.TI) * (st->g.N[o2] + 1);
            L.smem = std::max(L.smem, pass_shared_bytes(L.pass, c.TI, c.LP, g.WPL));
            if (id == CFG_C) hdiag[b].nparts = diag_parts(st);
          }
          L.nctas = ctas;
          if (id == CFG_FC && !e->boxes[0]->p.filter_on) continue;
          e->plan[variant].push_back(L);
        }
        if (s == 0 && id == CFG_C) {   // the stage-1 diagnostics of every box
          EnsLaunch L;
          L.pass = 0; L.nbox = (int)e->boxes.size();
          e->plan[variant].push_back(L);
        }
      }
    }
  }
  for (size_t b = 0; b < e->boxes.size(); ++b)
    for (int id = 0; id < NCFG; ++id) e->boxes[b]->cfg[id] = saved[b][id];
  ens_free_plan(e);
  CK(cudaMalloc(&e->dargs, hargs.size() * sizeof(PassArgs)));
  CK(cudaMalloc(&e->dcum, hcum.size() * sizeof(int)));
  CK(cudaMalloc(&e->ddiag, hdiag.size() * sizeof(DiagArgs)));
  CK(cudaMemcpy(e->dargs, hargs.data(), hargs.size() * sizeof(PassArgs), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e->dcum, hcum.data(), hcum.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e->ddiag, hdiag.data(), hdiag.size() * sizeof(DiagArgs), cudaMemcpyHostToDevice));
  return ASTR_OK;
}

cudaError_t ens_run(astr_ensemble* e, int variant) {
  cudaStream_t sm = e->ctx->stream;
  for (const EnsLaunch& L : e->plan[variant]) {
    cudaError_t err;
    if (L.pass == 0) err = launch_diag_reduce_batch(e->ddiag, L.nbox, sm);
    else err = launch_pass_batch(L.pass, L.dir, L.S, L.WPL, e->dargs + L.args_off, e->dcum + L.cum_off, L.nbox, L.nctas,
                                 L.threads, L.smem, sm);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

// Lines per CTA of each pass of each group: start from the largest power of two (<= 512
// threads) whose tiles fit in ~110 KB for every box of the group; with `timed`, also time the
// batched launch of each pass at that width, half and a quarter of it on scratch copies of the
// boxes' states (Q1) and keep the fastest.
int ens_tune(astr_ensemble* e, bool timed) {
  astr_ctx* ctx = e->ctx;
  for (auto& g : e->groups) {
    for (int id = 0; id < NCFG; ++id) {
      int ti = 16;
      for (int b : g.members) ti = std::min(ti, pick_ti(pass_tiles(CFG_PASS[id]), e->boxes[b]->g.N[CFG_DIR[id]], g.WPL, g.S));
      g.TI[id] = std::max(ti, 1);
    }
  }
  if (!timed) return ASTR_OK;
  cudaStream_t sm = ctx->stream;
  for (astr_state* st : e->boxes)
    CK(cudaMemcpyAsync(st->Q1, st->Q0, 5 * (size_t)st->g.fs * sizeof(double), cudaMemcpyDeviceToDevice, sm));
  PassArgs* dargs = nullptr;
  int* dcum = nullptr;
  CK(cudaMalloc(&dargs, e->boxes.size() * sizeof(PassArgs)));
  CK(cudaMalloc(&dcum, e->boxes.size() * sizeof(int)));
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int ids[6] = {CFG_A, CFG_B, CFG_C, CFG_VA, CFG_VB, CFG_FC};
  for (auto& g : e->groups) {
    for (int id : ids) {
      const int ti0 = g.TI[id];
      float best = 1e30f;
      int best_ti = ti0;
      for (int ti : {ti0, ti0 / 2, ti0 / 4}) {
        if (ti < 1) continue;
        std::vector<PassArgs> ha;
        std::vector<int> hc;
        int ctas = 0;
        size_t smem = 0;
        for (int b : g.members) {
          astr_state* st = e->boxes[b];
          const int dir = CFG_DIR[id];
          const PassCfg saved = st->cfg[id];
          PassCfg c;
          c.S = g.S; c.WPL = g.WPL; c.TI = ti; c.LP = tile_pitch(st->g.N[dir], ti, g.S);
          st->cfg[id] = c;
          PassArgs a = base_args(st, id);
          st->cfg[id] = saved;
          a.q = st->Q1; a.D = st->DA; a.DA = st->DA; a.DB = st->DB; a.partials = nullptr;
          // stage 2-3 form of the update: q (scratch) and qsave (live state, only read) distinct
          a.qsave = st->Q0; a.qout = st->Q1; a.mode = 1; a.do_filter = st->p.filter_on;
          a.c1 = 0.5; a.c2 = 0.5; a.c3 = 0.0; a.dt = 0.0;
          ha.push_back(a);
          hc.push_back(ctas);
          const int o1 = (dir == 0) ? 1 : 0, o2 = (dir == 2) ? 1 : 2;
          ctas += ((st->g.N[o1] + 1 + ti - 1) / ti) * (st->g.N[o2] + 1);
          smem = std::max(smem, pass_shared_bytes(CFG_PASS[id], ti, c.LP, g.WPL));
        }
        CK(cudaMemcpyAsync(dargs, ha.data(), ha.size() * sizeof(PassArgs), cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(dcum, hc.data(), hc.size() * sizeof(int), cudaMemcpyHostToDevice, sm));
        const int threads = ti * g.WPL * 32;
        float ms = 1e30f;
        cudaError_t err = launch_pass_batch(CFG_PASS[id], CFG_DIR[id], g.S, g.WPL, dargs, dcum, (int)ha.size(), ctas,
                                            threads, smem, sm);
        if (err == cudaSuccess) {
          cudaEventRecord(t0, sm);
          for (int r = 0; r < 2 && err == cudaSuccess; ++r)
            err = launch_pass_batch(CFG_PASS[id], CFG_DIR[id], g.S, g.WPL, dargs, dcum, (int)ha.size(), ctas, threads,
                                    smem, sm);
          cudaEventRecord(t1, sm);
          cudaEventSynchronize(t1);
          cudaEventElapsedTime(&ms, t0, t1);
        }
        if (err != cudaSuccess) { cudaGetLastError(); ms = 1e30f; }   // a width the device cannot launch
        if (ms < best) { best = ms; best_ti = ti; }
      }
      g.TI[id] = best_ti;
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(dargs);
  cudaFree(dcum);
  for (astr_state* st : e->boxes) CK(cudaMemsetAsync(st->err, 0, sizeof(int), sm));
  CK(cudaStreamSynchronize(sm));
  e->tuned = true;
  return ASTR_OK;
}

}  // namespace

extern "C" {

int astr_ensemble_create(astr_ctx* ctx, astr_state* const* boxes, int nbox, astr_ensemble** out) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx || !boxes || nbox < 1 || !out) return fail(ctx, ASTR_ERR_ARG, "null argument or empty ensemble");
  astr_ensemble* e = new astr_ensemble();
  e->ctx = ctx;
  for (int b = 0; b < nbox; ++b) {
    if (!boxes[b] || boxes[b]->ctx != ctx) { delete e; return fail(ctx, ASTR_ERR_ARG, "every box must belong to ctx"); }
    if (boxes[b]->p.filter_on != boxes[0]->p.filter_on) { delete e; return fail(ctx, ASTR_ERR_ARG, "mixed filter_on"); }
    e->boxes.push_back(boxes[b]);
  }
  for (int b = 0; b < nbox; ++b) {
    astr_state* st = boxes[b];
    int mx = 0;
    for (int d = 0; d < 3; ++d) mx = std::max(mx, st->hf[d].nsys());
    const Layout L = pick_layout(mx);
    bool found = false;
    for (auto& g : e->groups)
      if (g.S == L.S && g.WPL == L.WPL) { g.members.push_back(b); found = true; }
    if (!found) {
      astr_ensemble::Group g;
      g.S = L.S; g.WPL = L.WPL;
      g.members.push_back(b);
      e->groups.push_back(g);
    }
  }
  ens_tune(e, false);
  *out = e;
  return ASTR_OK;
}

int astr_ensemble_destroy(astr_ensemble* e) {
  const DeviceGuard dg_(e ? e->ctx->device : -1);
  if (!e) return ASTR_ERR_ARG;
  ens_drop_graphs(e);
  ens_free_plan(e);
  delete e;
  return ASTR_OK;
}

int astr_ensemble_step(astr_ensemble* e, const double* dt, int nsteps) {
  const DeviceGuard dg_(e ? e->ctx->device : -1);
  if (!e || !dt || nsteps < 0) return ASTR_ERR_ARG;
  astr_ctx* ctx = e->ctx;
  const int nbox = (int)e->boxes.size();
  for (int b = 0; b < nbox; ++b) {
    if (!(dt[b] > 0.0)) return fail(ctx, ASTR_ERR_ARG, "dt must be positive");
    if (hist_rows(e->boxes[b]) + nsteps > e->boxes[b]->hist_cap) return fail(ctx, ASTR_ERR_UNSUPPORTED, "history buffer full");
  }
  bool changed = e->dt.size() != (size_t)nbox;
  for (int b = 0; b < nbox && !changed; ++b) changed = e->dt[b] != dt[b];
  // The filter along A still owed by each box's last stage is applied by the first pass of
  // the step when every box owes it; otherwise the boxes that owe it apply it now.
  bool all_pending = true;
  for (int b = 0; b < nbox; ++b) all_pending = all_pending && e->boxes[b]->pending;
  if (!all_pending)
    for (int b = 0; b < nbox; ++b) CK(finalize_filter(e->boxes[b]));
  e->pending = all_pending;
  if (!e->tuned && nsteps > 0) {
    int rc = ens_tune(e, true);
    if (rc) return rc;
    changed = true;
  }
  if (changed) {
    e->dt.assign(dt, dt + nbox);
    ens_drop_graphs(e);
    int rc = ens_build(e);
    if (rc) return rc;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int variant = e->pending ? 1 : 0;
    for (int b = 0; b < nbox; ++b) {
      astr_state* st = e->boxes[b];
      st->row_key.push_back((double)st->nstep);
      st->row_key.push_back(st->time);
    }
    if (!e->gexec[variant]) {
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
      cudaError_t err = ens_run(e, variant);
      cudaError_t err2 = cudaStreamEndCapture(ctx->stream, &graph);
      if (err != cudaSuccess) return cuda_fail(ctx, err, "ensemble step capture");
      if (err2 != cudaSuccess) return cuda_fail(ctx, err2, "cudaStreamEndCapture");
      CK(cudaGraphInstantiate(&e->gexec[variant], graph, 0));
      cudaGraphDestroy(graph);
    }
    CK(cudaGraphLaunch(e->gexec[variant], ctx->stream));
    e->pending = e->boxes[0]->p.filter_on != 0;
    for (int b = 0; b < nbox; ++b) {
      astr_state* st = e->boxes[b];
      st->pending = e->pending;
      st->nstep += 1;
      st->time = st->time + dt[b];
    }
  }
  for (int b = 0; b < nbox; ++b) {
    int rc = check_err(e->boxes[b]);
    if (rc) return rc;
  }
  return ASTR_OK;
}

}  // extern "C"

// ====================================================================== discrete adjoint
// Gradient of J = <|rho u|^2 / (2 rho)> over nodes 1..N of the state after nsteps RK3 steps with
// respect to the initial conserved variables: checkpoints every `every` steps, each segment
// recomputed stage by stage (stage inputs kept), then reversed stage by stage.
struct astr_adjoint {
  astr_state* st = nullptr;
  int every = 20;
  AdjDevOp td[3], tf[3];        // transposed derivative / filter per direction
  PassCfg lcfg[3], gcfg[3];     // adjoint line kernels / gradient kernels per direction
  double* buf = nullptr;
  double *lam = nullptr, *lq = nullptr, *t1 = nullptr, *t2 = nullptr, *lnew = nullptr, *G = nullptr, *Y = nullptr,
         *lsave = nullptr, *U = nullptr, *lp = nullptr, *LG = nullptr, *part = nullptr, *jval = nullptr;
  std::vector<double*> ckpt;    // state at steps 0, every, 2*every, ...
  double* seg = nullptr;        // stage inputs of one segment: every x 3 states
  double* gstore = nullptr;     // their gradients (every x 3 x 12 fields) when memory allows
  int nsteps = 0;
  double dt = 0.0;
  double J = 0.0;
  bool have_forward = false;
};

namespace {

void adj_free(astr_adjoint* a) {
  for (int d = 0; d < 3; ++d) { free_adj_devop(a->td[d]); free_adj_devop(a->tf[d]); }
  if (a->buf) cudaFree(a->buf);
  a->buf = nullptr;
  for (double* c : a->ckpt) cudaFree(c);
  a->ckpt.clear();
  if (a->seg) cudaFree(a->seg);
  a->seg = nullptr;
  if (a->gstore) cudaFree(a->gstore);
  a->gstore = nullptr;
}

// One RK3 stage: qout = F(c1 qsave + c2 qin + c3 dt rhs(qin)) with the filter along A left
// owed, as in the time step: the next stage's first pass applies it to qout in place. With
// pending_in, qin still owes that filter and receives it here first (in place). With G, the
// velocity/temperature gradients of qin go to G[4d + k] (physical direction d, as the adjoint's
// gradient kernel lays them out).
cudaError_t run_stage_full(astr_state* st, int s, const double* qin, const double* qsave, double* qout, double dt,
                           double* G, bool pending_in) {
  static const double rk[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  double* qi = const_cast<double*>(qin);
  const int64_t fs = st->g.fs;
  double* DA = G ? G + 4 * DIR_A * fs : st->DA;
  double* DB = G ? G + 4 * DIR_B * fs : st->DB;
  cudaError_t e;
  const bool owed = pending_in && st->p.filter_on;
  if (owed && st->split_fa) {
    PassArgs f = base_args(st, CFG_FA);
    f.q = qi;
    if ((e = run_pass(st, CFG_FA, f)) != cudaSuccess) return e;
  }
  PassArgs a = base_args(st, CFG_A);
  a.q = qi; a.D = DA;
  a.do_filter = owed && !st->split_fa;
  if ((e = run_pass(st, CFG_A, a)) != cudaSuccess) return e;
  a = base_args(st, CFG_B);
  a.q = qi; a.D = DB;
  if ((e = run_pass(st, CFG_B, a)) != cudaSuccess) return e;
  a = base_args(st, CFG_C);
  a.q = qi; a.DA = DA; a.DB = DB; a.partials = nullptr;
  a.DC = G ? G + 4 * DIR_C * fs : nullptr;
  if ((e = run_pass(st, CFG_C, a)) != cudaSuccess) return e;
  a = base_args(st, CFG_VA);
  a.q = qi;
  if ((e = run_pass(st, CFG_VA, a)) != cudaSuccess) return e;
  a = base_args(st, CFG_VB);
  a.q = qi; a.qsave = qsave; a.qout = qout;
  a.mode = 1; a.do_filter = st->p.filter_on;
  a.c1 = rk[s][0]; a.c2 = rk[s][1]; a.c3 = rk[s][2]; a.dt = dt;
  if ((e = run_pass(st, CFG_VB, a)) != cudaSuccess) return e;
  if (st->p.filter_on) {
    a = base_args(st, CFG_FC);
    a.q = qout;
    if ((e = run_pass(st, CFG_FC, a)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

AdjLineArgs adj_line_args(astr_adjoint* A, int dir, bool filter, const double* in, double* out, int nf, double alpha,
                          bool acc) {
  astr_state* st = A->st;
  const AdjDevOp& op = filter ? A->tf[dir] : A->td[dir];
  AdjLineArgs a{};
  a.p.g = st->g;
  a.p.th = st->th;
  a.p.opd = op.tri.op;
  a.p.dir = dir;
  a.p.TI = A->lcfg[dir].TI;
  a.p.LP = A->lcfg[dir].LP;
  a.w = op.w;
  a.in = in;
  a.out = out;
  a.nf = nf;
  a.alpha = alpha;
  a.accumulate = acc ? 1 : 0;
  return a;
}

cudaError_t adj_lines(astr_adjoint* A, int dir, bool filter, const double* in, double* out, int nf, double alpha,
                      bool acc) {
  const AdjLineArgs a = adj_line_args(A, dir, filter, in, out, nf, alpha, acc);
  return launch_adj_lines(a, A->lcfg[dir].S, A->lcfg[dir].WPL, A->st->ctx->stream);
}

cudaError_t adj_grad(astr_adjoint* A, int dir, const double* q, double* D) {
  astr_state* st = A->st;
  const PassCfg& c = A->gcfg[dir];
  auto& o = get_ops(st, dir, c.S, c.WPL);
  PassArgs a{};
  a.g = st->g;
  a.th = st->th;
  a.opd = o.first.op;
  a.opf = o.second.op;
  a.dir = dir;
  a.dA = DIR_A; a.dB = DIR_B; a.dC = DIR_C;
  a.TI = c.TI;
  a.LP = c.LP;
  a.q = const_cast<double*>(q);
  a.D = D;
  a.err = st->err;
  return launch_adj_grad(a, c.S, c.WPL, st->ctx->stream);
}

// lam <- (d q_out / d q_in)^T lam for one RK3 step whose stage inputs are S0, S1, S2.
cudaError_t adj_step(astr_adjoint* A, const double* S0, const double* S1, const double* S2,
                     const double* const* Gs = nullptr) {
  static const double rk[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  astr_state* st = A->st;
  cudaStream_t sm = st->ctx->stream;
  const int64_t fs = st->g.fs;
  const double* Ss[3] = {S0, S1, S2};
  cudaError_t e;
  if ((e = cudaMemsetAsync(A->lsave, 0, 5 * fs * sizeof(double), sm)) != cudaSuccess) return e;
  for (int s = 2; s >= 0; --s) {
    const double* qs = Ss[s];
    const double c1 = rk[s][0], c2 = rk[s][1], c3 = rk[s][2];
    // filters: lam_new = F_A^T F_C^T F_B^T lam
    if (st->p.filter_on) {
      if ((e = adj_lines(A, DIR_B, true, A->lam, A->t1, 5, 1.0, false)) != cudaSuccess) return e;
      if ((e = adj_lines(A, DIR_C, true, A->t1, A->t2, 5, 1.0, false)) != cudaSuccess) return e;
      if ((e = adj_lines(A, DIR_A, true, A->t2, A->lnew, 5, 1.0, false)) != cudaSuccess) return e;
    } else {
      if ((e = cudaMemcpyAsync(A->lnew, A->lam, 5 * fs * sizeof(double), cudaMemcpyDeviceToDevice, sm)) != cudaSuccess)
        return e;
    }
    const double* Gq = Gs ? Gs[s] : A->G;
    for (int d = 0; d < 3; ++d) {
      if (!Gs && (e = adj_grad(A, d, qs, A->G + 4 * d * fs)) != cudaSuccess) return e;
      if ((e = adj_lines(A, d, false, A->lnew, A->Y + 5 * d * fs, 5, c3 * A->dt * st->g.rd[d], false)) != cudaSuccess)
        return e;
    }
    if ((e = launch_adj_point1(st->g, st->th, qs, Gq, A->Y, A->lnew, c1, c2, A->lsave, A->lq, A->U, A->lp, A->LG,
                               sm)) != cudaSuccess)
      return e;
    for (int d = 0; d < 3; ++d)
      if ((e = adj_lines(A, d, false, A->LG + 4 * d * fs, A->U, 4, st->g.rd[d], true)) != cudaSuccess) return e;
    if ((e = launch_adj_point2(st->g, st->th, qs, A->U, A->lp, A->lq, s == 0 ? A->lsave : nullptr, sm)) != cudaSuccess)
      return e;
    std::swap(A->lam, A->lq);
  }
  return cudaSuccess;
}

int adj_setup(astr_adjoint* A) {
  astr_state* st = A->st;
  astr_ctx* ctx = st->ctx;
  for (int d = 0; d < 3; ++d) {
    std::string err;
    AdjHostOp hd, hf;
    if (!build_adjoint_op(st->hd[d], hd, err) || !build_adjoint_op(st->hf[d], hf, err))
      return fail(ctx, ASTR_ERR_UNSUPPORTED, err);
    const Layout L = pick_layout(st->hf[d].nsys());
    if (L.S == 0) return fail(ctx, ASTR_ERR_UNSUPPORTED, "line too long for the adjoint layouts");
    CK(make_adj_devop(hd, L, A->td[d]));
    CK(make_adj_devop(hf, L, A->tf[d]));
    PassCfg lc;
    lc.S = L.S; lc.WPL = L.WPL;
    lc.TI = std::min(16, 512 / (32 * L.WPL));
    while (lc.TI > 1 && adj_lines_smem(lc.TI, tile_pitch(st->g.N[d], lc.TI, L.S), L.WPL) > 100 * 1024) lc.TI >>= 1;
    lc.LP = tile_pitch(st->g.N[d], lc.TI, L.S);
    A->lcfg[d] = lc;
    PassCfg gc;
    gc.S = L.S; gc.WPL = L.WPL;
    gc.TI = pick_ti(pass_tiles(PASS_A), st->g.N[d], L.WPL, L.S);
    gc.LP = tile_pitch(st->g.N[d], gc.TI, L.S);
    A->gcfg[d] = gc;
  }
  const int64_t fs = st->g.fs;
  const int nf = 5 * 5 + 12 + 15 + 5 + 4 + 1 + 12;
  CK(cudaMalloc(&A->buf, ((size_t)nf * fs + (st->g.N[2] + 1) + 8) * sizeof(double)));
  double* p = A->buf;
  auto take = [&](int n) { double* r = p; p += (size_t)n * fs; return r; };
  A->lam = take(5); A->lq = take(5); A->t1 = take(5); A->t2 = take(5); A->lnew = take(5);
  A->G = take(12); A->Y = take(15); A->lsave = take(5); A->U = take(4); A->lp = take(1); A->LG = take(12);
  A->part = p;
  A->jval = p + (st->g.N[2] + 1);
  CK(cudaMalloc(&A->seg, (size_t)A->every * 3 * 5 * fs * sizeof(double)));
  // keep the stage gradients of a segment from its recomputation when they fit in a quarter of
  // the free memory; otherwise the reverse sweep recomputes them stage by stage
  size_t free_b = 0, total_b = 0;
  const size_t need = (size_t)A->every * 3 * 12 * fs * sizeof(double);
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && need < free_b / 4) {
    if (cudaMalloc(&A->gstore, need) != cudaSuccess) { cudaGetLastError(); A->gstore = nullptr; }
  }
  return ASTR_OK;
}

}  // namespace

extern "C" {

int astr_adjoint_create(astr_state* st, int checkpoint_every, astr_adjoint** out) {
  const DeviceGuard dg_(st ? st->ctx->device : -1);
  if (!st || !out || checkpoint_every < 1) return ASTR_ERR_ARG;
  astr_adjoint* A = new astr_adjoint();
  A->st = st;
  A->every = checkpoint_every;
  int rc = adj_setup(A);
  if (rc) { adj_free(A); delete A; return rc; }
  *out = A;
  return ASTR_OK;
}

int astr_adjoint_destroy(astr_adjoint* A) {
  const DeviceGuard dg_(A ? A->st->ctx->device : -1);
  if (!A) return ASTR_ERR_ARG;
  adj_free(A);
  delete A;
  return ASTR_OK;
}

int astr_adjoint_forward(astr_adjoint* A, double dt, int nsteps, double* J) {
  const DeviceGuard dg_(A ? A->st->ctx->device : -1);
  if (!A || !(dt > 0.0) || nsteps < 1) return ASTR_ERR_ARG;
  astr_state* st = A->st;
  astr_ctx* ctx = st->ctx;
  const size_t qb = 5 * (size_t)st->g.fs * sizeof(double);
  // checkpoint buffers are kept across calls; the missing ones are allocated before any step
  const size_t nck = (size_t)((nsteps + A->every - 1) / A->every);
  while (A->ckpt.size() < nck) {
    double* c = nullptr;
    CK(cudaMalloc(&c, qb));
    A->ckpt.push_back(c);
  }
  CK(finalize_filter(st));
  for (int s0 = 0; s0 < nsteps; s0 += A->every) {
    double* c = A->ckpt[(size_t)(s0 / A->every)];
    CK(cudaMemcpyAsync(c, st->Q0, qb, cudaMemcpyDeviceToDevice, ctx->stream));
    const int n = std::min(A->every, nsteps - s0);
    int rc = astr_rk3_step(st, dt, n);
    if (rc) return rc;
    CK(finalize_filter(st));
  }
  CK(launch_kinetic_energy(st->g, st->Q0, A->part, A->jval, ctx->stream));
  CK(cudaMemcpyAsync(&A->J, A->jval, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  A->nsteps = nsteps;
  A->dt = dt;
  A->have_forward = true;
  if (J) *J = A->J;
  return check_err(st);
}

int astr_adjoint_backward(astr_adjoint* A, double* grad, const int64_t shape[3], const int64_t lbound[3], int where) {
  const DeviceGuard dg_(A ? A->st->ctx->device : -1);
  if (!A || !grad || !shape || !lbound) return ASTR_ERR_ARG;
  astr_state* st = A->st;
  astr_ctx* ctx = st->ctx;
  if (!A->have_forward) return fail(ctx, ASTR_ERR_STATE, "astr_adjoint_backward needs astr_adjoint_forward first");
  cudaStream_t sm = ctx->stream;
  const int64_t fs = st->g.fs;
  const size_t qb = 5 * (size_t)fs * sizeof(double);
  // dJ/dq at the final state (the state's Q0 after the forward run)
  CK(finalize_filter(st));
  CK(launch_adj_objective(st->g, st->Q0, A->lam, sm));
  const int nseg = (A->nsteps + A->every - 1) / A->every;
  for (int j = nseg - 1; j >= 0; --j) {
    const int s0 = j * A->every;
    const int len = std::min(A->every, A->nsteps - s0);
    auto stage = [&](int n, int s) { return A->seg + ((size_t)n * 3 + s) * 5 * fs; };
    auto grads = [&](int n, int s) -> double* {
      return A->gstore ? A->gstore + ((size_t)n * 3 + s) * 12 * fs : nullptr;
    };
    CK(cudaMemcpyAsync(stage(0, 0), A->ckpt[j], qb, cudaMemcpyDeviceToDevice, sm));
    for (int n = 0; n < len; ++n) {
      // every stage input receives the filter along A owed by the stage before it from its own
      // first pass (the checkpoint at n = 0 is fully filtered); the last step's third stage
      // still runs (into scratch) so that its input is filtered and its gradients are kept
      CK(run_stage_full(st, 0, stage(n, 0), stage(n, 0), stage(n, 1), A->dt, grads(n, 0), n > 0));
      CK(run_stage_full(st, 1, stage(n, 1), stage(n, 0), stage(n, 2), A->dt, grads(n, 1), true));
      CK(run_stage_full(st, 2, stage(n, 2), stage(n, 0), n + 1 < len ? stage(n + 1, 0) : A->t1, A->dt, grads(n, 2),
                        true));
    }
    for (int n = len - 1; n >= 0; --n) {
      const double* Gs[3] = {grads(n, 0), grads(n, 1), grads(n, 2)};
      CK(adj_step(A, stage(n, 0), stage(n, 1), stage(n, 2), A->gstore ? Gs : nullptr));
    }
  }
  int rc = copy_fields(st, A->lam, grad, shape, lbound, 0, where);
  if (rc) return rc;
  CK(cudaStreamSynchronize(sm));
  return check_err(st);
}

// lam_out = (d step / d q)^T lam_in for one RK3 step of size dt at the state's current q (the
// state is not advanced). Arrays hold 5 fields of nodes 0..N.
int astr_step_vjp(astr_adjoint* A, double dt, const double* lam_in, double* lam_out, const int64_t shape[3],
                  const int64_t lbound[3], int where) {
  const DeviceGuard dg_(A ? A->st->ctx->device : -1);
  if (!A || !lam_in || !lam_out || !shape || !lbound || !(dt > 0.0)) return ASTR_ERR_ARG;
  astr_state* st = A->st;
  astr_ctx* ctx = st->ctx;
  cudaStream_t sm = ctx->stream;
  const size_t qb = 5 * (size_t)st->g.fs * sizeof(double);
  CK(finalize_filter(st));
  double* S0 = A->seg;
  double* S1 = S0 + 5 * st->g.fs;
  double* S2 = S1 + 5 * st->g.fs;
  if (A->every < 1) return ASTR_ERR_ARG;
  CK(cudaMemcpyAsync(S0, st->Q0, qb, cudaMemcpyDeviceToDevice, sm));
  CK(run_stage_full(st, 0, S0, S0, S1, dt, nullptr, false));
  CK(run_stage_full(st, 1, S1, S0, S2, dt, nullptr, true));
  CK(run_stage_full(st, 2, S2, S0, A->t1, dt, nullptr, true));   // filters S2 in place
  int rc = copy_fields(st, A->lam, const_cast<double*>(lam_in), shape, lbound, 1, where);
  if (rc) return rc;
  const double keep = A->dt;
  A->dt = dt;
  cudaError_t e = adj_step(A, S0, S1, S2);
  A->dt = keep;
  CK(e);
  rc = copy_fields(st, A->lam, lam_out, shape, lbound, 0, where);
  if (rc) return rc;
  CK(cudaStreamSynchronize(sm));
  return ASTR_OK;
}

// out = scale * L^T g for every line along dir of nfields fields of nodes 0..N (periodic
// operators; device arrays of shape (n0, n1, n2) in Fortran order, fields contiguous).
int astr_scheme_apply_transpose(astr_ctx* ctx, astr_scheme* s, int dir, const double* g, const int64_t dims[3],
                                double* out, int nfields, double scale) {
  const DeviceGuard dg_(ctx ? ctx->device : -1);
  if (!ctx || !s || !g || !out || !dims || dir < 0 || dir > 2 || nfields < 1) return fail(ctx, ASTR_ERR_ARG, "bad argument");
  if (dims[dir] != s->h.dim + 1) return fail(ctx, ASTR_ERR_ARG, "dims[dir] must be dim+1");
  std::string err;
  AdjHostOp h;
  if (!build_adjoint_op(s->h, h, err)) return fail(ctx, ASTR_ERR_UNSUPPORTED, err);
  const Layout L = pick_layout(s->h.nsys());
  AdjDevOp op;
  CK(make_adj_devop(h, L, op));
  AdjLineArgs a{};
  a.p.g.N[0] = (int)dims[0] - 1; a.p.g.N[1] = (int)dims[1] - 1; a.p.g.N[2] = (int)dims[2] - 1;
  a.p.g.st[0] = 1; a.p.g.st[1] = dims[0]; a.p.g.st[2] = dims[0] * dims[1];
  a.p.g.fs = dims[0] * dims[1] * dims[2];
  a.p.opd = op.tri.op;
  a.p.dir = dir;
  a.p.TI = std::min(16, 512 / (32 * L.WPL));
  while (a.p.TI > 1 && adj_lines_smem(a.p.TI, tile_pitch(s->h.dim, a.p.TI, L.S), L.WPL) > 100 * 1024) a.p.TI >>= 1;
  a.p.LP = tile_pitch(s->h.dim, a.p.TI, L.S);
  a.w = op.w;
  a.in = g;
  a.out = out;
  a.nf = nfields;
  a.alpha = scale;
  a.accumulate = 0;
  cudaError_t e = launch_adj_lines(a, L.S, L.WPL, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  free_adj_devop(op);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "transposed line kernel");
  return ASTR_OK;
}

}  // extern "C"
