// C-ABI implementation (include/astr_b200.h): contexts, schemes, the solver state, and the
// orchestration of the RK3 step as fused passes (one CUDA graph per step).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/astr_b200.h"
#include "internal.h"
#include "tgv.cuh"

using namespace astr;

struct astr_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
};

struct astr_scheme {
  astr_ctx* ctx = nullptr;
  HostOp h;
  DevOp d;
};

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
  DevOp opd[3], opf[3];
  Layout lay[3]{};
  int TI[8][3]{};
  int LP[8][3]{};
  bool pending = false;       // filter along DIR_A of the last stage not yet applied
  int nstep = 0;
  double time = 0.0;
  std::vector<double> row_key;  // (nstep, time) per history row
  bool use_graph = true;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  double gdt[2] = {0.0, 0.0};
};

namespace {

int fail(astr_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
int cuda_fail(astr_ctx* c, cudaError_t e, const char* where) {
  return fail(c, ASTR_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

// Lines per CTA for a pass along a direction: at most 512 threads and ~110 KB of tiles so that
// two CTAs fit on an SM.
int pick_ti(int pass, int dim, int WPL) {
  int ti_thr = 512 / (WPL * 32);
  if (ti_thr < 1) ti_thr = 1;
  const int ntile = pass_tiles(pass);
  int ti = ti_thr > 16 ? 16 : ti_thr;
  while (ti > 1) {
    const size_t bytes = (size_t)ntile * ti * tile_pitch(dim, ti) * 8;
    if (bytes <= 110 * 1024) break;
    ti >>= 1;
  }
  return ti;
}

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

int line_call(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f, const int64_t* fsh, const int64_t* flb,
              double* out, const int64_t* osh, const int64_t* olb, int nfields, double scale, int where) {
  if (!ctx || !s || !f || !out || !fsh || !flb || !osh || !olb) return fail(ctx, ASTR_ERR_ARG, "null argument");
  if (dir < 0 || dir > 2 || nfields < 1) return fail(ctx, ASTR_ERR_ARG, "bad dir or nfields");
  const int dim = s->h.dim;
  for (int d = 0; d < 3; ++d)
    if (fsh[d] < 1 || osh[d] < 1) return fail(ctx, ASTR_ERR_ARG, "empty extent");
  if (!covers(osh, olb, dir, 0, dim)) return fail(ctx, ASTR_ERR_ARG, "output must cover nodes 0..dim along dir");
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
    CK(cudaMalloc(&tf, fb));
    CK(cudaMalloc(&to, ob));
    CK(cudaMemcpyAsync(tf, f, fb, cudaMemcpyHostToDevice, ctx->stream));
    df_ = tf;
    dout = to;
  }
  cudaError_t e = launch_line_api(s->d, dir, df_, fa, dout, oa, nfields, scale, ctx->stream);
  if (e != cudaSuccess) {
    if (tf) cudaFree(tf);
    if (to) cudaFree(to);
    return cuda_fail(ctx, e, "line kernel");
  }
  if (where == ASTR_HOST) {
    CK(cudaMemcpyAsync(out, to, ob, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(tf);
    cudaFree(to);
  }
  return ASTR_OK;
}

PassArgs base_args(astr_state* st, int pass, int dir) {
  PassArgs a{};
  a.g = st->g;
  a.th = st->th;
  a.opd = st->opd[dir].op;
  a.opf = st->opf[dir].op;
  a.dir = dir;
  a.dA = DIR_A; a.dB = DIR_B; a.dC = DIR_C;
  a.TI = st->TI[pass][dir];
  a.LP = st->LP[pass][dir];
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

cudaError_t run_pass(astr_state* st, int pass, PassArgs& a) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (g_timer) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st->ctx->stream);
  }
  cudaError_t e = launch_pass(pass, a, st->lay[a.dir].S, st->lay[a.dir].WPL, st->ctx->stream);
  if (g_timer) {
    cudaEventRecord(e1, st->ctx->stream);
    g_timer->ev.push_back(e0);
    g_timer->ev.push_back(e1);
    g_timer->kind.push_back(pass == PASS_F ? 5 : pass - 1);
  }
  return e;
}

// Filter along DIR_A still owed by the last stage.
cudaError_t finalize_filter(astr_state* st) {
  if (!st->pending) return cudaSuccess;
  PassArgs a = base_args(st, PASS_F, DIR_A);
  a.q = st->Q0;
  cudaError_t e = run_pass(st, PASS_F, a);
  if (e == cudaSuccess) st->pending = false;
  return e;
}

// rhscal of the state in q into R (no filter, no update).
cudaError_t run_rhs(astr_state* st, double* q) {
  PassArgs a = base_args(st, PASS_A, DIR_A);
  a.q = q; a.D = st->DA; a.do_filter = 0;
  cudaError_t e = run_pass(st, PASS_A, a);
  if (e != cudaSuccess) return e;
  a = base_args(st, PASS_B, DIR_B);
  a.q = q; a.D = st->DB;
  if ((e = run_pass(st, PASS_B, a)) != cudaSuccess) return e;
  a = base_args(st, PASS_C, DIR_C);
  a.q = q; a.DA = st->DA; a.DB = st->DB;
  if ((e = run_pass(st, PASS_C, a)) != cudaSuccess) return e;
  a = base_args(st, PASS_VA, DIR_A);
  if ((e = run_pass(st, PASS_VA, a)) != cudaSuccess) return e;
  a = base_args(st, PASS_VB, DIR_B);
  a.mode = 0;
  return run_pass(st, PASS_VB, a);
}

// One SSP-RK3 step (tgvsolver.F90:1037-1074): 6 passes per stage, diagnostics at stage 1.
cudaError_t run_step(astr_state* st, double dt, bool pending_at_start) {
  static const double rk[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  const int filt = st->p.filter_on;
  cudaError_t e;
  for (int s = 0; s < 3; ++s) {
    double* qin = (s == 0) ? st->Q0 : st->Q1;
    double* qout = (s == 2) ? st->Q0 : st->Q1;
    PassArgs a = base_args(st, PASS_A, DIR_A);
    a.q = qin; a.D = st->DA;
    a.do_filter = filt && (s > 0 || pending_at_start);
    if ((e = run_pass(st, PASS_A, a)) != cudaSuccess) return e;
    a = base_args(st, PASS_B, DIR_B);
    a.q = qin; a.D = st->DB;
    if ((e = run_pass(st, PASS_B, a)) != cudaSuccess) return e;
    a = base_args(st, PASS_C, DIR_C);
    a.q = qin; a.DA = st->DA; a.DB = st->DB;
    a.partials = (s == 0) ? st->partials : nullptr;
    if ((e = run_pass(st, PASS_C, a)) != cudaSuccess) return e;
    if (s == 0) {
      const double norm = (double)st->p.im * (double)st->p.jm * (double)st->p.km;
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (g_timer) { cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventRecord(e0, st->ctx->stream); }
      if ((e = launch_diag_reduce(st->partials, st->nparts, st->hist, st->counter, norm, st->ctx->stream)) != cudaSuccess)
        return e;
      if (g_timer) {
        cudaEventRecord(e1, st->ctx->stream);
        g_timer->ev.push_back(e0); g_timer->ev.push_back(e1); g_timer->kind.push_back(6);
      }
    }
    a = base_args(st, PASS_VA, DIR_A);
    if ((e = run_pass(st, PASS_VA, a)) != cudaSuccess) return e;
    a = base_args(st, PASS_VB, DIR_B);
    a.q = qin; a.qsave = st->Q0; a.qout = qout;
    a.mode = 1; a.do_filter = filt;
    a.c1 = rk[s][0]; a.c2 = rk[s][1]; a.c3 = rk[s][2]; a.dt = dt;
    if ((e = run_pass(st, PASS_VB, a)) != cudaSuccess) return e;
    if (filt) {
      a = base_args(st, PASS_F, DIR_C);
      a.q = qout;
      if ((e = run_pass(st, PASS_F, a)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

int check_err(astr_state* st) {
  astr_ctx* ctx = st->ctx;
  int h = 0;
  CK(cudaMemcpyAsync(&h, st->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
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

void drop_graphs(astr_state* st) {
  for (auto& g : st->gexec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

}  // namespace

extern "C" {

int astr_init(int device, astr_ctx** out) {
  if (!out) return ASTR_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return ASTR_ERR_CUDA;
  if (device < 0 || device >= n) return ASTR_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return ASTR_ERR_CUDA;
  astr_ctx* c = new (std::nothrow) astr_ctx();
  if (!c) return ASTR_ERR_NOMEM;
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return ASTR_ERR_CUDA; }
  c->own_stream = true;
  *out = c;
  return ASTR_OK;
}

int astr_destroy(astr_ctx* c) {
  if (!c) return ASTR_ERR_ARG;
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return ASTR_OK;
}

const char* astr_last_error(astr_ctx* c) { return c ? c->err.c_str() : "null context"; }

int astr_set_stream(astr_ctx* ctx, void* s) {
  if (!ctx) return ASTR_ERR_ARG;
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = (cudaStream_t)s;
  ctx->own_stream = false;
  return ASTR_OK;
}

int astr_synchronize(astr_ctx* ctx) {
  if (!ctx) return ASTR_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_fd_scheme_create(astr_ctx* ctx, const char scheme[4], int ntype, int dim, astr_scheme** out) {
  if (!ctx || !scheme || !out) return fail(ctx, ASTR_ERR_ARG, "null argument");
  astr_scheme* s = new astr_scheme();
  s->ctx = ctx;
  if (!build_fd_op(s->h, scheme, ntype, dim)) {
    delete s;
    return fail(ctx, ASTR_ERR_ARG, "scheme not defined (only 643c and 643e) or bad ntype/dim");
  }
  Layout lay = pick_layout(s->h.nsys());
  if (lay.S == 0) { delete s; return fail(ctx, ASTR_ERR_UNSUPPORTED, "line longer than 1280 rows"); }
  cudaError_t e = make_devop(s->h, lay, s->d);
  if (e != cudaSuccess) { free_devop(s->d); delete s; return cuda_fail(ctx, e, "scheme tables"); }
  *out = s;
  return ASTR_OK;
}

int astr_filter_create(astr_ctx* ctx, int ntype, int dim, double alpha_f, double beta_halo, double beta_bound,
                       int boundary_no_filter, astr_scheme** out) {
  if (!ctx || !out) return fail(ctx, ASTR_ERR_ARG, "null argument");
  if (ntype < 1 || ntype > 4 || dim < 16) return fail(ctx, ASTR_ERR_ARG, "bad ntype or dim < 16");
  astr_scheme* s = new astr_scheme();
  s->ctx = ctx;
  build_filter_op(s->h, ntype, dim, alpha_f, beta_halo, beta_bound, boundary_no_filter != 0);
  Layout lay = pick_layout(s->h.nsys());
  if (lay.S == 0) { delete s; return fail(ctx, ASTR_ERR_UNSUPPORTED, "line longer than 1280 rows"); }
  cudaError_t e = make_devop(s->h, lay, s->d);
  if (e != cudaSuccess) { free_devop(s->d); delete s; return cuda_fail(ctx, e, "scheme tables"); }
  *out = s;
  return ASTR_OK;
}

int astr_scheme_destroy(astr_scheme* s) {
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
  if (s && s->h.kind == OP_FILTER) return fail(ctx, ASTR_ERR_ARG, "scheme is a filter");
  return line_call(ctx, s, dir, f, f_shape, f_lbound, df, df_shape, df_lbound, nfields, scale, where);
}

int astr_filter_lines(astr_ctx* ctx, const astr_scheme* s, int dir, const double* f, const int64_t f_shape[3],
                      const int64_t f_lbound[3], double* ff, const int64_t ff_shape[3], const int64_t ff_lbound[3],
                      int nfields, int where) {
  if (s && s->h.kind != OP_FILTER) return fail(ctx, ASTR_ERR_ARG, "scheme is not a filter");
  return line_call(ctx, s, dir, f, f_shape, f_lbound, ff, ff_shape, ff_lbound, nfields, 1.0, where);
}

int astr_state_create(astr_ctx* ctx, const astr_params* p, astr_state** out) {
  if (!ctx || !p || !out) return fail(ctx, ASTR_ERR_ARG, "null argument");
  const int N[3] = {p->im, p->jm, p->km};
  for (int d = 0; d < 3; ++d)
    if (N[d] < 16) return fail(ctx, ASTR_ERR_ARG, "each dimension must be >= 16");
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
  st->th.reynolds = p->reynolds;
  st->th.prandtl = p->prandtl;
  st->th.tc = p->sutherland / p->ref_tem;
  st->th.tc1 = 1.0 + st->th.tc;
  st->th.mach = m;
  // operators and launch shapes per direction
  for (int d = 0; d < 3; ++d) {
    HostOp hd, hf;
    build_fd_op(hd, "643c", 3, N[d]);
    build_filter_op(hf, 3, N[d], p->alfa_filter, p->beta_halo, p->beta_bound, false);
    st->lay[d] = pick_layout(hf.nsys());
    if (st->lay[d].S == 0) { delete st; return fail(ctx, ASTR_ERR_UNSUPPORTED, "dimension too large (max 1273)"); }
    cudaError_t e1 = make_devop(hd, st->lay[d], st->opd[d]);
    cudaError_t e2 = make_devop(hf, st->lay[d], st->opf[d]);
    if (e1 != cudaSuccess || e2 != cudaSuccess) { delete st; return fail(ctx, ASTR_ERR_NOMEM, "scheme tables"); }
    for (int pass = 1; pass <= 6; ++pass) {
      st->TI[pass][d] = pick_ti(pass, N[d], st->lay[d].WPL);
      st->LP[pass][d] = tile_pitch(N[d], st->TI[pass][d]);
    }
  }
  // 30 fields: Q0(5) Q1(5) R(5) DA(4) DB(4) VF(7)
  const size_t nf = 30;
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
  const int ti = st->TI[PASS_C][DIR_C];
  const int o1 = (DIR_C == 0) ? 1 : 0, o2 = (DIR_C == 2) ? 1 : 2;
  st->nparts = (int)(((N[o1] + 1 + ti - 1) / ti) * (int64_t)(N[o2] + 1));
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
  if (!st) return ASTR_ERR_ARG;
  drop_graphs(st);
  for (int d = 0; d < 3; ++d) { free_devop(st->opd[d]); free_devop(st->opf[d]); }
  if (st->buf) cudaFree(st->buf);
  if (st->partials) cudaFree(st->partials);
  if (st->hist) cudaFree(st->hist);
  if (st->counter) cudaFree(st->counter);
  delete st;
  return ASTR_OK;
}

int astr_state_init_tgv(astr_state* st) {
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
  if (!st || !q || !shape || !lbound) return ASTR_ERR_ARG;
  int rc = copy_fields(st, st->Q0, const_cast<double*>(q), shape, lbound, 1, where);
  if (rc) return rc;
  st->pending = false;
  astr_ctx* ctx = st->ctx;
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_state_download(astr_state* st, double* q, const int64_t shape[3], const int64_t lbound[3], int where) {
  if (!st || !q || !shape || !lbound) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  CK(finalize_filter(st));
  int rc = copy_fields(st, st->Q0, q, shape, lbound, 0, where);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_cfl_dt(astr_state* st, double cfl, double* dt) {
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
  if (!st || !qrhs) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  CK(finalize_filter(st));
  CK(run_rhs(st, st->Q0));
  int rc = copy_fields(st, st->R, qrhs, shape, lbound, 0, where);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return check_err(st);
}

int astr_state_use_graph(astr_state* st, int on) {
  if (!st) return ASTR_ERR_ARG;
  st->use_graph = on != 0;
  return ASTR_OK;
}

int astr_rk3_step(astr_state* st, double dt, int nsteps) {
  if (!st || nsteps < 0 || !(dt > 0.0)) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  if (st->nstep + nsteps > st->hist_cap) return fail(ctx, ASTR_ERR_UNSUPPORTED, "history buffer full (65536 steps)");
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
  if (diag_out && st->nstep > 0) {
    CK(cudaMemcpyAsync(diag_out, st->hist + 3 * (size_t)(st->nstep - 1), 3 * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return ASTR_OK;
}

int astr_pass_timings(astr_state* st, double dt, int nsteps, double ms[7]) {
  if (!st || !ms || nsteps < 1) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  if (st->nstep + nsteps > st->hist_cap) return fail(ctx, ASTR_ERR_UNSUPPORTED, "history buffer full");
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
  double sum[7] = {0}, cnt[7] = {0};
  for (size_t i = 0; i < timer.kind.size(); ++i) {
    float t = 0.f;
    cudaEventElapsedTime(&t, timer.ev[2 * i], timer.ev[2 * i + 1]);
    sum[timer.kind[i]] += t;
    cnt[timer.kind[i]] += 1;
  }
  for (cudaEvent_t ev : timer.ev) cudaEventDestroy(ev);
  for (int k = 0; k < 7; ++k) ms[k] = cnt[k] > 0 ? sum[k] / cnt[k] : 0.0;
  return check_err(st);
}

int astr_history(astr_state* st, double* rows, int maxrows, int* nrows) {
  if (!st || !nrows) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  const int n = st->nstep;
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
  if (!st || !out) return ASTR_ERR_ARG;
  astr_ctx* ctx = st->ctx;
  CK(finalize_filter(st));
  // one gradient evaluation of the current state, reduced like stacal
  PassArgs a = base_args(st, PASS_A, DIR_A);
  a.q = st->Q0; a.D = st->DA; a.do_filter = 0;
  CK(run_pass(st, PASS_A, a));
  a = base_args(st, PASS_B, DIR_B);
  a.q = st->Q0; a.D = st->DB;
  CK(run_pass(st, PASS_B, a));
  a = base_args(st, PASS_C, DIR_C);
  a.q = st->Q0; a.DA = st->DA; a.DB = st->DB; a.partials = st->partials;
  CK(run_pass(st, PASS_C, a));
  int* cnt = nullptr;
  double* h = nullptr;
  CK(cudaMalloc(&cnt, sizeof(int)));
  CK(cudaMalloc(&h, 3 * sizeof(double)));
  CK(cudaMemsetAsync(cnt, 0, sizeof(int), ctx->stream));
  const double norm = (double)st->p.im * (double)st->p.jm * (double)st->p.km;
  CK(launch_diag_reduce(st->partials, st->nparts, h, cnt, norm, ctx->stream));
  CK(cudaMemcpyAsync(out, h, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(cnt);
  cudaFree(h);
  return check_err(st);
}

}  // extern "C"
