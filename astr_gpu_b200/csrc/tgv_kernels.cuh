// Pass kernels of the RK3 step (see tgv.cu for the pass structure). Included once per solve
// layout (S rows per lane, WPL warps per line) by tgv_l*.cu so the layouts compile in parallel.
//
// Thread roles in a CTA of TI lines x WPL warps:
//  * solve role: warp w works on line w / WPL, lanes own S consecutive rows (seg_solve);
//  * slot role (staging, pointwise work, stores): for x lines each line's 32*WPL threads walk
//    its contiguous nodes; for y/z lines consecutive threads take consecutive lines (TI adjacent
//    lines are contiguous in x) and walk the nodes with stride 32*WPL. Each thread keeps one
//    line in this role, so no index arithmetic beyond one multiply-add per node.
#pragma once
#include "tgv.cuh"

namespace astr {

namespace pass_detail {

template <int DIR, int WPL, bool LW = false>   // LW: warps may loop over lines (blockDim < TI*TPL)
struct TileCtx {
  static constexpr int o1 = (DIR == 0) ? 1 : 0;
  static constexpr int o2 = (DIR == 2) ? 1 : 2;
  static constexpr int TPL = 32 * WPL;   // threads per line (x lines)
  int dim, TI, LP;
  int sl, sn0;          // slot role: this thread's line and first node offset
  int nst;              // node stride of a slot: TPL, or blockDim / TI on y/z lines when LW
  bool svalid;          // that line exists
  int64_t sbase;        // element offset of node 0 of that line
  int64_t sd;
  __device__ __forceinline__ TileCtx(const PassArgs& a, int bx, int by) {
    dim = a.g.N[DIR];
    TI = a.TI;
    LP = a.LP;
    sd = a.g.st[DIR];
    if (DIR == 0) {
      sl = threadIdx.x / TPL;
      sn0 = threadIdx.x - sl * TPL;
      nst = TPL;
    } else {
      sl = threadIdx.x & (a.TI - 1);
      sn0 = threadIdx.x / a.TI;
      nst = LW ? (int)blockDim.x / a.TI : TPL;
    }
    const int64_t i1 = (int64_t)bx * a.TI + sl;
    svalid = i1 < a.g.N[o1] + 1;
    sbase = i1 * a.g.st[o1] + (int64_t)by * a.g.st[o2];
  }
  // f(tile offset of node n on the slot line, global offset) for n = n_lo.. n_hi
  template <class F>
  __device__ __forceinline__ void for_nodes(int n_lo, int n_hi, F f) const {
    const int tix0 = sl * LP + HT;
    for (int n = n_lo + sn0; n <= n_hi; n += nst) f(tix0 + n, n);
  }
  // Two-phase form for work that reads global memory: ld(n) -> P for NB nodes first (their
  // loads overlap), then use(tile offset, n, P) for the same nodes.
  template <int NB, class P, class Ld, class Use>
  __device__ __forceinline__ void for_nodes_batched(int n_lo, int n_hi, Ld ld, Use use) const {
    const int tix0 = sl * LP + HT;
    for (int nb = n_lo + sn0; nb <= n_hi; nb += NB * nst) {
      P r[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int n = nb + b * nst;
        if (n <= n_hi) r[b] = ld(n);
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int n = nb + b * nst;
        if (n <= n_hi) use(tix0 + n, n, r[b]);
      }
    }
  }
  // Two-phase form for read-modify-write of global fields: ld(n) for NB nodes first (their loads
  // overlap), then st(tile offset, n, loaded value).
  template <int NB, class Ld, class St>
  __device__ __forceinline__ void for_nodes_rmw(int n_lo, int n_hi, Ld ld, St st) const {
    const int tix0 = sl * LP + HT;
    for (int nb = n_lo + sn0; nb <= n_hi; nb += NB * nst) {
      double r[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int n = nb + b * nst;
        r[b] = (n <= n_hi) ? ld(n) : 0.0;
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int n = nb + b * nst;
        if (n <= n_hi) st(tix0 + n, n, r[b]);
      }
    }
  }
};

__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Wait until at most N committed groups of this thread are still in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void cp_async16(uint32_t sdst, const double* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sdst), "l"(gsrc) : "memory");
}

// Stage the slot line of one field, nodes -HT..dim+HT with the periodic wrap, asynchronously.
// The node progression of each thread runs through the low halo, the line and the high halo
// with the wrap applied per range; x lines (contiguous) copy node pairs with 16-byte copies
// when the line and the tile row start on 16-byte boundaries.
template <int DIR, int WPL, bool LW>
__device__ __forceinline__ void load_tile(const TileCtx<DIR, WPL, LW>& c, double* tile, const double* __restrict__ fld) {
  const int dim = c.dim;
  double* trow = tile + c.sl * c.LP + HT;   // node 0 of the slot line
  if (!c.svalid) {
    c.for_nodes(-HT, dim + HT, [&](int tix, int n) { tile[tix] = 1.0; });   // finite filler, never stored
    return;
  }
  const double* src = fld + c.sbase;
  const uint32_t s0 = (uint32_t)__cvta_generic_to_shared(trow);
  constexpr int TPL = TileCtx<DIR, WPL>::TPL;
  if (DIR == 0 && ((dim & 1) == 0) && ((c.LP & 1) == 0) && ((s0 & 15u) == 0)) {
    // pairs (n, n+1), n even, from -HT to dim+HT-1; then node dim+HT alone
    int n = -HT + 2 * c.sn0;
    for (; n < 0; n += 2 * TPL) cp_async16(s0 + 8 * n, src + (n + dim));
    for (; n + 1 <= dim; n += 2 * TPL) cp_async16(s0 + 8 * n, src + n);
    for (; n < dim + HT; n += 2 * TPL) {
      // the pair (dim, dim+1) straddles the wrap: node dim, then node 1
      if (n == dim) { cp_async8(trow + n, src + n); cp_async8(trow + n + 1, src + 1); }
      else cp_async16(s0 + 8 * n, src + (n - dim));
    }
    if (c.sn0 == 0) cp_async8(trow + dim + HT, src + HT);
    return;
  }
  const int64_t sd = c.sd;
  const int nst = c.nst;
  int n = -HT + c.sn0;
  for (; n < 0; n += nst) cp_async8(trow + n, src + (int64_t)(n + dim) * sd);
  for (; n <= dim; n += nst) cp_async8(trow + n, src + (int64_t)n * sd);
  for (; n <= dim + HT; n += nst) cp_async8(trow + n, src + (int64_t)(n - dim) * sd);
}

// ---- bulk copies completing on an mbarrier (the copy engine moves whole contiguous rows)
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Poll the barrier's phase `parity` at most `limit` times; false when it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit) {
  for (int it = 0; it < limit; ++it) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    if (done) return true;
  }
  return false;
}
constexpr int kBarrierPolls = 1 << 22;   // bounded wait (far beyond any copy's duration)

// Stage `nf` fields of the x lines of a tile with one bulk copy per line and field (nodes 0..dim
// are contiguous: one row of the padded box, 16-byte aligned), completing on one mbarrier; then
// the periodic halos -HT..-1 and dim+1..dim+HT are filled from the staged rows in shared memory.
// Needs an even tile pitch (16-byte aligned tile rows). A wait that does not complete sets bit 1
// of the error word; the kernel then runs to its end on whatever the tile holds.
template <int WPL>
__device__ __forceinline__ void stage_x_bulk(const TileCtx<0, WPL>& c, double* T, int tsz, const double* fld,
                                             int64_t fs, int nf, const PassArgs& a, int bx, int by, uint64_t* bar) {
  const int dim = c.dim;
  const unsigned bytes = (unsigned)(((dim + 1) * 8 + 15) & ~15);   // within the padded row
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    int nvalid = 0;
    for (int l = 0; l < c.TI; ++l) nvalid += ((int64_t)bx * c.TI + l < a.g.N[1] + 1) ? 1 : 0;
    mbar_arrive_expect_tx(bar, bytes * (unsigned)(nf * nvalid));
    for (int m = 0; m < nf; ++m)
      for (int l = 0; l < nvalid; ++l) {
        const int64_t row = ((int64_t)bx * c.TI + l) * a.g.st[1] + (int64_t)by * a.g.st[2];
        bulk_g2s(T + m * tsz + l * c.LP + HT, fld + m * fs + row, bytes, bar);
      }
  }
  if (!c.svalid) {
    for (int m = 0; m < nf; ++m) c.for_nodes(-HT, dim + HT, [&](int o, int) { T[m * tsz + o] = 1.0; });
  }
  if (!mbar_wait(bar, 0, kBarrierPolls) && threadIdx.x == 0) atomicOr(a.err, 2);
  if (c.svalid) {
    for (int m = 0; m < nf; ++m) {
      double* row = T + m * tsz + c.sl * c.LP + HT;
      for (int k = 1 + c.sn0; k <= HT; k += c.nst) {
        row[-k] = row[dim - k];
        row[dim + k] = row[k];
      }
    }
  }
}

// Write a lane's solution rows (nodes 0..dim) into a tile line, optionally with the periodic
// halo images of those nodes.
template <int S>
__device__ __forceinline__ void put_lane(double* line, const double (&v)[S], int seg, int ext, int dim, bool images) {
  const int n0 = seg * S - ext;
#pragma unroll
  for (int t = 0; t < S; ++t) {
    const int n = n0 + t;
    if ((unsigned)n > (unsigned)dim) continue;   // outside nodes 0..dim
    line[n] = v[t];
    if (images) {
      if (n >= 1 && n <= HT) line[dim + n] = v[t];
      if (n >= dim - HT && n <= dim - 1) line[n - dim] = v[t];
    }
  }
}

__device__ __forceinline__ void put_images(double* line, int n, int dim, double v) {
  if (n >= 1 && n <= HT) line[dim + n] = v;
  if (n >= dim - HT && n <= dim - 1) line[n - dim] = v;
}

// q -> (rho, u, v, w, p) in place over every staged node of the 5 tiles (q2fvar,
// tgvsolver.F90:92-121), once per node.
// With TEMP, tile 4 receives the temperature p/rho * gamma M^2 instead of the pressure (the
// gradient passes need only u, v, w, T). One reciprocal of rho per node; the results equal
// q2fvar's divisions to within an ulp.
template <int DIR, int WPL, bool TEMP = false, bool LW = false>
__device__ __forceinline__ void to_prims(const TileCtx<DIR, WPL, LW>& c, double* T, int tsz, const Thermo& th) {
  c.for_nodes(-HT, c.dim + HT, [&](int o, int) {
    const double q0 = T[o], q1 = T[tsz + o], q2 = T[2 * tsz + o], q3 = T[3 * tsz + o], q4 = T[4 * tsz + o];
    const double ri = 1.0 / q0;
    const double u = q1 * ri, v = q2 * ri, w = q3 * ri;
    const double p = (q4 - 0.5 * q0 * (u * u + v * v + w * w)) * th.gm1;
    T[tsz + o] = u;
    T[2 * tsz + o] = v;
    T[3 * tsz + o] = w;
    T[4 * tsz + o] = TEMP ? p * ri * th.const2 : p;
  });
}

// Pointwise function K of the primitive tiles at node n of a line (L = tile 0 of the line):
// 0..2 velocity, 3 temperature, 4..8 the Euler flux along DIR (convection,
// tgvsolver.F90:559-564; q_m = rho*u_m and E = p/(gamma-1) + rho|u|^2/2 as fvar2q rebuilds them).
template <int K, int DIR>
__device__ __forceinline__ double gprim(const double* L, int tsz, int n, const Thermo& th) {
  if (K < 3) return L[(K + 1) * tsz + n];
  if (K == 3) return L[4 * tsz + n] / L[n] * th.const2;
  const double rho = L[n];
  const double ud = L[(1 + DIR) * tsz + n];
  constexpr int m = K - 4;
  if (m == 0) return rho * ud;
  if (m <= 3) {
    const double f = rho * L[m * tsz + n] * ud;
    return (m - 1 == DIR) ? f + L[4 * tsz + n] : f;
  }
  const double u = L[tsz + n], v = L[2 * tsz + n], w = L[3 * tsz + n], p = L[4 * tsz + n];
  const double E = p * th.const6 + rho * (0.5 * (u * u + v * v + w * w));
  return (E + p) * ud;
}

template <int DIR>
__device__ __forceinline__ double gprim_rt(int K, const double* L, int tsz, int n, const Thermo& th) {
  switch (K) {
    case 0: return gprim<0, DIR>(L, tsz, n, th);
    case 1: return gprim<1, DIR>(L, tsz, n, th);
    case 2: return gprim<2, DIR>(L, tsz, n, th);
    case 3: return gprim<3, DIR>(L, tsz, n, th);
    case 4: return gprim<4, DIR>(L, tsz, n, th);
    case 5: return gprim<5, DIR>(L, tsz, n, th);
    case 6: return gprim<6, DIR>(L, tsz, n, th);
    case 7: return gprim<7, DIR>(L, tsz, n, th);
    default: return gprim<8, DIR>(L, tsz, n, th);
  }
}

// Window of pointwise function K (branch once per solve, not per node).
template <int W, int S, int DIR>
__device__ __forceinline__ void prim_window(double (&w)[W], int K, const double* L, int tsz, int n0, int dim,
                                            const Thermo& th) {
  switch (K) {
    case 0: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<0, DIR>(L, tsz, n, th); }); break;
    case 1: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<1, DIR>(L, tsz, n, th); }); break;
    case 2: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<2, DIR>(L, tsz, n, th); }); break;
    case 3: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<3, DIR>(L, tsz, n, th); }); break;
    case 4: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<4, DIR>(L, tsz, n, th); }); break;
    case 5: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<5, DIR>(L, tsz, n, th); }); break;
    case 6: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<6, DIR>(L, tsz, n, th); }); break;
    case 7: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<7, DIR>(L, tsz, n, th); }); break;
    default: fill_window<W, S>(w, n0, dim, [&](int n) { return gprim<8, DIR>(L, tsz, n, th); }); break;
  }
}

__device__ __forceinline__ int sidx(int a, int b) {
  // symmetric 3x3 stored as (11,12,13,22,23,33)
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

__device__ __forceinline__ double miucal(const Thermo& th, double t) {
  return t * sqrt(t) * th.tc1 / (t + th.tc);
}

struct LaneIds {
  int warp, lane, l, part, seg;
};
template <int WPL>
__device__ __forceinline__ LaneIds lane_ids() {
  LaneIds z;
  z.warp = threadIdx.x >> 5;
  z.lane = threadIdx.x & 31;
  z.l = z.warp / WPL;
  z.part = z.warp - z.l * WPL;
  z.seg = z.part * 32 + z.lane;
  return z;
}


// Closure-row RHS values of `ns` pending solves on every line of the tile, computed up front by
// a few threads so that no warp diverges on closure rows during its solve:
// sp[(l*ns + k)*2*NSP + j] for line l, solve k. getk(l, k, n) = input of solve k at node n.
template <int KIND = -1, class GetK>
__device__ __forceinline__ void compute_specials(const LineOp& op, int TI, double* sp, int ns, GetK getk) {
  const int per = 2 * NSP;
  for (int it = threadIdx.x; it < TI * ns * per; it += blockDim.x) {
    const int j = it % per, lk = it / per;
    const int k = lk % ns, l = lk / ns;
    const bool lo = j < NSP;
    if (lo ? (j >= op.spec_lo) : (j - NSP >= op.spec_hi)) continue;
    const int r = lo ? j : op.nsys - op.spec_hi + (j - NSP);
    sp[(l * ns + k) * per + j] = special_value<false, KIND>(op, r, [&](int n) { return getk(l, k, n); });
  }
}

// Derivatives of pointwise functions K0..K0+NV-1 along DIR for this lane's rows, solved together
// (scaled by 1/dx).
template <int S, int WPL, int DIR, int NV>
__device__ __forceinline__ void dsolve_n(double (&v)[NV][S], int K0, const PassArgs& a, const LaneIds& z,
                                         const double* L0, int tsz, double* scl, double rd, const double* sp) {
  const LineOp& op = a.opd;
  const int r0 = z.seg * S;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double w[S + 4];
    prim_window<S + 4, S, DIR>(w, K0 + i, L0, tsz, r0 - op.ext_lo - 2, op.dim, a.th);
    stencil_deriv<S>(v[i], w);
    apply_specials<S>(v[i], op, r0, sp + i * 2 * NSP);
  }
  seg_solve_n<S, WPL, NV>(v, op.tab, z.seg, z.lane, z.part, z.l, scl);
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int t = 0; t < S; ++t) v[i][t] *= rd;
}

// Solves of NV staged tile lines (derivative or filter) in place, together; `stride` separates
// the lines of consecutive solves.
// KIND: OP_DERIV or OP_FILTER, the operator's kind known at compile time, or -1: read from op
// (one instantiation serving both kinds, which some passes allocate registers better with).
template <int S, int WPL, int NV, int KIND>
__device__ __forceinline__ void solve_lines_n(double* line, int stride, const LineOp& op, const LaneIds& z, double* scl,
                                              double scale, bool images, const double* sp) {
  double v[NV][S];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const double* li = line + i * stride;
    if (KIND == OP_FILTER || (KIND < 0 && op.kind == OP_FILTER))
      rhs_filter<S>(v[i], op, z.seg, [li](int n) { return li[n]; }, sp + i * 2 * NSP);
    else rhs_deriv<S>(v[i], op, z.seg, [li](int n) { return li[n]; }, sp + i * 2 * NSP);
  }
  seg_solve_n<S, WPL, NV>(v, op.tab, z.seg, z.lane, z.part, z.l, scl);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    if (scale != 1.0) {
#pragma unroll
      for (int t = 0; t < S; ++t) v[i][t] *= scale;
    }
    put_lane<S>(line + i * stride, v[i], z.seg, op.ext_lo, op.dim, images);
  }
}

// Solve `count` staged lines spaced by `stride`: four at a time for 5 rows per lane, in pairs
// for 9 (independent recurrences and scans interleave; 512^3: pass C 11.8 -> 10.4 ms, A and B
// -7 %), one at a time for 17 rows per lane, where a pair's registers exceed the 128 cap, and
// for 3, the small boxes' layout.
// sp: this line's closure tables of the `count` solves (see compute_specials).
template <int S, int WPL, int KIND>
__device__ __forceinline__ void solve_lines(double* line, int stride, int count, const LineOp& op, const LaneIds& z,
                                            double* scl, double scale, bool images, const double* sp) {
  int i = 0;
  if (S == 5)
    for (; i + 3 < count; i += 4)
      solve_lines_n<S, WPL, 4, KIND>(line + i * stride, stride, op, z, scl, scale, images, sp + i * 2 * NSP);
  if (S == 5 || S == 9)
    for (; i + 1 < count; i += 2)
      solve_lines_n<S, WPL, 2, KIND>(line + i * stride, stride, op, z, scl, scale, images, sp + i * 2 * NSP);
  for (; i < count; ++i)
    solve_lines_n<S, WPL, 1, KIND>(line + i * stride, stride, op, z, scl, scale, images, sp + i * 2 * NSP);
}

// Closure tables of `count` tile lines spaced by `stride` (line l of solve k at
// base + k*stride + l*LP + HT).
template <int KIND>
__device__ __forceinline__ void tile_specials(const LineOp& op, int TI, int LP, const double* base, int stride, int count,
                                              double* sp) {
  compute_specials<KIND>(op, TI, sp, count, [&](int l, int k, int n) { return base[k * stride + l * LP + HT + n]; });
}

// Euler flux along DIR at one node from the primitives (convection, tgvsolver.F90:559-564, with
// q rebuilt by fvar2q): F0 = rho u_d, F_{1+j} = rho u_j u_d (+ p when j = d), F4 = (E + p) u_d.
template <int DIR>
__device__ __forceinline__ void euler_flux(double rho, double u, double v, double w, double p, const Thermo& th,
                                           double (&F)[5]) {
  const double ud = (DIR == 0) ? u : (DIR == 1 ? v : w);
  F[0] = rho * ud;
  F[1] = rho * u * ud;
  F[2] = rho * v * ud;
  F[3] = rho * w * ud;
  F[1 + DIR] = F[1 + DIR] + p;
  const double E = p * th.const6 + rho * (0.5 * (u * u + v * v + w * w));
  F[4] = (E + p) * ud;
}

// Store tiles [k0, k0 + nf) (nodes 0..dim of the slot line) to fields dst + m*fs (or add them).
// x lines store node pairs with 16-byte accesses when aligned.
template <int DIR, int WPL, bool ADD, bool LW>
__device__ __forceinline__ void store_tiles(const TileCtx<DIR, WPL, LW>& c, const double* T, int tsz, double* dst,
                                            int64_t fs, int nf) {
  if (!c.svalid) return;
  double* d = dst + c.sbase;
  const int dim = c.dim;
  constexpr int TPL = TileCtx<DIR, WPL>::TPL;
  const int row = c.sl * c.LP + HT;
  if (DIR == 0 && ((c.LP & 1) == 0) && ((reinterpret_cast<uintptr_t>(T + row) & 15u) == 0)) {
#pragma unroll 1
    for (int m = 0; m < nf; ++m) {
      double* dm = d + m * fs;
      const double* Tm = T + m * tsz + row;
      int n = 2 * c.sn0;
      for (; n + 1 <= dim; n += 2 * TPL) {
        double2 v = *reinterpret_cast<const double2*>(Tm + n);
        if (ADD) {
          const double2 r = *reinterpret_cast<const double2*>(dm + n);
          v.x += r.x;
          v.y += r.y;
        }
        *reinterpret_cast<double2*>(dm + n) = v;
      }
      if (n == dim) dm[n] = ADD ? dm[n] + Tm[n] : Tm[n];   // odd node count: the last node alone
    }
    return;
  }
#pragma unroll 1
  for (int m = 0; m < nf; ++m) {
    double* dm = d + m * fs;
    const double* Tm = T + m * tsz;
    if (ADD) c.for_nodes_rmw<8>(0, dim, [&](int n) { return dm[(int64_t)n * c.sd]; },
                                [&](int o, int n, double r) { dm[(int64_t)n * c.sd] = r + Tm[o]; });
    else c.for_nodes(0, dim, [&](int o, int n) { dm[(int64_t)n * c.sd] = Tm[o]; });
  }
}

// ------------------------------------------------------------------ pass A and pass B
// Gradients of (u, v, w, T) along DIR into D (gradcal, tgvsolver.F90:450-537); pass A first
// applies the filter along A still owed by the previous stage. Each solve writes its result over
// the primitive tile it no longer needs (u, v, w -> themselves, T -> the pressure tile).
template <int S, int WPL, int DIR, bool IS_A>
__device__ __forceinline__ void k_pass_ab_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  double* T = sm;
  double* scan = sm + 5 * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;   // closure tables
  const int64_t fs = a.g.fs;
  for (int m = 0; m < 5; ++m) load_tile(c, T + m * tsz, a.q + m * fs);
  cp_async_wait_all();
  __syncthreads();
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  const int dim = c.dim;

  if (IS_A && a.do_filter) {
    tile_specials<OP_FILTER>(a.opf, c.TI, c.LP, T, tsz, 5, spb);
    __syncthreads();
    solve_lines<S, WPL, OP_FILTER>(T + z.l * c.LP + HT, tsz, 5, a.opf, z, scl, 1.0, true, spb + z.l * 5 * 2 * NSP);
    __syncthreads();
    store_tiles<DIR, WPL, false>(c, T, tsz, a.q, fs, 5);
    __syncthreads();   // every filtered value is stored before the tiles turn into primitives
  }
  to_prims<DIR, WPL, true>(c, T, tsz, a.th);
  __syncthreads();
  tile_specials<OP_DERIV>(a.opd, c.TI, c.LP, T + tsz, tsz, 4, spb);
  __syncthreads();
  solve_lines<S, WPL, OP_DERIV>(T + tsz + z.l * c.LP + HT, tsz, 4, a.opd, z, scl, a.g.rd[DIR], false, spb + z.l * 4 * 2 * NSP);
  __syncthreads();
  store_tiles<DIR, WPL, false>(c, T + tsz, tsz, a.D, fs, 4);
}

// ------------------------------------------------------------------ pass C
// Gradients along C, viscous stress and heat flux at every node (diffusion,
// tgvsolver.F90:635-694) with the A and B gradients, the viscous fluxes of A and B stored for
// passes A' and B', diagnostics, then R = D_C(VF_C - F_C) (the first contribution to R).
// DIAG: the stage-1 form with the diagnostics partial sums (a.partials); stages 2 and 3 run a
// kernel without them (fewer live registers in the flux loop).
template <int S, int WPL, int DIR, bool DIAG>
__device__ __forceinline__ void k_pass_c_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  double* T = sm;
  double* G = sm + 5 * tsz;   // 4 gradient tiles, then the 5 combined-flux tiles G1..G4, G0
  double* scan = G + 5 * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;   // closure tables: 4 gradients, then 5 fluxes
  double* spv = spb + c.TI * 4 * 2 * NSP;
  double* red = spb + c.TI * SP_PER_LINE;
  const int64_t fs = a.g.fs;
  // the A and B gradients of the line (read by the flux loop after the C solves) start moving
  // into L2 now: one bulk prefetch per contiguous x line of each of the 8 fields
  if (DIR == 0 && c.svalid && c.sn0 < 8 && a.DA && a.DB) {
    const double* src = (c.sn0 < 4 ? a.DA + c.sn0 * fs : a.DB + (c.sn0 - 4) * fs) + c.sbase;
    const unsigned bytes = (unsigned)(((c.dim + 1) * 8 + 15) & ~15);   // within the padded row
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
  }
  __shared__ uint64_t bar;
  if (DIR == 0 && (c.LP & 1) == 0) {
    stage_x_bulk(c, T, tsz, a.q, fs, 5, a, bx, by, &bar);
  } else {
    for (int m = 0; m < 5; ++m) load_tile(c, T + m * tsz, a.q + m * fs);
    cp_async_wait_all();
  }
  __syncthreads();
  const int dim = c.dim;
  to_prims(c, T, tsz, a.th);
  __syncthreads();
  // gradients along C of (u, v, w, T), solved in place in the G tiles
  c.for_nodes(-HT, dim + HT, [&](int o, int) {
    G[o] = T[tsz + o];
    G[tsz + o] = T[2 * tsz + o];
    G[2 * tsz + o] = T[3 * tsz + o];
    G[3 * tsz + o] = T[4 * tsz + o] / T[o] * a.th.const2;
  });
  __syncthreads();
  tile_specials<OP_DERIV>(a.opd, c.TI, c.LP, G, tsz, 4, spb);
  __syncthreads();
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  const double rd = a.g.rd[DIR];
  solve_lines<S, WPL, OP_DERIV>(G + z.l * c.LP + HT, tsz, 4, a.opd, z, scl, rd, false, spb + z.l * 4 * 2 * NSP);
  __syncthreads();
  if (a.DC) {   // kept for the discrete adjoint
    store_tiles<DIR, WPL, false>(c, G, tsz, a.DC, fs, 4);
    __syncthreads();
  }

  const Thermo th = a.th;
  constexpr int dA = DIR_A, dB = DIR_B, dC = DIR_C;
  static_assert(DIR == DIR_C, "pass C runs along DIR_C");
  double ke = 0.0, en = 0.0, di = 0.0;
  const bool diag = DIAG && a.partials != nullptr;
  int bad = 0;
  if (c.svalid) {
    const double* DA = a.DA + c.sbase;
    const double* DB = a.DB + c.sbase;
    double* VF = a.VF + c.sbase;
    const bool row_ok = (bx * (int64_t)c.TI + c.sl) >= 1 && by >= 1;
    struct G8 { double ga[4], gb[4]; };
    c.template for_nodes_batched<2, G8>(0, dim, [&](int n) {
      const int64_t off = (int64_t)n * c.sd;
      G8 r;
#pragma unroll
      for (int k = 0; k < 4; ++k) { r.ga[k] = __ldg(DA + k * fs + off); r.gb[k] = __ldg(DB + k * fs + off); }
      return r;
    }, [&](int tix, int n, const G8& gl) {
      const int64_t off = (int64_t)n * c.sd;
      double gr[4][3];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        gr[k][dA] = gl.ga[k];
        gr[k][dB] = gl.gb[k];
        gr[k][dC] = G[k * tsz + tix];
      }
      const double q0 = T[tix], u = T[tsz + tix], v = T[2 * tsz + tix], w = T[3 * tsz + tix], p = T[4 * tsz + tix];
      // divisions by constants as products with their reciprocals (equal to within an ulp)
      const double tmp = p * (1.0 / q0) * th.const2;
      if (!(q0 > 0.0) || !isfinite(p)) bad = 1;
      const double s11 = gr[0][0];
      const double s12 = 0.5 * (gr[0][1] + gr[1][0]);
      const double s13 = 0.5 * (gr[0][2] + gr[2][0]);
      const double s22 = gr[1][1];
      const double s23 = 0.5 * (gr[1][2] + gr[2][1]);
      const double s33 = gr[2][2];
      const double skk = (1.0 / 3.0) * (s11 + s22 + s33);
      const double miu = miucal(th, tmp) * th.inv_re;
      const double miu2 = 2.0 * miu;
      const double hcc = miu * th.inv_prc5;
      double sg[6];
      sg[0] = miu2 * (s11 - skk);
      sg[1] = miu2 * s12;
      sg[2] = miu2 * s13;
      sg[3] = miu2 * (s22 - skk);
      sg[4] = miu2 * s23;
      sg[5] = miu2 * (s33 - skk);
      double qf[3];
      qf[0] = hcc * gr[3][0] + sg[0] * u + sg[1] * v + sg[2] * w;
      qf[1] = hcc * gr[3][1] + sg[1] * u + sg[3] * v + sg[4] * w;
      qf[2] = hcc * gr[3][2] + sg[2] * u + sg[4] * v + sg[5] * w;
      // combined fluxes G_d = VF_d - F_d along A and B for passes A' and B'
      {
        double FA[5], FB[5];
        euler_flux<dA>(q0, u, v, w, p, th, FA);
        euler_flux<dB>(q0, u, v, w, p, th, FB);
        VF[0 * fs + off] = -FA[0];
        VF[1 * fs + off] = sg[sidx(dA, 0)] - FA[1];
        VF[2 * fs + off] = sg[sidx(dA, 1)] - FA[2];
        VF[3 * fs + off] = sg[sidx(dA, 2)] - FA[3];
        VF[4 * fs + off] = qf[dA] - FA[4];
        VF[5 * fs + off] = -FB[0];
        VF[6 * fs + off] = sg[sidx(dB, 0)] - FB[1];
        VF[7 * fs + off] = sg[sidx(dB, 1)] - FB[2];
        VF[8 * fs + off] = sg[sidx(dB, 2)] - FB[3];
        VF[9 * fs + off] = qf[dB] - FB[4];
      }
      // combined fluxes along C, with their periodic images
      double F[5];
      euler_flux<DIR>(q0, u, v, w, p, th, F);
      const double gv[5] = {sg[sidx(dC, 0)] - F[1], sg[sidx(dC, 1)] - F[2], sg[sidx(dC, 2)] - F[3], qf[dC] - F[4], -F[0]};
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double* line = G + k * tsz + c.sl * c.LP + HT;
        line[n] = gv[k];
        put_images(line, n, dim, gv[k]);
      }
      if (diag && n >= 1 && row_ok) {
        // stacal (tgvsolver.F90:913-931) and diss_rate_cal (statistic.F90:1009-1034)
        ke += q0 * (u * u + v * v + w * w);
        const double om1 = gr[2][1] - gr[1][2];
        const double om2 = gr[0][2] - gr[2][0];
        const double om3 = gr[1][0] - gr[0][1];
        en += q0 * (om1 * om1 + om2 * om2 + om3 * om3);
        const double div = s11 + s22 + s33;
        di += 2.0 * miu * (s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23) -
                           (1.0 / 3.0) * (div * div));
      }
    });
  } else {
    // lines past the box: finite filler for the solves (never stored)
    c.for_nodes(-HT, dim + HT, [&](int tix, int) {
#pragma unroll
      for (int k = 0; k < 5; ++k) G[k * tsz + tix] = 0.0;
    });
  }
  if (bad) atomicOr(a.err, 1);
  if (diag) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ke += __shfl_down_sync(FULL, ke, off);
      en += __shfl_down_sync(FULL, en, off);
      di += __shfl_down_sync(FULL, di, off);
    }
    if (z.lane == 0) { red[3 * z.warp] = ke; red[3 * z.warp + 1] = en; red[3 * z.warp + 2] = di; }
  }
  __syncthreads();
  if (diag && threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; ++w) { s0 += red[3 * w]; s1 += red[3 * w + 1]; s2 += red[3 * w + 2]; }
    const int ntx = (a.g.N[TileCtx<DIR, WPL>::o1] + 1 + c.TI - 1) / c.TI;
    double* pp = a.partials + 3 * ((int64_t)by * ntx + bx);
    pp[0] = s0; pp[1] = s1; pp[2] = s2;
  }
  // R = D_C(VF_C - F_C): one solve per component (convection + diffusion, tgvsolver.F90:539-787)
  tile_specials<OP_DERIV>(a.opd, c.TI, c.LP, G, tsz, 5, spv);
  __syncthreads();
  solve_lines<S, WPL, OP_DERIV>(G + z.l * c.LP + HT, tsz, 5, a.opd, z, scl, rd, false, spv + z.l * 5 * 2 * NSP);
  __syncthreads();
  store_tiles<DIR, WPL, false>(c, G, tsz, a.R + fs, fs, 4);
  store_tiles<DIR, WPL, false>(c, G + 4 * tsz, tsz, a.R, fs, 1);
}

// ------------------------------------------------------------------ field streaming
// Passes whose fields are independent (A', B', F) can take their fields in groups of fps (the
// streamed kernels below use fps = 1) through one buffer or two. With two, the copies of group g+1
// are in flight while group g is solved; with one (warps looping over lines), each group is copied,
// waited for and processed in turn, and the overlap comes from the other CTAs on the SM, which the
// small footprint lets in. body(first field, count, tiles) runs between CTA barriers and leaves
// the tiles free for reuse.
template <int DIR, int WPL, bool LW, class Src, class Body>
__device__ __forceinline__ void stream_fields(const TileCtx<DIR, WPL, LW>& c, double* buf, int tsz, int nf, int nbuf,
                                              int fps, Src src, Body body) {
  const int ngrp = (nf + fps - 1) / fps;
  const int gsz = fps * tsz;
  auto load_group = [&](int g, double* dst) {
    for (int j = 0; j < fps && g * fps + j < nf; ++j) load_tile(c, dst + j * tsz, src(g * fps + j));
  };
  if (nbuf == 1) {
#pragma unroll 1
    for (int g = 0; g < ngrp; ++g) {
      load_group(g, buf);
      cp_async_wait_all();
      __syncthreads();
      body(g * fps, min(fps, nf - g * fps), buf);
      __syncthreads();
    }
    return;
  }
  load_group(0, buf);
  cp_async_commit();
#pragma unroll 1
  for (int g = 0; g < ngrp; ++g) {
    if (g + 1 < ngrp) {
      load_group(g + 1, buf + ((g + 1) & 1) * gsz);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    body(g * fps, min(fps, nf - g * fps), buf + (g & 1) * gsz);
    __syncthreads();
  }
}

// `count` solves (tiles spaced by tsz) on every line of a tile: the CTA's warps form TI / LPW
// line groups of WPL warps, and group g solves lines g, g + TI/LPW, ... (LPW lines per group;
// LPW = 1 on x lines). spb: closure tables laid out by tile_specials with `count` solves.
template <int S, int WPL, int KIND>
__device__ __forceinline__ void solve_tile(double* tile, int tsz, int count, int TI, int LP, int LPW, const LineOp& op,
                                           const LaneIds& z, double* scl, double scale, const double* spb) {
  const int ng = TI / LPW;
#pragma unroll 1
  for (int k = 0; k < LPW; ++k) {
    const int l = z.l + k * ng;
    solve_lines<S, WPL, KIND>(tile + l * LP + HT, tsz, count, op, z, scl, scale, false, spb + l * count * 2 * NSP);
  }
}

// Buffers of the streamed passes: one field tile, or two (shape_tiles on the host).
__device__ __forceinline__ int stream_nbuf(const PassArgs& a) { return a.LPW > 1 ? 1 : 2; }

// ------------------------------------------------------------------ streamed A', B', F
// The same passes with their fields streamed one at a time (FPS = 1), for large boxes; separate
// kernels, so that the all-fields forms below keep their own (smaller) register allocation.
template <int S, int WPL, int DIR>
__device__ __forceinline__ void k_pass_vas_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL, true> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  const int nbuf = stream_nbuf(a), fps = 1;
  double* scan = sm + nbuf * fps * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;
  const int64_t fs = a.g.fs;
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  stream_fields(c, sm, tsz, 5, nbuf, fps, [&](int m) { return a.VF + m * fs; }, [&](int m0, int cnt, double* T) {
    tile_specials<OP_DERIV>(a.opd, c.TI, c.LP, T, tsz, cnt, spb);
    __syncthreads();
    solve_tile<S, WPL, OP_DERIV>(T, tsz, cnt, c.TI, c.LP, a.LPW, a.opd, z, scl, a.g.rd[DIR], spb);
    __syncthreads();
    store_tiles<DIR, WPL, true>(c, T, tsz, a.R + m0 * fs, fs, cnt);
  });
}

template <int S, int WPL, int DIR>
__device__ __forceinline__ void k_pass_vbs_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL, true> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  const int nbuf = stream_nbuf(a), fps = 1;
  double* scan = sm + nbuf * fps * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;
  const int64_t fs = a.g.fs;
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  const int dim = c.dim;
  stream_fields(c, sm, tsz, 5, nbuf, fps, [&](int m) { return a.VF + (5 + m) * fs; }, [&](int m0, int cnt, double* T) {
    tile_specials<OP_DERIV>(a.opd, c.TI, c.LP, T, tsz, cnt, spb);
    __syncthreads();
    solve_tile<S, WPL, -1>(T, tsz, cnt, c.TI, c.LP, a.LPW, a.opd, z, scl, a.g.rd[DIR], spb);
    __syncthreads();
    if (a.mode == 0) {
      store_tiles<DIR, WPL, true>(c, T, tsz, a.R + m0 * fs, fs, cnt);
      return;
    }
    // SSP-RK3 stage update of the group's fields, with the periodic images for the filter
    if (c.svalid) {
      const double c1 = a.c1, c2 = a.c2, c3 = a.c3, dt = a.dt;
#pragma unroll 1
      for (int j = 0; j < cnt; ++j) {
        double* Tm = T + j * tsz;
        const int64_t fo = (m0 + j) * fs + c.sbase;
        const double* qs = a.qsave + fo;
        const double* qq = a.q + fo;
        const double* R = a.R + fo;
        double* sline = Tm + c.sl * c.LP + HT;
        struct L3 { double r, s, q; };
        c.template for_nodes_batched<4, L3>(0, dim, [&](int n) {
          const int64_t off = (int64_t)n * c.sd;
          return L3{R[off], qs[off], (c2 != 0.0) ? qq[off] : 0.0};
        }, [&](int o, int n, const L3& l) {
          const double r = l.r + Tm[o];
          // (c1 qsave + c2 q) + (c3 qrhs) dt in the reference's order, rounded at every step so
          // that the result does not depend on how the compiler contracts this kernel
          const double qc = (c2 != 0.0) ? __dmul_rn(c2, l.q) : 0.0;
          const double qn = __dadd_rn(__dadd_rn(__dmul_rn(c1, l.s), qc), __dmul_rn(__dmul_rn(c3, r), dt));
          Tm[o] = qn;
          put_images(sline, n, dim, qn);
        });
      }
    }
    __syncthreads();
    if (a.do_filter) {
      tile_specials<OP_FILTER>(a.opf, c.TI, c.LP, T, tsz, cnt, spb);
      __syncthreads();
      solve_tile<S, WPL, -1>(T, tsz, cnt, c.TI, c.LP, a.LPW, a.opf, z, scl, 1.0, spb);
      __syncthreads();
    }
    store_tiles<DIR, WPL, false>(c, T, tsz, a.qout + m0 * fs, fs, cnt);
  });
}

template <int S, int WPL, int DIR>
__device__ __forceinline__ void k_pass_fs_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL, true> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  const int nbuf = stream_nbuf(a), fps = 1;
  double* scan = sm + nbuf * fps * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;
  const int64_t fs = a.g.fs;
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  stream_fields(c, sm, tsz, 5, nbuf, fps, [&](int m) { return a.q + m * fs; }, [&](int m0, int cnt, double* T) {
    tile_specials<OP_FILTER>(a.opf, c.TI, c.LP, T, tsz, cnt, spb);
    __syncthreads();
    solve_tile<S, WPL, OP_FILTER>(T, tsz, cnt, c.TI, c.LP, a.LPW, a.opf, z, scl, 1.0, spb);
    __syncthreads();
    store_tiles<DIR, WPL, false>(c, T, tsz, a.q + m0 * fs, fs, cnt);
  });
}

// ------------------------------------------------------------------ pass A' (fluxes along A)
// R += D_A(G_A), G_A = VF_A - F_A as pass C stored it.
template <int S, int WPL, int DIR>
__device__ __forceinline__ void k_pass_va_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  double* T = sm;
  double* scan = sm + 5 * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;
  const int64_t fs = a.g.fs;
  for (int m = 0; m < 5; ++m) load_tile(c, T + m * tsz, a.VF + m * fs);
  cp_async_wait_all();
  __syncthreads();
  tile_specials<OP_DERIV>(a.opd, c.TI, c.LP, T, tsz, 5, spb);
  __syncthreads();
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  solve_lines<S, WPL, OP_DERIV>(T + z.l * c.LP + HT, tsz, 5, a.opd, z, scl, a.g.rd[DIR], false, spb + z.l * 5 * 2 * NSP);
  __syncthreads();
  store_tiles<DIR, WPL, true>(c, T, tsz, a.R, fs, 5);
}

// ------------------------------------------------------------------ pass B' (fluxes along B, update, filter)
// R += D_B(G_B); mode 1: q_out = F_B(c1 qsave + c2 q + c3 dt R) (rk3, tgvsolver.F90:1055-1057,
// filterq along B); mode 0: R only.
template <int S, int WPL, int DIR>
__device__ __forceinline__ void k_pass_vb_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  double* T = sm;
  double* scan = sm + 5 * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;
  const int64_t fs = a.g.fs;
  for (int m = 0; m < 5; ++m) load_tile(c, T + m * tsz, a.VF + (5 + m) * fs);
  cp_async_wait_all();
  __syncthreads();
  tile_specials<OP_DERIV>(a.opd, c.TI, c.LP, T, tsz, 5, spb);
  __syncthreads();
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  solve_lines<S, WPL, OP_DERIV>(T + z.l * c.LP + HT, tsz, 5, a.opd, z, scl, a.g.rd[DIR], false, spb + z.l * 5 * 2 * NSP);
  __syncthreads();
  if (a.mode == 0) {
    store_tiles<DIR, WPL, true>(c, T, tsz, a.R, fs, 5);
    return;
  }
  // SSP-RK3 stage update of every field, with the periodic images for the filter
  const int dim = c.dim;
  if (c.svalid) {
    const double c1 = a.c1, c2 = a.c2, c3 = a.c3, dt = a.dt;
    const double* qs = a.qsave + c.sbase;
    const double* qq = a.q + c.sbase;
    const double* R = a.R + c.sbase;
#pragma unroll 1
    for (int m = 0; m < 5; ++m) {
      double* Tm = T + m * tsz;
      double* sline = Tm + c.sl * c.LP + HT;
      struct L3 { double r, s, q; };
      c.template for_nodes_batched<4, L3>(0, dim, [&](int n) {
        const int64_t off = m * fs + (int64_t)n * c.sd;
        return L3{R[off], qs[off], (c2 != 0.0) ? qq[off] : 0.0};
      }, [&](int o, int n, const L3& l) {
        const double r = l.r + Tm[o];
        // (c1 qsave + c2 q) + (c3 qrhs) dt in the reference's order, rounded at every step so
        // that the result does not depend on how the compiler contracts this kernel
        const double qc = (c2 != 0.0) ? __dmul_rn(c2, l.q) : 0.0;
        const double qn = __dadd_rn(__dadd_rn(__dmul_rn(c1, l.s), qc), __dmul_rn(__dmul_rn(c3, r), dt));
        Tm[o] = qn;
        put_images(sline, n, dim, qn);
      });
    }
  }
  __syncthreads();
  if (a.do_filter) {
    tile_specials<OP_FILTER>(a.opf, c.TI, c.LP, T, tsz, 5, spb);
    __syncthreads();
    solve_lines<S, WPL, OP_FILTER>(T + z.l * c.LP + HT, tsz, 5, a.opf, z, scl, 1.0, false, spb + z.l * 5 * 2 * NSP);
    __syncthreads();
  }
  store_tiles<DIR, WPL, false>(c, T, tsz, a.qout, fs, 5);
}

// ------------------------------------------------------------------ pass F (filter only, 5 fields)
template <int S, int WPL, int DIR>
__device__ __forceinline__ void k_pass_f_body(const PassArgs& a, int bx, int by) {
  extern __shared__ double sm[];
  const TileCtx<DIR, WPL> c(a, bx, by);
  const int tsz = c.TI * c.LP;
  double* T = sm;
  double* scan = sm + 5 * tsz;
  double* spb = scan + c.TI * SCAN_PER_LINE * WPL;
  const int64_t fs = a.g.fs;
  for (int m = 0; m < 5; ++m) load_tile(c, T + m * tsz, a.q + m * fs);
  cp_async_wait_all();
  __syncthreads();
  tile_specials<OP_FILTER>(a.opf, c.TI, c.LP, T, tsz, 5, spb);
  __syncthreads();
  const LaneIds z = lane_ids<WPL>();
  double* scl = scan + z.l * SCAN_PER_LINE * WPL;
  solve_lines<S, WPL, OP_FILTER>(T + z.l * c.LP + HT, tsz, 5, a.opf, z, scl, 1.0, false, spb + z.l * 5 * 2 * NSP);
  __syncthreads();
  store_tiles<DIR, WPL, false>(c, T, tsz, a.q, fs, 5);
}

// ------------------------------------------------------------------ kernels
// One box: the grid is the box's tile grid. Batch: blockIdx.x walks the concatenated tile grids
// of nbox boxes (cum[k] = first CTA of box k); each CTA copies its box's arguments to shared
// memory and runs the same body.
struct BatchArgs {
  const PassArgs* args;
  const int* cum;
  int nbox;
};

__device__ __forceinline__ const PassArgs& batch_decode(const BatchArgs& b, PassArgs& sa, int& bx, int& by) {
  int lo = 0, hi = b.nbox - 1;
  const int blk = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(b.cum + mid) <= blk) lo = mid;
    else hi = mid - 1;
  }
  const PassArgs* src = b.args + lo;
  const int nwords = (int)(sizeof(PassArgs) / sizeof(unsigned long long));
  for (int w = threadIdx.x; w < nwords; w += blockDim.x)
    reinterpret_cast<unsigned long long*>(&sa)[w] = __ldg(reinterpret_cast<const unsigned long long*>(src) + w);
  __syncthreads();
  const int o1 = (sa.dir == 0) ? 1 : 0;
  const int ntx = (sa.g.N[o1] + 1 + sa.TI - 1) / sa.TI;
  const int local = blk - __ldg(b.cum + lo);
  by = local / ntx;
  bx = local - by * ntx;
  return sa;
}

// The small-box layout (3 rows per lane, one warp per line) is bounded for two 512-thread CTAs per
// SM where that costs no more than a few spilled words (every pass but C): the boxes that use it
// have small grids, and the SMs they fill need the second CTA to hide latency.
#define ASTR_MINB(S, WPL, SMALL) (((SMALL) && (S) == 3 && (WPL) == 1) ? 2 : 1)
#define ASTR_PASS_KERNELS(NAME, SMALL, TPARAMS, TARGS)                                          \
  template <TPARAMS>                                                                              \
  __global__ void __launch_bounds__(512, ASTR_MINB(S, WPL, SMALL)) NAME(PassArgs a) {             \
    NAME##_body<TARGS>(a, blockIdx.x, blockIdx.y);                                                \
  }                                                                                               \
  template <TPARAMS>                                                                              \
  __global__ void __launch_bounds__(512, ASTR_MINB(S, WPL, SMALL)) NAME##_batch(BatchArgs b) {    \
    __shared__ PassArgs sa;                                                            \
    int bx, by;                                                                        \
    const PassArgs& a = batch_decode(b, sa, bx, by);                                   \
    NAME##_body<TARGS>(a, bx, by);                                                     \
  }

#define ASTR_COMMA ,
ASTR_PASS_KERNELS(k_pass_ab, true, int S ASTR_COMMA int WPL ASTR_COMMA int DIR ASTR_COMMA bool IS_A, S ASTR_COMMA WPL ASTR_COMMA DIR ASTR_COMMA IS_A)
ASTR_PASS_KERNELS(k_pass_c, false, int S ASTR_COMMA int WPL ASTR_COMMA int DIR ASTR_COMMA bool DIAG, S ASTR_COMMA WPL ASTR_COMMA DIR ASTR_COMMA DIAG)
ASTR_PASS_KERNELS(k_pass_va, true, int S ASTR_COMMA int WPL ASTR_COMMA int DIR, S ASTR_COMMA WPL ASTR_COMMA DIR)
ASTR_PASS_KERNELS(k_pass_vb, true, int S ASTR_COMMA int WPL ASTR_COMMA int DIR, S ASTR_COMMA WPL ASTR_COMMA DIR)
ASTR_PASS_KERNELS(k_pass_f, true, int S ASTR_COMMA int WPL ASTR_COMMA int DIR, S ASTR_COMMA WPL ASTR_COMMA DIR)
#undef ASTR_PASS_KERNELS
#undef ASTR_COMMA

// streamed forms: single-box launches only (the batched ensemble passes take all fields at once)
#define ASTR_STREAM_KERNEL(NAME)                                         \
  template <int S, int WPL, int DIR>                                     \
  __global__ void __launch_bounds__(512, ASTR_MINB(S, WPL, true)) NAME(PassArgs a) { \
    NAME##_body<S, WPL, DIR>(a, blockIdx.x, blockIdx.y);                 \
  }
ASTR_STREAM_KERNEL(k_pass_vas)
ASTR_STREAM_KERNEL(k_pass_vbs)
ASTR_STREAM_KERNEL(k_pass_fs)
#undef ASTR_STREAM_KERNEL

}  // namespace pass_detail

using namespace pass_detail;

inline size_t pass_smem(int pass, int TI, int LP, int WPL, int LPW, int FPS);

template <class KernT>
cudaError_t launch_k(KernT kern, dim3 grid, int threads, size_t smem, cudaStream_t st, const PassArgs& a) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, threads, smem, st>>>(a);
  return cudaGetLastError();
}

template <int S, int WPL>
cudaError_t launch_pass_t(int pass, const PassArgs& a, cudaStream_t st) {
  const int o1 = (a.dir == 0) ? 1 : 0, o2 = (a.dir == 2) ? 1 : 2;
  const int lpw = a.LPW > 1 ? a.LPW : 1;
  const size_t smem = pass_smem(pass, a.TI, a.LP, WPL, lpw, a.FPS > 1 ? 5 : 1);
  dim3 grid((unsigned)((a.g.N[o1] + 1 + a.TI - 1) / a.TI), (unsigned)(a.g.N[o2] + 1));
  const int threads = (a.TI / lpw) * WPL * 32;
  switch (pass) {
    case PASS_A: return launch_k(k_pass_ab<S, WPL, DIR_A, true>, grid, threads, smem, st, a);
    case PASS_B: return launch_k(k_pass_ab<S, WPL, DIR_B, false>, grid, threads, smem, st, a);
    case PASS_C:
      return a.partials ? launch_k(k_pass_c<S, WPL, DIR_C, true>, grid, threads, smem, st, a)
                        : launch_k(k_pass_c<S, WPL, DIR_C, false>, grid, threads, smem, st, a);
    case PASS_VA:
      if (a.FPS == 1) return launch_k(k_pass_vas<S, WPL, DIR_A>, grid, threads, smem, st, a);
      return launch_k(k_pass_va<S, WPL, DIR_A>, grid, threads, smem, st, a);
    case PASS_VB:
      if (a.FPS == 1) return launch_k(k_pass_vbs<S, WPL, DIR_B>, grid, threads, smem, st, a);
      return launch_k(k_pass_vb<S, WPL, DIR_B>, grid, threads, smem, st, a);
    case PASS_F:
      if (a.FPS == 1) {
        if (a.dir == DIR_C) return launch_k(k_pass_fs<S, WPL, DIR_C>, grid, threads, smem, st, a);
        if (a.dir == DIR_A) return launch_k(k_pass_fs<S, WPL, DIR_A>, grid, threads, smem, st, a);
        return launch_k(k_pass_fs<S, WPL, DIR_B>, grid, threads, smem, st, a);
      }
      if (a.dir == DIR_C) return launch_k(k_pass_f<S, WPL, DIR_C>, grid, threads, smem, st, a);
      if (a.dir == DIR_A) return launch_k(k_pass_f<S, WPL, DIR_A>, grid, threads, smem, st, a);
      return launch_k(k_pass_f<S, WPL, DIR_B>, grid, threads, smem, st, a);
    default:
      return cudaErrorInvalidValue;
  }
}

// Dynamic shared memory of one pass launch for a tile of TI lines with pitch LP.
inline size_t pass_smem(int pass, int TI, int LP, int WPL, int LPW, int FPS) {
  return pass_shared_bytes(pass, TI, LP, WPL, LPW, FPS);
}

template <class KernT>
cudaError_t launch_kb(KernT kern, int nctas, int threads, size_t smem, cudaStream_t st, const BatchArgs& b) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<nctas, threads, smem, st>>>(b);
  return cudaGetLastError();
}

// One launch of a pass over several boxes of the same solve layout (see BatchArgs).
template <int S, int WPL>
cudaError_t launch_pass_batch_t(int pass, int dir, const PassArgs* dargs, const int* dcum, int nbox, int nctas,
                                int threads, size_t smem, cudaStream_t st) {
  const BatchArgs b{dargs, dcum, nbox};
  switch (pass) {
    case PASS_A: return launch_kb(k_pass_ab_batch<S, WPL, DIR_A, true>, nctas, threads, smem, st, b);
    case PASS_B: return launch_kb(k_pass_ab_batch<S, WPL, DIR_B, false>, nctas, threads, smem, st, b);
    case PASS_C: return launch_kb(k_pass_c_batch<S, WPL, DIR_C, true>, nctas, threads, smem, st, b);
    case PASS_VA: return launch_kb(k_pass_va_batch<S, WPL, DIR_A>, nctas, threads, smem, st, b);
    case PASS_VB: return launch_kb(k_pass_vb_batch<S, WPL, DIR_B>, nctas, threads, smem, st, b);
    case PASS_F:
      if (dir == DIR_C) return launch_kb(k_pass_f_batch<S, WPL, DIR_C>, nctas, threads, smem, st, b);
      if (dir == DIR_A) return launch_kb(k_pass_f_batch<S, WPL, DIR_A>, nctas, threads, smem, st, b);
      return launch_kb(k_pass_f_batch<S, WPL, DIR_B>, nctas, threads, smem, st, b);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace astr
