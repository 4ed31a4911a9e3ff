// batch.cu -- many log-stabilised Sinkhorn problems of different sizes in one
// cooperative launch, iterated in lockstep.
//
// Every problem has the semantics of rwig_sinkhorn_log (Sinkhorn::compute_log,
// src/sinkhorn_impl_log.cpp:225-295), solved in stabilised scaling form with
// f~ = g~ = 0 on K = exp(-C/eps):
//   init:      u_1 = a / (K 1)                     (the reference's first f update)
//   iteration: v = b / (K^T u), r = K v in the same pass over K,
//              err = ||log(u o r) - log a||_2 + ||log(v o K^T u) - log b||_2,
//              u = a / r unless the loop stops (err < tol or max_iter)
//   final:     f = eps log u, g = eps log v, P = exp(-((C - f) - g)/eps),
//              loss = sum C o P + eps sum P o (log P - 1) (:266-277), marginals.
//
// Work split.  Problem p owns a team of gp consecutive CTAs, gp = min(G, n_p,
// ceil(bytes of K_p / 128 KB)) -- a function of the problem alone
// (offset off_p, wrapping); team member k holds the column strip
// [k n/gp, (k+1) n/gp) of K_p with every row, so its column sums are complete
// in the CTA and its row partials go to rowp_p[k].  Rows are merged in units
// of 64 spread over the whole grid (lanes split the team's partials).  One iteration of the launch is
//   column pass over all my strips of the running problems (one bulk-copy
//   ring across problems) | grid barrier | row merge of my units | grid
//   barrier | every CTA takes the same continue / stop decision for every
//   problem.
// The column split, the merge order (team members 0..gp-1) and the error sums
// depend only on the problem, so a result is bitwise the same whatever else
// is in the batch.  A problem whose scalings leave [e^-650, e^650], whose
// masses are not all positive or whose sums leave the safe range is handed
// back (status kUnsafe) and re-solved by the per-call path.
//
// Every wait is bounded (2 s); on expiry the kernel sets an error word and
// returns, and the host reports RWIG_E_TIMEOUT.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "sk_common.cuh"
#include "sk_host.h"

namespace rwig {
namespace batch {

using sk::block_sum_cols;
using sk::STAGES;

constexpr int NTT = 512, NW = NTT / 32;
constexpr int kSlot = 8192;   // doubles per ring stage (CW x 512 RPT = 8192 for every row class)
constexpr int kMaxRows = 8192;
constexpr int kUnit = 64;     // rows per merge unit (4 per warp)
constexpr int kMaxProbs = 512;
constexpr int kMaxTeam = 160;       // CTAs of a team (the grid is one CTA per SM)
constexpr long long kStripBytes = 128 << 10;  // target bytes of K per team member
constexpr double kScaleMin = 5.1e-283, kScaleMax = 1.95e282;  // e^-650, e^650
enum { ST_RUN = 0, ST_FIN = 1, ST_RETIRED = 2 };
constexpr double kUnsafeStatus = -100.0;

struct Prob {
  const double* a;
  const double* b;
  const double* C;   // m x n, column-major, leading dimension m (built here when X, Y are given)
  const double* X;   // m x d source points (column-major) or null
  const double* Y;   // n x d target points or null
  int d;
  double* K;         // m x n, leading dimension ldk (even), 16-byte aligned
  long long ldk;
  double* P;         // optional plan (leading dimension m)
  double* f;         // m
  double* g;         // n; holds v during the iterations
  double* u0;        // u ping-pong (m each)
  double* u1;
  double* rowp;      // [gp][m] row partials
  double* colp;      // [gp][4] column-strip partials
  double* unitp;     // [nunits][4] merge-unit partials
  double* res;       // [10]: loss, err, iter, status, l1 row, l1 col, l2 row, l2 col, -, -
  int m, n, max_iter, cls, gp, off, nunits, unit0;
  double eps, tol;
};

struct State {  // per problem, identical in every CTA
  int st, iter, par, init;  // init: 2 cost from points pending, 1 first pass pending, 0 iterating
  double err, cmax;
};

__host__ __device__ constexpr size_t smem_bytes() {
  return (size_t)STAGES * kSlot * 8 + 64 + (size_t)2 * NW * 16 * 8 + (size_t)kMaxProbs * sizeof(State) + 256;
}

__device__ __forceinline__ int class_cw(int cls) { return cls == 0 ? 16 : cls == 1 ? 8 : cls == 2 ? 4 : cls == 3 ? 2 : 1; }

// Team membership of this CTA in problem p: index k, or -1.
__device__ __forceinline__ int team_index(const Prob& p, int cta, int G) {
  const int k = (cta - p.off + G) % G;
  return k < p.gp ? k : -1;
}
__device__ __forceinline__ int strip_begin(const Prob& p, int k) { return (int)(((long long)k * p.n) / p.gp); }

// Column groups of this CTA across the running problems, in problem order:
// the consumer and the issuer walk the same sequence.
struct Cursor {
  int p;   // problem index (np: exhausted; -1: before the first)
  int jb;  // first column of the current group
};

__device__ __forceinline__ void next_group(Cursor& c, const Prob* probs, const State* S, int np, int cta, int G) {
  if (c.p >= 0 && c.p < np) {
    const Prob& p = probs[c.p];
    const int k = team_index(p, cta, G);
    c.jb += class_cw(p.cls);
    if (c.jb < strip_begin(p, k + 1)) return;
  }
  for (int q = c.p + 1; q < np; ++q) {
    if (S[q].st != ST_RUN || S[q].init) continue;
    const Prob& p = probs[q];
    const int k = team_index(p, cta, G);
    if (k < 0) continue;
    c.p = q;
    c.jb = strip_begin(p, k);
    return;
  }
  c.p = np;
  c.jb = 0;
}

struct Ring {
  double* buf;
  uint64_t* bar;
  uint64_t pol;  // L2 evict_first: K is streamed once per iteration
  __device__ double* slot(unsigned seq) const { return buf + (size_t)(seq % STAGES) * kSlot; }
  // thread 0: copy the group starting at column jb of problem p (strip end c1) into stage seq
  __device__ void issue(unsigned seq, const Prob& p, int jb, int c1) const {
    const unsigned bytes = (unsigned)(min(class_cw(p.cls), c1 - jb) * p.ldk * 8);
    uint64_t* b = bar + (seq % STAGES);
    mbar_arrive_expect_tx(b, bytes);
    bulk_g2s_hint(slot(seq), p.K + (size_t)jb * p.ldk, bytes, b, pol);
  }
  __device__ bool wait(unsigned seq) const { return mbar_wait_bounded(bar + (seq % STAGES), (seq / STAGES) & 1u); }
};

// Thread 0 keeps up to STAGES groups in flight ahead of the consumer.
struct Issuer {
  Cursor c;
  unsigned seq;
};

__device__ __forceinline__ void issue_ahead(Issuer& is, const Ring& ring, unsigned limit, const Prob* probs,
                                            const State* S, int np, int cta, int G) {
  while (is.seq < limit && is.c.p < np) {
    const Prob& p = probs[is.c.p];
    ring.issue(is.seq, p, is.c.jb, strip_begin(p, team_index(p, cta, G) + 1));
    ++is.seq;
    next_group(is.c, probs, S, np, cta, G);
  }
}

// Column pass of one problem over this CTA's strip (its groups are the next
// ones in the ring): column sums with u, v = b / s, row partials r = K v ->
// rowp[k], column-strip partials -> colp[k].
// REREAD: the row update reads the stage from shared memory again instead of
// keeping it in registers (for 16 rows per thread, which would not fit), and
// the stage is refilled only after a block barrier that follows that read.
template <int RPT, int CW, bool REREAD>
__device__ bool column_pass(const Prob& p, const State& s, int k, const Ring& ring, unsigned& q, Issuer& is,
                            const Prob* probs, const State* S, int np, int cta, int G, double* red, int& par) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int m = p.m;
  const int c0 = strip_begin(p, k), c1 = strip_begin(p, k + 1);
  const double* ucur = s.par ? p.u1 : p.u0;
  double u[RPT], r[RPT];
  bool valid[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    valid[t] = tid + t * NTT < m;
    u[t] = valid[t] ? __ldcg(ucur + tid + t * NTT) : 0.0;
    r[t] = 0.0;
  }
  double errc = 0.0, bad = 0.0;
  for (int jb = c0; jb < c1; jb += CW) {
    const unsigned seq = q;
    if (!ring.wait(seq)) return false;
    const double* buf = ring.slot(seq) + tid;
    const int nc = min(CW, c1 - jb);
    double kv[REREAD ? 1 : RPT][CW], sum[CW];
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      sum[c] = 0.0;
#pragma unroll
      for (int t = 0; t < RPT; ++t) {
        const double x = (c < nc && valid[t]) ? buf[(size_t)c * p.ldk + t * NTT] : 0.0;
        if (!REREAD) kv[t][c] = x;
        sum[c] = fma(x, u[t], sum[c]);
      }
    }
    double v[CW];
    {
      block_sum_cols<CW, NW>(sum, red, par);  // (the stage is no longer read after this unless REREAD)
      double s_l = 1.0;
#pragma unroll
      for (int c = 0; c < CW; ++c)
        if (c == lane) s_l = sum[c];
      const bool owner = lane < nc;
      const double v_l = owner ? p.b[jb + lane] / s_l : 0.0;
      if (w == 0 && owner) {
        p.g[jb + lane] = v_l;
        // log(v s) - log(b) with v = b / s is a rounding-level residual; its
        // first-order form needs no logarithm
        const double d = (v_l * s_l) / p.b[jb + lane] - 1.0;
        errc += d * d;
        if (!(v_l >= kScaleMin && v_l <= kScaleMax) || !(s_l >= 1e-300 && s_l <= 1e300)) bad = 1.0;
      }
#pragma unroll
      for (int c = 0; c < CW; ++c) v[c] = __shfl_sync(0xffffffffu, v_l, c);
    }
    if (!REREAD && tid == 0) issue_ahead(is, ring, seq + 1 + STAGES, probs, S, np, cta, G);
    q = seq + 1;
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
      double acc = r[t];
#pragma unroll
      for (int c = 0; c < CW; ++c) {
        const double x = REREAD ? ((c < nc && valid[t]) ? buf[(size_t)c * p.ldk + t * NTT] : 0.0)
                                : kv[REREAD ? 0 : t][c];
        acc = fma(x, v[c], acc);
      }
      r[t] = acc;
    }
    if (REREAD) {
      __syncthreads();  // every thread is done with the stage
      if (tid == 0) issue_ahead(is, ring, seq + 1 + STAGES, probs, S, np, cta, G);
    }
  }
#pragma unroll
  for (int t = 0; t < RPT; ++t)
    if (valid[t]) p.rowp[(size_t)k * m + tid + t * NTT] = r[t];
  double tt[2] = {errc, bad};
  block_sum_cols<2, NW>(tt, red, par);
  if (tid == 0) {
    p.colp[(size_t)k * 4 + 0] = tt[0];
    p.colp[(size_t)k * 4 + 1] = tt[1];
  }
  return true;
}

// Final pass over this CTA's strip: g = eps log v, P, loss and marginal partials.
template <int RPT, int CW>
__device__ void final_pass(const Prob& p, const State& s, int k, double* red, int& par) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int m = p.m;
  const double eps = p.eps;
  const int c0 = strip_begin(p, k), c1 = strip_begin(p, k + 1);
  const double* ucur = s.par ? p.u1 : p.u0;
  double f[RPT], rs[RPT];
  bool valid[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    valid[t] = tid + t * NTT < m;
    f[t] = valid[t] ? eps * log(__ldcg(ucur + tid + t * NTT)) : 0.0;
    rs[t] = 0.0;
  }
  double s1 = 0.0, s2 = 0.0, l1c = 0.0, l2c = 0.0;
  for (int jb = c0; jb < c1; jb += CW) {
    const int nc = min(CW, c1 - jb);
    double gj[CW], cs[CW];
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      gj[c] = c < nc ? eps * log(p.g[jb + c]) : 0.0;
      cs[c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      if (c >= nc) continue;
      const double* cj = p.C + (size_t)(jb + c) * m;
#pragma unroll
      for (int t = 0; t < RPT; ++t)
        if (valid[t]) {
          const double cij = cj[tid + t * NTT];
          const double pij = exp(-((cij - f[t]) - gj[c]) / eps);
          if (p.P) p.P[(size_t)(jb + c) * m + tid + t * NTT] = pij;
          s1 += cij * pij;
          s2 += pij * (log(pij) - 1.0);
          rs[t] += pij;
          cs[c] += pij;
        }
    }
    block_sum_cols<CW, NW>(cs, red, par);  // every thread has read p.g[jb..] before this returns
    if (w == 0 && lane < nc) {
      double gl = 0.0, cl = 0.0;
#pragma unroll
      for (int c = 0; c < CW; ++c)
        if (c == lane) {
          gl = gj[c];
          cl = cs[c];
        }
      p.g[jb + lane] = gl;
      const double d = cl - p.b[jb + lane];
      l1c += fabs(d);
      l2c += d * d;
    }
  }
#pragma unroll
  for (int t = 0; t < RPT; ++t)
    if (valid[t]) p.rowp[(size_t)k * m + tid + t * NTT] = rs[t];
  double tt[4] = {s1, s2, l1c, l2c};
  block_sum_cols<4, NW>(tt, red, par);
  if (tid == 0)
    for (int i = 0; i < 4; ++i) p.colp[(size_t)k * 4 + i] = tt[i];
}

// Cost from points over this CTA's strip: C_ij = sum_k (x_ik - y_jk)^2 in
// ascending k, each step rounded separately (the same operations and order as
// a host that computes the differences, squares and sums elementwise, so the
// same bits), stored un-normalised; the strip's maximum -> colp[k][2].
__device__ void cost_pass(const Prob& p, int k, double* red, int& par) {
  const int c0 = strip_begin(p, k), c1 = strip_begin(p, k + 1);
  const int m = p.m, n = p.n;
  double mx = 0.0;
  for (int j = c0; j < c1; ++j)
    for (int i = threadIdx.x; i < m; i += NTT) {
      double acc = 0.0;
      for (int q = 0; q < p.d; ++q) {
        const double t = __dsub_rn(p.X[i + (size_t)q * m], p.Y[j + (size_t)q * n]);
        acc = __dadd_rn(acc, __dmul_rn(t, t));
      }
      const_cast<double*>(p.C)[i + (size_t)j * m] = acc;
      mx = fmax(mx, acc);
    }
  // block maximum (exact, order-free)
  mx = warp_max(mx);
  __syncthreads();  // red is free
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int q = 0; q < NW; ++q) v = fmax(v, red[q]);
    p.colp[(size_t)k * 4 + 2] = v;
  }
  __syncthreads();
}

// First pass of a problem over this CTA's strip: K = exp(-C/eps)
// (sinkhorn_impl_vanilla.cpp:41 form) into its buffer, row partials of K 1
// -> rowp[k] (the merge turns them into u_1 = a / (K 1)), and whether a mass
// of the strip's columns or (member 0) of the rows is not positive -> colp[k][1].
template <int RPT>
__device__ void init_pass(const Prob& p, int k, double cmax, double* red, int& par) {
  const int tid = threadIdx.x;
  const int c0 = strip_begin(p, k), c1 = strip_begin(p, k + 1);
  const int m = p.m;
  double r[RPT];
  bool valid[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    valid[t] = tid + t * NTT < m;
    r[t] = 0.0;
  }
#pragma unroll 2
  for (int j = c0; j < c1; ++j) {
    const double* cj = p.C + (size_t)j * m;
    double* kj = p.K + (size_t)j * p.ldk;
#pragma unroll
    for (int t = 0; t < RPT; ++t)
      if (valid[t]) {
        double c = cj[tid + t * NTT];
        if (p.X) {  // C /= max C
          c = c / cmax;
          const_cast<double*>(cj)[tid + t * NTT] = c;
        }
        const double x = exp(-c / p.eps);
        kj[tid + t * NTT] = x;
        r[t] += x;
      }
  }
  double bad = 0.0;
  for (int j = c0 + tid; j < c1; j += NTT)
    if (!(p.b[j] > 0.0)) bad = 1.0;
  if (k == 0)
    for (int i = tid; i < m; i += NTT)
      if (!(p.a[i] > 0.0)) bad = 1.0;
  asm volatile("fence.proxy.async.global;" ::: "memory");  // K is read next by bulk copies
#pragma unroll
  for (int t = 0; t < RPT; ++t)
    if (valid[t]) p.rowp[(size_t)k * m + tid + t * NTT] = r[t];
  double tt[1] = {bad};
  block_sum_cols<1, NW>(tt, red, par);
  if (tid == 0) {
    p.colp[(size_t)k * 4 + 0] = 0.0;
    p.colp[(size_t)k * 4 + 1] = tt[0];
  }
}

// Row totals of merge unit u (rows u*64 .. u*64+63): warp w sums rows
// 4w .. 4w+3 over the gp team partials, lane l taking members l, l+32, ...
// in order, then a fixed butterfly across the lanes.  Lane r < 4 of the warp
// receives the total of its row r (i = u*64 + 4w + r); rows past m give 0.
__device__ __forceinline__ double merge_unit(const double* rowp, int gp, int m, int u) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i0 = u * kUnit + 4 * w;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  double v[kMaxTeam / 32][4];  // every load in flight at once
#pragma unroll
  for (int j = 0; j < kMaxTeam / 32; ++j) {
    const int k = lane + 32 * j;
#pragma unroll
    for (int r = 0; r < 4; ++r) v[j][r] = (k < gp && i0 + r < m) ? __ldcg(rowp + (size_t)k * m + i0 + r) : 0.0;
  }
#pragma unroll
  for (int j = 0; j < kMaxTeam / 32; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[r] += v[j][r];
  double mine = 0.0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const double t = warp_sum(acc[r]);
    if (lane == r) mine = t;
  }
  return mine;
}

// Service loop.  probs[0, *pub) are the published problems (pub[0]: count,
// pub[1]: stop flag; host-mapped memory for a server, device memory for a
// batch call); done[q] is set (system scope) once problem q's results are in
// probs[q].res.  dctl: [0] barrier count, [2] error bits, [3..5] values CTA 0
// broadcasts to the grid each iteration.  The launch ends when no problem
// runs and either the stop flag is set or nothing new was published for
// idle_ns.  prof (may be null): CTA 0's nanoseconds in [1] column passes,
// [2] the first barrier, [3] merges, [4] the second barrier and decisions,
// [6] iterations; [8 + 2 it], [9 + 2 it]: column-pass time and running
// problems of iteration it < 4096; [8 + 8192 + cta]: each CTA's column time.
__global__ void __launch_bounds__(NTT, 1) batch_kernel(const Prob* probs, const volatile unsigned* pub,
                                                        volatile unsigned* done, unsigned* dctl, double* prof,
                                                        unsigned long long idle_ns) {
  extern __shared__ __align__(128) unsigned char smem[];
  double* ringbuf = reinterpret_cast<double*>(smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(ringbuf + (size_t)STAGES * kSlot);
  double* red = reinterpret_cast<double*>(smem + (size_t)STAGES * kSlot * 8 + 64);
  State* S = reinterpret_cast<State*>(red + 2 * NW * 16);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, cta = blockIdx.x, G = gridDim.x;
  int par = 0;
  unsigned nbar = 0;
  auto gsync = [&]() -> bool { ++nbar; return grid_sync(dctl, dctl + 2, nbar * (unsigned)G); };
  const bool timing = prof && cta == 0 && tid == 0;
  double pt[7] = {0, 0, 0, 0, 0, 0, 0};
  double my_col_ns = 0.0;
  unsigned long long tl = timing ? globaltimer_ns() : 0ull;
  auto lap = [&](int slot) {
    if (timing) {
      const unsigned long long t = globaltimer_ns();
      pt[slot] += (double)(t - tl);
      tl = t;
    }
  };
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(bar + s, 1);
    fence_mbar_init();
  }
  // the published problems at start: unfinished ones run, finished ones stay retired
  unsigned long long last_busy = globaltimer_ns();
  if (cta == 0 && tid == 0) dctl[3] = min(pub[0], (unsigned)kMaxProbs);
  if (!gsync()) return;
  int np = (int)__ldcg(dctl + 3);
  for (int q = tid; q < np; q += NTT) S[q] = State{done[q] ? ST_RETIRED : ST_RUN, 0, 0, probs[q].X ? 2 : 1, 1000.0, 1.0};
  __syncthreads();

  const Ring ring{ringbuf, bar, l2_policy_evict_first()};
  unsigned q = 0;
  Issuer is{{-1, 0}, 0};
  while (true) {
    // ---- column pass over my strips: first passes, iterations, final passes
    const unsigned long long tcol0 = (prof && tid == 0) ? globaltimer_ns() : 0ull;
    if (tid == 0) {
      is.c = Cursor{-1, 0};
      next_group(is.c, probs, S, np, cta, G);
      is.seq = q;
      issue_ahead(is, ring, q + STAGES, probs, S, np, cta, G);
    }
    bool ok = true;
    for (int pi = 0; pi < np && ok; ++pi) {
      const int st = S[pi].st;
      if (st != ST_RUN && st != ST_FIN) continue;
      const Prob& p = probs[pi];
      const int k = team_index(p, cta, G);
      if (k < 0) continue;
      if (st == ST_FIN) {
        switch (p.cls) {
          case 0: final_pass<1, 16>(p, S[pi], k, red, par); break;
          case 1: final_pass<2, 8>(p, S[pi], k, red, par); break;
          case 2: final_pass<4, 4>(p, S[pi], k, red, par); break;
          case 3: final_pass<8, 2>(p, S[pi], k, red, par); break;
          default: final_pass<16, 1>(p, S[pi], k, red, par); break;
        }
      } else if (S[pi].init == 2) {
        cost_pass(p, k, red, par);
      } else if (S[pi].init) {
        const double cm = S[pi].cmax;
        switch (p.cls) {
          case 0: init_pass<1>(p, k, cm, red, par); break;
          case 1: init_pass<2>(p, k, cm, red, par); break;
          case 2: init_pass<4>(p, k, cm, red, par); break;
          case 3: init_pass<8>(p, k, cm, red, par); break;
          default: init_pass<16>(p, k, cm, red, par); break;
        }
      } else {
        switch (p.cls) {
          case 0: ok = column_pass<1, 16, false>(p, S[pi], k, ring, q, is, probs, S, np, cta, G, red, par); break;
          case 1: ok = column_pass<2, 8, false>(p, S[pi], k, ring, q, is, probs, S, np, cta, G, red, par); break;
          case 2: ok = column_pass<4, 4, false>(p, S[pi], k, ring, q, is, probs, S, np, cta, G, red, par); break;
          case 3: ok = column_pass<8, 2, false>(p, S[pi], k, ring, q, is, probs, S, np, cta, G, red, par); break;
          default: ok = column_pass<16, 1, true>(p, S[pi], k, ring, q, is, probs, S, np, cta, G, red, par); break;
        }
      }
    }
    if (!ok) {
      if (tid == 0) atomicOr(dctl + 2, KERR_MBAR_TIMEOUT);
      return;
    }
    if (prof && tid == 0) my_col_ns += (double)(globaltimer_ns() - tcol0);
    if (timing && (int)pt[6] < 4096) prof[8 + 2 * (int)pt[6]] = (double)(globaltimer_ns() - tl);
    lap(1);
    if (!gsync()) return;
    lap(2);
    // ---- row merges: u_next = a / (sum over the team's partials) for the
    // running problems, f and the row marginals for the finishing ones
    for (int pi = 0; pi < np; ++pi) {
      const int st = S[pi].st;
      if ((st != ST_RUN && st != ST_FIN) || S[pi].init == 2) continue;
      const Prob& p = probs[pi];
      const double* ucur = S[pi].par ? p.u1 : p.u0;
      double* unext = S[pi].par ? p.u0 : p.u1;
      for (int u = (cta - p.unit0 + G) % G; u < p.nunits; u += G) {
        const double tot = merge_unit(p.rowp, p.gp, p.m, u);
        const int i = u * kUnit + 4 * w + lane;
        double t[2] = {0.0, 0.0};
        if (lane < 4 && i < p.m) {
          const double ai = p.a[i];
          if (st == ST_FIN) {
            p.f[i] = p.eps * log(__ldcg(ucur + i));
            const double d = tot - ai;
            t[0] = fabs(d);
            t[1] = d * d;
          } else {
            const double un = ai / tot;
            unext[i] = un;
            if (!S[pi].init) {
              const double d = log((__ldcg(ucur + i) * tot) / ai);
              t[0] = d * d;
            }
            if (!(un >= kScaleMin && un <= kScaleMax) || !(tot >= 1e-300 && tot <= 1e300)) t[1] = 1.0;
          }
        }
        block_sum_cols<2, NW>(t, red, par);
        if (tid == 0) {
          const int o = st == ST_FIN ? 2 : 0;
          p.unitp[(size_t)u * 4 + o] = t[0];
          p.unitp[(size_t)u * 4 + o + 1] = t[1];
        }
      }
    }
    if (cta == 0 && tid == 0) {
      dctl[3] = min(pub[0], (unsigned)kMaxProbs);
      dctl[4] = pub[1];
      dctl[5] = (globaltimer_ns() - last_busy > idle_ns) ? 1u : 0u;
    }
    lap(3);
    if (!gsync()) return;
    const int np_new = max(np, (int)__ldcg(dctl + 3));
    const bool stop = __ldcg(dctl + 4) != 0u, idle = __ldcg(dctl + 5) != 0u;
    // ---- the same decisions in every CTA: warp w takes problems w, w+16, ...
    int running = 0;
    for (int pi = w; pi < np; pi += NW) {
      State& s = S[pi];
      if (s.st != ST_RUN && s.st != ST_FIN) continue;
      const Prob& p = probs[pi];
      const bool reporter = (p.off == cta) && lane == 0;
      if (s.st == ST_FIN) {
        double c[6] = {0, 0, 0, 0, 0, 0};
        for (int k = lane; k < p.gp; k += 32)
          for (int j = 0; j < 4; ++j) c[j] += __ldcg(p.colp + (size_t)k * 4 + j);
        for (int u = lane; u < p.nunits; u += 32) {
          c[4] += __ldcg(p.unitp + (size_t)u * 4 + 2);
          c[5] += __ldcg(p.unitp + (size_t)u * 4 + 3);
        }
#pragma unroll
        for (int j = 0; j < 6; ++j) c[j] = warp_sum(c[j]);
        if (reporter) {
          p.res[0] = c[0] + p.eps * c[1];  // accu(C % P) + reg * accu(P % (log(P) - 1))
          p.res[1] = s.err;
          p.res[2] = s.iter;
          p.res[3] = (s.err <= p.tol) ? 0.0 : (s.iter == p.max_iter ? 1.0 : 2.0);
          p.res[4] = c[4];
          p.res[5] = c[2];
          p.res[6] = sqrt(c[5]);
          p.res[7] = sqrt(c[3]);
          __threadfence_system();
          done[pi] = 1u;
        }
        if (lane == 0) s.st = ST_RETIRED;
        continue;
      }
      if (s.init == 2) {  // maximum of the cost over the team's strips
        double mx = 0.0;
        for (int k = lane; k < p.gp; k += 32) mx = fmax(mx, __ldcg(p.colp + (size_t)k * 4 + 2));
        mx = warp_max(mx);
        if (lane == 0) {
          s.cmax = mx;
          s.init = 1;
          ++running;
        }
        continue;
      }
      double er = 0.0, ec = 0.0, bad = 0.0;
      for (int u = lane; u < p.nunits; u += 32) {
        er += __ldcg(p.unitp + (size_t)u * 4 + 0);
        bad += __ldcg(p.unitp + (size_t)u * 4 + 1);
      }
      for (int k = lane; k < p.gp; k += 32) {
        ec += __ldcg(p.colp + (size_t)k * 4 + 0);
        bad += __ldcg(p.colp + (size_t)k * 4 + 1);
      }
      er = warp_sum(er);
      ec = warp_sum(ec);
      bad = warp_sum(bad);
      if (lane != 0) continue;
      if (bad != 0.0) {
        if (reporter) {
          p.res[3] = kUnsafeStatus;
          __threadfence_system();
          done[pi] = 1u;
        }
        s.st = ST_RETIRED;
        continue;
      }
      ++running;
      if (s.init) {  // u_1 = a / (K 1): no iteration counted
        s.init = 0;
        s.par ^= 1;
        continue;
      }
      ++s.iter;
      s.err = sqrt(er) + sqrt(ec);
      if (s.iter < p.max_iter && s.err >= p.tol) s.par ^= 1;
      else s.st = ST_FIN;
    }
    for (int pi = np + tid; pi < np_new; pi += NTT) S[pi] = State{ST_RUN, 0, 0, probs[pi].X ? 2 : 1, 1000.0, 1.0};
    double t[1] = {(double)(running + (tid == 0 ? np_new - np : 0))};
    block_sum_cols<1, NW>(t, red, par);  // (also orders the state updates before the next pass)
    np = np_new;
    if (timing && (int)pt[6] < 4096) prof[9 + 2 * (int)pt[6]] = t[0];
    lap(4);
    pt[6] += 1.0;
    if (t[0] != 0.0) last_busy = globaltimer_ns();
    else if (stop || idle) break;
  }
  if (timing)
    for (int i = 0; i < 7; ++i) prof[i] = pt[i];
  if (prof && tid == 0) prof[8 + 2 * 4096 + cta] = my_col_ns;
}

int row_class(int m) { return m <= 512 ? 0 : m <= 1024 ? 1 : m <= 2048 ? 2 : m <= 4096 ? 3 : 4; }

}  // namespace batch

// Per-launch bounds: problem count (shared-memory state) and total elements
// (the K build of one launch must stay well inside the bounded barrier wait).
constexpr long long kLaunchMaxElems = 1LL << 30;
// Problems with more than this many elements go through the per-call path:
// its grid-wide sweep streams them at the bandwidth bound with less
// per-iteration overhead than a lockstep iteration.
constexpr long long kBatchMaxElems = 4LL << 20;

enum { SBT_DESC = 200, SBT_K, SBT_WORK, SBT_CTRL, SBT_PROF, SBT_RES, SBT_HOSTIO = 210 };

// Placement of problem q on the grid: team size, offset, merge units and the
// row class (all functions of the problem and of the running placement
// pointers), and the sizes of its work arrays.
void place(const rwig_problem& q, int G, int& ptr, int& unit0, batch::Prob& d, long long& kdoubles,
           long long& wdoubles) {
  using namespace batch;
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  d.m = q.M;
  d.n = q.N;
  d.ldk = ((q.M + 1) / 2) * 2;
  d.gp = (int)std::min<long long>(
      std::min(G, q.N), std::max<long long>(1, ((long long)d.ldk * q.N * 8 + kStripBytes - 1) / kStripBytes));
  d.off = ptr;
  ptr = (ptr + d.gp) % G;
  d.nunits = (q.M + kUnit - 1) / kUnit;
  d.unit0 = unit0;
  unit0 = (unit0 + d.nunits) % G;
  d.max_iter = q.max_iter;
  d.cls = row_class(q.M);
  d.eps = q.reg;
  d.tol = q.zero_tol;
  d.a = q.a;
  d.b = q.b;
  d.C = q.C;
  d.X = q.C ? nullptr : q.X;
  d.Y = q.C ? nullptr : q.Y;
  d.d = q.C ? 0 : q.d;
  d.P = q.P;
  d.f = q.f;
  d.g = q.g;
  kdoubles = al(d.ldk * q.N);
  wdoubles = 2 * al(q.M) + al((long long)d.gp * q.M) + al(4LL * d.gp) + al(4LL * d.nunits) + 32 +
             (q.C ? 0 : al((long long)q.M * q.N));  // the cost built from points
}

// Points the work arrays of d into w (wdoubles doubles) and K into k.
void bind(batch::Prob& d, double* k, double* w, double* res) {
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  d.K = k;
  d.u0 = w;
  d.u1 = w + al(d.m);
  d.rowp = d.u1 + al(d.m);
  d.colp = d.rowp + al((long long)d.gp * d.m);
  d.unitp = d.colp + al(4LL * d.gp);
  d.res = res;
  if (d.X) d.C = d.unitp + al(4LL * d.nunits) + 32;
}

int launch_service(Context* ctx, cudaStream_t st, const batch::Prob* dprob, const unsigned* pub, unsigned* done,
                   unsigned* dctl, double* dprof, unsigned long long idle_ns) {
  using namespace batch;
  static bool attr = false;
  if (!attr) {
    RWIG_CUDA_TRY(
        cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes()));
    attr = true;
  }
  int nblk = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nblk, batch_kernel, NTT, smem_bytes()));
  if (nblk < 1) return set_error(RWIG_E_UNSUPPORTED, "batched Sinkhorn kernel does not fit on an SM");
  RWIG_CUDA_TRY(cudaMemsetAsync(dctl, 0, sizeof(unsigned) * 8, st));
  const Prob* dp = dprob;
  const volatile unsigned* pb = pub;
  volatile unsigned* dn = done;
  unsigned* ctl = dctl;
  double* pr = dprof;
  unsigned long long idle = idle_ns;
  void* args[] = {(void*)&dp, (void*)&pb, (void*)&dn, (void*)&ctl, (void*)&pr, (void*)&idle};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((void*)batch_kernel, dim3(ctx->sm_count), dim3(NTT), args,
                                            smem_bytes(), st));
  return 0;
}

// Prints the optional per-phase profile of the last launch (rwig_set_option
// "batch.profile").
int print_profile(Context* ctx, const double* dprof, int np) {
  const int G = ctx->sm_count;
  std::vector<double> hpv(8 + 2 * 4096 + 256);
  RWIG_CUDA_TRY(cudaMemcpy(hpv.data(), dprof, sizeof(double) * hpv.size(), cudaMemcpyDeviceToHost));
  const double* h = hpv.data();
  double mx = 0.0, mn = 1e300, sm = 0.0;
  for (int c = 0; c < G; ++c) {
    mx = std::max(mx, h[8 + 2 * 4096 + c]);
    mn = std::min(mn, h[8 + 2 * 4096 + c]);
    sm += h[8 + 2 * 4096 + c];
  }
  const int nit = std::min(4096, (int)h[6]);
  std::vector<double> tsum(6, 0.0);
  std::vector<int> tcnt(6, 0);
  for (int it = 0; it < nit; ++it) {
    const int r = (int)h[9 + 2 * it];
    const int b = r <= 1 ? 0 : r <= 2 ? 1 : r <= 4 ? 2 : r <= 16 ? 3 : r <= 64 ? 4 : 5;
    tsum[b] += h[8 + 2 * it];
    ++tcnt[b];
  }
  std::fprintf(stderr,
               "batch_kernel profile (CTA 0, ms): column passes %.3f | barrier 1 %.3f | merges %.3f | barrier 2 + "
               "decisions %.3f | iterations %.0f | problems %d\n  column pass per CTA (ms): max %.3f mean %.3f min "
               "%.3f\n  column pass by running problems (iterations, us):",
               h[1] * 1e-6, h[2] * 1e-6, h[3] * 1e-6, h[4] * 1e-6, h[6], np, mx * 1e-6, sm / G * 1e-6, mn * 1e-6);
  const char* lab[6] = {"<=1", "2", "3-4", "5-16", "17-64", ">64"};
  for (int b = 0; b < 6; ++b) std::fprintf(stderr, " %s: %d, %.1f |", lab[b], tcnt[b], tcnt[b] ? tsum[b] / tcnt[b] * 1e-3 : 0.0);
  std::fprintf(stderr, "\n");
  return 0;
}

// One launch over problems `idx` (all eligible for the kernel), every one
// published up front with the stop flag set.
static int launch_group(Context* ctx, cudaStream_t st, const rwig_problem* probs, const std::vector<int>& idx,
                        rwig_result* out, std::vector<int>& percall, int* launches) {
  using namespace batch;
  const int np = (int)idx.size();
  const int G = ctx->sm_count;
  if (G > kMaxTeam) return set_error(RWIG_E_UNSUPPORTED, "more SMs than the batched kernel's team limit");
  std::vector<Prob> hp(np);
  std::vector<long long> koff(np), woff(np);
  long long kd = 0, wd = 0;
  int ptr = 0, unit0 = 0;
  // team placement, largest problems first; the problem order stays as given
  std::vector<int> ord(np);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
    return (long long)probs[idx[x]].M * probs[idx[x]].N > (long long)probs[idx[y]].M * probs[idx[y]].N;
  });
  for (int t : ord) {
    long long k1, w1;
    place(probs[idx[t]], G, ptr, unit0, hp[t], k1, w1);
    koff[t] = kd;
    woff[t] = wd;
    kd += k1;
    wd += w1;
  }
  Prob* dprob = (Prob*)scratch(ctx, SBT_DESC, sizeof(Prob) * np);
  double* dK = (double*)scratch(ctx, SBT_K, sizeof(double) * std::max<long long>(kd, 32));
  double* dW = (double*)scratch(ctx, SBT_WORK, sizeof(double) * std::max<long long>(wd, 32));
  double* dres = (double*)scratch(ctx, SBT_RES, sizeof(double) * 10 * np);
  unsigned* ctrl = (unsigned*)scratch(ctx, SBT_CTRL, sizeof(unsigned) * (8 + 2 + kMaxProbs));
  const bool profile = option("batch.profile", 0.0) != 0.0;
  double* dprof = profile ? (double*)scratch(ctx, SBT_PROF, sizeof(double) * (8 + 2 * 4096 + 256)) : nullptr;
  if (!dprob || !dK || !dW || !dres || !ctrl || (profile && !dprof)) return RWIG_E_NOMEM;
  for (int t = 0; t < np; ++t) bind(hp[t], dK + koff[t], dW + woff[t], dres + 10 * (size_t)t);
  unsigned* pub = ctrl + 8;
  unsigned* done = ctrl + 10;
  const unsigned hpub[2] = {(unsigned)np, 1u};
  RWIG_CUDA_TRY(cudaMemcpyAsync(dprob, hp.data(), sizeof(Prob) * np, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(pub, hpub, sizeof(hpub), cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(unsigned) * kMaxProbs, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(dres, 0, sizeof(double) * 10 * np, st));
  const int rc = launch_service(ctx, st, dprob, pub, done, ctrl, dprof, 0ull);
  if (rc) return rc;
  ++*launches;
  std::vector<double> hres(10 * (size_t)np);
  RWIG_CUDA_TRY(cudaMemcpyAsync(hres.data(), dres, sizeof(double) * 10 * np, cudaMemcpyDeviceToHost, st));
  unsigned hctl[4] = {0, 0, 0, 0};
  RWIG_CUDA_TRY(cudaMemcpyAsync(hctl, ctrl, sizeof(hctl), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (hctl[2]) return set_error(RWIG_E_TIMEOUT, "a bounded wait in the batched Sinkhorn kernel expired");
  if (profile) {
    const int rc2 = print_profile(ctx, dprof, np);
    if (rc2) return rc2;
  }
  for (int t = 0; t < np; ++t) {
    rwig_result& o = out[idx[t]];
    const double* r = hres.data() + 10 * (size_t)t;
    if (r[3] == kUnsafeStatus) {
      if (probs[idx[t]].C) percall.push_back(idx[t]);
      else o.status = RWIG_E_UNSUPPORTED;  // outside the scaling form; the per-call path takes C
      continue;
    }
    o.loss = r[0];
    o.err = r[1];
    o.iter = (int)r[2];
    o.status = (int)r[3];
    o.marg_l1_row = r[4];
    o.marg_l1_col = r[5];
    o.path = 0;
  }
  return 0;
}

// Batched solve on device pointers; out[i] receives each problem's result.
// Returns 0, or a negative error for the whole call.
int batch_device(Context* ctx, cudaStream_t st, const rwig_problem* probs, int count, rwig_result* out) {
  using namespace batch;
  if (count < 0 || (count > 0 && (!probs || !out))) return set_error(RWIG_E_INVALID, "bad batch arguments");
  std::vector<int> eligible, percall;
  for (int i = 0; i < count; ++i) {
    const rwig_problem& q = probs[i];
    out[i] = rwig_result{};
    const bool pts = !q.C && q.X && q.Y && q.d >= 1;
    if (!q.a || !q.b || !(q.C || pts) || !q.f || !q.g || q.M < 1 || q.N < 1 || !(q.reg > 0.0) ||
        !std::isfinite(q.reg)) {
      out[i].status = RWIG_E_INVALID;
      continue;
    }
    if (pts && (q.M > kMaxRows || q.max_iter < 1)) {
      out[i].status = RWIG_E_UNSUPPORTED;  // the per-call path takes a cost matrix
      continue;
    }
    if (q.M <= kMaxRows && q.max_iter >= 1 && (pts || (long long)q.M * q.N <= kBatchMaxElems))
      eligible.push_back(i);
    else
      percall.push_back(i);
  }
  int launches = 0;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->evs0, st));
  // launches of at most kMaxProbs problems and kLaunchMaxElems elements
  size_t s = 0;
  while (s < eligible.size()) {
    std::vector<int> grp;
    long long el = 0;
    while (s < eligible.size() && (int)grp.size() < kMaxProbs) {
      const long long e = (long long)probs[eligible[s]].M * probs[eligible[s]].N;
      if (!grp.empty() && el + e > kLaunchMaxElems) break;
      grp.push_back(eligible[s]);
      el += e;
      ++s;
    }
    const int rc = launch_group(ctx, st, probs, grp, out, percall, &launches);
    if (rc) return rc;
  }
  RWIG_CUDA_TRY(cudaEventRecord(ctx->evs1, st));
  RWIG_CUDA_TRY(cudaEventSynchronize(ctx->evs1));
  float bms = 0.f;
  cudaEventElapsedTime(&bms, ctx->evs0, ctx->evs1);
  for (int i : percall) {
    const rwig_problem& q = probs[i];
    rwig_result& o = out[i];
    double loss = 0.0, err = 0.0;
    int it = 0;
    const int rc = sinkhorn_device(ctx, st, false, q.P, nullptr, q.f, q.g, &loss, &it, &err, q.a, q.b, q.C, q.M,
                                   q.N, q.reg, 0, q.max_iter, q.zero_tol);
    const rwig_report& R = report();
    o.loss = loss;
    o.err = err;
    o.iter = it;
    o.status = rc;
    o.marg_l1_row = R.marg_l1_row;
    o.marg_l1_col = R.marg_l1_col;
    o.device_us = R.device_ms * 1e3;
    o.path = 1;
    launches += R.kernel_launches;
  }
  reset_report();
  report().kernel_launches = launches;
  report().sweep_ms = bms;  // device time of the batched launches
  return 0;
}

}  // namespace rwig

using namespace rwig;

extern "C" int rwig_batch_sinkhorn_log(const rwig_problem* probs, int count, rwig_result* out) {
  reset_report();
  if (count < 0 || (count > 0 && (!probs || !out))) return set_error(RWIG_E_INVALID, "bad batch arguments");
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = ctx->stream;
  // one device block for every problem's a, b, C, P, f, g (256-byte aligned slices)
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  std::vector<long long> off(count + 1, 0);
  auto cost_doubles = [&](const rwig_problem& q) -> long long {  // C, or the points
    const long long M = std::max(q.M, 0), N = std::max(q.N, 0);
    return q.C ? al(M * N) : al(M * std::max(q.d, 0)) + al(N * std::max(q.d, 0));
  };
  for (int i = 0; i < count; ++i) {
    const rwig_problem& q = probs[i];
    const long long M = std::max(q.M, 0), N = std::max(q.N, 0);
    off[i + 1] = off[i] + al(M) + al(N) + cost_doubles(q) + (q.P ? al(M * N) : 0) + al(M) + al(N);
  }
  double* dev = (double*)scratch(ctx, SBT_HOSTIO, sizeof(double) * std::max<long long>(off[count], 32));
  if (!dev) return RWIG_E_NOMEM;
  std::vector<rwig_problem> dp(probs, probs + count);
  for (int i = 0; i < count; ++i) {
    const rwig_problem& q = probs[i];
    const bool pts = !q.C && q.X && q.Y && q.d >= 1;
    if (!q.a || !q.b || !(q.C || pts) || !q.f || !q.g || q.M < 1 || q.N < 1) {
      dp[i].a = nullptr;  // rejected by the device driver with RWIG_E_INVALID
      continue;
    }
    const long long M = q.M, N = q.N;
    double* da = dev + off[i];
    double* db = da + al(M);
    double* dC = db + al(N);
    double* dP = q.P ? dC + cost_doubles(q) : nullptr;
    double* df = q.P ? dP + al(M * N) : dC + cost_doubles(q);
    double* dg = df + al(M);
    RWIG_CUDA_TRY(cudaMemcpyAsync(da, q.a, sizeof(double) * M, cudaMemcpyHostToDevice, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(db, q.b, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    if (pts) {
      double* dX = dC;
      double* dY = dC + al(M * q.d);
      RWIG_CUDA_TRY(cudaMemcpyAsync(dX, q.X, sizeof(double) * M * q.d, cudaMemcpyHostToDevice, st));
      RWIG_CUDA_TRY(cudaMemcpyAsync(dY, q.Y, sizeof(double) * N * q.d, cudaMemcpyHostToDevice, st));
      dp[i].X = dX;
      dp[i].Y = dY;
      dC = nullptr;
    } else {
      RWIG_CUDA_TRY(cudaMemcpyAsync(dC, q.C, sizeof(double) * M * N, cudaMemcpyHostToDevice, st));
    }
    dp[i].a = da;
    dp[i].b = db;
    dp[i].C = dC;
    dp[i].P = dP;
    dp[i].f = df;
    dp[i].g = dg;
  }
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
  const int rc = batch_device(ctx, st, dp.data(), count, out);
  if (rc) return rc;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  for (int i = 0; i < count; ++i) {
    if (!dp[i].a) continue;
    const long long M = probs[i].M, N = probs[i].N;
    if (probs[i].P)
      RWIG_CUDA_TRY(cudaMemcpyAsync(probs[i].P, dp[i].P, sizeof(double) * M * N, cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(probs[i].f, dp[i].f, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(probs[i].g, dp[i].g, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  }
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  report().device_ms = ms;
  report().kernel_ms = ms;
  return 0;
}

extern "C" int rwig_batch_sinkhorn_log_dev(const rwig_problem* probs, int count, rwig_result* out, void* stream) {
  reset_report();
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
  const int rc = batch_device(ctx, st, probs, count, out);
  if (rc) return rc;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  RWIG_CUDA_TRY(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  report().device_ms = ms;
  report().kernel_ms = ms;
  return 0;
}

// ---------------------------------------------------------------------------
// Serving: requests are admitted into the running service kernel as they
// arrive (continuous batching).  The caller drives the server from one
// thread: submit() copies a request in and publishes it, poll() collects
// finished ones.  Admission is bounded by a device-memory budget and by the
// slot table of one launch (kMaxProbs); a full table is reused once every
// slot of it has been collected and the kernel has gone idle.
// ---------------------------------------------------------------------------
struct rwig_server {
  rwig::Context* ctx = nullptr;
  cudaStream_t ks = nullptr, cs = nullptr;  // kernel stream, copy stream
  rwig::batch::Prob* dprob = nullptr;       // device, kMaxProbs descriptors
  unsigned* hpub = nullptr;                 // mapped: [0] published count, [1] stop
  unsigned* dpub = nullptr;
  unsigned* hdone = nullptr;                // mapped: done flag per slot
  unsigned* ddone = nullptr;
  double* hres = nullptr;                   // mapped: 10 results per slot
  double* dres = nullptr;
  unsigned* dctl = nullptr;                 // device control words
  unsigned hctl_err = 0;
  int nslots = 0, npub = 0, ptr = 0, unit0 = 0, next_ticket = 0;
  bool launched = false;
  double budget = 0.0, inflight = 0.0;
  unsigned long long idle_ns = 0;
  struct Slot {
    int ticket = -1;
    void* mem = nullptr;
    double bytes = 0.0;
    double *df = nullptr, *dg = nullptr, *dP = nullptr;
    double *hf = nullptr, *hg = nullptr, *hP = nullptr;
    int M = 0, N = 0;
    bool collected = true;
    cudaEvent_t ev = nullptr;  // the slot's copies have landed
  };
  std::vector<Slot> slots;
  std::vector<rwig::batch::Prob> staged;  // host copies of the descriptors (asynchronous copy sources)
};

namespace rwig {
namespace {

bool kernel_running(rwig_server* s) {
  if (!s->launched) return false;
  const cudaError_t e = cudaStreamQuery(s->ks);
  if (e == cudaErrorNotReady) return true;
  s->launched = false;
  (void)cudaGetLastError();
  return false;
}

int ensure_running(rwig_server* s) {
  if (kernel_running(s)) return 0;
  unsigned err = 0;
  RWIG_CUDA_TRY(cudaMemcpy(&err, s->dctl + 2, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (err) return set_error(RWIG_E_TIMEOUT, "a bounded wait in the serving kernel expired");
  bool pending = false;
  for (int i = 0; i < s->npub; ++i)
    if (!s->hdone[i]) pending = true;
  if (!pending) return 0;
  const int rc = launch_service(s->ctx, s->ks, s->dprob, s->dpub, s->ddone, s->dctl, nullptr, s->idle_ns);
  if (rc) return rc;
  s->launched = true;
  return 0;
}

// Publishes, in slot order, the submitted requests whose copies have landed.
int publish_ready(rwig_server* s) {
  const int before = s->npub;
  while (s->npub < s->nslots) {
    const cudaError_t e = cudaEventQuery(s->slots[s->npub].ev);
    if (e == cudaErrorNotReady) break;
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventQuery");
    ++s->npub;
  }
  if (s->npub != before) {
    std::atomic_thread_fence(std::memory_order_seq_cst);  // descriptors and buffers before the count
    *(volatile unsigned*)s->hpub = (unsigned)s->npub;
  }
  return ensure_running(s);
}

}  // namespace
}  // namespace rwig

extern "C" int rwig_server_create(rwig_server** out, double mem_budget_bytes, double idle_ms) {
  reset_report();
  if (!out) return set_error(RWIG_E_INVALID, "out is null");
  *out = nullptr;
  if (!(mem_budget_bytes > 0.0)) return set_error(RWIG_E_INVALID, "memory budget must be > 0");
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  if (ctx->sm_count > batch::kMaxTeam) return set_error(RWIG_E_UNSUPPORTED, "more SMs than the team limit");
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto* s = new rwig_server();
  s->ctx = ctx;
  s->budget = mem_budget_bytes;
  s->idle_ns = (unsigned long long)(std::max(0.0, idle_ms) * 1e6);
  s->slots.resize(batch::kMaxProbs);
  s->staged.resize(batch::kMaxProbs);
  auto fail = [&](cudaError_t e, const char* what) {
    rwig_server_destroy(s);
    return cuda_fail(e, what);
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s->ks, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
  if ((e = cudaStreamCreateWithFlags(&s->cs, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
  if ((e = cudaMalloc(&s->dprob, sizeof(batch::Prob) * batch::kMaxProbs)) != cudaSuccess) return fail(e, "descriptors");
  if ((e = cudaMalloc(&s->dctl, sizeof(unsigned) * 8)) != cudaSuccess) return fail(e, "control");
  if ((e = cudaHostAlloc(&s->hpub, sizeof(unsigned) * 2, cudaHostAllocMapped)) != cudaSuccess) return fail(e, "pub");
  if ((e = cudaHostAlloc(&s->hdone, sizeof(unsigned) * batch::kMaxProbs, cudaHostAllocMapped)) != cudaSuccess)
    return fail(e, "done");
  if ((e = cudaHostAlloc(&s->hres, sizeof(double) * 10 * batch::kMaxProbs, cudaHostAllocMapped)) != cudaSuccess)
    return fail(e, "results");
  if ((e = cudaHostGetDevicePointer(&s->dpub, s->hpub, 0)) != cudaSuccess) return fail(e, "pub map");
  if ((e = cudaHostGetDevicePointer(&s->ddone, s->hdone, 0)) != cudaSuccess) return fail(e, "done map");
  if ((e = cudaHostGetDevicePointer(&s->dres, s->hres, 0)) != cudaSuccess) return fail(e, "results map");
  if ((e = cudaMemset(s->dctl, 0, sizeof(unsigned) * 8)) != cudaSuccess) return fail(e, "control");
  for (auto& sl : s->slots)
    if ((e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "events");
  s->hpub[0] = 0;
  s->hpub[1] = 0;
  std::memset(s->hdone, 0, sizeof(unsigned) * batch::kMaxProbs);
  *out = s;
  return 0;
}

extern "C" int rwig_server_submit(rwig_server* s, const rwig_problem* q) {
  reset_report();
  if (!s || !q) return set_error(RWIG_E_INVALID, "null server or problem");
  const bool pts = !q->C && q->X && q->Y && q->d >= 1;
  if (!q->a || !q->b || !(q->C || pts) || !q->f || !q->g || q->M < 1 || q->N < 1 || !(q->reg > 0.0) ||
      !std::isfinite(q->reg) || q->max_iter < 1)
    return set_error(RWIG_E_INVALID, "bad problem");
  if (q->M > batch::kMaxRows) return set_error(RWIG_E_UNSUPPORTED, "M above 8192");
  std::lock_guard<std::mutex> lk(s->ctx->mu);
  using namespace batch;
  // a fresh slot table once every slot of the current one has been collected
  if (s->nslots == kMaxProbs) {
    bool all = true;
    for (int i = 0; i < s->nslots; ++i) all = all && s->slots[i].collected;
    if (!all || kernel_running(s)) return RWIG_E_BUSY;
    s->nslots = 0;
    s->npub = 0;
    std::memset(s->hdone, 0, sizeof(unsigned) * kMaxProbs);
    std::atomic_thread_fence(std::memory_order_seq_cst);
    *(volatile unsigned*)s->hpub = 0u;
  }
  Prob d{};
  long long kd = 0, wd = 0;
  int ptr = s->ptr, unit0 = s->unit0;
  place(*q, s->ctx->sm_count, ptr, unit0, d, kd, wd);
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  const long long M = q->M, N = q->N;
  const long long cd = pts ? al(M * q->d) + al(N * q->d) : al(M * N);  // C, or the points
  const long long io = al(M) + al(N) + cd + al(M) + al(N) + (q->P ? al(M * N) : 0);
  const double bytes = 8.0 * (double)(io + kd + wd);
  if (s->inflight + bytes > s->budget) return RWIG_E_BUSY;
  void* mem = nullptr;
  RWIG_CUDA_TRY(cudaMallocAsync(&mem, (size_t)bytes, s->cs));
  double* base = (double*)mem;
  double* da = base;
  double* db = da + al(M);
  double* dC = db + al(N);
  double* df = dC + cd;
  double* dg = df + al(M);
  double* dP = q->P ? dg + al(N) : nullptr;
  double* dk = base + io;
  double* dw = dk + kd;
  RWIG_CUDA_TRY(cudaMemcpyAsync(da, q->a, sizeof(double) * M, cudaMemcpyHostToDevice, s->cs));
  RWIG_CUDA_TRY(cudaMemcpyAsync(db, q->b, sizeof(double) * N, cudaMemcpyHostToDevice, s->cs));
  const int slot = s->nslots;
  if (pts) {
    RWIG_CUDA_TRY(cudaMemcpyAsync(dC, q->X, sizeof(double) * M * q->d, cudaMemcpyHostToDevice, s->cs));
    RWIG_CUDA_TRY(
        cudaMemcpyAsync(dC + al(M * q->d), q->Y, sizeof(double) * N * q->d, cudaMemcpyHostToDevice, s->cs));
    d.X = dC;
    d.Y = dC + al(M * q->d);
    d.C = nullptr;
  } else {
    RWIG_CUDA_TRY(cudaMemcpyAsync(dC, q->C, sizeof(double) * M * N, cudaMemcpyHostToDevice, s->cs));
    d.C = dC;
  }
  d.a = da;
  d.b = db;
  d.f = df;
  d.g = dg;
  d.P = dP;
  bind(d, dk, dw, s->dres + 10 * (size_t)slot);
  s->staged[slot] = d;  // the copy source must outlive the asynchronous copy
  RWIG_CUDA_TRY(cudaMemcpyAsync(s->dprob + slot, &s->staged[slot], sizeof(Prob), cudaMemcpyHostToDevice, s->cs));
  RWIG_CUDA_TRY(cudaEventRecord(s->slots[slot].ev, s->cs));
  s->ptr = ptr;
  s->unit0 = unit0;
  auto& sl = s->slots[slot];
  sl.ticket = s->next_ticket++;
  sl.mem = mem;
  sl.bytes = bytes;
  sl.df = df;
  sl.dg = dg;
  sl.dP = dP;
  sl.hf = q->f;
  sl.hg = q->g;
  sl.hP = q->P;
  sl.M = q->M;
  sl.N = q->N;
  sl.collected = false;
  s->inflight += bytes;
  s->hdone[slot] = 0u;
  s->nslots = slot + 1;
  const int rc = publish_ready(s);
  if (rc) return rc;
  return sl.ticket;
}

extern "C" int rwig_server_poll(rwig_server* s, int ticket, rwig_result* out) {
  reset_report();
  if (!s || !out) return set_error(RWIG_E_INVALID, "null server or result");
  std::lock_guard<std::mutex> lk(s->ctx->mu);
  int slot = -1;
  for (int i = 0; i < s->nslots; ++i)
    if (s->slots[i].ticket == ticket && !s->slots[i].collected) slot = i;
  if (slot < 0) return set_error(RWIG_E_INVALID, "unknown or already collected ticket");
  if (slot >= s->npub || !*(volatile unsigned*)(s->hdone + slot)) {
    const int rc = publish_ready(s);  // and restart a kernel that went idle before seeing it
    return rc ? rc : 0;
  }
  std::atomic_thread_fence(std::memory_order_seq_cst);
  auto& sl = s->slots[slot];
  const double* r = s->hres + 10 * (size_t)slot;
  *out = rwig_result{};
  if (r[3] == batch::kUnsafeStatus) {
    out->status = RWIG_E_UNSUPPORTED;  // outside the scaling form: solve with rwig_sinkhorn_log
  } else {
    out->loss = r[0];
    out->err = r[1];
    out->iter = (int)r[2];
    out->status = (int)r[3];
    out->marg_l1_row = r[4];
    out->marg_l1_col = r[5];
    RWIG_CUDA_TRY(cudaMemcpyAsync(sl.hf, sl.df, sizeof(double) * sl.M, cudaMemcpyDeviceToHost, s->cs));
    RWIG_CUDA_TRY(cudaMemcpyAsync(sl.hg, sl.dg, sizeof(double) * sl.N, cudaMemcpyDeviceToHost, s->cs));
    if (sl.hP)
      RWIG_CUDA_TRY(cudaMemcpyAsync(sl.hP, sl.dP, sizeof(double) * sl.M * sl.N, cudaMemcpyDeviceToHost, s->cs));
  }
  out->path = 0;
  RWIG_CUDA_TRY(cudaFreeAsync(sl.mem, s->cs));
  RWIG_CUDA_TRY(cudaStreamSynchronize(s->cs));
  s->inflight -= sl.bytes;
  sl.collected = true;
  sl.mem = nullptr;
  return 1;
}

extern "C" int rwig_server_destroy(rwig_server* s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->ctx->mu);
    if (s->hpub) {
      s->hpub[1] = 1u;  // stop: the kernel ends once nothing runs
      std::atomic_thread_fence(std::memory_order_seq_cst);
    }
    if (s->ks) cudaStreamSynchronize(s->ks);
    for (auto& sl : s->slots)
      if (sl.mem) cudaFreeAsync(sl.mem, s->cs);
    if (s->cs) cudaStreamSynchronize(s->cs);
    if (s->dprob) cudaFree(s->dprob);
    if (s->dctl) cudaFree(s->dctl);
    if (s->hpub) cudaFreeHost(s->hpub);
    if (s->hdone) cudaFreeHost(s->hdone);
    if (s->hres) cudaFreeHost(s->hres);
    for (auto& sl : s->slots)
      if (sl.ev) cudaEventDestroy(sl.ev);
    if (s->ks) cudaStreamDestroy(s->ks);
    if (s->cs) cudaStreamDestroy(s->cs);
  }
  delete s;
  return 0;
}
