// batch.cu -- many log-stabilised Sinkhorn problems of different sizes in one
// persistent launch, each solved by its own team of CTAs.
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
// Scheduling.  The grid is one CTA per SM.  Problem p is solved by a team of
// gp CTAs (gp a function of the problem alone); a free CTA claims the next
// member slot of the oldest problem whose team is not yet complete (one
// atomic counter per problem), so teams form in problem order and at most one
// team is incomplete at any time: its members wait only for CTAs that are
// finishing other problems, never for each other in a cycle.  A team
// synchronises through its own counter in global memory; nothing waits on the
// whole grid.
//
// Work split.  Member k holds the column strip [k n/gp, (k+1) n/gp) of K with
// every row, so its column sums are complete inside the CTA.
//  * resident strips (<= 184 KB): K is built straight into shared memory by
//    the first pass and stays there, so an iteration reads no K from memory;
//  * streamed strips (larger problems): K is built in global memory and
//    streamed through a bulk-copy ring every iteration (kept in L2 when it fits).
// Rows with m <= 512 are processed warp per column (lanes own rows, a warp
// reduction per column); larger m thread per row (a block reduction per
// group of columns).  Row sums of the members are merged in a fixed order
// either redundantly by every member (small teams: one team barrier per
// iteration) or split over the members (two barriers).  Every reduction order
// depends only on the problem, so a result is bitwise the same whatever else
// is in the batch.  A problem whose scalings leave [e^-650, e^650], whose
// masses are not all positive or whose sums leave the safe range is handed
// back (status kUnsafe) and re-solved by the per-call path.
//
// Every wait is bounded: team barriers after 2 s, and a member waiting for its
// team to form as long as other teams progress (2 s without progress ends it);
// on expiry the kernel sets an error word, drains its copies and returns, and
// the host reports RWIG_E_TIMEOUT.
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
constexpr int kSlot = 8192;                // doubles per streamed stage (64 KB: CW x 512 RPT for every row class)
constexpr int kArea = 27648;               // doubles of the strip area (216 KB): stage ring or resident strip
constexpr int kTree = 4096;                // doubles at the end of the area for the warp-mode row tree
constexpr int kResident = kArea - kTree;   // largest resident strip (184 KB)
constexpr int kWarpRows = 512;             // m <= this: warp-per-column passes
constexpr int kMaxRows = 8192;
constexpr int kUnit = 64;                  // rows per merge unit (4 per warp)
constexpr int kMaxProbs = 512;             // descriptor slots; problem number h lives in slot h % kMaxProbs
constexpr int kCtlPerSlot = 8;             // control words per slot (Prob::ctl)
constexpr int kMaxTeam = 160;              // CTAs of a team (the grid is one CTA per SM)
constexpr double kScaleMin = 5.1e-283, kScaleMax = 1.95e282;  // e^-650, e^650
constexpr double kUnsafeStatus = -100.0;
constexpr unsigned kClosed = 0x80000000u;
constexpr int kResStride = 16;  // doubles of results per problem

enum : int { MODE_RESIDENT = 1, MODE_WARP = 2, MODE_REDUNDANT = 4, MODE_KEEP_L2 = 8 };

// Device control words of a launch.
enum : int { DC_AVAIL = 0, DC_HEAD = 1, DC_ERR = 2, DC_PROGRESS = 3, DC_ACTIVE = 4, DC_FREE = 5, DC_OLDEST = 6,
             DC_OLDEST_T = 7, DC_PUB_T = 8, kCtlWords = 16 };

struct Prob {
  const double* a;
  const double* b;
  const double* C;   // m x n, column-major, leading dimension m (built here when X, Y are given)
  const double* X;   // m x d source points (column-major) or null
  const double* Y;   // n x d target points or null
  int d;
  double* K;         // streamed strips: m x n, leading dimension ldk
  long long ldk;     // even, >= m
  double* P;         // optional plan (leading dimension m)
  double* f;         // m
  double* g;         // n; holds v during the iterations
  double* rowp;      // [2][gp][m] row partials (by round parity)
  double* colp;      // [2][gp][4] column-strip partials
  double* mrgp;      // [2][gp][4] merge partials (split merges)
  double* ug;        // [2][m] u (split merges)
  unsigned* ctl;     // kCtlPerSlot words: 64-bit claim word at [0] (problem number << 32 | gp << 16 |
                     // claimed member slots), 64-bit state word at [2] (problem number << 32 | 0 unopened,
                     // 1 opened, 2 opening), [4] team barrier arrivals
  double* res;       // [16]: loss, err, iter, status, l1 row, l1 col, l2 row, l2 col, device ns, formation
                     // ns, then member 0's ns in column passes, merges + decisions, team barriers
  int m, n, max_iter, gp, mode, nunits;
  double eps, tol;
};

struct Shared {
  double* area;      // kArea doubles
  uint64_t* bar;     // STAGES mbarriers
  double* su;        // kWarpRows doubles: u in warp mode
  double* red;       // 2 * NW * 16 doubles: block reductions
  double* dec;       // 8 doubles: values broadcast to the CTA
  double* tim;       // 4 doubles: thread 0's phase timers
  int* flag;         // 4 ints
};

// dynamic shared memory of one CTA
__host__ __device__ constexpr size_t smem_bytes() {
  return (size_t)kArea * 8 + 64 + (size_t)kWarpRows * 8 + (size_t)2 * NW * 16 * 8 + 8 * 8 + 4 * 8 + 4 * 4 +
         sizeof(Prob) + 64;
}

__device__ __forceinline__ int strip_begin(int n, int gp, int k) { return (int)(((long long)k * n) / gp); }

// Waits until the team counter reaches target (thread 0).  A forming team
// waits as long as some other team makes progress; a formed team 2 s at most.
__device__ bool team_wait(unsigned* cnt, unsigned target, unsigned* dctl, bool forming) {
  __threadfence();
  asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(cnt) : "memory");
  unsigned long long t0 = 0;
  unsigned p0 = 0;
  for (unsigned spin = 0;; ++spin) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
    if ((int)(v - target) >= 0) return true;
    if ((spin & 63u) == 0u) {
      if (*(volatile unsigned*)(dctl + DC_ERR) != 0u) return false;
      const unsigned long long now = globaltimer_ns();
      if (forming) {
        const unsigned pv = *(volatile unsigned*)(dctl + DC_PROGRESS);
        if (t0 == 0 || pv != p0) {
          p0 = pv;
          t0 = now;
        }
      } else if (t0 == 0) {
        t0 = now;
      }
      if (now - t0 > kWaitLimitNs) {
        atomicOr(dctl + DC_ERR, KERR_BARRIER_TIMEOUT);
        return false;
      }
    }
  }
}

// Team barrier (all threads).  Single-member teams need only the block barrier.
__device__ __forceinline__ bool team_sync(const Prob& p, unsigned& nb, bool forming, unsigned* dctl, const Shared sh,
                                          double* prof_wait) {
  __syncthreads();
  if (p.gp == 1) return true;
  ++nb;
  if (threadIdx.x == 0) {
    const unsigned long long t = prof_wait ? globaltimer_ns() : 0ull;
    sh.flag[0] = team_wait(p.ctl + 4, nb * (unsigned)p.gp, dctl, forming) ? 1 : 0;
    if (prof_wait) *prof_wait += (double)(globaltimer_ns() - t);
  }
  __syncthreads();
  return sh.flag[0] != 0;
}

// ---------------------------------------------------------------- stage ring
// Streamed strips: the strip's column groups cycle through STAGES shared
// buffers; the q-th consumed stage (q counts across problems, so the mbarrier
// phases stay consistent) holds group (q - q0) mod ngroups.  Thread 0 issues.
struct Ring {
  double* buf;
  uint64_t* bar;
  uint64_t pol;
  const double* K;
  long long ldk;
  int c0, c1, cw, ngroups;
  unsigned q0;
  __device__ double* slot(unsigned seq) const { return buf + (size_t)(seq % STAGES) * kSlot; }
  __device__ int group_begin(unsigned seq) const { return c0 + (int)((seq - q0) % (unsigned)ngroups) * cw; }
  __device__ void issue(unsigned seq) const {
    const int jb = group_begin(seq);
    const unsigned bytes = (unsigned)(min(cw, c1 - jb) * ldk * 8);
    uint64_t* b = bar + (seq % STAGES);
    mbar_arrive_expect_tx(b, bytes);
    bulk_g2s_hint(slot(seq), K + (size_t)jb * ldk, bytes, b, pol);
  }
  __device__ bool wait(unsigned seq) const { return mbar_wait_bounded(bar + (seq % STAGES), (seq / STAGES) & 1u); }
};

// ---------------------------------------------------------------- passes
// Cost from points over this member's strip: C_ij = sum_k (x_ik - y_jk)^2 in
// ascending k, each step rounded separately (the same operations and order as
// a host that computes the differences, squares and sums elementwise, so the
// same bits), stored un-normalised; the strip's maximum is returned (block max).
__device__ double cost_pass(const Prob& p, int c0, int c1, double* red) {
  const int m = p.m, n = p.n, dim = p.d;
  const double* const X = p.X;
  const double* const Y = p.Y;
  double* const C = const_cast<double*>(p.C);
  double mx = 0.0;
  for (int j = c0; j < c1; ++j)
    for (int i = threadIdx.x; i < m; i += NTT) {
      double acc = 0.0;
      for (int q = 0; q < dim; ++q) {
        const double t = __dsub_rn(X[i + (size_t)q * m], Y[j + (size_t)q * n]);
        acc = __dadd_rn(acc, __dmul_rn(t, t));
      }
      C[i + (size_t)j * m] = acc;
      mx = fmax(mx, acc);
    }
  mx = warp_max(mx);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  double v = 0.0;
  for (int q = 0; q < NW; ++q) v = fmax(v, red[q]);
  __syncthreads();
  return v;  // exact and order-free
}

// First pass over the strip: K = exp(-C/eps) (sinkhorn_impl_vanilla.cpp:41
// form) into shared memory (resident) or global memory (streamed), row
// partials of K 1 -> rowp[0][k] (merged into u_1 = a / (K 1)), and whether a
// mass of the strip's columns or (member 0) of the rows is not positive.
template <int RPT>
__device__ double init_pass(const Prob& p, int k, int c0, int c1, double cmax, double* Kres, double* red, int& par) {
  const int tid = threadIdx.x;
  const int m = p.m;
  double r[RPT];
  bool valid[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    valid[t] = tid + t * NTT < m;
    r[t] = 0.0;
  }
  const bool res = (p.mode & MODE_RESIDENT) != 0;
  double* const C = const_cast<double*>(p.C);
  double* const Kg = p.K;
  const long long ldk = p.ldk;
  const bool pts = p.X != nullptr;
  const double eps = p.eps;
#pragma unroll 2
  for (int j = c0; j < c1; ++j) {
    double* cj = C + (size_t)j * m;
    double* kj = res ? Kres + (size_t)(j - c0) * ldk : Kg + (size_t)j * ldk;
#pragma unroll
    for (int t = 0; t < RPT; ++t)
      if (valid[t]) {
        double c = cj[tid + t * NTT];
        if (pts) {  // C /= max C
          c = c / cmax;
          cj[tid + t * NTT] = c;
        }
        const double x = exp(-c / eps);
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
  if (!res) asm volatile("fence.proxy.async.global;" ::: "memory");  // K is read next by bulk copies
#pragma unroll
  for (int t = 0; t < RPT; ++t)
    if (valid[t]) p.rowp[(size_t)k * m + tid + t * NTT] = r[t];
  double tt[1] = {bad};
  block_sum_cols<1, NW>(tt, red, par);
  return tt[0];
}

// Column pass, warp per column (m <= 32 RPL <= 512, resident strip): warp w
// takes the strip's columns w, w + NW, ...; lanes own rows lane + 32 j.
// Column sum with u (from su), v = b / s, row partials r += K v.  The warps'
// row partials are added in a fixed tree; the CTA's go to rowp[buf][k].
template <int RPL>
__device__ __noinline__ void warp_pass(const Prob& p, int k, int buf, int c0, int c1, const double* Ks, const Shared sh, int& par,
                          double& errc, double& bad) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  // every field used in the loops is read once here: stores through the
  // plan pointers would otherwise force reloads of the descriptor
  const int m = p.m;
  const long long ldk = p.ldk;
  const double* const bb = p.b + c0;
  double* const gg = p.g + c0;
  double* const rp_out = p.rowp + ((size_t)buf * p.gp + k) * m;
  const double* const su = sh.su;
  double* const tree = sh.area + kResident;
  double* const red = sh.red;
  // u in registers, or (16 rows per lane) read from su at each use
  constexpr bool kUReg = RPL <= 8;
  double u[kUReg ? RPL : 1], r[RPL];
#pragma unroll
  for (int j = 0; j < RPL; ++j) {
    const int i = lane + 32 * j;
    if (kUReg) u[kUReg ? j : 0] = i < m ? su[i] : 0.0;
    r[j] = 0.0;
  }
  double e = 0.0, bd = 0.0;
  const int nc = c1 - c0;
  auto column = [&](int c, double (&kv)[RPL], double& s) {
    const double* col = Ks + (size_t)c * ldk;
    s = 0.0;
#pragma unroll
    for (int j = 0; j < RPL; ++j) {
      const int i = lane + 32 * j;
      kv[j] = i < m ? col[i] : 0.0;
      s = fma(kv[j], kUReg ? u[kUReg ? j : 0] : (i < m ? su[i] : 0.0), s);
    }
  };
  auto finish = [&](int c, const double (&kv)[RPL], double s) {
    const double bj = bb[c];
    s = warp_sum(s);  // the same bits in every lane
    const double v = bj / s;
#pragma unroll
    for (int j = 0; j < RPL; ++j) r[j] = fma(kv[j], v, r[j]);
    if (lane == 0) {
      gg[c] = v;
      const double d = (v * s) / bj - 1.0;  // first-order form of log(v s) - log b
      e += d * d;
      if (!(v >= kScaleMin && v <= kScaleMax) || !(s >= 1e-300 && s <= 1e300)) bd = 1.0;
    }
  };
  int c = w;
  if (RPL <= 8)
    for (; c + NW < nc; c += 2 * NW) {  // two columns in flight
      double k1[RPL], k2[RPL], s1, s2;
      column(c, k1, s1);
      column(c + NW, k2, s2);
      finish(c, k1, s1);
      finish(c + NW, k2, s2);
    }
#pragma unroll 1
  for (; c < nc; c += NW) {
    double k1[RPL], s1;
    column(c, k1, s1);
    finish(c, k1, s1);
  }
  // fixed tree over the warps: w + h is added into w for h = 8, 4, 2, 1
#pragma unroll 1
  for (int h = NW / 2; h >= 1; h >>= 1) {
    if (w >= h && w < 2 * h)
#pragma unroll
      for (int j = 0; j < RPL; ++j) tree[((w - h) * RPL + j) * 32 + lane] = r[j];
    __syncthreads();
    if (w < h)
#pragma unroll
      for (int j = 0; j < RPL; ++j) r[j] += tree[(w * RPL + j) * 32 + lane];
    __syncthreads();
  }
  if (w == 0)
#pragma unroll
    for (int j = 0; j < RPL; ++j) {
      const int i = lane + 32 * j;
      if (i < m) rp_out[i] = r[j];
    }
  double tt[2] = {e, bd};
  block_sum_cols<2, NW>(tt, red, par);
  errc = tt[0];
  bad = tt[1];
}

// Column sums of a group of CW (a power of two, <= 16) columns over the
// block, returned to lane c < CW of every warp as the total of column c.
// Inside a warp a transposed reduction: at each of log2 CW levels a lane
// trades half of the columns it holds with its partner (lane ^ o) and keeps
// the sum of the other half, then a butterfly over the remaining lane bits --
// CW - 1 + 5 - log2 CW shuffles instead of 5 CW.  One partial per warp and
// column goes to shared memory; the owning lanes add the NW partials in warp
// order.  A fixed pattern: the same bits on every run.
template <int CW>
__device__ __forceinline__ double block_col_sums(const double (&v)[CW], double* red, int& par) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  constexpr int LG = CW >= 16 ? 4 : CW >= 8 ? 3 : CW >= 4 ? 2 : CW >= 2 ? 1 : 0;
  double x[CW];
#pragma unroll
  for (int c = 0; c < CW; ++c) x[c] = v[c];
  int col = 0;
#pragma unroll
  for (int st = 0; st < LG; ++st) {
    const int o = 16 >> st;
    const int half = CW >> (st + 1);
    const bool upper = (lane & o) != 0;
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const double send = upper ? x[j] : x[j + half];
      const double recv = __shfl_xor_sync(0xffffffffu, send, o);
      x[j] = (upper ? x[j + half] : x[j]) + recv;
    }
    if (upper) col += half;
  }
  double sum = x[0];
#pragma unroll
  for (int o = 16 >> LG; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((lane & ((32 >> LG) - 1)) == 0) red[(par * NW + w) * CW + col] = sum;
  __syncthreads();
  double tot = 0.0;
  if (lane < CW)
#pragma unroll
    for (int q = 0; q < NW; ++q) tot += red[(par * NW + q) * CW + lane];
  par ^= 1;
  return tot;
}

// One group of CW columns, thread per row (RPT rows per thread): column sums
// with u, v = b / s (warp 0, lane c owns column jb + c), r += K v.  `buf`
// points at column jb's row 0 (+ tid), leading dimension ldk.
template <int RPT, int CW, bool REREAD>
__device__ __forceinline__ void block_group(const Prob& p, const double* buf, int jb, int nc, const double (&u)[RPT],
                                            double (&r)[RPT], const bool (&valid)[RPT], double* red, int& par,
                                            double& e, double& bd, const Ring* ring, unsigned seq) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const long long ldk = p.ldk;
  double* const gg = p.g;
  const double bl = lane < nc ? p.b[jb + lane] : 1.0;  // issued before the reduction's barrier
  double kv[REREAD ? 1 : RPT][CW], sum[CW];
#pragma unroll
  for (int c = 0; c < CW; ++c) {
    sum[c] = 0.0;
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
      const double x = (c < nc && valid[t]) ? buf[(size_t)c * ldk + t * NTT] : 0.0;
      if (!REREAD) kv[t][c] = x;
      sum[c] = fma(x, u[t], sum[c]);
    }
  }
  double s_l = block_col_sums<CW>(sum, red, par);  // (its barrier: every thread has read the stage)
  if (lane >= CW) s_l = 1.0;
  const bool owner = lane < nc;
  const double v_l = owner ? bl / s_l : 0.0;
  if (w == 0 && owner) {
    gg[jb + lane] = v_l;
    const double d = (v_l * s_l) / bl - 1.0;  // first-order form of log(v s) - log b
    e += d * d;
    if (!(v_l >= kScaleMin && v_l <= kScaleMax) || !(s_l >= 1e-300 && s_l <= 1e300)) bd = 1.0;
  }
  double v[CW];
#pragma unroll
  for (int c = 0; c < CW; ++c) v[c] = __shfl_sync(0xffffffffu, v_l, c);
  // streamed, registers hold the stage: every thread has read it (block_col_sums)
  if (!REREAD && ring && tid == 0) ring->issue(seq + STAGES);
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    double acc = r[t];
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      const double x = REREAD ? ((c < nc && valid[t]) ? buf[(size_t)c * ldk + t * NTT] : 0.0) : kv[REREAD ? 0 : t][c];
      acc = fma(x, v[c], acc);
    }
    r[t] = acc;
  }
  if (REREAD && ring) {
    __syncthreads();  // every thread is done with the stage
    if (tid == 0) ring->issue(seq + STAGES);
  }
}

// Final pass over the strip with u in shared memory (area): g = eps log v,
// P, loss and column-marginal partials -> colp[buf][k], row sums -> rowp[buf][k].
template <int RPT, int CW>
__device__ void final_pass(const Prob& p, int k, int buf, int c0, int c1, const double* us, double* red, int& par) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int m = p.m;
  const double eps = p.eps;
  double f[RPT], rs[RPT];
  bool valid[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    valid[t] = tid + t * NTT < m;
    f[t] = valid[t] ? eps * log(us[tid + t * NTT]) : 0.0;
    rs[t] = 0.0;
  }
  double s1 = 0.0, s2 = 0.0, l1c = 0.0, l2c = 0.0;
  const double* const C = p.C;
  double* const Pp = p.P;
  double* const gg = p.g;
  const double* const bb = p.b;
  for (int jb = c0; jb < c1; jb += CW) {
    const int nc = min(CW, c1 - jb);
    double gj[CW], cs[CW];
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      gj[c] = c < nc ? eps * log(gg[jb + c]) : 0.0;
      cs[c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      if (c >= nc) continue;
      const double* cj = C + (size_t)(jb + c) * m;
#pragma unroll
      for (int t = 0; t < RPT; ++t)
        if (valid[t]) {
          const double cij = cj[tid + t * NTT];
          const double pij = exp(-((cij - f[t]) - gj[c]) / eps);
          if (Pp) Pp[(size_t)(jb + c) * m + tid + t * NTT] = pij;
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
      gg[jb + lane] = gl;
      const double d = cl - bb[jb + lane];
      l1c += fabs(d);
      l2c += d * d;
    }
  }
#pragma unroll
  for (int t = 0; t < RPT; ++t)
    if (valid[t]) p.rowp[((size_t)buf * p.gp + k) * m + tid + t * NTT] = rs[t];
  double tt[4] = {s1, s2, l1c, l2c};
  block_sum_cols<4, NW>(tt, red, par);
  if (tid == 0)
    for (int i = 0; i < 4; ++i) p.colp[((size_t)buf * p.gp + k) * 4 + i] = tt[i];
}

// Row totals of merge unit u (rows u*64 .. u*64+63) over the team's partials
// `rp` ([gp][m]): warp w sums rows 4w .. 4w+3, lane l taking members l, l+32,
// ... in order, then a fixed butterfly.  Lane r < 4 receives row u*64+4w+r.
__device__ __forceinline__ double merge_unit(const double* rp, int gp, int m, int u) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i0 = u * kUnit + 4 * w;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  double v[kMaxTeam / 32][4];  // every load in flight at once
#pragma unroll
  for (int j = 0; j < kMaxTeam / 32; ++j) {
    const int k = lane + 32 * j;
#pragma unroll
    for (int r = 0; r < 4; ++r) v[j][r] = (k < gp && i0 + r < m) ? __ldcg(rp + (size_t)k * m + i0 + r) : 0.0;
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

// Row total of row i over the team's partials rp ([gp][m]), members in order.
// Loads go out in batches of 8 (one memory round trip per batch); the sum
// is sequential in member order.
__device__ __forceinline__ double row_total(const double* rp, int gp, int m, int i) {
  double acc = 0.0;
  for (int k = 0; k < gp; k += 8) {
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = k + j < gp ? __ldcg(rp + (size_t)(k + j) * m + i) : 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (k + j < gp) acc += x[j];
  }
  return acc;
}

// The row update of one row: u_next = a / tot, the squared row error (not in
// the init round) and the range check.
__device__ __forceinline__ double row_update(double ai, double ucur, double tot, bool init, double& e, double& bd) {
  const double un = ai / tot;
  if (!init) {
    const double d = log((ucur * tot) / ai);
    e += d * d;
  }
  if (!(un >= kScaleMin && un <= kScaleMax) || !(tot >= 1e-300 && tot <= 1e300)) bd = 1.0;
  return un;
}

// Sums of the team's partials part[gp][4] (all four columns) in a fixed
// order, computed by warp 0 and returned to every thread.
__device__ __forceinline__ void team_sum4(const double* part, int gp, const Shared sh, double (&t)[4]) {
  if ((threadIdx.x >> 5) == 0) {
    const int lane = threadIdx.x & 31;
    double x[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = lane; k < gp; k += 32)
#pragma unroll
      for (int j = 0; j < 4; ++j) x[j] += __ldcg(part + (size_t)k * 4 + j);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      x[j] = warp_sum(x[j]);
      if (lane == 0) sh.dec[j] = x[j];
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 4; ++j) t[j] = sh.dec[j];
  __syncthreads();
}

// Sums of the team's partials part[gp][4] (columns j0, j1) in a fixed order,
// computed by warp 0 and returned to every thread.
__device__ __forceinline__ void team_sum2(const double* part, int gp, int j0, int j1, const Shared sh, double& t0,
                                          double& t1) {
  if ((threadIdx.x >> 5) == 0) {
    const int lane = threadIdx.x & 31;
    double x0 = 0.0, x1 = 0.0;
    for (int k = lane; k < gp; k += 32) {
      x0 += __ldcg(part + (size_t)k * 4 + j0);
      x1 += __ldcg(part + (size_t)k * 4 + j1);
    }
    x0 = warp_sum(x0);
    x1 = warp_sum(x1);
    if (lane == 0) {
      sh.dec[0] = x0;
      sh.dec[1] = x1;
    }
  }
  __syncthreads();
  t0 = sh.dec[0];
  t1 = sh.dec[1];
  __syncthreads();
}

// Solves problem pi as member k of its team.  RPT / CW: thread-per-row shape
// of the row class; WARP: warp-per-column passes (resident, m <= 512); RES:
// resident strip; REREAD: 16 rows per thread, the group is read from shared
// memory twice instead of held in registers.  Rounds: 0 builds K and merges
// u_1; round t >= 1 is iteration t (column pass, merge, decision).  Round
// parity selects the partial buffers, so a member may run one round ahead of
// another that is still reading.  Returns false after a failed wait.
template <int RPT, int CW, bool WARP, bool RES, bool REREAD>
__device__ __noinline__ bool solve(const Prob& p, int pi, int k, const Shared sh, unsigned& q, unsigned* dctl,
                      volatile unsigned* done, double* pw) {
  const int tid = threadIdx.x;
  const int m = p.m, gp = p.gp;
  const int c0 = strip_begin(p.n, gp, k), c1 = strip_begin(p.n, gp, k + 1);
  const bool redundant = RPT <= 8 && (p.mode & MODE_REDUNDANT) != 0;  // the host sets it for m <= 4096 only
  const double* const pa = p.a;
  double* const su = sh.su;
  const unsigned long long t_start = globaltimer_ns();
  int par = 0;
  unsigned nb = 0;
  bool valid[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) valid[t] = tid + t * NTT < m;

  // ---- round 0: cost from points, K, row sums of K
  double cmax = 1.0;
  bool forming = true;
  unsigned long long t_form = 0;  // time waiting for the team to form
  if (p.X) {
    const double mx = cost_pass(p, c0, c1, sh.red);
    if (tid == 0) p.colp[((size_t)1 * gp + k) * 4 + 2] = mx;  // read before round 1 writes colp[1]
    const unsigned long long tf = globaltimer_ns();
    if (!team_sync(p, nb, true, dctl, sh, pw)) return false;
    t_form = globaltimer_ns() - tf;
    forming = false;
    if (tid < 32) {
      double v = 0.0;
      for (int j = tid; j < gp; j += 32) v = fmax(v, __ldcg(p.colp + ((size_t)1 * gp + j) * 4 + 2));
      v = warp_max(v);
      if (tid == 0) sh.dec[2] = v;
    }
    __syncthreads();
    cmax = sh.dec[2];
  }
  {
    const double bad0 = init_pass<RPT>(p, k, c0, c1, cmax, sh.area, sh.red, par);
    if (tid == 0) {
      p.colp[(size_t)k * 4 + 0] = 0.0;
      p.colp[(size_t)k * 4 + 1] = bad0;
    }
  }
  {
    const unsigned long long tf = globaltimer_ns();
    if (!team_sync(p, nb, forming, dctl, sh, pw)) return false;
    if (forming) t_form = globaltimer_ns() - tf;
  }

  // stage ring of a streamed strip: its groups, prefetched across rounds
  Ring ring{};
  ring.buf = sh.area;
  ring.bar = sh.bar;
  ring.pol = (p.mode & MODE_KEEP_L2) ? l2_policy_evict_last() : l2_policy_evict_first();
  ring.K = p.K;
  ring.ldk = p.ldk;
  ring.c0 = c0;
  ring.c1 = c1;
  ring.cw = CW;
  ring.ngroups = (c1 - c0 + CW - 1) / CW;
  ring.q0 = q;
  unsigned issued = q;  // the same in every thread; thread 0 issues
  auto drain = [&]() {
    if (!RES)
      for (; q < issued; ++q) ring.wait(q);
    __syncthreads();
  };

  // u of the current round: registers (thread per row), su (warp mode) or
  // ug[round parity] (split merges); un: the merged u of the next round
  double u[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) u[t] = 0.0;
  int rd = 0, iter = 0;
  double err = 1000.0;
  bool unsafe = false;
  // phase timers of member 0 (column passes, merges + decisions, team
  // barriers), kept by thread 0 in shared memory: tim[3] holds the last stamp
  const bool timing = k == 0 && tid == 0;
  if (timing) {
    sh.tim[0] = sh.tim[1] = sh.tim[2] = 0.0;
    sh.tim[3] = (double)globaltimer_ns();
  }
  auto lap = [&](int i) {
    if (timing) {
      const double t = (double)globaltimer_ns();
      sh.tim[i] += t - sh.tim[3];
      sh.tim[3] = t;
    }
  };
  while (true) {
    const int buf = rd & 1;
    const double* rp = p.rowp + (size_t)buf * gp * m;
    const bool init = rd == 0;
    // ---- merge of round rd: un = a / (row totals), row error with u
    double er = 0.0, rbad = 0.0, ec = 0.0, cbad = 0.0;
    double un[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) un[t] = 0.0;
    if (redundant) {
      // the column partials of the team ride along in the merge's reduction
      // (thread t adds member t's), so the decision needs no further round trip
      const double* cp = p.colp + (size_t)buf * gp * 4;
      const double ce = tid < gp ? __ldcg(cp + (size_t)tid * 4 + 0) : 0.0;
      const double cb = tid < gp ? __ldcg(cp + (size_t)tid * 4 + 1) : 0.0;
      double e = 0.0, bd = 0.0;
      if (WARP) {
        if (tid < m) un[0] = row_update(pa[tid], su[tid], row_total(rp, gp, m, tid), init, e, bd);
      } else {
#pragma unroll
        for (int t = 0; t < RPT; ++t)
          if (valid[t]) {
            const int i = tid + t * NTT;
            un[t] = row_update(pa[i], u[t], row_total(rp, gp, m, i), init, e, bd);
          }
      }
      double tt[4] = {e, bd, ce, cb};
      block_sum_cols<4, NW>(tt, sh.red, par);
      er = tt[0];
      rbad = tt[1];
      ec = tt[2];
      cbad = tt[3];
    } else {
      const double* ucur = p.ug + (size_t)buf * m;
      double* unext = p.ug + (size_t)(buf ^ 1) * m;
      double e = 0.0, bd = 0.0;
      for (int un_ = k; un_ < p.nunits; un_ += gp) {
        const double tot = merge_unit(rp, gp, m, un_);
        const int i = un_ * kUnit + 4 * (tid >> 5) + (tid & 31);
        if ((tid & 31) < 4 && i < m) unext[i] = row_update(pa[i], init ? 1.0 : __ldcg(ucur + i), tot, init, e, bd);
      }
      double tt[2] = {e, bd};
      block_sum_cols<2, NW>(tt, sh.red, par);
      if (tid == 0) {  // with this member's column partials
        double* mp = p.mrgp + ((size_t)buf * gp + k) * 4;
        mp[0] = tt[0];
        mp[1] = tt[1];
        mp[2] = p.colp[((size_t)buf * gp + k) * 4 + 0];
        mp[3] = p.colp[((size_t)buf * gp + k) * 4 + 1];
      }
      lap(1);
      if (!team_sync(p, nb, false, dctl, sh, pw)) {
        drain();
        return false;
      }
      lap(2);
      double t4[4];
      team_sum4(p.mrgp + (size_t)buf * gp * 4, gp, sh, t4);
      er = t4[0];
      rbad = t4[1];
      ec = t4[2];
      cbad = t4[3];
    }
    // ---- decision of round rd (the same inputs and order in every member)
    if (k == 0 && tid == 0) atomicAdd(dctl + DC_PROGRESS, 1u);
    lap(1);
    if (rbad != 0.0 || cbad != 0.0) {
      unsafe = true;
      break;
    }
    if (!init) {
      iter = rd;
      err = sqrt(er) + sqrt(ec);
      if (!(iter < p.max_iter && err >= p.tol)) break;  // u, v of round rd are the final ones
    }
    // ---- the merged u becomes current
    ++rd;
    const int nbuf = rd & 1;
    if (redundant) {
      if (WARP) {
        if (tid < m) su[tid] = un[0];
        __syncthreads();
      } else {
#pragma unroll
        for (int t = 0; t < RPT; ++t) u[t] = un[t];
      }
    } else {
      const double* ucur = p.ug + (size_t)nbuf * m;
      if (WARP) {
        for (int i = tid; i < m; i += NTT) su[i] = __ldcg(ucur + i);
        __syncthreads();
      } else {
#pragma unroll
        for (int t = 0; t < RPT; ++t) u[t] = valid[t] ? __ldcg(ucur + tid + t * NTT) : 0.0;
      }
    }
    // ---- column pass of round rd: v = b / (K^T u), row partials of K v
    double ecol = 0.0, bcol = 0.0;
    if constexpr (WARP) {
      if (m <= 64) warp_pass<2>(p, k, nbuf, c0, c1, sh.area, sh, par, ecol, bcol);
      else if (m <= 128) warp_pass<4>(p, k, nbuf, c0, c1, sh.area, sh, par, ecol, bcol);
      else if (m <= 256) warp_pass<8>(p, k, nbuf, c0, c1, sh.area, sh, par, ecol, bcol);
      else warp_pass<16>(p, k, nbuf, c0, c1, sh.area, sh, par, ecol, bcol);
    } else {
      double r[RPT];
#pragma unroll
      for (int t = 0; t < RPT; ++t) r[t] = 0.0;
      double e = 0.0, bd = 0.0;
      if constexpr (RES) {
        for (int jb = c0; jb < c1; jb += CW)
          block_group<RPT, CW, REREAD>(p, sh.area + (size_t)(jb - c0) * p.ldk + tid, jb, min(CW, c1 - jb), u, r,
                                       valid, sh.red, par, e, bd, nullptr, 0u);
      } else {
        if (tid == 0)
          for (unsigned s2 = issued; s2 < q + STAGES; ++s2) ring.issue(s2);
        issued = max(issued, q + STAGES);
        for (int gi = 0; gi < ring.ngroups; ++gi) {
          const unsigned seq = q;
          if (!ring.wait(seq)) {
            atomicOr(dctl + DC_ERR, KERR_MBAR_TIMEOUT);
            drain();
            return false;
          }
          const int jb = ring.group_begin(seq);
          block_group<RPT, CW, REREAD>(p, ring.slot(seq) + tid, jb, min(CW, c1 - jb), u, r, valid, sh.red, par, e,
                                       bd, &ring, seq);
          q = seq + 1;
          issued = seq + STAGES + 1;  // block_group issued stage seq + STAGES
        }
      }
#pragma unroll
      for (int t = 0; t < RPT; ++t)
        if (valid[t]) p.rowp[((size_t)nbuf * gp + k) * m + tid + t * NTT] = r[t];
      double tt[2] = {e, bd};
      block_sum_cols<2, NW>(tt, sh.red, par);
      ecol = tt[0];
      bcol = tt[1];
    }
    if (tid == 0) {
      p.colp[((size_t)nbuf * gp + k) * 4 + 0] = ecol;
      p.colp[((size_t)nbuf * gp + k) * 4 + 1] = bcol;
    }
    lap(0);
    if (!team_sync(p, nb, false, dctl, sh, pw)) {
      drain();
      return false;
    }
    lap(2);
  }
  drain();

  if (unsafe) {
    if (k == 0 && tid == 0) {
      p.res[3] = kUnsafeStatus;
      __threadfence_system();
      done[pi] = 1u;
    }
    return true;
  }

  // ---- final round: u of the last column pass into the area (K is no longer
  // read), then P, g, loss and marginal partials
  double* us = sh.area;
  if (rd == 0) {
    // no iteration ran (cannot happen with max_iter >= 1): u = u_1
    for (int i = tid; i < m; i += NTT) us[i] = 0.0;
  } else if (redundant || !WARP) {
    if (WARP) {
      for (int i = tid; i < m; i += NTT) us[i] = su[i];
    } else if (redundant) {
#pragma unroll
      for (int t = 0; t < RPT; ++t)
        if (valid[t]) us[tid + t * NTT] = u[t];
    } else {
      const double* ucur = p.ug + (size_t)(rd & 1) * m;
      for (int i = tid; i < m; i += NTT) us[i] = __ldcg(ucur + i);
    }
  } else {
    for (int i = tid; i < m; i += NTT) us[i] = su[i];
  }
  __syncthreads();
  const int fbuf = (rd + 1) & 1;
  final_pass<RPT, 16 / RPT>(p, k, fbuf, c0, c1, us, sh.red, par);
  if (!team_sync(p, nb, false, dctl, sh, pw)) return false;
  if (k == 0) {
    const double* rp = p.rowp + (size_t)fbuf * gp * m;
    double l1 = 0.0, l2 = 0.0;
    for (int i = tid; i < m; i += NTT) {
      const double d = row_total(rp, gp, m, i) - p.a[i];
      l1 += fabs(d);
      l2 += d * d;
      p.f[i] = p.eps * log(us[i]);
    }
    double tt[2] = {l1, l2};
    block_sum_cols<2, NW>(tt, sh.red, par);
    double s1, s2, lc1, lc2;
    team_sum2(p.colp + (size_t)fbuf * gp * 4, gp, 0, 1, sh, s1, s2);
    team_sum2(p.colp + (size_t)fbuf * gp * 4, gp, 2, 3, sh, lc1, lc2);
    if (tid == 0) {
      p.res[0] = s1 + p.eps * s2;  // accu(C % P) + reg * accu(P % (log(P) - 1))
      p.res[1] = err;
      p.res[2] = iter;
      p.res[3] = (err <= p.tol) ? 0.0 : (iter == p.max_iter ? 1.0 : 2.0);
      p.res[4] = tt[0];
      p.res[5] = lc1;
      p.res[6] = sqrt(tt[1]);
      p.res[7] = sqrt(lc2);
      p.res[8] = (double)(globaltimer_ns() - t_start);
      p.res[9] = (double)t_form;
      p.res[10] = sh.tim[0];
      p.res[11] = sh.tim[1];
      p.res[12] = sh.tim[2];
      __threadfence_system();
      done[pi] = 1u;
    }
  }
  return true;
}

constexpr int kBackfillWindow = 64;
constexpr int kScanWindow = 256;  // problems from the scan start examined per pass

__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__host__ __device__ __forceinline__ unsigned slot_of(unsigned h) { return h & (unsigned)(kMaxProbs - 1); }

// Control words of problem number h: [0] the claim word, [1] the state word.
__device__ __forceinline__ unsigned long long* problem_ctl(const Prob* probs, unsigned h) {
  return reinterpret_cast<unsigned long long*>(
      __ldcg(reinterpret_cast<const unsigned long long*>(&probs[slot_of(h)].ctl)));
}
__host__ __device__ __forceinline__ unsigned long long claim_word(unsigned h, int gp, int claimed) {
  return ((unsigned long long)h << 32) | ((unsigned long long)(unsigned)gp << 16) | (unsigned)claimed;
}
__host__ __device__ __forceinline__ unsigned long long state_word(unsigned h, unsigned st) {
  return ((unsigned long long)h << 32) | st;
}

// Claim of a member slot (thread 0).  Team formation with reservation:
// F = (CTAs looking for work) - (unfilled slots of opened problems) never goes
// below zero.  A CTA that starts looking adds one to F; it first takes an
// unfilled slot of an opened problem; else it opens one -- the oldest
// unopened problem, or (backfilling, while that one has waited less than
// backfill_us) a later one in a window of kBackfillWindow -- by taking the
// problem's gp from F with a compare-and-swap.  So every opened team has
// enough free CTAs to fill it and no team waits on CTAs that are busy
// elsewhere.  Problems are numbered in publication order and problem h lives
// in descriptor slot h % kMaxProbs, which a server reuses once h has been
// collected: the claim and state words carry the problem number and change
// only by compare-and-swap, so a scan that meets a reused slot (its number is
// no longer h) counts h as finished and never touches the new problem.
// Returns the slot and member index, or pi = -1 when the launch is closing
// (or on an error).  The published count is taken from pub[0] until the
// launch closes (stop flag, or idle_ns with nothing to do and no work in
// flight).
__device__ void claim(const Prob* probs, const volatile unsigned* pub, unsigned* dctl, unsigned long long idle_ns,
                      unsigned backfill_us, int& pi, int& k) {
  pi = -1;
  k = -1;
  int* F = reinterpret_cast<int*>(dctl + DC_FREE);
  atomicAdd(F, 1);
  const unsigned long long t_idle = globaltimer_ns();
  unsigned nap = 256;  // sleep between empty passes, doubled up to 8 us
  while (true) {
    if (ld_relaxed(dctl + DC_ERR) != 0u) return;
    const unsigned W = ld_relaxed(dctl + DC_AVAIL);
    const unsigned npx = W & ~kClosed;
    if (!(W & kClosed)) {
      // the published count lives in host memory for a server: one CTA of
      // the grid reads it at most every 20 us, the others see DC_AVAIL
      const unsigned now_us = (unsigned)(globaltimer_ns() / 1000ull);
      const unsigned last = ld_relaxed(dctl + DC_PUB_T);
      if (now_us - last >= 20u && atomicCAS(dctl + DC_PUB_T, last, now_us) == last) {
        const unsigned p0 = pub[0] & ~kClosed;
        if (p0 > npx) {
          atomicCAS(dctl + DC_AVAIL, W, p0);
          continue;
        }
      }
    }
    // 1. an unfilled slot of an opened problem; the state and claim words are
    // read 8 problems at a time (the loads overlap)
    const unsigned head = ld_relaxed(dctl + DC_HEAD);
    const unsigned end = min(npx, head + kScanWindow);
    unsigned oldest = npx;  // oldest problem not yet opened
    bool open_slots = false, prefix_full = true;
    for (unsigned h0 = head; h0 < end; h0 += 8) {
      unsigned long long sw[8], cw[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const unsigned h = h0 + u;
        unsigned long long* ctl = h < end ? problem_ctl(probs, h) : nullptr;
        sw[u] = ctl ? ld_relaxed64(ctl + 1) : 0ull;
        cw[u] = ctl ? ld_relaxed64(ctl) : 0ull;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const unsigned h = h0 + u;
        if (h >= end) break;
        // a slot that no longer carries h was reused: h is finished
        const bool mine = (unsigned)(sw[u] >> 32) == h && (unsigned)(cw[u] >> 32) == h;
        const unsigned st = mine ? (unsigned)sw[u] : 1u;
        const int gp = (int)((cw[u] >> 16) & 0xffffu), cl = (int)(cw[u] & 0xffffu);
        const bool unfilled = mine && st == 1u && cl < gp;
        if (st == 1u) {
          if (unfilled) {
            open_slots = true;
            unsigned long long* ctl = problem_ctl(probs, h);
            unsigned long long w = cw[u];
            while ((unsigned)(w >> 32) == h && (int)(w & 0xffffu) < (int)((w >> 16) & 0xffffu)) {
              const unsigned long long prev = atomicCAS(ctl, w, w + 1ull);
              if (prev == w) {
                pi = (int)slot_of(h);
                k = (int)(w & 0xffffu);
                return;
              }
              w = prev;
            }
          } else if (prefix_full) {
            atomicMax(dctl + DC_HEAD, h + 1);  // opened and full up to here: later scans start after it
          }
        } else {
          prefix_full = false;
          if (oldest == npx) oldest = h;
        }
        if (unfilled) prefix_full = false;
      }
    }
    // 2. open a problem
    if (oldest < npx) {
      const unsigned now_us = (unsigned)(globaltimer_ns() / 1000ull);
      if (ld_relaxed(dctl + DC_OLDEST) != oldest + 1u) {
        atomicExch(dctl + DC_OLDEST_T, now_us);
        atomicExch(dctl + DC_OLDEST, oldest + 1u);
      }
      const bool backfill = now_us - ld_relaxed(dctl + DC_OLDEST_T) < backfill_us;
      bool opened = false;
      for (unsigned h = oldest; h < end && h < oldest + kBackfillWindow && !opened; ++h) {
        if (h != oldest && !backfill) break;
        unsigned long long* ctl = problem_ctl(probs, h);
        if (ld_relaxed64(ctl + 1) != state_word(h, 0u)) continue;
        const unsigned long long cw = ld_relaxed64(ctl);
        if ((unsigned)(cw >> 32) != h) continue;
        const int gp = (int)((cw >> 16) & 0xffffu);
        if (gp > (int)ld_relaxed(reinterpret_cast<unsigned*>(F))) continue;
        if (atomicCAS(ctl + 1, state_word(h, 0u), state_word(h, 2u)) != state_word(h, 0u)) continue;  // another CTA is opening it
        while (true) {
          const int f = (int)ld_relaxed(reinterpret_cast<unsigned*>(F));
          if (f < gp) break;
          if (atomicCAS(F, f, f - gp) == f) {
            opened = true;
            break;
          }
        }
        atomicExch(ctl + 1, state_word(h, opened ? 1u : 0u));
      }
      if (opened) continue;
    }
    // 3. nothing to take now
    if (W & kClosed) {
      if (oldest == npx && !open_slots && end == npx) return;  // everything published is opened and full
    } else {
      const bool idle = oldest == npx && !open_slots && globaltimer_ns() - t_idle > idle_ns &&
                        ld_relaxed(dctl + DC_ACTIVE) == 0u;
      if (pub[1] != 0u || idle) {
        atomicCAS(dctl + DC_AVAIL, W, W | kClosed);
        continue;
      }
    }
    __nanosleep(nap);
    nap = min(nap * 2, 8192u);
  }
}

int __host__ __device__ row_class(int m) { return m <= 512 ? 0 : m <= 1024 ? 1 : m <= 2048 ? 2 : m <= 4096 ? 3 : 4; }

// Service loop: CTAs claim member slots of the published problems
// probs[0, pub[0]) (pub[1]: stop flag; host-mapped memory for a server,
// device memory for a batch call) until the launch closes.  done[q] is set
// (system scope) once problem q's results are in probs[q].res.  dctl: see
// DC_*.  prof (may be null): per CTA [4 c + 0] busy ns, [1] team-wait ns,
// [2] claim ns, [3] member slots solved.
__global__ void __launch_bounds__(NTT, 1) service_kernel(const Prob* probs, const volatile unsigned* pub,
                                                          volatile unsigned* done, unsigned* dctl, double* prof,
                                                          unsigned long long idle_ns, unsigned backfill_us) {
  extern __shared__ __align__(128) unsigned char smem[];
  Shared sh;
  sh.area = reinterpret_cast<double*>(smem);
  sh.bar = reinterpret_cast<uint64_t*>(smem + (size_t)kArea * 8);
  sh.su = reinterpret_cast<double*>(smem + (size_t)kArea * 8 + 64);
  sh.red = sh.su + kWarpRows;
  sh.dec = sh.red + 2 * NW * 16;
  sh.tim = sh.dec + 8;
  sh.flag = reinterpret_cast<int*>(sh.tim + 4);
  Prob* sp = reinterpret_cast<Prob*>(sh.flag + 4);
  const int tid = threadIdx.x, cta = blockIdx.x;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(sh.bar + s, 1);
    fence_mbar_init();
  }
  __syncthreads();
  unsigned q = 0;
  double t_busy = 0.0, t_wait = 0.0, t_claim = 0.0, slots = 0.0;
  double* pw = prof ? &t_wait : nullptr;
  while (true) {
    const unsigned long long t0 = globaltimer_ns();
    if (tid == 0) {
      int pi, k;
      claim(probs, pub, dctl, idle_ns, backfill_us, pi, k);
      sh.flag[1] = pi;
      sh.flag[2] = k;
      if (pi >= 0) {
        atomicAdd(dctl + DC_ACTIVE, 1u);
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(probs + pi);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(sp);
        for (int w = 0; w < (int)(sizeof(Prob) / 8); ++w) dst[w] = __ldcg(src + w);
      }
    }
    __syncthreads();
    const int pi = sh.flag[1], k = sh.flag[2];
    const unsigned long long t1 = globaltimer_ns();
    t_claim += (double)(t1 - t0);
    if (pi < 0) break;
    const Prob& p = *sp;
    bool ok;
    if (p.mode & MODE_RESIDENT) {
      if (p.mode & MODE_WARP) {
        ok = solve<1, 16, true, true, false>(p, pi, k, sh, q, dctl, done, pw);
      } else {
        switch (row_class(p.m)) {
          case 0: ok = solve<1, 16, false, true, false>(p, pi, k, sh, q, dctl, done, pw); break;
          case 1: ok = solve<2, 8, false, true, false>(p, pi, k, sh, q, dctl, done, pw); break;
          case 2: ok = solve<4, 4, false, true, false>(p, pi, k, sh, q, dctl, done, pw); break;
          case 3: ok = solve<8, 2, false, true, false>(p, pi, k, sh, q, dctl, done, pw); break;
          default: ok = solve<16, 1, false, true, true>(p, pi, k, sh, q, dctl, done, pw); break;
        }
      }
    } else {
      switch (row_class(p.m)) {
        case 0: ok = solve<1, 16, false, false, false>(p, pi, k, sh, q, dctl, done, pw); break;
        case 1: ok = solve<2, 8, false, false, false>(p, pi, k, sh, q, dctl, done, pw); break;
        case 2: ok = solve<4, 4, false, false, false>(p, pi, k, sh, q, dctl, done, pw); break;
        case 3: ok = solve<8, 2, false, false, false>(p, pi, k, sh, q, dctl, done, pw); break;
        default: ok = solve<16, 1, false, false, true>(p, pi, k, sh, q, dctl, done, pw); break;
      }
    }
    __syncthreads();  // sp and flags are rewritten by the next claim
    if (tid == 0) atomicSub(dctl + DC_ACTIVE, 1u);
    t_busy += (double)(globaltimer_ns() - t1);
    slots += 1.0;
    if (!ok) break;
  }
  if (prof && tid == 0) {
    prof[4 * cta + 0] = t_busy - t_wait;
    prof[4 * cta + 1] = t_wait;
    prof[4 * cta + 2] = t_claim;
    prof[4 * cta + 3] = slots;
  }
}

}  // namespace batch

// Per-launch bound on the elements of the streamed problems' K and the
// points-built costs (device memory of one launch).
constexpr long long kLaunchMaxElems = 1LL << 31;

enum { SBT_DESC = 200, SBT_K, SBT_WORK, SBT_CTRL, SBT_PROF, SBT_RES, SBT_PCTL, SBT_HOSTIO = 210 };

// Placement of problem q: team size, strip mode, merge mode (functions of the
// problem, the SM count and the engine options batch.strip_kb,
// batch.max_team, batch.redundant_rows and batch.l2_keep_mb) and the sizes of
// its K and work arrays.
void place(const rwig_problem& q, int G, batch::Prob& d, long long& kdoubles, long long& wdoubles, bool server) {
  using namespace batch;
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  d = Prob{};
  d.m = q.M;
  d.n = q.N;
  d.ldk = ((q.M + 1) / 2) * 2;
  const long long strip_target = (long long)(option("batch.strip_kb", 184.0) * 1024.0 / 8.0);
  const long long cols = std::max<long long>(1, std::min<long long>(kResident, strip_target) / d.ldk);
  const int gp_res = (int)((q.N + cols - 1) / cols);
  // largest team: a quarter of the SMs for a batched call (throughput: more
  // problems side by side), 0.4 for a server (latency: each request done sooner)
  const int maxteam =
      std::max(1, std::min(G, (int)option("batch.max_team", std::floor((server ? 0.4 : 0.25) * G))));
  const int res_team = std::min(maxteam, (int)option("batch.resident_team", 32.0));
  int mode = 0;
  if (gp_res <= res_team || (q.M <= kWarpRows && gp_res <= maxteam)) {
    mode |= MODE_RESIDENT;
    d.gp = gp_res;
    if (q.M <= kWarpRows) mode |= MODE_WARP;
  } else {
    // streamed strips of about batch.stream_strip_kb each
    const double kbytes = (double)d.ldk * q.N * 8.0;
    const double sst = std::max(64.0, option("batch.stream_strip_kb", 1024.0)) * 1024.0;
    d.gp = (int)std::min<double>(std::min(maxteam, q.N), std::max(1.0, std::ceil(kbytes / sst)));
    if (kbytes <= option("batch.l2_keep_mb", 48.0) * 1048576.0) mode |= MODE_KEEP_L2;
  }
  const long long red_rows = (long long)option("batch.redundant_rows", 16384.0);
  if (q.M <= 4096 && (d.gp == 1 || (long long)d.gp * q.M <= red_rows)) mode |= MODE_REDUNDANT;
  d.mode = mode;
  d.nunits = (q.M + kUnit - 1) / kUnit;
  d.max_iter = q.max_iter;
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
  kdoubles = (mode & MODE_RESIDENT) ? 0 : al(d.ldk * q.N);
  wdoubles = al(2LL * d.gp * q.M) + 2 * al(8LL * d.gp) + al(2LL * q.M) + 32 +
             (q.C ? 0 : al((long long)q.M * q.N));  // the cost built from points
}

// Points the work arrays of d into w (wdoubles doubles), K into k, the
// results into res and the control words into ctl (4, zeroed by the caller).
void bind(batch::Prob& d, double* k, double* w, double* res, unsigned* ctl) {
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  d.K = k;
  d.rowp = w;
  d.colp = d.rowp + al(2LL * d.gp * d.m);
  d.mrgp = d.colp + al(8LL * d.gp);
  d.ug = d.mrgp + al(8LL * d.gp);
  d.res = res;
  d.ctl = ctl;
  if (d.X) d.C = d.ug + al(2LL * d.m) + 32;
}

int launch_service(Context* ctx, cudaStream_t st, const batch::Prob* dprob, const unsigned* pub, unsigned* done,
                   unsigned* dctl, double* dprof, unsigned long long idle_ns, unsigned avail0, unsigned head0) {
  using namespace batch;
  static bool attr = false;
  if (!attr) {
    RWIG_CUDA_TRY(
        cudaFuncSetAttribute(service_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes()));
    attr = true;
  }
  int nblk = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nblk, service_kernel, NTT, smem_bytes()));
  if (nblk < 1) return set_error(RWIG_E_UNSUPPORTED, "batched Sinkhorn kernel does not fit on an SM");
  unsigned h0[kCtlWords] = {};
  h0[DC_AVAIL] = avail0;
  h0[DC_HEAD] = head0;
  RWIG_CUDA_TRY(cudaMemcpyAsync(dctl, h0, sizeof(h0), cudaMemcpyHostToDevice, st));
  const Prob* dp = dprob;
  const volatile unsigned* pb = pub;
  volatile unsigned* dn = done;
  unsigned* ctl = dctl;
  double* pr = dprof;
  unsigned long long idle = idle_ns;
  unsigned bf = (unsigned)std::max(0.0, option("batch.backfill_us", 5000.0));
  void* args[] = {(void*)&dp, (void*)&pb, (void*)&dn, (void*)&ctl, (void*)&pr, (void*)&idle, (void*)&bf};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((void*)service_kernel, dim3(ctx->sm_count), dim3(NTT), args,
                                            smem_bytes(), st));
  return 0;
}

// Prints the optional per-CTA profile of the last launch (rwig_set_option
// "batch.profile"): busy, team-wait and claim time, member slots.
int print_profile(Context* ctx, const double* dprof, int np, float kernel_ms) {
  const int G = ctx->sm_count;
  std::vector<double> h(4 * (size_t)G);
  RWIG_CUDA_TRY(cudaMemcpy(h.data(), dprof, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
  double s[4] = {0, 0, 0, 0}, mx[4] = {0, 0, 0, 0};
  for (int c = 0; c < G; ++c)
    for (int j = 0; j < 4; ++j) {
      s[j] += h[4 * c + j];
      mx[j] = std::max(mx[j], h[4 * c + j]);
    }
  std::fprintf(stderr,
               "service_kernel profile: %d problems, kernel %.3f ms | per CTA mean (max) ms: busy %.3f (%.3f), "
               "team waits %.3f (%.3f), claim/idle %.3f (%.3f) | member slots %.0f\n",
               np, kernel_ms, s[0] / G * 1e-6, mx[0] * 1e-6, s[1] / G * 1e-6, mx[1] * 1e-6, s[2] / G * 1e-6,
               mx[2] * 1e-6, s[3]);
  return 0;
}

// One launch over problems `idx` (all eligible for the kernel), published up
// front in descending size (the claim order) with the launch closed.
static int launch_group(Context* ctx, cudaStream_t st, const rwig_problem* probs, const std::vector<int>& idx,
                        rwig_result* out, std::vector<int>& percall, int* launches) {
  using namespace batch;
  const int np = (int)idx.size();
  const int G = ctx->sm_count;
  if (G > kMaxTeam) return set_error(RWIG_E_UNSUPPORTED, "more SMs than the batched kernel's team limit");
  std::vector<int> ord(np);  // descriptor slot -> position in idx
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
    return (long long)probs[idx[x]].M * probs[idx[x]].N > (long long)probs[idx[y]].M * probs[idx[y]].N;
  });
  std::vector<Prob> hp(np);
  std::vector<long long> koff(np), woff(np);
  long long kd = 0, wd = 0;
  for (int s = 0; s < np; ++s) {
    long long k1, w1;
    place(probs[idx[ord[s]]], G, hp[s], k1, w1, false);
    koff[s] = kd;
    woff[s] = wd;
    kd += k1;
    wd += w1;
  }
  Prob* dprob = (Prob*)scratch(ctx, SBT_DESC, sizeof(Prob) * np);
  double* dK = (double*)scratch(ctx, SBT_K, sizeof(double) * std::max<long long>(kd, 32));
  double* dW = (double*)scratch(ctx, SBT_WORK, sizeof(double) * std::max<long long>(wd, 32));
  double* dres = (double*)scratch(ctx, SBT_RES, sizeof(double) * kResStride * np);
  unsigned* ctrl = (unsigned*)scratch(ctx, SBT_CTRL, sizeof(unsigned) * (kCtlWords + 2 + kMaxProbs));
  unsigned* pctl = (unsigned*)scratch(ctx, SBT_PCTL, sizeof(unsigned) * kCtlPerSlot * kMaxProbs);
  const bool profile = option("batch.profile", 0.0) != 0.0;
  double* dprof = profile ? (double*)scratch(ctx, SBT_PROF, sizeof(double) * 4 * G) : nullptr;
  if (!dprob || !dK || !dW || !dres || !ctrl || !pctl || (profile && !dprof)) return RWIG_E_NOMEM;
  // problem s in slot s: claim word (s, gp, 0), state word (s, unopened), team barrier 0
  std::vector<unsigned long long> hwords((size_t)np * kCtlPerSlot / 2, 0ull);
  for (int s = 0; s < np; ++s) {
    bind(hp[s], dK + koff[s], dW + woff[s], dres + kResStride * (size_t)s, pctl + kCtlPerSlot * s);
    hwords[(size_t)s * kCtlPerSlot / 2 + 0] = claim_word((unsigned)s, hp[s].gp, 0);
    hwords[(size_t)s * kCtlPerSlot / 2 + 1] = state_word((unsigned)s, 0u);
  }
  unsigned* pub = ctrl + kCtlWords;
  unsigned* done = ctrl + kCtlWords + 2;
  const unsigned hpub[2] = {(unsigned)np, 1u};
  RWIG_CUDA_TRY(cudaMemcpyAsync(dprob, hp.data(), sizeof(Prob) * np, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(pub, hpub, sizeof(hpub), cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(unsigned) * kMaxProbs, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(pctl, hwords.data(), sizeof(unsigned long long) * hwords.size(),
                                cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(dres, 0, sizeof(double) * kResStride * np, st));
  if (profile) RWIG_CUDA_TRY(cudaEventRecord(ctx->evk, st));
  const int rc = launch_service(ctx, st, dprob, pub, done, ctrl, dprof, 0ull, (unsigned)np | kClosed, 0u);
  if (rc) return rc;
  if (profile) RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  ++*launches;
  std::vector<double> hres(kResStride * (size_t)np);
  RWIG_CUDA_TRY(cudaMemcpyAsync(hres.data(), dres, sizeof(double) * kResStride * np, cudaMemcpyDeviceToHost, st));
  unsigned hctl[4] = {0, 0, 0, 0};
  RWIG_CUDA_TRY(cudaMemcpyAsync(hctl, ctrl, sizeof(hctl), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (hctl[2]) return set_error(RWIG_E_TIMEOUT, "a bounded wait in the batched Sinkhorn kernel expired");
  if (profile) {
    float kms = 0.f;
    cudaEventElapsedTime(&kms, ctx->evk, ctx->ev1);
    const int rc2 = print_profile(ctx, dprof, np, kms);
    if (rc2) return rc2;
    // per placement class: problems, member-iterations, solve and formation time, K bytes per member-us
    struct Agg { int n = 0; double mi = 0, dev = 0, form = 0, bytes = 0, mus = 0, it = 0, ph[3] = {0, 0, 0}; };
    Agg agg[4];
    for (int s2 = 0; s2 < np; ++s2) {
      const Prob& d = hp[s2];
      const double* r = hres.data() + kResStride * (size_t)s2;
      const int c = ((d.mode & MODE_RESIDENT) ? 0 : 2) + (d.m > kWarpRows ? 1 : 0);
      agg[c].n += 1;
      agg[c].mi += r[2] * d.gp;
      agg[c].dev += r[8] * 1e-6;
      agg[c].form += r[9] * 1e-6;
      agg[c].bytes += r[2] * (double)d.ldk * d.n * 8.0;
      agg[c].mus += (r[8] - r[9]) * 1e-3 * d.gp;
      agg[c].it += r[2];
      for (int j = 0; j < 3; ++j) agg[c].ph[j] += r[10 + j] * 1e-3;
    }
    const char* lab[4] = {"resident m<=512", "resident m>512", "streamed m<=512", "streamed m>512"};
    for (int c = 0; c < 4; ++c)
      if (agg[c].n)
        std::fprintf(stderr,
                     "  %-16s problems %3d | member-iterations %9.0f | solve ms (sum) %9.2f | formation ms (sum) "
                     "%8.2f | member-us per member-iteration %6.2f | GB/s per member %6.1f\n",
                     lab[c], agg[c].n, agg[c].mi, agg[c].dev, agg[c].form,
                     agg[c].mi > 0 ? agg[c].mus / agg[c].mi : 0.0, agg[c].mus > 0 ? agg[c].bytes / agg[c].mus * 1e-3 : 0.0);
    for (int c = 0; c < 4; ++c)
      if (agg[c].it > 0)
        std::fprintf(stderr, "  %-16s per iteration (member 0, us): column pass %.2f | merge + decision %.2f | team barriers %.2f\n",
                     lab[c], agg[c].ph[0] / agg[c].it, agg[c].ph[1] / agg[c].it, agg[c].ph[2] / agg[c].it);
  }
  for (int s = 0; s < np; ++s) {
    const int i = idx[ord[s]];
    rwig_result& o = out[i];
    const double* r = hres.data() + kResStride * (size_t)s;
    if (r[3] == kUnsafeStatus) {
      if (probs[i].C) percall.push_back(i);
      else o.status = RWIG_E_UNSUPPORTED;  // outside the scaling form; the per-call path takes C
      continue;
    }
    o.loss = r[0];
    o.err = r[1];
    o.iter = (int)r[2];
    o.status = (int)r[3];
    o.marg_l1_row = r[4];
    o.marg_l1_col = r[5];
    o.device_us = r[8] * 1e-3;
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
    if (q.M <= kMaxRows && q.max_iter >= 1 &&
        (pts || (double)q.M * q.N <= option("batch.max_elems", (double)(1LL << 26))))
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
  cudaStream_t st = call_stream(ctx, stream);
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
// finished ones.  Requests are numbered in submission order (the ticket) and
// request h lives in descriptor slot h % kMaxProbs, reused as soon as its
// previous occupant has been collected (the kernel's claim and state words
// carry the request number, so a reused slot is never mistaken for the old
// request).  Admission is bounded by a device-memory budget and by the
// kMaxProbs requests that may be out at once.
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
  unsigned* dpctl = nullptr;                // device, kCtlPerSlot control words per slot
  // the requests' memory: a pool of the server's own that keeps what it has
  // mapped (release threshold: unlimited), so freeing a collected request
  // never unmaps device memory -- which would wait for the running launch
  cudaMemPool_t pool = nullptr;
  unsigned hctl_err = 0;
  int nsub = 0, npub = 0;  // requests submitted (the next ticket) and published
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
  std::vector<unsigned long long> staged_ctl;  // and of the control words, kCtlPerSlot / 2 per slot
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
  // only the last kMaxProbs published requests can be unfinished; the new
  // launch's scan starts at the first of them
  bool pending = false;
  int head0 = s->npub;
  for (int h = std::max(0, s->npub - batch::kMaxProbs); h < s->npub; ++h) {
    const int slot = h % batch::kMaxProbs;
    if (s->slots[slot].ticket == h && !s->hdone[slot]) {
      pending = true;
      head0 = std::min(head0, h);
    }
  }
  if (!pending) return 0;
  const int rc =
      launch_service(s->ctx, s->ks, s->dprob, s->dpub, s->ddone, s->dctl, nullptr, s->idle_ns, 0u, (unsigned)head0);
  if (rc) return rc;
  s->launched = true;
  return 0;
}

// Publishes, in slot order, the submitted requests whose copies have landed.
int publish_ready(rwig_server* s) {
  const int before = s->npub;
  while (s->npub < s->nsub) {
    const cudaError_t e = cudaEventQuery(s->slots[s->npub % batch::kMaxProbs].ev);
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
  s->staged_ctl.assign((size_t)batch::kMaxProbs * batch::kCtlPerSlot / 2, 0ull);
  auto fail = [&](cudaError_t e, const char* what) {
    rwig_server_destroy(s);
    return cuda_fail(e, what);
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s->ks, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
  if ((e = cudaStreamCreateWithFlags(&s->cs, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
  if ((e = cudaMalloc(&s->dprob, sizeof(batch::Prob) * batch::kMaxProbs)) != cudaSuccess) return fail(e, "descriptors");
  if ((e = cudaMalloc(&s->dctl, sizeof(unsigned) * batch::kCtlWords)) != cudaSuccess) return fail(e, "control");
  {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    if ((e = cudaMemPoolCreate(&s->pool, &props)) != cudaSuccess) return fail(e, "memory pool");
    unsigned long long keep = ~0ull;
    if ((e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
      return fail(e, "memory pool");
    // map the whole budget now (at most 80 % of the free memory), while no
    // launch runs: growing the pool later waits for the running launch, which
    // stalled admission whenever the requests out at once outgrew the mapping
    void* prime = nullptr;
    size_t free_b = 0, total_b = 0;
    if ((e = cudaMemGetInfo(&free_b, &total_b)) != cudaSuccess) return fail(e, "memory info");
    const size_t pb = (size_t)std::min(mem_budget_bytes, 0.8 * (double)free_b);
    if ((e = cudaMallocFromPoolAsync(&prime, pb, s->pool, s->cs)) != cudaSuccess) return fail(e, "memory pool");
    if ((e = cudaFreeAsync(prime, s->cs)) != cudaSuccess) return fail(e, "memory pool");
    if ((e = cudaStreamSynchronize(s->cs)) != cudaSuccess) return fail(e, "memory pool");
  }
  if ((e = cudaMalloc(&s->dpctl, sizeof(unsigned) * batch::kCtlPerSlot * batch::kMaxProbs)) != cudaSuccess)
    return fail(e, "slot control");
  if ((e = cudaHostAlloc(&s->hpub, sizeof(unsigned) * 2, cudaHostAllocMapped)) != cudaSuccess) return fail(e, "pub");
  if ((e = cudaHostAlloc(&s->hdone, sizeof(unsigned) * batch::kMaxProbs, cudaHostAllocMapped)) != cudaSuccess)
    return fail(e, "done");
  if ((e = cudaHostAlloc(&s->hres, sizeof(double) * batch::kResStride * batch::kMaxProbs, cudaHostAllocMapped)) != cudaSuccess)
    return fail(e, "results");
  if ((e = cudaHostGetDevicePointer(&s->dpub, s->hpub, 0)) != cudaSuccess) return fail(e, "pub map");
  if ((e = cudaHostGetDevicePointer(&s->ddone, s->hdone, 0)) != cudaSuccess) return fail(e, "done map");
  if ((e = cudaHostGetDevicePointer(&s->dres, s->hres, 0)) != cudaSuccess) return fail(e, "results map");
  if ((e = cudaMemset(s->dctl, 0, sizeof(unsigned) * batch::kCtlWords)) != cudaSuccess) return fail(e, "control");
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
  // request numbers stay below the kernel's closed flag (bit 31): start again
  // from 0 once everything is collected and no launch runs
  if (s->nsub >= 0x7fff0000) {
    bool all = true;
    for (const auto& sl : s->slots) all = all && sl.collected;
    if (!all || kernel_running(s)) return RWIG_E_BUSY;
    s->nsub = 0;
    s->npub = 0;
    for (auto& sl : s->slots) sl.ticket = -1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    *(volatile unsigned*)s->hpub = 0u;
  }
  const int slot = s->nsub % kMaxProbs;
  if (!s->slots[slot].collected) return RWIG_E_BUSY;  // its previous request is still out
  Prob d{};
  long long kd = 0, wd = 0;
  place(*q, s->ctx->sm_count, d, kd, wd, true);
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  const long long M = q->M, N = q->N;
  const long long cd = pts ? al(M * q->d) + al(N * q->d) : al(M * N);  // C, or the points
  const long long io = al(M) + al(N) + cd + al(M) + al(N) + (q->P ? al(M * N) : 0);
  const double bytes = 8.0 * (double)(io + kd + wd);
  if (s->inflight + bytes > s->budget) return RWIG_E_BUSY;
  void* mem = nullptr;
  RWIG_CUDA_TRY(cudaMallocFromPoolAsync(&mem, (size_t)bytes, s->pool, s->cs));
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
  bind(d, dk, dw, s->dres + batch::kResStride * (size_t)slot, s->dpctl + kCtlPerSlot * (size_t)slot);
  // control words: claim (request, gp, 0), state (request, unopened), team barrier 0
  unsigned long long* hc = s->staged_ctl.data() + (size_t)slot * kCtlPerSlot / 2;
  for (int w = 0; w < kCtlPerSlot / 2; ++w) hc[w] = 0ull;
  hc[0] = claim_word((unsigned)s->nsub, d.gp, 0);
  hc[1] = state_word((unsigned)s->nsub, 0u);
  RWIG_CUDA_TRY(cudaMemcpyAsync(s->dpctl + kCtlPerSlot * (size_t)slot, hc, sizeof(unsigned) * kCtlPerSlot,
                                cudaMemcpyHostToDevice, s->cs));
  s->staged[slot] = d;  // the copy source must outlive the asynchronous copy
  RWIG_CUDA_TRY(cudaMemcpyAsync(s->dprob + slot, &s->staged[slot], sizeof(Prob), cudaMemcpyHostToDevice, s->cs));
  RWIG_CUDA_TRY(cudaEventRecord(s->slots[slot].ev, s->cs));
  auto& sl = s->slots[slot];
  sl.ticket = s->nsub;
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
  ++s->nsub;
  const int rc = publish_ready(s);
  if (rc) return rc;
  return sl.ticket;
}

extern "C" int rwig_server_poll(rwig_server* s, int ticket, rwig_result* out) {
  reset_report();
  if (!s || !out) return set_error(RWIG_E_INVALID, "null server or result");
  std::lock_guard<std::mutex> lk(s->ctx->mu);
  const int slot = ticket >= 0 ? ticket % batch::kMaxProbs : -1;
  if (slot < 0 || ticket >= s->nsub || s->slots[slot].ticket != ticket || s->slots[slot].collected)
    return set_error(RWIG_E_INVALID, "unknown or already collected ticket");
  if (ticket >= s->npub || !*(volatile unsigned*)(s->hdone + slot)) {
    const int rc = publish_ready(s);  // and restart a kernel that went idle before seeing it
    return rc ? rc : 0;
  }
  std::atomic_thread_fence(std::memory_order_seq_cst);
  auto& sl = s->slots[slot];
  const double* r = s->hres + batch::kResStride * (size_t)slot;
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
    out->device_us = r[8] * 1e-3;
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
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->dprob) cudaFree(s->dprob);
    if (s->dctl) cudaFree(s->dctl);
    if (s->dpctl) cudaFree(s->dpctl);
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
