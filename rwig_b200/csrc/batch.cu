// batch.cu -- many log-stabilised Sinkhorn problems of different sizes in one
// persistent launch.
//
// Every problem has the semantics of rwig_sinkhorn_log (Sinkhorn::compute_log,
// src/sinkhorn_impl_log.cpp:225-295) and is solved by ONE CTA, so it needs no
// synchronisation with any other CTA: the launch is a pool of 512-thread
// workers (one per SM) that take problems from a device work list, largest
// first.  A problem's result does not depend on which worker solves it or on
// what else is in the batch (fixed-order reductions inside one CTA).
//
// Per problem, in stabilised scaling form with f~ = g~ = 0:
//   K = exp(-C/eps), u_1 = a / (K 1)                  (the reference's first f update)
//   iteration: v = b / (K^T u) column by column, r = K v row-wise in the same
//              pass over K (the column strip is streamed through a 3-stage
//              bulk-copy ring), err = ||log(u o r) - log a||_2 + ||log(v o K^T u) - log b||_2,
//              then u = a / r unless the loop stops (err < tol or max_iter)
//   final:    f = eps log u, g = eps log v, P = exp(-(C - f - g)/eps),
//             loss = sum C o P + eps sum P o (log P - 1), marginal violations.
// This is the log-domain iteration of the reference written over u = exp(f/eps),
// v = exp(g/eps).  A problem whose scalings leave [e^-650, e^650], whose
// masses are not all positive, or whose sums leave the safe range is handed
// back (status kUnsafe) and re-solved by the per-call path.
#include <algorithm>
#include <cmath>
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
constexpr int kSlot = 8192;           // doubles per ring stage (CW x 512 RPT = 8192 for every class)
constexpr int kMaxRows = 8192;
constexpr double kUnsafeStatus = -100.0;
constexpr double kTimeoutStatus = -5.0;
constexpr double kLogRange = 650.0;   // |log u|, |log v| bound of the scaling form

struct Prob {
  const double* a;
  const double* b;
  const double* C;  // m x n, column-major, leading dimension m
  double* K;        // scratch m x n, leading dimension ldk (even), 16-byte aligned
  long long ldk;
  double* P;        // optional plan (leading dimension m)
  double* f;        // m
  double* g;        // n; holds v during the iterations
  double* res;      // [8]: loss, err, iter, status, l1 row, l1 col, l2 row, l2 col
  int m, n, max_iter, cls;
  double eps, tol;
};

__host__ __device__ constexpr size_t smem_bytes() {
  return (size_t)STAGES * kSlot * 8 + 64 + (size_t)2 * NW * 16 * 8 + 256;
}

// Bulk-copy ring over one problem's column groups.  Sequence numbers continue
// from problem to problem (base), so the mbarrier phases stay consistent.
template <int CW>
struct PRing {
  double* buf;
  uint64_t* bar;
  const double* K;
  long long ldk;
  int n, nst;
  unsigned base, q;
  __device__ int group(unsigned seq) const { return (int)((seq - base) % (unsigned)nst); }
  __device__ double* slot(unsigned seq) const { return buf + (size_t)(seq % STAGES) * kSlot; }
  __device__ void issue(unsigned seq) const {  // thread 0
    const int jb = group(seq) * CW;
    const unsigned bytes = (unsigned)(min(CW, n - jb) * ldk * 8);
    uint64_t* b = bar + (seq % STAGES);
    mbar_arrive_expect_tx(b, bytes);
    bulk_g2s(slot(seq), K + (size_t)jb * ldk, bytes, b);
  }
  __device__ bool wait(unsigned seq) const { return mbar_wait_bounded(bar + (seq % STAGES), (seq / STAGES) & 1u); }
};

// Block-wide fixed-order sums of NV values; every thread gets the totals.
template <int NV>
__device__ __forceinline__ void block_sums(double (&v)[NV], double* red, int& par) {
  block_sum_cols<NV, NW>(v, red, par);
}

// Solves problem p on this CTA; returns false after a timed-out wait (the
// CTA must then stop).  q: the ring's next sequence number (updated).
template <int RPT, int CW>
__device__ bool solve(const Prob& p, double* ringbuf, uint64_t* bar, unsigned& q, double* red, int& par,
                      double* sflag) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int m = p.m, n = p.n;
  const double eps = p.eps;
  int row[RPT];
  bool valid[RPT];
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    row[k] = tid + k * NTT;
    valid[k] = row[k] < m;
  }
  // ---- K = exp(-C/eps) (sinkhorn_impl_vanilla.cpp:41 form) and r = K 1;
  // masses must be positive for the scaling form
  double r[RPT], u[RPT];
  double bad = 0.0;
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    r[k] = 0.0;
    if (valid[k] && !(p.a[row[k]] > 0.0)) bad = 1.0;
  }
  for (int j = tid; j < n; j += NTT)
    if (!(p.b[j] > 0.0)) bad = 1.0;
  for (int j = 0; j < n; ++j) {
    const double* cj = p.C + (size_t)j * m;
    double* kj = p.K + (size_t)j * p.ldk;
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (valid[k]) {
        const double x = exp(-cj[row[k]] / eps);
        kj[row[k]] = x;
        r[k] += x;
      }
  }
  asm volatile("fence.proxy.async.global;" ::: "memory");  // K is read next by bulk copies
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    u[k] = valid[k] ? p.a[row[k]] / r[k] : 0.0;
    if (valid[k] && !(fabs(log(u[k])) <= kLogRange)) bad = 1.0;
  }
  {
    double t[1] = {bad};
    block_sums<1>(t, red, par);
    bad = t[0];
  }
  int iter = 0;
  double err = 1000.0;
  bool ok = true;
  if (bad == 0.0) {
    PRing<CW> ring{ringbuf, bar, p.K, p.ldk, n, (n + CW - 1) / CW, q, q};
    if (tid == 0)
      for (int s = 0; s < STAGES; ++s) ring.issue(ring.q + s);
    while (iter < p.max_iter && err >= p.tol) {
      ++iter;
      double errc = 0.0, vbad = 0.0;
#pragma unroll
      for (int k = 0; k < RPT; ++k) r[k] = 0.0;
      for (int s = 0; s < ring.nst; ++s) {
        const unsigned seq = ring.q;
        if (!ring.wait(seq)) {
          ok = false;
          break;
        }
        const double* buf = ring.slot(seq) + tid;
        const int jb = ring.group(seq) * CW, nc = min(CW, n - jb);
        double kv[RPT][CW], sum[CW];
#pragma unroll
        for (int c = 0; c < CW; ++c) {
          sum[c] = 0.0;
#pragma unroll
          for (int k = 0; k < RPT; ++k) {
            const double x = (c < nc && valid[k]) ? buf[(size_t)c * p.ldk + k * NTT] : 0.0;
            kv[k][c] = x;
            sum[c] = fma(x, u[k], sum[c]);
          }
        }
        block_sum_cols<CW, NW>(sum, red, par);  // (the stage is no longer read after this)
        if (tid == 0) ring.issue(seq + STAGES);
        ring.q = seq + 1;
        double s_l = 1.0;
#pragma unroll
        for (int c = 0; c < CW; ++c)
          if (c == lane) s_l = sum[c];
        const bool owner = lane < nc;
        const double v_l = owner ? p.b[jb + lane] / s_l : 0.0;
        if (w == 0 && owner) {
          p.g[jb + lane] = v_l;
          const double d = log(v_l * s_l) - log(p.b[jb + lane]);
          errc += d * d;
          if (!(fabs(log(v_l)) <= kLogRange) || !(s_l >= 1e-300 && s_l <= 1e300)) vbad = 1.0;
        }
        double v[CW];
#pragma unroll
        for (int c = 0; c < CW; ++c) v[c] = __shfl_sync(0xffffffffu, v_l, c);
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          double acc = r[k];
#pragma unroll
          for (int c = 0; c < CW; ++c) acc = fma(kv[k][c], v[c], acc);
          r[k] = acc;
        }
      }
      if (!ok) break;
      // row half of the error (u of this iteration against the new row sums)
      double errr = 0.0, ubad = 0.0, un[RPT];
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        un[k] = 0.0;
        if (valid[k]) {
          const double ai = p.a[row[k]];
          const double d = log(u[k] * r[k]) - log(ai);
          errr += d * d;
          un[k] = ai / r[k];
          if (!(fabs(log(un[k])) <= kLogRange) || !(r[k] >= 1e-300 && r[k] <= 1e300)) ubad = 1.0;
        }
      }
      double t[4] = {errr, errc, ubad, vbad};
      block_sums<4>(t, red, par);
      err = sqrt(t[0]) + sqrt(t[1]);
      if (t[2] != 0.0 || t[3] != 0.0) {
        bad = 1.0;
        break;
      }
      if (iter < p.max_iter && err >= p.tol) {
#pragma unroll
        for (int k = 0; k < RPT; ++k) u[k] = un[k];
      }
    }
    // drain the prefetched stages before the ring moves on
    if (tid == 0)
      for (int s = 0; s < STAGES; ++s)
        if (!ring.wait(ring.q + s)) ok = false;
    q = ring.q + STAGES;
    if (tid == 0 && !ok) *sflag = 1.0;
    __syncthreads();
    if (*sflag != 0.0) ok = false;
  }
  if (!ok) {
    if (tid == 0) p.res[3] = kTimeoutStatus;
    return false;
  }
  if (bad != 0.0) {
    if (tid == 0) p.res[3] = kUnsafeStatus;
    return true;
  }
  // ---- final pass: f, g, P = exp(-(C - f - g)/eps) (:266), loss (:277), marginals
  double f[RPT], rs[RPT];
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    f[k] = valid[k] ? eps * log(u[k]) : 0.0;
    if (valid[k]) p.f[row[k]] = f[k];
    rs[k] = 0.0;
  }
  double s1 = 0.0, s2 = 0.0, l1c = 0.0, l2c = 0.0;
  for (int jb = 0; jb < n; jb += CW) {
    const int nc = min(CW, n - jb);
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
      for (int k = 0; k < RPT; ++k)
        if (valid[k]) {
          const double cij = cj[row[k]];
          const double pij = exp(-((cij - f[k]) - gj[c]) / eps);
          if (p.P) p.P[(size_t)(jb + c) * m + row[k]] = pij;
          s1 += cij * pij;
          s2 += pij * (log(pij) - 1.0);
          rs[k] += pij;
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
  double l1r = 0.0, l2r = 0.0;
#pragma unroll
  for (int k = 0; k < RPT; ++k)
    if (valid[k]) {
      const double d = rs[k] - p.a[row[k]];
      l1r += fabs(d);
      l2r += d * d;
    }
  double t[6] = {s1, s2, l1r, l1c, l2r, l2c};
  block_sums<6>(t, red, par);
  if (tid == 0) {
    p.res[0] = t[0] + eps * t[1];  // accu(C % P) + reg * accu(P % (log(P) - 1))
    p.res[1] = err;
    p.res[2] = iter;
    p.res[3] = (err <= p.tol) ? 0.0 : (iter == p.max_iter ? 1.0 : 2.0);
    p.res[4] = t[2];
    p.res[5] = t[3];
    p.res[6] = sqrt(t[4]);
    p.res[7] = sqrt(t[5]);
  }
  return true;
}

// Persistent workers: each CTA takes the next problem of `order` until the
// list is exhausted.
__global__ void __launch_bounds__(NTT, 1) batch_kernel(const Prob* probs, const int* order, int count,
                                                        unsigned* head, unsigned* errflag) {
  extern __shared__ __align__(128) unsigned char smem[];
  double* ringbuf = reinterpret_cast<double*>(smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(ringbuf + (size_t)STAGES * kSlot);
  double* red = reinterpret_cast<double*>(smem + (size_t)STAGES * kSlot * 8 + 64);
  double* sflag = red + 2 * NW * 16;
  __shared__ int s_idx;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(bar + s, 1);
    fence_mbar_init();
    *sflag = 0.0;
  }
  __syncthreads();
  unsigned q = 0;
  int par = 0;
  while (true) {
    if (tid == 0) {
      const unsigned i = atomicAdd(head, 1u);
      s_idx = (i < (unsigned)count) ? order[i] : -1;
    }
    __syncthreads();
    const int idx = s_idx;
    __syncthreads();
    if (idx < 0) break;
    const Prob p = probs[idx];
    bool ok = true;
    switch (p.cls) {
      case 0: ok = solve<1, 16>(p, ringbuf, bar, q, red, par, sflag); break;
      case 1: ok = solve<2, 8>(p, ringbuf, bar, q, red, par, sflag); break;
      case 2: ok = solve<4, 4>(p, ringbuf, bar, q, red, par, sflag); break;
      case 3: ok = solve<8, 2>(p, ringbuf, bar, q, red, par, sflag); break;
      default: ok = solve<16, 1>(p, ringbuf, bar, q, red, par, sflag); break;
    }
    if (!ok) {
      if (tid == 0) atomicOr(errflag, 1u);
      break;
    }
  }
}

int row_class(int m) { return m <= 512 ? 0 : m <= 1024 ? 1 : m <= 2048 ? 2 : m <= 4096 ? 3 : 4; }

}  // namespace batch

// Largest M*N solved by the batched kernel; larger problems use the per-call
// path, whose grid-wide sweep is bandwidth-bound at that size.
constexpr long long kBatchMaxElems = 16LL << 20;

enum { SBT_DESC = 200, SBT_ORDER, SBT_RES, SBT_K, SBT_HEAD };

// Batched solve on device pointers.  probs[i] holds device pointers; out[i]
// receives the result.  Returns 0, or a negative error for the whole call
// (individual problems report their own status in out[i].status).
int batch_device(Context* ctx, cudaStream_t st, const rwig_problem* probs, int count, rwig_result* out) {
  using namespace batch;
  if (count < 0 || (count > 0 && (!probs || !out))) return set_error(RWIG_E_INVALID, "bad batch arguments");
  if (count == 0) return 0;
  std::vector<int> inkernel, percall;
  std::vector<long long> koff(count, -1);
  long long ktotal = 0;
  for (int i = 0; i < count; ++i) {
    const rwig_problem& q = probs[i];
    out[i] = rwig_result{};
    if (!q.a || !q.b || !q.C || !q.f || !q.g || q.M < 1 || q.N < 1 || !(q.reg > 0.0) || !std::isfinite(q.reg)) {
      out[i].status = RWIG_E_INVALID;
      continue;
    }
    if (q.M <= kMaxRows && q.max_iter >= 1 && (long long)q.M * q.N <= kBatchMaxElems) {
      inkernel.push_back(i);
      const long long ldk = ((q.M + 1) / 2) * 2;
      koff[i] = ktotal;
      ktotal += ((ldk * q.N + 31) / 32) * 32;  // 256-byte aligned slices
    } else {
      percall.push_back(i);
    }
  }
  int launches = 0;
  if (!inkernel.empty()) {
    const int nb = (int)inkernel.size();
    Prob* dprob = (Prob*)scratch(ctx, SBT_DESC, sizeof(Prob) * nb);
    int* dorder = (int*)scratch(ctx, SBT_ORDER, sizeof(int) * nb);
    double* dres = (double*)scratch(ctx, SBT_RES, sizeof(double) * 8 * nb);
    double* dK = (double*)scratch(ctx, SBT_K, sizeof(double) * std::max<long long>(ktotal, 32));
    unsigned* dhead = (unsigned*)scratch(ctx, SBT_HEAD, sizeof(unsigned) * 2);
    if (!dprob || !dorder || !dres || !dK || !dhead) return RWIG_E_NOMEM;
    std::vector<Prob> hp(nb);
    for (int t = 0; t < nb; ++t) {
      const rwig_problem& q = probs[inkernel[t]];
      Prob& d = hp[t];
      d.a = q.a;
      d.b = q.b;
      d.C = q.C;
      d.ldk = ((q.M + 1) / 2) * 2;
      d.K = dK + koff[inkernel[t]];
      d.P = q.P;
      d.f = q.f;
      d.g = q.g;
      d.res = dres + 8 * (size_t)t;
      d.m = q.M;
      d.n = q.N;
      d.max_iter = q.max_iter;
      d.cls = row_class(q.M);
      d.eps = q.reg;
      d.tol = q.zero_tol;
    }
    // largest first, so the last problems to start are the short ones
    std::vector<int> order(nb);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      return (long long)hp[x].m * hp[x].n > (long long)hp[y].m * hp[y].n;
    });
    RWIG_CUDA_TRY(cudaMemcpyAsync(dprob, hp.data(), sizeof(Prob) * nb, cudaMemcpyHostToDevice, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(dorder, order.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st));
    RWIG_CUDA_TRY(cudaMemsetAsync(dhead, 0, sizeof(unsigned) * 2, st));
    static bool attr = false;
    if (!attr) {
      RWIG_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bytes()));
      attr = true;
    }
    const int grid = std::min(nb, ctx->sm_count);
    batch_kernel<<<grid, NTT, smem_bytes(), st>>>(dprob, dorder, nb, dhead, dhead + 1);
    ++launches;
    RWIG_CUDA_TRY(cudaGetLastError());
    std::vector<double> hres(8 * (size_t)nb);
    unsigned herr = 0;
    RWIG_CUDA_TRY(cudaMemcpyAsync(hres.data(), dres, sizeof(double) * 8 * nb, cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(&herr, dhead + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) return set_error(RWIG_E_TIMEOUT, "a bounded wait in the batched Sinkhorn kernel expired");
    for (int t = 0; t < nb; ++t) {
      rwig_result& o = out[inkernel[t]];
      const double* r = hres.data() + 8 * (size_t)t;
      if (r[3] == kUnsafeStatus) {
        percall.push_back(inkernel[t]);
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
  }
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
    o.path = 1;
    launches += R.kernel_launches;
  }
  reset_report();
  report().kernel_launches = launches;
  return 0;
}

}  // namespace rwig

using namespace rwig;

extern "C" int rwig_batch_sinkhorn_log(const rwig_problem* probs, int count, rwig_result* out) {
  if (count < 0 || (count > 0 && (!probs || !out))) {
    reset_report();
    return set_error(RWIG_E_INVALID, "bad batch arguments");
  }
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = ctx->stream;
  // one device block for every problem's a, b, C, P, f, g (256-byte aligned slices)
  auto al = [](long long x) { return ((x + 31) / 32) * 32; };
  std::vector<long long> off(count + 1, 0);
  for (int i = 0; i < count; ++i) {
    const rwig_problem& q = probs[i];
    const long long M = std::max(q.M, 0), N = std::max(q.N, 0);
    off[i + 1] = off[i] + al(M) + al(N) + al(M * N) + (q.P ? al(M * N) : 0) + al(M) + al(N);
  }
  double* dev = (double*)scratch(ctx, 210, sizeof(double) * std::max<long long>(off[count], 32));
  if (!dev) return RWIG_E_NOMEM;
  std::vector<rwig_problem> dp(probs, probs + count);
  for (int i = 0; i < count; ++i) {
    const rwig_problem& q = probs[i];
    if (!q.a || !q.b || !q.C || !q.f || !q.g || q.M < 1 || q.N < 1) {
      dp[i].a = nullptr;  // rejected by the device driver with RWIG_E_INVALID
      continue;
    }
    const long long M = q.M, N = q.N;
    double* x = dev + off[i];
    double* da = x;
    double* db = da + al(M);
    double* dC = db + al(N);
    double* dP = q.P ? dC + al(M * N) : nullptr;
    double* df = (q.P ? dP + al(M * N) : dC + al(M * N));
    double* dg = df + al(M);
    RWIG_CUDA_TRY(cudaMemcpyAsync(da, q.a, sizeof(double) * M, cudaMemcpyHostToDevice, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(db, q.b, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(dC, q.C, sizeof(double) * M * N, cudaMemcpyHostToDevice, st));
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
    if (probs[i].P) RWIG_CUDA_TRY(cudaMemcpyAsync(probs[i].P, dp[i].P, sizeof(double) * M * N, cudaMemcpyDeviceToHost, st));
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
