// sinkhorn_log.cu -- log-stabilised Sinkhorn on one B200, one persistent
// cooperative launch per solve.
//
// Restates Sinkhorn::compute_log / _fwd_log (src/sinkhorn_impl_log.cpp:225-376):
//   f <- f + eps log a + Rminrow                       (:336)
//   g <- g + eps log b + mincol(R(f, g))               (:348-349)
//   (Rminrow, Rmincol) <- minrowcol(R(f, g)), err      (:359-360)
// with R = C - f 1^T - 1 g^T and softmin_eps(x) = min x - eps log sum exp(-(x - min x)/eps).
//
// Layout and work split.  C is column-major, so a set of whole columns is one
// contiguous range: each CTA owns a strip of columns and streams it through a
// 3-stage shared-memory ring filled by 1-D bulk copies (cp.async.bulk + mbarrier).
// Threads own rows.  One read of C per iteration serves both halves:
//   * column soft-min of D = C - f (complete inside the CTA) -> g update;
//   * the plan after the g update, P'_ij = exp(-(D_ij - g'_j)/eps)
//     = e_ij * b_j / s_j with e_ij the column pass's own exponentials, summed
//     per row into per-CTA partials (no second exponential);
// the row partials are merged across CTAs after a bounded grid barrier, giving
// Rminrow(f, g') = -eps log(sum_j P'_ij), the next f and the stopping error.
// The column half of the error uses softmin(D - g') = softmin(D) - g'.
// The column shift is the exact column minimum in the first iteration and the
// previous iteration's column soft-min afterwards (any shift gives the same
// value; a sum outside [1e-280, 1e280] re-runs that stage with the exact min).
// A row whose merged sum underflows re-runs the row soft-min with a per-row
// running minimum (the reference's shift), as does the initial minrow(C).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace rwig {
namespace sklog {

constexpr int NT = 512;
constexpr int NW = NT / 32;
constexpr int STAGES = 3;

struct Params {
  const double* C;
  long long ldc;
  const double* a;  // reduced marginals
  const double* b;
  int m, n, G;
  double eps, inv_eps;
  int max_iter;
  double tol;
  const double* loga;
  const double* eloga;
  const double* logb;
  const double* elogb;
  double* f0;
  double* f1;
  double* g;
  double* mu;
  double* rowp;   // [G][m]
  double* rowpm;  // [G][m]
  double* part;   // [G][8]
  unsigned* ctrl; // [0] count [1] generation [2] error bits [3] robust events
  double* P;      // optional full-size plan
  long long ldp;
  const int* ridx;  // reduced -> full row index (nullptr = identity)
  const int* cidx;
  double* f_out;  // optional, full size
  double* g_out;
  double* res;    // [8] iter, err, loss, l1row, l1col, l2row, l2col, robust events
};

// Stage ring over this CTA's column groups; the q-th consumed stage holds
// column group (q mod nst) and lives in buffer q mod STAGES.
template <int CW>
struct Ring {
  double* buf;
  uint64_t* bar;
  const double* C;
  long long ldc;
  int c0, c1, nst;
  unsigned q;  // next stage to consume (identical in every thread)

  __device__ int group_begin(unsigned seq) const { return c0 + (int)(seq % (unsigned)nst) * CW; }
  __device__ int group_cols(unsigned seq) const { return min(CW, c1 - group_begin(seq)); }
  __device__ double* slot(unsigned seq) const { return buf + (size_t)(seq % STAGES) * CW * ldc; }

  // thread 0 only
  __device__ void issue(unsigned seq) const {
    const int jb = group_begin(seq);
    const unsigned bytes = (unsigned)(group_cols(seq) * ldc * 8);
    uint64_t* b = bar + (seq % STAGES);
    mbar_arrive_expect_tx(b, bytes);
    bulk_g2s(slot(seq), C + (size_t)jb * ldc, bytes, b);
  }
  __device__ bool wait(unsigned seq) const { return mbar_wait_bounded(bar + (seq % STAGES), (seq / STAGES) & 1u); }
};

__device__ __forceinline__ void flag_error(unsigned* ctrl, unsigned bits) { atomicOr(ctrl + 2, bits); }

// Per-column block reduction: every warp ends with the same total per column.
template <int CW>
__device__ __forceinline__ void block_sum_cols(double (&v)[CW], double* red, int& par) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < CW; ++c) {
    double t = warp_sum(v[c]);
    if (lane == 0) red[(par * NW + w) * CW + c] = t;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < CW; ++c) v[c] = warp_sum(lane < NW ? red[(par * NW + lane) * CW + c] : 0.0);
  par ^= 1;
}

template <int CW>
__device__ __forceinline__ void block_min_cols(double (&v)[CW], double* red, int& par) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < CW; ++c) {
    double t = warp_min(v[c]);
    if (lane == 0) red[(par * NW + w) * CW + c] = t;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < CW; ++c) v[c] = warp_min(lane < NW ? red[(par * NW + lane) * CW + c] : INFINITY);
  par ^= 1;
}

template <int RPT, int CW>
__global__ void __launch_bounds__(NT, 1) sinkhorn_log_kernel(Params p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int cta = blockIdx.x, G = p.G;
  const int m = p.m;
  const double eps = p.eps, inv_eps = p.inv_eps;

  Ring<CW> ring;
  ring.buf = reinterpret_cast<double*>(smem);
  ring.bar = reinterpret_cast<uint64_t*>(smem + (size_t)STAGES * CW * p.ldc * 8);
  double* red = reinterpret_cast<double*>(ring.bar + STAGES);  // [2][NW][CW]
  double* red3 = red + 2 * NW * CW;                            // [NW][32]
  __shared__ double s_scalar[4];
  ring.C = p.C;
  ring.ldc = p.ldc;
  ring.c0 = (int)(((long long)cta * p.n) / G);
  ring.c1 = (int)(((long long)(cta + 1) * p.n) / G);
  ring.nst = (ring.c1 - ring.c0 + CW - 1) / CW;
  ring.q = 0;
  const int r0 = (int)(((long long)cta * m) / G), r1 = (int)(((long long)(cta + 1) * m) / G);
  int par = 0;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(ring.bar + s, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0 && ring.nst > 0)
    for (int s = 0; s < STAGES; ++s) ring.issue(s);

  bool ok = true;
  double f[RPT];
  double* fcur = p.f0;
  double* fnext = p.f1;
  unsigned robust_seen = 0;

  // ---------------------------------------------------------------- helpers
  auto load_f = [&](const double* src) {
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int i = tid + k * NT;
      f[k] = (i < m) ? __ldcg(src + i) : 0.0;
    }
  };

  // Robust row soft-min partials of R = (C - f) - g over this CTA's columns:
  // running (min, sum) per row, one exponential per element.
  auto robust_row_sweep = [&]() -> bool {
    double rm[RPT], rs[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      rm[k] = INFINITY;
      rs[k] = 0.0;
    }
    for (int s = 0; s < ring.nst; ++s) {
      const unsigned seq = ring.q;
      if (!ring.wait(seq)) {
        flag_error(p.ctrl, KERR_MBAR_TIMEOUT);
        return false;
      }
      const double* buf = ring.slot(seq);
      const int jb = ring.group_begin(seq), nc = ring.group_cols(seq);
      for (int c = 0; c < nc; ++c) {
        const double gj = p.g[jb + c];
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          const int i = tid + k * NT;
          if (i < m) {
            const double x = (buf[(size_t)c * p.ldc + i] - f[k]) - gj;
            const double d = x - rm[k];
            const double e = exp(-fabs(d) * inv_eps);
            if (d < 0.0) {
              rs[k] = rs[k] * e + 1.0;
              rm[k] = x;
            } else {
              rs[k] += e;
            }
          }
        }
      }
      __syncthreads();
      if (tid == 0) ring.issue(seq + STAGES);
      ring.q = seq + 1;
    }
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int i = tid + k * NT;
      if (i < m) {
        p.rowpm[(size_t)cta * m + i] = rm[k];
        p.rowp[(size_t)cta * m + i] = rs[k];
      }
    }
    return true;
  };

  // Row merge over all CTAs for rows [r0, r1).  robust: partials are
  // (min, sum) pairs; otherwise plain sums of the plan.  Writes fnext and the
  // CTA's squared row error into part[cta][0].
  auto row_merge = [&](bool robust) {
    double errr = 0.0;
    for (int rb = r0; rb < r1; rb += 32) {
      const int i = rb + lane;
      const bool valid = i < r1;
      double Rrow = 0.0;
      if (robust) {
        double mn = INFINITY;
        if (valid)
          for (int q2 = w; q2 < G; q2 += NW) mn = fmin(mn, __ldcg(p.rowpm + (size_t)q2 * m + i));
        red3[w * 32 + lane] = mn;
        __syncthreads();
        mn = INFINITY;
        for (int ww = 0; ww < NW; ++ww) mn = fmin(mn, red3[ww * 32 + lane]);
        __syncthreads();
        double acc = 0.0;
        if (valid)
          for (int q2 = w; q2 < G; q2 += NW) {
            const double mp = __ldcg(p.rowpm + (size_t)q2 * m + i);
            if (mp < INFINITY) acc += __ldcg(p.rowp + (size_t)q2 * m + i) * exp(-(mp - mn) * inv_eps);
          }
        red3[w * 32 + lane] = acc;
        __syncthreads();
        double tot = 0.0;
        for (int ww = 0; ww < NW; ++ww) tot += red3[ww * 32 + lane];
        Rrow = mn - eps * log(tot);
      } else {
        double acc = 0.0;
        if (valid)
          for (int q2 = w; q2 < G; q2 += NW) acc += __ldcg(p.rowp + (size_t)q2 * m + i);
        red3[w * 32 + lane] = acc;
        __syncthreads();
        double tot = 0.0;
        for (int ww = 0; ww < NW; ++ww) tot += red3[ww * 32 + lane];
        if (w == 0 && valid && !(tot >= 1e-290 && tot <= 1e290)) atomicAdd(p.ctrl + 3, 1u);
        Rrow = -eps * log(tot);
      }
      if (w == 0 && valid) {
        const double d = -Rrow * inv_eps - p.loga[i];
        errr += d * d;
        fnext[i] = __ldcg(fcur + i) + (p.eloga[i] + Rrow);
      }
      __syncthreads();
    }
    if (w == 0) {
      errr = warp_sum(errr);
      if (lane == 0) p.part[(size_t)cta * 8 + 0] = errr;
    }
  };

  // Deterministic sum of part[*][k] over CTAs (same order in every CTA).
  auto total = [&](int k) -> double {
    if (w == 0) {
      double acc = 0.0;
      for (int q2 = lane; q2 < G; q2 += 32) acc += __ldcg(p.part + (size_t)q2 * 8 + k);
      acc = warp_sum(acc);
      if (lane == 0) s_scalar[0] = acc;
    }
    __syncthreads();
    const double v = s_scalar[0];
    __syncthreads();
    return v;
  };

  // -------------------------------------------------------------- init
  int iter = 0;
  double err = 1000.0;
  if (p.max_iter > 0) {
    load_f(fcur);  // zeros
    ok = robust_row_sweep();
    ok = grid_barrier(p.ctrl, p.ctrl + 2, G) && ok;
    if (ok) {
      row_merge(true);
      ok = grid_barrier(p.ctrl, p.ctrl + 2, G);
    }
    { double* t = fcur; fcur = fnext; fnext = t; }
  }

  // -------------------------------------------------------------- iterations
  while (ok && iter < p.max_iter && err >= p.tol) {
    ++iter;
    load_f(fcur);
    double r[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) r[k] = 0.0;
    double errc = 0.0;
    const bool first = (iter == 1);

    for (int s = 0; s < ring.nst && ok; ++s) {
      const unsigned seq = ring.q;
      if (!ring.wait(seq)) {
        flag_error(p.ctrl, KERR_MBAR_TIMEOUT);
        ok = false;
        break;
      }
      const double* buf = ring.slot(seq);
      const int jb = ring.group_begin(seq), nc = ring.group_cols(seq);
      double mu[CW], sum[CW], e[RPT][CW];
      bool exact = first;
      for (int attempt = 0; attempt < 2; ++attempt) {
        if (exact) {
#pragma unroll
          for (int c = 0; c < CW; ++c) {
            double lm = INFINITY;
            if (c < nc) {
#pragma unroll
              for (int k = 0; k < RPT; ++k) {
                const int i = tid + k * NT;
                if (i < m) lm = fmin(lm, buf[(size_t)c * p.ldc + i] - f[k]);
              }
            }
            mu[c] = lm;
          }
          block_min_cols<CW>(mu, red, par);
        } else {
#pragma unroll
          for (int c = 0; c < CW; ++c) mu[c] = (c < nc) ? p.mu[jb + c] : 0.0;
        }
#pragma unroll
        for (int c = 0; c < CW; ++c) {
          sum[c] = 0.0;
#pragma unroll
          for (int k = 0; k < RPT; ++k) {
            const int i = tid + k * NT;
            double ev = 0.0;
            if (c < nc && i < m) ev = exp((mu[c] - (buf[(size_t)c * p.ldc + i] - f[k])) * inv_eps);
            e[k][c] = ev;
            sum[c] += ev;
          }
        }
        block_sum_cols<CW>(sum, red, par);
        bool bad = false;
#pragma unroll
        for (int c = 0; c < CW; ++c)
          if (c < nc && !(sum[c] >= 1e-280 && sum[c] <= 1e280)) bad = true;
        if (!bad || exact) break;
        exact = true;  // block-uniform: every warp holds the same sums
      }
      // every thread has finished reading this slot
      if (tid == 0) ring.issue(seq + STAGES);
      ring.q = seq + 1;

      double beta[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) beta[c] = (c < nc) ? p.b[jb + c] / sum[c] : 0.0;
      if (w == 0 && lane < nc) {
        // column finalisation for column jb + lane (lane < nc <= CW)
        double sml = 0.0, mul = 0.0;
#pragma unroll
        for (int c = 0; c < CW; ++c)
          if (c == lane) {
            sml = sum[c];
            mul = mu[c];
          }
        const int j = jb + lane;
        const double sm = mul - eps * log(sml);   // softmin_i(C_ij - f_i)
        const double gj = p.g[j];
        const double rmin = sm - gj;              // mincol(R(f, g))_j
        const double gn = gj + (p.elogb[j] + rmin);
        p.g[j] = gn;
        p.mu[j] = sm;
        const double d = -(sm - gn) * inv_eps - p.logb[j];
        errc += d * d;
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < CW; ++c) acc += e[k][c] * beta[c];
        r[k] += acc;
      }
    }
    if (!ok) break;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int i = tid + k * NT;
      if (i < m) p.rowp[(size_t)cta * m + i] = r[k];
    }
    if (w == 0) {
      errc = warp_sum(errc);
      if (lane == 0) p.part[(size_t)cta * 8 + 1] = errc;
    }
    if (!grid_barrier(p.ctrl, p.ctrl + 2, G)) { ok = false; break; }
    row_merge(false);
    if (!grid_barrier(p.ctrl, p.ctrl + 2, G)) { ok = false; break; }
    const unsigned rob = *(volatile unsigned*)(p.ctrl + 3);
    if (rob != robust_seen) {
      // some merged row sum left the safe range: redo the row soft-min with
      // the reference's per-row minimum shift, with g already updated
      robust_seen = rob;
      if (!robust_row_sweep()) { ok = false; break; }
      if (!grid_barrier(p.ctrl, p.ctrl + 2, G)) { ok = false; break; }
      row_merge(true);
      if (!grid_barrier(p.ctrl, p.ctrl + 2, G)) { ok = false; break; }
    }
    const double er = total(0), ec = total(1);
    err = sqrt(er) + sqrt(ec);
    if (iter < p.max_iter && err >= p.tol) {
      double* t = fcur;
      fcur = fnext;
      fnext = t;
    }
  }

  // -------------------------------------------------------------- final plan, loss, report
  if (ok) {
    load_f(fcur);
    double rr[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) rr[k] = 0.0;
    double l1 = 0.0, l2 = 0.0, c1 = 0.0, c2 = 0.0;
    for (int s = 0; s < ring.nst && ok; ++s) {
      const unsigned seq = ring.q;
      if (!ring.wait(seq)) {
        flag_error(p.ctrl, KERR_MBAR_TIMEOUT);
        ok = false;
        break;
      }
      const double* buf = ring.slot(seq);
      const int jb = ring.group_begin(seq), nc = ring.group_cols(seq);
      double cs[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) {
        cs[c] = 0.0;
        if (c < nc) {
          const int j = jb + c;
          const double gj = p.g[j];
          const long long jf = p.cidx ? p.cidx[j] : j;
#pragma unroll
          for (int k = 0; k < RPT; ++k) {
            const int i = tid + k * NT;
            if (i < m) {
              const double cij = buf[(size_t)c * p.ldc + i];
              const double R = (cij - f[k]) - gj;
              const double Pv = exp(-R * inv_eps);
              if (p.P) {
                const long long ifull = p.ridx ? p.ridx[i] : i;
                p.P[ifull + jf * p.ldp] = Pv;
              }
              l1 += cij * Pv;
              l2 += Pv * (log(Pv) - 1.0);
              rr[k] += Pv;
              cs[c] += Pv;
            }
          }
        }
      }
      block_sum_cols<CW>(cs, red, par);
      if (tid == 0) ring.issue(seq + STAGES);
      ring.q = seq + 1;
      if (w == 0 && lane < nc) {
        double csl = 0.0;
#pragma unroll
        for (int c = 0; c < CW; ++c)
          if (c == lane) csl = cs[c];
        const int j = jb + lane;
        const double d = csl - p.b[j];
        c1 += fabs(d);
        c2 += d * d;
        if (p.g_out) p.g_out[p.cidx ? p.cidx[j] : j] = p.g[j];
      }
    }
    if (ok) {
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int i = tid + k * NT;
        if (i < m) p.rowp[(size_t)cta * m + i] = rr[k];
      }
      // block-reduce the loss and column-violation partials
      double v[4] = {l1, l2, c1, c2};
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        double x = warp_sum(v[t]);
        if (lane == 0) red3[w * 4 + t] = x;
      }
      __syncthreads();
      if (tid < 4) {
        double acc = 0.0;
        for (int ww = 0; ww < NW; ++ww) acc += red3[ww * 4 + tid];
        p.part[(size_t)cta * 8 + 2 + tid] = acc;
      }
      __syncthreads();
      ok = grid_barrier(p.ctrl, p.ctrl + 2, G);
    }
    if (ok) {
      double a1 = 0.0, a2 = 0.0;
      for (int rb = r0; rb < r1; rb += 32) {
        const int i = rb + lane;
        const bool valid = i < r1;
        double acc = 0.0;
        if (valid)
          for (int q2 = w; q2 < G; q2 += NW) acc += __ldcg(p.rowp + (size_t)q2 * m + i);
        red3[w * 32 + lane] = acc;
        __syncthreads();
        if (w == 0 && valid) {
          double tot = 0.0;
          for (int ww = 0; ww < NW; ++ww) tot += red3[ww * 32 + lane];
          const double d = tot - p.a[i];
          a1 += fabs(d);
          a2 += d * d;
          if (p.f_out) p.f_out[p.ridx ? p.ridx[i] : i] = __ldcg(fcur + i);
        }
        __syncthreads();
      }
      if (w == 0) {
        a1 = warp_sum(a1);
        a2 = warp_sum(a2);
        if (lane == 0) {
          p.part[(size_t)cta * 8 + 6] = a1;
          p.part[(size_t)cta * 8 + 7] = a2;
        }
      }
      ok = grid_barrier(p.ctrl, p.ctrl + 2, G);
    }
    if (ok && cta == 0) {
      const double tl1 = total(2), tl2 = total(3), tc1 = total(4), tc2 = total(5), tr1 = total(6),
                   tr2 = total(7);
      if (tid == 0) {
        p.res[0] = iter;
        p.res[1] = err;
        p.res[2] = tl1 + eps * tl2;
        p.res[3] = tr1;
        p.res[4] = tc1;
        p.res[5] = sqrt(tr2);
        p.res[6] = sqrt(tc2);
        p.res[7] = *(volatile unsigned*)(p.ctrl + 3);
      }
    }
  }

  // drain the bulk copies still in flight into this CTA's ring
  if (tid == 0 && ring.nst > 0) {
    for (unsigned s = 0; s < (unsigned)STAGES; ++s) {
      const unsigned seq = ring.q + s;
      if (!ring.wait(seq)) flag_error(p.ctrl, KERR_MBAR_TIMEOUT);
    }
  }
}

// Small helpers --------------------------------------------------------------
__global__ void prep_kernel(const double* a, const double* b, int m, int n, double eps, double* loga,
                            double* eloga, double* logb, double* elogb, double* f0, double* g,
                            double* mu, unsigned* ctrl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int i = t; i < m; i += stride) {
    const double la = log(a[i]);
    loga[i] = la;
    eloga[i] = eps * la;
    f0[i] = 0.0;
  }
  for (int j = t; j < n; j += stride) {
    const double lb = log(b[j]);
    logb[j] = lb;
    elogb[j] = eps * lb;
    g[j] = 0.0;
    mu[j] = 0.0;
  }
  if (t < 4) ctrl[t] = 0u;
}

__global__ void gather_kernel(const double* C, long long ldC, const int* ridx, const int* cidx, int m,
                              int n, double* out, long long ldo) {
  const long long total = (long long)ldo * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldo);
    const int j = (int)(k / ldo);
    double v = 0.0;
    if (i < m) v = C[(ridx ? ridx[i] : i) + (long long)(cidx ? cidx[j] : j) * ldC];
    out[k] = v;
  }
}

__global__ void gather_vec(const double* x, const int* idx, int n, double* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[k] = x[idx ? idx[k] : k];
}

__global__ void fill_kernel(double* x, long long n, double v) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    x[k] = v;
}

template <int RPT, int CW>
int launch(Context* ctx, Params& p, cudaStream_t st, int* launches) {
  auto kern = sinkhorn_log_kernel<RPT, CW>;
  const size_t smem = (size_t)STAGES * CW * p.ldc * 8 + STAGES * 8 + (2 * NW * CW + NW * 32) * 8;
  if ((int)smem > ctx->smem_optin) return set_error(RWIG_E_UNSUPPORTED, "stage ring exceeds shared memory");
  RWIG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NT, smem));
  if (occ < 1) return set_error(RWIG_E_UNSUPPORTED, "kernel does not fit on an SM");
  const int maxG = occ * ctx->sm_count;
  p.G = std::min(p.G, maxG);  // p.G arrives as the scratch-sized cap
  void* args[] = {&p};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(p.G), dim3(NT), args, smem, st));
  ++*launches;
  return 0;
}

}  // namespace sklog

// Scratch slot numbers used by the log-Sinkhorn entry points.
enum {
  SL_LOGA = 0, SL_ELOGA, SL_LOGB, SL_ELOGB, SL_F0, SL_F1, SL_G, SL_MU, SL_ROWP, SL_ROWPM, SL_PART,
  SL_CTRL, SL_RES, SL_CRED, SL_AR, SL_BR, SL_RIDX, SL_CIDX, SL_HOST_C, SL_HOST_A, SL_HOST_B,
  SL_HOST_P, SL_HOST_F, SL_HOST_G
};

// Core of both log-Sinkhorn entry points: inputs on the device.
static int sinkhorn_log_device(Context* ctx, cudaStream_t st, double* P, double* grad_a, double* f,
                               double* g, double* loss, int* iter, double* err, const double* a,
                               const double* b, const double* C, int M, int N, double reg,
                               int withgrad, int max_iter, double zero_tol) {
  using namespace sklog;
  reset_report();
  if (!a || !b || !C) return set_error(RWIG_E_INVALID, "a, b and C must be non-null");
  if (M < 1 || N < 1) return set_error(RWIG_E_INVALID, "M and N must be >= 1");
  if (!(reg > 0.0) || !std::isfinite(reg)) return set_error(RWIG_E_INVALID, "reg must be finite and > 0");
  if (withgrad && grad_a)
    return set_error(RWIG_E_UNSUPPORTED, "log-Sinkhorn gradient is not available in this build");
  int launches = 0;

  // support reduction (src/sinkhorn_impl_log.cpp:238-249): drop zero masses
  std::vector<double> ha(M), hb(N);
  RWIG_CUDA_TRY(cudaMemcpyAsync(ha.data(), a, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(hb.data(), b, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<int> ri, ci;
  for (int i = 0; i < M; ++i)
    if (ha[i] != 0.0) ri.push_back(i);
  for (int j = 0; j < N; ++j)
    if (hb[j] != 0.0) ci.push_back(j);
  const int m = (int)ri.size(), n = (int)ci.size();
  if (m == 0 || n == 0)
    return set_error(RWIG_E_INVALID, "a and b must each have at least one non-zero entry");
  if (m > 16 * NT) return set_error(RWIG_E_UNSUPPORTED, "more than 8192 supported rows");
  const bool reduced = (m != M) || (n != N);
  // the stage ring bulk-copies whole columns: C must start on 16 bytes and
  // have an even leading dimension, otherwise it is repacked first
  const bool need_gather = reduced || (M % 2) != 0 || (reinterpret_cast<uintptr_t>(C) % 16) != 0;
  const long long ldc = need_gather ? ((m + 1) / 2) * 2 : M;

  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
  int* d_ridx = nullptr;
  int* d_cidx = nullptr;
  const double* Cr = C;
  const double* ar = a;
  const double* br = b;
  if (need_gather) {
    if (reduced) {
      d_ridx = (int*)scratch(ctx, SL_RIDX, sizeof(int) * m);
      d_cidx = (int*)scratch(ctx, SL_CIDX, sizeof(int) * n);
      if (!d_ridx || !d_cidx) return RWIG_E_NOMEM;
      RWIG_CUDA_TRY(cudaMemcpyAsync(d_ridx, ri.data(), sizeof(int) * m, cudaMemcpyHostToDevice, st));
      RWIG_CUDA_TRY(cudaMemcpyAsync(d_cidx, ci.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    }
    double* cbuf = (double*)scratch(ctx, SL_CRED, sizeof(double) * ldc * n);
    double* abuf = (double*)scratch(ctx, SL_AR, sizeof(double) * m);
    double* bbuf = (double*)scratch(ctx, SL_BR, sizeof(double) * n);
    if (!cbuf || !abuf || !bbuf) return RWIG_E_NOMEM;
    gather_kernel<<<4 * ctx->sm_count, 256, 0, st>>>(C, M, d_ridx, d_cidx, m, n, cbuf, ldc);
    gather_vec<<<(m + 255) / 256, 256, 0, st>>>(a, d_ridx, m, abuf);
    gather_vec<<<(n + 255) / 256, 256, 0, st>>>(b, d_cidx, n, bbuf);
    launches += 3;
    Cr = cbuf;
    ar = abuf;
    br = bbuf;
  }

  Params p{};
  p.C = Cr;
  p.ldc = ldc;
  p.a = ar;
  p.b = br;
  p.m = m;
  p.n = n;
  p.eps = reg;
  p.inv_eps = 1.0 / reg;
  p.max_iter = max_iter;
  p.tol = zero_tol;
  const int Gmax = std::min(n, 2 * ctx->sm_count);
  double* loga = (double*)scratch(ctx, SL_LOGA, sizeof(double) * m);
  double* eloga = (double*)scratch(ctx, SL_ELOGA, sizeof(double) * m);
  double* logb = (double*)scratch(ctx, SL_LOGB, sizeof(double) * n);
  double* elogb = (double*)scratch(ctx, SL_ELOGB, sizeof(double) * n);
  p.f0 = (double*)scratch(ctx, SL_F0, sizeof(double) * m);
  p.f1 = (double*)scratch(ctx, SL_F1, sizeof(double) * m);
  p.g = (double*)scratch(ctx, SL_G, sizeof(double) * n);
  p.mu = (double*)scratch(ctx, SL_MU, sizeof(double) * n);
  p.rowp = (double*)scratch(ctx, SL_ROWP, sizeof(double) * (size_t)Gmax * m);
  p.rowpm = (double*)scratch(ctx, SL_ROWPM, sizeof(double) * (size_t)Gmax * m);
  p.part = (double*)scratch(ctx, SL_PART, sizeof(double) * (size_t)Gmax * 8);
  p.ctrl = (unsigned*)scratch(ctx, SL_CTRL, sizeof(unsigned) * 4);
  p.res = (double*)scratch(ctx, SL_RES, sizeof(double) * 8);
  if (!loga || !eloga || !logb || !elogb || !p.f0 || !p.f1 || !p.g || !p.mu || !p.rowp || !p.rowpm ||
      !p.part || !p.ctrl || !p.res)
    return RWIG_E_NOMEM;
  p.loga = loga;
  p.eloga = eloga;
  p.logb = logb;
  p.elogb = elogb;
  p.P = P;
  p.ldp = M;
  p.ridx = d_ridx;
  p.cidx = d_cidx;
  p.f_out = f;
  p.g_out = g;
  p.G = Gmax;

  prep_kernel<<<std::max(1, (std::max(m, n) + 255) / 256), 256, 0, st>>>(
      ar, br, m, n, reg, loga, eloga, logb, elogb, p.f0, p.g, p.mu, p.ctrl);
  ++launches;
  if (reduced) {
    if (P) {
      RWIG_CUDA_TRY(cudaMemsetAsync(P, 0, sizeof(double) * (size_t)M * N, st));
    }
    if (f && m < M) {
      fill_kernel<<<(M + 255) / 256, 256, 0, st>>>(f, M, -INFINITY);
      ++launches;
    }
    if (g && n < N) {
      fill_kernel<<<(N + 255) / 256, 256, 0, st>>>(g, N, -INFINITY);
      ++launches;
    }
  }

  const int rpt_need = (m + NT - 1) / NT;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->evk, st));
  int rc;
  if (rpt_need <= 1) rc = launch<1, 16>(ctx, p, st, &launches);
  else if (rpt_need <= 2) rc = launch<2, 8>(ctx, p, st, &launches);
  else if (rpt_need <= 4) rc = launch<4, 4>(ctx, p, st, &launches);
  else if (rpt_need <= 8) rc = launch<8, 2>(ctx, p, st, &launches);
  else rc = launch<16, 1>(ctx, p, st, &launches);
  if (rc != 0) return rc;
  RWIG_CUDA_TRY(cudaGetLastError());
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));

  double res[8];
  unsigned ctrl[4];
  RWIG_CUDA_TRY(cudaMemcpyAsync(res, p.res, sizeof(res), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(ctrl, p.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (ctrl[2] != 0u) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "log-Sinkhorn kernel stopped by a bounded wait (error bits 0x%x)", ctrl[2]);
    return set_error(RWIG_E_TIMEOUT, buf);
  }
  float ms = 0.f, kms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  cudaEventElapsedTime(&kms, ctx->evk, ctx->ev1);
  const int it = (int)res[0];
  const double e = res[1];
  if (loss) *loss = res[2];
  if (iter) *iter = it;
  if (err) *err = e;
  const int status = (e <= zero_tol) ? 0 : (it == max_iter ? 1 : 2);
  rwig_report& R = report();
  R.iter = it;
  R.status = status;
  R.err = e;
  R.marg_l1_row = res[3];
  R.marg_l1_col = res[4];
  R.marg_l2_row = res[5];
  R.marg_l2_col = res[6];
  R.device_ms = ms;
  R.kernel_ms = kms;
  R.fallback_events = (int)res[7];
  R.kernel_launches = launches;
  R.support_m = m;
  R.support_n = n;
  return status;
}

}  // namespace rwig

using namespace rwig;

extern "C" int rwig_sinkhorn_log_dev(double* P, double* grad_a, double* f, double* g, double* loss,
                                     int* iter, double* err, const double* a, const double* b,
                                     const double* C, int M, int N, double reg, int withgrad,
                                     int max_iter, double zero_tol, void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  return sinkhorn_log_device(ctx, st, P, grad_a, f, g, loss, iter, err, a, b, C, M, N, reg, withgrad,
                             max_iter, zero_tol);
}

extern "C" int rwig_sinkhorn_log(double* P, double* grad_a, double* f, double* g, double* loss,
                                 int* iter, double* err, const double* a, const double* b,
                                 const double* C, int M, int N, double reg, int withgrad,
                                 int max_iter, double zero_tol) {
  if (!a || !b || !C || M < 1 || N < 1) return set_error(RWIG_E_INVALID, "bad arguments");
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = ctx->stream;
  const size_t MN = (size_t)M * N;
  double* dC = (double*)scratch(ctx, SL_HOST_C, sizeof(double) * MN);
  double* da = (double*)scratch(ctx, SL_HOST_A, sizeof(double) * M);
  double* db = (double*)scratch(ctx, SL_HOST_B, sizeof(double) * N);
  double* dP = P ? (double*)scratch(ctx, SL_HOST_P, sizeof(double) * MN) : nullptr;
  double* df = f ? (double*)scratch(ctx, SL_HOST_F, sizeof(double) * M) : nullptr;
  double* dg = g ? (double*)scratch(ctx, SL_HOST_G, sizeof(double) * N) : nullptr;
  if (!dC || !da || !db || (P && !dP) || (f && !df) || (g && !dg)) return RWIG_E_NOMEM;
  RWIG_CUDA_TRY(cudaMemcpyAsync(dC, C, sizeof(double) * MN, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(da, a, sizeof(double) * M, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(db, b, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  int rc = sinkhorn_log_device(ctx, st, dP, grad_a, df, dg, loss, iter, err, da, db, dC, M, N, reg,
                               withgrad, max_iter, zero_tol);
  if (rc < 0) return rc;
  if (P) RWIG_CUDA_TRY(cudaMemcpyAsync(P, dP, sizeof(double) * MN, cudaMemcpyDeviceToHost, st));
  if (f) RWIG_CUDA_TRY(cudaMemcpyAsync(f, df, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
  if (g) RWIG_CUDA_TRY(cudaMemcpyAsync(g, dg, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  return rc;
}

// ===========================================================================
// Allocation-free log-Sinkhorn (rwig_sinkhorn_log_noalloc).
//
// Some callers cannot let a library allocate device memory: a host framework
// that has reserved the GPU's memory for its own pool, a process running under
// a hard device-memory quota where a failed allocation in the middle of a
// request is not acceptable, or a serving loop that must not pay for the
// device-wide synchronisation that cudaMalloc / cudaFree can cause.  For them
// this entry point runs the same solver kernel on a fixed scratch block that
// lives in the library image itself: a file-scope __device__ array, created
// when the library's device code is loaded and held by every GPU that loads
// it until the process exits.  The caller passes all inputs and outputs.
//
// Limits: M <= 4096, N <= 4096, at most 148 CTAs, strictly positive a and b
// (no support reduction, which would need a packed copy of C), M even and C
// 16-byte aligned (the stage ring bulk-copies whole columns of C in place).
// Larger or other inputs are rejected with RWIG_E_UNSUPPORTED.
//
// The scratch block is shared by every call on a device and keeps the last
// call's contents; the control words, the potentials and the shifts are reset
// at the start of each call by the preparation kernel.  Two calls whose work
// overlaps on the GPU (different streams or host threads on the same device)
// race on the block and give wrong results: callers must serialise them.
// The first call on a device looks up the block's device address
// (cudaGetSymbolAddress, with that device current) and caches it; make that
// first call before any stream capture on the device.
// ===========================================================================
namespace rwig {
namespace sklog_noalloc {

constexpr int kMaxM = 4096;
constexpr int kMaxN = 4096;
constexpr int kMaxCtas = 148;
// layout in doubles
constexpr size_t kOffLogA = 0;
constexpr size_t kOffELogA = kOffLogA + kMaxM;
constexpr size_t kOffF0 = kOffELogA + kMaxM;
constexpr size_t kOffF1 = kOffF0 + kMaxM;
constexpr size_t kOffLogB = kOffF1 + kMaxM;
constexpr size_t kOffELogB = kOffLogB + kMaxN;
constexpr size_t kOffG = kOffELogB + kMaxN;
constexpr size_t kOffMu = kOffG + kMaxN;
constexpr size_t kOffRowP = kOffMu + kMaxN;
constexpr size_t kOffRowPM = kOffRowP + (size_t)kMaxCtas * kMaxM;
constexpr size_t kOffPart = kOffRowPM + (size_t)kMaxCtas * kMaxM;
constexpr size_t kOffRes = kOffPart + (size_t)kMaxCtas * 8;
constexpr size_t kOffCtrl = kOffRes + 8;  // 8 unsigned words = 4 doubles
constexpr size_t kDoubles = kOffCtrl + 4;  // about 10.0 MB in total

static __device__ __align__(256) double g_scratch[kDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_ptr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};
int g_smem_optin[kMaxDevices] = {};

// Once per device, with that device current: device address of g_scratch.
int setup(int dev, double** base, int* sms, int* smem_optin) {
  if (dev < 0 || dev >= kMaxDevices) return set_error(RWIG_E_NODEVICE, "device index beyond 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    int major = 0;
    RWIG_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major < 10) return set_error(RWIG_E_NODEVICE, "device is not sm_100 class (this build targets sm_100a)");
    RWIG_CUDA_TRY(cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    RWIG_CUDA_TRY(cudaDeviceGetAttribute(&g_smem_optin[dev], cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    g_ptr[dev] = static_cast<double*>(p);
  }
  *base = g_ptr[dev];
  *sms = g_sms[dev];
  *smem_optin = g_smem_optin[dev];
  return 0;
}

// Counts zero entries of a and b into *out (one block).
__global__ void count_zero_masses(const double* a, const double* b, int m, int n, unsigned* out) {
  __shared__ unsigned s_cnt;
  if (threadIdx.x == 0) s_cnt = 0u;
  __syncthreads();
  unsigned c = 0u;
  for (int i = threadIdx.x; i < m; i += blockDim.x) c += (a[i] == 0.0);
  for (int j = threadIdx.x; j < n; j += blockDim.x) c += (b[j] == 0.0);
  atomicAdd(&s_cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) *out = s_cnt;
}

template <int RPT, int CW>
int launch_noalloc(sklog::Params& p, int sms, int smem_optin, cudaStream_t st) {
  using namespace sklog;
  auto kern = sinkhorn_log_kernel<RPT, CW>;
  const size_t smem = (size_t)STAGES * CW * p.ldc * 8 + STAGES * 8 + (2 * NW * CW + NW * 32) * 8;
  if ((int)smem > smem_optin) return set_error(RWIG_E_UNSUPPORTED, "stage ring exceeds shared memory");
  RWIG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NT, smem));
  if (occ < 1) return set_error(RWIG_E_UNSUPPORTED, "kernel does not fit on an SM");
  p.G = std::min(std::min(p.n, occ * sms), kMaxCtas);
  void* args[] = {&p};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(p.G), dim3(NT), args, smem, st));
  return 0;
}

}  // namespace sklog_noalloc
}  // namespace rwig

extern "C" int rwig_sinkhorn_log_noalloc(double* P, double* f, double* g, double* loss, int* iter,
                                         double* err, const double* a, const double* b, const double* C,
                                         int M, int N, double reg, int max_iter, double zero_tol,
                                         void* stream) {
  using namespace rwig;
  using namespace rwig::sklog_noalloc;
  reset_report();
  if (!a || !b || !C) return set_error(RWIG_E_INVALID, "a, b and C must be non-null");
  if (M < 1 || N < 1) return set_error(RWIG_E_INVALID, "M and N must be >= 1");
  if (!(reg > 0.0) || !std::isfinite(reg)) return set_error(RWIG_E_INVALID, "reg must be finite and > 0");
  if (M > kMaxM || N > kMaxN)
    return set_error(RWIG_E_UNSUPPORTED,
                     "problem exceeds the no-allocation limit of M <= 4096 and N <= 4096; "
                     "use rwig_sinkhorn_log_dev");
  if (M % 2 != 0 || (reinterpret_cast<uintptr_t>(C) % 16) != 0)
    return set_error(RWIG_E_UNSUPPORTED,
                     "the no-allocation entry needs an even M and a 16-byte aligned C; "
                     "use rwig_sinkhorn_log_dev");
  int dev = 0;
  RWIG_CUDA_TRY(cudaGetDevice(&dev));
  double* base = nullptr;
  int sms = 0, smem_optin = 0;
  int rc = setup(dev, &base, &sms, &smem_optin);
  if (rc != 0) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  sklog::Params p{};
  p.C = C;
  p.ldc = M;
  p.a = a;
  p.b = b;
  p.m = M;
  p.n = N;
  p.eps = reg;
  p.inv_eps = 1.0 / reg;
  p.max_iter = max_iter;
  p.tol = zero_tol;
  p.loga = base + kOffLogA;
  p.eloga = base + kOffELogA;
  p.logb = base + kOffLogB;
  p.elogb = base + kOffELogB;
  p.f0 = base + kOffF0;
  p.f1 = base + kOffF1;
  p.g = base + kOffG;
  p.mu = base + kOffMu;
  p.rowp = base + kOffRowP;
  p.rowpm = base + kOffRowPM;
  p.part = base + kOffPart;
  p.res = base + kOffRes;
  p.ctrl = reinterpret_cast<unsigned*>(base + kOffCtrl);
  p.P = P;
  p.ldp = M;
  p.ridx = nullptr;
  p.cidx = nullptr;
  p.f_out = f;
  p.g_out = g;

  // every word the solver reads before writing is reset here: control words,
  // f, g and the column shifts
  sklog::prep_kernel<<<std::max(1, (std::max(M, N) + 255) / 256), 256, 0, st>>>(
      a, b, M, N, reg, base + kOffLogA, base + kOffELogA, base + kOffLogB, base + kOffELogB,
      base + kOffF0, base + kOffG, base + kOffMu, p.ctrl);
  count_zero_masses<<<1, 256, 0, st>>>(a, b, M, N, p.ctrl + 4);
  RWIG_CUDA_TRY(cudaGetLastError());
  unsigned zeros = 0u;
  RWIG_CUDA_TRY(cudaMemcpyAsync(&zeros, p.ctrl + 4, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (zeros != 0u)
    return set_error(RWIG_E_UNSUPPORTED,
                     "the no-allocation entry needs strictly positive a and b (zero masses need the "
                     "support-reducing rwig_sinkhorn_log_dev)");

  const int rpt_need = (M + sklog::NT - 1) / sklog::NT;
  if (rpt_need <= 1) rc = launch_noalloc<1, 16>(p, sms, smem_optin, st);
  else if (rpt_need <= 2) rc = launch_noalloc<2, 8>(p, sms, smem_optin, st);
  else if (rpt_need <= 4) rc = launch_noalloc<4, 4>(p, sms, smem_optin, st);
  else rc = launch_noalloc<8, 2>(p, sms, smem_optin, st);
  if (rc != 0) return rc;
  RWIG_CUDA_TRY(cudaGetLastError());

  double res[8];
  unsigned ctrl[4];
  RWIG_CUDA_TRY(cudaMemcpyAsync(res, p.res, sizeof(res), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(ctrl, p.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (ctrl[2] != 0u) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "log-Sinkhorn kernel stopped by a bounded wait (error bits 0x%x)", ctrl[2]);
    return set_error(RWIG_E_TIMEOUT, buf);
  }
  const int it = (int)res[0];
  const double e = res[1];
  if (loss) *loss = res[2];
  if (iter) *iter = it;
  if (err) *err = e;
  const int status = (e <= zero_tol) ? 0 : (it == max_iter ? 1 : 2);
  rwig_report& R = report();
  R.iter = it;
  R.status = status;
  R.err = e;
  R.marg_l1_row = res[3];
  R.marg_l1_col = res[4];
  R.marg_l2_row = res[5];
  R.marg_l2_col = res[6];
  R.fallback_events = (int)res[7];
  R.kernel_launches = 3;
  R.support_m = M;
  R.support_n = N;
  return status;
}
