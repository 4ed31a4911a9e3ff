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
#include "fastexp.cuh"
#include "sk_common.cuh"
#include "sk_host.h"

namespace rwig {
namespace sklog {

using sk::STAGES;
using sk::Ring;
using sk::flag_error;
using sk::block_sum_cols;
using sk::block_min_cols;
using sk::sum_partials;

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
  double* res;    // [9] iter, err, loss, l1row, l1col, l2row, l2col, robust events, finished
  int ncol_max;   // upper bound of columns per CTA (sizes the shared column arrays)
  // Resumable runs.  resume = 1 starts from f = f0 (reduced, set by the host)
  // and g = g_state after iter0 iterations with error err0, skipping the
  // initial row sweep.  iter_cap > 0 stops after that many iterations of this
  // launch.  At exit f_state / g_state hold the state to resume from (the f
  // of the next iteration and the current g) or, once the solve is finished
  // (err < tol or max_iter), the final f and g; res[8] = 1 when finished.
  // do_final = 0 skips the plan / loss / marginal pass.
  int resume, iter0, iter_cap, do_final;
  double err0;
  double* f_state;
  double* g_state;
  // optional history for the gradient: f_l at fh[l * m] (l = 1..L+1, the f
  // computed at the end of iteration l - 1) and g_l at gh[l * n] (l = 1..L)
  double* fh;
  double* gh;
};

// Dynamic shared memory of one CTA: stage ring, mbarriers, reduction scratch,
// exp table and the per-column state of the CTA's strip (b, log b, eps log b, g, shift).
template <int CW, int NWARPS>
__host__ __device__ constexpr size_t smem_bytes(long long ldc, int ncol_max) {
  return (size_t)STAGES * CW * ldc * 8 + STAGES * 8 +
         (size_t)(2 * NWARPS * CW + NWARPS * 32 + 64 * kExpTableSpread) * 8 +
         (size_t)6 * ncol_max * 8;
}

// RPT rows per thread, CW columns per stage, NTT threads per CTA; FULL when
// every thread row is a real row (m == RPT * NTT), which drops the row masks.
template <int RPT, int CW, int NTT, bool FULL>
__global__ void __launch_bounds__(NTT, 1) sinkhorn_log_kernel(Params p) {
  constexpr int NT = NTT;
  constexpr int NW = NTT / 32;
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
  double* tbl = red3 + NW * 32;                                // [64 x 16] 2^(j/64), bank-spread
  const double* tbl_l = tbl + (tid & (kExpTableSpread - 1));  // this lane's replica
  const int NCM = p.ncol_max;
  double* cb = tbl + 64 * kExpTableSpread;  // b_j of this CTA's columns
  double* clogb = cb + NCM;     // log b_j
  double* celogb = clogb + NCM; // eps log b_j
  double* cg = celogb + NCM;    // g_j
  double* cmu = cg + NCM;       // column shift (previous column soft-min / eps)
  double* csum = cmu + NCM;     // column sums of the current sweep
  __shared__ double s_scalar[4];
  ring.C = p.C;
  ring.ldc = p.ldc;
  ring.c0 = (int)(((long long)cta * p.n) / G);
  ring.c1 = (int)(((long long)(cta + 1) * p.n) / G);
  ring.nst = (ring.c1 - ring.c0 + CW - 1) / CW;
  ring.q = 0;
  // C streams through L2 once per sweep: mark it first to evict, which keeps
  // the small per-iteration vectors and partials resident
  ring.hot_groups = 0;
  ring.pol_cold = l2_policy_evict_first();
  const int r0 = (int)(((long long)cta * m) / G), r1 = (int)(((long long)(cta + 1) * m) / G);
  int par = 0;

  load_exp_table_spread(tbl);
  for (int c = tid; c < ring.c1 - ring.c0; c += NT) {
    const int j = ring.c0 + c;
    cb[c] = p.b[j];
    clogb[c] = p.logb[j];
    celogb[c] = p.elogb[j];
    cg[c] = p.resume ? p.g_state[j] : 0.0;
    cmu[c] = 0.0;
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(ring.bar + s, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0 && ring.nst > 0)
    for (int s = 0; s < STAGES; ++s) ring.issue(s);

  bool ok = true;
  unsigned nbar = 0;  // grid barriers passed so far (same in every CTA)
  auto gsync = [&]() -> bool { ++nbar; return grid_sync(p.ctrl, p.ctrl + 2, nbar * (unsigned)G); };
  // fr[k]: this thread's rows of f, scaled by 1/eps during the iterations
  double fr[RPT];
  bool valid[RPT];
#pragma unroll
  for (int k = 0; k < RPT; ++k) valid[k] = FULL || (tid + k * NT) < m;
  double* fcur = p.f0;
  double* fnext = p.f1;
  unsigned robust_seen = 0;
  int hist = 1;  // history row the next row merge writes (iteration + 1)

  // ---------------------------------------------------------------- helpers
  auto load_f = [&](const double* src, double scale) {
#pragma unroll
    for (int k = 0; k < RPT; ++k) fr[k] = valid[k] ? __ldcg(src + tid + k * NT) * scale : 0.0;
  };

  // Robust row soft-min partials of R/eps = (C - f - g)/eps over this CTA's
  // columns: running (min, sum) per row, one exponential per element; fr holds f/eps.
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
        const double gj = cg[jb - ring.c0 + c] * inv_eps;
        const double* col = buf + (size_t)c * p.ldc + tid;
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          if (valid[k]) {
            const double x = fma(col[k * NT], inv_eps, -(fr[k] + gj));
            const double d = x - rm[k];
            const double e = exp_tbl<kExpTableSpread>(-fabs(d), tbl_l);
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
      if (valid[k]) {
        const int i = tid + k * NT;
        p.rowpm[(size_t)cta * m + i] = rm[k];
        p.rowp[(size_t)cta * m + i] = rs[k];
      }
    }
    return true;
  };

  // Row merge over all CTAs for rows [r0, r1).  robust: partials are
  // (min, sum) pairs of R/eps; otherwise plain sums of the plan.  Writes
  // fnext and the CTA's squared row error into part[cta][0].
  auto row_merge = [&](bool robust) {
    double errr = 0.0;
    for (int rb = r0; rb < r1; rb += 32) {
      const int i = rb + lane;
      const bool vi = i < r1;
      double Rrow = 0.0;
      if (robust) {
        double mn = INFINITY;
        if (vi)
          for (int q2 = w; q2 < G; q2 += 4 * NW) {
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
              v[u] = (q2 + u * NW < G) ? __ldcg(p.rowpm + (size_t)(q2 + u * NW) * m + i) : INFINITY;
#pragma unroll
            for (int u = 0; u < 4; ++u) mn = fmin(mn, v[u]);
          }
        red3[w * 32 + lane] = mn;
        __syncthreads();
        mn = INFINITY;
        for (int ww = 0; ww < NW; ++ww) mn = fmin(mn, red3[ww * 32 + lane]);
        __syncthreads();
        double acc = 0.0;
        if (vi)
          for (int q2 = w; q2 < G; q2 += NW) {
            const double mp = __ldcg(p.rowpm + (size_t)q2 * m + i);
            if (mp < INFINITY) acc += __ldcg(p.rowp + (size_t)q2 * m + i) * exp(-(mp - mn));
          }
        red3[w * 32 + lane] = acc;
        __syncthreads();
        double tot = 0.0;
        for (int ww = 0; ww < NW; ++ww) tot += red3[ww * 32 + lane];
        Rrow = eps * (mn - log(tot));
      } else {
        double acc = 0.0;
        if (vi) acc = sum_partials<NW>(p.rowp, i, m, G, w);
        red3[w * 32 + lane] = acc;
        __syncthreads();
        double tot = 0.0;
        for (int ww = 0; ww < NW; ++ww) tot += red3[ww * 32 + lane];
        if (w == 0 && vi && !(tot >= 1e-250 && tot <= 1e250)) atomicAdd(p.ctrl + 3, 1u);
        Rrow = -eps * log(tot);
      }
      if (w == 0 && vi) {
        const double la = p.loga[i], ela = p.eloga[i], fc = __ldcg(fcur + i);
        const double d = -Rrow * inv_eps - la;
        errr += d * d;
        const double fn = fc + (ela + Rrow);
        fnext[i] = fn;
        if (p.fh) p.fh[(size_t)hist * m + i] = fn;
      }
      __syncthreads();
    }
    if (w == 0) {
      errr = warp_sum(errr);
      if (lane == 0) p.part[(size_t)cta * 8 + 0] = errr;
    }
  };

  // Deterministic sums of part[*][k0] and part[*][k1] over CTAs (same order
  // in every CTA).
  auto total2 = [&](int k0, int k1, double& t0, double& t1) {
    if (w == 0) {
      double a0 = 0.0, a1 = 0.0;
      for (int q2 = lane; q2 < G; q2 += 64) {
        const bool h = q2 + 32 < G;
        const double x0 = __ldcg(p.part + (size_t)q2 * 8 + k0), x1 = __ldcg(p.part + (size_t)q2 * 8 + k1);
        const double y0 = h ? __ldcg(p.part + (size_t)(q2 + 32) * 8 + k0) : 0.0;
        const double y1 = h ? __ldcg(p.part + (size_t)(q2 + 32) * 8 + k1) : 0.0;
        a0 += x0 + y0;
        a1 += x1 + y1;
      }
      a0 = warp_sum(a0);
      a1 = warp_sum(a1);
      if (lane == 0) {
        s_scalar[0] = a0;
        s_scalar[1] = a1;
      }
    }
    __syncthreads();
    t0 = s_scalar[0];
    t1 = s_scalar[1];
    __syncthreads();
  };

  // -------------------------------------------------------------- init
  int iter = p.resume ? p.iter0 : 0;
  double err = p.resume ? p.err0 : 1000.0;
  if (!p.resume && p.max_iter > 0) {
    load_f(fcur, inv_eps);  // zeros
    ok = robust_row_sweep();
    ok = gsync() && ok;
    if (ok) {
      row_merge(true);
      ok = gsync();
    }
    { double* t = fcur; fcur = fnext; fnext = t; }
  }

  // -------------------------------------------------------------- iterations
  // Column pass in units of 1/eps: y_ij = C_ij/eps - f_i/eps, shift mu_j,
  // e_ij = exp(mu_j - y_ij), s_j = sum_i e_ij, softmin_i(C_ij - f_i) = eps (mu_j - log s_j).
  while (ok && iter < p.max_iter && err >= p.tol) {
    ++iter;
    load_f(fcur, inv_eps);
    double r[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) r[k] = 0.0;
    double errc = 0.0;
    const bool first = (iter == (p.resume ? p.iter0 : 0) + 1);

    for (int s = 0; s < ring.nst && ok; ++s) {
      const unsigned seq = ring.q;
      if (!ring.wait(seq)) {
        flag_error(p.ctrl, KERR_MBAR_TIMEOUT);
        ok = false;
        break;
      }
      const double* buf = ring.slot(seq) + tid;
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
              for (int k = 0; k < RPT; ++k)
                if (valid[k]) lm = fmin(lm, fma(buf[(size_t)c * p.ldc + k * NT], inv_eps, -fr[k]));
            }
            mu[c] = lm;
          }
          block_min_cols<CW, NW>(mu, red, par);
        } else {
#pragma unroll
          for (int c = 0; c < CW; ++c) mu[c] = (c < nc) ? cmu[jb - ring.c0 + c] : 0.0;
        }
#pragma unroll
        for (int c = 0; c < CW; ++c) {
          sum[c] = 0.0;
          if (c < nc) {
            const double* col = buf + (size_t)c * p.ldc;
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
              double ev = 0.0;
              if (valid[k]) ev = exp_tbl<kExpTableSpread>(fma(col[k * NT], -inv_eps, mu[c] + fr[k]), tbl_l);
              e[k][c] = ev;
              sum[c] += ev;
            }
          } else {
#pragma unroll
            for (int k = 0; k < RPT; ++k) e[k][c] = 0.0;
          }
        }
        block_sum_cols<CW, NW>(sum, red, par);
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

      // lane c of every warp owns column jb + c: b_j / s_j, and (warp 0) the
      // column update; the ratio is shared across the warp by shuffles
      double mine_s = 0.0, mine_mu = 0.0;
#pragma unroll
      for (int c = 0; c < CW; ++c)
        if (c == lane) {
          mine_s = sum[c];
          mine_mu = mu[c];
        }
      const bool owner = lane < nc;
      const int jl = jb - ring.c0 + lane;  // local column index
      const double beta_l = owner ? cb[jl] * rcp_nr(mine_s) : 0.0;
      double beta[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) beta[c] = __shfl_sync(0xffffffffu, beta_l, c);
      if (w == 0 && owner) {
        cmu[jl] = mine_mu;  // shift used by this sweep
        csum[jl] = mine_s;
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < CW; ++c) acc = fma(e[k][c], beta[c], acc);
        r[k] += acc;
      }
    }
    if (!ok) break;
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (valid[k]) p.rowp[(size_t)cta * m + tid + k * NT] = r[k];
    // column updates of the whole strip, off the per-stage critical path
    __syncthreads();
    if (w == 0) {
      for (int c = lane; c < ring.c1 - ring.c0; c += 32) {
        const double sm = cmu[c] - log(csum[c]);  // softmin_i(C_ij - f_i) / eps
        const double gj = cg[c];
        const double rmin = eps * sm - gj;        // mincol(R(f, g))_j
        const double gn = gj + (celogb[c] + rmin);
        cg[c] = gn;
        cmu[c] = sm;
        if (p.gh) p.gh[(size_t)iter * p.n + ring.c0 + c] = gn;
        const double d = -(eps * sm - gn) * inv_eps - clogb[c];
        errc += d * d;
      }
    }
    if (w == 0) {
      errc = warp_sum(errc);
      if (lane == 0) p.part[(size_t)cta * 8 + 1] = errc;
    }
    if (!gsync()) { ok = false; break; }
    hist = iter + 1;
    row_merge(false);
    if (!gsync()) { ok = false; break; }
    const unsigned rob = *(volatile unsigned*)(p.ctrl + 3);
    if (rob != robust_seen) {
      // some merged row sum left the safe range: redo the row soft-min with
      // the reference's per-row minimum shift, with g already updated
      robust_seen = rob;
      if (!robust_row_sweep()) { ok = false; break; }
      if (!gsync()) { ok = false; break; }
      row_merge(true);
      if (!gsync()) { ok = false; break; }
    }
    double er, ec;
    total2(0, 1, er, ec);
    err = sqrt(er) + sqrt(ec);
    if (iter < p.max_iter && err >= p.tol) {
      double* t = fcur;
      fcur = fnext;
      fnext = t;
      if (p.iter_cap > 0 && iter - (p.resume ? p.iter0 : 0) >= p.iter_cap) break;  // hand-off
    }
  }
  const bool finished = !(iter < p.max_iter && err >= p.tol);

  // state for a resumed run: fcur and this CTA's columns of g
  if (ok && p.f_state) {
    for (int c = tid; c < ring.c1 - ring.c0; c += NT) p.g_state[ring.c0 + c] = cg[c];
    for (int i = r0 + tid; i < r1; i += NT) p.f_state[i] = __ldcg(fcur + i);
    if (cta == 0 && tid == 0) {
      p.res[0] = iter;
      p.res[1] = err;
      p.res[8] = finished ? 1.0 : 0.0;
    }
  }

  // -------------------------------------------------------------- final plan, loss, report
  if (ok && finished && p.do_final) {
    load_f(fcur, 1.0);
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
          const double gj = cg[j - ring.c0];
          const long long jf = p.cidx ? p.cidx[j] : j;
#pragma unroll
          for (int k = 0; k < RPT; ++k) {
            if (valid[k]) {
              const int i = tid + k * NT;
              const double cij = buf[(size_t)c * p.ldc + i];
              const double R = (cij - fr[k]) - gj;
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
      block_sum_cols<CW, NW>(cs, red, par);
      if (tid == 0) ring.issue(seq + STAGES);
      ring.q = seq + 1;
      if (w == 0 && lane < nc) {
        double csl = 0.0;
#pragma unroll
        for (int c = 0; c < CW; ++c)
          if (c == lane) csl = cs[c];
        const int j = jb + lane;
        const double d = csl - cb[j - ring.c0];
        c1 += fabs(d);
        c2 += d * d;
        p.g[j] = cg[j - ring.c0];
        if (p.g_out) p.g_out[p.cidx ? p.cidx[j] : j] = cg[j - ring.c0];
      }
    }
    if (ok) {
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (valid[k]) p.rowp[(size_t)cta * m + tid + k * NT] = rr[k];
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
      ok = gsync();
    }
    if (ok) {
      double a1 = 0.0, a2 = 0.0;
      for (int rb = r0; rb < r1; rb += 32) {
        const int i = rb + lane;
        const bool vi = i < r1;
        double acc = 0.0;
        if (vi) acc = sum_partials<NW>(p.rowp, i, m, G, w);
        red3[w * 32 + lane] = acc;
        __syncthreads();
        if (w == 0 && vi) {
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
      ok = gsync();
    }
    if (ok && cta == 0) {
      double tl1, tl2, tc1, tc2, tr1, tr2;
      total2(2, 3, tl1, tl2);
      total2(4, 5, tc1, tc2);
      total2(6, 7, tr1, tr2);
      if (tid == 0) {
        p.res[0] = iter;
        p.res[1] = err;
        p.res[2] = tl1 + eps * tl2;
        p.res[3] = tr1;
        p.res[4] = tc1;
        p.res[5] = sqrt(tr2);
        p.res[6] = sqrt(tc2);
        p.res[7] = *(volatile unsigned*)(p.ctrl + 3);
        p.res[8] = 1.0;
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

template <int RPT, int CW, int NTT>
int launch(Context* ctx, Params& p, cudaStream_t st, int* launches) {
  auto kern = (p.m == RPT * NTT) ? sinkhorn_log_kernel<RPT, CW, NTT, true> : sinkhorn_log_kernel<RPT, CW, NTT, false>;
  p.ncol_max = (p.n + ctx->sm_count - 1) / ctx->sm_count;
  const size_t smem = smem_bytes<CW, NTT / 32>(p.ldc, p.ncol_max);
  if ((int)smem > ctx->smem_optin)
    return set_error(RWIG_E_UNSUPPORTED, "stage ring and column state exceed shared memory");
  RWIG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NTT, smem));
  if (occ < 1) return set_error(RWIG_E_UNSUPPORTED, "kernel does not fit on an SM");
  const int maxG = occ * ctx->sm_count;
  p.G = std::min(p.G, maxG);  // p.G arrives as the scratch-sized cap
  void* args[] = {&p};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(p.G), dim3(NTT), args, smem, st));
  ++*launches;
  return 0;
}

// Shape choice by rows m: 512 threads, 1, 2, 4, 8 or 16 rows per thread and
// 16, 8, 4, 2 or 1 columns per stage (64 KB stages at the largest m of each).
inline int dispatch_launch(Context* ctx, Params& p, cudaStream_t st, int* launches) {
  const int m = p.m;
  if (m <= 512) return launch<1, 16, 512>(ctx, p, st, launches);
  if (m <= 1024) return launch<2, 8, 512>(ctx, p, st, launches);
  if (m <= 2048) return launch<4, 4, 512>(ctx, p, st, launches);
  if (m <= 4096) return launch<8, 2, 512>(ctx, p, st, launches);
  return launch<16, 1, 512>(ctx, p, st, launches);
}

}  // namespace sklog

// Scratch slot numbers used by the log-Sinkhorn entry points.
enum {
  SL_LOGA = 0, SL_ELOGA, SL_LOGB, SL_ELOGB, SL_F0, SL_F1, SL_G, SL_MU, SL_ROWP, SL_ROWPM, SL_PART,
  SL_CTRL, SL_RES, SL_CRED, SL_AR, SL_BR, SL_RIDX, SL_CIDX, SL_HOST_C, SL_HOST_A, SL_HOST_B,
  SL_HOST_P, SL_HOST_F, SL_HOST_G, SL_FST, SL_GST, SL_FT, SL_GT, SL_KT, SL_U0, SL_U1, SL_FH, SL_GH, SL_HOST_GA
};

// Largest forward history kept for the gradient (f and g of every iteration).
constexpr size_t kMaxHistoryBytes = size_t(32) << 30;

// Core of both log-Sinkhorn entry points: inputs on the device.
__global__ void scatter_kernel(const double* x, const int* idx, int n, double* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[idx ? idx[k] : k] = x[k];
}

// Shared driver of the vanilla and log-stabilised Sinkhorn entry points; inputs
// on the device.  Log: f, g are the dual potentials (-inf off the support).
// Vanilla: f, g receive the scalings u, v (0 off the support).
int sinkhorn_device(Context* ctx, cudaStream_t st, bool vanilla, double* P, double* grad_a, double* f,
                           double* g, double* loss, int* iter, double* err, const double* a,
                           const double* b, const double* C, int M, int N, double reg,
                           int withgrad, int max_iter, double zero_tol) {
  using namespace sklog;
  reset_report();
  if (!a || !b || !C) return set_error(RWIG_E_INVALID, "a, b and C must be non-null");
  if (M < 1 || N < 1) return set_error(RWIG_E_INVALID, "M and N must be >= 1");
  if (!(reg > 0.0) || !std::isfinite(reg)) return set_error(RWIG_E_INVALID, "reg must be finite and > 0");
  const bool want_grad = withgrad && grad_a;
  double grad_ms = 0.0;
  if (want_grad && max_iter < 0) return set_error(RWIG_E_INVALID, "max_iter must be >= 0");
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
  if (m > 8192) return set_error(RWIG_E_UNSUPPORTED, "more than 8192 supported rows");
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
  const int Gmax = std::min(std::min(n, 2 * ctx->sm_count), 320);  // merge loads assume G <= 20 warps' worth
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
  p.res = (double*)scratch(ctx, SL_RES, sizeof(double) * 16);
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
  p.f_out = vanilla ? nullptr : f;
  p.g_out = vanilla ? nullptr : g;
  p.G = Gmax;
  p.do_final = 1;

  // gradient: every iteration's potentials (log) or scalings (vanilla), rows
  // 1..max_iter+1 of f / u and 1..max_iter of g / v
  double* fh = nullptr;
  double* gh = nullptr;
  if (want_grad) {
    if (m > 8192) return set_error(RWIG_E_UNSUPPORTED, "the Sinkhorn gradient supports up to 8192 rows of support");
    const size_t hb_f = sizeof(double) * ((size_t)max_iter + 2) * m, hb_g = sizeof(double) * ((size_t)max_iter + 1) * n;
    if (hb_f + hb_g > kMaxHistoryBytes)
      return set_error(RWIG_E_UNSUPPORTED, "the gradient's iteration history (max_iter x (M + N)) exceeds 32 GiB");
    fh = (double*)scratch(ctx, SL_FH, hb_f);
    gh = (double*)scratch(ctx, SL_GH, hb_g);
    if (!fh || !gh) return RWIG_E_NOMEM;
    if (!vanilla) {
      p.fh = fh;
      p.gh = gh;
    }
  }

  prep_kernel<<<std::max(1, (std::max(m, n) + 255) / 256), 256, 0, st>>>(
      ar, br, m, n, reg, loga, eloga, logb, elogb, p.f0, p.g, p.mu, p.ctrl);
  ++launches;
  if (reduced) {
    if (P) {
      RWIG_CUDA_TRY(cudaMemsetAsync(P, 0, sizeof(double) * (size_t)M * N, st));
    }
    const double off = vanilla ? 0.0 : -INFINITY;  // sinkhorn_impl_vanilla.cpp:59-62, _log.cpp:267-268
    if (f && m < M) {
      fill_kernel<<<(M + 255) / 256, 256, 0, st>>>(f, M, off);
      ++launches;
    }
    if (g && n < N) {
      fill_kernel<<<(N + 255) / 256, 256, 0, st>>>(g, N, off);
      ++launches;
    }
  }

  double res[16];
  unsigned ctrl[4];
  int fallbacks = 0;
  double sweep_ms = 0.0;
  int sweep_iters = 0;
  // Runs one cooperative launch of `launch_fn` and reads back its results.
  auto run = [&](auto&& launch_fn) -> int {
    RWIG_CUDA_TRY(cudaMemsetAsync(p.ctrl, 0, sizeof(unsigned) * 4, st));
    int r = launch_fn();
    if (r != 0) return r;
    RWIG_CUDA_TRY(cudaGetLastError());
    ++launches;
    RWIG_CUDA_TRY(cudaMemcpyAsync(res, p.res, sizeof(res), cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaMemcpyAsync(ctrl, p.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaStreamSynchronize(st));
    if (ctrl[2] != 0u) {
      char buf[160];
      std::snprintf(buf, sizeof(buf), "log-Sinkhorn kernel stopped by a bounded wait (error bits 0x%x)", ctrl[2]);
      return set_error(RWIG_E_TIMEOUT, buf);
    }
    fallbacks += (int)ctrl[3];
    return 0;
  };
  auto log_launch = [&]() { int dummy = 0; return dispatch_launch(ctx, p, st, &dummy); };

  RWIG_CUDA_TRY(cudaEventRecord(ctx->evk, st));
  int rc = 0;
  // the gradient replays the log-domain iterations, so its forward runs there
  const bool scaled = option("log_sinkhorn.scaled", 1.0) != 0.0 && max_iter > 1 && !want_grad;
  if (vanilla) {
    // K = exp(-C/eps) (sinkhorn_impl_vanilla.cpp:41); u = a / (K 1), then the
    // scaled sweeps; P, loss and marginals from C with f = eps log u, g = eps log v
    double* fst = (double*)scratch(ctx, SL_FST, sizeof(double) * m);
    double* gst = (double*)scratch(ctx, SL_GST, sizeof(double) * n);
    double* Kt = (double*)scratch(ctx, SL_KT, sizeof(double) * ldc * n);
    double* u0 = (double*)scratch(ctx, SL_U0, sizeof(double) * m);
    double* u1 = (double*)scratch(ctx, SL_U1, sizeof(double) * m);
    if (!fst || !gst || !Kt || !u0 || !u1) return RWIG_E_NOMEM;
    rc = launch_absorb(ctx, Cr, ldc, p.f0, p.g, m, n, 1.0 / reg, Kt, st);  // f0, g are zero here
    if (rc != 0) return rc;
    ++launches;
    int it_now = 0;
    double err_now = 1000.0;
    if (max_iter > 0) {
      rc = launch_fill_ones(ctx, u0, m, st);
      if (rc != 0) return rc;
      ++launches;
      ScaledParams sp{};
      sp.K = Kt;
      sp.ldk = ldc;
      sp.a = ar;
      sp.b = br;
      sp.loga = loga;
      sp.logb = logb;
      sp.m = m;
      sp.n = n;
      sp.G = Gmax;
      sp.eps = reg;
      sp.inv_eps = 1.0 / reg;
      sp.tol = zero_tol;
      sp.tau = INFINITY;
      sp.iter0 = 0;
      sp.max_iter = max_iter;
      sp.err0 = 1000.0;
      sp.u0 = u0;
      sp.u1 = u1;
      sp.ft = p.f0;
      sp.gt = p.g;
      sp.rowp = p.rowp;
      sp.part = p.part;
      sp.ctrl = p.ctrl;
      sp.res = p.res;
      sp.f_state = fst;
      sp.g_state = gst;
      sp.l2_hot_fraction = option("log_sinkhorn.l2_hot", 0.0);
      sp.vanilla_init = 1;
      sp.uh = fh;
      sp.vh = gh;
      RWIG_CUDA_TRY(cudaEventRecord(ctx->evs0, st));
      rc = run([&]() {
        int r = launch_scaled(ctx, sp, st, true);
        if (r == 0) r = cudaEventRecord(ctx->evs1, st) == cudaSuccess ? 0 : RWIG_E_CUDA;
        return r;
      });
      if (rc != 0) return rc;
      float sms = 0.f;
      cudaEventElapsedTime(&sms, ctx->evs0, ctx->evs1);
      sweep_ms += sms;
      sweep_iters += (int)res[0];
      it_now = (int)res[0];
      err_now = res[1];
    } else {
      // no iteration: u = v = 1 (sinkhorn_impl_vanilla.cpp:96-97)
      rc = launch_fill_ones(ctx, fst, m, st);
      if (rc == 0) rc = launch_fill_ones(ctx, gst, n, st);
      if (rc != 0) return rc;
      launches += 2;
    }
    if (f) {
      scatter_kernel<<<std::max(1, (m + 255) / 256), 256, 0, st>>>(fst, d_ridx, m, f);
      ++launches;
    }
    if (g) {
      scatter_kernel<<<std::max(1, (n + 255) / 256), 256, 0, st>>>(gst, d_cidx, n, g);
      ++launches;
    }
    rc = launch_uv_to_potentials(ctx, fst, gst, m, n, reg, fst, gst, st);
    if (rc != 0) return rc;
    ++launches;
    RWIG_CUDA_TRY(cudaMemcpyAsync(p.f0, fst, sizeof(double) * m, cudaMemcpyDeviceToDevice, st));
    p.f_state = fst;
    p.g_state = gst;
    p.resume = 1;
    p.iter0 = it_now;
    p.err0 = err_now;
    p.max_iter = it_now;
    p.iter_cap = 0;
    rc = run(log_launch);
    if (rc != 0) return rc;
    res[0] = it_now;
    res[1] = err_now;
  } else if (!scaled) {
    // every iteration in the log domain, one launch
    rc = run(log_launch);
    if (rc != 0) return rc;
  } else {
    // first iteration in the log domain (robust start), then the scaled form
    // with absorptions; the plan / loss pass reads C with the final f, g
    double* fst = (double*)scratch(ctx, SL_FST, sizeof(double) * m);
    double* gst = (double*)scratch(ctx, SL_GST, sizeof(double) * n);
    double* ft = (double*)scratch(ctx, SL_FT, sizeof(double) * m);
    double* gt = (double*)scratch(ctx, SL_GT, sizeof(double) * n);
    double* Kt = (double*)scratch(ctx, SL_KT, sizeof(double) * ldc * n);
    double* u0 = (double*)scratch(ctx, SL_U0, sizeof(double) * m);
    double* u1 = (double*)scratch(ctx, SL_U1, sizeof(double) * m);
    if (!fst || !gst || !ft || !gt || !Kt || !u0 || !u1) return RWIG_E_NOMEM;
    p.f_state = fst;
    p.g_state = gst;
    p.iter_cap = 1;
    rc = run(log_launch);
    if (rc != 0) return rc;
    int it_now = (int)res[0];
    double err_now = res[1];
    bool finished = res[8] != 0.0;
    bool final_done = finished;
    const double tau = option("log_sinkhorn.tau", 100.0);
    while (!finished) {
      RWIG_CUDA_TRY(cudaMemcpyAsync(ft, fst, sizeof(double) * m, cudaMemcpyDeviceToDevice, st));
      RWIG_CUDA_TRY(cudaMemcpyAsync(gt, gst, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      rc = launch_absorb(ctx, Cr, ldc, ft, gt, m, n, 1.0 / reg, Kt, st);
      if (rc != 0) return rc;
      rc = launch_fill_ones(ctx, u0, m, st);
      if (rc != 0) return rc;
      launches += 2;
      ScaledParams sp{};
      sp.K = Kt;
      sp.ldk = ldc;
      sp.a = ar;
      sp.b = br;
      sp.loga = loga;
      sp.logb = logb;
      sp.m = m;
      sp.n = n;
      sp.G = Gmax;
      sp.eps = reg;
      sp.inv_eps = 1.0 / reg;
      sp.tol = zero_tol;
      sp.tau = tau;
      sp.iter0 = it_now;
      sp.max_iter = max_iter;
      sp.err0 = err_now;
      sp.u0 = u0;
      sp.u1 = u1;
      sp.ft = ft;
      sp.gt = gt;
      sp.rowp = p.rowp;
      sp.part = p.part;
      sp.ctrl = p.ctrl;
      sp.res = p.res;
      sp.f_state = fst;
      sp.g_state = gst;
      sp.l2_hot_fraction = option("log_sinkhorn.l2_hot", 0.0);
      RWIG_CUDA_TRY(cudaEventRecord(ctx->evs0, st));
      rc = run([&]() {
        int r = launch_scaled(ctx, sp, st, false);
        if (r == 0) r = cudaEventRecord(ctx->evs1, st) == cudaSuccess ? 0 : RWIG_E_CUDA;
        return r;
      });
      if (rc != 0) return rc;
      {
        float sms = 0.f;
        cudaEventElapsedTime(&sms, ctx->evs0, ctx->evs1);
        sweep_ms += sms;
        sweep_iters += (int)res[0] - sp.iter0;
      }
      it_now = (int)res[0];
      err_now = res[1];
      const int stt = (int)res[2];
      if (stt == kScaledFinished) {
        finished = true;
      } else if (stt == kScaledUnsafe) {
        // the rest of the solve in the log domain, from the state handed back
        ++fallbacks;
        RWIG_CUDA_TRY(cudaMemcpyAsync(p.f0, fst, sizeof(double) * m, cudaMemcpyDeviceToDevice, st));
        p.resume = 1;
        p.iter0 = it_now;
        p.err0 = err_now;
        p.iter_cap = 0;
        rc = run(log_launch);
        if (rc != 0) return rc;
        finished = final_done = true;
      }
    }
    if (!final_done) {
      // plan, loss and marginals from C with the final f, g (no iterations)
      RWIG_CUDA_TRY(cudaMemcpyAsync(p.f0, fst, sizeof(double) * m, cudaMemcpyDeviceToDevice, st));
      p.resume = 1;
      p.iter0 = it_now;
      p.err0 = err_now;
      p.max_iter = it_now;
      p.iter_cap = 0;
      rc = run(log_launch);
      if (rc != 0) return rc;
    }
  }
  if (want_grad) {
    // vanilla: K = exp(-C/eps) is the kernel the scalings were computed on
    const double* Kv = vanilla ? (const double*)scratch(ctx, SL_KT, sizeof(double) * ldc * n) : nullptr;
    RWIG_CUDA_TRY(cudaEventRecord(ctx->evs0, st));
    rc = sinkhorn_grad(ctx, st, vanilla, Cr, Kv, ldc, ar, br, loga, logb, fh, gh, m, n, (int)res[0], reg, d_ridx, M,
                       vanilla ? 1.0 : reg, grad_a, &launches);
    if (rc != 0) return rc;
    RWIG_CUDA_TRY(cudaEventRecord(ctx->evs1, st));
    RWIG_CUDA_TRY(cudaEventSynchronize(ctx->evs1));
    float gms = 0.f;
    cudaEventElapsedTime(&gms, ctx->evs0, ctx->evs1);
    grad_ms = gms;
  }
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  RWIG_CUDA_TRY(cudaEventSynchronize(ctx->ev1));
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
  R.sweep_ms = sweep_ms;
  R.sweep_iters = sweep_iters;
  R.fallback_events = fallbacks;
  R.kernel_launches = launches;
  R.support_m = m;
  R.support_n = n;
  R.grad_ms = grad_ms;
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
  cudaStream_t st = call_stream(ctx, stream);
  return sinkhorn_device(ctx, st, false, P, grad_a, f, g, loss, iter, err, a, b, C, M, N, reg, withgrad,
                         max_iter, zero_tol);
}

extern "C" int rwig_sinkhorn_vanilla_dev(double* P, double* grad_a, double* u, double* v, double* loss,
                                         int* iter, double* err, const double* a, const double* b,
                                         const double* C, int M, int N, double reg, int withgrad,
                                         int max_iter, double zero_tol, void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = call_stream(ctx, stream);
  return sinkhorn_device(ctx, st, true, P, grad_a, u, v, loss, iter, err, a, b, C, M, N, reg, withgrad,
                         max_iter, zero_tol);
}

static int sinkhorn_host(bool vanilla, double* P, double* grad_a, double* f, double* g, double* loss,
                         int* iter, double* err, const double* a, const double* b, const double* C, int M,
                         int N, double reg, int withgrad, int max_iter, double zero_tol) {
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
  const bool want_grad = withgrad && grad_a;
  double* dga = want_grad ? (double*)scratch(ctx, SL_HOST_GA, sizeof(double) * M) : nullptr;
  if (!dC || !da || !db || (P && !dP) || (f && !df) || (g && !dg) || (want_grad && !dga)) return RWIG_E_NOMEM;
  RWIG_CUDA_TRY(cudaMemcpyAsync(dC, C, sizeof(double) * MN, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(da, a, sizeof(double) * M, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(db, b, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  int rc = sinkhorn_device(ctx, st, vanilla, dP, dga, df, dg, loss, iter, err, da, db, dC, M, N, reg,
                           withgrad, max_iter, zero_tol);
  if (rc < 0) return rc;
  if (want_grad) RWIG_CUDA_TRY(cudaMemcpyAsync(grad_a, dga, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
  if (P) RWIG_CUDA_TRY(cudaMemcpyAsync(P, dP, sizeof(double) * MN, cudaMemcpyDeviceToHost, st));
  if (f) RWIG_CUDA_TRY(cudaMemcpyAsync(f, df, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
  if (g) RWIG_CUDA_TRY(cudaMemcpyAsync(g, dg, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  return rc;
}

extern "C" int rwig_sinkhorn_log(double* P, double* grad_a, double* f, double* g, double* loss,
                                 int* iter, double* err, const double* a, const double* b,
                                 const double* C, int M, int N, double reg, int withgrad,
                                 int max_iter, double zero_tol) {
  return sinkhorn_host(false, P, grad_a, f, g, loss, iter, err, a, b, C, M, N, reg, withgrad, max_iter,
                       zero_tol);
}

extern "C" int rwig_sinkhorn_vanilla(double* P, double* grad_a, double* u, double* v, double* loss,
                                     int* iter, double* err, const double* a, const double* b,
                                     const double* C, int M, int N, double reg, int withgrad,
                                     int max_iter, double zero_tol) {
  return sinkhorn_host(true, P, grad_a, u, v, loss, iter, err, a, b, C, M, N, reg, withgrad, max_iter,
                       zero_tol);
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
constexpr size_t kOffCtrl = kOffRes + 16;  // 8 unsigned words = 4 doubles
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

template <int RPT, int CW, int NTT>
int launch_noalloc(sklog::Params& p, int sms, int smem_optin, cudaStream_t st) {
  using namespace sklog;
  auto kern = (p.m == RPT * NTT) ? sinkhorn_log_kernel<RPT, CW, NTT, true> : sinkhorn_log_kernel<RPT, CW, NTT, false>;
  p.ncol_max = (p.n + std::min(sms, kMaxCtas) - 1) / std::min(sms, kMaxCtas);
  const size_t smem = smem_bytes<CW, NTT / 32>(p.ldc, p.ncol_max);
  if ((int)smem > smem_optin)
    return set_error(RWIG_E_UNSUPPORTED, "stage ring and column state exceed shared memory");
  RWIG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NTT, smem));
  if (occ < 1) return set_error(RWIG_E_UNSUPPORTED, "kernel does not fit on an SM");
  p.G = std::min(std::min(p.n, occ * sms), kMaxCtas);
  void* args[] = {&p};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(p.G), dim3(NTT), args, smem, st));
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
  if (max_iter < 0) return set_error(RWIG_E_INVALID, "max_iter must be >= 0");
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
  p.do_final = 1;

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

  if (M <= 512) rc = launch_noalloc<1, 16, 512>(p, sms, smem_optin, st);
  else if (M <= 1024) rc = launch_noalloc<2, 8, 512>(p, sms, smem_optin, st);
  else if (M <= 2048) rc = launch_noalloc<4, 4, 512>(p, sms, smem_optin, st);
  else rc = launch_noalloc<8, 2, 512>(p, sms, smem_optin, st);
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
