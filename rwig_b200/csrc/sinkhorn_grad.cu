// sinkhorn_grad.cu -- the unrolled gradient of the Sinkhorn loss w.r.t. a:
// Sinkhorn::_bwd_log (src/sinkhorn_impl_log.cpp:379-520) and _bwd_vanilla
// (src/sinkhorn_impl_vanilla.cpp:169-213), on the (support-reduced) problem,
// from the per-iteration history the forward recorded.
//
// Log (potentials f_l, g_l, l = 0..L, f_{L+1}):
//   l = L:  gbar = colsum(PbarP)/eps,  PbarP = (C + eps log P) o P (:383, :414)
//   l < L:  gbar = -X^T fbar with X = row-softmax(-R(f_l, g_l)/eps) (:418-454)
//   fbar = -W gbar (+ rowsum(PbarP)/eps at l = L), W = col-softmax(-R(f_l, g_l)/eps) (:458-488)
//   grad_a += fbar / a (:513);  grad_a *= eps at the end (:515).
// The soft-min normalisers come from the forward's own updates: the row
// soft-min at (f_l, g_l) is f_{l+1} - f_l - eps log a (the f update, :336), so
// X_ij = exp((f_{l+1,i} + g_{l,j} - C_ij)/eps - log a_i); the column soft-min
// at (f_l, g_l) is -eps log b (g has just been updated to it, :349), so
// W_ij = exp((f_{l,i} + g_{l,j} - C_ij)/eps - log b_j).  Both exponents are
// <= 0 up to rounding, as in the reference's shifted sweeps.
//
// Vanilla (scalings u_l, v_l, K = exp(-C/eps)):
//   l = L:  vbar = PbarK^T u,  ubar = PbarK v - K((vbar o v)/(K^T u)),  PbarK = (C + eps log P) o K
//   l < L:  vbar = -K^T((ubar o u_{l+1})/(K v_l)),  ubar = -K((vbar o v_l)/(K^T u_l))
//   grad_a += ubar / (K v_{l-1})
// with K v_l = a / u_{l+1} and K^T u_l = b / v_l (the forward's updates).
//
// One cooperative launch runs all L steps: each CTA owns a strip of columns
// with every row; per step one pass over C (and K) gives the strip's column
// sums and row partials, a bounded grid barrier, a fixed-order merge of the
// row partials over the CTAs, another barrier.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "fastexp.cuh"
#include "sk_common.cuh"
#include "sk_host.h"

namespace rwig {
namespace skgrad {

using sk::block_sum_cols;
using sk::sum_partials;

constexpr int NTT = 512, NW = NTT / 32;

struct Params {
  const double* C;   // m x n, leading dimension ldc
  const double* K;   // vanilla: exp(-C/eps), same layout
  long long ldc;
  const double* a;
  const double* b;
  const double* loga;
  const double* logb;
  const double* fh;  // log: f_l at fh[l*m] (l = 0..L+1); vanilla: u_l
  const double* gh;  // log: g_l at gh[l*n] (l = 0..L); vanilla: v_l
  double* rowp;      // [G][m]
  double* rowp2;     // [G][m] (log, step L: row sums of PbarP)
  double* xbar;      // m: fbar (log) or (ubar o u_l^2)/a (vanilla) of the last step
  double* ga;        // m: the gradient being accumulated
  unsigned* ctrl;    // [0] barrier count, [2] error bits
  int m, n, G, L;
  double eps;
};

template <int RPT, int CW, bool VAN>
__global__ void __launch_bounds__(NTT, 1) grad_kernel(Params p) {
  extern __shared__ __align__(16) double red[];  // [2][NW][max(CW, 32)], then the 2^(j/64) table
  double* tbl = red + 2 * NW * (CW > 32 ? CW : 32);
  load_exp_table_spread(tbl);
  __syncthreads();
  const double* tbl_l = tbl + (threadIdx.x & (kExpTableSpread - 1));
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, cta = blockIdx.x, G = p.G;
  const int m = p.m, n = p.n;
  const double eps = p.eps, inv_eps = 1.0 / eps;
  const int c0 = (int)(((long long)cta * n) / G), c1 = (int)(((long long)(cta + 1) * n) / G);
  const int r0 = (int)(((long long)cta * m) / G), r1 = (int)(((long long)(cta + 1) * m) / G);
  int par = 0;
  unsigned nbar = 0;
  auto gsync = [&]() -> bool { ++nbar; return grid_sync(p.ctrl, p.ctrl + 2, nbar * (unsigned)G); };
  bool valid[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) valid[t] = tid + t * NTT < m;

  for (int l = p.L; l >= 1; --l) {
    const bool last = (l == p.L);
    // ---- per-row inputs of this step
    double ra[RPT], rb[RPT], rx[RPT], r[RPT], s[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
      const int i = tid + t * NTT;
      r[t] = 0.0;
      s[t] = 0.0;
      if (!valid[t]) {
        ra[t] = rb[t] = rx[t] = 0.0;
        continue;
      }
      if (!VAN) {
        rb[t] = p.fh[(size_t)l * m + i];                                          // f_l
        ra[t] = last ? rb[t] : p.fh[(size_t)(l + 1) * m + i] - eps * p.loga[i];  // X's row term
        rx[t] = last ? 0.0 : __ldcg(p.xbar + i);                                 // fbar
      } else {
        rb[t] = p.fh[(size_t)l * m + i];                 // u_l
        rx[t] = last ? rb[t] : __ldcg(p.xbar + i);       // u_L (step L) or (ubar o u_{l+1}^2)/a
      }
    }
    // ---- column pass over the strip
    for (int jb = c0; jb < c1; jb += CW) {
      const int nc = min(CW, c1 - jb);
      double cs[CW], gl[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) {
        cs[c] = 0.0;
        gl[c] = c < nc ? p.gh[(size_t)l * n + jb + c] : 0.0;  // g_l (log) or v_l (vanilla)
      }
      double cij[RPT][CW], kij[VAN ? RPT : 1][VAN ? CW : 1];
#pragma unroll
      for (int c = 0; c < CW; ++c)
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
          const bool in = c < nc && valid[t];
          const size_t o = (size_t)(jb + c) * p.ldc + tid + t * NTT;
          cij[t][c] = in ? p.C[o] : 0.0;
          if (VAN) kij[VAN ? t : 0][VAN ? c : 0] = in ? p.K[o] : 0.0;
        }
      // column sums
#pragma unroll
      for (int c = 0; c < CW; ++c)
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
          if (!(c < nc && valid[t])) continue;
          double term;
          if (!VAN) {
            if (last) {
              const double P = exp(((rb[t] + gl[c]) - cij[t][c]) * inv_eps);  // exp(-R/eps) (:266)
              const double pb = (cij[t][c] + eps * log(P)) * P;               // PbarP (:383)
              s[t] += pb;
              term = pb;
            } else {
              // X_ij fbar_i; the table exponential (within 2 ulp, arguments below
              // -708 give 3e-308, negligible in this sum)
              term = exp_tbl<kExpTableSpread>(((ra[t] + gl[c]) - cij[t][c]) * inv_eps, tbl_l) * rx[t];
            }
          } else {
            if (last) {
              const double P = (rb[t] * kij[VAN ? t : 0][VAN ? c : 0]) * gl[c];                  // u K v (:58)
              const double pbk = (cij[t][c] + eps * log(P)) * kij[VAN ? t : 0][VAN ? c : 0];     // PbarK (:172)
              term = pbk * rb[t];
            } else {
              term = kij[VAN ? t : 0][VAN ? c : 0] * rx[t];
            }
          }
          cs[c] += term;
        }
      block_sum_cols<CW, NW>(cs, red, par);
      // column adjoints and the row partials of this group
#pragma unroll
      for (int c = 0; c < CW; ++c) {
        if (c >= nc) continue;
        const int j = jb + c;
        double col;  // gbar_j (log) or z_j = (vbar_j v_j^2) / b_j (vanilla)
        if (!VAN) col = last ? cs[c] * inv_eps : -cs[c];
        else col = ((last ? cs[c] : -cs[c]) * (gl[c] * gl[c])) / p.b[j];
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
          if (!valid[t]) continue;
          if (!VAN) {
            const double W = exp_tbl<kExpTableSpread>(((rb[t] + gl[c]) - cij[t][c]) * inv_eps - p.logb[j], tbl_l);
            r[t] += W * col;
          } else if (last) {
            const double P = (rb[t] * kij[VAN ? t : 0][VAN ? c : 0]) * gl[c];
            const double pbk = (cij[t][c] + eps * log(P)) * kij[VAN ? t : 0][VAN ? c : 0];
            r[t] += pbk * gl[c] - kij[VAN ? t : 0][VAN ? c : 0] * col;
          } else {
            r[t] += kij[VAN ? t : 0][VAN ? c : 0] * col;
          }
        }
      }
    }
#pragma unroll
    for (int t = 0; t < RPT; ++t)
      if (valid[t]) {
        p.rowp[(size_t)cta * m + tid + t * NTT] = r[t];
        if (last && !VAN) p.rowp2[(size_t)cta * m + tid + t * NTT] = s[t];
      }
    if (!gsync()) return;
    // ---- merge of this CTA's rows, fixed order over the CTAs
    for (int rb0 = r0; rb0 < r1; rb0 += 32) {
      const int i = rb0 + lane;
      const bool vi = i < r1;
      double tot = vi ? sum_partials<NW>(p.rowp, i, m, G, w) : 0.0;
      double tot2 = (vi && last && !VAN) ? sum_partials<NW>(p.rowp2, i, m, G, w) : 0.0;
      red[w * 32 + lane] = tot;
      red[NW * 32 + w * 32 + lane] = tot2;
      __syncthreads();
      if (w == 0 && vi) {
        double T = 0.0, T2 = 0.0;
        for (int q = 0; q < NW; ++q) {
          T += red[q * 32 + lane];
          T2 += red[NW * 32 + q * 32 + lane];
        }
        const double ai = p.a[i];
        if (!VAN) {
          const double fbar = -T + (last ? T2 * inv_eps : 0.0);
          p.ga[i] += fbar / ai;  // :513
          p.xbar[i] = fbar;
        } else {
          const double ul = p.fh[(size_t)l * m + i];
          const double ubar = last ? T : -T;
          p.ga[i] += (ubar * ul) / ai;           // ubar / (K v_{l-1}),  K v_{l-1} = a / u_l
          p.xbar[i] = (ubar * (ul * ul)) / ai;   // (ubar o u_l) / (K v_{l-1}) for step l-1
        }
      }
      __syncthreads();
    }
    if (!gsync()) return;
  }
}

template <int RPT, int CW, bool VAN>
int launch_t(Context* ctx, Params& p, cudaStream_t st) {
  auto kern = grad_kernel<RPT, CW, VAN>;
  const size_t smem = sizeof(double) * (2 * NW * std::max(CW, 32) + 64 * kExpTableSpread);
  int nblk = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nblk, kern, NTT, smem));
  if (nblk < 1) return set_error(RWIG_E_UNSUPPORTED, "gradient kernel does not fit on an SM");
  // every CTA must be resident (grid barrier); the merge sums at most 20 * NW partials
  p.G = std::min(std::min(p.n, ctx->sm_count * nblk), 20 * NW);
  p.rowp = (double*)scratch(ctx, 230, sizeof(double) * (size_t)p.G * p.m);
  p.rowp2 = (double*)scratch(ctx, 231, sizeof(double) * (size_t)p.G * p.m);
  if (!p.rowp || !p.rowp2) return RWIG_E_NOMEM;
  void* args[] = {(void*)&p};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((void*)kern, dim3(p.G), dim3(NTT), args, smem, st));
  return 0;
}

__global__ void scatter_scaled(const double* x, const int* idx, int n, double scale, double* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[idx ? idx[k] : k] = x[k] * scale;
}

}  // namespace skgrad

// Gradient of the reduced problem (m x n, rows ridx of the full M-row problem)
// into grad_a (M entries, zero off the support): the steps L..1 accumulate into
// a reduced buffer, which is scattered times out_scale (eps for the log form,
// src/sinkhorn_impl_log.cpp:515; 1 for vanilla).  fh / gh: the forward's
// history (see skgrad::Params).  Returns 0 or a negative engine error.
int sinkhorn_grad(Context* ctx, cudaStream_t st, bool vanilla, const double* C, const double* K, long long ldc,
                  const double* a, const double* b, const double* loga, const double* logb, const double* fh,
                  const double* gh, int m, int n, int L, double eps, const int* ridx, int M, double out_scale,
                  double* grad_a, int* launches) {
  using namespace skgrad;
  if (m > 8192) return set_error(RWIG_E_UNSUPPORTED, "the Sinkhorn gradient supports up to 8192 rows of support");
  double* ga = (double*)scratch(ctx, 232, sizeof(double) * m);
  double* xbar = (double*)scratch(ctx, 233, sizeof(double) * m);
  unsigned* ctrl = (unsigned*)scratch(ctx, 234, sizeof(unsigned) * 4);
  if (!ga || !xbar || !ctrl) return RWIG_E_NOMEM;
  RWIG_CUDA_TRY(cudaMemsetAsync(ga, 0, sizeof(double) * m, st));
  if (m < M) RWIG_CUDA_TRY(cudaMemsetAsync(grad_a, 0, sizeof(double) * M, st));
  if (L >= 1) {
    RWIG_CUDA_TRY(cudaMemsetAsync(ctrl, 0, sizeof(unsigned) * 4, st));
    Params p{C, K, ldc, a, b, loga, logb, fh, gh, nullptr, nullptr, xbar, ga, ctrl, m, n, 0, L, eps};
    int rc;
    if (vanilla) {
      if (m <= 512) rc = launch_t<1, 16, true>(ctx, p, st);
      else if (m <= 1024) rc = launch_t<2, 8, true>(ctx, p, st);
      else if (m <= 2048) rc = launch_t<4, 4, true>(ctx, p, st);
      else if (m <= 4096) rc = launch_t<8, 2, true>(ctx, p, st);
      else rc = launch_t<16, 1, true>(ctx, p, st);
    } else {
      if (m <= 512) rc = launch_t<1, 16, false>(ctx, p, st);
      else if (m <= 1024) rc = launch_t<2, 8, false>(ctx, p, st);
      else if (m <= 2048) rc = launch_t<4, 4, false>(ctx, p, st);
      else if (m <= 4096) rc = launch_t<8, 2, false>(ctx, p, st);
      else rc = launch_t<16, 1, false>(ctx, p, st);
    }
    if (rc) return rc;
    ++*launches;
  }
  scatter_scaled<<<std::max(1, std::min((m + 255) / 256, 4 * ctx->sm_count)), 256, 0, st>>>(ga, ridx, m, out_scale,
                                                                                           grad_a);
  RWIG_CUDA_TRY(cudaGetLastError());
  ++*launches;
  if (L >= 1) {
    unsigned err = 0;
    RWIG_CUDA_TRY(cudaMemcpyAsync(&err, ctrl + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaStreamSynchronize(st));
    if (err) return set_error(RWIG_E_TIMEOUT, "a bounded wait in the Sinkhorn gradient kernel expired");
  }
  return 0;
}

}  // namespace rwig
