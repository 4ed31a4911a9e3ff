// sinkhorn_scaled.cu -- the log-Sinkhorn iterations in stabilised scaling form.
//
// Same updates as Sinkhorn::_fwd_log (src/sinkhorn_impl_log.cpp:327-375), written
// over an absorbed kernel (B. Schmitzer, "Stabilized sparse scaling algorithms
// for entropy regularized transport problems", SIAM J. Sci. Comput. 41(3), 2019):
//   K~_ij = exp((f~_i + g~_j - C_ij) / eps),  f = f~ + eps log u,  g = g~ + eps log v.
// With these, exp((f_i + g_j - C_ij)/eps) = u_i K~_ij v_j, so one iteration
//   g <- g + eps log b + mincol(R(f, g))   is   v_j = b_j / sum_i K~_ij u_i
//   f <- f + eps log a + minrow(R(f, g))   is   u_i = a_i / sum_j K~_ij v_j
// and the stopping error's row term is log(u_i sum_j K~_ij v_j) - log a_i (the
// column term log(v_j s_j) - log b_j).  Two FMAs per element replace the
// exponential.  When |log u| or |log v| exceeds tau the host absorbs the
// scalings into f~, g~ and rebuilds K~ (absorb_kernel); entries of K~ that
// underflow at absorption are below exp(-708) relative to the dominant terms,
// as in the log domain.  A row sum outside [1e-250, 1e250] hands the solve back
// to the log-domain kernel from the previous iteration's state.
//
// Work split as in the log-domain kernel: CTAs own column strips of K~ streamed
// through the bulk-copy ring, threads own rows, column sums complete inside the
// CTA, row sums merged across CTAs in a fixed order after a bounded grid barrier.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "engine.h"
#include "fastexp.cuh"
#include "sk_common.cuh"
#include "sk_host.h"

namespace rwig {
namespace skscaled {

using sk::block_sum_cols;
using sk::flag_error;
using sk::Ring;
using sk::STAGES;
using sk::sum_partials;

template <int CW, int NW>
__host__ __device__ constexpr size_t smem_bytes(long long ldk, int ncol_max) {
  return (size_t)STAGES * CW * ldk * 8 + STAGES * 8 + (size_t)(2 * NW * CW + NW * 32) * 8 +
         (size_t)6 * ncol_max * 8;
}

// VAN: vanilla Sinkhorn (Sinkhorn::_fwd_vanilla, src/sinkhorn_impl_vanilla.cpp:93-166)
// on K = exp(-C/eps): the same sweeps, an initial pass u = a / (K 1) (:117),
// the stopping error ||u o Kv - a||_2 + ||v o K^T u - b||_2 (:139), no
// absorption; the exit state is u, v themselves.
template <int RPT, int CW, int NTT, bool FULL, bool VAN>
__global__ void __launch_bounds__(NTT, 1) scaled_kernel(ScaledParams p) {
  constexpr int NT = NTT;
  constexpr int NW = NTT / 32;
  extern __shared__ __align__(128) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int cta = blockIdx.x, G = p.G, m = p.m;
  const double eps = p.eps;

  Ring<CW> ring;
  ring.buf = reinterpret_cast<double*>(smem);
  ring.bar = reinterpret_cast<uint64_t*>(smem + (size_t)STAGES * CW * p.ldk * 8);
  double* red = reinterpret_cast<double*>(ring.bar + STAGES);  // [2][NW][CW]
  double* red3 = red + 2 * NW * CW;                            // [NW][32]
  const int NCM = p.ncol_max;
  double* cb = red3 + NW * 32;  // b_j
  double* clogb = cb + NCM;     // log b_j
  double* cgt = clogb + NCM;    // g~_j
  double* cv = cgt + NCM;       // v_j (current)
  double* cvp = cv + NCM;       // v_j of the previous iteration
  double* csum = cvp + NCM;     // s_j = sum_i K~_ij u_i
  __shared__ double s_tot[4];
  ring.C = p.K;
  ring.ldc = p.ldk;
  ring.c0 = (int)(((long long)cta * p.n) / G);
  ring.c1 = (int)(((long long)(cta + 1) * p.n) / G);
  ring.nst = (ring.c1 - ring.c0 + CW - 1) / CW;
  ring.q = 0;
  if (p.l2_hot_fraction >= 0.0) {
    ring.hot_groups = (int)(p.l2_hot_fraction * ring.nst + 0.5);
    ring.pol_hot = l2_policy_evict_last();
    ring.pol_cold = l2_policy_evict_first();
  }
  const int ncols = ring.c1 - ring.c0;
  const int r0 = (int)(((long long)cta * m) / G), r1 = (int)(((long long)(cta + 1) * m) / G);
  int par = 0;

  for (int c = tid; c < ncols; c += NT) {
    const int j = ring.c0 + c;
    cb[c] = p.b[j];
    clogb[c] = p.logb[j];
    cgt[c] = p.gt[j];
    cv[c] = 1.0;
    cvp[c] = 1.0;
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(ring.bar + s, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0 && ring.nst > 0)
    for (int s = 0; s < STAGES; ++s) ring.issue(s);

  bool ok = true;
  unsigned nbar = 0;
  auto gsync = [&]() -> bool { ++nbar; return grid_sync(p.ctrl, p.ctrl + 2, nbar * (unsigned)G); };
  bool valid[RPT];
#pragma unroll
  for (int k = 0; k < RPT; ++k) valid[k] = FULL || (tid + k * NT) < m;

  double* ucur = p.u0;
  double* unext = p.u1;
  int iter = p.iter0;
  double err = p.err0, err_prev = p.err0;
  int status = kScaledRunning;
  bool init = VAN && p.vanilla_init;  // the K 1 pass before the first iteration

  while (ok && (init || (iter < p.max_iter && err >= p.tol))) {
    if (!init) ++iter;
    double u[RPT], r[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      u[k] = valid[k] ? __ldcg(ucur + tid + k * NT) : 0.0;
      r[k] = 0.0;
    }
    // ---- column pass over this CTA's strip of K~
    for (int s = 0; s < ring.nst; ++s) {
      const unsigned seq = ring.q;
      if (!ring.wait(seq)) {
        flag_error(p.ctrl, KERR_MBAR_TIMEOUT);
        ok = false;
        break;
      }
      const double* buf = ring.slot(seq) + tid;
      const int jb = ring.group_begin(seq), nc = ring.group_cols(seq);
      double kv[RPT][CW], sum[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) {
        sum[c] = 0.0;
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          const double x = (c < nc && valid[k]) ? buf[(size_t)c * p.ldk + k * NT] : 0.0;
          kv[k][c] = x;
          sum[c] = fma(x, u[k], sum[c]);
        }
      }
      block_sum_cols<CW, NW>(sum, red, par);
      if (tid == 0) ring.issue(seq + STAGES);
      ring.q = seq + 1;
      double mine_s = 1.0;
#pragma unroll
      for (int c = 0; c < CW; ++c)
        if (c == lane) mine_s = sum[c];
      const bool owner = lane < nc;
      const int jl = jb - ring.c0 + lane;
      // vanilla: v = b / (K^T u) by IEEE division, as the reference
      // (sinkhorn_impl_vanilla.cpp:133), also where K^T u is subnormal or 0
      const double v_l = owner ? (init ? 1.0 : (VAN ? cb[jl] / mine_s : cb[jl] * rcp_nr(mine_s))) : 0.0;
      double v[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) v[c] = __shfl_sync(0xffffffffu, v_l, c);
      if (w == 0 && owner) {
        cvp[jl] = cv[jl];
        cv[jl] = v_l;
        csum[jl] = mine_s;
        if (VAN && p.vh && !init) p.vh[(size_t)iter * p.n + jb + lane] = v_l;
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        double acc = r[k];
#pragma unroll
        for (int c = 0; c < CW; ++c) acc = fma(kv[k][c], v[c], acc);
        r[k] = acc;
      }
    }
    if (!ok) break;
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (valid[k]) p.rowp[(size_t)cta * m + tid + k * NT] = r[k];
    // column error and drift of log v over the strip
    __syncthreads();
    if (w == 0) {
      double errc = 0.0, vmax = 0.0;
      for (int c = lane; c < ncols; c += 32) {
        if (VAN) {
          const double d = cv[c] * csum[c] - cb[c];
          errc += d * d;
        } else {
          const double d = log(cv[c] * csum[c]) - clogb[c];
          errc += d * d;
          vmax = fmax(vmax, fabs(log(cv[c])));
          if (!(csum[c] >= 1e-250 && csum[c] <= 1e250)) vmax = INFINITY;
        }
      }
      errc = warp_sum(errc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
      if (lane == 0) {
        p.part[(size_t)cta * 8 + 1] = errc;
        p.part[(size_t)cta * 8 + 3] = vmax;
      }
    }
    if (!gsync()) { ok = false; break; }
    // ---- row merge for rows [r0, r1)
    {
      double errr = 0.0, umax = 0.0, unsafe = 0.0;
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
          const double ui = __ldcg(ucur + i);
          const double un = p.a[i] / tot;
          unext[i] = un;
          if (VAN && p.uh) p.uh[(size_t)(iter + 1) * m + i] = un;
          if (VAN) {
            const double d = ui * tot - p.a[i];
            errr += d * d;
          } else {
            const double d = log(ui * tot) - p.loga[i];
            errr += d * d;
            umax = fmax(umax, fabs(log(un)));
            if (!(tot >= 1e-250 && tot <= 1e250)) unsafe = 1.0;
          }
        }
        __syncthreads();
      }
      if (w == 0) {
        errr = warp_sum(errr);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          umax = fmax(umax, __shfl_xor_sync(0xffffffffu, umax, o));
          unsafe = fmax(unsafe, __shfl_xor_sync(0xffffffffu, unsafe, o));
        }
        if (lane == 0) {
          p.part[(size_t)cta * 8 + 0] = errr;
          p.part[(size_t)cta * 8 + 2] = umax;
          p.part[(size_t)cta * 8 + 4] = unsafe;
        }
      }
    }
    if (!gsync()) { ok = false; break; }
    // ---- totals, same order in every CTA
    if (w == 0) {
      double e0 = 0.0, e1 = 0.0, mu = 0.0, mv = 0.0, un = 0.0;
      for (int q2 = lane; q2 < G; q2 += 32) {
        const double* pp = p.part + (size_t)q2 * 8;
        e0 += __ldcg(pp + 0);
        e1 += __ldcg(pp + 1);
        mu = fmax(mu, __ldcg(pp + 2));
        mv = fmax(mv, __ldcg(pp + 3));
        un = fmax(un, __ldcg(pp + 4));
      }
      e0 = warp_sum(e0);
      e1 = warp_sum(e1);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        mu = fmax(mu, __shfl_xor_sync(0xffffffffu, mu, o));
        mv = fmax(mv, __shfl_xor_sync(0xffffffffu, mv, o));
        un = fmax(un, __shfl_xor_sync(0xffffffffu, un, o));
      }
      if (lane == 0) {
        s_tot[0] = sqrt(e0) + sqrt(e1);
        s_tot[1] = fmax(mu, mv);
        s_tot[2] = un;
      }
    }
    __syncthreads();
    const double err_t = s_tot[0], drift = s_tot[1], unsafe = s_tot[2];
    __syncthreads();
    if (init) {
      // u = a / (K 1); no iteration counted, no error
      double* t = ucur;
      ucur = unext;
      unext = t;
      init = false;
      continue;
    }
    if (!VAN && (unsafe != 0.0 || !(drift <= 1e300))) {
      // hand back to the log domain from the state before this iteration
      status = kScaledUnsafe;
      --iter;
      err = err_prev;
      break;
    }
    err_prev = err = err_t;
    if (!(iter < p.max_iter && err >= p.tol)) {
      status = kScaledFinished;
      break;
    }
    double* t = ucur;
    ucur = unext;
    unext = t;
    if (!VAN && drift > p.tau) {
      status = kScaledAbsorb;
      break;
    }
  }
  if (ok && status == kScaledRunning) status = kScaledFinished;

  // ---- exit state: f = f~ + eps log u, g = g~ + eps log v (vanilla: u, v)
  if (ok) {
    for (int i = r0 + tid; i < r1; i += NT)
      p.f_state[i] = VAN ? __ldcg(ucur + i) : p.ft[i] + eps * log(__ldcg(ucur + i));
    for (int c = tid; c < ncols; c += NT)
      p.g_state[ring.c0 + c] = VAN ? cv[c] : cgt[c] + eps * log(status == kScaledUnsafe ? cvp[c] : cv[c]);
    if (cta == 0 && tid == 0) {
      p.res[0] = iter;
      p.res[1] = err;
      p.res[2] = status;
    }
  }
  if (tid == 0 && ring.nst > 0) {
    for (unsigned s = 0; s < (unsigned)STAGES; ++s)
      if (!ring.wait(ring.q + s)) flag_error(p.ctrl, KERR_MBAR_TIMEOUT);
  }
}

// K~_ij = exp((f~_i + g~_j - C_ij) / eps) for i < m; padding rows are zero.
__global__ void absorb_kernel(const double* C, long long ldc, const double* ft, const double* gt, int m,
                              int n, double inv_eps, double* K) {
  const long long total = ldc * (long long)n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldc);
    const int j = (int)(k / ldc);
    K[k] = (i < m) ? exp((ft[i] + gt[j] - C[k]) * inv_eps) : 0.0;
  }
}

__global__ void fill_ones(double* x, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] = 1.0;
}

template <int RPT, int CW, int NTT, bool VAN>
int launch_one(Context* ctx, ScaledParams& p, cudaStream_t st) {
  auto kern = (p.m == RPT * NTT) ? scaled_kernel<RPT, CW, NTT, true, VAN> : scaled_kernel<RPT, CW, NTT, false, VAN>;
  p.ncol_max = (p.n + ctx->sm_count - 1) / ctx->sm_count;
  const size_t smem = smem_bytes<CW, NTT / 32>(p.ldk, p.ncol_max);
  if ((int)smem > ctx->smem_optin)
    return set_error(RWIG_E_UNSUPPORTED, "stage ring and column state exceed shared memory");
  RWIG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  RWIG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NTT, smem));
  if (occ < 1) return set_error(RWIG_E_UNSUPPORTED, "kernel does not fit on an SM");
  p.G = std::min(p.G, occ * ctx->sm_count);
  void* args[] = {&p};
  RWIG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)kern, dim3(p.G), dim3(NTT), args, smem, st));
  return 0;
}

}  // namespace skscaled

template <bool VAN>
static int launch_by_rows(Context* ctx, ScaledParams& p, cudaStream_t st) {
  using namespace skscaled;
  const int m = p.m;
  if (m <= 512) return launch_one<1, 16, 512, VAN>(ctx, p, st);
  if (m <= 1024) return launch_one<2, 8, 512, VAN>(ctx, p, st);
  if (m <= 2048) return launch_one<4, 4, 512, VAN>(ctx, p, st);
  if (m <= 4096) return launch_one<8, 2, 512, VAN>(ctx, p, st);
  return launch_one<16, 1, 512, VAN>(ctx, p, st);
}

int launch_scaled(Context* ctx, ScaledParams& p, cudaStream_t st, bool vanilla) {
  return vanilla ? launch_by_rows<true>(ctx, p, st) : launch_by_rows<false>(ctx, p, st);
}

__global__ void uv_to_potentials(const double* u, const double* v, int m, int n, double eps, double* f,
                                 double* g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = t; i < m; i += stride) f[i] = eps * log(u[i]);
  for (int j = t; j < n; j += stride) g[j] = eps * log(v[j]);
}

int launch_uv_to_potentials(Context* ctx, const double* u, const double* v, int m, int n, double eps,
                            double* f, double* g, cudaStream_t st) {
  uv_to_potentials<<<std::max(1, (std::max(m, n) + 255) / 256), 256, 0, st>>>(u, v, m, n, eps, f, g);
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_absorb(Context* ctx, const double* C, long long ldc, const double* ft, const double* gt, int m,
                  int n, double inv_eps, double* K, cudaStream_t st) {
  skscaled::absorb_kernel<<<8 * ctx->sm_count, 256, 0, st>>>(C, ldc, ft, gt, m, n, inv_eps, K);
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_fill_ones(Context* ctx, double* x, int n, cudaStream_t st) {
  skscaled::fill_ones<<<std::max(1, std::min((n + 255) / 256, 4 * ctx->sm_count)), 256, 0, st>>>(x, n);
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace rwig
