// barycenter.cu -- Wasserstein barycenters of S histograms on a shared cost,
// parallel (Barycenter::compute_parallel, src/barycenter_impl_parallel.cpp:19)
// and log-domain (Barycenter::compute_log, src/barycenter_impl_log.cpp:23),
// with their unrolled gradients w.r.t. A and w.
//
// Both run in scaling form on K = exp(-C/eps): with U = exp(F/eps),
// V = exp(G/eps) the log-domain soft-min sweeps of the reference become the
// dense products K V and K^T U over the S histograms, done by the FP64
// tensor-core GEMM (dgemm.cuh); every elementwise step is fused into the
// split-K reduction that follows each product.  One iteration l:
//   U_l = A / Y_{l-1},  Z_l = K^T U_l,  b_l = prod_s Z_l^{w_s},  V_l = b_l / Z_l,
//   Y_l = K V_l                           (Y_0 = K 1)
// The log-domain residual -minrow(R)/eps - log A equals log(U_l o Y_l) - log A;
// the parallel residual is U_l o Y_l - A.  The adjoints (derived from
// _bwd_parallel :154-206 and _bwd_log :275-382) are, per step l = L..1,
//   parallel: Vbar = -K^T((Ubar o U_{l+1}) / Y_l), bbar = sum_s Vbar / Z_l,
//             Ubar = K((bbar w^T - Vbar / Z_l) o V_l), grad_A += Ubar / Y_{l-1},
//             grad_w += log(Z_l)^T (bbar o b_l)
//   log:      Gbar = -V_l o K^T(Fbar / Y_l), logbbar = eps sum_s Gbar,
//             Fbar = U_l o K(((w/eps) logbbar - Gbar) / Z_l), grad_A += Fbar / A,
//             grad_w += log(Z_l)^T logbbar,  grad_A *= eps at the end
// with the seeds of step L as in the reference.  The history U_l, V_l, Z_l,
// Y_l, b_l of every iteration is kept on the device (the backward reads it
// once, newest first); all reductions run in a fixed order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "dgemm.cuh"
#include "engine.h"

namespace rwig {

int dgemm_splitk(Context* ctx, const dg::GemmArgs& args, cudaStream_t st);
int dgemm_pick_splits(Context* ctx, int Mo, int Kd, int S);

namespace bary {

constexpr int TPB = 256;

__global__ void gibbs_kernel(const double* C, int M, int N, long long ldk, double reg, double* K) {
  const long long total = ldk * (long long)N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldk), j = (int)(k / ldk);
    K[k] = (i < M) ? exp(-C[i + (long long)j * M] / reg) : 0.0;  // exp(-C / reg)
  }
}

__global__ void fill_kernel(double* x, long long n, double v) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    x[k] = v;
}

// After Z = K^T U: per support point j, store Z, the barycenter entry and V.
// logdomain: b_j = exp(sum_s w_s log Z_js) and bl[j] = log b_j;
// parallel: b_j = prod_s Z_js^{w_s} (barycenter_impl_parallel.cpp:120), bl[j] = b_j.
__global__ void epi_z(const double* part, int splits, int N, int S, const double* w, int logdomain, double* Z,
                      double* V, double* bl) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    double acc = logdomain ? 0.0 : 1.0;
    for (int s = 0; s < S; ++s) {
      const double z = dg::reduce_splits(part, splits, N, S, j, s);
      Z[j + (size_t)s * N] = z;
      if (logdomain) acc += w[s] * log(z);
      else acc *= pow(z, w[s]);
    }
    const double b = logdomain ? exp(acc) : acc;
    bl[j] = acc;
    for (int s = 0; s < S; ++s) V[j + (size_t)s * N] = b / Z[j + (size_t)s * N];
  }
}

// After Y = K V: store Y, the next U = A / Y, and (when D != nullptr) the
// stopping residual of this iteration's U.
__global__ void epi_y(const double* part, int splits, int M, int S, const double* A, const double* logA,
                      const double* Ucur, int logdomain, double* Y, double* Unext, double* D, int ldd) {
  const long long total = (long long)M * S;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), s = (int)(k / M);
    const double y = dg::reduce_splits(part, splits, M, S, i, s);
    Y[k] = y;
    if (Unext) Unext[k] = A[k] / y;
    if (D) D[i + (size_t)s * ldd] = logdomain ? log(Ucur[k] * y) - logA[k] : Ucur[k] * y - A[k];
  }
}

// Backward, after T' = K^T T: per support point j the column adjoints, the
// operand of the next product (T2, N x S) and this block's share of grad_w.
// seed = 1 at step L.  bn: normalised barycenter (log seed); b_l: barycenter
// history entry of this step (parallel: b_l, log: unused); bext: data b.
__global__ void epi_b1(const double* part, int splits, int N, int S, const double* Z, const double* V,
                       const double* w, const double* bl, const double* bn, const double* bext, double eps,
                       int logdomain, int seed, double* T2, double* gw_part) {
  extern __shared__ double sh[];  // [S][blockDim.x / 32]
  const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double gw_local[64];
  for (int s = 0; s < S; ++s) gw_local[s] = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    if (!logdomain) {
      double bbar = 0.0;
      if (seed) {
        bbar = 2.0 * (bl[j] - bext[j]);  // un-normalised b (barycenter_impl_parallel.cpp:180)
      } else {
        for (int s = 0; s < S; ++s) {
          const double vbar = -dg::reduce_splits(part, splits, N, S, j, s);
          bbar += vbar / Z[j + (size_t)s * N];
        }
      }
      for (int s = 0; s < S; ++s) {
        const size_t k = j + (size_t)s * N;
        double t = bbar * w[s];
        if (!seed) t -= (-dg::reduce_splits(part, splits, N, S, j, s)) / Z[k];
        T2[k] = t * V[k];
        gw_local[s] += log(Z[k]) * (bbar * bl[j]);
      }
    } else {
      double lbb = 0.0;
      if (seed) {
        lbb = 2.0 * (bn[j] - bext[j]) * bn[j];  // barycenter_impl_log.cpp:324
      } else {
        for (int s = 0; s < S; ++s) lbb += -V[j + (size_t)s * N] * dg::reduce_splits(part, splits, N, S, j, s);
        lbb *= eps;
      }
      for (int s = 0; s < S; ++s) {
        const size_t k = j + (size_t)s * N;
        double y = (w[s] / eps) * lbb;
        if (!seed) y -= -V[k] * dg::reduce_splits(part, splits, N, S, j, s);
        T2[k] = y / Z[k];
        gw_local[s] += log(Z[k]) * lbb;
      }
    }
  }
  // block sums of the grad_w shares, fixed order, added to this block's slot
  for (int s = 0; s < S; ++s) {
    double v = gw_local[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[s * nw + warp] = v;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double v = 0.0;
    for (int q = 0; q < nw; ++q) v += sh[s * nw + q];
    gw_part[(size_t)blockIdx.x * S + s] += v;
  }
}

// Backward, after T'' = K T2: row adjoints, grad_A and the next step's operand.
__global__ void epi_b2(const double* part, int splits, int M, int S, const double* Ul, const double* Yprev,
                       const double* A, int logdomain, double* gradA, double* Tnext) {
  const long long total = (long long)M * S;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), s = (int)(k / M);
    const double y = dg::reduce_splits(part, splits, M, S, i, s);
    if (!logdomain) {
      gradA[k] += y / Yprev[k];                 // Ubar / (K V_{l-1})
      Tnext[k] = (y * Ul[k]) / Yprev[k];        // (Ubar o U_l) / (K V_{l-1})
    } else {
      const double fbar = Ul[k] * y;            // U_l o K(...)
      gradA[k] += fbar / A[k];
      Tnext[k] = fbar / Yprev[k];               // Fbar / (K V_{l-1})
    }
  }
}

__global__ void scale_kernel(double* x, long long n, double a) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    x[k] *= a;
}

__global__ void log_scaled(const double* x, long long n, double eps, double* out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    out[k] = eps * log(x[k]);
}

__global__ void log_kernel(const double* x, long long n, double* out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    out[k] = log(x[k]);
}

// One block: b = (logdomain ? exp(bl) : bl) / sum; loss = sum (b - bext)^2 when bext.
// Fixed-order tree reduction.
__global__ void normalise_b(const double* bl, int N, int logdomain, const double* bext, double* bn,
                            double* out2) {
  __shared__ double sh[1024];
  double acc = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) acc += logdomain ? exp(bl[j]) : bl[j];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double tot = sh[0];
  __syncthreads();
  double l = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    const double v = (logdomain ? exp(bl[j]) : bl[j]) / tot;
    bn[j] = v;
    if (bext) {
      const double d = v - bext[j];
      l += d * d;
    }
  }
  sh[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out2[0] = tot;
    out2[1] = sh[0];
  }
}

__global__ void reduce_gw(const double* gw_part, int nblk, int S, double* gw) {
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double v = 0.0;
    for (int q = 0; q < nblk; ++q) v += gw_part[(size_t)q * S + s];
    gw[s] = v;
  }
}

// Largest eigenvalue of a symmetric S x S matrix (cyclic Jacobi), host side.
double lambda_max(std::vector<double> G, int S) {
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < S; ++p)
      for (int q = p + 1; q < S; ++q) off += G[p + q * S] * G[p + q * S];
    if (off < 1e-300) break;
    for (int p = 0; p < S; ++p)
      for (int q = p + 1; q < S; ++q) {
        const double apq = G[p + q * S];
        if (apq == 0.0) continue;
        const double theta = (G[q + q * S] - G[p + p * S]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < S; ++k) {
          const double gkp = G[k + p * S], gkq = G[k + q * S];
          G[k + p * S] = c * gkp - sn * gkq;
          G[k + q * S] = sn * gkp + c * gkq;
        }
        for (int k = 0; k < S; ++k) {
          const double gpk = G[p + k * S], gqk = G[q + k * S];
          G[p + k * S] = c * gpk - sn * gqk;
          G[q + k * S] = sn * gpk + c * gqk;
        }
      }
  }
  double l = 0.0;
  for (int p = 0; p < S; ++p) l = std::max(l, G[p + p * S]);
  return l;
}

int grid_for(Context* ctx, long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + TPB - 1) / TPB, 8LL * ctx->sm_count));
}

enum {
  SB_K = 60, SB_PART, SB_UH, SB_VH, SB_ZH, SB_YH, SB_BH, SB_ONES, SB_LOGA, SB_D, SB_GRAM, SB_BN, SB_SCAL,
  SB_T, SB_T2, SB_GA, SB_GWP, SB_GW, SB_A, SB_W, SB_C, SB_BEXT, SB_OUTU, SB_OUTV, SB_OUTB
};

// Core driver; all pointers on the device.  Outputs (any may be null):
// U, V (parallel) or F, G (log) as X1, X2; b (normalised); grad_A, grad_w.
int run(Context* ctx, cudaStream_t st, bool logdomain, double* X1, double* X2, double* b, double* gradA,
        double* gradw, double* loss, int* iter_out, double* err_out, const double* A, const double* w,
        const double* C, const double* bext, int M, int N, int S, double reg, int withgrad, int max_iter,
        double tol) {
  reset_report();
  if (!A || !w || !C) return set_error(RWIG_E_INVALID, "A, w and C must be non-null");
  if (M < 1 || N < 1 || S < 1) return set_error(RWIG_E_INVALID, "M, N and S must be >= 1");
  if (S > 64) return set_error(RWIG_E_UNSUPPORTED, "more than 64 histograms");
  if (!(reg > 0.0) || !std::isfinite(reg)) return set_error(RWIG_E_INVALID, "reg must be finite and > 0");
  if (withgrad && !bext) return set_error(RWIG_E_INVALID, "b_ext is required with withgrad");
  const int L = std::max(0, max_iter);
  const size_t MS = (size_t)M * S, NS = (size_t)N * S;
  const long long ldk = ((M + 1) / 2) * 2;
  const int splits_y = dgemm_pick_splits(ctx, M, N, S), splits_z = dgemm_pick_splits(ctx, N, M, S);
  const int splits_max = std::max(splits_y, splits_z);
  // history depth: every iteration's state when gradients are needed, else two
  const int H = withgrad ? L + 2 : 2;
  double* K = (double*)scratch(ctx, SB_K, sizeof(double) * ldk * N);
  double* part = (double*)scratch(ctx, SB_PART, sizeof(double) * (size_t)splits_max * S * std::max(M, N));
  double* Uh = (double*)scratch(ctx, SB_UH, sizeof(double) * MS * H);
  double* Vh = (double*)scratch(ctx, SB_VH, sizeof(double) * NS * H);
  double* Zh = (double*)scratch(ctx, SB_ZH, sizeof(double) * NS * H);
  double* Yh = (double*)scratch(ctx, SB_YH, sizeof(double) * MS * H);
  double* Bh = (double*)scratch(ctx, SB_BH, sizeof(double) * (size_t)N * H);
  double* logA = (double*)scratch(ctx, SB_LOGA, sizeof(double) * MS);
  const long long ldd = ((M + 1) / 2) * 2;
  double* D = (double*)scratch(ctx, SB_D, sizeof(double) * ldd * S);
  double* gram = (double*)scratch(ctx, SB_GRAM, sizeof(double) * (size_t)splits_max * S * S + 64);
  double* bn = (double*)scratch(ctx, SB_BN, sizeof(double) * N);
  double* scal = (double*)scratch(ctx, SB_SCAL, sizeof(double) * 8);
  if (!K || !part || !Uh || !Vh || !Zh || !Yh || !Bh || !logA || !D || !gram || !bn || !scal)
    return RWIG_E_NOMEM;
  auto slot = [&](double* base, size_t sz, int l) { return base + sz * (size_t)(withgrad ? l : (l & 1)); };
  int launches = 0;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));

  gibbs_kernel<<<grid_for(ctx, ldk * N), TPB, 0, st>>>(C, M, N, ldk, reg, K);  // K = exp(-C/reg)
  log_kernel<<<grid_for(ctx, MS), TPB, 0, st>>>(A, MS, logA);
  fill_kernel<<<grid_for(ctx, NS), TPB, 0, st>>>(slot(Vh, NS, 0), NS, 1.0);  // V_0 = 1
  launches += 3;

  auto gemm = [&](int trans, const double* X, long long ldx, int Mo, int Kd, int splits) -> int {
    dg::GemmArgs g{K, ldk, trans, Mo, Kd, S, X, ldx, part, splits};
    ++launches;
    return dgemm_splitk(ctx, g, st);
  };
  // Y_0 = K V_0, U_1 = A / Y_0
  int rc = gemm(0, slot(Vh, NS, 0), N, M, N, splits_y);
  if (rc) return rc;
  epi_y<<<grid_for(ctx, MS), TPB, 0, st>>>(part, splits_y, M, S, A, logA, nullptr, logdomain,
                                            slot(Yh, MS, 0), slot(Uh, MS, 1), nullptr, (int)ldd);
  ++launches;

  double err = 1000.0;
  int iter = 0;
  auto compute_err = [&]() -> int {
    // err from the residual D: Frobenius (parallel, :134) or spectral (log, :252)
    dg::GemmArgs g{D, ldd, 1, S, M, S, D, ldd, gram, 1};
    ++launches;
    int r = dgemm_splitk(ctx, g, st);
    if (r) return r;
    std::vector<double> G(S * S);
    RWIG_CUDA_TRY(cudaMemcpyAsync(G.data(), gram, sizeof(double) * S * S, cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaStreamSynchronize(st));
    if (logdomain) {
      err = std::sqrt(lambda_max(G, S));
    } else {
      double tr = 0.0;
      for (int s = 0; s < S; ++s) tr += G[s + s * S];
      err = std::sqrt(tr);
    }
    return 0;
  };
  while (iter < L && err >= tol) {
    ++iter;
    const int l = iter;
    double* Ul = slot(Uh, MS, l);
    // Z_l = K^T U_l; b_l; V_l = b_l / Z_l
    rc = gemm(1, Ul, M, N, M, splits_z);
    if (rc) return rc;
    epi_z<<<grid_for(ctx, N), TPB, 0, st>>>(part, splits_z, N, S, w, logdomain, slot(Zh, NS, l),
                                             slot(Vh, NS, l), slot(Bh, N, l));
    ++launches;
    // Y_l = K V_l; U_{l+1} = A / Y_l; residual when the stopping test needs it
    rc = gemm(0, slot(Vh, NS, l), N, M, N, splits_y);
    if (rc) return rc;
    const bool need_err = (tol > 0.0) || (iter == L);
    epi_y<<<grid_for(ctx, MS), TPB, 0, st>>>(part, splits_y, M, S, A, logA, Ul, logdomain, slot(Yh, MS, l),
                                              slot(Uh, MS, l + 1), need_err ? D : nullptr, (int)ldd);
    ++launches;
    if (need_err) {
      rc = compute_err();
      if (rc) return rc;
    }
  }
  RWIG_CUDA_TRY(cudaGetLastError());

  // normalised barycenter and loss (log: before the backward, :268-271;
  // parallel: the backward uses the un-normalised b, :35-42)
  if (iter > 0) {
    normalise_b<<<1, 1024, 0, st>>>(slot(Bh, N, iter), N, logdomain, withgrad ? bext : nullptr, bn, scal);
  } else {
    // no iteration: parallel b = 0 / sum(0) (barycenter_impl_parallel.cpp:64, :39);
    // log b = exp(0) / N (barycenter_impl_log.cpp:193, :268-269)
    fill_kernel<<<grid_for(ctx, N), TPB, 0, st>>>(bn, N, logdomain ? 1.0 / N : NAN);
  }
  ++launches;

  if (withgrad && iter > 0) {
    double* T = (double*)scratch(ctx, SB_T, sizeof(double) * MS);
    double* T2 = (double*)scratch(ctx, SB_T2, sizeof(double) * NS);
    double* gA = (double*)scratch(ctx, SB_GA, sizeof(double) * MS);
    const int nb1 = grid_for(ctx, N);
    double* gwp = (double*)scratch(ctx, SB_GWP, sizeof(double) * (size_t)nb1 * S);
    double* gw = (double*)scratch(ctx, SB_GW, sizeof(double) * S);
    if (!T || !T2 || !gA || !gwp || !gw) return RWIG_E_NOMEM;
    RWIG_CUDA_TRY(cudaMemsetAsync(gA, 0, sizeof(double) * MS, st));
    RWIG_CUDA_TRY(cudaMemsetAsync(gwp, 0, sizeof(double) * (size_t)nb1 * S, st));
    const int nw = TPB / 32;
    for (int l = iter; l >= 1; --l) {
      const bool seed = (l == iter);
      if (!seed) {
        rc = gemm(1, T, M, N, M, splits_z);  // K^T T
        if (rc) return rc;
      }
      epi_b1<<<nb1, TPB, sizeof(double) * S * nw, st>>>(part, seed ? 0 : splits_z, N, S, slot(Zh, NS, l),
                                                       slot(Vh, NS, l), w, slot(Bh, N, l), bn, bext, reg,
                                                       logdomain, seed ? 1 : 0, T2, gwp);
      ++launches;
      rc = gemm(0, T2, N, M, N, splits_y);  // K T2
      if (rc) return rc;
      epi_b2<<<grid_for(ctx, MS), TPB, 0, st>>>(part, splits_y, M, S, slot(Uh, MS, l), slot(Yh, MS, l - 1), A,
                                                 logdomain, gA, T);
      ++launches;
    }
    reduce_gw<<<1, 64, 0, st>>>(gwp, nb1, S, gw);
    ++launches;
    if (logdomain) {
      scale_kernel<<<grid_for(ctx, MS), TPB, 0, st>>>(gA, MS, reg);  // :376
      ++launches;
    }
    if (gradA) RWIG_CUDA_TRY(cudaMemcpyAsync(gradA, gA, sizeof(double) * MS, cudaMemcpyDeviceToDevice, st));
    if (gradw) RWIG_CUDA_TRY(cudaMemcpyAsync(gradw, gw, sizeof(double) * S, cudaMemcpyDeviceToDevice, st));
  }

  // outputs: U, V (parallel) or F = eps log U, G = eps log V (log) of the last iteration
  const double* Ufin = slot(Uh, MS, iter > 0 ? iter : 0);
  const double* Vfin = slot(Vh, NS, iter);
  if (iter == 0) {
    fill_kernel<<<grid_for(ctx, MS), TPB, 0, st>>>(slot(Uh, MS, 0), MS, 1.0);  // U = 1 (:67)
    ++launches;
  }
  if (X1) {
    if (logdomain) log_scaled<<<grid_for(ctx, MS), TPB, 0, st>>>(Ufin, MS, reg, X1);
    else RWIG_CUDA_TRY(cudaMemcpyAsync(X1, Ufin, sizeof(double) * MS, cudaMemcpyDeviceToDevice, st));
  }
  if (X2) {
    if (logdomain) log_scaled<<<grid_for(ctx, NS), TPB, 0, st>>>(Vfin, NS, reg, X2);
    else RWIG_CUDA_TRY(cudaMemcpyAsync(X2, Vfin, sizeof(double) * NS, cudaMemcpyDeviceToDevice, st));
  }
  if (b) RWIG_CUDA_TRY(cudaMemcpyAsync(b, bn, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
  double sc[2] = {0.0, 0.0};
  if (iter > 0) RWIG_CUDA_TRY(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  RWIG_CUDA_TRY(cudaGetLastError());
  if (loss) *loss = withgrad ? sc[1] : 0.0;
  if (iter_out) *iter_out = iter;
  if (err_out) *err_out = err;
  const int status = (err <= tol) ? 0 : (iter == L ? 1 : 2);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  rwig_report& R = report();
  R.iter = iter;
  R.status = status;
  R.err = err;
  R.device_ms = ms;
  R.kernel_ms = ms;
  R.kernel_launches = launches;
  R.support_m = M;
  R.support_n = N;
  R.bary_norm = sc[0];
  return status;
}

// Host-pointer wrapper: copies in, runs, copies out.
int run_host(bool logdomain, double* X1, double* X2, double* b, double* gradA, double* gradw, double* loss,
             int* iter, double* err, const double* A, const double* w, const double* C, const double* bext, int M,
             int N, int S, double reg, int withgrad, int max_iter, double tol) {
  if (!A || !w || !C || M < 1 || N < 1 || S < 1) return set_error(RWIG_E_INVALID, "bad arguments");
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = ctx->stream;
  const size_t MS = (size_t)M * S, NS = (size_t)N * S, MN = (size_t)M * N;
  double* dA = (double*)scratch(ctx, SB_A, sizeof(double) * MS);
  double* dw = (double*)scratch(ctx, SB_W, sizeof(double) * S);
  double* dC = (double*)scratch(ctx, SB_C, sizeof(double) * MN);
  double* dbe = (withgrad && bext) ? (double*)scratch(ctx, SB_BEXT, sizeof(double) * N) : nullptr;
  double* d1 = X1 ? (double*)scratch(ctx, SB_OUTU, sizeof(double) * MS) : nullptr;
  double* d2 = X2 ? (double*)scratch(ctx, SB_OUTV, sizeof(double) * NS) : nullptr;
  double* db = (double*)scratch(ctx, SB_OUTB, sizeof(double) * (N + MS + S));
  if (!dA || !dw || !dC || (withgrad && bext && !dbe) || (X1 && !d1) || (X2 && !d2) || !db) return RWIG_E_NOMEM;
  double* dgA = db + N;
  double* dgw = dgA + MS;
  RWIG_CUDA_TRY(cudaMemcpyAsync(dA, A, sizeof(double) * MS, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(dw, w, sizeof(double) * S, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(dC, C, sizeof(double) * MN, cudaMemcpyHostToDevice, st));
  if (dbe) RWIG_CUDA_TRY(cudaMemcpyAsync(dbe, bext, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  int rc = run(ctx, st, logdomain, d1, d2, db, gradA ? dgA : nullptr, gradw ? dgw : nullptr, loss, iter, err, dA,
               dw, dC, dbe, M, N, S, reg, withgrad, max_iter, tol);
  if (rc < 0) return rc;
  if (X1) RWIG_CUDA_TRY(cudaMemcpyAsync(X1, d1, sizeof(double) * MS, cudaMemcpyDeviceToHost, st));
  if (X2) RWIG_CUDA_TRY(cudaMemcpyAsync(X2, d2, sizeof(double) * NS, cudaMemcpyDeviceToHost, st));
  if (b) RWIG_CUDA_TRY(cudaMemcpyAsync(b, db, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  if (withgrad && gradA) RWIG_CUDA_TRY(cudaMemcpyAsync(gradA, dgA, sizeof(double) * MS, cudaMemcpyDeviceToHost, st));
  if (withgrad && gradw) RWIG_CUDA_TRY(cudaMemcpyAsync(gradw, dgw, sizeof(double) * S, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  return rc;
}

}  // namespace bary
}  // namespace rwig

using namespace rwig;

extern "C" int rwig_barycenter_parallel(double* U, double* V, double* b, double* grad_A, double* grad_w,
                                        double* loss, int* iter, double* err, const double* A, const double* w,
                                        const double* C, const double* b_ext, int M, int N, int S, double reg,
                                        int withgrad, int max_iter, double zero_tol) {
  return bary::run_host(false, U, V, b, grad_A, grad_w, loss, iter, err, A, w, C, b_ext, M, N, S, reg, withgrad,
                        max_iter, zero_tol);
}

extern "C" int rwig_barycenter_log(double* F, double* G, double* b, double* grad_A, double* grad_w, double* loss,
                                   int* iter, double* err, const double* A, const double* w, const double* C,
                                   const double* b_ext, int M, int N, int S, double reg, int withgrad,
                                   int max_iter, double zero_tol) {
  return bary::run_host(true, F, G, b, grad_A, grad_w, loss, iter, err, A, w, C, b_ext, M, N, S, reg, withgrad,
                        max_iter, zero_tol);
}

extern "C" int rwig_barycenter_parallel_dev(double* U, double* V, double* b, double* grad_A, double* grad_w,
                                            double* loss, int* iter, double* err, const double* A, const double* w,
                                            const double* C, const double* b_ext, int M, int N, int S, double reg,
                                            int withgrad, int max_iter, double zero_tol, void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return bary::run(ctx, stream ? (cudaStream_t)stream : ctx->stream, false, U, V, b, grad_A, grad_w, loss, iter,
                   err, A, w, C, b_ext, M, N, S, reg, withgrad, max_iter, zero_tol);
}

extern "C" int rwig_barycenter_log_dev(double* F, double* G, double* b, double* grad_A, double* grad_w,
                                       double* loss, int* iter, double* err, const double* A, const double* w,
                                       const double* C, const double* b_ext, int M, int N, int S, double reg,
                                       int withgrad, int max_iter, double zero_tol, void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return bary::run(ctx, stream ? (cudaStream_t)stream : ctx->stream, true, F, G, b, grad_A, grad_w, loss, iter,
                   err, A, w, C, b_ext, M, N, S, reg, withgrad, max_iter, zero_tol);
}
