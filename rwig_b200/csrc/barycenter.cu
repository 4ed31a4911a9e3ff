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
//
// The scaling form equals the log-domain updates only while every K_ij is a
// normal double and the products stay well inside the double range.  For the
// log method the Gibbs kernel and the epilogues check this as they go (K_ij
// normal and finite; every entry of Y = K V and Z = K^T U in [1e-290,
// 1e290]; the adjoint operands finite) and raise a flag word; a flagged solve
// is re-run by the log-domain kernels of barycenter_log.cu, which follow the
// reference's soft-min sweeps over C - F and C - G directly.  With Y, Z >=
// 1e-290 and normal K the products lost to underflow change each sum by
// less than N 2^-1074 / 1e-290, far below rounding.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "barycenter.h"
#include "dgemm.cuh"
#include "engine.h"

namespace rwig {

namespace bary {

constexpr int TPB = 256;

// Range checks of the scaling form (log method): a value outside the range
// sets *flag (the solve is then re-run in the log domain).
constexpr double kRangeLo = 1e-290, kRangeHi = 1e290;
__device__ __forceinline__ void check_range(double* flag, double x) {
  if (flag && !(x >= kRangeLo && x <= kRangeHi)) *flag = 1.0;
}
__device__ __forceinline__ void check_finite(double* flag, double x) {
  if (flag && !(fabs(x) <= 1.79e308)) *flag = 1.0;
}

__global__ void gibbs_kernel(const double* C, int M, int N, long long ldk, double reg, double* K, double* flag) {
  const long long total = ldk * (long long)N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldk), j = (int)(k / ldk);
    const double v = (i < M) ? exp(-C[i + (long long)j * M] / reg) : 0.0;  // exp(-C / reg)
    K[k] = v;
    if (flag && i < M && !(v >= 2.2250738585072014e-308 && v <= 1.79e308)) *flag = 1.0;  // subnormal, 0, inf
  }
}

__global__ void fill_kernel(double* x, long long n, double v) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    x[k] = v;
}

// GEMM epilogues (dgemm.cuh interface): each receives rows r0 .. r0+nr-1 of
// the product, column s at t[s*ldt + r], and uses ws ((S+1)*ldt doubles of
// it) as scratch.  Per-row reductions over s run in the fixed order s = 0..S-1.

// After Z = K^T U_l: store Z, V = b / Z and the barycenter entry.
// logdomain: b_j = exp(sum_s w_s log Z_js), bl[j] = log b_j;
// parallel: b_j = prod_s Z_js^{w_s} (barycenter_impl_parallel.cpp:120), bl[j] = b_j.
struct EpiZ {
  const double* w;
  double* Z;
  double* V;
  double* bl;
  int N, S, logdomain;
  double* flag;
  __device__ void operator()(int r0, int nr, int, int, double* t, int ldt, double* ws) const {
    if (nr <= 0) return;
    const int n = nr * S;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const int r = e % nr, s = e / nr;
      const double z = t[s * ldt + r];
      check_range(flag, z);
      ws[s * ldt + r] = logdomain ? w[s] * log(z) : pow(z, w[s]);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
      double acc = logdomain ? 0.0 : 1.0;
      for (int s = 0; s < S; ++s) acc = logdomain ? acc + ws[s * ldt + r] : acc * ws[s * ldt + r];
      bl[r0 + r] = acc;
      ws[S * ldt + r] = logdomain ? exp(acc) : acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const int r = e % nr, s = e / nr;
      const size_t k = (size_t)(r0 + r) + (size_t)s * N;
      const double z = t[s * ldt + r];
      Z[k] = z;
      V[k] = ws[S * ldt + r] / z;
    }
  }
};

// After Y = K V: store Y, the next U = A / Y, and (when D != nullptr) the
// stopping residual of this iteration's U.
struct EpiY {
  const double* A;
  const double* logA;
  const double* Ucur;
  double* Y;
  double* Unext;
  double* D;
  int M, S, ldd, logdomain;
  double* flag;
  __device__ void operator()(int r0, int nr, int, int, double* t, int ldt, double*) const {
    if (nr <= 0) return;
    for (int e = threadIdx.x; e < nr * S; e += blockDim.x) {
      const int r = e % nr, s = e / nr, i = r0 + r;
      const size_t k = (size_t)i + (size_t)s * M;
      const double y = t[s * ldt + r];
      check_range(flag, y);
      Y[k] = y;
      if (Unext) Unext[k] = A[k] / y;
      if (D) D[i + (size_t)s * ldd] = logdomain ? log(Ucur[k] * y) - logA[k] : Ucur[k] * y - A[k];
    }
  }
};

// Backward, after T' = K^T T (t == nullptr at the seed step L, which has no
// product): per support point j the column adjoint, the operand T2 (N x S) of
// the next product and the grad_w shares, summed per 8-row group into
// gw_part[(j/8)*S + s].  bl: barycenter history entry of this step
// (parallel: b_l); bn: normalised barycenter (log seed); bext: data b.
struct EpiB1 {
  const double* Z;
  const double* V;
  const double* w;
  const double* bl;
  const double* bn;
  const double* bext;
  double eps;
  int N, S, logdomain, seed;
  double* T2;
  double* gw_part;
  double* flag;
  __device__ void operator()(int r0, int nr, int, int, double* t, int ldt, double* ws) const {
    if (nr <= 0) return;
    const int n = nr * S;
    if (!seed) {
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int r = e % nr, s = e / nr;
        const size_t k = (size_t)(r0 + r) + (size_t)s * N;
        const double y = t[s * ldt + r];
        ws[s * ldt + r] = logdomain ? -V[k] * y : (-y) / Z[k];
      }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
      const int j = r0 + r;
      double c;
      if (seed) {
        c = logdomain ? 2.0 * (bn[j] - bext[j]) * bn[j]   // barycenter_impl_log.cpp:324
                      : 2.0 * (bl[j] - bext[j]);          // un-normalised b (barycenter_impl_parallel.cpp:180)
      } else {
        c = 0.0;
        for (int s = 0; s < S; ++s) c += ws[s * ldt + r];
        if (logdomain) c *= eps;
      }
      ws[S * ldt + r] = c;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const int r = e % nr, s = e / nr, j = r0 + r;
      const size_t k = (size_t)j + (size_t)s * N;
      const double c = ws[S * ldt + r];
      const double lz = log(Z[k]);
      if (!logdomain) {
        double tt = c * w[s];
        if (!seed) tt -= (-t[s * ldt + r]) / Z[k];
        T2[k] = tt * V[k];
        ws[s * ldt + r] = lz * (c * bl[j]);
      } else {
        double y = (w[s] / eps) * c;
        if (!seed) y -= -V[k] * t[s * ldt + r];
        T2[k] = y / Z[k];
        check_finite(flag, T2[k]);
        ws[s * ldt + r] = lz * c;
      }
    }
    __syncthreads();
    const int ngrp = (nr + 7) / 8;
    for (int p = threadIdx.x; p < ngrp * S; p += blockDim.x) {
      const int s = p % S, q = p / S;
      double v = 0.0;
      for (int r = q * 8; r < min(nr, q * 8 + 8); ++r) v += ws[s * ldt + r];
      gw_part[(size_t)(r0 / 8 + q) * S + s] += v;
    }
  }
};

// Backward, after T'' = K T2: row adjoints, grad_A and the next step's operand.
struct EpiB2 {
  const double* Ul;
  const double* Yprev;
  const double* A;
  int M, S, logdomain;
  double* gradA;
  double* Tnext;
  double* flag;
  __device__ void operator()(int r0, int nr, int, int, double* t, int ldt, double*) const {
    if (nr <= 0) return;
    for (int e = threadIdx.x; e < nr * S; e += blockDim.x) {
      const int r = e % nr, s = e / nr;
      const size_t k = (size_t)(r0 + r) + (size_t)s * M;
      const double y = t[s * ldt + r];
      if (!logdomain) {
        gradA[k] += y / Yprev[k];           // Ubar / (K V_{l-1})
        Tnext[k] = (y * Ul[k]) / Yprev[k];  // (Ubar o U_l) / (K V_{l-1})
      } else {
        const double fbar = Ul[k] * y;  // U_l o K(...)
        gradA[k] += fbar / A[k];
        Tnext[k] = fbar / Yprev[k];  // Fbar / (K V_{l-1})
        check_finite(flag, Tnext[k]);
        check_finite(flag, gradA[k]);
      }
    }
  }
};

// The seed step of the backward, which has no product: the EpiB1 epilogue
// over 8-row groups.
__global__ void seed_b1(EpiB1 epi, int N) {
  extern __shared__ double ws[];  // (S + 1) * 8
  const int r0 = blockIdx.x * 8;
  epi(r0, min(8, N - r0), 0, 0, nullptr, 8, ws);
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

// grad_w[s] = sum over the 8-row groups of gw_part[q*S + s]; one block per s,
// fixed-order strided sums and tree.
__global__ void reduce_gw(const double* gw_part, int ngrp, int S, double* gw) {
  __shared__ double sh[256];
  const int s = blockIdx.x;
  double v = 0.0;
  for (int q = threadIdx.x; q < ngrp; q += blockDim.x) v += gw_part[(size_t)q * S + s];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) gw[s] = sh[0];
}

// Largest eigenvalue of a symmetric positive semi-definite S x S matrix
// (column-major), host side: Householder reduction to tridiagonal form,
// then bisection on the Sturm sequence of the tridiagonal matrix (the number
// of eigenvalues below x is the number of negative pivots of T - xI).
double lambda_max(std::vector<double> G, int n) {
  auto at = [&](int i, int j) -> double& { return G[i + (size_t)j * n]; };
  std::vector<double> v(n), p(n);
  for (int k = 0; k + 2 < n; ++k) {
    double a2 = 0.0;
    for (int i = k + 1; i < n; ++i) a2 += at(i, k) * at(i, k);
    const double x1 = at(k + 1, k);
    if (a2 == x1 * x1) continue;  // column already tridiagonal
    const double alpha = x1 >= 0.0 ? -std::sqrt(a2) : std::sqrt(a2);
    // v = x - alpha e1 (entries k+1..n-1), H = I - 2 v v^T / (v^T v)
    for (int i = k + 1; i < n; ++i) v[i] = at(i, k);
    v[k + 1] -= alpha;
    double vtv = 0.0;
    for (int i = k + 1; i < n; ++i) vtv += v[i] * v[i];
    if (vtv == 0.0) continue;
    // trailing block A <- H A H: p = 2 A v / vtv, q = p - (v^T p / vtv) v,
    // A -= v q^T + q v^T
    for (int i = k + 1; i < n; ++i) {
      double acc = 0.0;
      for (int j = k + 1; j < n; ++j) acc += at(i, j) * v[j];
      p[i] = 2.0 * acc / vtv;
    }
    double vp = 0.0;
    for (int i = k + 1; i < n; ++i) vp += v[i] * p[i];
    const double kf = vp / vtv;
    for (int i = k + 1; i < n; ++i) p[i] -= kf * v[i];
    for (int j = k + 1; j < n; ++j)
      for (int i = k + 1; i < n; ++i) at(i, j) -= v[i] * p[j] + p[i] * v[j];
    at(k + 1, k) = alpha;
    at(k, k + 1) = alpha;
    for (int i = k + 2; i < n; ++i) at(i, k) = at(k, i) = 0.0;
  }
  std::vector<double> d(n), e2(n, 0.0);
  double lo = 0.0, hi = 0.0;
  for (int i = 0; i < n; ++i) {
    d[i] = at(i, i);
    const double el = i > 0 ? std::fabs(at(i, i - 1)) : 0.0;
    const double er = i + 1 < n ? std::fabs(at(i + 1, i)) : 0.0;
    if (i > 0) e2[i] = at(i, i - 1) * at(i, i - 1);
    lo = i == 0 ? d[i] - el - er : std::min(lo, d[i] - el - er);
    hi = i == 0 ? d[i] + el + er : std::max(hi, d[i] + el + er);
  }
  const double tiny = 1e-300 + 1e-16 * std::max(std::fabs(lo), std::fabs(hi));
  auto below = [&](double x) {  // eigenvalues < x
    int cnt = 0;
    double q = 1.0;
    for (int i = 0; i < n; ++i) {
      q = d[i] - x - (i > 0 ? e2[i] / q : 0.0);
      if (q == 0.0) q = -tiny;
      if (q < 0.0) ++cnt;
    }
    return cnt;
  };
  for (int it = 0; it < 200 && hi - lo > 2e-16 * std::max(std::fabs(lo), std::fabs(hi)); ++it) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (below(mid) == n) hi = mid;
    else lo = mid;
  }
  return std::max(0.0, 0.5 * (lo + hi));
}

int grid_for(Context* ctx, long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + TPB - 1) / TPB, 8LL * ctx->sm_count));
}

enum {
  SB_K = 60, SB_UH, SB_VH, SB_ZH, SB_YH, SB_BH, SB_ONES, SB_LOGA, SB_D, SB_GRAM, SB_BN, SB_SCAL,
  SB_T, SB_T2, SB_GA, SB_GWP, SB_GW, SB_A, SB_W, SB_C, SB_BEXT, SB_OUTU, SB_OUTV, SB_OUTB
};

// One barycenter solve: its device buffers (engine scratch slots, numbered
// from `off` so that several solves can be enqueued side by side) and its
// launch sequence.  All pointers on the device.
struct Solve {
  Context* ctx = nullptr;
  bool logdomain = false;
  double *X1 = nullptr, *X2 = nullptr, *b = nullptr, *gradA = nullptr, *gradw = nullptr;
  const double *A = nullptr, *w = nullptr, *C = nullptr, *bext = nullptr;
  int M = 0, N = 0, S = 0, withgrad = 0, L = 0;
  double reg = 0.0, tol = 0.0;
  size_t MS = 0, NS = 0;
  long long ldk = 0, ldd = 0;
  int H = 0, ngrp = 0;
  // tol <= 0: the iteration count is fixed (L) and err is only needed after
  // the last iteration, so the whole launch sequence is known up front
  bool fixed = true;
  double *K = nullptr, *Uh = nullptr, *Vh = nullptr, *Zh = nullptr, *Yh = nullptr, *Bh = nullptr;
  double *logA = nullptr, *D = nullptr, *gram = nullptr, *bn = nullptr, *scal = nullptr;
  double *T = nullptr, *T2 = nullptr, *gA = nullptr, *gwp = nullptr, *gw = nullptr;
  int launches = 0, iter = 0;
  double err = 1000.0;
  bool needs_log = false;  // the range flag was seen set during the solve (tol > 0)

  double* slot(double* base, size_t sz, int l) const { return base + sz * (size_t)(withgrad ? l : (l & 1)); }

  // Sizes from the arguments; buffers from scratch slots off + SB_*,
  // allocated before anything is enqueued (a captured sequence must not
  // allocate).
  int alloc(int off) {
    L = std::max(0, L);
    MS = (size_t)M * S;
    NS = (size_t)N * S;
    ldk = ((M + 1) / 2) * 2;
    ldd = ((M + 1) / 2) * 2;
    // history depth: every iteration's state when gradients are needed, else two
    H = withgrad ? L + 2 : 2;
    ngrp = (N + 7) / 8;
    fixed = !(tol > 0.0);
    K = (double*)scratch(ctx, off + SB_K, sizeof(double) * ldk * N);
    Uh = (double*)scratch(ctx, off + SB_UH, sizeof(double) * MS * H);
    Vh = (double*)scratch(ctx, off + SB_VH, sizeof(double) * NS * H);
    Zh = (double*)scratch(ctx, off + SB_ZH, sizeof(double) * NS * H);
    Yh = (double*)scratch(ctx, off + SB_YH, sizeof(double) * MS * H);
    Bh = (double*)scratch(ctx, off + SB_BH, sizeof(double) * (size_t)N * H);
    logA = (double*)scratch(ctx, off + SB_LOGA, sizeof(double) * MS);
    D = (double*)scratch(ctx, off + SB_D, sizeof(double) * ldd * S);
    gram = (double*)scratch(ctx, off + SB_GRAM, sizeof(double) * (size_t)S * S);
    bn = (double*)scratch(ctx, off + SB_BN, sizeof(double) * N);
    scal = (double*)scratch(ctx, off + SB_SCAL, sizeof(double) * 8);
    if (!K || !Uh || !Vh || !Zh || !Yh || !Bh || !logA || !D || !gram || !bn || !scal) return RWIG_E_NOMEM;
    if (withgrad) {
      T = (double*)scratch(ctx, off + SB_T, sizeof(double) * MS);
      T2 = (double*)scratch(ctx, off + SB_T2, sizeof(double) * NS);
      gA = (double*)scratch(ctx, off + SB_GA, sizeof(double) * MS);
      gwp = (double*)scratch(ctx, off + SB_GWP, sizeof(double) * (size_t)ngrp * S);
      gw = (double*)scratch(ctx, off + SB_GW, sizeof(double) * S);
      if (!T || !T2 || !gA || !gwp || !gw) return RWIG_E_NOMEM;
    }
    return 0;
  }

  // err from the Gram matrix of the residual D: Frobenius (parallel, :134) or
  // spectral (log, :252)
  void err_from_gram(const double* G) {
    if (logdomain) {
      err = std::sqrt(lambda_max(std::vector<double>(G, G + (size_t)S * S), S));
    } else {
      double tr = 0.0;
      for (int s = 0; s < S; ++s) tr += G[s + s * S];
      err = std::sqrt(tr);
    }
  }

  // The whole solve on stream q (with tol > 0 the stopping test reads err
  // on the host after every iteration).
  // Log method: the range flag of the scaling form (scal[2]), else null.
  double* flag() const { return logdomain ? scal + 2 : nullptr; }

  int enqueue(cudaStream_t q) {
  launches = 0;
  iter = 0;
  err = 1000.0;
  needs_log = false;
  RWIG_CUDA_TRY(cudaMemsetAsync(scal + 2, 0, sizeof(double), q));
  gibbs_kernel<<<grid_for(ctx, ldk * N), TPB, 0, q>>>(C, M, N, ldk, reg, K, flag());  // K = exp(-C/reg)
  log_kernel<<<grid_for(ctx, MS), TPB, 0, q>>>(A, MS, logA);
  fill_kernel<<<grid_for(ctx, NS), TPB, 0, q>>>(slot(Vh, NS, 0), NS, 1.0);  // V_0 = 1
  launches += 3;
  // Y = K X (rows M, contraction N) and Z = K^T X (rows N, contraction M)
  auto gemm_y = [&](const double* X, auto epi) -> int {
    return dg::gemm<0>(ctx, dg::GemmArgs{K, ldk, M, N, S, X, N, 0}, epi, q, 0, &launches);
  };
  auto gemm_z = [&](const double* X, auto epi) -> int {
    return dg::gemm<1>(ctx, dg::GemmArgs{K, ldk, N, M, S, X, M, 0}, epi, q, 0, &launches);
  };
  // Y_0 = K V_0, U_1 = A / Y_0
  int rc = gemm_y(slot(Vh, NS, 0), EpiY{A, logA, nullptr, slot(Yh, MS, 0), slot(Uh, MS, 1), nullptr, M, S,
                                        (int)ldd, logdomain ? 1 : 0, flag()});
  if (rc) return rc;
  while (iter < L && err >= tol) {
    ++iter;
    const int l = iter;
    double* Ul = slot(Uh, MS, l);
    // Z_l = K^T U_l; b_l; V_l = b_l / Z_l
    rc = gemm_z(Ul, EpiZ{w, slot(Zh, NS, l), slot(Vh, NS, l), slot(Bh, N, l), N, S, logdomain ? 1 : 0, flag()});
    if (rc) return rc;
    // Y_l = K V_l; U_{l+1} = A / Y_l; residual when the stopping test needs it
    const bool need_err = !fixed || (iter == L);
    rc = gemm_y(slot(Vh, NS, l), EpiY{A, logA, Ul, slot(Yh, MS, l), slot(Uh, MS, l + 1),
                                      need_err ? D : nullptr, M, S, (int)ldd, logdomain ? 1 : 0, flag()});
    if (rc) return rc;
    if (need_err) {
      rc = dg::gemm<1>(ctx, dg::GemmArgs{D, ldd, S, M, S, D, ldd, 0}, dg::EpiStore{gram, S, S}, q, 0, &launches);
      if (rc) return rc;
      if (!fixed) {  // the stopping test needs err now
        std::vector<double> G((size_t)S * S + 1);
        RWIG_CUDA_TRY(cudaMemcpyAsync(G.data(), gram, sizeof(double) * S * S, cudaMemcpyDeviceToHost, q));
        RWIG_CUDA_TRY(cudaMemcpyAsync(G.data() + (size_t)S * S, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, q));
        RWIG_CUDA_TRY(cudaStreamSynchronize(q));
        if (G[(size_t)S * S] != 0.0) {  // out of the scaling form's range: stop, re-run in the log domain
          needs_log = true;
          return 0;
        }
        err_from_gram(G.data());
      }
    }
  }
  RWIG_CUDA_TRY(cudaGetLastError());

  // normalised barycenter and loss (log: before the backward, :268-271;
  // parallel: the backward uses the un-normalised b, :35-42)
  if (iter == 0) {
    // no iteration: the initial b is 0 (parallel, barycenter_impl_parallel.cpp:64)
    // or log b = 0 (log, barycenter_impl_log.cpp:193), normalised as below to
    // 0 / 0 = NaN or 1/N, and the loss taken against b_ext all the same
    fill_kernel<<<grid_for(ctx, N), TPB, 0, q>>>(slot(Bh, N, 0), N, 0.0);
    ++launches;
  }
  normalise_b<<<1, 1024, 0, q>>>(slot(Bh, N, iter), N, logdomain, withgrad ? bext : nullptr, bn, scal);
  ++launches;

  if (withgrad && iter > 0) {
    RWIG_CUDA_TRY(cudaMemsetAsync(gA, 0, sizeof(double) * MS, q));
    RWIG_CUDA_TRY(cudaMemsetAsync(gwp, 0, sizeof(double) * (size_t)ngrp * S, q));
    for (int l = iter; l >= 1; --l) {
      const bool seed = (l == iter);
      const EpiB1 e1{slot(Zh, NS, l), slot(Vh, NS, l), w, slot(Bh, N, l), bn, bext, reg, N, S,
                     logdomain ? 1 : 0, seed ? 1 : 0, T2, gwp, flag()};
      if (seed) {
        seed_b1<<<ngrp, dg::NTH, sizeof(double) * (S + 1) * 8, q>>>(e1, N);
        ++launches;
      } else {
        rc = gemm_z(T, e1);  // K^T T
        if (rc) return rc;
      }
      rc = gemm_y(T2, EpiB2{slot(Uh, MS, l), slot(Yh, MS, l - 1), A, M, S, logdomain ? 1 : 0, gA, T, flag()});  // K T2
      if (rc) return rc;
    }
    reduce_gw<<<S, 256, 0, q>>>(gwp, ngrp, S, gw);
    ++launches;
    if (logdomain) {
      scale_kernel<<<grid_for(ctx, MS), TPB, 0, q>>>(gA, MS, reg);  // :376
      ++launches;
    }
    if (gradA) RWIG_CUDA_TRY(cudaMemcpyAsync(gradA, gA, sizeof(double) * MS, cudaMemcpyDeviceToDevice, q));
    if (gradw) RWIG_CUDA_TRY(cudaMemcpyAsync(gradw, gw, sizeof(double) * S, cudaMemcpyDeviceToDevice, q));
  } else if (withgrad) {  // no iteration to unroll: the gradient is zero
    if (gradA) RWIG_CUDA_TRY(cudaMemsetAsync(gradA, 0, sizeof(double) * MS, q));
    if (gradw) RWIG_CUDA_TRY(cudaMemsetAsync(gradw, 0, sizeof(double) * S, q));
  }

  // outputs: U, V (parallel) or F = eps log U, G = eps log V (log) of the last iteration
  const double* Ufin = slot(Uh, MS, iter > 0 ? iter : 0);
  const double* Vfin = slot(Vh, NS, iter);
  if (iter == 0) {
    fill_kernel<<<grid_for(ctx, MS), TPB, 0, q>>>(slot(Uh, MS, 0), MS, 1.0);  // U = 1 (:67)
    ++launches;
  }
  if (X1) {
    if (logdomain) {
      log_scaled<<<grid_for(ctx, MS), TPB, 0, q>>>(Ufin, MS, reg, X1);
      ++launches;
    } else {
      RWIG_CUDA_TRY(cudaMemcpyAsync(X1, Ufin, sizeof(double) * MS, cudaMemcpyDeviceToDevice, q));
    }
  }
  if (X2) {
    if (logdomain) {
      log_scaled<<<grid_for(ctx, NS), TPB, 0, q>>>(Vfin, NS, reg, X2);
      ++launches;
    } else {
      RWIG_CUDA_TRY(cudaMemcpyAsync(X2, Vfin, sizeof(double) * NS, cudaMemcpyDeviceToDevice, q));
    }
  }
  if (b) RWIG_CUDA_TRY(cudaMemcpyAsync(b, bn, sizeof(double) * N, cudaMemcpyDeviceToDevice, q));
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
  }
};

// Checks of the arguments common to the single and batched entries.
int check_args(const double* A, const double* w, const double* C, const double* bext, int M, int N, int S,
               double reg, int withgrad) {
  if (!A || !w || !C) return set_error(RWIG_E_INVALID, "A, w and C must be non-null");
  if (M < 1 || N < 1 || S < 1) return set_error(RWIG_E_INVALID, "M, N and S must be >= 1");
  if (S > 64) return set_error(RWIG_E_UNSUPPORTED, "more than 64 histograms");
  if (!(reg > 0.0) || !std::isfinite(reg)) return set_error(RWIG_E_INVALID, "reg must be finite and > 0");
  if (withgrad && !bext) return set_error(RWIG_E_INVALID, "b_ext is required with withgrad");
  return 0;
}

// Core driver; all pointers on the device.  Outputs (any may be null):
// U, V (parallel) or F, G (log) as X1, X2; b (normalised); grad_A, grad_w.
// Option "barycenter.log_path" for the log method: 0 (default) the scaling
// form with its range check, re-run in the log domain when it fails; 1 the
// log-domain kernels always; -1 the scaling form only.
int log_path_option() { return (int)option("barycenter.log_path", 0.0); }

// run_log with the call's report filled (device time from ev0 on `st`).
int run_log_reported(Context* ctx, cudaStream_t st, double* X1, double* X2, double* b, double* gradA,
                     double* gradw, double* loss, int* iter_out, double* err_out, const double* A, const double* w,
                     const double* C, const double* bext, int M, int N, int S, double reg, int withgrad,
                     int max_iter, double tol, int prior_launches) {
  int nl = 0, it = 0;
  double er = 0.0;
  const int status = run_log(ctx, st, X1, X2, b, gradA, gradw, loss, &it, &er, A, w, C, bext, M, N, S, reg,
                             withgrad, max_iter, tol, &nl);
  if (status < 0) return status;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  RWIG_CUDA_TRY(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (iter_out) *iter_out = it;
  if (err_out) *err_out = er;
  rwig_report& R = report();
  R.iter = it;
  R.status = status;
  R.err = er;
  R.device_ms = ms;
  R.kernel_ms = ms;
  R.kernel_launches = prior_launches + nl;
  R.fallback_events = 1;
  R.support_m = M;
  R.support_n = N;
  return status;
}

int run(Context* ctx, cudaStream_t st, bool logdomain, double* X1, double* X2, double* b, double* gradA,
        double* gradw, double* loss, int* iter_out, double* err_out, const double* A, const double* w,
        const double* C, const double* bext, int M, int N, int S, double reg, int withgrad, int max_iter,
        double tol) {
  reset_report();
  if (int rc = check_args(A, w, C, bext, M, N, S, reg, withgrad)) return rc;
  const int lp = logdomain ? log_path_option() : 0;
  if (lp == 1) {
    RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
    return run_log_reported(ctx, st, X1, X2, b, gradA, gradw, loss, iter_out, err_out, A, w, C, bext, M, N, S,
                            reg, withgrad, max_iter, tol, 0);
  }
  Solve sv;
  sv.ctx = ctx;
  sv.logdomain = logdomain;
  sv.X1 = X1;
  sv.X2 = X2;
  sv.b = b;
  sv.gradA = gradA;
  sv.gradw = gradw;
  sv.A = A;
  sv.w = w;
  sv.C = C;
  sv.bext = bext;
  sv.M = M;
  sv.N = N;
  sv.S = S;
  sv.reg = reg;
  sv.withgrad = withgrad;
  sv.L = max_iter;
  sv.tol = tol;
  if (int rc = sv.alloc(0)) return rc;
  const bool fixed = sv.fixed;
  const int L = sv.L;
  auto enqueue = [&](cudaStream_t q) { return sv.enqueue(q); };
  int& launches = sv.launches;
  int& iter = sv.iter;
  double& err = sv.err;
  const double *K = sv.K, *Uh = sv.Uh, *Vh = sv.Vh, *Zh = sv.Zh, *Yh = sv.Yh, *Bh = sv.Bh, *logA = sv.logA;
  const double *D = sv.D, *gram = sv.gram, *bn = sv.bn, *scal = sv.scal;
  const double *T = sv.T, *T2 = sv.T2, *gA = sv.gA, *gwp = sv.gwp, *gw = sv.gw;

  // A fixed sequence that repeats the previous call's arguments and buffers
  // is captured once into a CUDA graph and replayed from then on.
  std::vector<unsigned long long> key;
  if (fixed) {
    for (const void* p : {(const void*)X1, (const void*)X2, (const void*)b, (const void*)gradA, (const void*)gradw,
                          (const void*)A, (const void*)w, (const void*)C, (const void*)bext, (const void*)st,
                          (const void*)K, (const void*)Uh, (const void*)Vh, (const void*)Zh, (const void*)Yh,
                          (const void*)Bh, (const void*)logA, (const void*)D, (const void*)gram, (const void*)bn,
                          (const void*)scal, (const void*)T, (const void*)T2, (const void*)gA, (const void*)gwp,
                          (const void*)gw})
      key.push_back((unsigned long long)(uintptr_t)p);
    unsigned long long r;
    std::memcpy(&r, &reg, sizeof(r));
    for (unsigned long long v : {(unsigned long long)M, (unsigned long long)N, (unsigned long long)S, r,
                                 (unsigned long long)withgrad, (unsigned long long)L, options_generation()})
      key.push_back(v);
  }
  const int site = logdomain ? kGraphBaryLog : kGraphBaryParallel;
  GraphEntry& ge = ctx->graphs[site];
  // graphs are captured and launched on the engine's own stream, fenced
  // against the caller's stream by events (the legacy default stream cannot
  // be captured)
  const cudaStream_t gs = ctx->stream;
  auto fence = [&](cudaStream_t from, cudaStream_t to) -> int {
    if (from == to) return 0;
    RWIG_CUDA_TRY(cudaEventRecord(ctx->evk, from));
    RWIG_CUDA_TRY(cudaStreamWaitEvent(to, ctx->evk, 0));
    return 0;
  };
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
  if (fixed && ge.exec && ge.key == key) {
    if (fence(st, gs)) return RWIG_E_CUDA;
    RWIG_CUDA_TRY(cudaGraphLaunch(ge.exec, gs));
    if (fence(gs, st)) return RWIG_E_CUDA;
    launches = ge.launches;
    iter = L;
  } else if (fixed && ctx->seen[site] == key) {
    cudaGraph_t graph = nullptr;
    if (fence(st, gs)) return RWIG_E_CUDA;
    RWIG_CUDA_TRY(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue(gs);
    const cudaError_t ce = cudaStreamEndCapture(gs, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    cudaGraphExec_t exec = nullptr;
    cudaError_t ie = ce;
    if (ce == cudaSuccess) {
      ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
    }
    if (ie != cudaSuccess) {
      // capture or instantiation refused: run this call eagerly, stop trying
      (void)cudaGetLastError();
      ctx->seen[site].clear();
      const int rc2 = enqueue(st);
      if (rc2) return rc2;
    } else {
      if (ge.exec) cudaGraphExecDestroy(ge.exec);
      ge.exec = exec;
      ge.key = key;
      ge.launches = launches;
      RWIG_CUDA_TRY(cudaGraphLaunch(exec, gs));
      if (fence(gs, st)) return RWIG_E_CUDA;
    }
  } else {
    const int rc = enqueue(st);
    if (rc) return rc;
    if (fixed) ctx->seen[site] = key;
  }
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  double sc[3] = {0.0, 0.0, 0.0};
  RWIG_CUDA_TRY(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
  std::vector<double> G;
  if (fixed && iter > 0) {
    G.resize((size_t)S * S);
    RWIG_CUDA_TRY(cudaMemcpyAsync(G.data(), gram, sizeof(double) * S * S, cudaMemcpyDeviceToHost, st));
  }
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  RWIG_CUDA_TRY(cudaGetLastError());
  if (logdomain && lp == 0 && (sv.needs_log || sc[2] != 0.0))
    return run_log_reported(ctx, st, X1, X2, b, gradA, gradw, loss, iter_out, err_out, A, w, C, bext, M, N, S,
                            reg, withgrad, max_iter, tol, launches);
  if (fixed && iter > 0) sv.err_from_gram(G.data());
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

// Side streams of the batched entry: the context's (engine.h).
constexpr int kSideStreams = Context::kSideStreams;

// First scratch slot of the solves enqueued on side stream i (clear of every
// other entry's slot numbers).  Solves on one stream run in stream order, so
// they share one slot set, grown to the largest of them.
constexpr int kBatchSlotBase = 1000, kBatchSlotStride = 32;

// Many barycenter problems: those with a fixed iteration count enqueued
// side by side on the side streams (each with its own scratch slots), their
// Gram matrices and scalars copied to pinned memory, one wait at the end;
// the others through run() one after another.
int run_batch(Context* ctx, cudaStream_t st, const rwig_bary_problem* probs, int count, rwig_bary_result* out) {
  reset_report();
  std::vector<Solve> sv((size_t)count);
  std::vector<int> fixed_ids, serial_ids;
  for (int i = 0; i < count; ++i) {
    const rwig_bary_problem& q = probs[i];
    out[i] = rwig_bary_result{0.0, 0.0, 0, 0};
    const int rc = (q.method == 0 || q.method == 1)
                       ? check_args(q.A, q.w, q.C, q.b_ext, q.M, q.N, q.S, q.reg, q.withgrad)
                       : set_error(RWIG_E_INVALID, "method must be 0 (parallel) or 1 (log)");
    if (rc) {
      out[i].status = rc;
      continue;
    }
    if (q.zero_tol > 0.0 || (q.method == 1 && log_path_option() == 1)) {
      serial_ids.push_back(i);
      continue;
    }
    Solve& s = sv[i];
    s.ctx = ctx;
    s.logdomain = q.method == 1;
    s.X1 = q.X1;
    s.X2 = q.X2;
    s.b = q.b;
    s.gradA = q.grad_A;
    s.gradw = q.grad_w;
    s.A = q.A;
    s.w = q.w;
    s.C = q.C;
    s.bext = q.b_ext;
    s.M = q.M;
    s.N = q.N;
    s.S = q.S;
    s.reg = q.reg;
    s.withgrad = q.withgrad;
    s.L = q.max_iter;
    s.tol = q.zero_tol;
    const int rc2 = s.alloc(kBatchSlotBase + kBatchSlotStride * (int)(fixed_ids.size() % kSideStreams));
    if (rc2) {
      out[i].status = rc2;
      continue;
    }
    fixed_ids.push_back(i);
  }
  // a later, larger solve on the same stream may have regrown a slot: take
  // every solve's pointers again now that the slots have their final sizes
  for (size_t k = 0; k < fixed_ids.size(); ++k) {
    Solve& s = sv[fixed_ids[k]];
    if (const int rc = s.alloc(kBatchSlotBase + kBatchSlotStride * (int)(k % kSideStreams))) return rc;
  }
  int launches = 0;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
  if (!fixed_ids.empty()) {
    // pinned results: per solve the Gram matrix (S x S) and two scalars
    size_t need = 0;
    std::vector<size_t> at(fixed_ids.size());
    for (size_t k = 0; k < fixed_ids.size(); ++k) {
      at[k] = need;
      need += (size_t)sv[fixed_ids[k]].S * sv[fixed_ids[k]].S + 3;
    }
    if (ctx->pinned_bytes < need * sizeof(double)) {
      if (ctx->pinned) cudaFreeHost(ctx->pinned);
      ctx->pinned = nullptr;
      ctx->pinned_bytes = 0;
      RWIG_CUDA_TRY(cudaHostAlloc(&ctx->pinned, need * sizeof(double), cudaHostAllocDefault));
      ctx->pinned_bytes = need * sizeof(double);
    }
    double* hp = (double*)ctx->pinned;
    RWIG_CUDA_TRY(cudaEventRecord(ctx->evk, st));  // inputs ready on the caller's stream
    bool used[kSideStreams] = {};
    // on an error part-way, wait for what was enqueued (it writes the
    // caller's outputs and the pinned buffer) and mark the rest as failed
    auto fail_from = [&](size_t k0, int rc) -> int {
      for (int si = 0; si < kSideStreams; ++si)
        if (used[si]) cudaStreamSynchronize(ctx->side[si]);
      for (size_t k = k0; k < fixed_ids.size(); ++k) out[fixed_ids[k]].status = rc;
      return rc;
    };
    for (size_t k = 0; k < fixed_ids.size(); ++k) {
      Solve& s = sv[fixed_ids[k]];
      const int si = (int)(k % kSideStreams);
      cudaStream_t q = side_stream(ctx, si);
      if (!q) return fail_from(k, set_error(RWIG_E_CUDA, "could not create a side stream"));
      if (!used[si] && cudaStreamWaitEvent(q, ctx->evk, 0) != cudaSuccess)
        return fail_from(k, set_error(RWIG_E_CUDA, "cudaStreamWaitEvent on a side stream failed"));
      used[si] = true;
      if (int rc = s.enqueue(q)) return fail_from(k, rc);
      launches += s.launches;
      if (cudaMemcpyAsync(hp + at[k], s.gram, sizeof(double) * s.S * s.S, cudaMemcpyDeviceToHost, q) !=
              cudaSuccess ||
          cudaMemcpyAsync(hp + at[k] + (size_t)s.S * s.S, s.scal, sizeof(double) * 3, cudaMemcpyDeviceToHost,
                          q) != cudaSuccess)
        return fail_from(k, set_error(RWIG_E_CUDA, "result copy of a batched barycenter failed"));
    }
    for (int si = 0; si < kSideStreams; ++si)
      if (used[si]) RWIG_CUDA_TRY(cudaStreamSynchronize(ctx->side[si]));
    RWIG_CUDA_TRY(cudaGetLastError());
    // log problems whose scaling form left its range: re-run in the log domain
    const int lp = log_path_option();
    for (size_t k = 0; k < fixed_ids.size(); ++k) {
      Solve& s = sv[fixed_ids[k]];
      if (!(s.logdomain && lp == 0 && hp[at[k] + (size_t)s.S * s.S + 2] != 0.0)) continue;
      const rwig_bary_problem& q = probs[fixed_ids[k]];
      rwig_bary_result& r = out[fixed_ids[k]];
      int nl = 0;
      const int rc = run_log(ctx, st, q.X1, q.X2, q.b, q.grad_A, q.grad_w, &r.loss, &r.iter, &r.err, q.A, q.w, q.C,
                             q.b_ext, q.M, q.N, q.S, q.reg, q.withgrad, q.max_iter, q.zero_tol, &nl);
      launches += nl;
      r.status = rc;
      s.iter = -1;  // done
    }
    for (size_t k = 0; k < fixed_ids.size(); ++k) {
      Solve& s = sv[fixed_ids[k]];
      rwig_bary_result& r = out[fixed_ids[k]];
      if (s.iter < 0) continue;
      if (s.iter > 0) s.err_from_gram(hp + at[k]);
      r.loss = s.withgrad ? hp[at[k] + (size_t)s.S * s.S + 1] : 0.0;
      r.err = s.err;
      r.iter = s.iter;
      r.status = (s.err <= s.tol) ? 0 : (s.iter == s.L ? 1 : 2);
    }
  }
  for (int i : serial_ids) {
    const rwig_bary_problem& q = probs[i];
    int it = 0;
    double loss = 0.0, err = 0.0;
    const int rc = run(ctx, st, q.method == 1, q.X1, q.X2, q.b, q.grad_A, q.grad_w, &loss, &it, &err, q.A, q.w, q.C,
                       q.b_ext, q.M, q.N, q.S, q.reg, q.withgrad, q.max_iter, q.zero_tol);
    launches += report().kernel_launches;
    out[i] = rwig_bary_result{loss, err, it, rc};
  }
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  RWIG_CUDA_TRY(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  reset_report();
  rwig_report& R = report();
  R.device_ms = ms;
  R.kernel_ms = ms;
  R.kernel_launches = launches;
  return 0;
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
  return bary::run(ctx, call_stream(ctx, stream), false, U, V, b, grad_A, grad_w, loss, iter,
                   err, A, w, C, b_ext, M, N, S, reg, withgrad, max_iter, zero_tol);
}

extern "C" int rwig_batch_barycenter_dev(const rwig_bary_problem* probs, int count, rwig_bary_result* out,
                                         void* stream) {
  if (count < 0 || (count > 0 && (!probs || !out))) return set_error(RWIG_E_INVALID, "bad problem array");
  if (count == 0) return 0;
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return bary::run_batch(ctx, call_stream(ctx, stream), probs, count, out);
}

extern "C" int rwig_barycenter_log_dev(double* F, double* G, double* b, double* grad_A, double* grad_w,
                                       double* loss, int* iter, double* err, const double* A, const double* w,
                                       const double* C, const double* b_ext, int M, int N, int S, double reg,
                                       int withgrad, int max_iter, double zero_tol, void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return bary::run(ctx, call_stream(ctx, stream), true, F, G, b, grad_A, grad_w, loss, iter,
                   err, A, w, C, b_ext, M, N, S, reg, withgrad, max_iter, zero_tol);
}
