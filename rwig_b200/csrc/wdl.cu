// wdl.cu -- Wasserstein dictionary learning (WassersteinDictionaryLearning,
// src/wdl_impl.cpp; GPU path cuda_wdl, src/cuda_wdl.cu).
//
// Batched step (_train_batch_batched, wdl_impl.cpp:87-247; wdl_batch,
// cuda_wdl.cu:385): the D documents of a batch are D parallel barycenters
// sharing the topics A (N x S) and K = exp(-C/eps), stacked as SD = S*D
// columns (column d*S + s).  Forward, L fixed iterations l = 0..L-1:
//   KVB_l = K VB_l (VB_0 = 1),  UB_{l+1} = A_tiled / KVB_l,
//   KTUB_{l+1} = K^T UB_{l+1},  bB_{l+1}[:,d] = prod_s KTUB[:,dS+s]^{W_B[s,d]},
//   VB_{l+1} = bB_{l+1} / KTUB_{l+1};
// backward l = L..1 (the parallel-barycenter adjoint, per document):
//   l = L: bBbar = 2 (bB_L - Y_B), T2 = (bBbar W_B) o VB_L
//   l < L: VBbar = -K^T T, bBbar = sum_s VBbar / KTUB_l,
//          T2 = (bBbar W_B - VBbar / KTUB_l) o VB_l
//   UBbar = K T2;  ABbar += UBbar / KVB_{l-1};  T = UBbar o UB_l / KVB_{l-1}
//   wBbar += log(KTUB_l)^T (bBbar o bB_l)
// then the softmax Jacobians and the batch means (:223-243).  Each product
// is one FP64 tensor-core GEMM (dgemm.cuh) over all SD columns, its column
// tiles holding whole documents, with the elementwise work fused into the
// epilogue; every reduction runs in a fixed order.
//
// Training (_compute_serial, wdl_impl.cpp:254-347; cuda_wdl.cu:539-730):
// per batch the step above, one optimizer update of the logits Alpha (N x S)
// and Lambda (S x M) -- the Lambda gradient is g_lambda broadcast to every
// document (:246) -- and the column softmaxes A = softmax(Alpha),
// W = softmax(Lambda).  Inference (:349-377): the parallel barycenter of
// every document under the learned A and W.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "barycenter.h"
#include "dgemm.cuh"
#include "engine.h"
#include "ozaki.cuh"

namespace rwig {
namespace wdl {

constexpr int TPB = 256;

int grid_for(const Context* ctx, long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + TPB - 1) / TPB, 8LL * ctx->sm_count));
}

__global__ void gibbs(const double* C, int N, long long ldk, double reg, double* K) {
  const long long total = ldk * (long long)N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldk), j = (int)(k / ldk);
    K[k] = (i < N) ? exp(-C[i + (long long)j * N] / reg) : 0.0;
  }
}

// K given: copy into the padded layout.
__global__ void copy_k(const double* Kin, int N, long long ldk, double* K) {
  const long long total = ldk * (long long)N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldk), j = (int)(k / ldk);
    K[k] = (i < N) ? Kin[i + (long long)j * N] : 0.0;
  }
}

__global__ void fill(double* x, long long n, double v) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    x[k] = v;
}

// ---------------------------------------------------------------------------
// GEMM epilogues over document groups of S columns (tile columns are whole
// groups, c0 a multiple of S); W = S*D columns in all.
// ---------------------------------------------------------------------------
// After KVB_l = K VB_l: store it and UB_{l+1} = A_tiled / KVB_l.
struct EpiY {
  const double* A;
  int N, S, W;
  double* KVB;
  double* UB;
  __device__ void operator()(int r0, int nr, int c0, int nc, double* t, int ldt, double*) const {
    if (nr <= 0) return;
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      if (gc >= W) continue;
      const int i = r0 + r;
      const size_t k = (size_t)i + (size_t)gc * N;
      const double y = t[c * ldt + r];
      KVB[k] = y;
      UB[k] = A[i + (size_t)(gc % S) * N] / y;
    }
  }
};

// After KTUB = K^T UB: store it, the barycenters bB (N x D) and VB = bB / KTUB.
struct EpiZ {
  const double* Wb;  // S x D weights of the batch, flat index = column
  int N, S, W;
  double* KTUB;
  double* VB;
  double* bB;
  __device__ void operator()(int r0, int nr, int c0, int nc, double* t, int ldt, double* ws) const {
    if (nr <= 0) return;
    double* wb = ws + nc * ldt;  // per (group, row) barycenter entry
    const int ng = nc / S;
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      ws[c * ldt + r] = gc < W ? pow(t[c * ldt + r], Wb[gc]) : 1.0;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < nr * ng; p += blockDim.x) {
      const int r = p % nr, q = p / nr, g0 = c0 + q * S;
      if (g0 >= W) continue;
      double acc = 1.0;  // barycenter_impl_parallel.cpp:120 order
      for (int s = 0; s < S; ++s) acc *= ws[(q * S + s) * ldt + r];
      bB[(size_t)(r0 + r) + (size_t)(g0 / S) * N] = acc;
      wb[q * ldt + r] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      if (gc >= W) continue;
      const size_t k = (size_t)(r0 + r) + (size_t)gc * N;
      const double z = t[c * ldt + r];
      KTUB[k] = z;
      VB[k] = wb[(c / S) * ldt + r] / z;
    }
  }
};

// Backward after K^T T (t == nullptr at the seed step L, which has no
// product): bBbar per (row, document), the next operand T2 and the wBbar
// shares, summed per 8-row group into gw_part[(j/8)*W + column].
struct EpiB1 {
  const double* KTU;  // KTUB_l
  const double* VB;   // VB_l
  const double* Wb;
  const double* bBl;  // bB_l (N x D)
  const double* Yb;   // documents of the batch (N x D)
  int N, S, W, seed;
  double* T2;
  double* gw_part;
  __device__ void operator()(int r0, int nr, int c0, int nc, double* t, int ldt, double* ws) const {
    if (nr <= 0) return;
    double* wg = ws + nc * ldt;  // bBbar per (group, row)
    const int ng = nc / S;
    if (!seed) {
      for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
        const int r = e % nr, c = e / nr, gc = c0 + c;
        if (gc >= W) continue;
        const size_t k = (size_t)(r0 + r) + (size_t)gc * N;
        ws[c * ldt + r] = (-t[c * ldt + r]) / KTU[k];  // VBbar / KTUB_l
      }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < nr * ng; p += blockDim.x) {
      const int r = p % nr, q = p / nr, g0 = c0 + q * S;
      if (g0 >= W) continue;
      const size_t jd = (size_t)(r0 + r) + (size_t)(g0 / S) * N;
      double bb;
      if (seed) {
        bb = 2.0 * (bBl[jd] - Yb[jd]);  // wdl_impl.cpp:176
      } else {
        bb = 0.0;
        for (int s = 0; s < S; ++s) bb += ws[(q * S + s) * ldt + r];
      }
      wg[q * ldt + r] = bb;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      if (gc >= W) {
        ws[c * ldt + r] = 0.0;
        continue;
      }
      const size_t k = (size_t)(r0 + r) + (size_t)gc * N;
      const double bb = wg[(c / S) * ldt + r];
      double tt = bb * Wb[gc];
      if (!seed) tt -= (-t[c * ldt + r]) / KTU[k];
      T2[k] = tt * VB[k];
      ws[c * ldt + r] = log(KTU[k]) * (bb * bBl[(size_t)(r0 + r) + (size_t)(gc / S) * N]);
    }
    __syncthreads();
    const int n8 = (nr + 7) / 8;
    for (int p = threadIdx.x; p < n8 * nc; p += blockDim.x) {
      const int c = p % nc, g8 = p / nc, gc = c0 + c;
      if (gc >= W) continue;
      double v = 0.0;
      for (int r = g8 * 8; r < min(nr, g8 * 8 + 8); ++r) v += ws[c * ldt + r];
      gw_part[(size_t)(r0 / 8 + g8) * W + gc] += v;
    }
  }
};

// Backward after UBbar = K T2: ABbar += UBbar / KVB_{l-1} and the next
// step's operand T = UBbar o UB_l / KVB_{l-1}.
struct EpiB2 {
  const double* UBl;
  const double* KVBprev;
  int N, W;
  double* ABbar;
  double* T;
  __device__ void operator()(int r0, int nr, int c0, int nc, double* t, int ldt, double*) const {
    if (nr <= 0) return;
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      if (gc >= W) continue;
      const size_t k = (size_t)(r0 + r) + (size_t)gc * N;
      const double y = t[c * ldt + r];
      ABbar[k] += y / KVBprev[k];
      T[k] = (y * UBl[k]) / KVBprev[k];
    }
  }
};

// The seed step: EpiB1 over 8-row groups x column tiles, without a product.
__global__ void seed_b1(EpiB1 epi, int N, int tc) {
  extern __shared__ double ws[];  // 2 * tc * 8
  const int r0 = blockIdx.x * 8, c0 = blockIdx.y * tc;
  epi(r0, min(8, N - r0), c0, tc, nullptr, 8, ws);
}

// dot[c] = sum_i A[i, c % S] * X[i, c]; one block per column, fixed tree.
__global__ void col_dots(const double* A, const double* X, int N, int S, double* dot) {
  __shared__ double sh[TPB];
  const int c = blockIdx.x, s = c % S;
  double v = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) v += A[i + (size_t)s * N] * X[i + (size_t)c * N];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) dot[c] = sh[0];
}

// g_Alpha[i,s] = sum_d (a x_d - a dot_d) / D with a = A[i,s], x_d = ABbar[i, dS+s]
// (softmax Jacobian per column, wdl_impl.cpp:223-228, then the batch mean :236-238).
__global__ void alpha_grad(const double* A, const double* X, const double* dot, int N, int S, int D, double* g) {
  const long long total = (long long)N * S;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % N), s = (int)(k / N);
    const double a = A[k];
    double acc = 0.0;
    for (int d = 0; d < D; ++d) {
      const int c = d * S + s;
      acc += a * X[i + (size_t)c * N] - a * dot[c];
    }
    g[k] = acc / D;
  }
}

// out[c] = sum over the 8-row groups of part[q*W + c]; one block per column.
__global__ void reduce_cols(const double* part, int ngrp, int W, double* out) {
  __shared__ double sh[TPB];
  const int c = blockIdx.x;
  double v = 0.0;
  for (int q = threadIdx.x; q < ngrp; q += blockDim.x) v += part[(size_t)q * W + c];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = sh[0];
}

// Softmax Jacobian of every document's weights (wdl_impl.cpp:229-233) and the
// batch mean g_lambda (:239-243); x = wBbar (S x D), updated in place.
__global__ void lambda_grad(const double* Wb, double* x, int S, int D, double* gl) {
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    const double* wd = Wb + (size_t)d * S;
    double* xd = x + (size_t)d * S;
    double dot = 0.0;
    for (int s = 0; s < S; ++s) dot += wd[s] * xd[s];
    for (int s = 0; s < S; ++s) xd[s] = wd[s] * xd[s] - wd[s] * dot;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double acc = 0.0;
    for (int d = 0; d < D; ++d) acc += x[s + (size_t)d * S];
    gl[s] = acc / D;
  }
}

// Column softmax of an r x c matrix (wdl_impl.hpp:80-96; cuda_wdl.cu:45),
// one block per column, fixed-order trees.
__global__ void col_softmax(const double* X, int r, double* out) {
  __shared__ double sh[TPB];
  const double* x = X + (size_t)blockIdx.x * r;
  double* o = out + (size_t)blockIdx.x * r;
  double mx = -INFINITY;
  for (int i = threadIdx.x; i < r; i += blockDim.x) mx = fmax(mx, x[i]);
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + h]);
    __syncthreads();
  }
  mx = sh[0];
  __syncthreads();
  double sum = 0.0;
  for (int i = threadIdx.x; i < r; i += blockDim.x) {
    const double e = exp(x[i] - mx);
    o[i] = e;
    sum += e;
  }
  sh[threadIdx.x] = sum;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  sum = sh[0];
  for (int i = threadIdx.x; i < r; i += blockDim.x) o[i] = o[i] / sum;
}

// One optimizer update (optimizer.hpp:72-99; cuda_optimizer.cu:64): opt 0 SGD,
// 1 Adam, 2 AdamW; c1 = 1 - beta1^step, c2 = 1 - beta2^step.  The gradient of
// element k is g[gmod ? k % gmod : k] (gmod = S broadcasts g_lambda over the
// documents).
__global__ void opt_step(double* th, double* m, double* v, const double* g, int gmod, long long n, int opt,
                         double eta, double gamma, double b1, double b2, double eps, double c1, double c2) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const double gk = g[gmod ? k % gmod : k];
    if (opt == 0) {
      th[k] = th[k] - eta * gk;
      continue;
    }
    m[k] = b1 * m[k] + (1.0 - b1) * gk;
    v[k] = b2 * v[k] + (1.0 - b2) * (gk * gk);
    const double mh = m[k] / c1, vh = v[k] / c2;
    if (opt == 1) th[k] = th[k] - eta * (mh / (sqrt(vh) + eps));
    else th[k] = (1.0 - eta * gamma) * th[k] - eta * (mh / (sqrt(vh) + eps));
  }
}

enum {
  SW_UH = 120, SW_VH, SW_KVH, SW_KTH, SW_BH, SW_T, SW_T2, SW_AB, SW_GWP, SW_DOT, SW_WBAR, SW_K,
  SW_Y, SW_C, SW_ALPHA, SW_LAMBDA, SW_A, SW_W, SW_MA, SW_VA, SW_ML, SW_VL, SW_GA, SW_GL, SW_YHAT,
  SW_HA, SW_HW, SW_HY, SW_HK, SW_HOUT, SW_IU, SW_IV, SW_IKV, SW_IKT, SW_IB, SW_IERR, SW_IST, SW_VCK
};

// Columns per GEMM tile: whole documents, at most 64.
int tile_cols(int S, int SD) { return std::min((64 / S) * S, SD); }

// ---------------------------------------------------------------------------
// Inference (wdl_impl.cpp:349-377; cuda_wdl.cu:754-776): the parallel
// barycenter of every document, each with its own stopping test
// (Barycenter::compute_parallel: `iter < max_iter && err >= tol`, err the
// Frobenius norm of U o KV - A).  The reference solves the documents one by
// one; here a chunk of documents is one set of stacked columns, as in the
// training step, and a document whose test stops it is frozen: the
// epilogues skip its columns, so its state -- and its barycenter -- stays
// that of its own last iteration.
// ---------------------------------------------------------------------------
// After KVB = K VB: store KVB and UB = A / KVB for the running documents;
// unless `first`, the squared residual (U_l o KVB - A, with U_l the UB this
// overwrites) summed over each row's S columns -> errp[document * N + row]
// (one entry per row whatever rows the GEMM hands this call: with split-K a
// tile's rows are divided among the cluster's CTAs).
struct EpiYInf {
  const double* A;
  const int* active;
  int N, S, W, D, first;
  double* KVB;
  double* UB;
  double* errp;
  __device__ void operator()(int r0, int nr, int c0, int nc, double* t, int ldt, double* ws) const {
    if (nr <= 0) return;
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      double sq = 0.0;
      if (gc < W && active[gc / S]) {
        const int i = r0 + r;
        const size_t k = (size_t)i + (size_t)gc * N;
        const double y = t[c * ldt + r];
        const double a = A[i + (size_t)(gc % S) * N];
        if (!first) {
          const double res = UB[k] * y - a;
          sq = res * res;
        }
        KVB[k] = y;
        UB[k] = a / y;
      }
      ws[c * ldt + r] = sq;
    }
    if (first) return;
    __syncthreads();
    const int ng = nc / S;
    for (int p = threadIdx.x; p < nr * ng; p += blockDim.x) {
      const int r = p % nr, q = p / nr, g0 = c0 + q * S;
      if (g0 >= W) continue;
      double acc = 0.0;
      for (int s = 0; s < S; ++s) acc += ws[(q * S + s) * ldt + r];
      errp[(size_t)(g0 / S) * N + r0 + r] = acc;
    }
  }
};

// After KTUB = K^T UB: for the running documents KTUB, their barycenters bB
// and VB = bB / KTUB (EpiZ's arithmetic).
struct EpiZInf {
  const double* Wb;
  const int* active;
  int N, S, W;
  double* KTUB;
  double* VB;
  double* bB;
  __device__ void operator()(int r0, int nr, int c0, int nc, double* t, int ldt, double* ws) const {
    if (nr <= 0) return;
    double* wb = ws + nc * ldt;
    const int ng = nc / S;
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      ws[c * ldt + r] = gc < W ? pow(t[c * ldt + r], Wb[gc]) : 1.0;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < nr * ng; p += blockDim.x) {
      const int r = p % nr, q = p / nr, g0 = c0 + q * S;
      if (g0 >= W || !active[g0 / S]) continue;
      double acc = 1.0;  // barycenter_impl_parallel.cpp:120 order
      for (int s = 0; s < S; ++s) acc *= ws[(q * S + s) * ldt + r];
      bB[(size_t)(r0 + r) + (size_t)(g0 / S) * N] = acc;
      wb[q * ldt + r] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr, gc = c0 + c;
      if (gc >= W || !active[gc / S]) continue;
      const size_t k = (size_t)(r0 + r) + (size_t)gc * N;
      const double z = t[c * ldt + r];
      KTUB[k] = z;
      VB[k] = wb[(c / S) * ldt + r] / z;
    }
  }
};

// One iteration's bookkeeping, one block per document: err = sqrt of the
// document's per-row residual sums (256 strided partial sums, then a tree:
// a fixed order), then the stopping test.  state[d] = iterations run,
// state[D + d] = running flag, state[2 D] counts the documents still running.
__global__ void infer_update(const double* errp, int N, int D, int L, double tol, int* state) {
  __shared__ double sh[256];
  const int d = blockIdx.x;
  if (!state[D + d]) return;  // the same for every thread of the block
  double acc = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) acc += errp[(size_t)d * N + j];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double err = sqrt(sh[0]);
    const int it = ++state[d];
    if (!(it < L && err >= tol)) {
      state[D + d] = 0;
      atomicSub(state + 2 * D, 1);
    }
  }
}

__global__ void infer_init(int D, int* state) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < D; d += gridDim.x * blockDim.x) {
    state[d] = 0;
    state[D + d] = 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) state[2 * D] = D;
}

// Yhat[:, d] = bB[:, d] / sum(bB[:, d]) (normalise_b's order: 1024 strided
// partial sums, then a tree).
__global__ void infer_output(const double* bB, int N, double* Yhat) {
  __shared__ double sh[1024];
  const double* b = bB + (size_t)blockIdx.x * N;
  double acc = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) acc += b[j];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double tot = sh[0];
  for (int j = threadIdx.x; j < N; j += blockDim.x) Yhat[(size_t)blockIdx.x * N + j] = b[j] / tot;
}

// Inference of documents [0, M): A (N x S), W (S x M), K padded (ldk); Yhat
// (N x M).  Chunks of at most wdl.infer_docs documents (default 1024).
int infer(Context* ctx, cudaStream_t st, const double* A, const double* W, const double* K, long long ldk, int N,
          int S, int M, int L, double tol, double* Yhat, int* launches, const oz::Prepared* pr) {
  const int chunk = std::max(1, std::min(M, (int)option("wdl.infer_docs", 1024.0)));
  const size_t NWc = (size_t)N * S * chunk;
  double* UB = (double*)scratch(ctx, SW_IU, sizeof(double) * NWc);
  double* VB = (double*)scratch(ctx, SW_IV, sizeof(double) * NWc);
  double* KV = (double*)scratch(ctx, SW_IKV, sizeof(double) * NWc);
  double* KT = (double*)scratch(ctx, SW_IKT, sizeof(double) * NWc);
  double* bB = (double*)scratch(ctx, SW_IB, sizeof(double) * (size_t)N * chunk);
  double* errp = (double*)scratch(ctx, SW_IERR, sizeof(double) * (size_t)N * chunk);
  int* state = (int*)scratch(ctx, SW_IST, sizeof(int) * (2 * (size_t)chunk + 1));
  if (!UB || !VB || !KV || !KT || !bB || !errp || !state) return RWIG_E_NOMEM;
  for (int m0 = 0; m0 < M; m0 += chunk) {
    const int D = std::min(chunk, M - m0);
    const int SD = S * D;
    const size_t NW = (size_t)N * SD;
    const double* Wb = W + (size_t)m0 * S;
    const int tc = tile_cols(S, SD);
    auto gemm = [&](int trans, const double* X, auto epi) -> int {
      if (pr) return oz::gemm(ctx, *pr, trans, X, N, SD, tc, epi, st, launches);
      const dg::GemmArgs g{K, ldk, N, N, SD, X, N, 0, tc};
      return trans ? dg::gemm<1>(ctx, g, epi, st, 0, launches) : dg::gemm<0>(ctx, g, epi, st, 0, launches);
    };
    fill<<<grid_for(ctx, NW), TPB, 0, st>>>(VB, NW, 1.0);
    infer_init<<<std::max(1, (D + 255) / 256), 256, 0, st>>>(D, state);
    *launches += 2;
    int rc = gemm(0, VB, EpiYInf{A, state + D, N, S, SD, D, 1, KV, UB, errp});  // U_1 = A / K 1
    if (rc) return rc;
    for (int l = 0; l < L; ++l) {
      rc = gemm(1, UB, EpiZInf{Wb, state + D, N, S, SD, KT, VB, bB});
      if (rc) return rc;
      rc = gemm(0, VB, EpiYInf{A, state + D, N, S, SD, D, 0, KV, UB, errp});
      if (rc) return rc;
      infer_update<<<D, 256, 0, st>>>(errp, N, D, L, tol, state);
      ++*launches;
      if (tol > 0.0 && l + 1 < L) {  // stop early once every document has stopped
        int running = 0;
        RWIG_CUDA_TRY(cudaMemcpyAsync(&running, state + 2 * D, sizeof(int), cudaMemcpyDeviceToHost, st));
        RWIG_CUDA_TRY(cudaStreamSynchronize(st));
        if (running == 0) break;
      }
    }
    infer_output<<<D, 1024, 0, st>>>(bB, N, Yhat + (size_t)m0 * N);
    ++*launches;
    RWIG_CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

// Batched gradient on device buffers: K padded (ldk), A (N x S), Wb (S x D),
// Yb (N x D); outputs gA (N x S) and gl (S).
//
// Checkpointing (option "wdl.checkpoint" = k, 0 or >= L: none).  The state
// the backward step l reads -- KVB_{l-1}, UB_l, KTUB_l, VB_l, bB_l -- is what
// forward iteration l-1 writes from VB_{l-1} alone.  The forward keeps VB at
// every k-th iteration (VB_0, VB_k, ...) and the full state of one segment of
// k iterations; the backward runs the segments newest first, recomputing each
// earlier segment's states from its checkpoint into the segment buffers
// before unrolling it.  The recomputation runs the same products on the same
// inputs, so the gradient is bitwise that of the full history; it costs
// 2 (L - k') extra products (k' the last segment's length) and holds
// ceil(L / k) + 4 k + 3 state slots of N x S D doubles instead of 4 (L + 1).
int batch_grad(Context* ctx, cudaStream_t st, double* gA, double* gl, const double* A, const double* Wb,
               const double* Yb, const double* K, long long ldk, int N, int S, int D, int L, int* launches,
               const oz::Prepared* pr) {
  const int SD = S * D;
  const size_t NW = (size_t)N * SD, ND = (size_t)N * D;
  if (L <= 0) {
    RWIG_CUDA_TRY(cudaMemsetAsync(gA, 0, sizeof(double) * N * S, st));
    RWIG_CUDA_TRY(cudaMemsetAsync(gl, 0, sizeof(double) * S, st));
    return 0;
  }
  const int kopt = (int)option("wdl.checkpoint", 0.0);
  const int k = (kopt <= 0 || kopt >= L) ? L : kopt;  // segment length
  const int nseg = (L + k - 1) / k;
  const int ngrp = (N + 7) / 8;
  // Option wdl.halves = 2 runs the batch's documents as two independent
  // halves on two streams (the documents of a batch share nothing until the
  // final means), for one half's tensor-core products to overlap the other
  // half's residue and reconstruction kernels; one stream is the default,
  // measured as fast on the 5000-word batch.
  const int halves = (pr && D >= 2 && (int)option("wdl.halves", 1.0) >= 2) ? 2 : 1;
  // segment buffers, local index t = l - j k (t = 0..k); V's slot 0 is the checkpoint
  double* Us = (double*)scratch(ctx, SW_UH, sizeof(double) * NW * (k + 1));
  double* Vs = (double*)scratch(ctx, SW_VH, sizeof(double) * NW * (k + 1));
  double* KVs = (double*)scratch(ctx, SW_KVH, sizeof(double) * NW * k);
  double* KTs = (double*)scratch(ctx, SW_KTH, sizeof(double) * NW * (k + 1));
  double* Bs = (double*)scratch(ctx, SW_BH, sizeof(double) * ND * (k + 1));
  double* Vck = (double*)scratch(ctx, SW_VCK, sizeof(double) * NW * nseg);  // VB_{j k}
  double* T = (double*)scratch(ctx, SW_T, sizeof(double) * NW);
  double* T2 = (double*)scratch(ctx, SW_T2, sizeof(double) * NW);
  double* AB = (double*)scratch(ctx, SW_AB, sizeof(double) * NW);
  double* gwp = (double*)scratch(ctx, SW_GWP, sizeof(double) * (size_t)ngrp * SD);  // per half: [ngrp][W_h]
  double* dot = (double*)scratch(ctx, SW_DOT, sizeof(double) * SD);
  double* wbar = (double*)scratch(ctx, SW_WBAR, sizeof(double) * SD);
  if (!Us || !Vs || !KVs || !KTs || !Bs || !Vck || !T || !T2 || !AB || !gwp || !dot || !wbar) return RWIG_E_NOMEM;
  cudaStream_t qs[2] = {st, st};
  if (halves == 2) {
    qs[1] = side_stream(ctx, 0);
    if (!qs[1]) return set_error(RWIG_E_CUDA, "could not create a side stream");
    RWIG_CUDA_TRY(cudaEventRecord(ctx->evfork, st));
    RWIG_CUDA_TRY(cudaStreamWaitEvent(qs[1], ctx->evfork, 0));
  }
  auto seg_len = [&](int j) { return std::min(k, L - j * k); };
  // one half: documents [d0, d1), columns [c0, c0 + Wh) of every buffer
  auto run_half = [&](int h, int d0, int d1) -> int {
    cudaStream_t q = qs[h];
    const int c0 = d0 * S, Wh = (d1 - d0) * S;
    const size_t o = (size_t)N * c0, od = (size_t)N * d0;
    double* gw = gwp + (size_t)ngrp * c0;  // [ngrp][Wh]
    auto U = [&](int t) { return Us + NW * t + o; };
    auto V = [&](int j, int t) { return (t == 0 ? Vck + NW * j : Vs + NW * t) + o; };
    auto KV = [&](int t) { return KVs + NW * t + o; };
    auto KT = [&](int t) { return KTs + NW * t + o; };
    auto Bb = [&](int t) { return Bs + ND * t + od; };
    const int tc = tile_cols(S, Wh);
    auto gemm = [&](int trans, const double* X, auto epi) -> int {
      if (pr) return oz::gemm(ctx, *pr, trans, X, N, Wh, tc, epi, q, launches, h);
      const dg::GemmArgs g{K, ldk, N, N, Wh, X, N, 0, tc};
      return trans ? dg::gemm<1>(ctx, g, epi, q, 0, launches) : dg::gemm<0>(ctx, g, epi, q, 0, launches);
    };
    const double* Wbh = Wb + c0;
    // forward iterations j k .. j k + len - 1 (wdl_impl.cpp:124-160)
    auto forward_segment = [&](int j) -> int {
      for (int t = 0; t < seg_len(j); ++t) {
        if (int rc = gemm(0, V(j, t), EpiY{A, N, S, Wh, KV(t), U(t + 1)})) return rc;
        if (int rc = gemm(1, U(t + 1), EpiZ{Wbh, N, S, Wh, KT(t + 1), V(j, t + 1), Bb(t + 1)})) return rc;
      }
      return 0;
    };
    fill<<<grid_for(ctx, (long long)N * Wh), TPB, 0, q>>>(V(0, 0), (long long)N * Wh, 1.0);
    ++*launches;
    int rc;
    for (int j = 0; j < nseg; ++j) {
      if ((rc = forward_segment(j))) return rc;
      if (j + 1 < nseg)  // VB_{(j+1) k}, the next segment's checkpoint
        RWIG_CUDA_TRY(
            cudaMemcpyAsync(V(j + 1, 0), V(j, k), sizeof(double) * N * Wh, cudaMemcpyDeviceToDevice, q));
    }
    RWIG_CUDA_TRY(cudaMemsetAsync(AB + o, 0, sizeof(double) * N * Wh, q));
    RWIG_CUDA_TRY(cudaMemsetAsync(gw, 0, sizeof(double) * (size_t)ngrp * Wh, q));
    for (int j = nseg - 1; j >= 0; --j) {  // :169-218, segments newest first
      if (j != nseg - 1 && (rc = forward_segment(j))) return rc;  // recompute from VB_{j k}
      for (int t = seg_len(j); t >= 1; --t) {
        const bool seed = (j * k + t == L);
        const EpiB1 e1{KT(t), V(j, t), Wbh, Bb(t), Yb + od, N, S, Wh, seed ? 1 : 0, T2 + o, gw};
        if (seed) {
          dim3 grid(ngrp, (Wh + tc - 1) / tc);
          seed_b1<<<grid, TPB, sizeof(double) * 2 * tc * 8, q>>>(e1, N, tc);
          ++*launches;
        } else {
          if ((rc = gemm(1, T + o, e1))) return rc;  // K^T T
        }
        if ((rc = gemm(0, T2 + o, EpiB2{U(t), KV(t - 1), N, Wh, AB + o, T + o}))) return rc;  // K T2
      }
    }
    reduce_cols<<<Wh, TPB, 0, q>>>(gw, ngrp, Wh, wbar + c0);
    ++*launches;
    RWIG_CUDA_TRY(cudaGetLastError());
    return 0;
  };
  const int dsplit = halves == 2 ? D / 2 : D;
  if (int rc = run_half(0, 0, dsplit)) return rc;
  if (halves == 2) {
    if (int rc = run_half(1, dsplit, D)) return rc;
    RWIG_CUDA_TRY(cudaEventRecord(ctx->evjoin, qs[1]));
    RWIG_CUDA_TRY(cudaStreamWaitEvent(st, ctx->evjoin, 0));
  }
  col_dots<<<SD, TPB, 0, st>>>(A, AB, N, S, dot);
  alpha_grad<<<grid_for(ctx, (long long)N * S), TPB, 0, st>>>(A, AB, dot, N, S, D, gA);
  lambda_grad<<<1, TPB, 0, st>>>(Wb, wbar, S, D, gl);
  *launches += 3;
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Whether the WDL products of an N x N kernel run on the INT8 tensor cores
// (ozaki.cuh) rather than the FP64 ones: option "wdl.int8" 0 never, 2
// whenever the device and size allow, 1 (default) from N = 1024 up.
bool use_int8(Context* ctx, int N) {
  const int o = (int)option("wdl.int8", 1.0);
  if (o == 0 || N > oz::kMaxKd || !oz::available(ctx)) return false;
  return o == 2 || N >= 1024;
}

int check_dims(int N, int S, int D) {
  if (N < 1 || S < 1 || D < 1) return set_error(RWIG_E_INVALID, "N, S and D must be >= 1");
  if (S > 64) return set_error(RWIG_E_UNSUPPORTED, "more than 64 topics");
  if ((long long)S * D > (1LL << 24)) return set_error(RWIG_E_UNSUPPORTED, "S * D too large");
  return 0;
}

// K (padded, ldk) from K itself (mode 0) or from C (mode 1).
int make_k(Context* ctx, cudaStream_t st, const double* KorC, int N, double reg, int mode, double** Kout,
           long long* ldk_out) {
  const long long ldk = ((N + 1) / 2) * 2;
  double* K = (double*)scratch(ctx, SW_K, sizeof(double) * ldk * N);
  if (!K) return RWIG_E_NOMEM;
  if (mode == 1) gibbs<<<grid_for(ctx, ldk * N), TPB, 0, st>>>(KorC, N, ldk, reg, K);
  else copy_k<<<grid_for(ctx, ldk * N), TPB, 0, st>>>(KorC, N, ldk, K);
  RWIG_CUDA_TRY(cudaGetLastError());
  *Kout = K;
  *ldk_out = ldk;
  return 0;
}

int batch_grad_entry(Context* ctx, cudaStream_t st, double* gA, double* gl, const double* A, const double* Wb,
                     const double* Yb, const double* KorC, int N, int S, int D, double reg, int L, int mode) {
  reset_report();
  if (!gA || !gl || !A || !Wb || !Yb || !KorC) return set_error(RWIG_E_INVALID, "null pointer argument");
  int rc = check_dims(N, S, D);
  if (rc) return rc;
  if (mode != 0 && mode != 1) return set_error(RWIG_E_INVALID, "mode must be 0 (K given) or 1 (C given)");
  if (mode == 1 && (!(reg > 0.0) || !std::isfinite(reg))) return set_error(RWIG_E_INVALID, "reg must be > 0");
  if (L < 0) return set_error(RWIG_E_INVALID, "L must be >= 0");
  if ((rc = gemm_timer_begin(ctx))) return rc;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
  double* K = nullptr;
  long long ldk = 0;
  rc = make_k(ctx, st, KorC, N, reg, mode, &K, &ldk);
  if (rc) return rc;
  int launches = 1;
  oz::Prepared pr;
  const bool i8 = use_int8(ctx, N) && L > 0;
  if (i8 && (rc = oz::prepare_reuse(ctx, K, ldk, N, &pr, st, &launches))) return rc;
  rc = batch_grad(ctx, st, gA, gl, A, Wb, Yb, K, ldk, N, S, D, L, &launches, i8 ? &pr : nullptr);
  if (rc) return rc;
  if (i8 && (rc = oz::status(ctx, st))) return rc;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  rwig_report& R = report();
  R.iter = L;
  R.device_ms = ms;
  R.kernel_ms = ms;
  R.kernel_launches = launches;
  gemm_timer_end(ctx, &R.gemm_ms, &R.gemm_launches);
  return 0;
}

}  // namespace wdl
}  // namespace rwig

using namespace rwig;

extern "C" int rwig_wdl_batch_grad_dev(double* g_Alpha, double* g_lambda, const double* A, const double* W_B,
                                       const double* Y_B, const double* K_or_C, int N, int S, int D, double reg,
                                       int L, int mode, void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return wdl::batch_grad_entry(ctx, call_stream(ctx, stream), g_Alpha, g_lambda, A, W_B, Y_B,
                               K_or_C, N, S, D, reg, L, mode);
}

extern "C" int rwig_wdl_update_dev(double* Alpha, double* Lambda, double* A, double* W, double* mA, double* vA,
                                   double* mL, double* vL, const double* g_Alpha, const double* g_lambda, int N,
                                   int S, int M, int opt, double eta, double gamma, double beta1, double beta2,
                                   double eps, int step, void* stream) {
  reset_report();
  if (!Alpha || !Lambda || !A || !W || !g_Alpha || !g_lambda || (opt != 0 && (!mA || !vA || !mL || !vL)))
    return set_error(RWIG_E_INVALID, "null pointer argument");
  if (N < 1 || S < 1 || M < 1 || step < 1) return set_error(RWIG_E_INVALID, "N, S, M and step must be >= 1");
  if (opt < 0 || opt > 2) return set_error(RWIG_E_INVALID, "opt must be 0 (SGD), 1 (Adam) or 2 (AdamW)");
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = call_stream(ctx, stream);
  const long long NS = (long long)N * S, SM = (long long)S * M;
  // the same bias corrections and kernels as the training loop of rwig_wdl
  const double c1 = 1.0 - std::pow(beta1, step), c2 = 1.0 - std::pow(beta2, step);
  wdl::opt_step<<<wdl::grid_for(ctx, NS), wdl::TPB, 0, st>>>(Alpha, mA, vA, g_Alpha, 0, NS, opt, eta, gamma, beta1,
                                                            beta2, eps, c1, c2);
  wdl::opt_step<<<wdl::grid_for(ctx, SM), wdl::TPB, 0, st>>>(Lambda, mL, vL, g_lambda, S, SM, opt, eta, gamma,
                                                            beta1, beta2, eps, c1, c2);
  wdl::col_softmax<<<S, wdl::TPB, 0, st>>>(Alpha, N, A);
  wdl::col_softmax<<<M, wdl::TPB, 0, st>>>(Lambda, S, W);
  RWIG_CUDA_TRY(cudaGetLastError());
  report().kernel_launches = 4;
  return 0;
}

extern "C" int rwig_wdl_batch_grad(double* g_Alpha, double* g_lambda, const double* A, const double* W_B,
                                   const double* Y_B, const double* K_or_C, int N, int S, int D, double reg, int L,
                                   int mode) {
  if (!g_Alpha || !g_lambda || !A || !W_B || !Y_B || !K_or_C) {
    reset_report();
    return set_error(RWIG_E_INVALID, "null pointer argument");
  }
  {
    const int rc = wdl::check_dims(N, S, D);
    if (rc) return rc;
  }
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = ctx->stream;
  const size_t NS = (size_t)N * S, SD = (size_t)S * D, ND = (size_t)N * D, NN = (size_t)N * N;
  double* dA = (double*)scratch(ctx, wdl::SW_HA, sizeof(double) * NS);
  double* dW = (double*)scratch(ctx, wdl::SW_HW, sizeof(double) * SD);
  double* dY = (double*)scratch(ctx, wdl::SW_HY, sizeof(double) * ND);
  double* dK = (double*)scratch(ctx, wdl::SW_HK, sizeof(double) * NN);
  double* dO = (double*)scratch(ctx, wdl::SW_HOUT, sizeof(double) * (NS + S));
  if (!dA || !dW || !dY || !dK || !dO) return RWIG_E_NOMEM;
  RWIG_CUDA_TRY(cudaMemcpyAsync(dA, A, sizeof(double) * NS, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(dW, W_B, sizeof(double) * SD, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(dY, Y_B, sizeof(double) * ND, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(dK, K_or_C, sizeof(double) * NN, cudaMemcpyHostToDevice, st));
  const int rc = wdl::batch_grad_entry(ctx, st, dO, dO + NS, dA, dW, dY, dK, N, S, D, reg, L, mode);
  if (rc) return rc;
  RWIG_CUDA_TRY(cudaMemcpyAsync(g_Alpha, dO, sizeof(double) * NS, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(g_lambda, dO + NS, sizeof(double) * S, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  return 0;
}

extern "C" int rwig_wdl(double* A, double* W, double* Yhat, const double* Y, const double* C, int N, int M, int S,
                        double reg, int max_iter, double zero_tol, int B, int E, int opt, double eta, double gamma,
                        double beta1, double beta2, double eps, int seed, int verbose, const double* Alpha0,
                        const double* Lambda0, int max_steps) {
  reset_report();
  if (!Y || !C) return set_error(RWIG_E_INVALID, "Y and C must be non-null");
  if (M < 1 || B < 1 || E < 0) return set_error(RWIG_E_INVALID, "M, B must be >= 1 and E >= 0");
  if (opt < 0 || opt > 2) return set_error(RWIG_E_INVALID, "opt must be 0 (SGD), 1 (Adam) or 2 (AdamW)");
  if (!(reg > 0.0) || !std::isfinite(reg)) return set_error(RWIG_E_INVALID, "reg must be finite and > 0");
  if (max_iter < 0) return set_error(RWIG_E_INVALID, "max_iter must be >= 0");
  {
    const int rc = wdl::check_dims(N, S, std::min(B, M));
    if (rc) return rc;
  }
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = ctx->stream;
  using namespace wdl;
  const size_t NS = (size_t)N * S, SM = (size_t)S * M, NM = (size_t)N * M, NN = (size_t)N * N;
  double* dY = (double*)scratch(ctx, SW_Y, sizeof(double) * NM);
  double* dC = (double*)scratch(ctx, SW_C, sizeof(double) * NN);
  double* dAl = (double*)scratch(ctx, SW_ALPHA, sizeof(double) * NS);
  double* dLa = (double*)scratch(ctx, SW_LAMBDA, sizeof(double) * SM);
  double* dA = (double*)scratch(ctx, SW_A, sizeof(double) * NS);
  double* dW = (double*)scratch(ctx, SW_W, sizeof(double) * SM);
  double* mA = (double*)scratch(ctx, SW_MA, sizeof(double) * NS);
  double* vA = (double*)scratch(ctx, SW_VA, sizeof(double) * NS);
  double* mL = (double*)scratch(ctx, SW_ML, sizeof(double) * SM);
  double* vL = (double*)scratch(ctx, SW_VL, sizeof(double) * SM);
  double* gA = (double*)scratch(ctx, SW_GA, sizeof(double) * NS);
  double* gl = (double*)scratch(ctx, SW_GL, sizeof(double) * S);
  if (!dY || !dC || !dAl || !dLa || !dA || !dW || !mA || !vA || !mL || !vL || !gA || !gl) return RWIG_E_NOMEM;
  RWIG_CUDA_TRY(cudaMemcpyAsync(dY, Y, sizeof(double) * NM, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpyAsync(dC, C, sizeof(double) * NN, cudaMemcpyHostToDevice, st));
  // initial logits: given, or N(0, 1) draws from mt19937(seed), Alpha first
  // then Lambda (cuda_wdl.cu:592-689)
  std::vector<double> h;
  if (!Alpha0 || !Lambda0) {
    std::mt19937 rng((unsigned)seed);
    std::normal_distribution<double> randn(0.0, 1.0);
    h.resize(NS + SM);
    for (auto& x : h) x = randn(rng);
  }
  RWIG_CUDA_TRY(cudaMemcpyAsync(dAl, Alpha0 ? Alpha0 : h.data(), sizeof(double) * NS, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(
      cudaMemcpyAsync(dLa, Lambda0 ? Lambda0 : h.data() + NS, sizeof(double) * SM, cudaMemcpyHostToDevice, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(mA, 0, sizeof(double) * NS, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(vA, 0, sizeof(double) * NS, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(mL, 0, sizeof(double) * SM, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(vL, 0, sizeof(double) * SM, st));
  int rc = gemm_timer_begin(ctx);  // training GEMMs only
  if (rc) return rc;
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev0, st));
  int launches = 0;
  double* K = nullptr;
  long long ldk = 0;
  rc = make_k(ctx, st, dC, N, reg, 1, &K, &ldk);  // K = exp(-C/reg) (wdl_impl.cpp:297)
  if (rc) return rc;
  oz::Prepared pr;  // K's residue planes, once for the whole training and inference
  const bool i8 = use_int8(ctx, N);
  if (i8 && (rc = oz::prepare(ctx, K, ldk, N, &pr, st, &launches))) return rc;
  col_softmax<<<S, TPB, 0, st>>>(dAl, N, dA);
  col_softmax<<<M, TPB, 0, st>>>(dLa, S, dW);
  launches += 3;
  const int batches = (M % B) ? (M / B + 1) : (M / B);
  int steps = 0;
  for (int e = 0; e < E; ++e) {
    for (int bi = 0; bi < batches; ++bi) {
      if (max_steps > 0 && steps >= max_steps) break;
      const int D = (bi == M / B) ? (M % B) : B;  // wdl_impl.cpp:91
      rc = batch_grad(ctx, st, gA, gl, dA, dW + (size_t)bi * B * S, dY + (size_t)bi * B * N, K, ldk, N, S, D,
                      max_iter, &launches, i8 ? &pr : nullptr);
      if (rc) return rc;
      ++steps;
      const double c1 = 1.0 - std::pow(beta1, steps), c2 = 1.0 - std::pow(beta2, steps);
      opt_step<<<grid_for(ctx, NS), TPB, 0, st>>>(dAl, mA, vA, gA, 0, NS, opt, eta, gamma, beta1, beta2, eps, c1,
                                                  c2);
      opt_step<<<grid_for(ctx, SM), TPB, 0, st>>>(dLa, mL, vL, gl, S, SM, opt, eta, gamma, beta1, beta2, eps, c1,
                                                  c2);
      col_softmax<<<S, TPB, 0, st>>>(dAl, N, dA);
      col_softmax<<<M, TPB, 0, st>>>(dLa, S, dW);
      launches += 4;
      RWIG_CUDA_TRY(cudaGetLastError());
      if (verbose) {
        RWIG_CUDA_TRY(cudaStreamSynchronize(st));
        std::fprintf(stderr, "rwig_wdl: epoch %d of %d, batch %d of %d done\n", e + 1, E, bi + 1, batches);
      }
    }
  }
  RWIG_CUDA_TRY(cudaEventRecord(ctx->ev1, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (i8 && (rc = oz::status(ctx, st))) return rc;
  float train_ms = 0.f;
  cudaEventElapsedTime(&train_ms, ctx->ev0, ctx->ev1);
  double gemm_ms = 0.0;
  int gemm_n = 0;
  gemm_timer_end(ctx, &gemm_ms, &gemm_n);
  if (A) RWIG_CUDA_TRY(cudaMemcpyAsync(A, dA, sizeof(double) * NS, cudaMemcpyDeviceToHost, st));
  if (W) RWIG_CUDA_TRY(cudaMemcpyAsync(W, dW, sizeof(double) * SM, cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (Yhat) {
    // inference: the parallel barycenter of every document (wdl_impl.cpp:349-377),
    // all documents at once; without iterations the reference's b is 0 / 0
    double* dYh = (double*)scratch(ctx, SW_YHAT, sizeof(double) * NM);
    if (!dYh) return RWIG_E_NOMEM;
    if (max_iter >= 1) {
      rc = infer(ctx, st, dA, dW, K, ldk, N, S, M, max_iter, zero_tol, dYh, &launches, i8 ? &pr : nullptr);
      if (rc < 0) return rc;
      if (i8 && (rc = oz::status(ctx, st))) return rc;
    } else {
      for (int m = 0; m < M; ++m) {
        rc = bary::run(ctx, st, false, nullptr, nullptr, dYh + (size_t)m * N, nullptr, nullptr, nullptr, nullptr,
                       nullptr, dA, dW + (size_t)m * S, dC, nullptr, N, N, S, reg, 0, max_iter, zero_tol);
        if (rc < 0) return rc;
      }
    }
    RWIG_CUDA_TRY(cudaMemcpyAsync(Yhat, dYh, sizeof(double) * NM, cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  }
  reset_report();
  rwig_report& R = report();
  R.iter = steps;
  R.device_ms = train_ms;
  R.kernel_ms = train_ms;
  R.kernel_launches = launches;
  R.gemm_ms = gemm_ms;
  R.gemm_launches = gemm_n;
  return 0;
}
