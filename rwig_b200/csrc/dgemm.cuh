// dgemm.cuh -- FP64 tensor-core (DMMA, mma.sync m16n8k4 .f64) GEMM for the
// skinny products of the barycenter and WDL paths:
//     Y (Mo x S) = op(K) * X (Kd x S),   op(K) = K or K^T,
// K column-major (ldk), X and Y column-major.  Split-K: each CTA computes a
// 64 x 32 tile of Y over one slice of the contraction and writes it to a
// partial buffer [split][S][Mo]; callers reduce the splits in a fixed order
// (deterministic) inside their own epilogue kernels.
//
// Tiles: 4 warps per CTA, each 16 rows x 32 columns (four m16n8k4 n-tiles);
// BK = 16 contraction steps per stage, two stages through cp.async (16-byte
// copies, zero-filled at the edges).
#pragma once

#include <cstdint>

namespace rwig {
namespace dg {

constexpr int BM = 64, BN = 32, BK = 16, NTH = 128;
constexpr int PAD = 4;  // doubles of padding per shared row

struct GemmArgs {
  const double* K;
  long long ldk;
  int trans;         // 0: Y = K X (Mo = rows of K), 1: Y = K^T X (Mo = cols of K)
  int Mo, Kd, S;     // output rows, contraction length, output columns
  const double* X;   // Kd x S, column-major
  long long ldx;
  double* part;      // [splits][S][Mo]
  int splits;        // contraction slices (gridDim.z)
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ void mma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// Shared tiles: A as [BK][BM + PAD] (k-major), B as [BK][BN + PAD].
struct Smem {
  double A[2][BK][BM + PAD];
  double B[2][BK][BN + PAD];
};

// Loads the A and B tiles of contraction step k0 into stage `st`.
__device__ __forceinline__ void load_stage(const GemmArgs& g, Smem& sm, int st, int m0, int n0, int k0, int kend) {
  const int tid = threadIdx.x;
  // A tile: BK x BM doubles = 512 16-byte chunks, 4 per thread
  if (!g.trans) {
    // A[m][k] = K[m + k*ldk]: chunk = (k, pair of m)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int idx = tid + c * NTH;  // 0..511
      const int kk = idx >> 5, mp = (idx & 31) * 2;
      const int gk = k0 + kk, gm = m0 + mp;
      int bytes = 0;
      const double* src = g.K;
      if (gk < kend && gm < g.Mo) {
        bytes = (gm + 1 < g.Mo) ? 16 : 8;
        src = g.K + gm + (long long)gk * g.ldk;
      }
      cp_async16(&sm.A[st][kk][mp], src, bytes);
    }
  } else {
    // A[m][k] = K[k + m*ldk]: chunk = (m, pair of k), stored transposed
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int idx = tid + c * NTH;
      const int mm = idx >> 3, kp = (idx & 7) * 2;
      const int gk = k0 + kp, gm = m0 + mm;
      double v0 = 0.0, v1 = 0.0;
      if (gm < g.Mo) {
        const double* src = g.K + gk + (long long)gm * g.ldk;
        if (gk < kend) v0 = __ldg(src);
        if (gk + 1 < kend) v1 = __ldg(src + 1);
      }
      sm.A[st][kp][mm] = v0;
      sm.A[st][kp + 1][mm] = v1;
    }
  }
  // B tile: BK x BN doubles = 256 chunks, 2 per thread; B[k][n] = X[k + n*ldx]
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int idx = tid + c * NTH;  // 0..255
    const int nn = idx >> 3, kp = (idx & 7) * 2;
    const int gk = k0 + kp, gn = n0 + nn;
    double v0 = 0.0, v1 = 0.0;
    if (gn < g.S) {
      const double* src = g.X + gk + (long long)gn * g.ldx;
      if (gk < kend) v0 = __ldg(src);
      if (gk + 1 < kend) v1 = __ldg(src + 1);
    }
    sm.B[st][kp][nn] = v0;
    sm.B[st][kp + 1][nn] = v1;
  }
}

#ifdef RWIG_DGEMM_DEFINE_KERNEL  // defined in dgemm.cu only
__global__ void __launch_bounds__(NTH) dgemm_splitk_kernel(GemmArgs g) {
  __shared__ __align__(16) Smem sm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int slice = (g.Kd + g.splits - 1) / g.splits;
  const int kbeg = blockIdx.z * slice;
  const int kend = min(g.Kd, kbeg + slice);
  double acc[4][4];
#pragma unroll
  for (int t = 0; t < 4; ++t)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[t][e] = 0.0;

  const int nsteps = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
  if (nsteps > 0) load_stage(g, sm, 0, m0, n0, kbeg, kend);
  cp_async_commit();
  const int wm = warp * 16;
  for (int s = 0; s < nsteps; ++s) {
    const int st = s & 1;
    if (s + 1 < nsteps) load_stage(g, sm, st ^ 1, m0, n0, kbeg + (s + 1) * BK, kend);
    cp_async_commit();
    cp_async_wait_one();
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      const double a0 = sm.A[st][kk + tig][wm + gid];
      const double a1 = sm.A[st][kk + tig][wm + gid + 8];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const double b0 = sm.B[st][kk + tig][t * 8 + gid];
        mma_16x8x4(acc[t], a0, a1, b0);
      }
    }
    __syncthreads();
  }
  cp_async_wait_all();
  // C fragment: c0,c1 at row gid, cols 2*tig + {0,1}; c2,c3 at row gid + 8
  double* out = g.part + (size_t)blockIdx.z * g.S * g.Mo;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int r = m0 + wm + gid + ((e >> 1) << 3);
      const int c = n0 + t * 8 + tig * 2 + (e & 1);
      if (r < g.Mo && c < g.S) out[(size_t)c * g.Mo + r] = acc[t][e];
    }
  }
}

#endif  // RWIG_DGEMM_DEFINE_KERNEL

// Fixed-order sum of the split partials of entry (r, c).
__device__ __forceinline__ double reduce_splits(const double* part, int splits, int Mo, int S, int r, int c) {
  double s = 0.0;
  const size_t stride = (size_t)S * Mo, off = (size_t)c * Mo + r;
  for (int z = 0; z < splits; ++z) s += part[z * stride + off];
  return s;
}

}  // namespace dg
}  // namespace rwig
