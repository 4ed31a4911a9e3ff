// dgemm.cuh -- FP64 tensor-core (DMMA, mma.sync m16n8k4 .f64) GEMM for the
// skinny products of the barycenter and WDL paths:
//     Y (Mo x W) = op(K) * X (Kd x W),   op(K) = K or K^T,
// K column-major (ldk even, 16-byte aligned), X column-major.
//
// One CTA (8 warps) computes a BM x BN tile of Y over one slice of the
// contraction; each warp owns 16 rows x BN columns (NT m16n8k4 n-tiles) and
// one half of every BK step (warps 0-3 the first 16 k, warps 4-7 the second),
// the two halves being added in a fixed order at the end.  Operands stream
// through a STAGES-deep cp.async ring in their natural global layout (K^T
// tiles m-major, K tiles k-major, X tiles column-major), padded so the
// fragment reads are free of bank conflicts.
//
// Split-K runs inside a thread-block cluster of `splits` CTAs stacked along
// z: every CTA parks its partial tile in shared memory, and after a cluster
// barrier CTA z sums rows [z*BM/splits, (z+1)*BM/splits) of all partials
// through distributed shared memory, in the fixed order 0..splits-1 (the
// result is bitwise repeatable and independent of scheduling).  The summed
// rows then go to an epilogue functor, so the elementwise work that follows
// each product never makes a separate pass over HBM.
//
// Epilogue interface (called by all NTH threads of the CTA; may use
// __syncthreads):
//     epi(r0, nr, c0, nc, t, ldt, ws)
// rows r0 .. r0+nr-1 of Y (nr <= 0: nothing to do), columns c0 .. c0+nc-1
// (nc = the tile's column count, tcols), value (r0 + r, c0 + c) at
// t[c * ldt + r] (the epilogue may overwrite t); ws: 2 * (BN + 1) * ldt
// doubles of shared scratch.  Columns at
// or beyond W hold zeros.  Tiles are numbered with the column tiles fastest,
// so the CTAs resident at one time share rows of K (one HBM pass over K when
// it does not fit in L2).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace rwig {
namespace dg {

constexpr int BM = 64, BK = 32, NTH = 256, STAGES = 4;
constexpr int PAD = 4;  // doubles of padding per shared row
constexpr int kMaxSplits = 8;

struct GemmArgs {
  const double* K;
  long long ldk;
  int Mo, Kd, W;     // output rows, contraction length, output columns
  const double* X;   // Kd x W, column-major
  long long ldx;
  int splits;        // cluster size along z: 1, 2, 4 or 8
  int tcols;         // output columns per tile (<= BN; 0: BN).  A multiple of an
                     // epilogue's column group keeps every group inside one tile.
};

template <int TRANS>
__host__ __device__ constexpr int a_stage_doubles() {
  return TRANS ? BM * (BK + PAD) : BK * (BM + PAD);
}
template <int NT>
__host__ __device__ constexpr int b_stage_doubles() {
  return NT * 8 * (BK + PAD);
}
template <int TRANS, int NT>
__host__ __device__ constexpr int smem_doubles() {
  // pipeline ring, or (after the main loop) partial tile + summed rows +
  // epilogue scratch (two blocks of (BN + 1) x BM)
  return (STAGES * (a_stage_doubles<TRANS>() + b_stage_doubles<NT>()) > NT * 8 * (2 * BM + 1) + 2 * (NT * 8 + 1) * BM)
             ? STAGES * (a_stage_doubles<TRANS>() + b_stage_doubles<NT>())
             : NT * 8 * (2 * BM + 1) + 2 * (NT * 8 + 1) * BM;
}

__device__ __forceinline__ void cp_async16(double* smem, const double* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ unsigned cluster_nctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
// Load a double from the same shared-memory offset in cluster CTA `rank`.
__device__ __forceinline__ double ld_cluster(const double* p, unsigned rank) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  unsigned ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(ra) : "memory");
  return v;
}

// Issues the copies of contraction step [k0, k0 + BK) into one ring stage.
// XV = 2: X columns copied as 16-byte pairs (ldx even, X 16-byte aligned);
// XV = 1: 8-byte copies.  Out-of-range elements are zero-filled.
template <int TRANS, int NT, int XV>
__device__ __forceinline__ void load_stage(const GemmArgs& g, double* As, double* Bs, int m0, int n0, int tc,
                                           int k0, int kend) {
  const int tid = threadIdx.x;
  if (!TRANS) {
    // A[k][m] = K[m + k*ldk]: 32 k x 32 m-pairs
#pragma unroll
    for (int c = 0; c < (BK * BM / 2) / NTH; ++c) {
      const int idx = tid + c * NTH;
      const int kk = idx >> 5, mp = (idx & 31) * 2;
      const int gk = k0 + kk, gm = m0 + mp;
      int bytes = 0;
      const double* src = g.K;
      if (gk < kend && gm < g.Mo) {
        bytes = (gm + 1 < g.Mo) ? 16 : 8;
        src = g.K + gm + (long long)gk * g.ldk;
      }
      cp_async16(As + kk * (BM + PAD) + mp, src, bytes);
    }
  } else {
    // A[m][k] = K[k + m*ldk]: 64 m x 16 k-pairs
#pragma unroll
    for (int c = 0; c < (BM * BK / 2) / NTH; ++c) {
      const int idx = tid + c * NTH;
      const int mm = idx >> 4, kp = (idx & 15) * 2;
      const int gk = k0 + kp, gm = m0 + mm;
      int bytes = 0;
      const double* src = g.K;
      if (gk < kend && gm < g.Mo) {
        bytes = (gk + 1 < kend) ? 16 : 8;
        src = g.K + gk + (long long)gm * g.ldk;
      }
      cp_async16(As + mm * (BK + PAD) + kp, src, bytes);
    }
  }
  // B[n][k] = X[k + n*ldx]
  if (XV == 2) {
#pragma unroll
    for (int c = 0; c < NT * 8 * 16 / NTH; ++c) {  // NT*8 columns x 16 k-pairs
      const int idx = tid + c * NTH;
      const int nn = idx >> 4, kp = (idx & 15) * 2;
      const int gk = k0 + kp, gn = n0 + nn;
      int bytes = 0;
      const double* src = g.X;
      if (gk < kend && gn < g.W && nn < tc) {
        bytes = (gk + 1 < kend) ? 16 : 8;
        src = g.X + gk + (long long)gn * g.ldx;
      }
      cp_async16(Bs + nn * (BK + PAD) + kp, src, bytes);
    }
  } else {
#pragma unroll
    for (int c = 0; c < NT * 8 * 32 / NTH; ++c) {  // NT*8 columns x 32 k
      const int idx = tid + c * NTH;
      const int nn = idx >> 5, kk = idx & 31;
      const int gk = k0 + kk, gn = n0 + nn;
      int bytes = 0;
      const double* src = g.X;
      if (gk < kend && gn < g.W && nn < tc) {
        bytes = 8;
        src = g.X + gk + (long long)gn * g.ldx;
      }
      cp_async8(Bs + nn * (BK + PAD) + kk, src, bytes);
    }
  }
}

template <int TRANS, int NT, int XV, class Epi>
__global__ void __launch_bounds__(NTH) dgemm_kernel(GemmArgs g, Epi epi) {
  extern __shared__ __align__(16) double smem[];
  constexpr int BN = NT * 8;
  constexpr int ASZ = a_stage_doubles<TRANS>(), BSZ = b_stage_doubles<NT>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int tc = g.tcols > 0 ? g.tcols : BN;
  const int ntiles = (g.W + tc - 1) / tc;
  const int m0 = (blockIdx.x / ntiles) * BM, n0 = (blockIdx.x % ntiles) * tc;
  const int splits = g.splits;
  // the launch must form one cluster of `splits` CTAs along z
  if (splits > 1 && (int)cluster_nctarank() != splits) return;
  const int z = blockIdx.z;
  int slice = (g.Kd + splits - 1) / splits;
  slice = ((slice + BK - 1) / BK) * BK;
  const int kbeg = z * slice;
  const int kend = min(g.Kd, kbeg + slice);
  const int nsteps = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;

  double acc[NT][4];
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[t][e] = 0.0;

  double* As = smem;
  double* Bs = smem + STAGES * ASZ;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nsteps) load_stage<TRANS, NT, XV>(g, As + s * ASZ, Bs + s * BSZ, m0, n0, tc, kbeg + s * BK, kend);
    cp_async_commit();
  }
  const int wm = (warp & 3) * 16, kh = (warp >> 2) * (BK / 2);
  for (int s = 0; s < nsteps; ++s) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();  // stage s visible; stage s-1 no longer read
    const int nx = s + STAGES - 1;
    if (nx < nsteps) {
      const int q = nx % STAGES;
      load_stage<TRANS, NT, XV>(g, As + q * ASZ, Bs + q * BSZ, m0, n0, tc, kbeg + nx * BK, kend);
    }
    cp_async_commit();
    const double* A = As + (s % STAGES) * ASZ;
    const double* B = Bs + (s % STAGES) * BSZ;
#pragma unroll
    for (int k4 = 0; k4 < BK / 2; k4 += 4) {
      const int kk = kh + k4;
      double a0, a1;
      if (!TRANS) {
        a0 = A[(kk + tig) * (BM + PAD) + wm + gid];
        a1 = A[(kk + tig) * (BM + PAD) + wm + gid + 8];
      } else {
        a0 = A[(wm + gid) * (BK + PAD) + kk + tig];
        a1 = A[(wm + gid + 8) * (BK + PAD) + kk + tig];
      }
#pragma unroll
      for (int t = 0; t < NT; ++t) mma_16x8x4(acc[t], a0, a1, B[(t * 8 + gid) * (BK + PAD) + kk + tig]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();

  // partial tile -> shared memory, [c][r] with row stride BM + 1; the second
  // k half is added to the first in a fixed order
  double* red = smem;
  double* fin = red + BN * (BM + 1);
  double* ws = fin + BN * BM;
  for (int h = 0; h < 2; ++h) {
    if ((warp >> 2) == h) {
#pragma unroll
      for (int t = 0; t < NT; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int r = wm + gid + ((e >> 1) << 3);
          const int c = t * 8 + tig * 2 + (e & 1);
          if (h == 0) red[c * (BM + 1) + r] = acc[t][e];
          else red[c * (BM + 1) + r] += acc[t][e];
        }
    }
    if (h == 0) __syncthreads();
  }
  if (splits > 1) {
    cluster_arrive();
    cluster_wait();
  } else {
    __syncthreads();
  }
  // sum this CTA's rows over the cluster's partials, fixed order
  const int rows = BM / splits;
  const int rl0 = z * rows;
  for (int e = threadIdx.x; e < rows * BN; e += NTH) {
    const int r = e % rows, c = e / rows;
    const double* p = red + c * (BM + 1) + rl0 + r;
    double v = 0.0;
    if (splits > 1) {
      for (int q = 0; q < splits; ++q) v += ld_cluster(p, (unsigned)q);
    } else {
      v += *p;
    }
    fin[c * rows + r] = v;
  }
  if (splits > 1) cluster_arrive();  // this CTA is done reading its peers
  __syncthreads();
  epi(m0 + rl0, min(rows, g.Mo - (m0 + rl0)), n0, tc, fin, rows, ws);
  if (splits > 1) cluster_wait();  // peers are done reading this CTA
}

// Epilogue that stores the tile: Y[r + c*ldy] for columns < W.
struct EpiStore {
  double* Y;
  long long ldy;
  int W;
  __device__ void operator()(int r0, int nr, int c0, int nc, double* t, int ldt, double*) const {
    if (nr <= 0) return;
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
      const int r = e % nr, c = e / nr;
      if (c0 + c < W) Y[(r0 + r) + (long long)(c0 + c) * ldy] = t[c * ldt + r];
    }
  }
};

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Largest power of two <= kMaxSplits that keeps the grid within about the
// resident CTAs of one wave (two per SM for NT = 4, one for NT = 8) and
// leaves every slice at least four BK steps.
inline int pick_splits(const Context* ctx, int Mo, int Kd, int W, int NT, int tc = 0) {
  if (tc <= 0) tc = NT * 8;
  const long long tiles = (long long)((Mo + BM - 1) / BM) * ((W + tc - 1) / tc);
  const long long target = (NT <= 4 ? 2LL : 1LL) * ctx->sm_count;
  int s = 1;
  while (s < kMaxSplits && tiles * s * 2 <= target && Kd >= s * 2 * 4 * BK) s *= 2;
  return s;
}

inline int clamp_splits(int s) { return s >= 8 ? 8 : s >= 4 ? 4 : s >= 2 ? 2 : 1; }

template <int TRANS, int NT, int XV, class Epi>
int launch_kernel(const GemmArgs& g, const Epi& epi, cudaStream_t st) {
  constexpr size_t bytes = sizeof(double) * smem_doubles<TRANS, NT>();
  auto kern = dgemm_kernel<TRANS, NT, XV, Epi>;
  static bool attr_set = false;  // once per instantiation (callers hold the context lock)
  if (!attr_set) {
    RWIG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    attr_set = true;
  }
  cudaLaunchConfig_t cfg = {};
  const int tc = g.tcols > 0 ? g.tcols : NT * 8;
  cfg.gridDim = dim3((unsigned)(((g.Mo + BM - 1) / BM) * ((g.W + tc - 1) / tc)), 1, g.splits);
  cfg.blockDim = dim3(NTH);
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 1;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = (unsigned)g.splits;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  RWIG_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, g, epi));
  return 0;
}

// Y = op(K) X with epilogue `epi`.  g.splits <= 0 picks the split count,
// otherwise it is rounded down to 1, 2, 4 or 8.  Tiles of at most 32 columns
// run on 32-column CTAs, wider ones on 64-column CTAs; g.tcols (<= 64) fixes
// the columns per tile.  Returns 0 or an engine error code.
template <int TRANS, class Epi>
int gemm(const Context* ctx, GemmArgs g, const Epi& epi, cudaStream_t st) {
  if (!g.K || !g.X || g.Mo < 1 || g.Kd < 1 || g.W < 1)
    return set_error(RWIG_E_INVALID, "GEMM: null operand or empty shape");
  if ((g.ldk % 2) != 0 || (reinterpret_cast<uintptr_t>(g.K) % 16) != 0)
    return set_error(RWIG_E_INVALID, "GEMM operand K needs an even leading dimension and 16-byte alignment");
  if (g.ldk < (TRANS ? g.Kd : g.Mo) || g.ldx < g.Kd)
    return set_error(RWIG_E_INVALID, "GEMM: leading dimension smaller than the operand");
  const int NT = (g.tcols > 0 ? g.tcols : g.W) <= 32 ? 4 : 8;
  if (g.tcols < 0 || g.tcols > NT * 8) return set_error(RWIG_E_INVALID, "GEMM: tile columns above 64");
  if ((long long)((g.Mo + BM - 1) / BM) * ((g.W + (g.tcols > 0 ? g.tcols : NT * 8) - 1) /
                                          (g.tcols > 0 ? g.tcols : NT * 8)) > 0x7fffffffLL)
    return set_error(RWIG_E_INVALID, "GEMM: too many tiles");
  g.splits = g.splits <= 0 ? pick_splits(ctx, g.Mo, g.Kd, g.W, NT, g.tcols) : clamp_splits(g.splits);
  const bool xv2 = (g.ldx % 2) == 0 && (reinterpret_cast<uintptr_t>(g.X) % 16) == 0;
  if (NT == 4) return xv2 ? launch_kernel<TRANS, 4, 2>(g, epi, st) : launch_kernel<TRANS, 4, 1>(g, epi, st);
  return xv2 ? launch_kernel<TRANS, 8, 2>(g, epi, st) : launch_kernel<TRANS, 8, 1>(g, epi, st);
}

}  // namespace dg
}  // namespace rwig
