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

#include <algorithm>
#include <cstdint>

#include "engine.h"

namespace rwig {
namespace dg {

constexpr int BM = 64, BK = 32, NTH = 256, STAGES = 4;
constexpr int PAD = 4;  // doubles of padding per shared row
constexpr int kMaxSplits = 8;
constexpr int kDmmaK = 4;  // DMMA shape of the product paths (m16n8k4)

struct GemmArgs {
  const double* K;
  long long ldk;
  int Mo, Kd, W;     // output rows, contraction length, output columns
  const double* X;   // Kd x W, column-major
  long long ldx;
  int splits;        // cluster size along z: 1, 2, 4 or 8
  int tcols;         // output columns per tile (<= BN; 0: BN).  A multiple of an
                     // epilogue's column group keeps every group inside one tile.
  int tile0;         // first tile of the launch (wide-tile kernel; 0 otherwise)
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

// m16n8k8 and m16n8k16 (PTX ISA 7.8, sm_90 and later): thread (gid, tig)
// holds A(gid + 8 (i % 2), tig + 4 (i / 2)) in a_i and B(tig + 4 i, gid) in b_i.
__device__ __forceinline__ void mma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
__device__ __forceinline__ void mma_16x8x16(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
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
template <int TRANS, int NT, int XV, int BMT = BM>
__device__ __forceinline__ void load_stage(const GemmArgs& g, double* As, double* Bs, int m0, int n0, int tc,
                                           int k0, int kend) {
  const int tid = threadIdx.x;
  if (!TRANS) {
    // A[k][m] = K[m + k*ldk]: 32 k x BMT/2 m-pairs
#pragma unroll
    for (int c = 0; c < (BK * BMT / 2) / NTH; ++c) {
      const int idx = tid + c * NTH;
      const int kk = idx / (BMT / 2), mp = (idx % (BMT / 2)) * 2;
      const int gk = k0 + kk, gm = m0 + mp;
      int bytes = 0;
      const double* src = g.K;
      if (gk < kend && gm < g.Mo) {
        bytes = (gm + 1 < g.Mo) ? 16 : 8;
        src = g.K + gm + (long long)gk * g.ldk;
      }
      cp_async16(As + kk * (BMT + PAD) + mp, src, bytes);
    }
  } else {
    // A[m][k] = K[k + m*ldk]: BMT m x 16 k-pairs
#pragma unroll
    for (int c = 0; c < (BMT * BK / 2) / NTH; ++c) {
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

// KM: k extent of one DMMA instruction (4, 8 or 16).
template <int TRANS, int NT, int XV, class Epi, int KM>
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
    for (int k0 = 0; k0 < BK / 2; k0 += KM) {
      const int kk = kh + k0;
      // A(wm + gid + 8 (i % 2), kk + tig + 4 (i / 2)), i < KM / 2
      double a[KM / 2];
#pragma unroll
      for (int i = 0; i < KM / 2; ++i) {
        const int r = wm + gid + 8 * (i & 1), k = kk + tig + 4 * (i >> 1);
        a[i] = !TRANS ? A[k * (BM + PAD) + r] : A[r * (BK + PAD) + k];
      }
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const double* bp = B + (t * 8 + gid) * (BK + PAD) + kk + tig;
        if constexpr (KM == 4) {
          mma_16x8x4(acc[t], a[0], a[1], bp[0]);
        } else if constexpr (KM == 8) {
          const double b[2] = {bp[0], bp[4]};
          mma_16x8x8(acc[t], *reinterpret_cast<const double(*)[4]>(a), b);
        } else {
          const double b[4] = {bp[0], bp[4], bp[8], bp[12]};
          mma_16x8x16(acc[t], *reinterpret_cast<const double(*)[8]>(a), b);
        }
      }
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

// ---------------------------------------------------------------------------
// Wide-tile variant for long products with 64-column tiles: a BM2 x 64 tile
// per CTA (one CTA per SM), the 8 warps in a 4 x 2 grid of 32 x 32 blocks,
// each over the whole BK step (two m16 x four n8 DMMA tiles per k chunk, so a
// warp issues BK / KM * 8 DMMAs between barriers and reads 8 fragments per 8
// DMMAs).  Same operand ring, split-K cluster and epilogue interface as
// dgemm_kernel; without split-K the partial tile itself (row stride BM2 + 1)
// goes to the epilogue.
constexpr int BM2 = 128, STAGES2 = 4;
template <int TRANS>
__host__ __device__ constexpr int a2_stage_doubles() {
  return TRANS ? BM2 * (BK + PAD) : BK * (BM2 + PAD);
}
template <int TRANS>
__host__ __device__ constexpr int smem2_doubles() {
  // ring, or partial tile + epilogue scratch (no split), or partial tile +
  // summed rows + scratch (split-K, at most BM2 / 2 rows per CTA)
  constexpr int ring = STAGES2 * (a2_stage_doubles<TRANS>() + b_stage_doubles<8>());
  constexpr int e1 = 64 * (BM2 + 1) + 2 * 65 * (BM2 + 1);
  constexpr int e2 = 64 * (BM2 + 1) + 64 * (BM2 / 2) + 2 * 65 * (BM2 / 2);
  return ring > e1 ? (ring > e2 ? ring : e2) : (e1 > e2 ? e1 : e2);
}

template <int TRANS, int XV, class Epi, int KM>
__global__ void __launch_bounds__(NTH, 1) dgemm2_kernel(GemmArgs g, Epi epi) {
  extern __shared__ __align__(16) double smem[];
  constexpr int NT = 8, BN = 64;
  constexpr int ASZ = a2_stage_doubles<TRANS>(), BSZ = b_stage_doubles<NT>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int tc = g.tcols > 0 ? g.tcols : BN;
  const int ntiles = (g.W + tc - 1) / tc;
  const int tile = (int)blockIdx.x + g.tile0;
  const int m0 = (tile / ntiles) * BM2, n0 = (tile % ntiles) * tc;
  const int splits = g.splits;
  if (splits > 1 && (int)cluster_nctarank() != splits) return;
  const int z = blockIdx.z;
  int slice = (g.Kd + splits - 1) / splits;
  slice = ((slice + BK - 1) / BK) * BK;
  const int kbeg = z * slice;
  const int kend = min(g.Kd, kbeg + slice);
  const int nsteps = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;

  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][t][e] = 0.0;

  double* As = smem;
  double* Bs = smem + STAGES2 * ASZ;
#pragma unroll
  for (int s = 0; s < STAGES2 - 1; ++s) {
    if (s < nsteps)
      load_stage<TRANS, NT, XV, BM2>(g, As + s * ASZ, Bs + s * BSZ, m0, n0, tc, kbeg + s * BK, kend);
    cp_async_commit();
  }
  const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
  for (int s = 0; s < nsteps; ++s) {
    cp_async_wait<STAGES2 - 2>();
    __syncthreads();  // stage s visible; stage s-1 no longer read
    const int nx = s + STAGES2 - 1;
    if (nx < nsteps) {
      const int q = nx % STAGES2;
      load_stage<TRANS, NT, XV, BM2>(g, As + q * ASZ, Bs + q * BSZ, m0, n0, tc, kbeg + nx * BK, kend);
    }
    cp_async_commit();
    const double* A = As + (s % STAGES2) * ASZ;
    const double* B = Bs + (s % STAGES2) * BSZ;
#pragma unroll
    for (int kk = 0; kk < BK; kk += KM) {
      double a[2][KM / 2], b[4][KM / 4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int i = 0; i < KM / 2; ++i) {
          const int r = wm + 16 * mi + gid + 8 * (i & 1), k = kk + tig + 4 * (i >> 1);
          a[mi][i] = !TRANS ? A[k * (BM2 + PAD) + r] : A[r * (BK + PAD) + k];
        }
#pragma unroll
      for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int i = 0; i < KM / 4; ++i) b[t][i] = B[(wn + 8 * t + gid) * (BK + PAD) + kk + tig + 4 * i];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          if constexpr (KM == 4) mma_16x8x4(acc[mi][t], a[mi][0], a[mi][1], b[t][0]);
          else if constexpr (KM == 8) mma_16x8x8(acc[mi][t], a[mi], b[t]);
          else mma_16x8x16(acc[mi][t], a[mi], b[t]);
        }
    }
  }
  cp_async_wait<0>();
  __syncthreads();

  // partial tile -> shared memory, [c][r] with row stride BM2 + 1
  double* red = smem;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = wm + 16 * mi + gid + ((e >> 1) << 3);
        const int c = wn + 8 * t + tig * 2 + (e & 1);
        red[c * (BM2 + 1) + r] = acc[mi][t][e];
      }
  if (splits == 1) {
    __syncthreads();
    epi(m0, min(BM2, g.Mo - m0), n0, tc, red, BM2 + 1, red + BN * (BM2 + 1));
    return;
  }
  cluster_arrive();
  cluster_wait();
  // CTA z sums rows [z * rows, z * rows + nrl) of the tile; rows is a multiple
  // of 8 (at most BM2 / 2), so every CTA's first row is too
  const int rows = ((BM2 + splits - 1) / splits + 7) / 8 * 8;
  const int rl0 = z * rows;
  const int nrl = min(rows, BM2 - rl0);
  double* fin = red + BN * (BM2 + 1);
  double* ws = fin + BN * rows;
  for (int e = threadIdx.x; e < nrl * BN; e += NTH) {
    const int r = e % nrl, c = e / nrl;
    const double* p = red + c * (BM2 + 1) + rl0 + r;
    double v = 0.0;
    for (int q = 0; q < splits; ++q) v += ld_cluster(p, (unsigned)q);
    fin[c * rows + r] = v;
  }
  cluster_arrive();  // this CTA is done reading its peers
  __syncthreads();
  epi(m0 + rl0, min(nrl, g.Mo - (m0 + rl0)), n0, tc, fin, rows, ws);
  cluster_wait();  // peers are done reading this CTA
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

template <int TRANS, int NT, int XV, class Epi, int KM>
int launch_kernel(const GemmArgs& g, const Epi& epi, cudaStream_t st) {
  constexpr size_t bytes = sizeof(double) * smem_doubles<TRANS, NT>();
  auto kern = dgemm_kernel<TRANS, NT, XV, Epi, KM>;
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

template <int TRANS, int XV, class Epi, int KM>
int prepare_kernel2() {
  constexpr size_t bytes = sizeof(double) * smem2_doubles<TRANS>();
  static_assert(bytes <= 227 * 1024, "wide-tile GEMM exceeds the shared memory of a CTA");
  static bool attr_set = false;  // once per instantiation (callers hold the context lock)
  if (!attr_set) {
    RWIG_CUDA_TRY(cudaFuncSetAttribute(dgemm2_kernel<TRANS, XV, Epi, KM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bytes));
    attr_set = true;
  }
  return 0;
}

// Clusters of `s` wide-tile CTAs that can be resident at once (cached per
// instantiation; 0 if the query fails).
template <int TRANS, int XV, class Epi, int KM>
int max_clusters2(int s) {
  static int cache[kMaxSplits + 1] = {};
  if (cache[s] == 0) {
    if (prepare_kernel2<TRANS, XV, Epi, KM>() != 0) return 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1, 1, (unsigned)s);
    cfg.blockDim = dim3(NTH);
    cfg.dynamicSmemBytes = sizeof(double) * smem2_doubles<TRANS>();
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 1;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = (unsigned)s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, dgemm2_kernel<TRANS, XV, Epi, KM>, &cfg) != cudaSuccess || n < 1) {
      (void)cudaGetLastError();
      n = -1;
    }
    cache[s] = n;
  }
  return cache[s] > 0 ? cache[s] : 0;
}

template <int TRANS, int XV, class Epi, int KM>
int launch_kernel2(const GemmArgs& g, const Epi& epi, cudaStream_t st, int ntile) {
  constexpr size_t bytes = sizeof(double) * smem2_doubles<TRANS>();
  auto kern = dgemm2_kernel<TRANS, XV, Epi, KM>;
  if (int rc = prepare_kernel2<TRANS, XV, Epi, KM>()) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ntile, 1, g.splits);
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
// Split count of the wide-tile kernel (one CTA per SM) for `tiles` tiles:
// the largest count up to 8 that keeps the CTAs within one wave and every
// slice at least four BK steps.
inline int pick_splits2(const Context* ctx, long long tiles, int Kd) {
  int s = 1;
  while (s < kMaxSplits && tiles * (s + 1) <= ctx->sm_count && Kd >= (s + 1) * 4 * BK) ++s;
  return s;
}
inline long long wide_tiles(int Mo, int W, int tc) {
  if (tc <= 0) tc = 64;
  return (long long)((Mo + BM2 - 1) / BM2) * ((W + tc - 1) / tc);
}

// Wide-tile product: whole waves of unsplit tiles, then the tiles of a last
// partial wave (when they fill at most half the SMs) as a second launch with
// split-K, so the tail takes a fraction of a wave.
template <int TRANS, int XV, class Epi, int KM>
int gemm_wide(const Context* ctx, GemmArgs g, const Epi& epi, cudaStream_t st, int* launches) {
  const long long tiles = wide_tiles(g.Mo, g.W, g.tcols);
  const int sm = ctx->sm_count;
  if (g.splits > 0 || tiles < sm) {
    g.splits = g.splits > 0 ? std::min(g.splits, kMaxSplits) : pick_splits2(ctx, tiles, g.Kd);
    g.tile0 = 0;
    if (launches) ++*launches;
    return launch_kernel2<TRANS, XV, Epi, KM>(g, epi, st, (int)tiles);
  }
  const long long tail = tiles % sm;
  const long long full = (tail > 0 && 2 * tail <= sm) ? tiles - tail : tiles;
  g.splits = 1;
  g.tile0 = 0;
  if (launches) ++*launches;
  int rc = launch_kernel2<TRANS, XV, Epi, KM>(g, epi, st, (int)full);
  if (rc != 0 || full == tiles) return rc;
  // split count of the tail: the least waves of resident clusters per slice,
  // ceil(tail / clusters(s)) / s (clusters wider than a TPC pair may leave SMs
  // idle, so the count of resident clusters is asked of the runtime)
  int best = 1;
  double best_t = 1.0;
  for (int s = 2; s <= kMaxSplits && g.Kd >= s * 4 * BK; ++s) {
    const int nc = max_clusters2<TRANS, XV, Epi, KM>(s);
    if (nc < 1) continue;
    const double t = (double)((tail + nc - 1) / nc) / s;
    if (t < best_t - 1e-9) {
      best_t = t;
      best = s;
    }
  }
  g.splits = best;
  g.tile0 = (int)full;
  if (launches) ++*launches;
  return launch_kernel2<TRANS, XV, Epi, KM>(g, epi, st, (int)(tiles - full));
}

// tile: 0 picks the tile height (128 rows for tiles of more than 32 columns
// when the unsplit 128-row tiles fill every SM, else 64), 64 or 128 forces it
// (128 only for tiles of more than 32 columns).  launches (optional) is
// incremented by the number of kernel launches made (1, or 2 with a split
// tail wave).
template <int TRANS, class Epi, int KM = kDmmaK>
int gemm(const Context* ctx, GemmArgs g, const Epi& epi, cudaStream_t st, int tile = 0, int* launches = nullptr) {
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
  const bool xv2 = (g.ldx % 2) == 0 && (reinterpret_cast<uintptr_t>(g.X) % 16) == 0;
  if (tile == 0) tile = (NT == 8 && wide_tiles(g.Mo, g.W, g.tcols) >= ctx->sm_count) ? 128 : 64;
  if (NT == 8 && tile == 128)
    return xv2 ? gemm_wide<TRANS, 2, Epi, KM>(ctx, g, epi, st, launches)
               : gemm_wide<TRANS, 1, Epi, KM>(ctx, g, epi, st, launches);
  g.splits = g.splits <= 0 ? pick_splits(ctx, g.Mo, g.Kd, g.W, NT, g.tcols) : clamp_splits(g.splits);
  if (launches) ++*launches;
  if (NT == 4)
    return xv2 ? launch_kernel<TRANS, 4, 2, Epi, KM>(g, epi, st) : launch_kernel<TRANS, 4, 1, Epi, KM>(g, epi, st);
  return xv2 ? launch_kernel<TRANS, 8, 2, Epi, KM>(g, epi, st) : launch_kernel<TRANS, 8, 1, Epi, KM>(g, epi, st);
}

}  // namespace dg
}  // namespace rwig
