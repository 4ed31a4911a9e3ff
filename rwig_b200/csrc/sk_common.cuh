// sk_common.cuh -- pieces shared by the column-strip Sinkhorn kernels: the
// bulk-copy stage ring over a CTA's columns, per-column block reductions and
// the fixed-order merge of per-CTA row partials.
#pragma once

#include "common.cuh"

namespace rwig {
namespace sk {

constexpr int STAGES = 3;

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

  // L2 priority: column groups below hot_groups are copied with an
  // evict_last hint (they stay resident between sweeps), the rest with
  // evict_first; hot_groups < 0 copies without a hint.
  int hot_groups = -1;
  uint64_t pol_hot = 0, pol_cold = 0;

  // thread 0 only
  __device__ void issue(unsigned seq) const {
    const int grp = (int)(seq % (unsigned)nst);
    const int jb = c0 + grp * CW;
    const unsigned bytes = (unsigned)(min(CW, c1 - jb) * ldc * 8);
    uint64_t* b = bar + (seq % STAGES);
    mbar_arrive_expect_tx(b, bytes);
    if (hot_groups < 0)
      bulk_g2s(slot(seq), C + (size_t)jb * ldc, bytes, b);
    else
      bulk_g2s_hint(slot(seq), C + (size_t)jb * ldc, bytes, b, grp < hot_groups ? pol_hot : pol_cold);
  }
  __device__ bool wait(unsigned seq) const { return mbar_wait_bounded(bar + (seq % STAGES), (seq / STAGES) & 1u); }
};

__device__ __forceinline__ void flag_error(unsigned* ctrl, unsigned bits) { atomicOr(ctrl + 2, bits); }

// Per-column block reduction: every warp ends with the same total per column.
template <int CW, int NW>
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

template <int CW, int NW>
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

// Sum over CTAs q = w, w + NW, ... of part[q * m + i], all loads in flight at
// once; the order is fixed, so every run gives the same bits.
template <int NW>
__device__ __forceinline__ double sum_partials(const double* part, int i, int m, int G, int w) {
  // every load of the batch is in flight at once (G <= 20 * NW)
  constexpr int U = 20;
  double v[U];
#pragma unroll
  for (int u = 0; u < U; ++u) v[u] = (w + u * NW < G) ? __ldcg(part + (size_t)(w + u * NW) * m + i) : 0.0;
  double acc = 0.0;
#pragma unroll
  for (int u = 0; u < U; ++u) acc += v[u];
  return acc;
}

}  // namespace sk
}  // namespace rwig
