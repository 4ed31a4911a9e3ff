// common.cuh -- device helpers shared by the rwig_b200 kernels (sm_100a).
//
//  * mbarrier + 1-D bulk-copy (TMA) primitives, written as inline PTX;
//  * a bounded grid-wide barrier for cooperative (persistent) launches;
//  * bounded waits everywhere: a wait that runs out sets an error word in
//    global memory and returns, it never traps and never spins forever.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rwig {

// Error bits written by kernels into their control block.
enum : unsigned {
  KERR_BARRIER_TIMEOUT = 1u,  // grid barrier wait ran out
  KERR_MBAR_TIMEOUT = 2u,     // mbarrier (bulk copy) wait ran out
  KERR_NONFINITE = 4u,        // non-finite intermediate detected
};

// Wall-clock limit for any single device-side wait.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier -------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar` to complete, bounded in time.  Returns
// false (and leaves the phase incomplete) when the limit runs out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > kWaitLimitNs) return false;
  }
}

// 1-D bulk copy global -> shared, completion signalled on `bar` (non-multicast).
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Same, with an L2 eviction-priority hint (policy from createpolicy).
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes,
                                              uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], "
      "%2, [%3], %4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// ---- grid barrier -----------------------------------------------------------
// Counting grid barrier for a cooperative launch: the CTAs add 1 to *count
// at every barrier and wait until it reaches `target` = (barrier index + 1) *
// nblocks, so no generation word and no last-arriver step are needed.  Thread 0
// of each CTA fences (cumulative over the CTA's writes, ordered by the block
// barrier), arrives with a relaxed reduction and polls with acquire loads.
// The count must start at zero; the wait is bounded and sets *err on expiry.
__device__ __forceinline__ bool grid_sync(unsigned* count, unsigned* err, unsigned target) {
  __shared__ int s_ok2;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    asm volatile("red.relaxed.gpu.global.add.u32 [%0], 1;" ::"l"(count) : "memory");
    unsigned long long t0 = 0;
    for (unsigned spin = 0;; ++spin) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
      if ((int)(v - target) >= 0) break;
      if ((spin & 255u) == 0u) {
        if (*(volatile unsigned*)err != 0u) break;
        const unsigned long long now = globaltimer_ns();
        if (t0 == 0) t0 = now;
        else if (now - t0 > kWaitLimitNs) {
          atomicOr(err, KERR_BARRIER_TIMEOUT);
          break;
        }
      }
    }
    s_ok2 = (*(volatile unsigned*)err == 0u);
  }
  __syncthreads();
  return s_ok2 != 0;
}

// ---- warp reductions ------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace rwig
