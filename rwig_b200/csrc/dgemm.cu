// dgemm.cu -- launch helpers for the FP64 DMMA GEMM (dgemm.cuh) and its
// self-check entry point.
#include <algorithm>

#define RWIG_DGEMM_DEFINE_KERNEL
#include "dgemm.cuh"
#include "engine.h"

namespace rwig {

int dgemm_splitk(Context* ctx, const dg::GemmArgs& args, cudaStream_t st) {
  if ((args.ldk % 2) != 0 || (reinterpret_cast<uintptr_t>(args.K) % 16) != 0)
    return set_error(RWIG_E_INVALID, "GEMM operand K needs an even leading dimension and 16-byte alignment");
  dim3 grid((args.Mo + dg::BM - 1) / dg::BM, (args.S + dg::BN - 1) / dg::BN, args.splits);
  dg::dgemm_splitk_kernel<<<grid, dg::NTH, 0, st>>>(args);
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Splits chosen to put about two waves of CTAs on the GPU, each slice at least
// 64 long.
int dgemm_pick_splits(Context* ctx, int Mo, int Kd, int S) {
  const long long tiles = (long long)((Mo + dg::BM - 1) / dg::BM) * ((S + dg::BN - 1) / dg::BN);
  long long want = (2LL * ctx->sm_count + tiles - 1) / tiles;
  want = std::min<long long>(want, std::max(1, Kd / 64));
  return (int)std::max<long long>(1, std::min<long long>(want, 64));
}

namespace {
__global__ void reduce_plain(const double* part, int splits, int Mo, int S, double* Y, long long ldy) {
  const long long total = (long long)Mo * S;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(k % Mo), c = (int)(k / Mo);
    Y[r + c * ldy] = dg::reduce_splits(part, splits, Mo, S, r, c);
  }
}
}  // namespace

}  // namespace rwig

using namespace rwig;

extern "C" int rwig_selftest_dgemm(const double* K, long long ldk, int trans, int Mo, int Kd, int S,
                                   const double* X, long long ldx, double* Y, long long ldy, int splits,
                                   void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!K || !X || !Y || Mo < 1 || Kd < 1 || S < 1) return set_error(RWIG_E_INVALID, "bad arguments");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  if (splits <= 0) splits = dgemm_pick_splits(ctx, Mo, Kd, S);
  double* part = (double*)scratch(ctx, 40, sizeof(double) * (size_t)splits * Mo * S);
  if (!part) return RWIG_E_NOMEM;
  dg::GemmArgs g{K, ldk, trans, Mo, Kd, S, X, ldx, part, splits};
  int rc = dgemm_splitk(ctx, g, st);
  if (rc != 0) return rc;
  reduce_plain<<<std::max(1, std::min((Mo * S + 255) / 256, 8 * ctx->sm_count)), 256, 0, st>>>(part, splits, Mo,
                                                                                                 S, Y, ldy);
  RWIG_CUDA_TRY(cudaGetLastError());
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  return splits;
}
