// dgemm.cu -- self-check entry point of the FP64 DMMA GEMM (dgemm.cuh).
#include "dgemm.cuh"
#include "engine.h"

using namespace rwig;

extern "C" int rwig_selftest_dgemm(const double* K, long long ldk, int trans, int Mo, int Kd, int S,
                                   const double* X, long long ldx, double* Y, long long ldy, int splits,
                                   void* stream) {
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!K || !X || !Y || Mo < 1 || Kd < 1 || S < 1 || ldy < Mo) return set_error(RWIG_E_INVALID, "bad arguments");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  const int NT = S <= 32 ? 4 : 8;
  splits = splits <= 0 ? dg::pick_splits(ctx, Mo, Kd, S, NT) : dg::clamp_splits(splits);
  dg::GemmArgs g{K, ldk, Mo, Kd, S, X, ldx, splits};
  dg::EpiStore epi{Y, ldy, S};
  const int rc = trans ? dg::gemm<1>(ctx, g, epi, st) : dg::gemm<0>(ctx, g, epi, st);
  if (rc != 0) return rc;
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  RWIG_CUDA_TRY(cudaGetLastError());
  return splits;
}
