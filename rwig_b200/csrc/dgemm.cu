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
  cudaStream_t st = call_stream(ctx, stream);
  // dgemm.kshape: the DMMA instruction's k extent (4, 8 or 16); dgemm.tile:
  // the tile height (0 automatic, 64, 128) for this check
  const int km = (int)option("dgemm.kshape", (double)dg::kDmmaK);
  const int tile = (int)option("dgemm.tile", 0.0);
  const bool forced = splits > 0;
  const int NT = S <= 32 ? 4 : 8;
  const bool wide = NT == 8 && (tile == 128 || (tile == 0 && dg::wide_tiles(Mo, S, 0) >= ctx->sm_count));
  // the split count of the (first) launch; the wide-tile path splits only a
  // tail wave on its own
  if (splits <= 0)
    splits = wide ? (dg::wide_tiles(Mo, S, 0) >= ctx->sm_count ? 1 : dg::pick_splits2(ctx, dg::wide_tiles(Mo, S, 0), Kd))
                  : dg::pick_splits(ctx, Mo, Kd, S, NT);
  else
    splits = wide ? std::min(splits, dg::kMaxSplits) : dg::clamp_splits(splits);
  dg::GemmArgs g{K, ldk, Mo, Kd, S, X, ldx, forced ? splits : 0};
  dg::EpiStore epi{Y, ldy, S};
  int rc;
  if (km == 16)
    rc = trans ? dg::gemm<1, dg::EpiStore, 16>(ctx, g, epi, st, tile) : dg::gemm<0, dg::EpiStore, 16>(ctx, g, epi, st, tile);
  else if (km == 8)
    rc = trans ? dg::gemm<1, dg::EpiStore, 8>(ctx, g, epi, st, tile) : dg::gemm<0, dg::EpiStore, 8>(ctx, g, epi, st, tile);
  else
    rc = trans ? dg::gemm<1, dg::EpiStore, 4>(ctx, g, epi, st, tile) : dg::gemm<0, dg::EpiStore, 4>(ctx, g, epi, st, tile);
  if (rc != 0) return rc;
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  RWIG_CUDA_TRY(cudaGetLastError());
  return splits;
}
