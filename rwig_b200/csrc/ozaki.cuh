// ozaki.cuh -- FP64 matrix products op(K) X on the INT8 tensor cores
// (tcgen05 kind::i8), exact integer products recombined by the Chinese
// remainder theorem: the scheme of Y. Uchino, K. Ozaki and T. Imamura,
// "Performance enhancement of the Ozaki Scheme on integer matrix
// multiplication unit" (Ozaki scheme II, 2024/2025), written here for the
// skinny products of the WDL step.
//
//   1. Scaling.  Row i of A = op(K) is scaled by 2^alpha_i and column j of X
//      by 2^beta_j (powers of two: exact) so that the largest magnitude of the
//      row / column is just below 2^q; truncation toward zero gives integer
//      matrices Ah, Xh with |entries| < 2^q (an entry loses bits only where it
//      is below 2^(53-q) of its row's / column's largest).
//   2. Residues.  For T pairwise coprime moduli p_t <= 256 the residues
//      Ah mod p_t, Xh mod p_t in [0, p_t) fit in uint8.
//   3. Products.  D_t = (Ah mod p_t)(Xh mod p_t) is exact in the tensor
//      cores' int32 accumulators (0 <= D_t <= Kd 255^2 < 2^31 for Kd <= 33000);
//      c_t = D_t mod p_t in [0, p_t) (ozaki.cu).
//   4. Reconstruction.  With P = prod p_t, M_t = P / p_t and e_t = M_t
//      (M_t^-1 mod p_t), Ch = Ah Xh is the representative in (-P/2, P/2) of
//      sum_t c_t e_t mod P.  Here frac(sum_t c_t e_t / P) is accumulated in
//      256-bit fixed point from F_t = floor(2^256 e_t / P) (the mod-1
//      reduction is the fixed point's overflow), read as a signed fraction s,
//      and Ch = s P; the result is 2^-(alpha_i + beta_j) Ch, rounded once.
//      Sizes keep Kd 2^(2q) < P / 2, so Ch is the exact integer product.
//
// With T = 24 moduli (log2 P = 184.09) and q = 85 the product is exact for
// the truncated inputs; the only errors are the truncation of entries far
// below their row's / column's maximum (relative 2^-85 of that maximum) and
// the final rounding.  The reconstruction writes the FP64 product; a tile
// kernel then hands each output tile to the same epilogue functors as the
// DMMA GEMM (dgemm.cuh contract).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dgemm.cuh"
#include "engine.h"

namespace rwig {
namespace oz {

constexpr int kT = 24;        // moduli
constexpr int kQ = 85;        // bits of the scaled integers
constexpr int kMaxKd = 8192;  // contraction length for which kQ is safe: Kd 2^(2 kQ) < P / 2
constexpr int kTileM = 128;   // UMMA M
constexpr int kBk = 64;       // bytes of K per pipeline stage (one 64-byte swizzle atom)
constexpr int kKpadTo = 128;  // the contraction is padded to a multiple of this
constexpr int kCrtRows = 16;  // rows per epilogue tile (26 KB of shared memory: fits beside a GEMM CTA)
constexpr int kCrtCols = 64;  // most columns per epilogue tile (the DMMA GEMM's widest tile)
constexpr int kCrtThreads = 256;

// Reconstruction constants, passed by value to the kernels.
struct Crt {
  int p[kT];
  double invp[kT];
  unsigned F32[kT][8];  // floor(2^256 e_t / P), little-endian 32-bit limbs
  double P;                     // P rounded to double
};

// Host: the moduli and reconstruction constants (computed once).
const Crt& crt_constants();

// op(K) as the tensor cores' A operand: residues [kT][Mpad][Kpad] (K-major
// uint8) and the row exponents alpha (Mo ints), for trans = 0 (K, rows of K)
// and trans = 1 (K^T, columns of K).
struct Prepared {
  const double* K = nullptr;
  long long ldk = 0;
  int Mo = 0, Kd = 0, Mpad = 0, Kpad = 0;
  int8_t* ares[2] = {nullptr, nullptr};
  int* alpha[2] = {nullptr, nullptr};
};

// Residues and exponents of op(K) for trans = 0 and 1 (square K: Mo = Kd),
// into engine scratch slots; starts a sequence of products whose bounded-wait
// failures status() reports.  Returns 0 or an engine error.
int prepare(Context* ctx, const double* K, long long ldk, int n, Prepared* pr, cudaStream_t st, int* launches);

// X's residues and the kT integer products: cres[t][j][i] = (A_t X_t)_ij mod
// p_t for i < Mo, j < W (pitch Mpad per column, Wpad columns per modulus),
// beta (W ints), in the scratch of `lane` (products on different streams at
// once use different lanes).  Returns 0 or an engine error.
int products(Context* ctx, const Prepared& pr, int trans, const double* X, long long ldx, int W, cudaStream_t st,
             const uint8_t** cres, const int** beta, int* Wpad, int* launches, int lane);

// Status of the bounded waits of the INT8 GEMMs enqueued on `st` since
// prepare() (synchronises): 0 or RWIG_E_TIMEOUT.
int status(Context* ctx, cudaStream_t st);

// Whether the INT8 tensor-core path can run: sm_100 class device with the
// driver's tensor-map entry point.
bool available(Context* ctx);

// Y (Mo x W, ldy) = op(K) X from the residue planes of products():
// reconstruction and scaling (ozaki.cu).
int reconstruct(Context* ctx, const Prepared& pr, int trans, const uint8_t* cres, int Wpad, const int* beta, int W,
                double* Y, long long ldy, cudaStream_t st, int* launches);

// Scratch of `lane` for the FP64 product (Mo x W doubles).
double* product_buffer(Context* ctx, size_t doubles, int lane);

// Tiles of kCrtRows x tc of Y handed to the epilogue (the dgemm.cuh
// contract: value (r0 + r, c0 + c) at t[c * ldt + r], columns >= W zero,
// 2 (kCrtCols + 1) ldt doubles of workspace).
template <class Epi>
__global__ void __launch_bounds__(kCrtThreads) epi_tiles(const double* __restrict__ Y, long long ldy, int Mo, int W,
                                                         int tc, Epi epi) {
  extern __shared__ double sm[];
  constexpr int ldt = kCrtRows + 1;
  double* tile = sm;                         // [tc][ldt]
  double* ws = sm + (size_t)kCrtCols * ldt;  // 2 (kCrtCols + 1) ldt doubles
  const int r0 = blockIdx.x * kCrtRows, c0 = blockIdx.y * tc;
  const int nr = min(kCrtRows, Mo - r0);
  for (int e = threadIdx.x; e < kCrtRows * tc; e += blockDim.x) {
    const int r = e % kCrtRows, cc = e / kCrtRows;
    tile[cc * ldt + r] = (r < nr && c0 + cc < W) ? Y[(long long)(r0 + r) + (long long)(c0 + cc) * ldy] : 0.0;
  }
  __syncthreads();
  epi(r0, nr, c0, tc, tile, ldt, ws);
}

inline size_t epi_smem_bytes() { return sizeof(double) * (size_t)(kCrtCols + 2 * (kCrtCols + 1)) * (kCrtRows + 1); }

// Y = op(K) X through the INT8 tensor cores, each output tile handed to
// `epi` (the dgemm.cuh epilogue contract, tiles of kCrtRows rows and tc
// columns).  *launches += the kernels launched.
template <class Epi>
int gemm(Context* ctx, const Prepared& pr, int trans, const double* X, long long ldx, int W, int tc, const Epi& epi,
         cudaStream_t st, int* launches, int lane = 0) {
  const uint8_t* cres = nullptr;
  const int* beta = nullptr;
  int Wpad = 0;
  if (int rc = products(ctx, pr, trans, X, ldx, W, st, &cres, &beta, &Wpad, launches, lane)) return rc;
  double* Y = product_buffer(ctx, (size_t)pr.Mo * W, lane);
  if (!Y) return RWIG_E_NOMEM;
  if (int rc = reconstruct(ctx, pr, trans, cres, Wpad, beta, W, Y, pr.Mo, st, launches)) return rc;
  if (tc <= 0 || tc > kCrtCols) tc = kCrtCols;
  static bool attr = false;  // once per instantiation (callers hold the context lock)
  const size_t smem = epi_smem_bytes();
  if (!attr) {
    RWIG_CUDA_TRY(cudaFuncSetAttribute(epi_tiles<Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  const dim3 grid((pr.Mo + kCrtRows - 1) / kCrtRows, (W + tc - 1) / tc);
  epi_tiles<Epi><<<grid, kCrtThreads, smem, st>>>(Y, pr.Mo, pr.Mo, W, tc, epi);
  if (launches) ++*launches;
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace oz
}  // namespace rwig
