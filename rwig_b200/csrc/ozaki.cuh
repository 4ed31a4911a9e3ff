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
// the final rounding.  The reconstruction runs tile by tile in the kernel
// that hands each output tile to the same epilogue functors as the DMMA GEMM
// (dgemm.cuh contract), so the FP64 product never goes through memory.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

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
constexpr int kCrtRows = 32;  // rows per epilogue tile: one 32-byte sector per residue column
constexpr int kCrtCols = 64;  // most columns per epilogue tile (the DMMA GEMM's widest tile)
constexpr int kCrtThreads = 256;
constexpr int kCrtRowsPerThread = 2;

// Reconstruction constants, passed by value to the kernels.
struct Crt {
  int p[kT];
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

// prepare(), unless the scratch already holds the residue planes of a K equal
// to this one bit for bit (compared against a device copy of the K they were
// made from: one read of both, a host synchronisation); then only the
// sequence's error word is reset.
int prepare_reuse(Context* ctx, const double* K, long long ldk, int n, Prepared* pr, cudaStream_t st,
                  int* launches);

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

// The signed fraction held in eight 32-bit limb sums (carries pending; limbs
// below l0 taken as zero), as |s| and its sign: the 256-bit fixed-point
// value read in [-1/2, 1/2).
__device__ __forceinline__ double limbs_to_fraction(const unsigned long long (&acc)[8], int l0, bool& neg) {
  unsigned limb[8];
  unsigned long long carry = 0ull;
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    const unsigned long long x = (l >= l0 ? acc[l] : 0ull) + carry;
    limb[l] = (unsigned)x;
    carry = x >> 32;
  }
  neg = (limb[7] >> 31) != 0;
  if (neg) {  // two's complement negation of the 256-bit value
    unsigned long long b = 1ull;
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const unsigned long long x = (unsigned long long)(~limb[l]) + b;
      limb[l] = (unsigned)x;
      b = x >> 32;
    }
  }
  return ldexp((double)(((unsigned long long)limb[7] << 32) | limb[6]), -64) +
         ldexp((double)(((unsigned long long)limb[5] << 32) | limb[4]), -128) +
         ldexp((double)(((unsigned long long)limb[3] << 32) | limb[2]), -192);
}

// Reconstruction of rows i0 .. i0 + RP - 1 (RP = 2 or 4, i0 a multiple of
// RP) of column j from the residue planes cres[t][j][i] (pitch Mpad, plane
// stride `plane` bytes): the fraction frac(sum_t c_t e_t / P) is accumulated
// as 32-bit limb sums in 64-bit registers (each below 24 * 255 * 2^32 <
// 2^45, so the carries wait until the end), read as a signed fraction s, and
// y = s P 2^-(alpha_i + beta).  Fast path: the four upper limbs alone.  The
// lower ones add less than 24 * 255 * 2^-128 < 2^-115 to s, within 2^-55 of
// |s| once |s| >= 2^-60; smaller values are recomputed with all eight.  Rows
// at or beyond Mo give 0.
template <int RP>
__device__ __forceinline__ void crt_rows(const Crt& c, const uint8_t* __restrict__ cres, size_t plane, int Mpad, int i0,
                                         int j, const int* __restrict__ alpha, int beta, int Mo, double (&y)[RP]) {
  using Word = typename std::conditional<RP == 4, unsigned, unsigned short>::type;
  const Word* q = reinterpret_cast<const Word*>(cres + (size_t)j * Mpad + i0);
  const size_t pw = plane / RP;  // plane stride in words
  unsigned long long acc[RP][4];
#pragma unroll
  for (int u = 0; u < RP; ++u)
#pragma unroll
    for (int l = 0; l < 4; ++l) acc[u][l] = 0ull;
  unsigned w[kT];
#pragma unroll
  for (int t = 0; t < kT; ++t) w[t] = __ldg(q + t * pw);  // all loads in flight at once
#pragma unroll
  for (int t = 0; t < kT; ++t)
#pragma unroll
    for (int u = 0; u < RP; ++u) {
      const unsigned ct = (w[t] >> (8 * u)) & 0xffu;
#pragma unroll
      for (int l = 0; l < 4; ++l) acc[u][l] += (unsigned long long)ct * c.F32[t][4 + l];
    }
#pragma unroll
  for (int u = 0; u < RP; ++u) {
    const int i = i0 + u;
    if (i >= Mo) {
      y[u] = 0.0;
      continue;
    }
    unsigned long long a8[8] = {0ull, 0ull, 0ull, 0ull, acc[u][0], acc[u][1], acc[u][2], acc[u][3]};
    bool neg;
    double mag = limbs_to_fraction(a8, 4, neg);
    if (mag < 0x1p-60) {  // small: the lower limbs matter (residues reloaded)
#pragma unroll
      for (int l = 0; l < 8; ++l) a8[l] = 0ull;
#pragma unroll 1
      for (int t = 0; t < kT; ++t) {
        const unsigned ct = ((unsigned)__ldg(q + t * pw) >> (8 * u)) & 0xffu;
#pragma unroll
        for (int l = 0; l < 8; ++l) a8[l] += (unsigned long long)ct * c.F32[t][l];
      }
      mag = limbs_to_fraction(a8, 0, neg);
    }
    y[u] = ldexp(neg ? -mag * c.P : mag * c.P, -(alpha[i] + beta));
  }
}

// Tiles of kCrtRows x tc of Y = op(K) X, reconstructed from the residue
// planes of products() into shared memory and handed to the epilogue (the
// dgemm.cuh contract: value (r0 + r, c0 + c) at t[c * ldt + r], columns >= W
// zero, 2 (kCrtCols + 1) ldt doubles of workspace).  Each thread takes
// kCrtRowsPerThread consecutive rows of one column: one load per residue
// plane.
template <class Epi>
__global__ void __launch_bounds__(kCrtThreads) crt_tiles(Crt c, const uint8_t* __restrict__ cres, int Mpad, int Wpad,
                                                         const int* __restrict__ alpha, const int* __restrict__ beta,
                                                         int Mo, int W, int tc, Epi epi) {
  extern __shared__ double sm[];
  constexpr int ldt = kCrtRows + 1;
  constexpr int RP = kCrtRowsPerThread, groups = kCrtRows / RP;
  double* tile = sm;                         // [tc][ldt]
  double* ws = sm + (size_t)kCrtCols * ldt;  // 2 (kCrtCols + 1) ldt doubles
  const int r0 = blockIdx.x * kCrtRows, c0 = blockIdx.y * tc;
  const int nr = min(kCrtRows, Mo - r0);
  const size_t plane = (size_t)Wpad * Mpad;
  for (int e = threadIdx.x; e < groups * tc; e += blockDim.x) {
    const int rg = e % groups, cc = e / groups, j = c0 + cc;
    double y[RP];
#pragma unroll
    for (int u = 0; u < RP; ++u) y[u] = 0.0;
    if (j < W && r0 + RP * rg < Mo) crt_rows<RP>(c, cres, plane, Mpad, r0 + RP * rg, j, alpha, beta[j], Mo, y);
#pragma unroll
    for (int u = 0; u < RP; ++u) tile[cc * ldt + RP * rg + u] = y[u];
  }
  __syncthreads();
  epi(r0, nr, c0, tc, tile, ldt, ws);
}

inline size_t epi_smem_bytes() { return sizeof(double) * (size_t)(kCrtCols + 2 * (kCrtCols + 1)) * (kCrtRows + 1); }

// Row exponents alpha of op(K) (trans) for the reconstruction.
inline const int* row_exponents(const Prepared& pr, int trans) { return pr.alpha[trans]; }

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
  if (tc <= 0 || tc > kCrtCols) tc = kCrtCols;
  static bool attr = false;  // once per instantiation (callers hold the context lock)
  const size_t smem = epi_smem_bytes();
  if (!attr) {
    RWIG_CUDA_TRY(cudaFuncSetAttribute(crt_tiles<Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  const dim3 grid((pr.Mo + kCrtRows - 1) / kCrtRows, (W + tc - 1) / tc);
  crt_tiles<Epi><<<grid, kCrtThreads, smem, st>>>(crt_constants(), cres, pr.Mpad, Wpad, row_exponents(pr, trans), beta,
                                                   pr.Mo, W, tc, epi);
  if (launches) ++*launches;
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace oz
}  // namespace rwig
