// fastexp.cuh -- table-driven FP64 exponential for the solver's inner loops.
//
// Method: P. T. P. Tang, "Table-driven implementation of the exponential
// function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989.
//   x = (64 m + j) ln2/64 + r,  |r| <= ln2/128,
//   exp(x) = 2^m * 2^(j/64) * exp(r),
// with k = round(x * 64/ln2) obtained by the 1.5*2^52 shifter, r reduced with
// a two-constant (Cody-Waite) split of ln2/64 evaluated by FMA, exp(r) - 1 by
// its degree-5 Taylor polynomial (truncation < 4e-17 relative for |r| <= ln2/128)
// and 2^(j/64) from a 64-entry table held in shared memory.  The table entries
// and the split of ln2/64 were computed in 60-digit decimal arithmetic and
// rounded to nearest.  Accuracy: within 2 ulp of the correctly rounded result
// for x in [-708, 709] (tests/test_gpu_fastexp.py compares it with CUDA's exp
// on the device).  The input is clamped to [-708, 709] first, so smaller
// arguments (and NaN) return exp(-708) ~ 3.3e-308 and larger ones exp(709):
// the solver only sums these values against terms of order one or checks the
// sums' range, so the floor is below its rounding.  No branches.
#pragma once

#include <cstdint>

namespace rwig {

static __constant__ unsigned long long kExp2J64[64] = {
    0x3ff0000000000000ull, 0x3ff02c9a3e778061ull, 0x3ff059b0d3158574ull, 0x3ff0874518759bc8ull,
    0x3ff0b5586cf9890full, 0x3ff0e3ec32d3d1a2ull, 0x3ff11301d0125b51ull, 0x3ff1429aaea92de0ull,
    0x3ff172b83c7d517bull, 0x3ff1a35beb6fcb75ull, 0x3ff1d4873168b9aaull, 0x3ff2063b88628cd6ull,
    0x3ff2387a6e756238ull, 0x3ff26b4565e27cddull, 0x3ff29e9df51fdee1ull, 0x3ff2d285a6e4030bull,
    0x3ff306fe0a31b715ull, 0x3ff33c08b26416ffull, 0x3ff371a7373aa9cbull, 0x3ff3a7db34e59ff7ull,
    0x3ff3dea64c123422ull, 0x3ff4160a21f72e2aull, 0x3ff44e086061892dull, 0x3ff486a2b5c13cd0ull,
    0x3ff4bfdad5362a27ull, 0x3ff4f9b2769d2ca7ull, 0x3ff5342b569d4f82ull, 0x3ff56f4736b527daull,
    0x3ff5ab07dd485429ull, 0x3ff5e76f15ad2148ull, 0x3ff6247eb03a5585ull, 0x3ff6623882552225ull,
    0x3ff6a09e667f3bcdull, 0x3ff6dfb23c651a2full, 0x3ff71f75e8ec5f74ull, 0x3ff75feb564267c9ull,
    0x3ff7a11473eb0187ull, 0x3ff7e2f336cf4e62ull, 0x3ff82589994cce13ull, 0x3ff868d99b4492edull,
    0x3ff8ace5422aa0dbull, 0x3ff8f1ae99157736ull, 0x3ff93737b0cdc5e5ull, 0x3ff97d829fde4e50ull,
    0x3ff9c49182a3f090ull, 0x3ffa0c667b5de565ull, 0x3ffa5503b23e255dull, 0x3ffa9e6b5579fdbfull,
    0x3ffae89f995ad3adull, 0x3ffb33a2b84f15fbull, 0x3ffb7f76f2fb5e47ull, 0x3ffbcc1e904bc1d2ull,
    0x3ffc199bdd85529cull, 0x3ffc67f12e57d14bull, 0x3ffcb720dcef9069ull, 0x3ffd072d4a07897cull,
    0x3ffd5818dcfba487ull, 0x3ffda9e603db3285ull, 0x3ffdfc97337b9b5full, 0x3ffe502ee78b3ff6ull,
    0x3ffea4afa2a490daull, 0x3ffefa1bee615a27ull, 0x3fff50765b6e4540ull, 0x3fffa7c1819e90d8ull,
};

// Copies the 2^(j/64) table into shared memory (64 doubles); the caller
// synchronises the block before the first exp_tbl.
__device__ __forceinline__ void load_exp_table(double* tbl) {
  for (int i = threadIdx.x; i < 64; i += blockDim.x) tbl[i] = __longlong_as_double((long long)kExp2J64[i]);
}

// Bank-spread copy: 16 replicas interleaved, entry j of replica r at
// [16 j + r] (1024 doubles).  Lane l reads replica l % 16, so the 16 lanes of
// a 64-bit shared-memory phase always hit 16 distinct bank pairs.
constexpr int kExpTableSpread = 16;
__device__ __forceinline__ void load_exp_table_spread(double* tbl) {
  for (int i = threadIdx.x; i < 64 * kExpTableSpread; i += blockDim.x)
    tbl[i] = __longlong_as_double((long long)kExp2J64[i / kExpTableSpread]);
}

// tbl: the table as laid out by load_exp_table (stride 1) or, with
// STRIDE = kExpTableSpread, by load_exp_table_spread offset by the lane's replica.
template <int STRIDE = 1>
__device__ __forceinline__ double exp_tbl(double x, const double* tbl) {
  const double kInvLn2_64 = 92.33248261689366;          // 64 / ln 2
  const double kLn2_64_hi = 0.010830424696249145;       // ln2/64 rounded to double
  const double kLn2_64_lo = 3.623510646634843e-19;      // ln2/64 - kLn2_64_hi
  const double kShifter = 6755399441055744.0;           // 1.5 * 2^52
  const double xc = fmin(fmax(x, -708.0), 709.0);
  const double t = fma(xc, kInvLn2_64, kShifter);
  const int k = __double2loint(t);
  const double kd = t - kShifter;
  double r = fma(kd, -kLn2_64_hi, xc);
  r = fma(kd, -kLn2_64_lo, r);
  double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = p * r;  // exp(r) - 1
  const double tj = tbl[(k & 63) * STRIDE];
  const double y = fma(tj, p, tj);
  const double scale = __hiloint2double(((k >> 6) + 1023) << 20, 0);
  return y * scale;
}

}  // namespace rwig

namespace rwig {
// 1/x to within 2 ulp: for |x| in [2^-120, 2^120] a single-precision seed
// refined by two Newton-Raphson steps y <- y + y (1 - x y) in FP64 (each step
// squares the relative error: 2^-22 -> 2^-44 -> below 2^-53).  Outside that
// range (where the float seed would be 0, inf or subnormal), and for 0, inf
// and NaN, the IEEE division 1.0 / x.
__device__ __forceinline__ double rcp_nr(double x) {
  const double ax = fabs(x);
  if (!(ax >= 0x1p-120 && ax <= 0x1p120)) return 1.0 / x;
  double y = (double)(1.0f / (float)x);
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
}  // namespace rwig
