// ozaki.cu -- the INT8 tensor-core half of the emulated FP64 products
// (ozaki.cuh): reconstruction constants, scaling exponents, residues, and
// the tcgen05 kind::i8 GEMM of the residue planes.
//
// GEMM kernel (one CTA per 256 x ntile output tile of one modulus, 256
// threads):
//   * operands are K-major uint8 planes [T][rows][Kpad]; TMA (3-D tensor
//     maps, 64-byte swizzle) copies 256 x 64-byte A tiles and ntile x 64-byte
//     B tiles into a 6-stage shared-memory ring, full / empty mbarriers (a
//     deep ring of small stages: the copies' latency, not the L2 bandwidth,
//     bounds a shallower one);
//   * thread 0 issues the copies, thread 32 the MMAs: per stage and per
//     128-row half two tcgen05.mma.cta_group::1.kind::i8 of K = 32 (the
//     shared-memory descriptors advanced by 32 bytes inside the swizzle
//     atom) into int32 accumulators in tensor memory, then tcgen05.commit
//     frees the stage;
//   * the eight warps read the accumulators back (tcgen05.ld 32x32b, warp w
//     owns lanes 32 (w % 4) .. +31 = rows of half w / 4), reduce them modulo
//     p_t and store one byte per entry.
// Every wait is bounded (2 s): a wait that runs out sets the error word and
// the kernel winds down (the MMA thread still commits what it issued, the
// tensor memory is freed), and the host reports RWIG_E_TIMEOUT.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "ozaki.cuh"

namespace rwig {
namespace oz {

// ---------------------------------------------------------------------------
// reconstruction constants (host, little-endian 32-bit limbs)
// ---------------------------------------------------------------------------
namespace {

using Big = std::vector<uint32_t>;

void trim(Big& a) {
  while (a.size() > 1 && a.back() == 0) a.pop_back();
}
Big mul_small(const Big& a, uint32_t m) {
  Big r(a.size() + 1, 0);
  uint64_t carry = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    const uint64_t v = (uint64_t)a[i] * m + carry;
    r[i] = (uint32_t)v;
    carry = v >> 32;
  }
  r[a.size()] = (uint32_t)carry;
  trim(r);
  return r;
}
Big div_small(const Big& a, uint32_t d) {
  Big r(a.size(), 0);
  uint64_t rem = 0;
  for (size_t i = a.size(); i-- > 0;) {
    const uint64_t cur = (rem << 32) | a[i];
    r[i] = (uint32_t)(cur / d);
    rem = cur % d;
  }
  trim(r);
  return r;
}
uint32_t mod_small(const Big& a, uint32_t d) {
  uint64_t rem = 0;
  for (size_t i = a.size(); i-- > 0;) rem = ((rem << 32) | a[i]) % d;
  return (uint32_t)rem;
}
int cmp(const Big& a, const Big& b) {
  if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
  for (size_t i = a.size(); i-- > 0;)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}
void sub_in(Big& a, const Big& b) {  // a -= b, a >= b
  int64_t borrow = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    int64_t v = (int64_t)a[i] - borrow - (i < b.size() ? (int64_t)b[i] : 0);
    borrow = v < 0;
    if (v < 0) v += (int64_t)1 << 32;
    a[i] = (uint32_t)v;
  }
  trim(a);
}
void shl1(Big& a) {
  uint32_t carry = 0;
  for (uint32_t& x : a) {
    const uint32_t nc = x >> 31;
    x = (x << 1) | carry;
    carry = nc;
  }
  if (carry) a.push_back(carry);
}

Crt make_crt() {
  // the 24 largest pairwise coprime integers up to 256
  static const int mods[kT] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211,
                               199, 197, 193, 191, 181, 179, 173, 167, 163, 157, 151, 149};
  Crt c{};
  Big P{1};
  for (int t = 0; t < kT; ++t) P = mul_small(P, (uint32_t)mods[t]);
  double Pd = 0.0;
  for (size_t i = P.size(); i-- > 0;) Pd = Pd * 4294967296.0 + (double)P[i];
  c.P = Pd;
  for (int t = 0; t < kT; ++t) {
    const uint32_t p = (uint32_t)mods[t];
    c.p[t] = (int)p;
    const Big Mt = div_small(P, p);
    const uint32_t mt = mod_small(Mt, p);
    uint32_t inv = 0;
    for (uint32_t x = 1; x < p; ++x)
      if ((uint64_t)mt * x % p == 1) {
        inv = x;
        break;
      }
    Big e = mul_small(Mt, inv);  // e_t = M_t (M_t^-1 mod p_t) < P
    // F_t = floor(2^256 e_t / P): 256 fraction bits by long division
    unsigned long long F[4] = {0, 0, 0, 0};
    for (int k = 255; k >= 0; --k) {
      shl1(e);
      if (cmp(e, P) >= 0) {
        sub_in(e, P);
        F[k / 64] |= 1ull << (k % 64);
      }
    }
    for (int l = 0; l < 4; ++l) {
      c.F32[t][2 * l] = (unsigned)(F[l] & 0xffffffffu);
      c.F32[t][2 * l + 1] = (unsigned)(F[l] >> 32);
    }
  }
  return c;
}

}  // namespace

const Crt& crt_constants() {
  static const Crt c = make_crt();
  return c;
}

// ---------------------------------------------------------------------------
// scaling exponents and residues
// ---------------------------------------------------------------------------
constexpr int kChunks = 4;     // chunks of a scaled integer (88 bits >= kQ)
constexpr int kChunkBits = 22;  // sum_b chunk_b w_b < 4 (2^22 - 1) 255 < 2^32

// Per-modulus constants, passed by value (uniform across a launch): p, the
// reduction multiplier ceil(2^32 / p) and the chunk weights 2^(22 b) mod p.
struct Mods {
  int p[kT];
  unsigned mg[kT];
  unsigned w[kT][kChunks];
};

Mods mods_of(const Crt& c) {
  Mods m;
  for (int t = 0; t < kT; ++t) {
    const unsigned long long p = (unsigned long long)c.p[t];
    m.p[t] = c.p[t];
    m.mg[t] = (unsigned)((0x100000000ull + p - 1) / p);
    unsigned long long v = 1 % p;
    for (int b = 0; b < kChunks; ++b) {
      m.w[t][b] = (unsigned)v;
      v = (v << kChunkBits) % p;
    }
  }
  return m;
}

__device__ __forceinline__ int scale_exp(double mx) { return mx > 0.0 ? kQ - 1 - ilogb(mx) : 0; }


// x mod p for x < 2^32 and p <= 256 (Barrett: the quotient estimate from the
// multiplier ceil(2^32 / p) is exact or one too large).
__device__ __forceinline__ unsigned bmod(unsigned x, unsigned p, unsigned mg) {
  const int r = (int)(x - __umulhi(x, mg) * p);
  return r < 0 ? (unsigned)(r + (int)p) : (unsigned)r;
}

// alpha[i] from max_k |K[i + k ldk]| (rows of K), one thread per row.
__global__ void exp_rows(const double* K, long long ldk, int n, int* alpha) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double mx = 0.0;
    for (int k = 0; k < n; ++k) mx = fmax(mx, fabs(K[i + (long long)k * ldk]));
    alpha[i] = scale_exp(mx);
  }
}

// trunc(|x| 2^sc) (< 2^88) as four 22-bit chunks; false for x = 0.
__device__ __forceinline__ bool chunks_scaled(double x, int sc, unsigned (&ch)[kChunks]) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
  if (bits == 0) {
#pragma unroll
    for (int b = 0; b < kChunks; ++b) ch[b] = 0;
    return false;
  }
  const int eb = (int)(bits >> 52);
  const unsigned long long mant = eb ? ((bits & 0xfffffffffffffull) | (1ull << 52)) : bits;
  const int sh = (eb ? eb : 1) - 1075 + sc;  // |x| 2^sc = mant 2^sh
  unsigned long long lo, hi;                 // the 128-bit integer trunc(mant 2^sh)
  if (sh >= 0) {
    lo = sh < 64 ? mant << sh : 0ull;
    hi = sh == 0 ? 0ull : (sh < 64 ? mant >> (64 - sh) : mant << (sh - 64));
  } else {
    lo = sh > -64 ? mant >> -sh : 0ull;
    hi = 0ull;
  }
  const unsigned m22 = (1u << kChunkBits) - 1;
  ch[0] = (unsigned)lo & m22;
  ch[1] = (unsigned)(lo >> 22) & m22;
  ch[2] = (unsigned)((lo >> 44) | (hi << 20)) & m22;
  ch[3] = (unsigned)(hi >> 2) & m22;
  return true;
}

// Residue in [0, p_t) of the chunked integer, negated modulo p_t for x < 0:
// sum_b ch_b (2^(22 b) mod p) < 4 (2^22 - 1) 255 < 2^32; one Barrett reduction.
__device__ __forceinline__ unsigned residue_chunks(const unsigned (&ch)[kChunks], bool neg, const Mods& m, int t) {
  unsigned s = 0;
#pragma unroll
  for (int b = 0; b < kChunks; ++b) s += ch[b] * m.w[t][b];
  const unsigned p = (unsigned)m.p[t];
  const unsigned r = bmod(s, p, m.mg[t]);
  return (neg && r) ? p - r : r;
}

// Row r of the operand is column r of src (A(r, k) = src[k + r ld]): one
// block per row finds the row's largest magnitude, stores its exponent
// ex[r] (r < rows), then writes out[t][r][k] for k < Kpad (zero outside rows
// x Kd), each thread 4 consecutive k as one 32-bit word per modulus.
__global__ void __launch_bounds__(256) res_cols(const double* __restrict__ src, long long ld, int Kd, int rows,
                                                int* __restrict__ ex, int Kpad, int rows_pad, Mods m,
                                                int8_t* __restrict__ out) {
  __shared__ double red[256 / 32];
  const int r = blockIdx.x;
  const double* col = src + (long long)r * ld;
  double mx = 0.0;
  if (r < rows)
    for (int k = threadIdx.x; k < Kd; k += blockDim.x) mx = fmax(mx, fabs(col[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  mx = red[0];
#pragma unroll
  for (int w = 1; w < 256 / 32; ++w) mx = fmax(mx, red[w]);
  const int sc = scale_exp(mx);
  if (threadIdx.x == 0 && r < rows) ex[r] = sc;
  const size_t plane4 = (size_t)rows_pad * Kpad / 4;
  for (int k0 = 4 * threadIdx.x; k0 < Kpad; k0 += 4 * blockDim.x) {
    unsigned ch[4][kChunks];
    bool ng[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = k0 + q;
      const double x = (r < rows && k < Kd) ? col[k] : 0.0;
      chunks_scaled(x, sc, ch[q]);
      ng[q] = x < 0.0;
    }
    unsigned* o = reinterpret_cast<unsigned*>(out + (size_t)r * Kpad + k0);
#pragma unroll
    for (int t = 0; t < kT; ++t) {
      unsigned w = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) w |= residue_chunks(ch[q], ng[q], m, t) << (8 * q);
      o[t * plane4] = w;
    }
  }
}

// Row i of the operand is row i of K (A(i, k) = K[i + k ldk]): 32 x 32 tiles
// transposed through shared memory, out[t][i][k].
__global__ void res_rows(const double* K, long long ldk, int n, const int* alpha, int Kpad, int Mpad, Mods m,
                         int8_t* out) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + threadIdx.x, k = k0 + r;
    tile[r][threadIdx.x] = (i < n && k < n) ? K[i + (long long)k * ldk] : 0.0;
  }
  __syncthreads();
  const size_t plane = (size_t)Mpad * Kpad;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, k = k0 + threadIdx.x;
    if (i < Mpad && k < Kpad) {
      const double x = tile[threadIdx.x][r];
      unsigned ch[kChunks];
      chunks_scaled(x, i < n ? alpha[i] : 0, ch);
      int8_t* o = out + (size_t)i * Kpad + k;
#pragma unroll 4
      for (int t = 0; t < kT; ++t) o[t * plane] = (int8_t)residue_chunks(ch, x < 0.0, m, t);
    }
  }
}

// ---------------------------------------------------------------------------
// the tcgen05 INT8 GEMM
// ---------------------------------------------------------------------------
constexpr int kStages = 6;
constexpr int kCtaM = 2 * kTileM;      // two M = 128 accumulators per CTA: 256 rows
constexpr int kAStage = kCtaM * kBk;   // 16 KB
constexpr int kBStage = 256 * kBk;     // room for ntile <= 256: 16 KB
constexpr size_t kGemmSmem = 1024 + (size_t)kStages * (kAStage + kBStage) + 256;  // + barriers and the TMEM slot

struct I8Args {
  int Mpad, Wpad, Kpad, ntile, nk;
  int sgn;        // 1: signed int8 operands (self-check), 0: unsigned residues
  uint8_t* cres;  // residue planes [T][Wpad][Mpad]
  int* raw;       // RAW: the int32 product [Wpad][Mpad]
  unsigned* err;
  Mods m;
};

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile in the 64-byte swizzle
// layout (rows of 64 bytes, eight-row atoms of 512 bytes): start address
// >> 4, leading byte offset 16 (unused by this layout), stride byte offset
// 512 (eight 64-byte rows), descriptor version 1, base offset 0 (tiles are
// 1024-byte aligned), layout type 4 (64B).
__device__ __forceinline__ uint64_t sw64_desc(const void* p) {
  const uint32_t a = smem_u32(p);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)(16 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

// Instruction descriptor of kind::i8: int32 accumulator, A and B signed
// (sgn = 1) or unsigned (sgn = 0) 8-bit, both K-major, N = n, M = 128.
__host__ __device__ constexpr uint32_t i8_idesc(int n, int sgn) {
  return (2u << 4) | ((uint32_t)sgn << 7) | ((uint32_t)sgn << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_local(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Persistent: one CTA per SM walks the tiles blockIdx.x, + gridDim.x, ...
// (column tiles fastest, then row tiles, then residue planes).  A tile is MT
// x ntile of the output, accumulated in tensor memory as MT / 128 row halves
// of 128 lanes; MT = 256 holds one tile in the 512 columns (half h at column
// 256 h), MT = 128 holds two (buffer b at column 256 b), so that the MMAs of
// the next tile run while the epilogue drains the last one.  Warp 0 (one
// thread) issues the copies, warp 1 (one thread) the MMAs, warps 2..9 read
// the accumulators back (warp w reaches tensor-memory lanes 32 (w % 4) ..
// +31).  The copy ring runs on across tiles (a global k-block count keeps its
// barrier phases); tfull[b] / tempty[b] hand accumulator buffer b between
// the MMA thread and the epilogue warps.
constexpr int kEpiWarps = 8;
constexpr int kPersistThreads = 64 + 32 * kEpiWarps;

template <bool RAW, int MT>
__global__ void __launch_bounds__(kPersistThreads, 1) i8_gemm(const __grid_constant__ CUtensorMap ta,
                                                              const __grid_constant__ CUtensorMap tb, I8Args g,
                                                              int ntn, int ntm, int planes) {
  constexpr int kHalves = MT / kTileM;
  constexpr int kBufs = 2 / kHalves;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = base;
  uint8_t* sB = base + (size_t)kStages * kAStage;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + (size_t)kStages * kBStage);
  uint64_t* empty = full + kStages;
  uint64_t* tfull = empty + kStages;  // [kBufs]
  uint64_t* tempty = tfull + 2;       // [kBufs]
  uint64_t* fin = tempty + 2;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr uint32_t ncols = 512;
  const int tiles = ntn * ntm * planes;
  const uint32_t stage_bytes = (uint32_t)(MT * kBk + g.ntile * kBk);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(tfull + b, 1);
      mbar_init(tempty + b, kEpiWarps);
    }
    mbar_init(fin, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if (warp == 0) {
    if (lane == 0) {  // copies
      long long kbg = 0;
      bool ok = true;
      for (int tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x) {
        const int n0 = (tile % ntn) * g.ntile, m0 = ((tile / ntn) % ntm) * MT, z = tile / (ntn * ntm);
        for (int kb = 0; kb < g.nk; ++kb, ++kbg) {
          const int s = (int)(kbg % kStages);
          if (kbg >= kStages && !mbar_wait_bounded(empty + s, (unsigned)((kbg / kStages) - 1) & 1)) {
            atomicOr(g.err, KERR_MBAR_TIMEOUT);
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(full + s, stage_bytes);
          tma_load_3d(sA + (size_t)s * kAStage, &ta, kb * kBk, m0, z, full + s);
          tma_load_3d(sB + (size_t)s * kBStage, &tb, kb * kBk, n0, z, full + s);
        }
      }
      // the copies of the last use of each stage land before the CTA leaves
      for (long long u = std::max(0LL, kbg - kStages); u < kbg; ++u)
        if (!mbar_wait_bounded(full + u % kStages, (unsigned)(u / kStages) & 1)) atomicOr(g.err, KERR_MBAR_TIMEOUT);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMAs
      const uint32_t idesc = i8_idesc(g.ntile, g.sgn);
      long long kbg = 0;
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x, ++it) {
        const int b = it % kBufs, use = it / kBufs;
        if (use > 0 && !mbar_wait_bounded(tempty + b, (unsigned)(use - 1) & 1)) {  // buffer b drained
          atomicOr(g.err, KERR_MBAR_TIMEOUT);
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(256 * b);
        for (int kb = 0; kb < g.nk; ++kb, ++kbg) {
          const int s = (int)(kbg % kStages);
          if (!mbar_wait_bounded(full + s, (unsigned)(kbg / kStages) & 1)) {
            atomicOr(g.err, KERR_MBAR_TIMEOUT);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint8_t* a = sA + (size_t)s * kAStage;
          const uint8_t* bb = sB + (size_t)s * kBStage;
#pragma unroll
          for (int h = 0; h < kHalves; ++h)
#pragma unroll
            for (int kk = 0; kk < kBk / 32; ++kk)
              tc_mma(acc + (uint32_t)(256 * h), sw64_desc(a + h * (kTileM * kBk) + kk * 32), sw64_desc(bb + kk * 32),
                     idesc, (kb | kk) != 0);
          tc_commit(empty + s);  // the stage is free once these MMAs have read it
        }
        if (ok) tc_commit(tfull + b);  // this tile's accumulators are complete
      }
      // every MMA issued has completed before the tensor memory is freed
      tc_commit(fin);
      if (!mbar_wait_bounded(fin, 0)) atomicOr(g.err, KERR_MBAR_TIMEOUT);
    }
  } else {  // epilogue warps
    const int ew = warp - 2, lq = warp & 3;
    const int h = kHalves == 2 ? ew >> 2 : 0;
    const int cfirst = kHalves == 2 ? 0 : (ew >> 2) * 32, cstep = kHalves == 2 ? 32 : 64;
    int it = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++it) {
      const int n0 = (tile % ntn) * g.ntile, m0 = ((tile / ntn) % ntm) * MT, z = tile / (ntn * ntm);
      const int b = it % kBufs;
      const unsigned par = (unsigned)(it / kBufs) & 1;
      bool have = mbar_try_wait(tfull + b, par);
      if (!have) {
        const unsigned long long t0 = globaltimer_ns();
        while (!(have = mbar_try_wait(tfull + b, par)) && globaltimer_ns() - t0 <= kWaitLimitNs) __nanosleep(100);
      }
      if (!have) {
        if (lane == 0) atomicOr(g.err, KERR_MBAR_TIMEOUT);
        break;
      }
      tc_fence_after();
      const int i = m0 + h * kTileM + lq * 32 + lane;  // output row
      const unsigned p = RAW ? 1u : (unsigned)g.m.p[z];
      const unsigned mg = RAW ? 1u : g.m.mg[z];
      const uint32_t acc = tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(256 * (b + h));
      for (int c = cfirst; c < g.ntile; c += cstep) {
        uint32_t v[32];
        tc_ld32(acc + (uint32_t)c, v);
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          if (c + q >= g.ntile) break;  // columns of the last load beyond the tile
          const int j = n0 + c + q;
          const int d = (int)v[q];
          if (RAW) {
            g.raw[(size_t)j * g.Mpad + i] = d;
          } else {  // 0 <= d < Kpad 255^2 < 2^31: one Barrett step in integer arithmetic
            g.cres[((size_t)z * g.Wpad + j) * g.Mpad + i] = (uint8_t)bmod((unsigned)d, p, mg);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_local(tempty + b);  // this warp is done with buffer b
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    (void)cudaGetLastError();
  }
  return fn;
}

// 3-D map over int8 planes [planes][rows][Kpad], boxes of kBk bytes x box_rows x 1
// in the 64-byte swizzle layout.
int make_map(CUtensorMap* map, const void* base, int Kpad, int rows, int planes, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return set_error(RWIG_E_UNSUPPORTED, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[3] = {(cuuint64_t)Kpad, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)Kpad, (cuuint64_t)Kpad * (cuuint64_t)rows};
  const cuuint32_t box[3] = {(cuuint32_t)kBk, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(RWIG_E_CUDA, "cuTensorMapEncodeTiled failed");
  return 0;
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }
int pick_ntile(int W) { return std::min(256, round_up(std::max(W, 16), 16)); }

enum { SO_ARES0 = 400, SO_ARES1, SO_ALPHA0, SO_ALPHA1, SO_ERR, SO_TA, SO_TB, SO_TD, SO_KKEEP, SO_KDIFF };
// per-lane scratch of the product pipeline: lanes are products in flight on
// different streams at once
enum { SO_LANE = 420, SO_BRES = 0, SO_BETA, SO_CRES, SO_PER_LANE = 3 };
int lane_slot(int lane, int k) { return SO_LANE + SO_PER_LANE * lane + k; }

// The kT (or, RAW, one) planes of A (Mpad x Kpad) and B (Wpad x Kpad): the
// int8 products into cres (or raw).
template <bool RAW>
int launch_i8(Context* ctx, const int8_t* A, int Mpad, const int8_t* B, int Wpad, int Kpad, int ntile, int planes,
              uint8_t* cres, int* raw, cudaStream_t st) {
  CUtensorMap ta, tb;
  unsigned* err = (unsigned*)scratch(ctx, SO_ERR, sizeof(unsigned) * 4);  // cleared by reset_err()
  if (!err) return RWIG_E_NOMEM;
  I8Args g{};
  g.Mpad = Mpad;
  g.Wpad = Wpad;
  g.Kpad = Kpad;
  g.ntile = ntile;
  g.nk = Kpad / kBk;
  g.sgn = RAW ? 1 : 0;
  g.cres = cres;
  g.raw = raw;
  g.err = err;
  g.m = mods_of(crt_constants());
  // 256-row tiles (one accumulator) by default: measured faster than 128-row
  // tiles with two accumulators on the 5000 x 1024 products; option "oz.tile_m".
  const int tm_opt = (int)option("oz.tile_m", 0.0);
  const int MT = tm_opt == 128 || tm_opt == 256 ? tm_opt : 256;
  if (int rc = make_map(&ta, A, Kpad, Mpad, planes, MT)) return rc;
  if (int rc = make_map(&tb, B, Kpad, Wpad, planes, ntile)) return rc;
  static bool attr[2] = {false, false};
  const int ntn = Wpad / ntile, ntm = Mpad / MT, tiles = ntn * ntm * planes;
  const int grid = std::min(tiles, ctx->sm_count);  // persistent: one CTA per SM
  const bool timed = gemm_timer_mark(ctx, st);
  if (MT == 256) {
    if (!attr[0]) {
      RWIG_CUDA_TRY(cudaFuncSetAttribute(i8_gemm<RAW, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
      attr[0] = true;
    }
    i8_gemm<RAW, 256><<<grid, kPersistThreads, kGemmSmem, st>>>(ta, tb, g, ntn, ntm, planes);
  } else {
    if (!attr[1]) {
      RWIG_CUDA_TRY(cudaFuncSetAttribute(i8_gemm<RAW, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
      attr[1] = true;
    }
    i8_gemm<RAW, 128><<<grid, kPersistThreads, kGemmSmem, st>>>(ta, tb, g, ntn, ntm, planes);
  }
  RWIG_CUDA_TRY(cudaGetLastError());
  if (timed) gemm_timer_mark(ctx, st);
  return 0;
}

// Clears the error word that the GEMMs of a sequence (prepare() .. status())
// accumulate their bounded-wait failures into.
int reset_err(Context* ctx, cudaStream_t st) {
  unsigned* err = (unsigned*)scratch(ctx, SO_ERR, sizeof(unsigned) * 4);
  if (!err) return RWIG_E_NOMEM;
  RWIG_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned), st));
  return 0;
}

int check_err(Context* ctx, cudaStream_t st) {
  unsigned h = 0;
  unsigned* err = (unsigned*)scratch(ctx, SO_ERR, sizeof(unsigned) * 4);
  RWIG_CUDA_TRY(cudaMemcpyAsync(&h, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  if (h) return set_error(RWIG_E_TIMEOUT, "INT8 tensor-core GEMM: a bounded wait ran out");
  return 0;
}

}  // namespace

bool available(Context* ctx) { return ctx && ctx->smem_optin >= (int)kGemmSmem && encode_fn() != nullptr; }

// Counts the positions where a and b differ bitwise (n doubles), into *diff.
__global__ void count_diff(const unsigned long long* __restrict__ a, const unsigned long long* __restrict__ b,
                           long long n, unsigned* diff) {
  unsigned d = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d |= (unsigned)(__ldcs(a + i) != __ldcs(b + i));
  if (__syncthreads_or(d) && threadIdx.x == 0) atomicOr(diff, 1u);
}

int prepare(Context* ctx, const double* K, long long ldk, int n, Prepared* pr, cudaStream_t st, int* launches) {
  ctx->oz_kept = false;  // the residue planes are about to hold another K
  if (n < 1 || n > kMaxKd) return set_error(RWIG_E_UNSUPPORTED, "INT8 product path: size above 8192");
  if (!available(ctx)) return set_error(RWIG_E_UNSUPPORTED, "INT8 product path unavailable on this device");
  pr->K = K;
  pr->ldk = ldk;
  pr->Mo = pr->Kd = n;
  pr->Mpad = round_up(n, kCtaM);
  pr->Kpad = round_up(n, kKpadTo);
  const size_t planes = (size_t)kT * pr->Mpad * pr->Kpad;
  const Mods m = mods_of(crt_constants());
  if (int rc = reset_err(ctx, st)) return rc;
  for (int tr = 0; tr < 2; ++tr) {
    pr->ares[tr] = (int8_t*)scratch(ctx, SO_ARES0 + tr, planes);
    pr->alpha[tr] = (int*)scratch(ctx, SO_ALPHA0 + tr, sizeof(int) * n);
    if (!pr->ares[tr] || !pr->alpha[tr]) return RWIG_E_NOMEM;
  }
  // trans = 0: rows of K
  exp_rows<<<std::max(1, (n + 255) / 256), 256, 0, st>>>(K, ldk, n, pr->alpha[0]);
  res_rows<<<dim3(pr->Kpad / 32, pr->Mpad / 32), dim3(32, 8), 0, st>>>(K, ldk, n, pr->alpha[0], pr->Kpad, pr->Mpad, m,
                                                                        pr->ares[0]);
  // trans = 1: columns of K
  res_cols<<<pr->Mpad, 256, 0, st>>>(K, ldk, n, n, pr->alpha[1], pr->Kpad, pr->Mpad, m, pr->ares[1]);
  if (launches) *launches += 3;
  RWIG_CUDA_TRY(cudaGetLastError());
  return 0;
}

int prepare_reuse(Context* ctx, const double* K, long long ldk, int n, Prepared* pr, cudaStream_t st, int* launches) {
  if (n < 1 || n > kMaxKd) return set_error(RWIG_E_UNSUPPORTED, "INT8 product path: size above 8192");
  const long long len = ldk * (long long)n;
  double* keep = (double*)scratch(ctx, SO_KKEEP, sizeof(double) * (size_t)len);
  unsigned* diff = (unsigned*)scratch(ctx, SO_KDIFF, sizeof(unsigned) * 4);
  if (!keep || !diff) return RWIG_E_NOMEM;
  if (ctx->oz_kept && ctx->oz_kept_n == n && ctx->oz_kept_ldk == ldk) {
    RWIG_CUDA_TRY(cudaMemsetAsync(diff, 0, sizeof(unsigned), st));
    const int grid = (int)std::max<long long>(1, std::min<long long>((len + 255) / 256, 4LL * ctx->sm_count));
    count_diff<<<grid, 256, 0, st>>>(reinterpret_cast<const unsigned long long*>(K),
                                     reinterpret_cast<const unsigned long long*>(keep), len, diff);
    RWIG_CUDA_TRY(cudaGetLastError());
    if (launches) ++*launches;
    unsigned h = 1;
    RWIG_CUDA_TRY(cudaMemcpyAsync(&h, diff, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    RWIG_CUDA_TRY(cudaStreamSynchronize(st));
    if (h == 0) {  // the same K, bit for bit: its residue planes are still in the scratch
      pr->K = K;
      pr->ldk = ldk;
      pr->Mo = pr->Kd = n;
      pr->Mpad = round_up(n, kCtaM);
      pr->Kpad = round_up(n, kKpadTo);
      const size_t planes = (size_t)kT * pr->Mpad * pr->Kpad;
      for (int tr = 0; tr < 2; ++tr) {
        pr->ares[tr] = (int8_t*)scratch(ctx, SO_ARES0 + tr, planes);
        pr->alpha[tr] = (int*)scratch(ctx, SO_ALPHA0 + tr, sizeof(int) * n);
        if (!pr->ares[tr] || !pr->alpha[tr]) return RWIG_E_NOMEM;
      }
      return reset_err(ctx, st);
    }
  }
  if (int rc = prepare(ctx, K, ldk, n, pr, st, launches)) return rc;
  RWIG_CUDA_TRY(cudaMemcpyAsync(keep, K, sizeof(double) * (size_t)len, cudaMemcpyDeviceToDevice, st));
  ctx->oz_kept = true;
  ctx->oz_kept_n = n;
  ctx->oz_kept_ldk = ldk;
  return 0;
}

int products(Context* ctx, const Prepared& pr, int trans, const double* X, long long ldx, int W, cudaStream_t st,
             const uint8_t** cres, const int** beta, int* Wpad_out, int* launches, int lane) {
  if (W < 1 || !X) return set_error(RWIG_E_INVALID, "INT8 product path: empty operand");
  const int ntile = pick_ntile(W);
  const int Wpad = round_up(W, ntile);
  int8_t* bres = (int8_t*)scratch(ctx, lane_slot(lane, SO_BRES), (size_t)kT * Wpad * pr.Kpad);
  int* be = (int*)scratch(ctx, lane_slot(lane, SO_BETA), sizeof(int) * W);
  uint8_t* cr = (uint8_t*)scratch(ctx, lane_slot(lane, SO_CRES), (size_t)kT * Wpad * pr.Mpad);
  if (!bres || !be || !cr) return RWIG_E_NOMEM;
  const Mods m = mods_of(crt_constants());
  res_cols<<<Wpad, 256, 0, st>>>(X, ldx, pr.Kd, W, be, pr.Kpad, Wpad, m, bres);
  if (int rc = launch_i8<false>(ctx, pr.ares[trans], pr.Mpad, bres, Wpad, pr.Kpad, ntile, kT, cr, nullptr, st)) return rc;
  if (launches) *launches += 2;
  *cres = cr;
  *beta = be;
  *Wpad_out = Wpad;
  return 0;
}

// Bounded-wait status of the last products() launches (a host read).
int status(Context* ctx, cudaStream_t st) { return check_err(ctx, st); }

}  // namespace oz
}  // namespace rwig

using namespace rwig;

// Self-check of the INT8 tensor-core GEMM (no counterpart in the reference):
// D (M x N, column-major, int32) = A B^T for A (M x Kd) and B (N x Kd) int8,
// both row-major (K-major); all device pointers.
extern "C" int rwig_selftest_i8gemm(const signed char* A, const signed char* B, int M, int N, int Kd, int* D,
                                    void* stream) {
  if (!A || !B || !D || M < 1 || N < 1 || Kd < 1 || Kd > (1 << 16))
    return set_error(RWIG_E_INVALID, "bad INT8 GEMM arguments");
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!oz::available(ctx)) return set_error(RWIG_E_UNSUPPORTED, "INT8 tensor-core GEMM unavailable");
  cudaStream_t st = call_stream(ctx, stream);
  const int ntile = oz::pick_ntile(N), Mpad = oz::round_up(M, oz::kCtaM), Npad = oz::round_up(N, ntile);
  const int Kpad = oz::round_up(Kd, oz::kKpadTo);
  int8_t* a = (int8_t*)scratch(ctx, oz::SO_TA, (size_t)Mpad * Kpad);
  int8_t* b = (int8_t*)scratch(ctx, oz::SO_TB, (size_t)Npad * Kpad);
  int* d = (int*)scratch(ctx, oz::SO_TD, sizeof(int) * (size_t)Mpad * Npad);
  if (!a || !b || !d) return RWIG_E_NOMEM;
  RWIG_CUDA_TRY(cudaMemsetAsync(a, 0, (size_t)Mpad * Kpad, st));
  RWIG_CUDA_TRY(cudaMemsetAsync(b, 0, (size_t)Npad * Kpad, st));
  RWIG_CUDA_TRY(cudaMemcpy2DAsync(a, Kpad, A, Kd, Kd, M, cudaMemcpyDeviceToDevice, st));
  RWIG_CUDA_TRY(cudaMemcpy2DAsync(b, Kpad, B, Kd, Kd, N, cudaMemcpyDeviceToDevice, st));
  if (int rc = oz::reset_err(ctx, st)) return rc;
  if (int rc = oz::launch_i8<true>(ctx, a, Mpad, b, Npad, Kpad, ntile, 1, nullptr, d, st)) return rc;
  RWIG_CUDA_TRY(cudaMemcpy2DAsync(D, sizeof(int) * M, d, sizeof(int) * Mpad, sizeof(int) * M, N,
                                  cudaMemcpyDeviceToDevice, st));
  return oz::check_err(ctx, st);
}

// Self-check of the emulated FP64 product (no counterpart in the reference):
// Y (n x W, ldy) = op(K) X, op(K) = K (trans = 0) or K^T (trans = 1), K
// n x n (ldk), X n x W (ldx); all device pointers.
extern "C" int rwig_selftest_ozaki(const double* K, long long ldk, int trans, int n, const double* X, long long ldx,
                                   int W, double* Y, long long ldy, void* stream) {
  if (!K || !X || !Y || n < 1 || W < 1 || (trans != 0 && trans != 1) || ldk < n || ldx < n || ldy < n)
    return set_error(RWIG_E_INVALID, "bad emulated-product arguments");
  Context* ctx = get_context();
  if (!ctx) return RWIG_E_NODEVICE;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t st = call_stream(ctx, stream);
  oz::Prepared pr;
  int launches = 0;
  reset_report();
  if (int rc = gemm_timer_begin(ctx)) return rc;
  if (int rc = oz::prepare(ctx, K, ldk, n, &pr, st, &launches)) return rc;
  if (int rc = oz::gemm(ctx, pr, trans, X, ldx, W, oz::kCrtCols, dg::EpiStore{Y, ldy, W}, st, &launches)) return rc;
  const int rc = oz::status(ctx, st);
  gemm_timer_end(ctx, &report().gemm_ms, &report().gemm_launches);
  report().kernel_launches = launches;
  return rc;
}
