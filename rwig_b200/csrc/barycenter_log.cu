// barycenter_log.cu -- the log barycenter in the log domain: the reference's
// own updates (Barycenter::_fwd_log, src/barycenter_impl_log.cpp:189-272, and
// _bwd_log, :275-382) with no Gibbs kernel K anywhere, for the regimes where
// the scaling form of barycenter.cu would leave the range of doubles (max
// C / eps above ~700, or scalings beyond 1e+-290).  barycenter.cu runs the
// scaling form first and hands the problem here when its range certificate
// fails (or always, with the option "barycenter.log_path" = 1).
//
// Every sweep is a soft-min over one axis of C minus a potential,
//   column pass  m_js = softmin_i (C_ij - F_is),   row pass  r_is = softmin_j (C_ij - G_js),
// softmin_k(x_k) = -eps log sum_k exp(-x_k / eps), evaluated with the running
// maximum of each tile as the shift (one exponential per element).  With
// R_s = C - F_s 1^T - 1 G_s^T one forward iteration l is
//   F_l      = F_{l-1} + (eps log A + KV_{l-1}),   KV_{l-1} = r_{l-1} - F_{l-1}   (:231)
//   m_l      = column pass over C - F_l,   KTU = m_l - G_{l-1}                   (:238)
//   logb_l   = -(sum_s w_s m_l,s) / eps,   G_l = eps logb_l + m_l                (:239, :245)
//   r_l      = row pass over C - G_l,      KV_l = r_l - F_l                      (:251)
//   err      = || -KV_l / eps - log A ||_2 (spectral norm, :252)
// and the adjoint step l reads the row- and column-softmax weights of the
// reference (:306-346) with their normalisers from the forward:
//   X_ij = exp((r_l,is + G_l,js - C_ij) / eps)    (row softmax at F_l, G_l)
//   W_ij = exp((m_l,js + F_l,is - C_ij) / eps)    (column softmax at F_l, G_{l-1})
//   Gbar_js = -sum_i X_ij Fbar_is,  logbbar_j = eps sum_s Gbar_js  (l < L)
//   y_js = (w_s / eps) logbbar_j - Gbar_js,  Fbar_is = sum_j W_ij y_js
//   grad_A += Fbar / A,  grad_w -= m_l^T logbbar,  then grad_A *= eps, grad_w /= eps.
// The histories F_l, G_l, m_l, r_l (l = 0..L) stay on the device.
//
// Pass kernel: a CTA owns 64 outputs x 16 histograms and one slice of the
// reduction axis; the 32 x 64 tile of C and the 32 x 16 tile of the
// potential sit in shared memory, each thread holds 2 x 2 outputs (4
// exponentials per 4 shared loads).  Partial (max, sum) pairs per slice are
// merged in a fixed order by the merge kernels, which also carry the
// elementwise updates above: results are bitwise repeatable.  The
// exponential is the table method of fastexp.cuh; it is FP64-pipe bound.
#include <algorithm>
#include <cmath>
#include <vector>

#include "barycenter.h"
#include "dgemm.cuh"
#include "engine.h"
#include "fastexp.cuh"

namespace rwig {
namespace barylog {

constexpr int TK = 32;   // reduction rows per shared tile
constexpr int TO = 64;   // outputs per CTA
constexpr int TS = 16;   // histograms per CTA
constexpr int NT = 256;  // 32 output groups x 8 histogram pairs

// One pass: for outputs o < O, histograms s < S and k in this CTA's slice,
//   forward  (WEIGHTED = false): max_k x and sum_k exp(x - max), x = (P_ks - C(k,o)) / eps;
//   weighted (WEIGHTED = true):  sum_k exp((P_ks + Q_os - C(k,o)) / eps) Y_ks,
// with C(k,o) = C_ko (column pass, k a row of C) or C_ok (row pass, ROWS).
// P = P1 + p2c P2 (P2 null, or ldp2 = 0 to add a K-vector to every column).
struct Pass {
  const double* C;
  long long ldc;
  int K, O, S;
  const double* P1;
  long long ldp1;
  const double* P2;
  long long ldp2;
  double p2c;
  const double* Q;  // O x S (weighted)
  long long ldq;
  const double* Y;  // K x S (weighted)
  long long ldy;
  double inv_eps;
  int kchunk;    // reduction rows per slice (a multiple of TK)
  double* pmax;  // [slices][S][O] (forward)
  double* psum;  // [slices][S][O]
};

// exp(x) by the table method, exactly 0 below -708 (where the table method
// returns its clamp value exp(-708)).
__device__ __forceinline__ double expz(double x, const double* tbl) {
  const double e = exp_tbl<kExpTableSpread>(x, tbl);
  return x < -708.0 ? 0.0 : e;
}

template <bool ROWS, bool WEIGHTED>
__global__ void __launch_bounds__(NT) pass_kernel(Pass a) {
  constexpr int LD = ROWS ? (TO + 2) : (TK + 1);  // shared C tile: ROWS [k][o], else [o][k]
  __shared__ double ct[ROWS ? TK * (TO + 2) : TO * (TK + 1)];
  __shared__ double pt[TS * TK];
  __shared__ double yt[WEIGHTED ? TS * TK : 1];
  __shared__ double tbl_all[64 * kExpTableSpread];
  const int tid = threadIdx.x, og = tid & 31, sg = tid >> 5;
  const int o0 = blockIdx.x * TO, s0 = blockIdx.y * TS;
  const int kb = blockIdx.z * a.kchunk, ke = min(a.K, kb + a.kchunk);
  load_exp_table_spread(tbl_all);
  const double* tbl = tbl_all + (tid & (kExpTableSpread - 1));
  const double ie = a.inv_eps;
  const int oo[2] = {og, og + 32};
  const int ss[2] = {2 * sg, 2 * sg + 1};
  double mx[2][2], sm[2][2], qv[2][2];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      mx[p][q] = -INFINITY;
      sm[p][q] = 0.0;
      qv[p][q] = 0.0;
      if (WEIGHTED && o0 + oo[p] < a.O && s0 + ss[q] < a.S)
        qv[p][q] = a.Q[(long long)(o0 + oo[p]) + (long long)(s0 + ss[q]) * a.ldq] * ie;
    }
  for (int kt = kb; kt < ke; kt += TK) {
    const int nk = min(TK, ke - kt);
    __syncthreads();  // the previous tile is consumed (and the table loaded)
    if (ROWS) {
      for (int e = tid; e < TK * TO; e += NT) {
        const int kk = e / TO, o = e % TO;
        ct[kk * LD + o] = (kk < nk && o0 + o < a.O) ? a.C[(long long)(o0 + o) + (long long)(kt + kk) * a.ldc] : 0.0;
      }
    } else {
      for (int e = tid; e < TK * TO; e += NT) {
        const int o = e / TK, kk = e % TK;
        ct[o * LD + kk] = (kk < nk && o0 + o < a.O) ? a.C[(long long)(kt + kk) + (long long)(o0 + o) * a.ldc] : 0.0;
      }
    }
    for (int e = tid; e < TS * TK; e += NT) {
      const int s = e / TK, kk = e % TK;
      double v = 0.0, y = 0.0;
      if (kk < nk && s0 + s < a.S) {
        const long long k = kt + kk;
        v = a.P1[k + (long long)(s0 + s) * a.ldp1];
        if (a.P2) v += a.p2c * a.P2[k + (long long)(s0 + s) * a.ldp2];
        if (WEIGHTED) y = a.Y[k + (long long)(s0 + s) * a.ldy];
      }
      pt[s * TK + kk] = v;
      if (WEIGHTED) yt[s * TK + kk] = y;
    }
    __syncthreads();
    const double* c0p = ROWS ? ct + oo[0] : ct + oo[0] * LD;
    const double* c1p = ROWS ? ct + oo[1] : ct + oo[1] * LD;
    constexpr int CK = ROWS ? LD : 1;  // stride of k in the C tile
    const double* p0p = pt + ss[0] * TK;
    const double* p1p = pt + ss[1] * TK;
    if (!WEIGHTED) {
      double tm[2][2] = {{-INFINITY, -INFINITY}, {-INFINITY, -INFINITY}};
      for (int kk = 0; kk < nk; ++kk) {
        const double c0 = c0p[kk * CK], c1 = c1p[kk * CK], p0 = p0p[kk], p1 = p1p[kk];
        tm[0][0] = fmax(tm[0][0], (p0 - c0) * ie);
        tm[0][1] = fmax(tm[0][1], (p1 - c0) * ie);
        tm[1][0] = fmax(tm[1][0], (p0 - c1) * ie);
        tm[1][1] = fmax(tm[1][1], (p1 - c1) * ie);
      }
#pragma unroll
      for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          if (tm[p][q] > mx[p][q]) {
            sm[p][q] *= expz(mx[p][q] - tm[p][q], tbl);
            mx[p][q] = tm[p][q];
          }
      for (int kk = 0; kk < nk; ++kk) {
        const double c0 = c0p[kk * CK], c1 = c1p[kk * CK], p0 = p0p[kk], p1 = p1p[kk];
        sm[0][0] += expz((p0 - c0) * ie - mx[0][0], tbl);
        sm[0][1] += expz((p1 - c0) * ie - mx[0][1], tbl);
        sm[1][0] += expz((p0 - c1) * ie - mx[1][0], tbl);
        sm[1][1] += expz((p1 - c1) * ie - mx[1][1], tbl);
      }
    } else {
      const double* y0p = yt + ss[0] * TK;
      const double* y1p = yt + ss[1] * TK;
      for (int kk = 0; kk < nk; ++kk) {
        const double c0 = c0p[kk * CK], c1 = c1p[kk * CK], p0 = p0p[kk], p1 = p1p[kk];
        const double y0 = y0p[kk], y1 = y1p[kk];
        sm[0][0] = fma(expz((p0 - c0) * ie + qv[0][0], tbl), y0, sm[0][0]);
        sm[0][1] = fma(expz((p1 - c0) * ie + qv[0][1], tbl), y1, sm[0][1]);
        sm[1][0] = fma(expz((p0 - c1) * ie + qv[1][0], tbl), y0, sm[1][0]);
        sm[1][1] = fma(expz((p1 - c1) * ie + qv[1][1], tbl), y1, sm[1][1]);
      }
    }
  }
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int o = o0 + oo[p], s = s0 + ss[q];
      if (o < a.O && s < a.S) {
        const long long idx = ((long long)blockIdx.z * a.S + s) * a.O + o;
        if (!WEIGHTED) a.pmax[idx] = mx[p][q];
        a.psum[idx] = sm[p][q];
      }
    }
}

// Merged soft-min of output o, histogram s over the slices (fixed order):
// -eps (max + log sum_slices psum exp(pmax - max)).
__device__ __forceinline__ double merged_softmin(const double* pmax, const double* psum, int slices, int S, int O,
                                                 int s, int o, double eps) {
  double mx = -INFINITY;
  for (int z = 0; z < slices; ++z) mx = fmax(mx, pmax[((long long)z * S + s) * O + o]);
  double sum = 0.0;
  for (int z = 0; z < slices; ++z) {
    const long long k = ((long long)z * S + s) * O + o;
    sum += psum[k] * exp(pmax[k] - mx);
  }
  return -eps * (mx + log(sum));
}

// Forward, after the column pass over C - F_l (thread per support point j):
// m_l (into Mh), logb_j = -(sum_s w_s m_js) / eps, G_l = eps logb + m.
__global__ void col_merge_fwd(const double* pmax, const double* psum, int slices, int N, int S, double eps,
                              const double* w, double* M_out, double* G, double* logb) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int s = 0; s < S; ++s) {
      const double m = merged_softmin(pmax, psum, slices, S, N, s, j, eps);
      M_out[j + (long long)s * N] = m;
      acc += m * w[s];
    }
    const double lb = -acc / eps;  // barycenter_impl_log.cpp:239
    logb[j] = lb;
    for (int s = 0; s < S; ++s) G[j + (long long)s * N] = eps * lb + M_out[j + (long long)s * N];  // :245
  }
}

// Forward, after the row pass over C - G (thread per (i, s)): r (into R_out
// when given), KV = r - F, the next F = F + (eps log A + KV) (:231) and, when
// D is given, the stopping residual -KV / eps - log A (:252).
__global__ void row_merge_fwd(const double* pmax, const double* psum, int slices, int M, int S, double eps,
                              const double* F, const double* logA, double* R_out, double* Fnext, double* D,
                              long long ldd) {
  const long long n = (long long)M * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % M), s = (int)(e / M);
    const double r = merged_softmin(pmax, psum, slices, S, M, s, i, eps);
    const double kv = r - F[e];
    if (R_out) R_out[e] = r;
    Fnext[e] = F[e] + (eps * logA[e] + kv);
    if (D) D[i + (long long)s * ldd] = -kv / eps - logA[e];
  }
}

// Adjoint seed and column step (thread per support point j).  seed: logbbar
// = 2 (b - b_ext) o b with the normalised b (:324), Gbar = 0; otherwise
// Gbar_js = -(sum over slices of the weighted pass), logbbar = eps sum_s Gbar.
// Then y = (w / eps) logbbar - Gbar (the right-hand side of the row step) and
// gwp[j S + s] -= m_l,js logbbar_j (:368-372).
__global__ void col_merge_bwd(const double* psum, int slices, int N, int S, double eps, int seed, const double* bn,
                              const double* bext, const double* w, const double* Ml, double* Yv, double* gwp) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    double lbb;
    if (seed) {
      lbb = 2.0 * (bn[j] - bext[j]) * bn[j];
      for (int s = 0; s < S; ++s) Yv[j + (long long)s * N] = (w[s] / eps) * lbb;
    } else {
      double acc = 0.0;
      for (int s = 0; s < S; ++s) {
        double g = 0.0;
        for (int z = 0; z < slices; ++z) g += psum[((long long)z * S + s) * N + j];
        g = -g;
        Yv[j + (long long)s * N] = g;  // Gbar, replaced by y below
        acc += g;
      }
      lbb = eps * acc;
      for (int s = 0; s < S; ++s) {
        const long long k = j + (long long)s * N;
        Yv[k] = (w[s] / eps) * lbb - Yv[k];
      }
    }
    for (int s = 0; s < S; ++s) gwp[(long long)j * S + s] -= Ml[j + (long long)s * N] * lbb;
  }
}

// Adjoint row step (thread per (i, s)): Fbar = sum over slices; grad_A += Fbar / A.
__global__ void row_merge_bwd(const double* psum, int slices, int M, int S, const double* A, double* Fbar,
                              double* gA) {
  const long long n = (long long)M * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % M), s = (int)(e / M);
    double f = 0.0;
    for (int z = 0; z < slices; ++z) f += psum[((long long)z * S + s) * M + i];
    Fbar[e] = f;
    gA[e] += f / A[e];
  }
}

__global__ void axpby_kernel(double* x, long long n, double a) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    x[k] *= a;
}

__global__ void zero_kernel(double* x, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    x[k] = 0.0;
}

__global__ void log_kernel(const double* x, long long n, double* out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = log(x[k]);
}

// grad_w[s] = (sum_j gwp[j S + s]) / eps, one block per s, fixed order.
__global__ void reduce_gw_eps(const double* gwp, int N, int S, double eps, double* gw) {
  __shared__ double sh[256];
  const int s = blockIdx.x;
  double v = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) v += gwp[(long long)j * S + s];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) gw[s] = sh[0] / eps;  // :377
}

// One block: b = exp(logb) / sum, loss = sum (b - b_ext)^2 when b_ext (:268-271).
__global__ void finish_b(const double* logb, int N, const double* bext, double* bn, double* out2) {
  __shared__ double sh[1024];
  double acc = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) acc += exp(logb[j]);
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double tot = sh[0];
  __syncthreads();
  double l = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    const double v = exp(logb[j]) / tot;
    bn[j] = v;
    if (bext) {
      const double d = v - bext[j];
      l += d * d;
    }
  }
  sh[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out2[0] = tot;
    out2[1] = sh[0];
  }
}

enum {
  SL_FH = 300, SL_GH, SL_MH, SL_RH, SL_LB, SL_LOGA, SL_D, SL_GRAM, SL_PMAX, SL_PSUM, SL_FBAR, SL_Y, SL_GA,
  SL_GWP, SL_GW, SL_BN, SL_SCAL
};

int grid1(const Context* ctx, long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 8LL * ctx->sm_count));
}

// Reduction slices for a pass with `tiles` CTAs per slice: about two CTAs
// per SM in all, each slice at least 4 shared tiles long.
int pick_slices(const Context* ctx, long long tiles, int K) {
  const long long want = (2LL * ctx->sm_count + tiles - 1) / tiles;
  const long long most = std::max(1, (K + 4 * TK - 1) / (4 * TK));
  return (int)std::max(1LL, std::min(want, most));
}

}  // namespace barylog

namespace bary {

using namespace barylog;

// The log barycenter in the log domain; arguments and outputs as run()
// (barycenter.h).  *launches is increased by the kernels launched.
int run_log(Context* ctx, cudaStream_t st, double* X1, double* X2, double* b, double* gradA, double* gradw,
            double* loss, int* iter_out, double* err_out, const double* A, const double* w, const double* C,
            const double* bext, int M, int N, int S, double reg, int withgrad, int max_iter, double tol,
            int* launches) {
  const int L = std::max(0, max_iter);
  const size_t MS = (size_t)M * S, NS = (size_t)N * S;
  const long long ldd = ((M + 1) / 2) * 2;
  const int H = withgrad ? L + 2 : 2;  // slots of F (l = 0..L+1) and of G, m, r
  const bool fixed = !(tol > 0.0);
  // slices of the passes (the column passes reduce over M, the row passes over N)
  const long long col_tiles = (long long)((N + TO - 1) / TO) * ((S + TS - 1) / TS);
  const long long row_tiles = (long long)((M + TO - 1) / TO) * ((S + TS - 1) / TS);
  const int zc = pick_slices(ctx, col_tiles, M), zr = pick_slices(ctx, row_tiles, N);
  const int kc_col = ((M + zc - 1) / zc + TK - 1) / TK * TK, kc_row = ((N + zr - 1) / zr + TK - 1) / TK * TK;
  const int zcol = (M + kc_col - 1) / kc_col, zrow = (N + kc_row - 1) / kc_row;
  const size_t part = std::max((size_t)zcol * NS, (size_t)zrow * MS);

  double* Fh = (double*)scratch(ctx, SL_FH, sizeof(double) * MS * H);
  double* Gh = (double*)scratch(ctx, SL_GH, sizeof(double) * NS * H);
  double* Mh = (double*)scratch(ctx, SL_MH, sizeof(double) * NS * H);
  double* Rh = (double*)scratch(ctx, SL_RH, sizeof(double) * MS * H);
  double* lb = (double*)scratch(ctx, SL_LB, sizeof(double) * N);
  double* logA = (double*)scratch(ctx, SL_LOGA, sizeof(double) * MS);
  double* D = (double*)scratch(ctx, SL_D, sizeof(double) * ldd * S);
  double* gram = (double*)scratch(ctx, SL_GRAM, sizeof(double) * S * S);
  double* pmax = (double*)scratch(ctx, SL_PMAX, sizeof(double) * part);
  double* psum = (double*)scratch(ctx, SL_PSUM, sizeof(double) * part);
  double* bn = (double*)scratch(ctx, SL_BN, sizeof(double) * N);
  double* scal = (double*)scratch(ctx, SL_SCAL, sizeof(double) * 8);
  if (!Fh || !Gh || !Mh || !Rh || !lb || !logA || !D || !gram || !pmax || !psum || !bn || !scal) return RWIG_E_NOMEM;
  double *Fbar = nullptr, *Yv = nullptr, *gA = nullptr, *gwp = nullptr, *gw = nullptr;
  if (withgrad) {
    Fbar = (double*)scratch(ctx, SL_FBAR, sizeof(double) * MS);
    Yv = (double*)scratch(ctx, SL_Y, sizeof(double) * NS);
    gA = (double*)scratch(ctx, SL_GA, sizeof(double) * MS);
    gwp = (double*)scratch(ctx, SL_GWP, sizeof(double) * NS);
    gw = (double*)scratch(ctx, SL_GW, sizeof(double) * S);
    if (!Fbar || !Yv || !gA || !gwp || !gw) return RWIG_E_NOMEM;
  }
  auto slot = [&](double* base, size_t sz, int l) { return base + sz * (size_t)(withgrad ? l : (l & 1)); };
  const double inv_eps = 1.0 / reg;
  int nl = 0;
  // column pass over C - P (P: M x S), row pass over C - P (P: N x S)
  auto col_pass = [&](const double* P1, const double* P2, long long ldp2, double p2c, const double* Q,
                      const double* Y) -> int {
    Pass p{C, (long long)M, M, N, S, P1, (long long)M, P2, ldp2, p2c, Q, (long long)N, Y, (long long)M,
           inv_eps, kc_col, pmax, psum};
    const dim3 grid((N + TO - 1) / TO, (S + TS - 1) / TS, zcol);
    if (Y) pass_kernel<false, true><<<grid, NT, 0, st>>>(p);
    else pass_kernel<false, false><<<grid, NT, 0, st>>>(p);
    ++nl;
    return 0;
  };
  auto row_pass = [&](const double* P1, const double* P2, long long ldp2, double p2c, const double* Q,
                      const double* Y) -> int {
    Pass p{C, (long long)M, N, M, S, P1, (long long)N, P2, ldp2, p2c, Q, (long long)M, Y, (long long)N,
           inv_eps, kc_row, pmax, psum};
    const dim3 grid((M + TO - 1) / TO, (S + TS - 1) / TS, zrow);
    if (Y) pass_kernel<true, true><<<grid, NT, 0, st>>>(p);
    else pass_kernel<true, false><<<grid, NT, 0, st>>>(p);
    ++nl;
    return 0;
  };

  // F_0 = G_0 = 0, log A; the initial row soft-min at (0, 0) gives F_1 (:221, :231)
  zero_kernel<<<grid1(ctx, MS), 256, 0, st>>>(slot(Fh, MS, 0), (long long)MS);
  zero_kernel<<<grid1(ctx, NS), 256, 0, st>>>(slot(Gh, NS, 0), (long long)NS);
  zero_kernel<<<grid1(ctx, N), 256, 0, st>>>(lb, N);
  log_kernel<<<grid1(ctx, MS), 256, 0, st>>>(A, (long long)MS, logA);
  nl += 4;
  row_pass(slot(Gh, NS, 0), nullptr, 0, 0.0, nullptr, nullptr);
  row_merge_fwd<<<grid1(ctx, MS), 256, 0, st>>>(pmax, psum, zrow, M, S, reg, slot(Fh, MS, 0), logA, nullptr,
                                                  slot(Fh, MS, 1), nullptr, ldd);
  ++nl;
  int iter = 0;
  double err = 1000.0;
  while (iter < L && err >= tol) {
    ++iter;
    const int l = iter;
    col_pass(slot(Fh, MS, l), nullptr, 0, 0.0, nullptr, nullptr);
    col_merge_fwd<<<grid1(ctx, N), 256, 0, st>>>(pmax, psum, zcol, N, S, reg, w, slot(Mh, NS, l), slot(Gh, NS, l),
                                                  lb);
    row_pass(slot(Gh, NS, l), nullptr, 0, 0.0, nullptr, nullptr);
    const bool need_err = !fixed || iter == L;
    row_merge_fwd<<<grid1(ctx, MS), 256, 0, st>>>(pmax, psum, zrow, M, S, reg, slot(Fh, MS, l), logA,
                                                    slot(Rh, MS, l), slot(Fh, MS, l + 1), need_err ? D : nullptr,
                                                    ldd);
    nl += 2;
    RWIG_CUDA_TRY(cudaGetLastError());
    if (need_err) {
      int gl = 0;
      if (int rc = dg::gemm<1>(ctx, dg::GemmArgs{D, ldd, S, M, S, D, ldd, 0}, dg::EpiStore{gram, S, S}, st, 0, &gl))
        return rc;
      nl += gl;
      std::vector<double> G((size_t)S * S);
      RWIG_CUDA_TRY(cudaMemcpyAsync(G.data(), gram, sizeof(double) * S * S, cudaMemcpyDeviceToHost, st));
      RWIG_CUDA_TRY(cudaStreamSynchronize(st));
      err = std::sqrt(lambda_max(G, S));  // Armadillo norm(X, 2) of a matrix: the spectral norm
    }
  }
  // normalised barycenter and loss (:268-271)
  finish_b<<<1, 1024, 0, st>>>(lb, N, withgrad ? bext : nullptr, bn, scal);
  ++nl;

  if (withgrad && iter > 0) {
    RWIG_CUDA_TRY(cudaMemsetAsync(gA, 0, sizeof(double) * MS, st));
    RWIG_CUDA_TRY(cudaMemsetAsync(gwp, 0, sizeof(double) * NS, st));
    for (int l = iter; l >= 1; --l) {
      const bool seed = (l == iter);
      if (!seed) {
        // Gbar: column pass weighted by the row softmax at (F_l, G_l) (:306-320)
        col_pass(slot(Rh, MS, l), nullptr, 0, 0.0, slot(Gh, NS, l), Fbar);
      }
      col_merge_bwd<<<grid1(ctx, N), 256, 0, st>>>(psum, zcol, N, S, reg, seed ? 1 : 0, bn, bext, w,
                                                    slot(Mh, NS, l), Yv, gwp);
      // Fbar: row pass weighted by the column softmax at (F_l, G_{l-1}) (:330-346)
      row_pass(slot(Mh, NS, l), nullptr, 0, 0.0, slot(Fh, MS, l), Yv);
      row_merge_bwd<<<grid1(ctx, MS), 256, 0, st>>>(psum, zrow, M, S, A, Fbar, gA);
      nl += 2;
    }
    axpby_kernel<<<grid1(ctx, MS), 256, 0, st>>>(gA, (long long)MS, reg);  // :376
    reduce_gw_eps<<<S, 256, 0, st>>>(gwp, N, S, reg, gw);                 // :377
    nl += 2;
    if (gradA) RWIG_CUDA_TRY(cudaMemcpyAsync(gradA, gA, sizeof(double) * MS, cudaMemcpyDeviceToDevice, st));
    if (gradw) RWIG_CUDA_TRY(cudaMemcpyAsync(gradw, gw, sizeof(double) * S, cudaMemcpyDeviceToDevice, st));
  } else if (withgrad) {  // nothing to unroll
    if (gradA) RWIG_CUDA_TRY(cudaMemsetAsync(gradA, 0, sizeof(double) * MS, st));
    if (gradw) RWIG_CUDA_TRY(cudaMemsetAsync(gradw, 0, sizeof(double) * S, st));
  }
  // outputs F_L, G_L (the reference keeps them as U, V: :386-387); b
  if (X1) RWIG_CUDA_TRY(cudaMemcpyAsync(X1, slot(Fh, MS, iter), sizeof(double) * MS, cudaMemcpyDeviceToDevice, st));
  if (X2) RWIG_CUDA_TRY(cudaMemcpyAsync(X2, slot(Gh, NS, iter), sizeof(double) * NS, cudaMemcpyDeviceToDevice, st));
  if (b) RWIG_CUDA_TRY(cudaMemcpyAsync(b, bn, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
  double sc[2] = {0.0, 0.0};
  RWIG_CUDA_TRY(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  RWIG_CUDA_TRY(cudaGetLastError());
  if (loss) *loss = withgrad ? sc[1] : 0.0;
  if (iter_out) *iter_out = iter;
  if (err_out) *err_out = err;
  if (launches) *launches += nl;
  report().bary_norm = sc[0];
  return (err <= tol) ? 0 : (iter == L ? 1 : 2);
}

}  // namespace bary
}  // namespace rwig
