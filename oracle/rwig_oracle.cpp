// rwig_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement, on the CPU and in FP64, of rwig's Armadillo code
// path for entropic optimal transport.  It is the parity oracle for the CUDA
// engine in rwig_b200/: only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline / reference arm may load it, and only as the checker or as the
// timed CPU baseline.  Nothing in the product links against it.
//
// Every function below cites the reference file:line it restates (paths are
// relative to the rwig source tree).  Layout is column-major (R / Armadillo),
// X[i + j*rows].  Differences from real Armadillo are confined to summation
// order (plain sequential loops instead of BLAS dgemv/dgemm and Armadillo's
// accu), which moves results by ~1e-15 relative.
//
// Pinned against the reference's own known-answer tests
// (inst/tinytest/test_sinkhorn.R, inst/tinytest/test_barycenter.R) by
// tests/test_oracle_golden.py.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

using std::vector;

namespace {

// ---------------------------------------------------------------------------
// small dense helpers (column-major)
// ---------------------------------------------------------------------------

// y = K * x      (K is m x n)
void matvec(const double* K, const double* x, double* y, int m, int n) {
  for (int i = 0; i < m; ++i) y[i] = 0.0;
  for (int j = 0; j < n; ++j) {
    const double xj = x[j];
    const double* col = K + (size_t)j * m;
    for (int i = 0; i < m; ++i) y[i] += col[i] * xj;
  }
}

// y = K^T * x    (K is m x n)
void matvec_t(const double* K, const double* x, double* y, int m, int n) {
  for (int j = 0; j < n; ++j) {
    const double* col = K + (size_t)j * m;
    double s = 0.0;
    for (int i = 0; i < m; ++i) s += col[i] * x[i];
    y[j] = s;
  }
}

// Y = K * X      (K m x n, X n x s, Y m x s)
void matmul(const double* K, const double* X, double* Y, int m, int n, int s) {
  for (int c = 0; c < s; ++c) matvec(K, X + (size_t)c * n, Y + (size_t)c * m, m, n);
}

// Y = K^T * X    (K m x n, X m x s, Y n x s)
void matmul_t(const double* K, const double* X, double* Y, int m, int n, int s) {
  for (int c = 0; c < s; ++c) matvec_t(K, X + (size_t)c * m, Y + (size_t)c * n, m, n);
}

double nrm2(const vector<double>& x) {
  double s = 0.0;
  for (double v : x) s += v * v;
  return std::sqrt(s);
}

// Largest singular value of an m x s matrix: Armadillo's norm(X, 2) for a
// matrix is the induced 2-norm (barycenter_impl_log.cpp:252 relies on it).
// Computed as sqrt(lambda_max(X^T X)) with cyclic Jacobi on the s x s Gram.
double spectral_norm(const double* X, int m, int s) {
  if (s == 0 || m == 0) return 0.0;
  vector<double> G((size_t)s * s, 0.0);
  for (int a = 0; a < s; ++a)
    for (int b = a; b < s; ++b) {
      double acc = 0.0;
      for (int i = 0; i < m; ++i) acc += X[i + (size_t)a * m] * X[i + (size_t)b * m];
      G[a + b * s] = G[b + a * s] = acc;
    }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < s; ++p)
      for (int q = p + 1; q < s; ++q) off += G[p + q * s] * G[p + q * s];
    if (off < 1e-300) break;
    for (int p = 0; p < s; ++p)
      for (int q = p + 1; q < s; ++q) {
        double apq = G[p + q * s];
        if (apq == 0.0) continue;
        double app = G[p + p * s], aqq = G[q + q * s];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < s; ++k) {
          double gkp = G[k + p * s], gkq = G[k + q * s];
          G[k + p * s] = c * gkp - sn * gkq;
          G[k + q * s] = sn * gkp + c * gkq;
        }
        for (int k = 0; k < s; ++k) {
          double gpk = G[p + k * s], gqk = G[q + k * s];
          G[p + k * s] = c * gpk - sn * gqk;
          G[q + k * s] = sn * gpk + c * gqk;
        }
      }
  }
  double lmax = 0.0;
  for (int p = 0; p < s; ++p) lmax = std::max(lmax, G[p + p * s]);
  return std::sqrt(lmax);
}

// Chunked std::thread fan-out with the reference's split: chunk = n / T and
// the last thread takes the remainder (sinkhorn_impl_log.cpp:89-94).
template <class F>
void chunked(int n_threads, int n, F&& body) {
  if (n_threads <= 1) {
    body(0, n);
    return;
  }
  vector<std::thread> th;
  int chunk = n / n_threads;
  for (int t = 0; t < n_threads; ++t) {
    int start = t * chunk;
    int end = (t == n_threads - 1) ? n : (t + 1) * chunk;
    th.emplace_back([&body, start, end]() { body(start, end); });
  }
  for (auto& t : th) t.join();
}

// R = C - f 1^T - 1 g^T, materialised the way Sinkhorn::_compute_R does
// (sinkhorn_impl_log.cpp:23-28): (C_ij - f_i) - g_j.
void compute_R(vector<double>& R, const vector<double>& C, const double* f,
               const double* g, int m, int n) {
  for (int j = 0; j < n; ++j) {
    const double gj = g[j];
    const double* c = C.data() + (size_t)j * m;
    double* r = R.data() + (size_t)j * m;
    for (int i = 0; i < m; ++i) r[i] = (c[i] - f[i]) - gj;
  }
}

// softmin over row i of R: min - eps * log(sum exp(-(R - min)/eps))
// (sinkhorn_impl_log.cpp:35-37, :101-105)
double softmin_row(const vector<double>& R, int i, int m, int n, double eps) {
  double mn = std::numeric_limits<double>::infinity();
  for (int j = 0; j < n; ++j) mn = std::min(mn, R[i + (size_t)j * m]);
  double s = 0.0;
  for (int j = 0; j < n; ++j) s += std::exp(-(R[i + (size_t)j * m] - mn) / eps);
  return mn - eps * std::log(s);
}

// softmin over column j of R (sinkhorn_impl_log.cpp:48-50, :138-142)
double softmin_col(const vector<double>& R, int j, int m, double eps) {
  const double* r = R.data() + (size_t)j * m;
  double mn = std::numeric_limits<double>::infinity();
  for (int i = 0; i < m; ++i) mn = std::min(mn, r[i]);
  double s = 0.0;
  for (int i = 0; i < m; ++i) s += std::exp(-(r[i] - mn) / eps);
  return mn - eps * std::log(s);
}

void minrow(const vector<double>& R, vector<double>& out, int m, int n, double eps, int nt) {
  chunked(nt, m, [&](int s, int e) {
    for (int i = s; i < e; ++i) out[i] = softmin_row(R, i, m, n, eps);
  });
}

void mincol(const vector<double>& R, vector<double>& out, int m, int n, double eps, int nt) {
  chunked(nt, n, [&](int s, int e) {
    for (int j = s; j < e; ++j) out[j] = softmin_col(R, j, m, eps);
  });
}

// Un-normalised barycenter of the last barycenter call on this thread (the
// backward passes differentiate losses built on it; see oracle_last_raw_b).
thread_local vector<double> t_raw_b;

int return_code(double err, double tol, int iter, int max_iter) {
  // sinkhorn_impl_vanilla.cpp:79-85
  if (err <= tol) return 0;
  if (iter == max_iter) return 1;
  return 2;
}

void support(const double* x, int n, vector<int>& idx) {
  idx.clear();
  for (int i = 0; i < n; ++i)
    if (x[i] != 0.0) idx.push_back(i);
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Vanilla Sinkhorn: Sinkhorn::compute_vanilla (sinkhorn_impl_vanilla.cpp:18),
// _fwd_vanilla (:93), _bwd_vanilla (:169).  Returns the reference's
// return_status (0 converged, 1 max_iter reached, 2 otherwise).
// ---------------------------------------------------------------------------
int oracle_sinkhorn_vanilla(double* P, double* grad_a, double* u_out, double* v_out,
                            double* loss_out, int* iter_out, double* err_out,
                            const double* a, const double* b, const double* C, int M,
                            int N, double reg, int withgrad, int max_iter, double tol) {
  vector<int> ai, bj;
  support(a, M, ai);
  support(b, N, bj);
  const int m = (int)ai.size(), n = (int)bj.size();
  vector<double> ar(m), br(n), Cr((size_t)m * n), K((size_t)m * n);
  for (int i = 0; i < m; ++i) ar[i] = a[ai[i]];
  for (int j = 0; j < n; ++j) br[j] = b[bj[j]];
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) Cr[i + (size_t)j * m] = C[ai[i] + (size_t)bj[j] * M];
  // K = exp(-C / reg) (:41); symmatu of an exactly symmetric K is a no-op (:43-45)
  for (size_t k = 0; k < K.size(); ++k) K[k] = std::exp(-Cr[k] / reg);

  vector<double> u(m, 1.0), v(n, 1.0), Kv(m), KTu(n);
  vector<vector<double>> uh, vh;
  if (withgrad) {
    uh.push_back(u);
    vh.push_back(v);
  }
  int iter = 0;
  double err = 1000.0;
  matvec(K.data(), v.data(), Kv.data(), m, n);  // :117
  while (iter < max_iter && err >= tol) {       // :119
    ++iter;
    for (int i = 0; i < m; ++i) u[i] = ar[i] / Kv[i];
    if (withgrad) uh.push_back(u);
    matvec_t(K.data(), u.data(), KTu.data(), m, n);
    for (int j = 0; j < n; ++j) v[j] = br[j] / KTu[j];
    if (withgrad) vh.push_back(v);
    matvec(K.data(), v.data(), Kv.data(), m, n);
    double e1 = 0.0, e2 = 0.0;  // :139
    for (int i = 0; i < m; ++i) {
      double d = u[i] * Kv[i] - ar[i];
      e1 += d * d;
    }
    for (int j = 0; j < n; ++j) {
      double d = v[j] * KTu[j] - br[j];
      e2 += d * d;
    }
    err = std::sqrt(e1) + std::sqrt(e2);
  }

  // P = diag(u) K diag(v) (:58), loss (:69)
  vector<double> Pr((size_t)m * n);
  double l1 = 0.0, l2 = 0.0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      size_t k = i + (size_t)j * m;
      Pr[k] = (u[i] * K[k]) * v[j];
      l1 += Cr[k] * Pr[k];
      l2 += Pr[k] * (std::log(Pr[k]) - 1.0);
    }
  if (loss_out) *loss_out = l1 + reg * l2;
  if (P) {
    std::fill(P, P + (size_t)M * N, 0.0);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) P[ai[i] + (size_t)bj[j] * M] = Pr[i + (size_t)j * m];
  }
  if (u_out) {
    std::fill(u_out, u_out + M, 0.0);
    for (int i = 0; i < m; ++i) u_out[ai[i]] = u[i];
  }
  if (v_out) {
    std::fill(v_out, v_out + N, 0.0);
    for (int j = 0; j < n; ++j) v_out[bj[j]] = v[j];
  }

  if (withgrad && grad_a) {
    // _bwd_vanilla (:169-213)
    vector<double> PbarK((size_t)m * n);
    for (size_t k = 0; k < PbarK.size(); ++k) PbarK[k] = (Cr[k] + reg * std::log(Pr[k])) * K[k];
    vector<double> ubar(m, 0.0), vbar(n, 0.0), g(m, 0.0), tm(m), tn(n), tn2(n), tm2(m);
    for (int l = iter; l > 0; --l) {
      if (l == iter) {
        matvec_t(PbarK.data(), u.data(), vbar.data(), m, n);  // vbar = PbarK^T u
        matvec_t(K.data(), u.data(), tn.data(), m, n);        // K^T u
        for (int j = 0; j < n; ++j) tn[j] = (vbar[j] * v[j]) / tn[j];
        matvec(PbarK.data(), v.data(), tm.data(), m, n);
        matvec(K.data(), tn.data(), tm2.data(), m, n);
        for (int i = 0; i < m; ++i) ubar[i] = tm[i] - tm2[i];
      } else {
        matvec(K.data(), vh[l].data(), tm.data(), m, n);  // K v_l
        for (int i = 0; i < m; ++i) tm[i] = (ubar[i] * uh[l + 1][i]) / tm[i];
        matvec_t(K.data(), tm.data(), vbar.data(), m, n);
        for (int j = 0; j < n; ++j) vbar[j] = -vbar[j];
        matvec_t(K.data(), uh[l].data(), tn.data(), m, n);  // K^T u_l
        for (int j = 0; j < n; ++j) tn[j] = (vbar[j] * vh[l][j]) / tn[j];
        matvec(K.data(), tn.data(), ubar.data(), m, n);
        for (int i = 0; i < m; ++i) ubar[i] = -ubar[i];
      }
      matvec(K.data(), vh[l - 1].data(), tm.data(), m, n);  // :212
      for (int i = 0; i < m; ++i) g[i] += ubar[i] / tm[i];
    }
    std::fill(grad_a, grad_a + M, 0.0);
    for (int i = 0; i < m; ++i) grad_a[ai[i]] = g[i];
  }
  if (iter_out) *iter_out = iter;
  if (err_out) *err_out = err;
  return return_code(err, tol, iter, max_iter);
}

// ---------------------------------------------------------------------------
// Log-stabilised Sinkhorn: Sinkhorn::compute_log (sinkhorn_impl_log.cpp:225),
// _fwd_log (:298), _bwd_log (:379).  n_threads > 0 fans the row / column
// soft-min sweeps out over std::threads with the reference's chunking
// (:82-217); n_threads == 0 runs them serially.  Both give identical numbers.
// ---------------------------------------------------------------------------
int oracle_sinkhorn_log(double* P, double* grad_a, double* f_out, double* g_out,
                        double* loss_out, int* iter_out, double* err_out, const double* a,
                        const double* b, const double* C, int M, int N, double reg,
                        int withgrad, int max_iter, double tol, int n_threads) {
  vector<int> ai, bj;
  support(a, M, ai);
  support(b, N, bj);
  const int m = (int)ai.size(), n = (int)bj.size();
  vector<double> ar(m), br(n), Cr((size_t)m * n), R((size_t)m * n);
  for (int i = 0; i < m; ++i) ar[i] = a[ai[i]];
  for (int j = 0; j < n; ++j) br[j] = b[bj[j]];
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) Cr[i + (size_t)j * m] = C[ai[i] + (size_t)bj[j] * M];

  vector<double> f(m, 0.0), g(n, 0.0), loga(m), logb(n), Rrow(m, 0.0), Rcol(n, 0.0);
  for (int i = 0; i < m; ++i) loga[i] = std::log(ar[i]);
  for (int j = 0; j < n; ++j) logb[j] = std::log(br[j]);
  vector<vector<double>> fh, gh;
  if (withgrad) {
    fh.push_back(f);
    gh.push_back(g);
  }
  int iter = 0;
  double err = 1000.0;
  compute_R(R, Cr, f.data(), g.data(), m, n);  // :325
  minrow(R, Rrow, m, n, reg, n_threads);
  while (iter < max_iter && err >= tol) {  // :327
    ++iter;
    for (int i = 0; i < m; ++i) f[i] += reg * loga[i] + Rrow[i];  // :336
    if (withgrad) fh.push_back(f);
    compute_R(R, Cr, f.data(), g.data(), m, n);  // :348
    mincol(R, Rcol, m, n, reg, n_threads);
    for (int j = 0; j < n; ++j) g[j] += reg * logb[j] + Rcol[j];  // :349
    if (withgrad) gh.push_back(g);
    compute_R(R, Cr, f.data(), g.data(), m, n);  // :359
    minrow(R, Rrow, m, n, reg, n_threads);
    mincol(R, Rcol, m, n, reg, n_threads);
    vector<double> d1(m), d2(n);  // :360
    for (int i = 0; i < m; ++i) d1[i] = -Rrow[i] / reg - loga[i];
    for (int j = 0; j < n; ++j) d2[j] = -Rcol[j] / reg - logb[j];
    err = nrm2(d1) + nrm2(d2);
  }

  // P = exp(-R / reg) from the last R (:266); loss (:277)
  vector<double> Pr((size_t)m * n);
  double l1 = 0.0, l2 = 0.0;
  for (size_t k = 0; k < Pr.size(); ++k) {
    Pr[k] = std::exp(-R[k] / reg);
    l1 += Cr[k] * Pr[k];
    l2 += Pr[k] * (std::log(Pr[k]) - 1.0);
  }
  if (loss_out) *loss_out = l1 + reg * l2;
  if (P) {
    std::fill(P, P + (size_t)M * N, 0.0);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) P[ai[i] + (size_t)bj[j] * M] = Pr[i + (size_t)j * m];
  }
  const double ninf = -std::numeric_limits<double>::infinity();
  if (f_out) {
    std::fill(f_out, f_out + M, ninf);  // :267
    for (int i = 0; i < m; ++i) f_out[ai[i]] = f[i];
  }
  if (g_out) {
    std::fill(g_out, g_out + N, ninf);  // :268
    for (int j = 0; j < n; ++j) g_out[bj[j]] = g[j];
  }

  if (withgrad && grad_a) {
    // _bwd_log (:379-520).  R holds R(f_L, g_L) on entry (:266).
    vector<double> PbarP((size_t)m * n);
    for (size_t k = 0; k < PbarP.size(); ++k) PbarP[k] = (Cr[k] + reg * std::log(Pr[k])) * Pr[k];
    vector<double> fbar(m, 0.0), gbar(n, 0.0), ga(m, 0.0);
    for (int l = iter; l > 0; --l) {
      if (l == iter) {
        for (int j = 0; j < n; ++j) {  // :414
          double s = 0.0;
          for (int i = 0; i < m; ++i) s += PbarP[i + (size_t)j * m];
          gbar[j] = s / reg;
        }
      } else {
        compute_R(R, Cr, fh[l].data(), gh[l].data(), m, n);  // :418-420
        // X = row-softmax(-R/reg)^T ; gbar = -X fbar   (:445-454)
        vector<double> gnew(n, 0.0);
        for (int i = 0; i < m; ++i) {
          double mn = std::numeric_limits<double>::infinity();
          for (int j = 0; j < n; ++j) mn = std::min(mn, R[i + (size_t)j * m]);
          double s = 0.0;
          for (int j = 0; j < n; ++j) s += std::exp(-(R[i + (size_t)j * m] - mn) / reg);
          for (int j = 0; j < n; ++j)
            gnew[j] += (std::exp(-(R[i + (size_t)j * m] - mn) / reg) / s) * fbar[i];
        }
        for (int j = 0; j < n; ++j) gbar[j] = -gnew[j];
      }
      // W = col-softmax(-R/reg) of the current R ; fbar = -W gbar (:480-488)
      vector<double> fnew(m, 0.0);
      for (int j = 0; j < n; ++j) {
        const double* r = R.data() + (size_t)j * m;
        double mn = std::numeric_limits<double>::infinity();
        for (int i = 0; i < m; ++i) mn = std::min(mn, r[i]);
        double s = 0.0;
        for (int i = 0; i < m; ++i) s += std::exp(-(r[i] - mn) / reg);
        for (int i = 0; i < m; ++i) fnew[i] += (std::exp(-(r[i] - mn) / reg) / s) * gbar[j];
      }
      for (int i = 0; i < m; ++i) fbar[i] = -fnew[i];
      if (l == iter) {
        for (int i = 0; i < m; ++i) {
          double s = 0.0;
          for (int j = 0; j < n; ++j) s += PbarP[i + (size_t)j * m];
          fbar[i] += s / reg;
        }
      }
      for (int i = 0; i < m; ++i) ga[i] += fbar[i] / ar[i];  // :513
    }
    std::fill(grad_a, grad_a + M, 0.0);
    for (int i = 0; i < m; ++i) grad_a[ai[i]] = ga[i] * reg;  // :515
  }
  if (iter_out) *iter_out = iter;
  if (err_out) *err_out = err;
  return return_code(err, tol, iter, max_iter);
}

// ---------------------------------------------------------------------------
// Parallel barycenter: Barycenter::compute_parallel
// (barycenter_impl_parallel.cpp:19), _fwd_parallel (:60), _bwd_parallel
// (:154).  A is M x S, C is M x N, w has S entries, b_ext N entries.
// ---------------------------------------------------------------------------
int oracle_barycenter_parallel(double* U_out, double* V_out, double* b_out, double* grad_A,
                               double* grad_w, double* loss_out, int* iter_out,
                               double* err_out, const double* A, const double* w,
                               const double* C, const double* b_ext, int M, int N, int S,
                               double reg, int withgrad, int max_iter, double tol) {
  const size_t MS = (size_t)M * S, NS = (size_t)N * S;
  vector<double> K((size_t)M * N);
  for (size_t k = 0; k < K.size(); ++k) K[k] = std::exp(-C[k] / reg);  // :84
  vector<double> U(MS, 1.0), V(NS, 1.0), b(N, 0.0), KV(MS), KTU(NS);
  vector<vector<double>> Uh, Vh, bh;
  if (withgrad) {
    Uh.push_back(U);
    Vh.push_back(V);
    bh.push_back(b);
  }
  int iter = 0;
  double err = 1000.0;
  matmul(K.data(), V.data(), KV.data(), M, N, S);  // :95
  while (iter < max_iter && err >= tol) {
    ++iter;
    for (size_t k = 0; k < MS; ++k) U[k] = A[k] / KV[k];  // :112
    if (withgrad) Uh.push_back(U);
    matmul_t(K.data(), U.data(), KTU.data(), M, N, S);  // :118
    for (int j = 0; j < N; ++j) {                       // :120 prod(pow(KTU, 1 w^T), 1)
      double p = 1.0;
      for (int s = 0; s < S; ++s) p *= std::pow(KTU[j + (size_t)s * N], w[s]);
      b[j] = p;
    }
    if (withgrad) bh.push_back(b);
    for (int s = 0; s < S; ++s)  // :126
      for (int j = 0; j < N; ++j) V[j + (size_t)s * N] = b[j] / KTU[j + (size_t)s * N];
    if (withgrad) Vh.push_back(V);
    matmul(K.data(), V.data(), KV.data(), M, N, S);  // :132
    double e = 0.0;                                  // :134
    for (size_t k = 0; k < MS; ++k) {
      double d = U[k] * KV[k] - A[k];
      e += d * d;
    }
    err = std::sqrt(e);
  }

  if (withgrad) {
    // _bwd_parallel (:154-206), uses the un-normalised b (:180)
    vector<double> gA(MS, 0.0), gw(S, 0.0), Ubar(MS, 0.0), Vbar(NS, 0.0), bbar(N, 0.0), KTUl(NS),
        T(NS), TM(MS), KVl(MS);
    for (int l = iter; l > 0; --l) {
      matmul_t(K.data(), Uh[l].data(), KTUl.data(), M, N, S);  // :177
      if (l == iter) {
        for (int j = 0; j < N; ++j) bbar[j] = 2.0 * (b[j] - b_ext[j]);  // :180
        for (int s = 0; s < S; ++s)
          for (int j = 0; j < N; ++j) T[j + (size_t)s * N] = (bbar[j] * w[s]) * V[j + (size_t)s * N];
        matmul(K.data(), T.data(), Ubar.data(), M, N, S);  // :181
      } else {
        matmul(K.data(), Vh[l].data(), KVl.data(), M, N, S);  // :183
        for (size_t k = 0; k < MS; ++k) TM[k] = (Ubar[k] * Uh[l + 1][k]) / KVl[k];
        matmul_t(K.data(), TM.data(), Vbar.data(), M, N, S);
        for (size_t k = 0; k < NS; ++k) Vbar[k] = -Vbar[k];
        for (int j = 0; j < N; ++j) {  // :184
          double s_ = 0.0;
          for (int s = 0; s < S; ++s) s_ += Vbar[j + (size_t)s * N] / KTUl[j + (size_t)s * N];
          bbar[j] = s_;
        }
        for (int s = 0; s < S; ++s)  // :185
          for (int j = 0; j < N; ++j) {
            size_t k = j + (size_t)s * N;
            T[k] = (bbar[j] * w[s] - Vbar[k] / KTUl[k]) * Vh[l][k];
          }
        matmul(K.data(), T.data(), Ubar.data(), M, N, S);
      }
      matmul(K.data(), Vh[l - 1].data(), KVl.data(), M, N, S);  // :204
      for (size_t k = 0; k < MS; ++k) gA[k] += Ubar[k] / KVl[k];
      for (int s = 0; s < S; ++s) {  // :205
        double acc = 0.0;
        for (int j = 0; j < N; ++j) acc += std::log(KTUl[j + (size_t)s * N]) * (bbar[j] * bh[l][j]);
        gw[s] += acc;
      }
    }
    if (grad_A) std::copy(gA.begin(), gA.end(), grad_A);
    if (grad_w) std::copy(gw.begin(), gw.end(), grad_w);
  }
  // b <- b / sum(b) after the backward (:39); loss with the normalised b (:42)
  t_raw_b = b;
  double sb = 0.0;
  for (int j = 0; j < N; ++j) sb += b[j];
  for (int j = 0; j < N; ++j) b[j] = b[j] / sb;
  if (withgrad && loss_out) {
    double ls = 0.0;
    for (int j = 0; j < N; ++j) {
      double d = b[j] - b_ext[j];
      ls += d * d;
    }
    *loss_out = ls;
  }
  if (b_out) std::copy(b.begin(), b.end(), b_out);
  if (U_out) std::copy(U.begin(), U.end(), U_out);
  if (V_out) std::copy(V.begin(), V.end(), V_out);
  if (iter_out) *iter_out = iter;
  if (err_out) *err_out = err;
  return return_code(err, tol, iter, max_iter);
}

// ---------------------------------------------------------------------------
// Log barycenter: Barycenter::compute_log (barycenter_impl_log.cpp:23),
// _fwd_log (:189), _bwd_log (:275).  F is M x S, G is N x S.
// The threaded soft-min sweeps shift each column by its own minimum (the
// serial form, :86-88); the reference's threaded column sweep uses a row
// minimum as the shift (:166), which is the same value in exact arithmetic.
// ---------------------------------------------------------------------------
namespace {
void bary_R(vector<double>& R, const double* C, const double* F, const double* G, int M, int N) {
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) R[i + (size_t)j * M] = (C[i + (size_t)j * M] - F[i]) - G[j];
}
void bary_minrow(const double* C, const vector<double>& F, const vector<double>& G,
                 vector<double>& KV, vector<double>& R, int M, int N, int S, double reg, int nt) {
  vector<double> tmp(M);
  for (int s = 0; s < S; ++s) {
    bary_R(R, C, F.data() + (size_t)s * M, G.data() + (size_t)s * N, M, N);
    minrow(R, tmp, M, N, reg, nt);
    std::copy(tmp.begin(), tmp.end(), KV.begin() + (size_t)s * M);
  }
}
void bary_mincol(const double* C, const vector<double>& F, const vector<double>& G,
                 vector<double>& KTU, vector<double>& R, int M, int N, int S, double reg, int nt) {
  vector<double> tmp(N);
  for (int s = 0; s < S; ++s) {
    bary_R(R, C, F.data() + (size_t)s * M, G.data() + (size_t)s * N, M, N);
    mincol(R, tmp, M, N, reg, nt);
    std::copy(tmp.begin(), tmp.end(), KTU.begin() + (size_t)s * N);
  }
}
}  // namespace

int oracle_barycenter_log(double* F_out, double* G_out, double* b_out, double* grad_A,
                          double* grad_w, double* loss_out, int* iter_out, double* err_out,
                          const double* A, const double* w, const double* C, const double* b_ext,
                          int M, int N, int S, double reg, int withgrad, int max_iter, double tol,
                          int n_threads) {
  const size_t MS = (size_t)M * S, NS = (size_t)N * S;
  vector<double> R((size_t)M * N), F(MS, 0.0), G(NS, 0.0), logb(N, 0.0), KV(MS, 0.0),
      KTU(NS, 0.0), logA(MS);
  for (size_t k = 0; k < MS; ++k) logA[k] = std::log(A[k]);
  vector<vector<double>> Fh, Gh, lbh;
  if (withgrad) {
    Fh.push_back(F);
    Gh.push_back(G);
    lbh.push_back(logb);
  }
  int iter = 0;
  double err = 1000.0;
  bary_minrow(C, F, G, KV, R, M, N, S, reg, n_threads);  // :221
  vector<double> D(MS);
  while (iter < max_iter && err >= tol) {
    ++iter;
    for (size_t k = 0; k < MS; ++k) F[k] += reg * logA[k] + KV[k];  // :231
    if (withgrad) Fh.push_back(F);
    bary_mincol(C, F, G, KTU, R, M, N, S, reg, n_threads);  // :238
    for (int j = 0; j < N; ++j) {                           // :239 logb = -(G + KTU) w / reg
      double acc = 0.0;
      for (int s = 0; s < S; ++s) acc += (G[j + (size_t)s * N] + KTU[j + (size_t)s * N]) * w[s];
      logb[j] = -acc / reg;
    }
    if (withgrad) lbh.push_back(logb);
    for (int s = 0; s < S; ++s)  // :245
      for (int j = 0; j < N; ++j) {
        size_t k = j + (size_t)s * N;
        G[k] += reg * logb[j] + KTU[k];
      }
    if (withgrad) Gh.push_back(G);
    bary_minrow(C, F, G, KV, R, M, N, S, reg, n_threads);  // :251
    for (size_t k = 0; k < MS; ++k) D[k] = -KV[k] / reg - logA[k];
    err = spectral_norm(D.data(), M, S);  // :252 norm(X, 2) of a matrix
  }
  vector<double> b(N);
  double sb = 0.0;
  for (int j = 0; j < N; ++j) {  // :268-269
    b[j] = std::exp(logb[j]);
    sb += b[j];
  }
  t_raw_b = b;
  for (int j = 0; j < N; ++j) b[j] = b[j] / sb;
  if (withgrad && loss_out) {  // :271
    double ls = 0.0;
    for (int j = 0; j < N; ++j) {
      double d = b[j] - b_ext[j];
      ls += d * d;
    }
    *loss_out = ls;
  }

  if (withgrad) {
    // _bwd_log (:275-382)
    vector<double> gA(MS, 0.0), gw(S, 0.0), Fbar(MS, 0.0), Gbar(NS, 0.0), lbbar(N, 0.0);
    for (int l = iter; l > 0; --l) {
      if (l != iter) {  // :306-320
        for (int s = 0; s < S; ++s) {
          bary_R(R, C, Fh[l].data() + (size_t)s * M, Gh[l].data() + (size_t)s * N, M, N);
          vector<double> acc(N, 0.0);
          for (int i = 0; i < M; ++i) {
            double mn = std::numeric_limits<double>::infinity();
            for (int j = 0; j < N; ++j) mn = std::min(mn, R[i + (size_t)j * M]);
            double sm = 0.0;
            for (int j = 0; j < N; ++j) sm += std::exp(-(R[i + (size_t)j * M] - mn) / reg);
            const double fb = Fbar[i + (size_t)s * M];
            for (int j = 0; j < N; ++j)
              acc[j] += (std::exp(-(R[i + (size_t)j * M] - mn) / reg) / sm) * fb;
          }
          for (int j = 0; j < N; ++j) Gbar[j + (size_t)s * N] = -acc[j];
        }
      }
      if (l == iter) {  // :323-327
        for (int j = 0; j < N; ++j) lbbar[j] = 2.0 * (b[j] - b_ext[j]) * b[j];
      } else {
        for (int j = 0; j < N; ++j) {
          double acc = 0.0;
          for (int s = 0; s < S; ++s) acc += Gbar[j + (size_t)s * N];
          lbbar[j] = reg * acc;
        }
      }
      for (int s = 0; s < S; ++s) {  // :330-346
        bary_R(R, C, Fh[l].data() + (size_t)s * M, Gh[l - 1].data() + (size_t)s * N, M, N);
        vector<double> acc(M, 0.0);
        const double ws = w[s] / reg;
        for (int j = 0; j < N; ++j) {
          const double* r = R.data() + (size_t)j * M;
          double mn = std::numeric_limits<double>::infinity();
          for (int i = 0; i < M; ++i) mn = std::min(mn, r[i]);
          double sm = 0.0;
          for (int i = 0; i < M; ++i) sm += std::exp(-(r[i] - mn) / reg);
          const double y = (l == iter) ? lbbar[j] : (ws * lbbar[j] - Gbar[j + (size_t)s * N]);
          for (int i = 0; i < M; ++i) acc[i] += (std::exp(-(r[i] - mn) / reg) / sm) * y;
        }
        for (int i = 0; i < M; ++i)
          Fbar[i + (size_t)s * M] = (l == iter) ? ws * acc[i] : acc[i];
      }
      for (size_t k = 0; k < MS; ++k) gA[k] += Fbar[k] / A[k];  // :364
      // grad_w -= (G_{l-1} + mincol(R(F_l, G_{l-1})))^T logbbar  (:368-372)
      bary_mincol(C, Fh[l], Gh[l - 1], KTU, R, M, N, S, reg, n_threads);
      for (int s = 0; s < S; ++s) {
        double acc = 0.0;
        for (int j = 0; j < N; ++j)
          acc += (Gh[l - 1][j + (size_t)s * N] + KTU[j + (size_t)s * N]) * lbbar[j];
        gw[s] -= acc;
      }
    }
    for (size_t k = 0; k < MS; ++k) gA[k] *= reg;  // :376-377
    for (int s = 0; s < S; ++s) gw[s] /= reg;
    if (grad_A) std::copy(gA.begin(), gA.end(), grad_A);
    if (grad_w) std::copy(gw.begin(), gw.end(), grad_w);
  }
  if (F_out) std::copy(F.begin(), F.end(), F_out);
  if (G_out) std::copy(G.begin(), G.end(), G_out);
  if (b_out) std::copy(b.begin(), b.end(), b_out);
  if (iter_out) *iter_out = iter;
  if (err_out) *err_out = err;
  return return_code(err, tol, iter, max_iter);
}

// ---------------------------------------------------------------------------
// WDL batched step: WassersteinDictionaryLearning::_train_batch_batched
// (wdl_impl.cpp:87-247).  K is the N x N Gibbs kernel, A (N x S) the current
// topics, WB (S x D) the batch's topic weights, YB (N x D) its documents.
// L fixed iterations; outputs the batch-averaged g_Alpha (N x S) and
// g_lambda (S) after the softmax Jacobians.
// ---------------------------------------------------------------------------
void oracle_wdl_batch_grad(double* g_Alpha, double* g_lambda, const double* A, const double* WB,
                           const double* YB, const double* K, int N, int S, int D, int L) {
  const int SD = S * D;
  const size_t NSD = (size_t)N * SD;
  vector<double> UB(NSD, 1.0), VB(NSD, 1.0), bB((size_t)N * D, 0.0), KVB(NSD), KTUB(NSD);
  vector<vector<double>> UBh(L + 1), VBh(L + 1), bBh(L + 1), KVBh(L), KTUBh(L + 1);
  UBh[0] = UB;
  VBh[0] = VB;
  bBh[0] = bB;
  for (int l = 0; l < L; ++l) {  // :124-160
    matmul(K, VB.data(), KVB.data(), N, N, SD);
    KVBh[l] = KVB;
    for (int d = 0; d < D; ++d)
      for (int s = 0; s < S; ++s)
        for (int i = 0; i < N; ++i) {
          size_t k = i + (size_t)(d * S + s) * N;
          UB[k] = A[i + (size_t)s * N] / KVB[k];
        }
    UBh[l + 1] = UB;
    matmul_t(K, UB.data(), KTUB.data(), N, N, SD);
    KTUBh[l + 1] = KTUB;
    for (int d = 0; d < D; ++d)
      for (int i = 0; i < N; ++i) {
        double p = 1.0;
        for (int s = 0; s < S; ++s)
          p *= std::pow(KTUB[i + (size_t)(d * S + s) * N], WB[s + (size_t)d * S]);
        bB[i + (size_t)d * N] = p;
      }
    bBh[l + 1] = bB;
    for (int d = 0; d < D; ++d)
      for (int s = 0; s < S; ++s)
        for (int i = 0; i < N; ++i) {
          size_t k = i + (size_t)(d * S + s) * N;
          VB[k] = bB[i + (size_t)d * N] / KTUB[k];
        }
    VBh[l + 1] = VB;
  }
  vector<double> UBbar(NSD, 0.0), VBbar(NSD, 0.0), bBbar((size_t)N * D, 0.0), ABbar(NSD, 0.0),
      wBbar((size_t)S * D, 0.0), tmp(NSD), t2(NSD);
  for (int l = L; l > 0; --l) {  // :169-218
    const vector<double>& KTU_l = KTUBh[l];  // equals K^T UB_hist[l] (:172)
    if (l == L) {
      for (int d = 0; d < D; ++d)
        for (int i = 0; i < N; ++i)
          bBbar[i + (size_t)d * N] = 2.0 * (bBh[l][i + (size_t)d * N] - YB[i + (size_t)d * N]);
      for (int d = 0; d < D; ++d)
        for (int s = 0; s < S; ++s)
          for (int i = 0; i < N; ++i) {
            size_t k = i + (size_t)(d * S + s) * N;
            tmp[k] = (bBbar[i + (size_t)d * N] * WB[s + (size_t)d * S]) * VBh[l][k];
          }
      matmul(K, tmp.data(), UBbar.data(), N, N, SD);
    } else {
      for (size_t k = 0; k < NSD; ++k) t2[k] = (UBbar[k] * UBh[l + 1][k]) / KVBh[l][k];
      matmul_t(K, t2.data(), VBbar.data(), N, N, SD);
      for (size_t k = 0; k < NSD; ++k) VBbar[k] = -VBbar[k];
      for (int d = 0; d < D; ++d)
        for (int i = 0; i < N; ++i) {
          double acc = 0.0;
          for (int s = 0; s < S; ++s) {
            size_t k = i + (size_t)(d * S + s) * N;
            acc += VBbar[k] / KTU_l[k];
          }
          bBbar[i + (size_t)d * N] = acc;
        }
      for (int d = 0; d < D; ++d)
        for (int s = 0; s < S; ++s)
          for (int i = 0; i < N; ++i) {
            size_t k = i + (size_t)(d * S + s) * N;
            tmp[k] = (bBbar[i + (size_t)d * N] * WB[s + (size_t)d * S] - VBbar[k] / KTU_l[k]) *
                     VBh[l][k];
          }
      matmul(K, tmp.data(), UBbar.data(), N, N, SD);
    }
    for (size_t k = 0; k < NSD; ++k) ABbar[k] += UBbar[k] / KVBh[l - 1][k];  // :210
    for (int d = 0; d < D; ++d)                                               // :213-217
      for (int s = 0; s < S; ++s) {
        double acc = 0.0;
        for (int i = 0; i < N; ++i)
          acc += std::log(KTU_l[i + (size_t)(d * S + s) * N]) *
                 (bBbar[i + (size_t)d * N] * bBh[l][i + (size_t)d * N]);
        wBbar[s + (size_t)d * S] += acc;
      }
  }
  // softmax Jacobians (:223-233)
  for (int j = 0; j < SD; ++j) {
    const int s = j % S;
    const double* as = A + (size_t)s * N;
    double* x = ABbar.data() + (size_t)j * N;
    double dot = 0.0;
    for (int i = 0; i < N; ++i) dot += as[i] * x[i];
    for (int i = 0; i < N; ++i) x[i] = as[i] * x[i] - as[i] * dot;
  }
  for (int d = 0; d < D; ++d) {
    const double* wd = WB + (size_t)d * S;
    double* x = wBbar.data() + (size_t)d * S;
    double dot = 0.0;
    for (int s = 0; s < S; ++s) dot += wd[s] * x[s];
    for (int s = 0; s < S; ++s) x[s] = wd[s] * x[s] - wd[s] * dot;
  }
  // batch averages (:236-243)
  for (size_t k = 0; k < (size_t)N * S; ++k) g_Alpha[k] = 0.0;
  for (int d = 0; d < D; ++d)
    for (size_t k = 0; k < (size_t)N * S; ++k) g_Alpha[k] += ABbar[k + (size_t)d * S * N];
  for (size_t k = 0; k < (size_t)N * S; ++k) g_Alpha[k] /= D;
  for (int s = 0; s < S; ++s) {
    double acc = 0.0;
    for (int d = 0; d < D; ++d) acc += wBbar[s + (size_t)d * S];
    g_lambda[s] = acc / D;
  }
}

// Copies the un-normalised barycenter of this thread's last barycenter call:
// prod_s KTU^w (parallel, barycenter_impl_parallel.cpp:120) or exp(logb)
// (log, barycenter_impl_log.cpp:268).  Returns its length.
int oracle_last_raw_b(double* out, int n) {
  const int k = std::min(n, (int)t_raw_b.size());
  for (int j = 0; j < k; ++j) out[j] = t_raw_b[j];
  return (int)t_raw_b.size();
}

// Column softmax of an r x c matrix (wdl_impl.hpp:80-96).
void oracle_col_softmax(double* out, const double* X, int r, int c) {
  for (int j = 0; j < c; ++j) {
    const double* x = X + (size_t)j * r;
    double* o = out + (size_t)j * r;
    double mx = -std::numeric_limits<double>::infinity();
    for (int i = 0; i < r; ++i) mx = std::max(mx, x[i]);
    double s = 0.0;
    for (int i = 0; i < r; ++i) {
      o[i] = std::exp(x[i] - mx);
      s += o[i];
    }
    for (int i = 0; i < r; ++i) o[i] = o[i] / s;
  }
}

// One optimizer update (optimizer.hpp:72-99).  opt: 0 SGD, 1 Adam, 2 AdamW.
// step is the 1-based step count after the increment.
void oracle_optimizer_step(double* theta, double* m, double* v, const double* g, size_t n, int opt,
                           int step, double eta, double gamma, double beta1, double beta2,
                           double eps) {
  if (opt == 0) {
    for (size_t k = 0; k < n; ++k) theta[k] = theta[k] - eta * g[k];
    return;
  }
  const double c1 = 1.0 - std::pow(beta1, step), c2 = 1.0 - std::pow(beta2, step);
  for (size_t k = 0; k < n; ++k) {
    m[k] = beta1 * m[k] + (1.0 - beta1) * g[k];
    v[k] = beta2 * v[k] + (1.0 - beta2) * std::pow(g[k], 2);
    const double mh = m[k] / c1, vh = v[k] / c2;
    if (opt == 1)
      theta[k] = theta[k] - eta * (mh / (std::sqrt(vh) + eps));
    else
      theta[k] = (1.0 - eta * gamma) * theta[k] - eta * (mh / (std::sqrt(vh) + eps));
  }
}

// WDL training loop: WassersteinDictionaryLearning::_compute_serial
// (wdl_impl.cpp:254-347) with the initial logits passed in (the reference
// draws them from randn, :277-278).  Runs E epochs over ceil(M/B) batches,
// stopping early after max_steps batches when max_steps > 0.  Writes A
// (N x S), W (S x M) and the final logits.
int oracle_wdl_train(double* A_out, double* W_out, double* Alpha, double* Lambda, const double* Y,
                     const double* C, int N, int M, int S, double reg, int L, int B, int E, int opt,
                     double eta, double gamma, double beta1, double beta2, double eps,
                     int max_steps) {
  vector<double> K((size_t)N * N);
  for (size_t k = 0; k < K.size(); ++k) K[k] = std::exp(-C[k] / reg);  // :297
  const size_t NS = (size_t)N * S, SM = (size_t)S * M;
  vector<double> A(NS), W(SM), mA(NS, 0.0), vA(NS, 0.0), mL(SM, 0.0), vL(SM, 0.0), gA(NS), gl(S),
      gL(SM);
  oracle_col_softmax(A.data(), Alpha, N, S);
  oracle_col_softmax(W.data(), Lambda, S, M);
  const int batches = (M % B) ? (M / B + 1) : (M / B);  // :307
  int steps = 0;
  for (int e = 0; e < E; ++e) {
    for (int bi = 0; bi < batches; ++bi) {
      if (max_steps > 0 && steps >= max_steps) goto done;
      const int D = (bi == M / B) ? (M % B) : B;  // :91
      oracle_wdl_batch_grad(gA.data(), gl.data(), A.data(), W.data() + (size_t)bi * B * S,
                            Y + (size_t)bi * B * N, K.data(), N, S, D, L);
      for (int mm = 0; mm < M; ++mm)  // :246 broadcast to every document
        for (int s = 0; s < S; ++s) gL[s + (size_t)mm * S] = gl[s];
      ++steps;
      oracle_optimizer_step(Alpha, mA.data(), vA.data(), gA.data(), NS, opt, steps, eta, gamma,
                            beta1, beta2, eps);
      oracle_optimizer_step(Lambda, mL.data(), vL.data(), gL.data(), SM, opt, steps, eta, gamma,
                            beta1, beta2, eps);
      oracle_col_softmax(A.data(), Alpha, N, S);
      oracle_col_softmax(W.data(), Lambda, S, M);
    }
  }
done:
  if (A_out) std::copy(A.begin(), A.end(), A_out);
  if (W_out) std::copy(W.begin(), W.end(), W_out);
  return steps;
}

}  // extern "C"
