// rwig_b200_glue.cpp -- the Rcpp glue rwig compiles to call this engine: the
// GPU branches of rwig's src/sinkhorn.cpp, src/barycenter.cpp and src/wdl.cpp,
// with the same R-level arguments and returned lists as the reference's own
// CUDA glue (sinkhorn_vanilla_cuda, src/sinkhorn.cpp:51-106;
// barycenter_parallel_cuda, src/barycenter.cpp:67-140; wdl_cpp_cuda,
// src/wdl.cpp:57-99), pointed at the C ABI of include/rwig_b200.h, plus the
// log-domain branches the reference has only on the CPU (sinkhorn_log_cpp
// :142, barycenter_log_cpp :168).  A maintainer adds this file to rwig's src/
// (and the two lines of INTEGRATION.md to src/Makevars.in); every engine
// error becomes an R error through Rcpp::stop.
#include <Rcpp.h>

#include "rwig_b200.h"

namespace {

int status_of(int rc) {
  if (rc < 0) Rcpp::stop(rwig_last_error());
  return rc;  // the reference's return_status (0 converged, 1 max_iter, 2 otherwise)
}

SEXP matrix(int rows, int cols) {
  SEXP x = PROTECT(Rf_allocVector(REALSXP, (R_xlen_t)rows * cols));
  SEXP dims = PROTECT(Rf_allocVector(INTSXP, 2));
  INTEGER(dims)[0] = rows;
  INTEGER(dims)[1] = cols;
  Rf_setAttrib(x, R_DimSymbol, dims);
  UNPROTECT(2);
  return x;
}

// Vanilla (log_domain = false) or log-stabilised Sinkhorn on the GPU.
Rcpp::List sinkhorn_gpu(bool log_domain, const SEXP& a, const SEXP& b, const SEXP& C, double reg, bool withgrad,
                        int maxiter, double zerotol) {
  const int m = Rf_nrows(C), n = Rf_ncols(C);
  SEXP P = PROTECT(matrix(m, n));
  SEXP x = PROTECT(Rf_allocVector(REALSXP, m));  // u (vanilla) or f (log)
  SEXP y = PROTECT(Rf_allocVector(REALSXP, n));  // v or g
  SEXP grad_a = PROTECT(Rf_allocVector(REALSXP, m));
  double loss = 0.0, err = 0.0;
  int iter = 0;
  auto entry = log_domain ? rwig_sinkhorn_log : rwig_sinkhorn_vanilla;
  const int rc = entry(REAL(P), withgrad ? REAL(grad_a) : nullptr, REAL(x), REAL(y), &loss, &iter, &err, REAL(a),
                       REAL(b), REAL(C), m, n, reg, withgrad ? 1 : 0, maxiter, zerotol);
  UNPROTECT(4);
  const int status = status_of(rc);
  const char* xn = log_domain ? "f" : "u";
  const char* yn = log_domain ? "g" : "v";
  if (withgrad)
    return Rcpp::List::create(Rcpp::Named("P") = P, Rcpp::Named("grad_a") = grad_a, Rcpp::Named(xn) = x,
                              Rcpp::Named(yn) = y, Rcpp::Named("loss") = loss, Rcpp::Named("iter") = iter,
                              Rcpp::Named("err") = err, Rcpp::Named("return_status") = status);
  return Rcpp::List::create(Rcpp::Named("P") = P, Rcpp::Named(xn) = x, Rcpp::Named(yn) = y,
                            Rcpp::Named("loss") = loss, Rcpp::Named("iter") = iter, Rcpp::Named("err") = err,
                            Rcpp::Named("return_status") = status);
}

// Parallel (log_domain = false) or log barycenter on the GPU.
Rcpp::List barycenter_gpu(bool log_domain, const SEXP& A, const SEXP& C, const SEXP& w, double reg,
                          const SEXP& b_ext, bool withgrad, int maxiter, double zerotol) {
  const int M = Rf_nrows(C), N = Rf_ncols(C), S = Rf_ncols(A);
  if (withgrad && Rf_length(b_ext) < N) Rcpp::stop("b_ext must have one entry per column of C");
  SEXP b = PROTECT(Rf_allocVector(REALSXP, N));
  SEXP X1 = PROTECT(matrix(M, S));  // U or F
  SEXP X2 = PROTECT(matrix(N, S));  // V or G
  SEXP grad_A = PROTECT(matrix(M, S));
  SEXP grad_w = PROTECT(Rf_allocVector(REALSXP, S));
  double loss = 0.0, err = 0.0;
  int iter = 0;
  auto entry = log_domain ? rwig_barycenter_log : rwig_barycenter_parallel;
  const int rc = entry(REAL(X1), REAL(X2), REAL(b), withgrad ? REAL(grad_A) : nullptr,
                       withgrad ? REAL(grad_w) : nullptr, &loss, &iter, &err, REAL(A), REAL(w), REAL(C),
                       withgrad ? REAL(b_ext) : nullptr, M, N, S, reg, withgrad ? 1 : 0, maxiter, zerotol);
  UNPROTECT(5);
  const int status = status_of(rc);
  const char* n1 = log_domain ? "F" : "U";
  const char* n2 = log_domain ? "G" : "V";
  if (withgrad)
    return Rcpp::List::create(Rcpp::Named("b") = b, Rcpp::Named("grad_A") = grad_A, Rcpp::Named("grad_w") = grad_w,
                              Rcpp::Named("loss") = loss, Rcpp::Named(n1) = X1, Rcpp::Named(n2) = X2,
                              Rcpp::Named("iter") = iter, Rcpp::Named("err") = err,
                              Rcpp::Named("return_status") = status);
  return Rcpp::List::create(Rcpp::Named("b") = b, Rcpp::Named(n1) = X1, Rcpp::Named(n2) = X2,
                            Rcpp::Named("iter") = iter, Rcpp::Named("err") = err,
                            Rcpp::Named("return_status") = status);
}

}  // namespace

Rcpp::List sinkhorn_vanilla_cuda(const SEXP& a, const SEXP& b, const SEXP& C, double reg, bool withgrad = false,
                                 int maxiter = 1000, double zerotol = 1e-6, int verbose = 0) {
  (void)verbose;
  return sinkhorn_gpu(false, a, b, C, reg, withgrad, maxiter, zerotol);
}

Rcpp::List sinkhorn_log_cuda(const SEXP& a, const SEXP& b, const SEXP& C, double reg, bool withgrad = false,
                             int maxiter = 1000, double zerotol = 1e-6, int verbose = 0) {
  (void)verbose;
  return sinkhorn_gpu(true, a, b, C, reg, withgrad, maxiter, zerotol);
}

Rcpp::List barycenter_parallel_cuda(const SEXP& A, const SEXP& C, const SEXP& w, double reg, const SEXP& b_ext,
                                    bool withgrad = false, int maxiter = 1000, double zerotol = 1e-6,
                                    int verbose = 0) {
  (void)verbose;
  return barycenter_gpu(false, A, C, w, reg, b_ext, withgrad, maxiter, zerotol);
}

Rcpp::List barycenter_log_cuda(const SEXP& A, const SEXP& C, const SEXP& w, double reg, const SEXP& b_ext,
                               bool withgrad = false, int maxiter = 1000, double zerotol = 1e-6, int verbose = 0) {
  (void)verbose;
  return barycenter_gpu(true, A, C, w, reg, b_ext, withgrad, maxiter, zerotol);
}

Rcpp::List wdl_cpp_cuda(const SEXP& Y, const SEXP& C, const double reg, const int S, const int batch_size,
                        const int epochs, int sinkhorn_mode = 1, const int max_iter = 1000,
                        const double zero_tol = 1e-6, const int optimizer = 2, const double eta = .001,
                        const double gamma = .01, const double beta1 = .9, const double beta2 = .999,
                        const double eps = 1e-8, const bool verbose = false, const int seed = 42) {
  (void)sinkhorn_mode;  // the GPU path's inference is the parallel barycenter, as in the reference
  const int N = Rf_nrows(Y), M = Rf_ncols(Y);
  SEXP A = PROTECT(matrix(N, S));
  SEXP W = PROTECT(matrix(S, M));
  SEXP Yhat = PROTECT(matrix(N, M));
  const int rc = rwig_wdl(REAL(A), REAL(W), REAL(Yhat), REAL(Y), REAL(C), N, M, S, reg, max_iter, zero_tol,
                          batch_size, epochs, optimizer, eta, gamma, beta1, beta2, eps, seed, verbose ? 1 : 0,
                          nullptr, nullptr, 0);
  UNPROTECT(3);
  status_of(rc);
  return Rcpp::List::create(Rcpp::Named("A") = A, Rcpp::Named("W") = W, Rcpp::Named("Yhat") = Yhat);
}
