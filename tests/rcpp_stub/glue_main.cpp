// glue_main.cpp -- drives the Rcpp glue (rwig_b200/rcpp/rwig_b200_glue.cpp)
// outside R through the stand-in Rcpp.h: one small call of each GPU branch,
// printing one line per call, "ok <name> <return_status> <iter> <number>" or
// "error <name> <R error message>".
#include <cmath>
#include <cstdio>

#include "Rcpp.h"

Rcpp::List sinkhorn_vanilla_cuda(const SEXP&, const SEXP&, const SEXP&, double, bool, int, double, int);
Rcpp::List sinkhorn_log_cuda(const SEXP&, const SEXP&, const SEXP&, double, bool, int, double, int);
Rcpp::List barycenter_parallel_cuda(const SEXP&, const SEXP&, const SEXP&, double, const SEXP&, bool, int, double,
                                    int);
Rcpp::List barycenter_log_cuda(const SEXP&, const SEXP&, const SEXP&, double, const SEXP&, bool, int, double, int);
Rcpp::List wdl_cpp_cuda(const SEXP&, const SEXP&, const double, const int, const int, const int, int, const int,
                        const double, const int, const double, const double, const double, const double,
                        const double, const bool, const int);

static SEXP vec(int n, double (*f)(int)) {
  SEXP x = Rf_allocVector(REALSXP, n);
  for (int i = 0; i < n; ++i) REAL(x)[i] = f(i);
  return x;
}
static SEXP mat(int r, int c, double (*f)(int, int)) {
  SEXP x = Rf_allocVector(REALSXP, (R_xlen_t)r * c);
  for (int j = 0; j < c; ++j)
    for (int i = 0; i < r; ++i) REAL(x)[i + (size_t)j * r] = f(i, j);
  SEXP d = Rf_allocVector(INTSXP, 2);
  INTEGER(d)[0] = r;
  INTEGER(d)[1] = c;
  Rf_setAttrib(x, R_DimSymbol, d);
  return x;
}

template <class F>
static void call(const char* name, F f, const char* num) {
  try {
    const Rcpp::List r = f();
    const int status = (int)(num[0] == '-' ? 0 : r["return_status"].num);
    const int iter = (int)(num[0] == '-' ? 0 : r["iter"].num);
    const double v = num[0] == '-' ? REAL(r["A"].sexp)[0] : (r[num].kind ? r[num].num : REAL(r[num].sexp)[0]);
    std::printf("ok %s %d %d %.17g\n", name, status, iter, v);
  } catch (const std::exception& e) {
    std::printf("error %s %s\n", name, e.what());
  }
}

int main() {
  const int n = 24, S = 3;
  auto cost = [](int i, int j) { const double d = (i - j) / 24.0; return d * d; };
  SEXP a = vec(n, [](int i) { return (1.0 + (i % 5)) / (3.0 * 24); });
  SEXP b = vec(n, [](int i) { return (1.0 + (i % 7)) / (4.0 * 24); });
  SEXP C = mat(n, n, cost);
  SEXP A = mat(n, S, [](int i, int s) { return (1.0 + ((i + s) % 4)) / (2.5 * 24); });
  SEXP w = vec(S, [](int s) { return 1.0 / 3 + 0 * s; });
  SEXP be = vec(n, [](int) { return 1.0 / 24; });
  SEXP Y = mat(n, 8, [](int i, int d) { return (1.0 + ((i * 3 + d) % 6)) / (3.5 * 24); });
  call("sinkhorn_vanilla", [&] { return sinkhorn_vanilla_cuda(a, b, C, 0.1, true, 1000, 1e-9, 0); }, "loss");
  call("sinkhorn_log", [&] { return sinkhorn_log_cuda(a, b, C, 0.05, false, 1000, 1e-9, 0); }, "loss");
  call("barycenter_parallel", [&] { return barycenter_parallel_cuda(A, C, w, 0.1, be, true, 20, 0.0, 0); }, "loss");
  call("barycenter_log", [&] { return barycenter_log_cuda(A, C, w, 0.1, be, true, 20, 0.0, 0); }, "loss");
  call("wdl", [&] { return wdl_cpp_cuda(Y, C, 0.1, 2, 4, 1, 1, 5, 1e-6, 1, 1e-3, 0.01, 0.9, 0.999, 1e-8, false, 3); },
       "-");
  return 0;
}
