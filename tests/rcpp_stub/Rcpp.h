// Rcpp.h -- a stand-in for R's C API and the parts of Rcpp that
// rwig_b200/rcpp/rwig_b200_glue.cpp uses, so that the glue compiles, links
// against the engine and runs outside R in the test suite.  Vectors are
// plain heap objects (never freed: a test process is short), PROTECT is a
// no-op, Rcpp::stop throws, and Rcpp::List keeps (name, value) pairs.
#pragma once
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

enum { REALSXP = 14, INTSXP = 13 };
typedef std::ptrdiff_t R_xlen_t;
struct SEXPREC {
  int type = 0;
  std::vector<double> real;
  std::vector<int> ints;
  std::vector<int> dim;
};
typedef SEXPREC* SEXP;

inline SEXP Rf_allocVector(int type, R_xlen_t n) {
  SEXP x = new SEXPREC;
  x->type = type;
  if (type == REALSXP) x->real.assign((size_t)n, 0.0);
  else x->ints.assign((size_t)n, 0);
  return x;
}
inline double* REAL(SEXP x) { return x->real.data(); }
inline int* INTEGER(SEXP x) { return x->ints.data(); }
inline int Rf_length(SEXP x) { return (int)(x->type == REALSXP ? x->real.size() : x->ints.size()); }
inline int Rf_nrows(SEXP x) { return x->dim.size() == 2 ? x->dim[0] : Rf_length(x); }
inline int Rf_ncols(SEXP x) { return x->dim.size() == 2 ? x->dim[1] : 1; }
static SEXPREC g_dim_symbol;
static const SEXP R_DimSymbol = &g_dim_symbol;
inline void Rf_setAttrib(SEXP x, SEXP sym, SEXP val) {
  if (sym == R_DimSymbol) x->dim = val->ints;
}
#define PROTECT(x) (x)
#define UNPROTECT(n) ((void)(n))

namespace Rcpp {
struct Value {
  std::string name;
  SEXP sexp = nullptr;
  double num = 0.0;
  int kind = 0;  // 0 SEXP, 1 number
};
struct Named {
  std::string name;
  explicit Named(const char* n) : name(n) {}
  Value operator=(SEXP x) const { return Value{name, x, 0.0, 0}; }
  Value operator=(double v) const { return Value{name, nullptr, v, 1}; }
  Value operator=(int v) const { return Value{name, nullptr, (double)v, 1}; }
};
struct List {
  std::vector<Value> items;
  template <class... T>
  static List create(T... xs) {
    List l;
    (l.items.push_back(xs), ...);
    return l;
  }
  const Value& operator[](const std::string& n) const {
    for (const Value& v : items)
      if (v.name == n) return v;
    throw std::out_of_range(n);
  }
};
[[noreturn]] inline void stop(const std::string& msg) { throw std::runtime_error(msg); }
}  // namespace Rcpp
