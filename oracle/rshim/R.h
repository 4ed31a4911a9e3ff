/* R.h -- stand-in for R's header, used only to compile the reference's GPU
 * WDL (src/cuda_wdl.cu) outside R for the parity tests and the reference
 * timing.  That file uses two of R's printing functions; here they print to
 * stdout / stderr.  Test infrastructure only. */
#ifndef RWIG_RSHIM_R_H
#define RWIG_RSHIM_R_H
#include <cstdarg>
#include <cstdio>

static inline void Rprintf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vprintf(fmt, ap);
  va_end(ap);
}

static inline void REprintf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vfprintf(stderr, fmt, ap);
  va_end(ap);
}
#endif
