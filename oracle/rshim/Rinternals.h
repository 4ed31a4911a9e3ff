/* Rinternals.h -- stand-in for R's header (see R.h beside it).  The
 * reference's WDL polls for a user interrupt through R_ToplevelExec(
 * R_CheckUserInterrupt); outside R there is no interrupt to see, so the call
 * runs the function and reports success (Rboolean TRUE = 1). */
#ifndef RWIG_RSHIM_RINTERNALS_H
#define RWIG_RSHIM_RINTERNALS_H
typedef int Rboolean;

static inline void R_CheckUserInterrupt(void) {}

static inline Rboolean R_ToplevelExec(void (*fun)(void*), void* data) {
  fun(data);
  return 1;
}
#endif
