// sk_host.h -- host-side interface of the scaled-form log-Sinkhorn iterations
// (sinkhorn_scaled.cu), used by the log-Sinkhorn driver (sinkhorn_log.cu).
#pragma once

#include <cuda_runtime.h>

#include "engine.h"

namespace rwig {

enum { kScaledRunning = 0, kScaledFinished = 1, kScaledAbsorb = 2, kScaledUnsafe = 3 };

struct ScaledParams {
  const double* K;  // absorbed kernel, reduced m x n, leading dimension ldk
  long long ldk;
  const double* a;
  const double* b;
  const double* loga;
  const double* logb;
  int m, n, G;
  double eps, inv_eps, tol, tau;
  int iter0, max_iter;
  double err0;
  double* u0;  // current u (all ones after an absorption); ping-pong with u1
  double* u1;
  const double* ft;  // absorbed potentials f~, g~
  const double* gt;
  double* rowp;  // [G][m]
  double* part;  // [G][8]
  unsigned* ctrl;
  double* res;       // iter, err, status
  double* f_state;   // exit state (reduced)
  double* g_state;
  int ncol_max;
  double l2_hot_fraction;  // share of each CTA's column groups kept in L2 (evict_last); < 0: no hint
  int vanilla_init;         // vanilla mode: start with the pass u = a / (K 1)
  // vanilla mode, optional: the scalings of every iteration for the gradient,
  // u_l at uh[l * m] (l = 1..L+1) and v_l at vh[l * n] (l = 1..L)
  double* uh;
  double* vh;
};

int launch_scaled(Context* ctx, ScaledParams& p, cudaStream_t st, bool vanilla);
int launch_uv_to_potentials(Context* ctx, const double* u, const double* v, int m, int n, double eps,
                            double* f, double* g, cudaStream_t st);
int launch_absorb(Context* ctx, const double* C, long long ldc, const double* ft, const double* gt, int m,
                  int n, double inv_eps, double* K, cudaStream_t st);
int launch_fill_ones(Context* ctx, double* x, int n, cudaStream_t st);

// The per-call Sinkhorn driver (sinkhorn_log.cu) on device inputs: vanilla
// (f, g receive u, v) or log-stabilised (f, g the potentials).  Returns the
// reference status (0, 1, 2) or a negative engine error; fills report().
// Unrolled gradient of the Sinkhorn loss w.r.t. a from the forward's history
// (sinkhorn_grad.cu); grad_a has M entries, zero off the support rows ridx.
int sinkhorn_grad(Context* ctx, cudaStream_t st, bool vanilla, const double* C, const double* K, long long ldc,
                  const double* a, const double* b, const double* loga, const double* logb, const double* fh,
                  const double* gh, int m, int n, int L, double eps, const int* ridx, int M, double out_scale,
                  double* grad_a, int* launches);

int sinkhorn_device(Context* ctx, cudaStream_t st, bool vanilla, double* P, double* grad_a, double* f, double* g,
                    double* loss, int* iter, double* err, const double* a, const double* b, const double* C,
                    int M, int N, double reg, int withgrad, int max_iter, double zero_tol);

}  // namespace rwig
