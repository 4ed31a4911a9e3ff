/* rwig_b200.h -- C ABI of the B200 (sm_100a) engine for rwig's entropic-OT path.
 *
 * Drop-in replacement for the GPU entry points that rwig's Rcpp glue calls
 * (inst/include/cuda_interface.cuh:13-39), plus the log-domain and gradient
 * entries that the reference only has on the CPU.  Every function:
 *   - takes plain pointers, sizes and scalars (no C++ or framework types);
 *   - uses column-major FP64 arrays with R's layout (X[i + j*rows]);
 *   - never throws, never calls R, never prints;
 *   - returns >= 0 on success, namely the reference's `return_status`
 *     (0: err <= zero_tol, 1: max_iter reached, 2: otherwise; src/sinkhorn.cpp:88-95),
 *     or a negative RWIG_E_* code on failure, with a message in rwig_last_error().
 * Calls are blocking and serialised per device; they may be made from any host
 * thread.  Host-pointer entries copy inputs in and results out themselves; the
 * *_dev entries take device pointers (inputs resident in HBM) and a CUDA stream
 * (NULL: the engine's own stream, made to wait first for the work already
 * queued on the legacy default stream).
 */
#ifndef RWIG_B200_H
#define RWIG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define RWIG_B200_VERSION 100

#if defined(__GNUC__)
#define RWIG_API __attribute__((visibility("default")))
#else
#define RWIG_API
#endif

/* error codes (negative return values) */
#define RWIG_E_INVALID     (-1) /* bad argument (size, pointer, reg <= 0, ...) */
#define RWIG_E_CUDA        (-2) /* a CUDA runtime call failed */
#define RWIG_E_NODEVICE    (-3) /* no usable sm_100 device */
#define RWIG_E_NOMEM       (-4) /* device allocation failed or admission refused */
#define RWIG_E_TIMEOUT     (-5) /* a bounded device-side wait expired */
#define RWIG_E_UNSUPPORTED (-6) /* shape outside what this build supports */
#define RWIG_E_BUSY        (-7) /* server queue full */

/* Per-call report, filled by every solve (see rwig_last_report). */
typedef struct rwig_report {
  int iter;              /* iterations run */
  int status;            /* reference return_status (0/1/2) */
  double err;            /* stopping error of the last iteration */
  double marg_l1_row;    /* || P 1 - a ||_1     (barycenters: || U o KV - A ||_1) */
  double marg_l1_col;    /* || P^T 1 - b ||_1   (barycenters: 0) */
  double marg_l2_row;    /* || P 1 - a ||_2 */
  double marg_l2_col;    /* || P^T 1 - b ||_2 */
  double device_ms;      /* device time of the whole call (CUDA events) */
  double kernel_ms;      /* device time of the solver kernels (first launch to last) */
  double sweep_ms;       /* device time of the launches that ran scaled-form iterations */
  int sweep_iters;       /* iterations run by those launches */
  int fallback_events;   /* sweeps re-run with exact per-row / per-column minima
                            (log barycenter: 1 when the log-domain kernels ran) */
  int kernel_launches;   /* engine kernels launched by the call */
  int support_m;         /* rows kept after dropping zero-mass entries of a */
  int support_n;         /* columns kept after dropping zero-mass entries of b */
  double bary_norm;      /* barycenters: sum of the un-normalised barycenter b */
  double grad_ms;        /* Sinkhorn with withgrad: device time of the backward launch */
  double gemm_ms;        /* with option "profile.gemm" = 1: summed device time of the
                            call's INT8 tensor-core GEMM launches (CUDA events) */
  int gemm_launches;     /* those launches (0 when the timer was off) */
} rwig_report;

/* ---- context ---------------------------------------------------------- */
RWIG_API int rwig_init(int device);            /* optional; the first call initialises device 0 */
RWIG_API void rwig_shutdown(void);             /* frees all device memory held by the engine */
RWIG_API const char* rwig_last_error(void);    /* message of the last failure on this thread */
RWIG_API int rwig_version(void);
RWIG_API int rwig_last_report(rwig_report* out); /* report of the last call on this thread */
/* Engine options (process-wide):
 *   "log_sinkhorn.scaled": 1 (default) runs the log-Sinkhorn iterations after
 *       the first in stabilised scaling form, 0 keeps every iteration in the
 *       log domain (same results within rounding; slower);
 *   "log_sinkhorn.tau": absorption bound on |log u|, |log v| (default 100);
 *   "log_sinkhorn.l2_hot": share of each CTA's column groups of the scaled
 *       kernel copied with an L2 evict_last hint, the rest evict_first
 *       (default 0: all evict_first; negative: no hint);
 *   "batch.profile": 1 prints each batched Sinkhorn launch's busy, team-wait
 *       and claim time per CTA to stderr (default 0);
 *   "batch.strip_kb": target K strip per team member of a batched problem,
 *       at most 184 (default); strips up to that stay in shared memory;
 *   "batch.max_team": largest team of CTAs per batched problem (default:
 *       0.25 x the SM count for rwig_batch_sinkhorn_log*, 0.4 x for a
 *       server);
 *   "batch.resident_team": problems with M > 512 keep their K strips in
 *       shared memory when that takes at most this many CTAs (default 32),
 *       else stream strips of about "batch.stream_strip_kb" (default 1024)
 *       from memory every iteration;
 *   "batch.redundant_rows": teams with gp * M up to this (and M <= 4096)
 *       merge row sums redundantly in every member, one team barrier per
 *       iteration (default 16384);
 *   "batch.l2_keep_mb": streamed problems whose K is at most this many MB
 *       read it with an L2 evict_last hint (default 48);
 *   "batch.max_elems": problems with more elements go through the per-call
 *       path (default 2^26);
 *   "batch.backfill_us": how long the oldest waiting problem may be passed
 *       over by later ones that fit the free CTAs (default 5000);
 *   "wdl.infer_docs": documents per stacked-column chunk of WDL inference
 *       (default 1024);
 *   "wdl.int8": where the WDL products run: 1 (default) on the INT8 tensor
 *       cores for N >= 1024 (each FP64 product emulated exactly by 24
 *       modular integer products and CRT reconstruction), else on the FP64
 *       tensor cores; 2 on the INT8 tensor cores whenever N <= 8192; 0
 *       always on the FP64 tensor cores;
 *   "wdl.halves": 2 runs the two halves of the document batch of an
 *       INT8-path WDL gradient on two streams (same gradient bits), 1
 *       (default) on one stream;
 *   "oz.tile_m": rows per tile of the INT8 GEMM: 256 (default; one
 *       accumulator per CTA) or 128 (two accumulators, the MMAs of one tile
 *       beside the epilogue of the last);
 *   "wdl.checkpoint": k > 0 keeps the WDL forward state only every k-th
 *       iteration plus one segment of k iterations and recomputes the other
 *       segments during the backward (same gradient bits; 2 (L - k) more
 *       products; ceil(L/k) + 4k + 3 history slots of N x S D doubles
 *       instead of 4 (L + 1)); 0 (default) or k >= L keeps every
 *       iteration;
 *   "profile.gemm": 1 brackets each INT8 tensor-core GEMM launch of a call
 *       with CUDA events and reports their summed duration
 *       (rwig_report.gemm_ms, gemm_launches); 0 (default) off;
 *   "dgemm.kshape", "dgemm.tile": DMMA instruction shape (k = 4, 8 or 16)
 *       and tile height (0 automatic, 64, 128) of rwig_selftest_dgemm only;
 *   "barycenter.log_path": the log barycenter's route: 0 (default) the
 *       scaling form on K = exp(-C/reg) with a range check, re-run by the
 *       log-domain kernels when K has subnormal entries or the sums leave
 *       [1e-290, 1e290]; 1 the log-domain kernels always; -1 the scaling
 *       form only.
 * The batch.* options change team shapes and therefore the summation order
 * of a batched result (within rounding); a result is the same alone and in
 * any mix under the same options.  A NaN value clears the option (its
 * built-in default applies again). */
RWIG_API int rwig_set_option(const char* name, double value);
/* The value set for option `name`: 0 and *value, or 1 when the option is not
 * set (its built-in default applies); RWIG_E_INVALID for an unknown name. */
RWIG_API int rwig_get_option(const char* name, double* value);

/* ---- vanilla Sinkhorn --------------------------------------------------
 * Replaces cuda_sinkhorn_vanilla (inst/include/cuda_interface.cuh:13-18,
 * src/cuda_sinkhorn.cu:181) called from sinkhorn_vanilla_cuda (src/sinkhorn.cpp:51),
 * with the semantics of the CPU path Sinkhorn::compute_vanilla
 * (src/sinkhorn_impl_vanilla.cpp:18): zero masses dropped, `err >= zero_tol`
 * continues, u, v zero off the support.  a: M, b: N, C: M x N.  Outputs (any
 * may be NULL): P (M x N), grad_a (M, needs withgrad), u (M), v (N), loss.
 * grad_a is the unrolled backward Sinkhorn::_bwd_vanilla (:169-213), zero off
 * the support; it needs at most 8192 non-zero entries of a and keeps every
 * iteration's scalings on the device (8 (max_iter + 2)(M + N) bytes, at most
 * 32 GiB), else RWIG_E_UNSUPPORTED.
 */
RWIG_API int rwig_sinkhorn_vanilla(double* P, double* grad_a, double* u, double* v, double* loss,
                                   int* iter, double* err, const double* a, const double* b,
                                   const double* C, int M, int N, double reg, int withgrad,
                                   int max_iter, double zero_tol);

/* Same on device pointers (see rwig_sinkhorn_log_dev). */
RWIG_API int rwig_sinkhorn_vanilla_dev(double* P, double* grad_a, double* u, double* v, double* loss,
                                       int* iter, double* err, const double* a, const double* b,
                                       const double* C, int M, int N, double reg, int withgrad,
                                       int max_iter, double zero_tol, void* stream);

/* ---- log-stabilised Sinkhorn ------------------------------------------
 * Replaces the CPU-only Sinkhorn::compute_log (src/sinkhorn_impl_log.cpp:225)
 * reached from sinkhorn_log_cpp (src/sinkhorn.cpp:142); the reference has no
 * GPU entry for it (inst/include/cuda_interface.cuh:41, "TODO").
 * a: M, b: N, C: M x N.  Outputs (any may be NULL): P (M x N), grad_a (M,
 * needs withgrad), f (M), g (N; -inf off the support, as :267-270), loss.
 * grad_a is the unrolled backward Sinkhorn::_bwd_log (:379-520), zero off the
 * support; the forward of a gradient call runs every iteration in the log
 * domain, with the limits of rwig_sinkhorn_vanilla's gradient.
 */
RWIG_API int rwig_sinkhorn_log(double* P, double* grad_a, double* f, double* g, double* loss,
                      int* iter, double* err, const double* a, const double* b,
                      const double* C, int M, int N, double reg, int withgrad,
                      int max_iter, double zero_tol);

/* Same, with every array a device pointer (C with leading dimension M) and the
 * work queued on `stream` (a cudaStream_t, NULL = the engine's stream).
 * loss / iter / err are host pointers, written before the call returns. */
RWIG_API int rwig_sinkhorn_log_dev(double* P, double* grad_a, double* f, double* g, double* loss,
                          int* iter, double* err, const double* a, const double* b,
                          const double* C, int M, int N, double reg, int withgrad,
                          int max_iter, double zero_tol, void* stream);

/* ---- Wasserstein barycenters -------------------------------------------
 * rwig_barycenter_parallel replaces cuda_barycenter_parallel
 * (inst/include/cuda_interface.cuh:20-26, src/cuda_barycenter.cu:268) called
 * from barycenter_parallel_cuda (src/barycenter.cpp:67), with the semantics of
 * Barycenter::compute_parallel (src/barycenter_impl_parallel.cpp:19);
 * rwig_barycenter_log is the GPU form of the CPU-only Barycenter::compute_log
 * (src/barycenter_impl_log.cpp:23, reached from src/barycenter.cpp:168).
 * A: M x S histograms, w: S weights, C: M x N cost, b_ext: N (only read when
 * withgrad).  Outputs (any may be NULL): parallel U (M x S), V (N x S); log
 * F (M x S), G (N x S); b (N, normalised); grad_A (M x S), grad_w (S), loss
 * (need withgrad).  S <= 64.
 */
RWIG_API int rwig_barycenter_parallel(double* U, double* V, double* b, double* grad_A, double* grad_w,
                                      double* loss, int* iter, double* err, const double* A,
                                      const double* w, const double* C, const double* b_ext, int M,
                                      int N, int S, double reg, int withgrad, int max_iter,
                                      double zero_tol);
RWIG_API int rwig_barycenter_log(double* F, double* G, double* b, double* grad_A, double* grad_w,
                                 double* loss, int* iter, double* err, const double* A, const double* w,
                                 const double* C, const double* b_ext, int M, int N, int S, double reg,
                                 int withgrad, int max_iter, double zero_tol);
/* Same on device pointers, work queued on `stream`; loss / iter / err are host pointers. */
RWIG_API int rwig_barycenter_parallel_dev(double* U, double* V, double* b, double* grad_A,
                                          double* grad_w, double* loss, int* iter, double* err,
                                          const double* A, const double* w, const double* C,
                                          const double* b_ext, int M, int N, int S, double reg,
                                          int withgrad, int max_iter, double zero_tol, void* stream);
RWIG_API int rwig_barycenter_log_dev(double* F, double* G, double* b, double* grad_A, double* grad_w,
                                     double* loss, int* iter, double* err, const double* A,
                                     const double* w, const double* C, const double* b_ext, int M,
                                     int N, int S, double reg, int withgrad, int max_iter,
                                     double zero_tol, void* stream);

/* Many independent barycenter problems in one call.  No counterpart in the
 * reference (one barycenter per call).  Each problem has its own sizes,
 * method (0 parallel, 1 log), regularisation and iteration control, and the
 * argument meaning of rwig_barycenter_*_dev; all arrays are device pointers
 * and the outputs X1 (U or F), X2 (V or G), b, grad_A, grad_w may be NULL.
 * Problems with a fixed iteration count (zero_tol <= 0) are queued side by
 * side on streams forked from `stream` (NULL = the engine's stream), so their
 * small products share the GPU; problems with a stopping test (zero_tol > 0)
 * read their error on the host every iteration and run one after another.
 * out[i]: loss, err, iter and status (0 converged, 1 max_iter, 2 other, < 0
 * an error of that problem alone).  Each result equals the single call's on
 * the same problem bitwise.  Returns 0 once every output is written, or a
 * negative error. */
typedef struct rwig_bary_problem {
  const double* A;     /* M x S */
  const double* w;     /* S */
  const double* C;     /* M x N */
  const double* b_ext; /* N (withgrad) */
  int M, N, S;
  double reg;
  int method;   /* 0 parallel, 1 log */
  int withgrad;
  int max_iter;
  double zero_tol;
  double* X1;     /* U (parallel) or F (log), M x S */
  double* X2;     /* V or G, N x S */
  double* b;      /* N */
  double* grad_A; /* M x S */
  double* grad_w; /* S */
} rwig_bary_problem;

typedef struct rwig_bary_result {
  double loss, err;
  int iter, status;
} rwig_bary_result;

RWIG_API int rwig_batch_barycenter_dev(const rwig_bary_problem* probs, int count, rwig_bary_result* out,
                                       void* stream);

/* Wasserstein dictionary learning.
 *
 * rwig_wdl replaces cuda_wdl (inst/include/cuda_interface.cuh:31-39, called
 * from src/wdl.cpp:76) with the same argument meaning, host pointers: Y
 * (N x M documents), C (N x N cost); outputs A (N x S topics), W (S x M
 * weights) and Yhat (N x M barycenters of the documents; NULL skips the
 * inference).  max_iter is the fixed iteration count L of each training
 * batch and the iteration cap of the inference barycenters (tolerance
 * zero_tol); B batch size, E epochs; opt 0 SGD, 1 Adam, 2 AdamW with eta,
 * gamma (AdamW decay), beta1, beta2, eps.  Added arguments: Alpha0 (N x S)
 * and Lambda0 (S x M) initial logits (NULL: N(0,1) draws from mt19937(seed),
 * Alpha first, as the reference GPU path does), and max_steps (> 0: stop
 * after that many batches).  S <= 64.  Returns 0 or a negative error.
 *
 * rwig_wdl_batch_grad is one batched step (WassersteinDictionaryLearning::
 * _train_batch_batched, src/wdl_impl.cpp:87-247; wdl_batch,
 * src/cuda_wdl.cu:385): the batch-mean gradients g_Alpha (N x S) and
 * g_lambda (S) of the D documents Y_B (N x D) with weights W_B (S x D) under
 * topics A (N x S), after the softmax Jacobians.  mode 0: K_or_C is the
 * Gibbs kernel K (N x N); mode 1: it is C and K = exp(-C/reg).  L fixed
 * iterations.  The _dev form takes device pointers and a stream. */
RWIG_API int rwig_wdl(double* A, double* W, double* Yhat, const double* Y, const double* C, int N, int M,
                      int S, double reg, int max_iter, double zero_tol, int B, int E, int opt, double eta,
                      double gamma, double beta1, double beta2, double eps, int seed, int verbose,
                      const double* Alpha0, const double* Lambda0, int max_steps);
RWIG_API int rwig_wdl_batch_grad(double* g_Alpha, double* g_lambda, const double* A, const double* W_B,
                                 const double* Y_B, const double* K_or_C, int N, int S, int D, double reg,
                                 int L, int mode);
RWIG_API int rwig_wdl_batch_grad_dev(double* g_Alpha, double* g_lambda, const double* A,
                                     const double* W_B, const double* Y_B, const double* K_or_C, int N,
                                     int S, int D, double reg, int L, int mode, void* stream);
/* One optimizer step of WDL training on device buffers, the step rwig_wdl
 * takes after each batch (src/wdl_impl.cpp:332-336, inst/include/optimizer.hpp:72-99,
 * src/cuda_optimizer.cu:64): Alpha (N x S) -= update(g_Alpha); every column
 * of Lambda (S x M) -= update(g_lambda) (the batch's Lambda gradient applied
 * to all documents, wdl_impl.cpp:246); then A = column softmax of Alpha and
 * W = column softmax of Lambda.  opt 0 SGD, 1 Adam, 2 AdamW (gamma the
 * decay); mA, vA (N x S) and mL, vL (S x M) are the moments (zero before the
 * first step); step >= 1 counts the steps taken, for the bias corrections.
 * With the same inputs every rank of a data-parallel run takes the same
 * step (the data-parallel training of rwig_b200/api.py). */
RWIG_API int rwig_wdl_update_dev(double* Alpha, double* Lambda, double* A, double* W, double* mA, double* vA,
                                 double* mL, double* vL, const double* g_Alpha, const double* g_lambda, int N,
                                 int S, int M, int opt, double eta, double gamma, double beta1, double beta2,
                                 double eps, int step, void* stream);

/* ---- batched log-Sinkhorn ---------------------------------------------
 * Many independent problems with the semantics of rwig_sinkhorn_log in one
 * call (no counterpart in the reference, whose GPU path solves one problem
 * per call; the semantics are those of Sinkhorn::compute_log,
 * src/sinkhorn_impl_log.cpp:225).  Problems with M <= 8192 and M*N <= 4 Mi
 * are iterated together in one cooperative launch, each on its own team of
 * CTAs (results bitwise identical whatever else is in the batch); larger
 * ones, and any problem the scaling form cannot treat (a zero mass, scalings
 * beyond e^650), go through the per-call path.  Host pointers for rwig_batch_sinkhorn_log, device pointers for the
 * _dev form.  P may be NULL.  The call returns 0 or a negative error for the
 * whole batch; each out[i].status is the problem's own status (0/1/2, or a
 * negative RWIG_E_* for a rejected problem). */
typedef struct rwig_problem {
  const double* a; /* M */
  const double* b; /* N */
  const double* C; /* M x N, column-major */
  int M, N;
  double reg;
  int max_iter;
  double zero_tol;
  double* P;       /* M x N plan or NULL */
  double* f;       /* M potentials */
  double* g;       /* N potentials */
  /* Instead of C (C = NULL): source points X (M x d) and target points Y
   * (N x d), column-major; the engine builds C_ij = sum_k (x_ik - y_jk)^2
   * (ascending k, every operation rounded separately) divided by its
   * maximum, on the device.  Batched and served problems only. */
  const double* X;
  const double* Y;
  int d;
} rwig_problem;

typedef struct rwig_result {
  double loss, err;
  int iter, status;
  double marg_l1_row, marg_l1_col;
  double device_us; /* device time of this problem's solve (start to end on its CTA, or the per-call solve) */
  int path;        /* 0: batched kernel, 1: per-call path */
  int reserved;
} rwig_result;

RWIG_API int rwig_batch_sinkhorn_log(const rwig_problem* probs, int count, rwig_result* out);

/* ---- serving (continuous batching of log-Sinkhorn requests) -------------
 * No counterpart in the reference.  A server keeps one service launch of the
 * batched kernel running while requests arrive: rwig_server_submit copies a
 * request (host pointers; M <= 8192) to the device and publishes it to the
 * running kernel, where free CTAs form its team as soon as enough are free
 * and solve it beside the others; rwig_server_poll returns 1 once the request is
 * finished (f, g and P copied to the pointers given at submit; out filled),
 * 0 while it runs.  submit returns the request's ticket (>= 0; tickets
 * number the requests in submission order), or RWIG_E_BUSY when admitting it
 * would exceed the device-memory budget or the request submitted 512 tickets
 * earlier has not been collected yet (at most 512 requests are out at once;
 * their descriptor slots are reused while the launch runs) -- poll and
 * retry.  The kernel ends after
 * idle_ms without work and is restarted by the next submit or poll; while it
 * runs it holds every SM (other work on the GPU waits), so idle_ms trades the
 * restart of the launch (tens of microseconds) against that.
 * Requests are allocated from a memory pool of the server's own, which keeps
 * what it maps until rwig_server_destroy; create maps the whole budget up
 * front (at most 80 % of the free device memory; beyond that the pool grows
 * on demand, which waits for the running launch).
 * Results are bitwise those of rwig_batch_sinkhorn_log for the same problem
 * under the same "batch.max_team" (set explicitly: the two defaults differ).
 * One thread drives a server. */
typedef struct rwig_server rwig_server;
RWIG_API int rwig_server_create(rwig_server** out, double mem_budget_bytes, double idle_ms);
RWIG_API int rwig_server_submit(rwig_server* server, const rwig_problem* prob);
RWIG_API int rwig_server_poll(rwig_server* server, int ticket, rwig_result* out);
RWIG_API int rwig_server_destroy(rwig_server* server);
RWIG_API int rwig_batch_sinkhorn_log_dev(const rwig_problem* probs, int count, rwig_result* out,
                                         void* stream);

/* Self-check of the engine's internal exponential (no counterpart in the
 * reference): evaluates it and CUDA's exp on n device doubles x, writing
 * y_engine and y_cuda (device).  Used by the test suite to bound its error. */
RWIG_API int rwig_selftest_exp(const double* x, double* y_engine, double* y_cuda, int n, void* stream);

/* Self-check of the engine's FP64 tensor-core GEMM (no counterpart in the
 * reference): Y (Mo x S, ldy) = op(K) X with op(K) = K (trans = 0) or K^T
 * (trans = 1), K column-major with even ldk, X (Kd x S, ldx); all device
 * pointers.  splits <= 0 picks the split-K count.  Returns the split count. */
RWIG_API int rwig_selftest_dgemm(const double* K, long long ldk, int trans, int Mo, int Kd, int S,
                                 const double* X, long long ldx, double* Y, long long ldy, int splits,
                                 void* stream);

/* Self-check of the INT8 tensor-core GEMM behind the emulated FP64 products
 * (no counterpart in the reference): D (M x N, column-major int32) = A B^T for
 * A (M x Kd) and B (N x Kd) row-major int8 (values as signed char), Kd <=
 * 65536; all device pointers. */
RWIG_API int rwig_selftest_i8gemm(const signed char* A, const signed char* B, int M, int N, int Kd, int* D,
                                  void* stream);

/* Self-check of the FP64 product emulated on the INT8 tensor cores (no
 * counterpart in the reference): Y (n x W, ldy) = op(K) X with op(K) = K
 * (trans = 0) or K^T (trans = 1), K n x n (ldk), X n x W (ldx), n <= 8192;
 * all device pointers.  Returns 0 or a negative error. */
RWIG_API int rwig_selftest_ozaki(const double* K, long long ldk, int trans, int n, const double* X, long long ldx,
                                 int W, double* Y, long long ldy, void* stream);

/* Allocation-free log-Sinkhorn.  No counterpart in the reference: it exists for
 * callers that cannot let a library allocate device memory (a host framework
 * that owns the GPU's memory pool, a process under a hard device-memory quota,
 * a serving loop that must not stall on cudaMalloc / cudaFree).  Same solver
 * and results as rwig_sinkhorn_log_dev, but all scratch lives in a fixed
 * ~10 MB block inside the library image, held by every GPU that loads the
 * library until exit; the call makes no device allocation.
 * Limits: M, N <= 4096, a and b strictly positive, M even, C 16-byte aligned
 * (column-major, leading dimension M); anything else returns
 * RWIG_E_UNSUPPORTED; a negative max_iter returns RWIG_E_INVALID.  P, f, g
 * are device outputs (any may be NULL); loss, iter, err are host pointers;
 * `stream` is a cudaStream_t (NULL: legacy default stream).  The call waits
 * for its work on `stream` before it returns (loss, iter and err are read
 * back to the host).  All calls on a device share the block: calls that overlap
 * on the GPU race and must be serialised by the caller.  The first call on a
 * device looks up the block's address; make it before any stream capture. */
RWIG_API int rwig_sinkhorn_log_noalloc(double* P, double* f, double* g, double* loss, int* iter,
                                       double* err, const double* a, const double* b,
                                       const double* C, int M, int N, double reg, int max_iter,
                                       double zero_tol, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RWIG_B200_H */
