// barycenter.h -- device-pointer driver of the barycenters (barycenter.cu),
// shared with the WDL inference.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "engine.h"

namespace rwig {
namespace bary {

// All pointers on the device; outputs may be null.  X1, X2: U, V (parallel)
// or F, G (log); b: normalised barycenter.  Returns the status code (0, 1, 2)
// or a negative engine error.
int run(Context* ctx, cudaStream_t st, bool logdomain, double* X1, double* X2, double* b, double* gradA,
        double* gradw, double* loss, int* iter_out, double* err_out, const double* A, const double* w,
        const double* C, const double* bext, int M, int N, int S, double reg, int withgrad, int max_iter,
        double tol);

// The log barycenter in the log domain (barycenter_log.cu), same arguments
// and outputs as run() with logdomain; *launches += the kernels launched.
int run_log(Context* ctx, cudaStream_t st, double* X1, double* X2, double* b, double* gradA, double* gradw,
            double* loss, int* iter_out, double* err_out, const double* A, const double* w, const double* C,
            const double* bext, int M, int N, int S, double reg, int withgrad, int max_iter, double tol,
            int* launches);

// Largest eigenvalue of a symmetric positive semi-definite n x n matrix.
double lambda_max(std::vector<double> G, int n);

}  // namespace bary
}  // namespace rwig
