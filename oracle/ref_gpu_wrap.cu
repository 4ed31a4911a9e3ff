// ref_gpu_wrap.cu -- C-linkage entry points onto rwig's own GPU Sinkhorn and
// parallel barycenter (src/cuda_sinkhorn.cu:181 cuda_sinkhorn_vanilla,
// src/cuda_barycenter.cu:268 cuda_barycenter_parallel, declared in
// inst/include/cuda_interface.cuh:13-26), which the Makefile's `ref` target
// compiles from the reference's sources into oracle/_ref/.  Test and
// benchmark infrastructure only: bench.py times the reference GPU path beside
// the engine; nothing in the engine links it.
#include "cuda_interface.cuh"

extern "C" void ref_gpu_sinkhorn_vanilla(double* P, double* grad_a, double* u, double* v, double* loss,
                                         int* iter_out, double* err_out, const double* a, const double* b,
                                         const double* C, int m, int n, double reg, int withgrad, int max_iter,
                                         double zero_tol) {
  cuda_sinkhorn_vanilla(P, grad_a, u, v, loss, iter_out, err_out, a, b, C, m, n, reg, withgrad != 0, max_iter,
                        zero_tol);
}

extern "C" void ref_gpu_barycenter_parallel(double* U, double* V, double* b, double* grad_A, double* grad_w,
                                            double* loss, int* iter_out, double* err_out, const double* A,
                                            const double* w, const double* C, const double* b_ext, int M, int N,
                                            int S, double reg, int withgrad, int max_iter, double zero_tol) {
  cuda_barycenter_parallel(U, V, b, grad_A, grad_w, loss, iter_out, err_out, A, w, C, b_ext, M, N, S, reg,
                           withgrad != 0, max_iter, zero_tol);
}
