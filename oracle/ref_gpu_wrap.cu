// ref_gpu_wrap.cu -- C-linkage entry points onto rwig's own GPU code, which
// the Makefile's `ref` target compiles from the reference's sources into
// oracle/_ref/:
//   * cuda_sinkhorn_vanilla (src/cuda_sinkhorn.cu:181) and
//     cuda_barycenter_parallel (src/cuda_barycenter.cu:268), declared in
//     inst/include/cuda_interface.cuh:13-26;
//   * cuda_wdl (src/cuda_wdl.cu:539, cuda_interface.cuh:31-39), the whole
//     GPU training + inference;
//   * wdl_batch (src/cuda_wdl.cu:385), the unrolled batched WDL gradient the
//     training loop calls once per batch (external linkage, no header: its
//     prototype is restated below with the definition's parameter list).
// src/cuda_wdl.cu includes R's headers for printing and interrupt checks;
// oracle/rshim/ supplies stand-ins for those four functions.  Test and
// benchmark infrastructure only: the tests compare the engine with these, and
// bench.py times them beside the engine; nothing in the engine links them.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <vector>

#include "cuda_interface.cuh"
#include "cuda_kernels.cuh"

void wdl_batch(double* g_Alpha, double* g_lambda, double* g_Lambda, double* A, double* W, double* Y, double* K,
               double* UB, double* VB, double* bB, double* KVB, double* KTUB, double* UB_hist, double* VB_hist,
               double* bB_hist, double* KVB_hist, double* KTUB_hist, double* UBbar, double* VBbar, double* bBbar,
               double* ABbar, double* wBbar, int batch_id, int B, int M, int N, int S, int max_iter,
               cudaStream_t& stream, cublasHandle_t& handle);

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

extern "C" void ref_gpu_wdl(double* A, double* W, double* Yhat, const double* Y, const double* C, int N, int M,
                            int S, double reg, int max_iter, double zero_tol, int B, int E, int opt, double eta,
                            double gamma, double beta1, double beta2, double eps, int seed) {
  cuda_wdl(A, W, Yhat, Y, C, N, M, S, reg, max_iter, zero_tol, B, E, opt, eta, gamma, beta1, beta2, eps, seed,
           false);
}

// One wdl_batch call on a batch of D documents (batch 0 of a corpus of D
// documents with batch size D, so the reference takes all D): host inputs A
// (N x S, topics after softmax), W_B (S x D), Y_B (N x D), K_or_C (N x N: the
// Gibbs kernel when mode == 0, the cost when mode == 1, turned into
// exp(-C/reg) by the reference's update_K); outputs g_Alpha (N x S), g_lambda
// (S).  The call is repeated `reps` times (>= 1) on the same inputs;
// *ms_out receives the mean device time of one wdl_batch call (CUDA events
// on its stream).  Returns 0, or the CUDA error code of a failed
// allocation or copy.
extern "C" int ref_gpu_wdl_batch_grad(double* g_Alpha, double* g_lambda, const double* A, const double* W_B,
                                      const double* Y_B, const double* K_or_C, int N, int S, int D, double reg,
                                      int L, int mode, int reps, float* ms_out) {
  const size_t NS = (size_t)N * S, NSD = NS * D, ND = (size_t)N * D, SD = (size_t)S * D, H = (size_t)L + 1;
  struct Buf {
    double** p;
    size_t n;
  };
  double *dA = nullptr, *dW = nullptr, *dY = nullptr, *dK = nullptr, *gA = nullptr, *gl = nullptr, *gL = nullptr;
  double *UB = nullptr, *VB = nullptr, *bB = nullptr, *KVB = nullptr, *KTUB = nullptr;
  double *UBh = nullptr, *VBh = nullptr, *bBh = nullptr, *KVBh = nullptr, *KTUBh = nullptr;
  double *UBbar = nullptr, *VBbar = nullptr, *bBbar = nullptr, *ABbar = nullptr, *wBbar = nullptr;
  std::vector<Buf> bufs = {{&dA, NS},        {&dW, SD},          {&dY, ND},         {&dK, (size_t)N * N},
                           {&gA, NS},        {&gl, (size_t)S},   {&gL, SD},         {&UB, NSD},
                           {&VB, NSD},       {&bB, ND},          {&KVB, NSD},       {&KTUB, NSD},
                           {&UBh, H * NSD},  {&VBh, H * NSD},    {&bBh, H * ND},    {&KVBh, H * NSD},
                           {&KTUBh, H * NSD}, {&UBbar, NSD},     {&VBbar, NSD},     {&bBbar, ND},
                           {&ABbar, NSD},    {&wBbar, SD}};
  cudaStream_t stream = nullptr;
  cublasHandle_t handle = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t rc = cudaSuccess;
  float total = 0.f;
  if (reps < 1) reps = 1;
  for (Buf& b : bufs) {
    rc = cudaMalloc((void**)b.p, sizeof(double) * b.n);
    if (rc != cudaSuccess) goto done;
  }
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  cublasCreate(&handle);
  cublasSetStream(handle, stream);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  if ((rc = cudaMemcpyAsync(dA, A, sizeof(double) * NS, cudaMemcpyHostToDevice, stream)) != cudaSuccess) goto done;
  if ((rc = cudaMemcpyAsync(dW, W_B, sizeof(double) * SD, cudaMemcpyHostToDevice, stream)) != cudaSuccess) goto done;
  if ((rc = cudaMemcpyAsync(dY, Y_B, sizeof(double) * ND, cudaMemcpyHostToDevice, stream)) != cudaSuccess) goto done;
  if ((rc = cudaMemcpyAsync(dK, K_or_C, sizeof(double) * N * N, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
    goto done;
  if (mode == 1) update_K(dK, N, N, reg, stream);
  for (int r = 0; r < reps; ++r) {
    float ms = 0.f;
    cudaEventRecord(e0, stream);
    wdl_batch(gA, gl, gL, dA, dW, dY, dK, UB, VB, bB, KVB, KTUB, UBh, VBh, bBh, KVBh, KTUBh, UBbar, VBbar, bBbar,
              ABbar, wBbar, 0, D, D, N, S, L, stream, handle);
    cudaEventRecord(e1, stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    total += ms;
  }
  if ((rc = cudaMemcpyAsync(g_Alpha, gA, sizeof(double) * NS, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    goto done;
  if ((rc = cudaMemcpyAsync(g_lambda, gl, sizeof(double) * S, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    goto done;
  rc = cudaStreamSynchronize(stream);
  if (rc == cudaSuccess) rc = cudaGetLastError();
  if (ms_out) *ms_out = total / reps;
done:
  if (stream) cudaStreamSynchronize(stream);
  for (Buf& b : bufs)
    if (*b.p) cudaFree(*b.p);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (handle) cublasDestroy(handle);
  if (stream) cudaStreamDestroy(stream);
  return (int)rc;
}
