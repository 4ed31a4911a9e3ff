// selftest.cu -- device self-checks exposed through the C ABI for the test suite.
#include <algorithm>
#include "engine.h"
#include "fastexp.cuh"

namespace rwig {
namespace {
__global__ void exp_pair_kernel(const double* x, double* y_tbl, double* y_ref, int n) {
  __shared__ double tbl[64];
  load_exp_table(tbl);
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    y_tbl[i] = exp_tbl<1>(x[i], tbl);
    y_ref[i] = exp(x[i]);
  }
}
}  // namespace
}  // namespace rwig

extern "C" int rwig_selftest_exp(const double* x, double* y_engine, double* y_cuda, int n, void* stream) {
  using namespace rwig;
  if (!x || !y_engine || !y_cuda || n < 0) return set_error(RWIG_E_INVALID, "bad arguments");
  if (n == 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  exp_pair_kernel<<<std::min((n + 255) / 256, 4096), 256, 0, st>>>(x, y_engine, y_cuda, n);
  RWIG_CUDA_TRY(cudaGetLastError());
  RWIG_CUDA_TRY(cudaStreamSynchronize(st));
  return 0;
}
