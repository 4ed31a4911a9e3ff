// context.cu -- per-device context, scratch arena and the error / report
// entry points of the C ABI.
#include <cstdio>
#include <cmath>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <string>

#include "engine.h"

namespace rwig {

namespace {
thread_local std::string t_last_error;
thread_local rwig_report t_report;

std::mutex g_ctx_mu;
std::vector<std::unique_ptr<Context>> g_ctx;  // indexed by device

int init_device(int dev, Context** out) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return set_error(RWIG_E_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= ndev) return set_error(RWIG_E_INVALID, "device index out of range");
  if ((int)g_ctx.size() < ndev) g_ctx.resize(ndev);
  if (!g_ctx[dev]) {
    auto c = std::make_unique<Context>();
    c->device = dev;
    RWIG_CUDA_TRY(cudaSetDevice(dev));
    cudaDeviceProp prop;
    RWIG_CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10)
      return set_error(RWIG_E_NODEVICE, "device is not sm_100 class (this build targets sm_100a)");
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = (int)prop.sharedMemPerBlockOptin;
    RWIG_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    RWIG_CUDA_TRY(cudaEventCreate(&c->ev0));
    RWIG_CUDA_TRY(cudaEventCreate(&c->ev1));
    RWIG_CUDA_TRY(cudaEventCreate(&c->evk));
    RWIG_CUDA_TRY(cudaEventCreate(&c->evs0));
    RWIG_CUDA_TRY(cudaEventCreate(&c->evs1));
    RWIG_CUDA_TRY(cudaEventCreateWithFlags(&c->evfork, cudaEventDisableTiming));
    RWIG_CUDA_TRY(cudaEventCreateWithFlags(&c->evlegacy, cudaEventDisableTiming));
    RWIG_CUDA_TRY(cudaEventCreateWithFlags(&c->evjoin, cudaEventDisableTiming));
    g_ctx[dev] = std::move(c);
  }
  *out = g_ctx[dev].get();
  return 0;
}
}  // namespace

namespace {
std::mutex g_opt_mu;
std::map<std::string, double> g_opts;
const char* const kOptionNames[] = {"log_sinkhorn.scaled", "log_sinkhorn.tau", "log_sinkhorn.l2_hot", "batch.profile",
                                   "batch.strip_kb", "batch.max_team", "batch.redundant_rows",
                                   "batch.l2_keep_mb", "batch.max_elems", "batch.resident_team",
                                   "batch.stream_strip_kb", "batch.backfill_us",
                                   "wdl.infer_docs", "wdl.checkpoint", "wdl.int8", "wdl.halves", "dgemm.kshape", "dgemm.tile", "barycenter.log_path", "oz.tile_m", "profile.gemm"};
}  // namespace

double option(const char* name, double dflt) {
  std::lock_guard<std::mutex> lk(g_opt_mu);
  auto it = g_opts.find(name);
  return it == g_opts.end() ? dflt : it->second;
}

int set_error(int code, const std::string& msg) {
  t_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
  t_last_error = buf;
  return e == cudaErrorMemoryAllocation ? RWIG_E_NOMEM : RWIG_E_CUDA;
}

rwig_report& report() { return t_report; }

cudaStream_t call_stream(Context* ctx, void* stream) {
  if (stream) return (cudaStream_t)stream;
  if (cudaEventRecord(ctx->evlegacy, cudaStreamLegacy) == cudaSuccess)
    (void)cudaStreamWaitEvent(ctx->stream, ctx->evlegacy, 0);
  (void)cudaGetLastError();
  return ctx->stream;
}

int gemm_timer_begin(Context* ctx) {
  ctx->gemm_ev_used = 0;
  ctx->gemm_timing = option("profile.gemm", 0.0) == 1.0;
  if (ctx->gemm_timing && ctx->gemm_ev.empty()) {
    ctx->gemm_ev.resize(2 * Context::kTimedGemms, nullptr);
    for (cudaEvent_t& e : ctx->gemm_ev) RWIG_CUDA_TRY(cudaEventCreate(&e));
  }
  return 0;
}

bool gemm_timer_mark(Context* ctx, cudaStream_t st) {
  if (!ctx->gemm_timing || ctx->gemm_ev_used >= (int)ctx->gemm_ev.size()) return false;
  return cudaEventRecord(ctx->gemm_ev[ctx->gemm_ev_used++], st) == cudaSuccess;
}

void gemm_timer_end(Context* ctx, double* ms_out, int* n_out) {
  double ms = 0.0;
  int n = 0;
  for (int k = 0; ctx->gemm_timing && k + 1 < ctx->gemm_ev_used; k += 2) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, ctx->gemm_ev[k], ctx->gemm_ev[k + 1]) == cudaSuccess) {
      ms += t;
      ++n;
    }
  }
  (void)cudaGetLastError();
  *ms_out = ms;
  *n_out = n;
  ctx->gemm_timing = false;
  ctx->gemm_ev_used = 0;
}

void reset_report() {
  std::memset(&t_report, 0, sizeof(t_report));
}

Context* get_context() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  Context* c = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (dev < (int)g_ctx.size() && g_ctx[dev]) return g_ctx[dev].get();
  }
  if (init_device(dev, &c) != 0) return nullptr;
  return c;
}

cudaStream_t side_stream(Context* ctx, int i) {
  cudaStream_t& q = ctx->side[i];
  if (!q && cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking) != cudaSuccess) {
    (void)cudaGetLastError();
    q = nullptr;
  }
  return q;
}

void* scratch(Context* ctx, int k, size_t bytes) {
  if ((int)ctx->slots.size() <= k) {
    ctx->slots.resize(k + 1, nullptr);
    ctx->slot_bytes.resize(k + 1, 0);
  }
  if (ctx->slot_bytes[k] >= bytes && ctx->slots[k]) return ctx->slots[k];
  if (ctx->slots[k]) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->slots[k]);
    ctx->slots[k] = nullptr;
    ctx->slot_bytes[k] = 0;
  }
  size_t want = bytes < 256 ? 256 : bytes;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cuda_fail(e, "cudaMalloc(scratch)");
    return nullptr;
  }
  ctx->slots[k] = p;
  ctx->slot_bytes[k] = want;
  return p;
}

}  // namespace rwig

using namespace rwig;

extern "C" int rwig_init(int device) {
  Context* c = nullptr;
  int rc = init_device(device, &c);
  if (rc != 0) return rc;
  if (cudaSetDevice(device) != cudaSuccess) return set_error(RWIG_E_CUDA, "cudaSetDevice failed");
  return 0;
}

extern "C" void rwig_shutdown(void) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  for (auto& c : g_ctx) {
    if (!c) continue;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto& ge : c->graphs)
      if (ge.exec) cudaGraphExecDestroy(ge.exec);
    for (void* p : c->slots)
      if (p) cudaFree(p);
    if (c->pinned) cudaFreeHost(c->pinned);
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaEventDestroy(c->evk);
    cudaEventDestroy(c->evs0);
    cudaEventDestroy(c->evs1);
    cudaEventDestroy(c->evfork);
    cudaEventDestroy(c->evlegacy);
    cudaEventDestroy(c->evjoin);
    for (cudaEvent_t e : c->gemm_ev) cudaEventDestroy(e);
    for (cudaStream_t& q : c->side)
      if (q) {
        cudaStreamSynchronize(q);
        cudaStreamDestroy(q);
      }
    cudaStreamDestroy(c->stream);
    c.reset();
  }
  g_ctx.clear();
}

extern "C" const char* rwig_last_error(void) { return t_last_error.c_str(); }

namespace rwig {
std::atomic<unsigned long long> g_opt_generation{0};
unsigned long long options_generation() { return g_opt_generation.load(std::memory_order_relaxed); }
}  // namespace rwig

extern "C" int rwig_set_option(const char* name, double value) {
  if (!name) return set_error(RWIG_E_INVALID, "option name is null");
  for (const char* known : kOptionNames)
    if (std::strcmp(known, name) == 0) {
      std::lock_guard<std::mutex> lk(g_opt_mu);
      if (std::isnan(value)) g_opts.erase(name);  // back to the built-in default
      else g_opts[name] = value;
      g_opt_generation.fetch_add(1, std::memory_order_relaxed);
      return 0;
    }
  return set_error(RWIG_E_INVALID, std::string("unknown option: ") + name);
}

extern "C" int rwig_get_option(const char* name, double* value) {
  if (!name || !value) return set_error(RWIG_E_INVALID, "option name or value pointer is null");
  for (const char* known : kOptionNames)
    if (std::strcmp(known, name) == 0) {
      std::lock_guard<std::mutex> lk(g_opt_mu);
      auto it = g_opts.find(name);
      if (it == g_opts.end()) return 1;
      *value = it->second;
      return 0;
    }
  return set_error(RWIG_E_INVALID, std::string("unknown option: ") + name);
}

extern "C" int rwig_version(void) { return RWIG_B200_VERSION; }

extern "C" int rwig_last_report(rwig_report* out) {
  if (!out) return RWIG_E_INVALID;
  *out = t_report;
  return 0;
}
