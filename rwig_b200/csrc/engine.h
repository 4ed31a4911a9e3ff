// engine.h -- host-side plumbing shared by the entry points: per-device
// context (stream, events, scratch arena), error / report bookkeeping.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rwig_b200.h"

namespace rwig {

// A captured launch sequence, replayed when a call repeats with the same
// arguments and buffers (key).
struct GraphEntry {
  std::vector<unsigned long long> key;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
};
enum { kGraphBaryParallel = 0, kGraphBaryLog = 1, kGraphSites = 4 };

struct Context {
  int device = -1;
  int sm_count = 0;
  int smem_optin = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk = nullptr, evs0 = nullptr, evs1 = nullptr;
  cudaEvent_t evfork = nullptr, evjoin = nullptr;  // ordering only (no timing)
  cudaEvent_t evlegacy = nullptr;                   // orders the engine's stream after the legacy default stream
  std::mutex mu;
  std::vector<void*> slots;
  std::vector<size_t> slot_bytes;
  void* pinned = nullptr;  // small pinned staging buffer for scalars
  size_t pinned_bytes = 0;
  GraphEntry graphs[kGraphSites];
  std::vector<unsigned long long> seen[kGraphSites];  // key of the previous call per site
  // side streams of the batched barycenter entry, created on this device on
  // first use (under mu) and destroyed by rwig_shutdown
  static constexpr int kSideStreams = 8;
  cudaStream_t side[kSideStreams] = {};
  // GEMM launch timer (option "profile.gemm"): event pairs around each
  // tensor-core GEMM launch of a call, created on first use
  static constexpr int kTimedGemms = 512;
  std::vector<cudaEvent_t> gemm_ev;
  int gemm_ev_used = 0;
  bool gemm_timing = false;
  // the K whose INT8 residue planes the scratch holds (oz::prepare_reuse):
  // its size and leading dimension, valid while no other prepare ran
  bool oz_kept = false;
  int oz_kept_n = 0;
  long long oz_kept_ldk = 0;
};

// Returns the context of the current (or first) device, initialising it on
// first use.  nullptr on failure (last error set).
Context* get_context();

// The stream a *_dev entry runs on: the caller's, or for a null handle the
// engine's own stream, first made to wait for the work already queued on the
// legacy default stream (the engine's stream is non-blocking, so nothing else
// orders it after a caller that wrote the inputs there).
cudaStream_t call_stream(Context* ctx, void* stream);

// Side stream i (< Context::kSideStreams) of the context's device, created on
// first use (the caller holds ctx->mu with the device current); nullptr on
// failure.
cudaStream_t side_stream(Context* ctx, int i);

// GEMM timer of a call: gemm_timer_begin() arms it when option
// "profile.gemm" is 1; gemm_timer_mark() records an event on `st` (before and
// after each timed launch); gemm_timer_end() (after the timed work has
// completed) returns the summed launch durations and their count, and
// disarms the timer.
int gemm_timer_begin(Context* ctx);
bool gemm_timer_mark(Context* ctx, cudaStream_t st);
void gemm_timer_end(Context* ctx, double* ms, int* launches);

// Grow-only scratch slot `k` of at least `bytes`; nullptr on failure.
void* scratch(Context* ctx, int k, size_t bytes);

// Engine options (rwig_set_option); unknown names return `dflt`.
double option(const char* name, double dflt);
// Count of rwig_set_option calls so far: part of the key of a captured launch
// sequence, so that a sequence captured under other options is not replayed.
unsigned long long options_generation();

// Error / report plumbing (thread-local).
int set_error(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
rwig_report& report();
void reset_report();

#define RWIG_CUDA_TRY(expr)                              \
  do {                                                   \
    cudaError_t _e = (expr);                             \
    if (_e != cudaSuccess) return ::rwig::cuda_fail(_e, #expr); \
  } while (0)

}  // namespace rwig
