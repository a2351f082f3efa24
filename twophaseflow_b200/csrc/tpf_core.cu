// Library-wide entry points: version, last-error string and the launch-shape
// autotuner.
#include "tpf_common.cuh"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <string>

namespace tpf {

namespace {
thread_local std::string g_last_error;
}

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

const char* last_error() { return g_last_error.c_str(); }

namespace {
std::mutex g_tune_mu;
std::map<std::array<int64_t, 6>, int> g_tuned;
bool g_tune_on = true;
int g_tune_force = -1;   // >= 0: every tuned kernel takes this candidate (clamped)
}  // namespace

int tuned_choice_impl(const TuneKey& key, int ncand, int fallback, size_t scratch_bytes, cudaStream_t s, TuneRun run,
                      void* ctx) {
  const std::array<int64_t, 6> k{key.kernel, key.dtype, key.d[0], key.d[1], key.d[2], key.d[3]};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune_force >= 0) return std::min(g_tune_force, ncand - 1);
    auto it = g_tuned.find(k);
    if (it != g_tuned.end()) return it->second;
    if (!g_tune_on) return fallback;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return fallback;
  }
  void* scratch = nullptr;
  if (scratch_bytes && cudaMalloc(&scratch, scratch_bytes) != cudaSuccess) {
    cudaGetLastError();
    return fallback;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int best = fallback;
  bool ok = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  if (ok && scratch_bytes) ok = cudaMemsetAsync(scratch, 0, scratch_bytes, s) == cudaSuccess;
  float best_t = INFINITY;
  for (int c = 0; ok && c < ncand; ++c) {
    if (run(c, scratch, s, ctx) != TPF_OK || cudaGetLastError() != cudaSuccess) continue;
    float t = INFINITY;
    for (int r = 0; r < 3; ++r) {
      float ms = 0.0f;
      if (cudaEventRecord(e0, s) != cudaSuccess || run(c, scratch, s, ctx) != TPF_OK ||
          cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        ok = false;
        break;
      }
      t = std::fmin(t, ms);
    }
    if (ok && t < best_t) {
      best_t = t;
      best = c;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (scratch) {
    cudaStreamSynchronize(s);
    cudaFree(scratch);
  }
  cudaGetLastError();
  if (!ok) return fallback;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[k] = best;
  return best;
}

}  // namespace tpf

extern "C" {

int tpf_version(void) { return 10000; }

const char* tpf_last_error(void) { return tpf::last_error(); }

int tpf_set_launch_autotune(int mode) {
  TPF_CHECK_ARG(mode >= 0, "autotune mode must be 0 (off), 1 (on) or 2 + k (candidate k), got %d", mode);
  std::lock_guard<std::mutex> lk(tpf::g_tune_mu);
  tpf::g_tune_on = mode == 1;
  tpf::g_tune_force = mode >= 2 ? mode - 2 : -1;
  if (mode != 1) tpf::g_tuned.clear();
  return TPF_OK;
}

int tpf_launch_autotune_entries(void) {
  std::lock_guard<std::mutex> lk(tpf::g_tune_mu);
  return (int)tpf::g_tuned.size();
}

}  // extern "C"
