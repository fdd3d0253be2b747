// SPDX-License-Identifier: Apache-2.0
// Instrumentation: the count of the engine's kernel launches, and for the dominant kernel (the cube
// passes) the CUDA-event duration of every launch and its algorithmic bytes. Off by default; the
// benchmark enables it over its timed region (eda_profile / eda_profile_read of the C ABI).
#include "../../include/eda_b200.h"
#include "engine.cuh"

#include <atomic>
#include <mutex>
#include <set>
#include <utility>
#include <vector>

namespace edab {
namespace {

std::atomic<long long> g_launches{0};
std::atomic<bool> g_on{false};
std::mutex g_mu;
// Events are created once and reused across eda_profile resets (no event creation inside a timed
// region once the pool holds enough): launch i uses events 2 i and 2 i + 1.
std::vector<cudaEvent_t> g_pool;
size_t g_used = 0;
__device__ unsigned long long g_cube_bytes;

}  // namespace

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void once_on_device(const void* key, const std::function<void()>& set) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> seen;
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);  // held while set() runs: later callers wait for it
  if (seen.count({dev, key})) return;
  set();
  seen.emplace(dev, key);
}

bool profiling() { return g_on.load(std::memory_order_relaxed); }

unsigned long long* cube_bytes_counter() {
  if (!profiling()) return nullptr;
  void* p = nullptr;
  EDAB_CUDA(cudaGetSymbolAddress(&p, g_cube_bytes));
  return static_cast<unsigned long long*>(p);
}

void profile_cube_launch(cudaStream_t s, bool begin) {
  if (!profiling()) return;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!begin && g_used % 2 == 0) return;  // an end without its begin
  if (begin && g_used % 2 == 1) --g_used;  // a begin whose launch failed before its end
  if (g_used == g_pool.size()) {
    cudaEvent_t e;
    EDAB_CUDA(cudaEventCreate(&e));
    g_pool.push_back(e);
  }
  EDAB_CUDA(cudaEventRecord(g_pool[g_used++], s));
}

}  // namespace edab

extern "C" {

// Resets the counters and turns the instrumentation on (enable != 0) or off.
EDA_API int eda_profile(int enable) {
  try {
    std::lock_guard<std::mutex> lock(edab::g_mu);
    edab::g_used = 0;
    // enough events for a long timed region, made before it starts
    while (enable && edab::g_pool.size() < 4096) {
      cudaEvent_t e;
      EDAB_CUDA(cudaEventCreate(&e));
      edab::g_pool.push_back(e);
    }
    edab::g_launches.store(0);
    const unsigned long long zero = 0;
    EDAB_CUDA(cudaMemcpyToSymbol(edab::g_cube_bytes, &zero, sizeof zero));
    EDAB_CUDA(cudaDeviceSynchronize());  // the reset lands before work on any stream counts
    edab::g_on.store(enable != 0);
    return EDA_OK;
  } catch (...) {
    return EDA_CUDA_ERROR;
  }
}

// Kernel launches since eda_profile, and for the cube passes: launches, algorithmic bytes and the
// summed CUDA-event milliseconds (synchronizes the device).
EDA_API int eda_profile_read(int64_t* launches, int64_t* cube_launches, double* cube_bytes, double* cube_ms) {
  try {
    EDAB_CUDA(cudaDeviceSynchronize());
    std::lock_guard<std::mutex> lock(edab::g_mu);
    double ms = 0.0;
    const size_t pairs = edab::g_used / 2;
    for (size_t i = 0; i < pairs; ++i) {
      float t = 0.f;
      EDAB_CUDA(cudaEventElapsedTime(&t, edab::g_pool[2 * i], edab::g_pool[2 * i + 1]));
      ms += t;
    }
    unsigned long long bytes = 0;
    EDAB_CUDA(cudaMemcpyFromSymbol(&bytes, edab::g_cube_bytes, sizeof bytes));
    if (launches) *launches = edab::g_launches.load();
    if (cube_launches) *cube_launches = static_cast<int64_t>(pairs);
    if (cube_bytes) *cube_bytes = static_cast<double>(bytes);
    if (cube_ms) *cube_ms = ms;
    return EDA_OK;
  } catch (...) {
    return EDA_CUDA_ERROR;
  }
}

}  // extern "C"
