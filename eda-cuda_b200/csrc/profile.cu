// SPDX-License-Identifier: Apache-2.0
// Instrumentation: the count of the engine's kernel launches, and for the dominant kernel (the cube
// passes) the CUDA-event duration of every launch and its algorithmic bytes. Off by default; the
// benchmark enables it over its timed region (eda_profile / eda_profile_read of the C ABI).
#include "../../include/eda_b200.h"
#include "engine.cuh"

#include <atomic>
#include <mutex>
#include <vector>

namespace edab {
namespace {

std::atomic<long long> g_launches{0};
std::atomic<bool> g_on{false};
std::mutex g_mu;
struct Pair {
  cudaEvent_t a, b;
};
std::vector<Pair> g_events;
cudaEvent_t g_open = nullptr;
__device__ unsigned long long g_cube_bytes;

}  // namespace

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

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
  cudaEvent_t e;
  EDAB_CUDA(cudaEventCreate(&e));
  EDAB_CUDA(cudaEventRecord(e, s));
  if (begin) {
    g_open = e;
  } else {
    g_events.push_back(Pair{g_open, e});
    g_open = nullptr;
  }
}

}  // namespace edab

extern "C" {

// Resets the counters and turns the instrumentation on (enable != 0) or off.
EDA_API int eda_profile(int enable) {
  try {
    std::lock_guard<std::mutex> lock(edab::g_mu);
    for (const auto& p : edab::g_events) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    edab::g_events.clear();
    edab::g_launches.store(0);
    const unsigned long long zero = 0;
    EDAB_CUDA(cudaMemcpyToSymbol(edab::g_cube_bytes, &zero, sizeof zero));
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
    for (const auto& p : edab::g_events) {
      float t = 0.f;
      EDAB_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
      ms += t;
    }
    unsigned long long bytes = 0;
    EDAB_CUDA(cudaMemcpyFromSymbol(&bytes, edab::g_cube_bytes, sizeof bytes));
    if (launches) *launches = edab::g_launches.load();
    if (cube_launches) *cube_launches = static_cast<int64_t>(edab::g_events.size());
    if (cube_bytes) *cube_bytes = static_cast<double>(bytes);
    if (cube_ms) *cube_ms = ms;
    return EDA_OK;
  } catch (...) {
    return EDA_CUDA_ERROR;
  }
}

}  // extern "C"
