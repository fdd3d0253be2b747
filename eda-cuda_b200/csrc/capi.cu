// SPDX-License-Identifier: Apache-2.0
// The C ABI (include/eda_b200.h): exceptions become status codes and a per-thread message.
#include "../../include/eda_b200.h"
#include "driver.hpp"
#include "orient.cuh"

#include <cstdio>
#include <cstring>
#include <string>

struct eda_run {
  std::unique_ptr<edab::Run> run;
};
struct eda_ragged_run {
  std::unique_ptr<edab::RaggedRun> run;
};

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return EDA_OK;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return EDA_INVALID_ARGUMENT;
  } catch (const edab::OutOfMemory& e) {
    g_last_error = e.what();
    return EDA_OUT_OF_MEMORY;
  } catch (const std::bad_alloc& e) {
    g_last_error = std::string("eda: host memory exhausted: ") + e.what();
    return EDA_OUT_OF_MEMORY;
  } catch (const edab::CudaError& e) {
    g_last_error = e.what();
    return e.code == cudaErrorMemoryAllocation ? EDA_OUT_OF_MEMORY : EDA_CUDA_ERROR;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return EDA_INTERNAL;
  } catch (...) {
    g_last_error = "eda: unknown failure";
    return EDA_INTERNAL;
  }
}

void put(char* buf, size_t len, const std::string& s) {
  if (!buf || len == 0) return;
  const size_t k = std::min(len - 1, s.size());
  std::memcpy(buf, s.data(), k);
  buf[k] = 0;
}

}  // namespace

namespace edab {
// The calling thread's last error message, for entry points defined in other files.
void set_last_error(const char* message) { g_last_error = message; }
}  // namespace edab

extern "C" {

int eda_decompose(const void* x, int x_on_device, int dtype, int dim, int64_t batch, const int64_t* n,
                  const eda_params* params, void* stream, eda_run** out) {
  return guarded([&] {
    if (!out || !n || !params) throw std::invalid_argument("eda: null argument");
    if (batch > 0 && !x) throw std::invalid_argument("eda: null input");
    edab::Params p;
    p.max_imf = params->max_imf;
    p.tie_tolerance = params->tie_tolerance;
    p.sifts = params->sifts;
    p.check_finite = params->check_finite != 0;
    p.max_chunk = params->max_chunk;
    p.orientation = params->orientation != 0;
    auto r = std::make_unique<eda_run>();
    r->run = edab::decompose(x, x_on_device != 0, dtype, dim, batch, n, p, static_cast<cudaStream_t>(stream));
    *out = r.release();
  });
}

int eda_decompose_strided(const void* x, const eda_source* src, int dtype, int dim, const int64_t* n,
                          const eda_params* params, void* stream, eda_run** out) {
  return guarded([&] {
    if (!out || !n || !params || !src) throw std::invalid_argument("eda: null argument");
    if (dim < 1 || dim > edab::kMaxDim) throw std::invalid_argument("eda: D must be 1, 2 or 3");
    if (src->batch_axes < 0 || src->batch_axes > edab::kMaxBatchAxes) {
      throw std::invalid_argument("eda: at most 64 batch axes");
    }
    if (!src->stride || (src->batch_axes > 0 && (!src->batch_shape || !src->batch_stride))) {
      throw std::invalid_argument("eda: null layout array");
    }
    edab::SourceView v;
    v.type = src->type;
    v.batch_axes = src->batch_axes;
    for (int k = 0; k < src->batch_axes; ++k) {
      v.batch_shape[k] = src->batch_shape[k];
      v.batch_stride[k] = src->batch_stride[k];
    }
    for (int a = 0; a < dim; ++a) v.stride[a] = src->stride[a];
    edab::Params p;
    p.max_imf = params->max_imf;
    p.tie_tolerance = params->tie_tolerance;
    p.sifts = params->sifts;
    p.check_finite = params->check_finite != 0;
    p.max_chunk = params->max_chunk;
    p.orientation = params->orientation != 0;
    auto r = std::make_unique<eda_run>();
    r->run = edab::decompose_strided(x, v, dtype, dim, n, p, static_cast<cudaStream_t>(stream));
    *out = r.release();
  });
}

int eda_decompose_ragged(const void* const* x, int x_on_device, int dtype, int dim, int64_t count, const int64_t* n,
                         const eda_params* params, int32_t workers, void* stream, eda_ragged_run** out) {
  return guarded([&] {
    if (!out || !params) throw std::invalid_argument("eda: null argument");
    edab::Params p;
    p.max_imf = params->max_imf;
    p.tie_tolerance = params->tie_tolerance;
    p.sifts = params->sifts;
    p.check_finite = params->check_finite != 0;
    p.max_chunk = params->max_chunk;
    p.orientation = params->orientation != 0;
    auto r = std::make_unique<eda_ragged_run>();
    r->run = edab::decompose_ragged(x, x_on_device != 0, dtype, dim, count, n, p, workers,
                                    static_cast<cudaStream_t>(stream));
    *out = r.release();
  });
}

int eda_ragged_element(const eda_ragged_run* run, int64_t i, int32_t* rows, int32_t* n_imfs, int32_t* error,
                       int32_t* windows, int32_t* sifts, double* spacing, double* energy) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("eda: null run");
    const edab::RaggedRun& R = *run->run;
    if (i < 0 || i >= static_cast<int64_t>(R.group.size())) throw std::invalid_argument("eda: element index out of range");
    const edab::Run& r = *R.groups[static_cast<size_t>(R.group[static_cast<size_t>(i)])];
    const int64_t j = R.index[static_cast<size_t>(i)];
    const size_t cap1 = static_cast<size_t>(r.rows_cap > 0 ? r.rows_cap - 1 : 0);
    const int32_t err = r.error[static_cast<size_t>(j)];
    const int32_t k = err ? 0 : r.n_imfs[static_cast<size_t>(j)];
    if (rows) *rows = r.rows_of(j);
    if (n_imfs) *n_imfs = r.n_imfs[static_cast<size_t>(j)];
    if (error) *error = err;
    for (int32_t m = 0; m < k; ++m) {
      const size_t at = static_cast<size_t>(j) * cap1 + static_cast<size_t>(m);
      if (windows) windows[m] = r.hist_scale[at];
      if (sifts) sifts[m] = r.hist_sifts[at];
      if (spacing) spacing[m] = r.hist_spacing[at];
      if (energy) energy[m] = r.hist_energy[at];
    }
  });
}

int eda_ragged_collect(eda_ragged_run* run, int64_t i, void* dst, int dst_on_device, void* stream) {
  return guarded([&] {
    if (!run || !dst) throw std::invalid_argument("eda: null argument");
    edab::RaggedRun& R = *run->run;
    if (i < 0 || i >= static_cast<int64_t>(R.group.size())) throw std::invalid_argument("eda: element index out of range");
    edab::Run& r = *R.groups[static_cast<size_t>(R.group[static_cast<size_t>(i)])];
    int prev = 0;
    EDAB_CUDA(cudaGetDevice(&prev));
    if (prev != r.device) EDAB_CUDA(cudaSetDevice(r.device));
    r.collect_one(R.index[static_cast<size_t>(i)], dst, dst_on_device != 0, static_cast<cudaStream_t>(stream));
    if (prev != r.device) EDAB_CUDA(cudaSetDevice(prev));
  });
}

int eda_ragged_collect_all(eda_ragged_run* run, void* dst, int dst_on_device, const int64_t* offsets, void* stream) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("eda: null run");
    run->run->collect_all(dst, dst_on_device != 0, offsets, static_cast<cudaStream_t>(stream));
  });
}

void eda_ragged_free(eda_ragged_run* run) { delete run; }

int eda_run_shape(const eda_run* run, int64_t* batch, int32_t* rows, int32_t* K, int64_t* count, int64_t* chunk) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("eda: null run");
    const edab::Run& r = *run->run;
    if (batch) *batch = r.batch;
    if (rows) *rows = r.rows;
    if (K) *K = r.K;
    if (count) *count = r.count;
    if (chunk) *chunk = r.chunk;
  });
}

int eda_run_info(const eda_run* run, int32_t* n_imfs, int32_t* error, int32_t* windows, int32_t* sifts,
                 double* spacing, double* energy) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("eda: null run");
    const edab::Run& r = *run->run;
    const size_t B = static_cast<size_t>(r.batch), K = static_cast<size_t>(r.K);
    const size_t cap1 = static_cast<size_t>(r.rows_cap > 0 ? r.rows_cap - 1 : 0);
    for (size_t b = 0; b < B; ++b) {
      if (n_imfs) n_imfs[b] = r.n_imfs[b];
      if (error) error[b] = r.error[b];
      const int32_t kb = r.error[b] ? 0 : r.n_imfs[b];
      for (size_t k = 0; k < K; ++k) {
        const bool have = static_cast<int32_t>(k) < kb;
        if (windows) windows[b * K + k] = have ? r.hist_scale[b * cap1 + k] : 0;
        if (sifts) sifts[b * K + k] = have ? r.hist_sifts[b * cap1 + k] : 0;
        if (spacing) spacing[b * K + k] = have ? r.hist_spacing[b * cap1 + k] : 0.0;
        if (energy) energy[b * K + k] = have ? r.hist_energy[b * cap1 + k] : 0.0;
      }
    }
  });
}

int eda_run_collect(eda_run* run, void* dst, int dst_on_device, void* stream) {
  return guarded([&] {
    if (!run) throw std::invalid_argument("eda: null run");
    edab::Run& r = *run->run;
    int prev = 0;
    EDAB_CUDA(cudaGetDevice(&prev));
    if (prev != r.device) EDAB_CUDA(cudaSetDevice(r.device));
    r.collect(dst, dst_on_device != 0, static_cast<cudaStream_t>(stream));
    if (prev != r.device) EDAB_CUDA(cudaSetDevice(prev));
  });
}

int eda_run_collect_orientation(eda_run* run, void* dir, void* coh, int dst_on_device, void* stream) {
  return guarded([&] {
    if (!run || !dir || !coh) throw std::invalid_argument("eda: null argument");
    edab::Run& r = *run->run;
    int prev = 0;
    EDAB_CUDA(cudaGetDevice(&prev));
    if (prev != r.device) EDAB_CUDA(cudaSetDevice(r.device));
    r.collect_orientation(dir, coh, dst_on_device != 0, static_cast<cudaStream_t>(stream));
    if (prev != r.device) EDAB_CUDA(cudaSetDevice(prev));
  });
}

int eda_monogenic(const void* x, int x_on_device, int dtype, int dim, int64_t batch, const int64_t* n,
                  int64_t max_chunk, void* out, int out_on_device, int32_t* nonfinite, void* stream) {
  return guarded([&] {
    if (!n || !nonfinite || (batch > 0 && (!x || !out))) throw std::invalid_argument("eda: null argument");
    if (batch == 0) return;
    edab::monogenic(x, x_on_device != 0, dtype, dim, batch, n, max_chunk, out, out_on_device != 0, nonfinite,
                    static_cast<cudaStream_t>(stream));
  });
}

void eda_run_free(eda_run* run) { delete run; }

size_t eda_last_error(char* buf, size_t len) {
  put(buf, len, g_last_error);
  return g_last_error.size();
}

int eda_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

int eda_build_info(char* buf, size_t len) {
  int rt = 0, drv = 0;
  cudaRuntimeGetVersion(&rt);
  cudaDriverGetVersion(&drv);
  (void)cudaGetLastError();
  char s[512];
  std::snprintf(s, sizeof s,
                "{\"version\": \"0.1.0\", \"engine\": \"b200\", \"cuda_architectures\": \"100a\", \"sass\": [\"sm_100a\"], "
                "\"ptx\": [], \"cuda_toolkit\": \"%d.%d\", \"cuda_runtime\": %d, \"cuda_driver\": %d, "
                "\"build_type\": \"Release\", \"cufft_version\": null}",
                CUDART_VERSION / 1000, (CUDART_VERSION % 1000) / 10, rt, drv);
  put(buf, len, s);
  return EDA_OK;
}

int eda_device_info(int device, char* buf, size_t len) {
  return guarded([&] {
    int n = eda_device_count();
    if (device < 0 || device >= n) throw std::invalid_argument("eda: CUDA device " + std::to_string(device) + " is not visible");
    cudaDeviceProp p{};
    EDAB_CUDA(cudaGetDeviceProperties(&p, device));
    int rt = 0, drv = 0;
    cudaRuntimeGetVersion(&rt);
    cudaDriverGetVersion(&drv);
    char bus[32] = {0};
    cudaDeviceGetPCIBusId(bus, sizeof bus, device);
    size_t fr = 0, tot = 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaMemGetInfo(&fr, &tot);
    cudaSetDevice(prev);
    (void)cudaGetLastError();
    char s[1024];
    std::snprintf(s, sizeof s,
                  "{\"device\": %d, \"name\": \"%s\", \"pci_bus_id\": \"%s\", \"compute_capability\": [%d, %d], "
                  "\"multiprocessors\": %d, \"total_memory\": %zu, \"free_memory\": %zu, \"l2_cache\": %d, "
                  "\"driver_version\": %d, \"runtime_version\": %d}",
                  device, p.name, bus, p.major, p.minor, p.multiProcessorCount, tot, fr, p.l2CacheSize, drv, rt);
    put(buf, len, s);
  });
}

int eda_release_workspace(void) {
  return guarded([&] {
    edab::thread_workspace().release();
    edab::thread_staging().release();
    edab::release_leased_workspaces();
  });
}

int eda_set_transform_precision(int mode) {
  return guarded([&] {
    if (mode < 0 || mode > 2) throw std::invalid_argument("eda: transform precision must be 0 (3xTF32), 1 (BF16x3) or 2 (FP32)");
    edab::set_transform_precision(static_cast<edab::TransformPrecision>(mode));
  });
}

int eda_transform_precision(void) { return static_cast<int>(edab::transform_precision()); }

int eda_set_length_classes(int32_t on) {
  return guarded([&] { edab::set_length_classes(on != 0); });
}

int eda_length_classes(void) { return edab::length_classes() ? 1 : 0; }

}  // extern "C"
