// SPDX-License-Identifier: Apache-2.0
// An allocation-free decomposition for callers that must not allocate device memory: plugin hosts
// whose device allocator belongs to the host application (an allocation behind its back breaks its
// accounting or its memory limits), and real-time loops that forbid allocation after start-up (an
// allocation can block on the driver for milliseconds). It computes exactly what eda_decompose
// computes (the same engine and kernels, bit for bit), for 1-D signals of bounded size, with all of
// its scratch memory in the file-scope device array below.
//
// The call is synchronous: the engine reads per-element state back to the host between the steps
// of a mode and at the end of the call, so it blocks the host on the caller's stream several times.
//
// The array (kScratchBytes per device) is part of the library's image: every GPU that loads the
// library holds it until the process exits. Every call shares it, and it keeps the last call's
// contents: each call clears what must start at zero. Calls that overlap on the GPU (from several
// threads or streams at once) race on the array, so callers serialize them.
#include "../../include/eda_b200.h"
#include "driver.hpp"

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

namespace edab {
namespace {

constexpr size_t kScratchBytes = size_t{24} << 20;  // 24 MiB per device
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The device address of the array on the current device. In host code the array's name is only a
// host-side stand-in, so the address comes from cudaGetSymbolAddress, once per device, with that
// device current; the first call on a device does this set-up.
void* scratch_address() {
  static std::mutex mu;
  static void* addr[256] = {};
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) throw std::invalid_argument("eda: device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      (void)cudaGetLastError();
      throw CudaError(std::string("eda: cudaGetSymbolAddress of the allocation-free scratch failed: ") +
                          cudaGetErrorString(e),
                      static_cast<int>(e));
    }
    addr[dev] = p;
  }
  return addr[dev];
}

// A caller's buffer must be device memory of the current device (the scratch is that device's).
void require_on_current_device(const void* ptr, const char* name) {
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  cudaPointerAttributes at{};
  const cudaError_t e = cudaPointerGetAttributes(&at, ptr);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw std::invalid_argument(std::string("eda: eda_decompose_noalloc: ") + name + " is not a CUDA pointer");
  }
  if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != dev) {
    throw std::invalid_argument(std::string("eda: eda_decompose_noalloc: ") + name + " must be device memory of the current device (" +
                                std::to_string(dev) + ")");
  }
}

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

// rows (B, P_out, count) of the caller: NaN rows for failed elements, the rows 0..n_imfs, zeros above.
template <class T>
__global__ void collect_into(int64_t B, int32_t P_out, int32_t cap, int64_t count, const int32_t* meta,
                             const T* __restrict__ src, T* __restrict__ dst) {
  const int64_t total = B * P_out * count;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx % count;
    const int64_t bk = idx / count;
    const int64_t k = bk % P_out;
    const int64_t b = bk / P_out;
    T v;
    if (meta[B + b] != 0) v = static_cast<T>(d_nan());
    else if (k <= meta[b] && k < cap) v = src[(b * cap + k) * count + i];
    else v = T(0);
    dst[idx] = v;
  }
}

template <class T>
void run_noalloc(const T* x, int64_t batch, int64_t len, const Params& p, T* rows_dev, int32_t rows_capacity,
                 int32_t* rows_out, int32_t* n_imfs, int32_t* error, int32_t* windows, int32_t* sifts,
                 double* spacing, double* energy, cudaStream_t s) {
  const bool f32 = sizeof(T) == 4;
  const int64_t n[1] = {len};
  const Geom g = make_geom(1, batch, n);
  const double tau = p.tie_tolerance >= 0 ? p.tie_tolerance : (f32 ? std::ldexp(1.0, -14) : std::ldexp(1.0, -30));
  Ctl c = make_ctl(g, f32, p.sifts, tau, p.max_imf, p.check_finite, 0);
  const int32_t bound = mode_bound(c);
  const int32_t cap = (p.max_imf > 0 ? std::min(bound, p.max_imf) : bound) + 2;
  c.rows_cap = cap;
  const size_t he = static_cast<size_t>(batch) * static_cast<size_t>(cap - 1);
  const size_t rows_bytes = up256(static_cast<size_t>(batch) * cap * static_cast<size_t>(g.count) * sizeof(T));
  const size_t hist_bytes = up256(2 * std::max<size_t>(he, 1) * sizeof(int32_t)) + up256(2 * std::max<size_t>(he, 1) * sizeof(double));
  const size_t meta_bytes = up256(2 * static_cast<size_t>(batch) * sizeof(int32_t));
  const size_t engine = engine_bytes<T>(g);
  const size_t need = rows_bytes + hist_bytes + meta_bytes + engine;
  if (need > kScratchBytes) {
    throw std::invalid_argument("eda: eda_decompose_noalloc: the call needs " + std::to_string(need >> 10) +
                                " KiB of scratch and the allocation-free scratch holds " +
                                std::to_string(kScratchBytes >> 10) + " KiB (1-D signals, batch x length up to "
                                "about 32768 float32 or 16384 float64 samples); use eda_decompose");
  }
  unsigned char* base = static_cast<unsigned char*>(scratch_address());
  T* rows_int = reinterpret_cast<T*>(base);
  int32_t* hist_i = reinterpret_cast<int32_t*>(base + rows_bytes);
  double* hist_d = reinterpret_cast<double*>(base + rows_bytes + up256(2 * std::max<size_t>(he, 1) * sizeof(int32_t)));
  int32_t* meta = reinterpret_cast<int32_t*>(base + rows_bytes + hist_bytes);
  unsigned char* ws_base = base + rows_bytes + hist_bytes + meta_bytes;
  // the array keeps the previous call's contents: start from zeros
  EDAB_CUDA(cudaMemsetAsync(base, 0, need, s));
  Workspace ws(ws_base, engine);
  std::vector<Elem> elems;
  run_chunk<T>(g, c, s, ws, x, rows_int, hist_i, hist_i + he, hist_d, hist_d + he, elems);
  // the per-element results, as eda_decompose maps them
  std::vector<int32_t> ni(static_cast<size_t>(batch)), er(static_cast<size_t>(batch));
  int32_t P = 0;
  bool any_error = false;
  for (int64_t b = 0; b < batch; ++b) {
    const Elem& e = elems[static_cast<size_t>(b)];
    int32_t err = 0, k = 0;
    if (e.status == kError) err = e.error ? e.error : kErrInternal;
    else if (e.error == kErrNonFiniteResult) err = kErrNonFiniteResult;
    else if (e.status != kDone || e.n_imfs + 1 > cap) err = kErrInternal;
    else k = e.n_imfs;
    ni[static_cast<size_t>(b)] = k;
    er[static_cast<size_t>(b)] = err;
    if (err) any_error = true;
    else P = std::max(P, k + 1);
  }
  if (any_error) P = std::max(P, 1);
  if (rows_out) *rows_out = P;
  if (P > rows_capacity) {
    throw std::invalid_argument("eda: eda_decompose_noalloc: the result has " + std::to_string(P) +
                                " rows per element and rows_capacity is " + std::to_string(rows_capacity));
  }
  std::vector<int32_t> hs(he), hf(he);
  std::vector<double> hp(he), hen(he);
  if (he) {
    EDAB_CUDA(cudaMemcpyAsync(hs.data(), hist_i, he * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaMemcpyAsync(hf.data(), hist_i + he, he * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaMemcpyAsync(hp.data(), hist_d, he * sizeof(double), cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaMemcpyAsync(hen.data(), hist_d + he, he * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  EDAB_CUDA(cudaMemcpyAsync(meta, ni.data(), sizeof(int32_t) * batch, cudaMemcpyHostToDevice, s));
  EDAB_CUDA(cudaMemcpyAsync(meta + batch, er.data(), sizeof(int32_t) * batch, cudaMemcpyHostToDevice, s));
  const int64_t total = batch * rows_capacity * g.count;
  const unsigned grid = static_cast<unsigned>(std::min<int64_t>((total + kThreads - 1) / kThreads, 1 << 20));
  collect_into<T><<<std::max(grid, 1u), kThreads, 0, s>>>(batch, rows_capacity, cap, g.count, meta, rows_int, rows_dev);
  EDAB_LAUNCH("collect_into");
  EDAB_CUDA(cudaStreamSynchronize(s));
  // the information: [batch] and [batch, rows_capacity - 1], 0 beyond n_imfs and for failures
  const int64_t Kc = rows_capacity - 1;
  for (int64_t b = 0; b < batch; ++b) {
    const int32_t kb = er[static_cast<size_t>(b)] ? 0 : ni[static_cast<size_t>(b)];
    const int32_t k_exp = elems[static_cast<size_t>(b)].exp;
    if (n_imfs) n_imfs[b] = ni[static_cast<size_t>(b)];
    if (error) error[b] = er[static_cast<size_t>(b)];
    for (int64_t k = 0; k < Kc; ++k) {
      const bool have = k < kb;
      const size_t h = static_cast<size_t>(b) * static_cast<size_t>(cap - 1) + static_cast<size_t>(k);
      if (windows) windows[b * Kc + k] = have ? hs[h] : 0;
      if (sifts) sifts[b * Kc + k] = have ? hf[h] : 0;
      if (spacing) spacing[b * Kc + k] = have ? hp[h] : 0.0;
      if (energy) energy[b * Kc + k] = have ? (k_exp ? std::ldexp(hen[h], 2 * k_exp) : hen[h]) : 0.0;
    }
  }
}

}  // namespace

void set_last_error(const char* message);  // capi.cu: the message eda_last_error returns

}  // namespace edab

extern "C" {

EDA_API int eda_decompose_noalloc(const void* x_dev, int dtype, int64_t batch, int64_t length,
                                  const eda_params* params, void* rows_dev, int32_t rows_capacity, int32_t* rows,
                                  int32_t* n_imfs, int32_t* error, int32_t* windows, int32_t* sifts, double* spacing,
                                  double* energy, void* stream) {
  try {
    if (!x_dev || !rows_dev || !params) throw std::invalid_argument("eda: eda_decompose_noalloc: null argument");
    if (rows_capacity < 1) throw std::invalid_argument("eda: eda_decompose_noalloc: rows_capacity must be >= 1");
    edab::Params p;
    p.max_imf = params->max_imf;
    p.tie_tolerance = params->tie_tolerance;
    p.sifts = params->sifts;
    p.check_finite = params->check_finite != 0;
    p.max_chunk = 0;
    const int64_t n[1] = {length};
    edab::validate(dtype, 1, batch, n, p);
    edab::require_on_current_device(x_dev, "x_dev");
    edab::require_on_current_device(rows_dev, "rows_dev");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == EDA_FLOAT32) {
      edab::run_noalloc<float>(static_cast<const float*>(x_dev), batch, length, p, static_cast<float*>(rows_dev),
                               rows_capacity, rows, n_imfs, error, windows, sifts, spacing, energy, s);
    } else {
      edab::run_noalloc<double>(static_cast<const double*>(x_dev), batch, length, p, static_cast<double*>(rows_dev),
                                rows_capacity, rows, n_imfs, error, windows, sifts, spacing, energy, s);
    }
    edab::set_last_error("");
    return EDA_OK;
  } catch (const std::invalid_argument& e) {
    edab::set_last_error(e.what());
    return EDA_INVALID_ARGUMENT;
  } catch (const edab::CudaError& e) {
    edab::set_last_error(e.what());
    return EDA_CUDA_ERROR;
  } catch (const std::exception& e) {
    edab::set_last_error(e.what());
    return EDA_INTERNAL;
  }
}

}  // extern "C"
