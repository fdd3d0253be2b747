// SPDX-License-Identifier: Apache-2.0
// eda.monogenic on the engine (cpp/src/method/monogenic.cpp:61-158 of eda-cuda define the behaviour
// this follows): the batch in chunks sized by the free device memory; per chunk the input staged,
// the padded field, the per-element max |x| and non-finite flag, the exact prescale f = x 2^-k with
// k = ilogb(max |x|) (max |f| in [1, 2)), and the monogenic signal (orient.cu, monogenic_fields)
// into the call's output planes. An element's result depends on its own samples only.
#include "../../include/eda_b200.h"
#include "driver.hpp"
#include "orient.cuh"

#include <algorithm>
#include <vector>

namespace edab {
namespace {

template <class T>
__global__ void pad_field(Geom g, const T* __restrict__ x, T* __restrict__ f) {
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const int64_t row = pitch_row(g, v), col = v - row * g.pitch;
      f[b * g.field + v] = col < g.n_last ? x[b * g.count + row * g.n_last + col] : T(0);
    }
  }
}

// max |v| over the finite samples (as integer bits of a non-negative value) and the non-finite flag
template <class T>
__global__ void field_max(Geom g, const T* __restrict__ f, unsigned long long* amax_bits, int32_t* bad) {
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    unsigned long long m = 0;
    int32_t nf = 0;
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const double a = fabs(static_cast<double>(f[b * g.field + v]));
      if (!isfinite(a)) {
        nf = 1;
        continue;
      }
      const unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(a));
      m = u > m ? u : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long w = __shfl_xor_sync(0xffffffffu, m, o);
      m = w > m ? w : m;
      nf |= __shfl_xor_sync(0xffffffffu, nf, o);
    }
    if ((threadIdx.x & 31) == 0) {
      if (m) atomicMax(amax_bits + b, m);
      if (nf) atomicOr(bad + b, 1);
    }
  }
}

template <class T>
__global__ void prescale(Geom g, const unsigned long long* amax_bits, int32_t* exp, T* __restrict__ f) {
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    const double am = __longlong_as_double(static_cast<long long>(amax_bits[b]));
    const int k = am > 0.0 ? ilogb(am) : 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) exp[b] = k;
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      T& y = f[b * g.field + v];
      y = static_cast<T>(ldexp(static_cast<double>(y), -k));
    }
  }
}

template <class T>
void run_monogenic(const void* x, bool on_device, int dim, int64_t batch, const int64_t* n, int64_t max_chunk,
                   T* out, int32_t* nonfinite, cudaStream_t s) {
  const Geom g = make_geom(dim, batch, n);
  const size_t es = sizeof(T);
  const auto need = [&](int64_t nb) {
    const Geom gc = make_geom(dim, nb, n);
    return static_cast<size_t>(nb) * g.count * es + static_cast<size_t>(gc.batch * gc.field) * es +
           static_cast<size_t>(monogenic_work_samples(gc)) * es +
           static_cast<size_t>(nb) * (sizeof(Elem) + 4 * sizeof(int64_t)) + 64 * 256;
  };
  int64_t Bc = max_chunk > 0 ? std::min(batch, max_chunk) : batch;
  size_t free_b = 0, total_b = 0;
  EDAB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t margin = std::max<size_t>(size_t{256} << 20, free_b / 20);
  Workspace& ws = thread_workspace();
  while (Bc > 1 && need(Bc) + margin > free_b) Bc = (Bc + 1) / 2;
  ws.reserve(need(Bc), s);
  const OrientPlan& plan = orient_plan(g, std::is_same_v<T, double>);
  std::vector<int32_t> bad(static_cast<size_t>(Bc));
  for (int64_t b0 = 0; b0 < batch; b0 += Bc) {
    const int64_t nb = std::min(Bc, batch - b0);
    const Geom gc = make_geom(dim, nb, n);
    ws.reset();
    T* staged = ws.take<T>(static_cast<size_t>(nb) * g.count);
    T* f = ws.take<T>(static_cast<size_t>(gc.batch * gc.field));
    T* work = ws.take<T>(static_cast<size_t>(monogenic_work_samples(gc)));
    Elem* el = ws.take<Elem>(static_cast<size_t>(nb));
    unsigned long long* amax = ws.take<unsigned long long>(static_cast<size_t>(nb));
    int32_t* exp = ws.take<int32_t>(static_cast<size_t>(nb));
    int32_t* flag = ws.take<int32_t>(static_cast<size_t>(nb));
    int32_t* run = ws.take<int32_t>(static_cast<size_t>(nb));
    int32_t* err = ws.take<int32_t>(1);
    const T* src = static_cast<const T*>(x) + b0 * g.count;
    EDAB_CUDA(cudaMemcpyAsync(staged, src, static_cast<size_t>(nb) * g.count * es,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    EDAB_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * nb, s));
    EDAB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int32_t) * nb, s));
    EDAB_CUDA(cudaMemsetAsync(el, 0, sizeof(Elem) * nb, s));
    EDAB_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), s));
    const std::vector<int32_t> ones(static_cast<size_t>(nb), 1);
    EDAB_CUDA(cudaMemcpyAsync(run, ones.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice, s));
    const dim3 grid = voxel_grid(gc);
    pad_field<T><<<grid, kThreads, 0, s>>>(gc, staged, f);
    EDAB_LAUNCH("pad_field");
    field_max<T><<<grid, kThreads, 0, s>>>(gc, f, amax, flag);
    EDAB_LAUNCH("field_max");
    prescale<T><<<grid, kThreads, 0, s>>>(gc, amax, exp, f);
    EDAB_LAUNCH("prescale");
    monogenic_fields<T>(s, gc, plan, f, run, exp, el, work, out, batch, b0, err);
    int32_t herr = 0;
    EDAB_CUDA(cudaMemcpyAsync(bad.data(), flag, sizeof(int32_t) * nb, cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaStreamSynchronize(s));
    if (herr) {
      throw CudaError("eda: a tensor-core transform of the monogenic signal gave up waiting for its pipeline",
                      static_cast<int>(cudaErrorLaunchTimeout));
    }
    for (int64_t b = 0; b < nb; ++b) nonfinite[b0 + b] = bad[static_cast<size_t>(b)];
  }
}

}  // namespace

void monogenic(const void* x, bool on_device, int dtype, int dim, int64_t batch, const int64_t* n, int64_t max_chunk,
               void* out, bool out_on_device, int32_t* nonfinite, cudaStream_t s) {
  Params p;
  validate(dtype, dim, batch, n, p);
  // the monogenic transforms are dense products with n x n bases: every axis stays within the
  // 2-D / 3-D limits (the reference's), also in 1-D
  const int64_t lim = dtype == 0 ? 8192 : 4096;
  for (int a = 0; a < dim; ++a) {
    if (n[a] > lim) {
      throw std::invalid_argument("eda: axis extent " + std::to_string(n[a]) + " exceeds the limit " + std::to_string(lim) +
                                  (dtype == 0 ? " for float32" : " for float64"));
    }
  }
  if (max_chunk < 0) throw std::invalid_argument("eda: max_chunk must be >= 0");
  int64_t count = 1;
  for (int a = 0; a < dim; ++a) count *= n[a];
  const size_t es = dtype == 0 ? 4 : 8;
  const size_t planes = dim == 1 ? 3 : static_cast<size_t>(4 + dim);
  const size_t bytes = planes * static_cast<size_t>(batch) * static_cast<size_t>(count) * es;
  void* dst = out;
  if (!out_on_device) {
    const cudaError_t e = cudaMallocAsync(&dst, bytes, s);
    if (e == cudaErrorMemoryAllocation) {
      (void)cudaGetLastError();
      throw OutOfMemory("eda: the monogenic output (" + std::to_string(bytes >> 20) + " MiB) does not fit the device memory");
    }
    EDAB_CUDA(e);
  }
  try {
    if (dtype == 0) run_monogenic<float>(x, on_device, dim, batch, n, max_chunk, static_cast<float*>(dst), nonfinite, s);
    else run_monogenic<double>(x, on_device, dim, batch, n, max_chunk, static_cast<double*>(dst), nonfinite, s);
    if (!out_on_device) copy_to_pageable(out, dst, bytes, s);
  } catch (...) {
    if (!out_on_device) cudaFreeAsync(dst, s);
    throw;
  }
  if (!out_on_device) EDAB_CUDA(cudaFreeAsync(dst, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace edab
