// SPDX-License-Identifier: Apache-2.0
// Stage-level hooks for the parity tests (include/eda_b200_testing.h): one stage of the engine on a
// dense batch, so that a test compares it bit for bit with the oracle's restatement of the same
// stage. The reference tests its stages the same way through C++ harnesses against host twins
// (cpp/tests/test_cube.cu:52-128 for the cube filter, against cpp/tests/twin.hpp).
#include "../../include/eda_b200_testing.h"
#include "driver.hpp"
#include "orient.cuh"

#include <vector>

namespace edab {
void set_last_error(const char* message);
}

namespace {

using namespace edab;

// dense (B, count) <-> padded (B, field); pads of the padded layout are zero
template <class T>
__global__ void to_padded(Geom g, const T* __restrict__ x, T* __restrict__ f) {
  const int64_t total = g.batch * g.field;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = elem_of(g, i), v = i - b * g.field;
    const int64_t col = v % g.pitch, row = v / g.pitch;
    const int32_t nl = g.n_last;
    f[i] = col < nl ? x[b * g.count + row * nl + col] : T(0);
  }
}
template <class T>
__global__ void to_dense(Geom g, int64_t blocks, const T* __restrict__ f, T* __restrict__ y) {
  const int32_t nl = g.n_last;
  const int64_t total = blocks * g.count;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = i / g.count, c = i - b * g.count;
    const int64_t row = c / nl, col = c - row * nl;
    y[i] = f[b * g.field + row * g.pitch + col];
  }
}

template <class T>
void run_cube(const void* x_dev, int dim, int64_t batch, const int64_t* n, int op, const int32_t* win, int32_t rungs,
              void* out0, void* out1, cudaStream_t s) {
  const Geom g = make_geom(dim, batch, n);
  const int64_t fe = batch * g.field;
  const size_t es = sizeof(T);
  T *in = nullptr, *o0 = nullptr, *o1 = nullptr;
  int32_t* dw = nullptr;
  EDAB_CUDA(cudaMalloc(&in, fe * es));
  EDAB_CUDA(cudaMalloc(&o0, fe * rungs * es));
  EDAB_CUDA(cudaMalloc(&o1, fe * rungs * es));
  EDAB_CUDA(cudaMalloc(&dw, sizeof(int32_t) * batch * rungs));
  EDAB_CUDA(cudaMemcpyAsync(dw, win, sizeof(int32_t) * batch * rungs, cudaMemcpyHostToDevice, s));
  // NaN sentinels: an element with window < 1 keeps them
  EDAB_CUDA(cudaMemsetAsync(o0, 0xff, fe * rungs * es, s));
  EDAB_CUDA(cudaMemsetAsync(o1, 0xff, fe * rungs * es, s));
  const unsigned blocks = blocks_for(fe);
  to_padded<T><<<std::min(blocks, 1u << 16), kThreads, 0, s>>>(g, static_cast<const T*>(x_dev), in);
  EDAB_LAUNCH("to_padded");
  CubeArgs<T> a{};
  a.in = in;
  a.out0 = o0;
  a.out1 = op == static_cast<int>(CubeOp::kMaxMin) ? o1 : nullptr;
  a.win = dw;
  a.rungs = rungs;
  a.out_stride = fe;
  a.epi = BoxEpi::kStore;
  cube<T>(s, g, static_cast<CubeOp>(op), a);
  const unsigned ob = blocks_for(batch * rungs * g.count);
  to_dense<T><<<std::min(ob, 1u << 16), kThreads, 0, s>>>(g, batch * rungs, o0, static_cast<T*>(out0));
  EDAB_LAUNCH("to_dense");
  if (op == static_cast<int>(CubeOp::kMaxMin) && out1) {
    to_dense<T><<<std::min(ob, 1u << 16), kThreads, 0, s>>>(g, batch * rungs, o1, static_cast<T*>(out1));
    EDAB_LAUNCH("to_dense");
  }
  EDAB_CUDA(cudaStreamSynchronize(s));
  cudaFree(in);
  cudaFree(o0);
  cudaFree(o1);
  cudaFree(dw);
}

template <class T>
void run_transform(const void* x_dev, int dim, int64_t batch, const int64_t* n, const int32_t* kinds, void* out_dev,
                   cudaStream_t s) {
  const Geom g = make_geom(dim, batch, n);
  const int64_t fe = batch * g.field;
  const int64_t fw = batch * orient_layout_samples(g);
  const size_t es = sizeof(T);
  T *in = nullptr, *b0 = nullptr, *b1 = nullptr, *out = nullptr;
  int32_t *run = nullptr, *err = nullptr;
  EDAB_CUDA(cudaMalloc(&in, fe * es));
  EDAB_CUDA(cudaMalloc(&b0, fw * es));
  EDAB_CUDA(cudaMalloc(&b1, fw * es));
  EDAB_CUDA(cudaMalloc(&out, fe * es));
  EDAB_CUDA(cudaMalloc(&run, sizeof(int32_t) * batch));
  EDAB_CUDA(cudaMalloc(&err, sizeof(int32_t)));
  std::vector<int32_t> ones(static_cast<size_t>(batch), 1);
  EDAB_CUDA(cudaMemcpyAsync(run, ones.data(), sizeof(int32_t) * batch, cudaMemcpyHostToDevice, s));
  EDAB_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), s));
  const unsigned blocks = blocks_for(fe);
  to_padded<T><<<std::min(blocks, 1u << 16), kThreads, 0, s>>>(g, static_cast<const T*>(x_dev), in);
  EDAB_LAUNCH("to_padded");
  const OrientPlan& plan = orient_plan(g, std::is_same_v<T, double>);
  int k3[kMaxDim] = {0, 0, 0};
  for (int a = 0; a < dim; ++a) k3[a] = kinds[a];
  transform_axes<T>(s, g, plan, in, out, b0, b1, k3, run, err);
  const unsigned ob = blocks_for(batch * g.count);
  to_dense<T><<<std::min(ob, 1u << 16), kThreads, 0, s>>>(g, batch, out, static_cast<T*>(out_dev));
  EDAB_LAUNCH("to_dense");
  int32_t herr = 0;
  EDAB_CUDA(cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
  cudaFree(in);
  cudaFree(b0);
  cudaFree(b1);
  cudaFree(out);
  cudaFree(run);
  cudaFree(err);
  if (herr) throw std::runtime_error("eda_testing_transform: the tensor-core pass gave up waiting for its pipeline");
}

}  // namespace

extern "C" int eda_testing_cube(const void* x_dev, int dtype, int dim, int64_t batch, const int64_t* n, int op,
                                const int32_t* win, int32_t rungs, void* out0_dev, void* out1_dev, void* stream) {
  try {
    if (!x_dev || !n || !win || !out0_dev || batch < 1 || rungs < 1 || rungs > 32 || dim < 1 || dim > kMaxDim ||
        op < 0 || op > 3 || (op == static_cast<int>(CubeOp::kMaxMin) && !out1_dev)) {
      throw std::invalid_argument("eda_testing_cube: invalid argument");
    }
    Params p;
    validate(dtype, dim, batch, n, p);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == 0) run_cube<float>(x_dev, dim, batch, n, op, win, rungs, out0_dev, out1_dev, s);
    else run_cube<double>(x_dev, dim, batch, n, op, win, rungs, out0_dev, out1_dev, s);
    set_last_error("");
    return EDA_OK;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return EDA_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return EDA_CUDA_ERROR;
  }
}

extern "C" int eda_testing_transform(const void* x_dev, int dtype, int dim, int64_t batch, const int64_t* n,
                                     const int32_t* kinds, void* out_dev, void* stream) {
  try {
    if (!x_dev || !n || !kinds || !out_dev || batch < 1 || dim < 2 || dim > kMaxDim) {
      throw std::invalid_argument("eda_testing_transform: invalid argument");
    }
    for (int a = 0; a < dim; ++a) {
      if (kinds[a] < 0 || kinds[a] > 2) throw std::invalid_argument("eda_testing_transform: kinds are 0, 1 or 2");
    }
    Params p;
    validate(dtype, dim, batch, n, p);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == 0) run_transform<float>(x_dev, dim, batch, n, kinds, out_dev, s);
    else run_transform<double>(x_dev, dim, batch, n, kinds, out_dev, s);
    set_last_error("");
    return EDA_OK;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return EDA_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return EDA_CUDA_ERROR;
  }
}
