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
  // 1-D lines beyond the staged capacity fold through a global scratch of batch x pitch samples
  const size_t lb = long_line_scratch_bytes(g, sizeof(T));
  void* ls = nullptr;
  if (lb) EDAB_CUDA(cudaMalloc(&ls, lb));
  set_long_line_scratch(ls, lb);
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
  set_long_line_scratch(nullptr, 0);
  cudaFree(ls);
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

template <class T>
void run_select(const void* x_dev, int dim, int64_t batch, const int64_t* n, int src, int axes, const uint8_t* mask_dev,
                int bits, const double* center, double q, double* out, int64_t* count, cudaStream_t s) {
  const Geom g = make_geom(dim, batch, n);
  const int64_t fe = batch * g.field;
  T* f = nullptr;
  uint8_t* m = nullptr;
  double *c = nullptr, *o = nullptr;
  int64_t* k = nullptr;
  EDAB_CUDA(cudaMalloc(&f, fe * sizeof(T)));
  EDAB_CUDA(cudaMalloc(&o, sizeof(double) * batch));
  EDAB_CUDA(cudaMalloc(&k, sizeof(int64_t) * batch));
  to_padded<T><<<std::min(blocks_for(fe), 1u << 16), kThreads, 0, s>>>(g, static_cast<const T*>(x_dev), f);
  EDAB_LAUNCH("to_padded");
  if (mask_dev) {
    EDAB_CUDA(cudaMalloc(&m, fe));
    to_padded<uint8_t><<<std::min(blocks_for(fe), 1u << 16), kThreads, 0, s>>>(g, mask_dev, m);
    EDAB_LAUNCH("to_padded");
  }
  if (center) {
    EDAB_CUDA(cudaMalloc(&c, sizeof(double) * batch));
    EDAB_CUDA(cudaMemcpyAsync(c, center, sizeof(double) * batch, cudaMemcpyHostToDevice, s));
  }
  Sel<T> sel{};
  sel.src = src == 0 ? SelSrc::kField : SelSrc::kDiff;
  sel.field = f;
  sel.mask = m;
  sel.bits = static_cast<uint8_t>(bits);
  sel.axes = static_cast<uint8_t>(axes);
  sel.center = c;
  void* scratch = nullptr;
  EDAB_CUDA(cudaMalloc(&scratch, select_scratch_bytes(g)));
  select<T>(s, g, sel, q, nullptr, o, k, scratch);
  EDAB_CUDA(cudaMemcpyAsync(out, o, sizeof(double) * batch, cudaMemcpyDeviceToHost, s));
  if (count) EDAB_CUDA(cudaMemcpyAsync(count, k, sizeof(int64_t) * batch, cudaMemcpyDeviceToHost, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
  cudaFree(f);
  cudaFree(m);
  cudaFree(c);
  cudaFree(o);
  cudaFree(k);
  cudaFree(scratch);
}

template <class T>
void run_flags(const void* r_dev, const void* tau_dev, int dim, int64_t batch, const int64_t* n, uint8_t* flags_dev,
               uint64_t* ext, cudaStream_t s) {
  const Geom g = make_geom(dim, batch, n);
  const int64_t fe = batch * g.field;
  T *r = nullptr, *tau = nullptr;
  uint8_t* fl = nullptr;
  Elem* el = nullptr;
  EDAB_CUDA(cudaMalloc(&r, fe * sizeof(T)));
  EDAB_CUDA(cudaMalloc(&tau, fe * sizeof(T)));
  EDAB_CUDA(cudaMalloc(&fl, fe));
  EDAB_CUDA(cudaMalloc(&el, sizeof(Elem) * batch));
  EDAB_CUDA(cudaMemsetAsync(el, 0, sizeof(Elem) * batch, s));
  EDAB_CUDA(cudaMemsetAsync(fl, 0xff, fe, s));  // the pass clears the flags of the running elements itself
  const unsigned blocks = std::min(blocks_for(fe), 1u << 16);
  to_padded<T><<<blocks, kThreads, 0, s>>>(g, static_cast<const T*>(r_dev), r);
  EDAB_LAUNCH("to_padded");
  to_padded<T><<<blocks, kThreads, 0, s>>>(g, static_cast<const T*>(tau_dev), tau);
  EDAB_LAUNCH("to_padded");
  sig_flags<T>(s, g, r, tau, fl, el, nullptr);
  to_dense<uint8_t><<<std::min(blocks_for(batch * g.count), 1u << 16), kThreads, 0, s>>>(g, batch, fl, flags_dev);
  EDAB_LAUNCH("to_dense");
  std::vector<Elem> h(static_cast<size_t>(batch));
  EDAB_CUDA(cudaMemcpyAsync(h.data(), el, sizeof(Elem) * batch, cudaMemcpyDeviceToHost, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
  for (int64_t b = 0; b < batch; ++b) {
    for (int a = 0; a < dim; ++a) ext[b * dim + a] = h[static_cast<size_t>(b)].ext[a];
  }
  cudaFree(r);
  cudaFree(tau);
  cudaFree(fl);
  cudaFree(el);
}

// padded labels (the smallest padded index of the component) to dense ones (its dense index)
__global__ void labels_dense(Geom g, const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
  const int32_t nl = g.n_last;
  const int64_t total = g.batch * g.count;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = i / g.count, c = i - b * g.count;
    const int64_t row = c / nl, col = c - row * nl;
    const int32_t v = lab[b * g.field + row * g.pitch + col];
    out[i] = v < 0 ? -1 : static_cast<int32_t>((v / g.pitch) * nl + v % g.pitch);
  }
}

void run_components(const uint8_t* mask_dev, int bits, int dim, int64_t batch, const int64_t* n, int32_t* labels_dev,
                    cudaStream_t s) {
  const Geom g = make_geom(dim, batch, n);
  const int64_t fe = batch * g.field;
  uint8_t* m = nullptr;
  int32_t* lab = nullptr;
  EDAB_CUDA(cudaMalloc(&m, fe));
  EDAB_CUDA(cudaMalloc(&lab, fe * sizeof(int32_t)));
  to_padded<uint8_t><<<std::min(blocks_for(fe), 1u << 16), kThreads, 0, s>>>(g, mask_dev, m);
  EDAB_LAUNCH("to_padded");
  ccl(s, g, m, static_cast<uint8_t>(bits), lab, nullptr);
  labels_dense<<<std::min(blocks_for(batch * g.count), 1u << 16), kThreads, 0, s>>>(g, lab, labels_dev);
  EDAB_LAUNCH("labels_dense");
  EDAB_CUDA(cudaStreamSynchronize(s));
  cudaFree(m);
  cudaFree(lab);
}

template <class F>
int guarded(const char* name, F f) {
  try {
    f();
    set_last_error("");
    return EDA_OK;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return EDA_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    set_last_error((std::string(name) + ": " + e.what()).c_str());
    return EDA_CUDA_ERROR;
  }
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

extern "C" int eda_testing_select(const void* x_dev, int dtype, int dim, int64_t batch, const int64_t* n, int src,
                                  int axes, const uint8_t* mask_dev, int bits, const double* center, double q,
                                  double* out, int64_t* count, void* stream) {
  return guarded("eda_testing_select", [&] {
    if (!x_dev || !n || !out || batch < 1 || dim < 1 || dim > kMaxDim || src < 0 || src > 1 ||
        (src == 1 && (axes <= 0 || axes >= (1 << dim))) || (src == 0 && mask_dev && (bits <= 0 || bits > 255)) ||
        (q >= 0 && q > 1)) {
      throw std::invalid_argument("eda_testing_select: invalid argument");
    }
    Params p;
    validate(dtype, dim, batch, n, p);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == 0) run_select<float>(x_dev, dim, batch, n, src, axes, mask_dev, bits, center, q, out, count, s);
    else run_select<double>(x_dev, dim, batch, n, src, axes, mask_dev, bits, center, q, out, count, s);
  });
}

extern "C" int eda_testing_flags(const void* r_dev, const void* tau_dev, int dtype, int dim, int64_t batch,
                                 const int64_t* n, uint8_t* flags_dev, uint64_t* ext, void* stream) {
  return guarded("eda_testing_flags", [&] {
    if (!r_dev || !tau_dev || !n || !flags_dev || !ext || batch < 1 || dim < 1 || dim > kMaxDim) {
      throw std::invalid_argument("eda_testing_flags: invalid argument");
    }
    Params p;
    validate(dtype, dim, batch, n, p);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == 0) run_flags<float>(r_dev, tau_dev, dim, batch, n, flags_dev, ext, s);
    else run_flags<double>(r_dev, tau_dev, dim, batch, n, flags_dev, ext, s);
  });
}

extern "C" int eda_testing_components(const uint8_t* mask_dev, int bits, int dim, int64_t batch, const int64_t* n,
                                      int32_t* labels_dev, void* stream) {
  return guarded("eda_testing_components", [&] {
    if (!mask_dev || !n || !labels_dev || batch < 1 || dim < 1 || dim > kMaxDim || bits <= 0 || bits > 255) {
      throw std::invalid_argument("eda_testing_components: invalid argument");
    }
    Params p;
    validate(0, dim, batch, n, p);
    run_components(mask_dev, bits, dim, batch, n, labels_dev, static_cast<cudaStream_t>(stream));
  });
}
