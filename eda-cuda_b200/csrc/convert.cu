// SPDX-License-Identifier: Apache-2.0
// Device input that cannot be read in place (cpp/src/field/convert.hpp and convert.cu:69-170 of
// eda-cuda define the behaviour): any of 13 element types, any strides (of either sign) over any
// number of batch axes and the spatial axes. One kernel per chunk gathers the chunk's elements and
// casts them to the compute type, straight into the chunk's staging buffer (the dense
// (B, n_0..n_{D-1}) layout that a C-contiguous input is copied into), so no converted copy of the
// whole input is made. Casts round to nearest even (integers of more than 24 / 53 bits, float64 to
// float32); bool gives 0 or 1; float16, bfloat16 and float32 widen exactly.
#include "driver.hpp"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

namespace edab {
namespace {

struct BoolByte {  // a bool stored as one byte: any non-zero byte is true
  uint8_t v;
};

template <class T, class S>
__device__ __forceinline__ T cast_in(S v) {
  if constexpr (std::is_same_v<S, BoolByte>) {
    return v.v != 0 ? T(1) : T(0);
  } else if constexpr (std::is_same_v<S, __half>) {
    return static_cast<T>(__half2float(v));
  } else if constexpr (std::is_same_v<S, __nv_bfloat16>) {
    return static_cast<T>(__bfloat162float(v));
  } else if constexpr (std::is_same_v<T, float>) {
    if constexpr (std::is_same_v<S, double>) return __double2float_rn(v);
    else if constexpr (std::is_same_v<S, int64_t>) return __ll2float_rn(v);
    else if constexpr (std::is_same_v<S, uint64_t>) return __ull2float_rn(v);
    else if constexpr (std::is_same_v<S, int32_t>) return __int2float_rn(v);
    else if constexpr (std::is_same_v<S, uint32_t>) return __uint2float_rn(v);
    else return static_cast<float>(v);  // exact: 8- and 16-bit integers, float32
  } else {
    if constexpr (std::is_same_v<S, int64_t>) return __ll2double_rn(v);
    else if constexpr (std::is_same_v<S, uint64_t>) return __ull2double_rn(v);
    else return static_cast<double>(v);  // exact
  }
}

// dst[j * count + v] <- element b0 + j of x, spatial offset v (C order over n), cast to T.
template <class S, class T>
__global__ void __launch_bounds__(kThreads) convert_gather(SourceView src, const S* __restrict__ x, int64_t b0,
                                                          int64_t nb, int dim, int32_t n1, int32_t n2, int64_t count,
                                                          T* __restrict__ dst) {
  __shared__ int64_t base_s;
  for (int64_t j = blockIdx.y; j < nb; j += gridDim.y) {
    if (threadIdx.x == 0) {
      // the element's offset: its C-order multi-index over the batch shape
      int64_t b = b0 + j, off = 0;
      for (int k = src.batch_axes - 1; k >= 0; --k) {
        const int64_t e = src.batch_shape[k];
        off += (b % e) * src.batch_stride[k];
        b /= e;
      }
      base_s = off;
    }
    __syncthreads();
    const int64_t base = base_s;
    const int64_t s0 = src.stride[0], s1 = src.stride[1], s2 = src.stride[2];
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < count;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      // 32-bit coordinates: an element holds fewer than 2^31 samples
      const uint32_t u = static_cast<uint32_t>(v);
      int64_t at;
      if (dim == 1) {
        at = base + static_cast<int64_t>(u) * s0;
      } else if (dim == 2) {
        const uint32_t i0 = u / static_cast<uint32_t>(n1), i1 = u - i0 * static_cast<uint32_t>(n1);
        at = base + static_cast<int64_t>(i0) * s0 + static_cast<int64_t>(i1) * s1;
      } else {
        const uint32_t q = u / static_cast<uint32_t>(n2), i2 = u - q * static_cast<uint32_t>(n2);
        const uint32_t i0 = q / static_cast<uint32_t>(n1), i1 = q - i0 * static_cast<uint32_t>(n1);
        at = base + static_cast<int64_t>(i0) * s0 + static_cast<int64_t>(i1) * s1 + static_cast<int64_t>(i2) * s2;
      }
      dst[j * count + v] = cast_in<T>(x[at]);
    }
    __syncthreads();  // base_s is rewritten for the next element
  }
}

template <class S, class T>
void launch_convert(cudaStream_t s, const SourceView& src, const void* x, int64_t b0, int64_t nb, int dim,
                    const int64_t* n, T* dst) {
  int64_t count = 1;
  for (int a = 0; a < dim; ++a) count *= n[a];
  const unsigned gx = std::min<unsigned>(blocks_for(count), 1024u);
  const unsigned gy = static_cast<unsigned>(std::min<int64_t>(nb, 65535));
  convert_gather<S, T><<<dim3(gx, gy), kThreads, 0, s>>>(src, static_cast<const S*>(x), b0, nb, dim,
                                                          dim >= 2 ? static_cast<int32_t>(n[1]) : 1,
                                                          dim >= 3 ? static_cast<int32_t>(n[2]) : 1, count, dst);
  EDAB_LAUNCH("convert_gather");
}

}  // namespace

size_t source_item_size(int type) {
  switch (type) {
    case kSrcBool: case kSrcI8: case kSrcU8: return 1;
    case kSrcI16: case kSrcU16: case kSrcF16: case kSrcBF16: return 2;
    case kSrcI32: case kSrcU32: case kSrcF32: return 4;
    case kSrcI64: case kSrcU64: case kSrcF64: return 8;
    default: throw std::invalid_argument("eda: unknown source element type " + std::to_string(type));
  }
}

template <class T>
void convert_chunk(cudaStream_t s, const SourceView& src, const void* x, int64_t b0, int64_t nb, int dim,
                   const int64_t* n, T* dst) {
  switch (src.type) {
    case kSrcBool: launch_convert<BoolByte, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcI8: launch_convert<int8_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcI16: launch_convert<int16_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcI32: launch_convert<int32_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcI64: launch_convert<int64_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcU8: launch_convert<uint8_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcU16: launch_convert<uint16_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcU32: launch_convert<uint32_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcU64: launch_convert<uint64_t, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcF16: launch_convert<__half, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcBF16: launch_convert<__nv_bfloat16, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcF32: launch_convert<float, T>(s, src, x, b0, nb, dim, n, dst); break;
    case kSrcF64: launch_convert<double, T>(s, src, x, b0, nb, dim, n, dst); break;
    default: throw std::invalid_argument("eda: unknown source element type " + std::to_string(src.type));
  }
}

template void convert_chunk<float>(cudaStream_t, const SourceView&, const void*, int64_t, int64_t, int,
                                   const int64_t*, float*);
template void convert_chunk<double>(cudaStream_t, const SourceView&, const void*, int64_t, int64_t, int,
                                    const int64_t*, double*);

}  // namespace edab
