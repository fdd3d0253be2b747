// SPDX-License-Identifier: Apache-2.0
// Device buffers for results handed to callers that hold no array library (the reference's output
// pool and DLPack export, cpp/src/runtime/memory.hpp:44-75 and src/eda/_device.py:228-334 of
// eda-cuda): a buffer is reference-counted; the caller's array object holds one reference and
// every DLPack tensor exported from it holds one, released by the tensor's deleter, so the memory
// lives until the last holder lets go. The DLPack structures are those of the DLPack 0.8 ABI
// (DLManagedTensor), laid out here without the dlpack header.
#include "../../include/eda_b200.h"
#include "engine.cuh"

#include <atomic>
#include <cstdlib>
#include <cstring>

namespace edab {
void set_last_error(const char* message);
}

struct eda_buffer {
  void* ptr;
  int device;
  std::atomic<int> refs;
};

namespace {

struct DLDeviceAbi {
  int32_t device_type;  // kDLCUDA = 2
  int32_t device_id;
};
struct DLDataTypeAbi {
  uint8_t code;  // kDLInt 0, kDLUInt 1, kDLFloat 2, kDLBfloat 4, kDLBool 6
  uint8_t bits;
  uint16_t lanes;
};
struct DLTensorAbi {
  void* data;
  DLDeviceAbi device;
  int32_t ndim;
  DLDataTypeAbi dtype;
  int64_t* shape;
  int64_t* strides;
  uint64_t byte_offset;
};
struct DLManagedTensorAbi {
  DLTensorAbi dl_tensor;
  void* manager_ctx;
  void (*deleter)(DLManagedTensorAbi*);
};
// one allocation: the managed tensor, then its shape and strides
struct Exported {
  DLManagedTensorAbi t;
  int64_t dims[2 * 8];
};

void release(eda_buffer* b) {
  if (b == nullptr) return;
  if (b->refs.fetch_sub(1) == 1) {
    int prev = 0;
    if (cudaGetDevice(&prev) == cudaSuccess) {
      cudaSetDevice(b->device);
      cudaFree(b->ptr);  // at interpreter exit the context may be gone: errors are ignored
      cudaSetDevice(prev);
    }
    (void)cudaGetLastError();
    delete b;
  }
}

void exported_deleter(DLManagedTensorAbi* t) {
  if (t == nullptr) return;
  release(static_cast<eda_buffer*>(t->manager_ctx));
  std::free(reinterpret_cast<Exported*>(t));
}

}  // namespace

extern "C" {

EDA_API int eda_buffer_alloc(int device, size_t bytes, eda_buffer** out, void** ptr) {
  try {
    if (!out || !ptr) throw std::invalid_argument("eda: eda_buffer_alloc: null argument");
    int prev = 0;
    EDAB_CUDA(cudaGetDevice(&prev));
    EDAB_CUDA(cudaSetDevice(device));
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes ? bytes : 1);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      if (e == cudaErrorMemoryAllocation) {
        edab::set_last_error("eda: out of device memory for the result");
        return EDA_OUT_OF_MEMORY;
      }
      EDAB_CUDA(e);
    }
    *out = new eda_buffer{p, device, {1}};
    *ptr = p;
    edab::set_last_error("");
    return EDA_OK;
  } catch (const std::invalid_argument& e) {
    edab::set_last_error(e.what());
    return EDA_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    edab::set_last_error(e.what());
    return EDA_CUDA_ERROR;
  }
}

EDA_API void eda_buffer_release(eda_buffer* b) { release(b); }

EDA_API int eda_buffer_dlpack(eda_buffer* b, size_t byte_offset, int dtype_code, int bits, int ndim,
                              const int64_t* shape, const int64_t* strides, void** managed) {
  if (!b || !managed || ndim < 0 || ndim > 8 || (ndim > 0 && (!shape || !strides))) {
    edab::set_last_error("eda: eda_buffer_dlpack: invalid argument");
    return EDA_INVALID_ARGUMENT;
  }
  auto* x = static_cast<Exported*>(std::calloc(1, sizeof(Exported)));
  if (!x) {
    edab::set_last_error("eda: eda_buffer_dlpack: out of host memory");
    return EDA_OUT_OF_MEMORY;
  }
  for (int i = 0; i < ndim; ++i) {
    x->dims[i] = shape[i];
    x->dims[8 + i] = strides[i];
  }
  b->refs.fetch_add(1);
  x->t.dl_tensor.data = b->ptr;
  x->t.dl_tensor.device = DLDeviceAbi{2, b->device};
  x->t.dl_tensor.ndim = ndim;
  x->t.dl_tensor.dtype = DLDataTypeAbi{static_cast<uint8_t>(dtype_code), static_cast<uint8_t>(bits), 1};
  x->t.dl_tensor.shape = x->dims;
  x->t.dl_tensor.strides = x->dims + 8;
  x->t.dl_tensor.byte_offset = byte_offset;
  x->t.manager_ctx = b;
  x->t.deleter = exported_deleter;
  *managed = &x->t;
  edab::set_last_error("");
  return EDA_OK;
}

EDA_API int eda_copy_to_host(void* dst, const void* src, size_t bytes, int device) {
  try {
    int prev = 0;
    EDAB_CUDA(cudaGetDevice(&prev));
    EDAB_CUDA(cudaSetDevice(device));
    const cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    cudaSetDevice(prev);
    EDAB_CUDA(e);
    edab::set_last_error("");
    return EDA_OK;
  } catch (const std::exception& e) {
    edab::set_last_error(e.what());
    return EDA_CUDA_ERROR;
  }
}

EDA_API int eda_pointer_device(const void* p, int* device) {
  if (!device) {
    edab::set_last_error("eda: eda_pointer_device: null argument");
    return EDA_INVALID_ARGUMENT;
  }
  cudaPointerAttributes at{};
  const cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess || (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
    (void)cudaGetLastError();
    edab::set_last_error("eda: the CUDA array's pointer is not device memory");
    return EDA_INVALID_ARGUMENT;
  }
  *device = at.device;
  edab::set_last_error("");
  return EDA_OK;
}

}  // extern "C"
