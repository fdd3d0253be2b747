/* SPDX-License-Identifier: Apache-2.0
 *
 * eda_b200: the C ABI of the B200 engine of eda's decomposition (the sifting hot path behind
 * eda.decompose). Plain pointers, sizes and status codes; no C++ or framework types. A host binding
 * (ctypes, cgo, JNI, N-API) binds these entry points; eda-cuda_b200/eda/_native.py is the Python
 * one and mirrors the reference's extension module eda._core.
 *
 * Every entry point returns EDA_OK or an error status; eda_last_error() returns the message of the
 * calling thread's last failure. Calls may come from several threads; each thread keeps its own
 * device workspace. The reference interfaces each entry point replaces are cited beside it (paths
 * inside giorgioangel/eda-cuda).
 */
#ifndef EDA_B200_H_
#define EDA_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define EDA_API __attribute__((visibility("default")))
#else
#define EDA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the reference's exceptions, cpp/python/module.cpp:28-51: invalid_argument ->
 * ValueError, bad_alloc -> MemoryError, CudaError -> eda.CudaError). */
#define EDA_OK 0
#define EDA_INVALID_ARGUMENT 1
#define EDA_OUT_OF_MEMORY 2
#define EDA_CUDA_ERROR 3
#define EDA_INTERNAL 4

/* Per-element error codes of info.error (cpp/src/field/state.hpp:16). */
#define EDA_ERR_NONE 0
#define EDA_ERR_NON_FINITE 1
#define EDA_ERR_NON_FINITE_RESULT 2
#define EDA_ERR_INTERNAL 255

#define EDA_FLOAT32 0
#define EDA_FLOAT64 1

/* The call parameters (cpp/src/decompose.hpp:69-76, Params). */
typedef struct eda_params {
  int32_t max_imf;        /* <= 0: no limit */
  double tie_tolerance;   /* relative tie tolerance; < 0: 2^-14 (float32) / 2^-30 (float64) */
  int32_t sifts;          /* sifts per mode, >= 1 (3 by default) */
  int32_t check_finite;   /* non-zero: an element holding inf or NaN fails with code 1 */
  int64_t max_chunk;      /* > 0: at most this many elements per chunk; 0: by free device memory */
  int32_t orientation;    /* non-zero (D >= 2): keep every mode's direction and coherence for
                             eda_run_collect_orientation (the binding's orientation flag,
                             cpp/python/decompose.cpp:325-509) */
} eda_params;

/* One call's results: the rows on the device and the per-element information (the reference's
 * eda::Run, cpp/src/decompose.hpp:85-104). */
typedef struct eda_run eda_run;

/* Decomposes x, a C-contiguous (batch, n[0], .., n[dim-1]) array of float32 (dtype 0) or
 * float64 (dtype 1) on the host (x_on_device 0) or on the calling thread's current CUDA device,
 * on `stream` (a cudaStream_t; NULL: the legacy default stream). On EDA_OK *out receives the run,
 * released by eda_run_free. Replaces eda::decompose (cpp/src/decompose.hpp:106) and the argument
 * rules of the binding's decompose_host / decompose_device (cpp/python/decompose.cpp:325-509). */
EDA_API int eda_decompose(const void* x, int x_on_device, int dtype, int dim, int64_t batch, const int64_t* n,
                  const eda_params* params, void* stream, eda_run** out);

/* Element types of a device input that eda_decompose_strided reads where it lies (the reference's
 * SourceType, cpp/src/field/convert.hpp:18). */
#define EDA_SRC_BOOL 0
#define EDA_SRC_INT8 1
#define EDA_SRC_INT16 2
#define EDA_SRC_INT32 3
#define EDA_SRC_INT64 4
#define EDA_SRC_UINT8 5
#define EDA_SRC_UINT16 6
#define EDA_SRC_UINT32 7
#define EDA_SRC_UINT64 8
#define EDA_SRC_FLOAT16 9
#define EDA_SRC_BFLOAT16 10
#define EDA_SRC_FLOAT32 11
#define EDA_SRC_FLOAT64 12

/* The layout of a device input (the reference's SourceLayout, cpp/src/field/convert.hpp:28-36):
 * element (j, i_0..i_{dim-1}) lies at x + sum_k j_k batch_stride[k] + sum_a i_a stride[a], with
 * j_0..j_{batch_axes-1} the C-order multi-index of batch element j over batch_shape; strides in
 * elements of the source type, either sign; at most 64 batch axes (none: one element). */
typedef struct eda_source {
  int32_t type;                 /* EDA_SRC_* */
  int32_t batch_axes;
  const int64_t* batch_shape;   /* [batch_axes] */
  const int64_t* batch_stride;  /* [batch_axes] */
  const int64_t* stride;        /* [dim] */
} eda_source;

/* eda_decompose of a CUDA input on the current device in any layout and element type: each chunk
 * is gathered and cast to dtype (round to nearest even; bool to 0 / 1) by one kernel into the
 * chunk's staging buffer, with no converted copy of the whole input. The batch is the product of
 * batch_shape. Replaces the strided gather and cast of the reference's decompose_device
 * (cpp/src/field/convert.cu:69-170, cpp/python/decompose.cpp:25-82). */
EDA_API int eda_decompose_strided(const void* x, const eda_source* src, int dtype, int dim, const int64_t* n,
                                  const eda_params* params, void* stream, eda_run** out);

/* The shape of a run: batch, P (the output rows per element: one more than the largest IMF count
 * of the elements without an error), K (the largest IMF count: the width of the information
 * arrays), the samples per element and the elements per chunk (cpp/python/decompose.cpp:188-214). */
EDA_API int eda_run_shape(const eda_run* run, int64_t* batch, int32_t* rows, int32_t* K, int64_t* count, int64_t* chunk);

/* The per-element information: n_imfs[batch], error[batch], and the [batch, K] arrays windows,
 * sifts (int32), spacing, energy (float64), zero beyond an element's n_imfs and for failed
 * elements (cpp/python/decompose.cpp:188-214, info_dict). Any pointer may be NULL. */
EDA_API int eda_run_info(const eda_run* run, int32_t* n_imfs, int32_t* error, int32_t* windows, int32_t* sifts,
                 double* spacing, double* energy);

/* The rows (batch, P, count) in the compute dtype into dst (host memory, or device memory of the
 * run's device with dst_on_device), complete on return: NaN rows for failed elements, the IMFs
 * then the residue, zeros above (cpp/src/field/field_ops.hpp:43-47, Run::collect). */
EDA_API int eda_run_collect(eda_run* run, void* dst, int dst_on_device, void* stream);

/* return_orientation (a call with params->orientation and 2 or 3 axes): dir (batch, K, D, count)
 * receives every mode's unit direction n across the stripes (component a along axis a; the first
 * component of magnitude above the dtype's default tie tolerance positive) and coh (batch, K,
 * count) its coherence in [0, 1], both as computed at the start of the mode; rows beyond an
 * element's n_imfs and all rows of a failed element are 0 (cpp/src/decompose.hpp:97-104,
 * Run::collect_orientation). Host or device memory of the run's device, complete on return. */
EDA_API int eda_run_collect_orientation(eda_run* run, void* dir, void* coh, int dst_on_device, void* stream);

EDA_API void eda_run_free(eda_run* run);

/* eda.monogenic (cpp/src/method/monogenic.cpp:145-155, run_monogenic; the binding's monogenic_host /
 * monogenic_device): the monogenic signal of every field of x (C-contiguous (batch, n[0], ..,
 * n[dim-1]), float32 or float64, host or current device). out (host, or device with out_on_device)
 * receives the reference's native planes: amplitude, phase (-pi, pi], frequency (cycles per sample
 * along the direction), each [batch][count], then in 2-D / 3-D the direction [batch][D][count]
 * (first component above the dtype's default tie tolerance positive) and the coherence
 * [batch][count]; nonfinite[batch] (host) receives 1 for a field holding inf or NaN. max_chunk > 0
 * caps the elements per chunk. Complete on return. */
EDA_API int eda_monogenic(const void* x, int x_on_device, int dtype, int dim, int64_t batch, const int64_t* n,
                          int64_t max_chunk, void* out, int out_on_device, int32_t* nonfinite, void* stream);

/* Ragged batches: count elements of different shapes (same dtype and dim) in one call. Element i is
 * the C-contiguous array x[i] with extents n[i * dim .. i * dim + dim - 1], all on the host
 * (x_on_device 0) or all on the calling thread's current device and ready once `stream` (a
 * cudaStream_t; NULL: the legacy default stream) reaches the call. Equal shapes (1-D signals: length
 * classes, eda_set_length_classes) are decomposed together and up to `workers` groups run
 * concurrently, each on its own stream and workspace; every element's rows and information are
 * those a one-element eda_decompose call gives. The reference
 * takes one shape per call (cpp/src/decompose.hpp:106): a ragged workload there is one call per
 * shape. On EDA_OK *out receives the run, released by eda_ragged_free. */
typedef struct eda_ragged_run eda_ragged_run;
EDA_API int eda_decompose_ragged(const void* const* x, int x_on_device, int dtype, int dim, int64_t count,
                                 const int64_t* n, const eda_params* params, int32_t workers, void* stream,
                                 eda_ragged_run** out);
/* Element i's rows P (n_imfs + 1, or 1 for a failed element), n_imfs, error, and its windows,
 * sifts, spacing, energy (n_imfs entries each, none for a failed element; any pointer may be NULL). */
EDA_API int eda_ragged_element(const eda_ragged_run* run, int64_t i, int32_t* rows, int32_t* n_imfs, int32_t* error,
                               int32_t* windows, int32_t* sifts, double* spacing, double* energy);
/* Element i's rows (P, *n_i) into dst (host, or device memory of the run's device), complete on
 * return: a NaN row for a failed element, the IMFs then the residue otherwise. */
EDA_API int eda_ragged_collect(eda_ragged_run* run, int64_t i, void* dst, int dst_on_device, void* stream);
/* Every element's rows at once (no counterpart in the reference): element i's (P_i, *n_i) rows into
 * dst + offsets[i] (offsets in samples of the run's dtype; dst on the host, or device memory of the
 * run's device, large enough for every element), complete on return. One device pass per group of
 * the run instead of one collect per element. */
EDA_API int eda_ragged_collect_all(eda_ragged_run* run, void* dst, int dst_on_device, const int64_t* offsets,
                                   void* stream);
EDA_API void eda_ragged_free(eda_ragged_run* run);

/* The calling thread's last error message (NUL-terminated, truncated to len). Returns its full
 * length. */
EDA_API size_t eda_last_error(char* buf, size_t len);

/* The visible CUDA devices (0 without a driver or device); the build and a device's properties as
 * JSON text (cpp/python/module.cpp:64-129, build_info / device_info). */
EDA_API int eda_device_count(void);
EDA_API int eda_build_info(char* buf, size_t len);
EDA_API int eda_device_info(int device, char* buf, size_t len);

/* Frees the calling thread's device workspace and its pinned host staging of device-to-host copies
 * (the reference's Context::release_unused_memory, cpp/src/runtime/context.cpp:154-160), and the
 * idle workspaces that ragged-batch workers keep between calls. */
EDA_API int eda_release_workspace(void);

/* Device buffers for results returned to callers without an array library (the reference's output
 * pool and DLPack export, cpp/src/runtime/memory.hpp:44-75, src/eda/_device.py:228-334):
 * eda_buffer_alloc allocates `bytes` on `device` and returns the buffer (one reference, the
 * caller's) and its pointer; eda_buffer_release drops a reference (the memory is freed with the
 * last one); eda_buffer_dlpack exports a view of it (byte_offset, DLPack dtype code 0 int / 1 uint /
 * 2 float / 4 bfloat / 6 bool, bits, ndim <= 8, shape and strides in elements) as a
 * DLManagedTensor* (DLPack 0.8 ABI) that holds one reference until its deleter runs.
 * eda_copy_to_host copies device memory of `device` to the host (synchronous). eda_pointer_device
 * gives the device of device (or managed) memory at p (the reference's pointer_device,
 * cpp/python/module.cpp), EDA_INVALID_ARGUMENT for other memory. */
typedef struct eda_buffer eda_buffer;
EDA_API int eda_buffer_alloc(int device, size_t bytes, eda_buffer** out, void** ptr);
EDA_API void eda_buffer_release(eda_buffer* b);
EDA_API int eda_buffer_dlpack(eda_buffer* b, size_t byte_offset, int dtype_code, int bits, int ndim,
                              const int64_t* shape, const int64_t* strides, void** managed);
EDA_API int eda_copy_to_host(void* dst, const void* src, size_t bytes, int device);
EDA_API int eda_pointer_device(const void* p, int* device);

/* The cube passes' autotuner (no counterpart in the reference, whose launch shapes are fixed,
 * cpp/src/field/vhgw.cu:540-559). eda_autotune times the candidate launch shapes of the cube passes
 * (lines per CTA, line groups per CTA, the segment share from which windows fold whole segments)
 * on a synthetic field of the geometry (dtype, dim, batch, n) on the current device, records the
 * fastest for that geometry (results are bit-identical under every shape) and, with cache_path,
 * writes every record to that text file; report receives a JSON summary. eda_tuning_load reads a
 * cache file into the records (the environment variable EDA_TUNING_CACHE names one that the first
 * cube pass of the process loads); eda_tuning_dump writes the records as text; eda_tuning_clear
 * forgets them. */
EDA_API int eda_autotune(int dtype, int dim, int64_t batch, const int64_t* n, const char* cache_path, char* report,
                         size_t len);
EDA_API int eda_tuning_load(const char* cache_path);
EDA_API int eda_tuning_dump(char* buf, size_t len);
EDA_API int eda_tuning_clear(void);

/* The product of the float32 orientation transforms, process-wide (no counterpart in the reference,
 * whose transforms are cuFFT's float32 FFTs, cpp/src/method/orientation.cu:674-767): 0 = 3xTF32
 * split products on the tensor cores (the default), 1 = BF16x3 split products on the tensor cores,
 * 2 = the plain float32 SIMT product. Float64 fields always use the float64 product. Changing it
 * between calls changes float32 2-D / 3-D results within the transforms' precision (about 1e-6 of
 * the field for 3xTF32 and FP32, 1e-5 for BF16x3). eda_transform_precision returns the current one. */
EDA_API int eda_set_transform_precision(int mode);
EDA_API int eda_transform_precision(void);

/* How eda_decompose_ragged groups 1-D signals, process-wide (no counterpart in the reference, which
 * takes one shape per call, cpp/src/decompose.hpp:106): non-zero (the default) = by length class,
 * the lengths in [2^k, 2^(k+1)) decomposed together as one batch of uneven lengths (every kernel
 * reads each signal's own length); 0 = by exact length. Either way every signal's rows and
 * information are those of a one-element eda_decompose call. eda_length_classes returns the
 * current setting (1 or 0). */
EDA_API int eda_set_length_classes(int32_t on);
EDA_API int eda_length_classes(void);

/* The allocation-free decomposition (no counterpart in the reference), for callers that must not
 * allocate device memory: plugin hosts whose device allocator belongs to the host application, and
 * real-time loops that forbid allocation after start-up. It computes what eda_decompose computes,
 * bit for bit, for 1-D signals: x_dev holds batch x length samples (C-contiguous, dtype 0 float32 /
 * 1 float64) in device memory of the current device; rows_dev (device memory of the current device)
 * receives (batch, rows_capacity, length) in the same layout as eda_run_collect with
 * P = rows_capacity (NaN rows for failed elements, zeros above an element's residue); *rows receives
 * the P an eda_decompose call would have (EDA_INVALID_ARGUMENT when it exceeds rows_capacity); the
 * host arrays n_imfs, error [batch] and windows, sifts, spacing, energy [batch, rows_capacity - 1]
 * are filled as eda_run_info fills them (NULL allowed). All scratch lives in a 24 MiB device array
 * inside the library, held by every GPU that loads the library until the process exits: batch x
 * length up to about 32768 float32 or 16384 float64 samples; larger calls are rejected with
 * EDA_INVALID_ARGUMENT, as are buffers that are not device memory of the current device. The first
 * call on a device looks the array's address up. The call is synchronous: it blocks the host on the
 * stream several times (per-element state is read back between the steps of a mode). Calls share the array: calls that overlap on the
 * GPU race, so serialize them. It calls no cudaMalloc, cudaFree or allocating library routine. */
EDA_API int eda_decompose_noalloc(const void* x_dev, int dtype, int64_t batch, int64_t length,
                                  const eda_params* params, void* rows_dev, int32_t rows_capacity, int32_t* rows,
                                  int32_t* n_imfs, int32_t* error, int32_t* windows, int32_t* sifts, double* spacing,
                                  double* energy, void* stream);

/* Instrumentation (no counterpart in the reference): eda_profile(1) resets and enables the counters
 * of the engine's kernel launches and, for the dominant kernel (the cube-filter passes), of the
 * CUDA-event duration and algorithmic bytes of every launch; eda_profile_read synchronizes the
 * device and returns them. */
EDA_API int eda_profile(int enable);
EDA_API int eda_profile_read(int64_t* launches, int64_t* cube_launches, double* cube_bytes, double* cube_ms);

#ifdef __cplusplus
}
#endif

#endif /* EDA_B200_H_ */
