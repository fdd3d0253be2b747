// SPDX-License-Identifier: Apache-2.0
// The host side of a call: the device workspace, the chunking of a batch by free device memory and
// the Run that holds a call's rows on the device (cpp/src/decompose.hpp:35-106 and
// cpp/src/method/driver.cpp:754-923 of eda-cuda define the behaviour this follows).
#pragma once

#include "engine.cuh"

#include <memory>
#include <vector>

namespace edab {

// A grow-only device buffer carved into 256-byte aligned slices (one per thread and device).
class Workspace {
 public:
  Workspace() = default;
  // A view of caller-owned device memory: never allocates, resized or freed by the view.
  Workspace(void* external, size_t bytes)
      : base_(static_cast<unsigned char*>(external)), size_(bytes), owned_(false) {}
  ~Workspace();
  // frees and reallocates when the buffer is smaller; a new buffer is zeroed on stream s (the
  // caller's stream, which may be a non-blocking one: a legacy-stream memset would not be ordered
  // before the caller's work on it)
  void reserve(size_t bytes, cudaStream_t s);
  void reset() { used_ = 0; }
  template <class T>
  T* take(size_t count) {
    const size_t bytes = (count * sizeof(T) + 255) / 256 * 256;
    if (used_ + bytes > size_) throw std::logic_error("eda: workspace layout exceeds its reservation");
    T* p = reinterpret_cast<T*>(base_ + used_);
    used_ += bytes;
    return p;
  }
  void release();

 private:
  unsigned char* base_ = nullptr;
  size_t size_ = 0;
  size_t used_ = 0;
  int device_ = -1;
  bool owned_ = true;
};
// The calling thread's workspace: its own, or the one it leases (set_thread_workspace).
Workspace& thread_workspace();
void set_thread_workspace(Workspace* ws);  // nullptr: the thread's own again
// Workspaces of ragged-batch workers, kept across calls: a worker thread lives for one call, and a
// workspace of its own would be allocated on every call and freed when the thread ends (cudaFree
// synchronises the device, so the workers' ends would wait for one another's work).
Workspace* lease_workspace();
void return_workspace(Workspace* ws);
void release_leased_workspaces();  // frees the idle ones

// Pinned host memory of the calling thread for device-to-host copies into pageable memory: two
// pieces of kPiece bytes, allocated on first use and kept until released.
class HostStaging {
 public:
  static constexpr size_t kPiece = size_t{32} << 20;
  ~HostStaging();
  unsigned char* piece(int i);  // i = 0 or 1
  void release();

 private:
  unsigned char* base_ = nullptr;
};
HostStaging& thread_staging();

// Copies bytes from device memory src to pageable host memory dst on stream s: the transfers land
// in the pinned pieces (double-buffered) and host threads copy each piece on while the next one
// transfers. Returns when dst holds every byte.
void copy_to_pageable(void* dst, const void* src, size_t bytes, cudaStream_t s);
// Whether p is page-locked host memory (copied by DMA directly, not through the staging).
bool is_pinned(const void* p);

struct Params {
  int32_t max_imf = -1;
  double tie_tolerance = -1.0;  // < 0: 2^-14 (float32) / 2^-30 (float64)
  int32_t sifts = 3;
  bool check_finite = true;
  int64_t max_chunk = 0;
  int64_t mem_budget = 0;  // > 0: the device bytes this call may hold (else the free memory)
  bool orientation = false;  // keep n and c of every mode (D >= 2): return_orientation
};

// One call's results: the rows (B, cap, count) on the device and the per-element information.
// The stream-ordered pool of the runs' rows on one device and the stream they are returned on.
struct RowsPool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t free_stream = nullptr;
};
RowsPool& rows_pool(int dev);
// bytes from the current device's rows pool, ordered on stream s (OutOfMemory when they do not fit).
void* rows_alloc(size_t bytes, cudaStream_t s, const char* what);

struct Run {
  int dtype = 0;  // 0 float32, 1 float64
  int device = 0;
  Geom geom{};
  int64_t batch = 0, count = 0, chunk = 0;
  int32_t rows = 1, rows_cap = 0, K = 0;
  std::vector<int32_t> n_imfs, error, hist_scale, hist_sifts;
  std::vector<double> hist_spacing, hist_energy;
  std::vector<int32_t> lens;  // a 1-D batch of uneven lengths: every element's length (else empty)
  void* dev_rows = nullptr;  // from the device's rows pool (rows_alloc)
  void* dev_orient = nullptr;  // (B, cap - 1, D + 1, count) with Params::orientation, rows pool
  ~Run();
  // (B, P, count) into dst: NaN rows for failed elements, zeros above an element's residue.
  void collect(void* dst, bool dst_on_device, cudaStream_t s);
  // Element j alone: (P_j, count) with P_j = n_imfs + 1 (1 for a failed element: a NaN row).
  void collect_one(int64_t j, void* dst, bool dst_on_device, cudaStream_t s);
  // return_orientation: dir (B, K, D, count) and coh (B, K, count), zero beyond n_imfs and for failed
  // elements (cpp/src/method/orientation.cu:524-549, eda_orientation_collect).
  void collect_orientation(void* dir, void* coh, bool dst_on_device, cudaStream_t s);
  int32_t rows_of(int64_t j) const { return error[static_cast<size_t>(j)] ? 1 : n_imfs[static_cast<size_t>(j)] + 1; }
  // samples of element j (its length in a batch of uneven lengths)
  int64_t count_of(int64_t j) const { return lens.empty() ? count : lens[static_cast<size_t>(j)]; }
};

// A ragged batch: elements of different shapes, decomposed in groups (equal shapes, or 1-D length
// classes run as batches of uneven lengths; an element's results do not depend on the batch around
// it) by concurrent workers, each with its own stream and workspace.
struct RaggedRun {
  int dtype = 0, dim = 1, device = 0;
  std::vector<std::unique_ptr<Run>> groups;
  std::vector<int32_t> group;   // per element: its group
  std::vector<int64_t> index;   // per element: its index in the group
  // Every element's rows (P_i, count_i) into one buffer dst (host, or device memory of the run's
  // device) at dst + offsets[i] samples: one table copy and one kernel per group (and, for a host
  // dst, one device-to-host copy of all of them). Complete on return.
  void collect_all(void* dst, bool dst_on_device, const int64_t* offsets, cudaStream_t s);
};
// xs[i]: element i, C-contiguous with extents n[i * dim .. i * dim + dim - 1]; on_device: every
// element on the current device, ready once `s` reaches the call. workers: concurrent groups (>= 1).
std::unique_ptr<RaggedRun> decompose_ragged(const void* const* xs, bool on_device, int dtype, int dim, int64_t count,
                                            const int64_t* n, const Params& p, int workers, cudaStream_t s);
// 1-D ragged batches in length classes (on: the default) or by exact length (off), process-wide.
void set_length_classes(bool on);
bool length_classes();

// Decomposes x (B, n_0..n_{D-1}), C-contiguous, float32 (dtype 0) or float64 (1), on the host or
// the current device, on stream s. Throws std::invalid_argument, OutOfMemory or CudaError.
std::unique_ptr<Run> decompose(const void* x, bool on_device, int dtype, int dim, int64_t batch, const int64_t* n,
                               const Params& p, cudaStream_t s);
// Decomposes a 1-D batch of uneven lengths in one engine run: x (batch, max(lens)) holds element b
// in its first lens[b] samples (the rest is not read). Element b's results are those of a call on
// that element alone; collect them with Run::collect_one.
std::unique_ptr<Run> decompose_lengths(const void* x, bool on_device, int dtype, int64_t batch, const int32_t* lens,
                                       const Params& p, cudaStream_t s);

// A device input read where it lies: element type (the C ABI's EDA_SRC_* codes), batch axes (C
// order) and strides in elements of that type, of either sign.
constexpr int kSrcBool = 0, kSrcI8 = 1, kSrcI16 = 2, kSrcI32 = 3, kSrcI64 = 4, kSrcU8 = 5, kSrcU16 = 6, kSrcU32 = 7,
              kSrcU64 = 8, kSrcF16 = 9, kSrcBF16 = 10, kSrcF32 = 11, kSrcF64 = 12;
constexpr int kMaxBatchAxes = 64;
struct SourceView {
  int32_t type = kSrcF32;
  int32_t batch_axes = 0;
  int64_t batch_shape[kMaxBatchAxes] = {};
  int64_t batch_stride[kMaxBatchAxes] = {};
  int64_t stride[kMaxDim] = {};
};
size_t source_item_size(int type);
// dst (nb, count) dense <- elements b0 .. b0 + nb - 1 of x (src's layout), cast to T, on stream s.
template <class T>
void convert_chunk(cudaStream_t s, const SourceView& src, const void* x, int64_t b0, int64_t nb, int dim,
                   const int64_t* n, T* dst);
// decompose() of a device input in any layout and element type (converted chunk by chunk).
std::unique_ptr<Run> decompose_strided(const void* x, const SourceView& src, int dtype, int dim, const int64_t* n,
                                       const Params& p, cudaStream_t s);
void validate(int dtype, int dim, int64_t batch, const int64_t* n, const Params& p);

// eda.monogenic of the batch x (host or current device, C-contiguous (batch, n..)): out (host or
// device) receives the planes amplitude, phase, frequency [batch][count], then in 2-D / 3-D
// direction [batch][D][count] and coherence [batch][count]; nonfinite[b] (host) = 1 where element b
// holds inf or NaN. Complete on return.
void monogenic(const void* x, bool on_device, int dtype, int dim, int64_t batch, const int64_t* n, int64_t max_chunk,
               void* out, bool out_on_device, int32_t* nonfinite, cudaStream_t s);

template <class T>
size_t engine_bytes(const Geom& g);
template <class T>
void run_chunk(const Geom& g, const Ctl& c, cudaStream_t s, Workspace& ws, const T* x, T* rows, int32_t* hs,
               int32_t* hf, double* hp, double* he, std::vector<Elem>& out, T* orient = nullptr);

}  // namespace edab
