// SPDX-License-Identifier: Apache-2.0
// A call: validation, the output rows, the chunking by free device memory, the host-to-device copy
// of each chunk, the engine, the per-element results and the collect of the public rows
// (cpp/src/method/driver.cpp:754-923 and cpp/src/method/driver.cpp:962-987 of eda-cuda).
#include "driver.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstring>
#include <mutex>
#include <thread>

#include <sys/mman.h>

namespace edab {

Workspace::~Workspace() { release(); }

void Workspace::release() {
  if (!owned_) return;  // a view of caller-owned memory
  if (base_) {
    int prev = -1;
    cudaGetDevice(&prev);
    if (device_ >= 0 && prev != device_) cudaSetDevice(device_);
    cudaFree(base_);
    if (device_ >= 0 && prev != device_ && prev >= 0) cudaSetDevice(prev);
  }
  base_ = nullptr;
  size_ = 0;
  used_ = 0;
}

void Workspace::reserve(size_t bytes, cudaStream_t s) {
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  if (base_ && size_ >= bytes && dev == device_) return;
  release();
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    throw OutOfMemory("eda: the workspace (" + std::to_string(bytes >> 20) + " MiB) does not fit the device memory");
  }
  EDAB_CUDA(e);
  // deterministic contents: pad samples of every field start at zero (ordered on the caller's stream)
  EDAB_CUDA(cudaMemsetAsync(p, 0, bytes, s));
  base_ = static_cast<unsigned char*>(p);
  size_ = bytes;
  device_ = dev;
}

namespace {
thread_local Workspace* t_leased = nullptr;
std::mutex g_pool_mu;
std::vector<std::unique_ptr<Workspace>>& idle_workspaces() {
  static std::vector<std::unique_ptr<Workspace>> v;
  return v;
}
}  // namespace

Workspace& thread_workspace() {
  thread_local Workspace ws;
  return t_leased ? *t_leased : ws;
}

void set_thread_workspace(Workspace* ws) { t_leased = ws; }

Workspace* lease_workspace() {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  auto& v = idle_workspaces();
  if (v.empty()) return new Workspace();
  Workspace* w = v.back().release();
  v.pop_back();
  return w;
}

void return_workspace(Workspace* ws) {
  if (!ws) return;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  idle_workspaces().emplace_back(ws);
}

void release_leased_workspaces() {
  std::vector<std::unique_ptr<Workspace>> v;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    v.swap(idle_workspaces());
  }
  for (auto& w : v) w->release();
}

HostStaging::~HostStaging() { release(); }

unsigned char* HostStaging::piece(int i) {
  if (!base_) {
    void* p = nullptr;
    EDAB_CUDA(cudaHostAlloc(&p, 2 * kPiece, cudaHostAllocPortable));
    base_ = static_cast<unsigned char*>(p);
  }
  return base_ + static_cast<size_t>(i) * kPiece;
}

void HostStaging::release() {
  if (base_) cudaFreeHost(base_);
  base_ = nullptr;
}

HostStaging& thread_staging() {
  thread_local HostStaging st;
  return st;
}

namespace {
// dst[0, bytes) = src[0, bytes) by up to `threads` host threads
void parallel_memcpy(unsigned char* dst, const unsigned char* src, size_t bytes, unsigned threads) {
  const size_t min_share = size_t{1} << 20;
  const unsigned k = static_cast<unsigned>(std::min<size_t>(threads, std::max<size_t>(1, bytes / min_share)));
  if (k <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  std::vector<std::thread> pool;
  const size_t share = (bytes + k - 1) / k;
  for (unsigned t = 1; t < k; ++t) {
    const size_t off = t * share;
    if (off >= bytes) break;
    pool.emplace_back([=] { std::memcpy(dst + off, src + off, std::min(share, bytes - off)); });
  }
  std::memcpy(dst, src, std::min(share, bytes));
  for (auto& th : pool) th.join();
}
}  // namespace

void copy_to_pageable(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (is_pinned(dst)) {  // page-locked already: one DMA
    EDAB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaStreamSynchronize(s));
    return;
  }
  // A large destination not touched yet (a fresh output array) takes a page fault per 4 KiB page
  // during the copy: ask for huge pages on its whole 2 MiB pages first (a hint on this process's
  // own mapping; ignored where the kernel does not support it).
  if (bytes >= (size_t{8} << 20)) {
    const uintptr_t huge = uintptr_t{2} << 20;
    const uintptr_t a = (reinterpret_cast<uintptr_t>(dst) + huge - 1) & ~(huge - 1);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(dst) + bytes) & ~(huge - 1);
    if (e > a) (void)madvise(reinterpret_cast<void*>(a), e - a, MADV_HUGEPAGE);
  }
  HostStaging& st = thread_staging();
  const unsigned threads = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  const size_t P = HostStaging::kPiece;
  const size_t pieces = (bytes + P - 1) / P;
  cudaEvent_t done[2];
  EDAB_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
  EDAB_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
  auto issue = [&](size_t i) {
    const size_t off = i * P, len = std::min(P, bytes - off);
    EDAB_CUDA(cudaMemcpyAsync(st.piece(static_cast<int>(i & 1)), static_cast<const unsigned char*>(src) + off, len,
                              cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaEventRecord(done[i & 1], s));
  };
  issue(0);
  for (size_t i = 0; i < pieces; ++i) {
    EDAB_CUDA(cudaEventSynchronize(done[i & 1]));
    if (i + 1 < pieces) issue(i + 1);  // the other piece was copied on in the previous step
    const size_t off = i * P, len = std::min(P, bytes - off);
    parallel_memcpy(static_cast<unsigned char*>(dst) + off, st.piece(static_cast<int>(i & 1)), len, threads);
  }
  cudaEventDestroy(done[0]);
  cudaEventDestroy(done[1]);
}

bool is_pinned(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// The rows of the runs come from a stream-ordered pool per device that keeps up to 2 GiB cached
// between calls (no cudaMalloc / cudaFree, which synchronizes the device, per call); they are
// returned on the pool's own stream once the run's work is complete (every call and collect ends
// with a synchronization of its stream).
RowsPool& rows_pool(int dev) {
  static std::mutex mu;
  static RowsPool pools[64];
  std::lock_guard<std::mutex> lock(mu);
  RowsPool& p = pools[dev];
  if (!p.pool) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    EDAB_CUDA(cudaMemPoolCreate(&p.pool, &props));
    uint64_t keep = uint64_t{2} << 30;
    EDAB_CUDA(cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    EDAB_CUDA(cudaStreamCreateWithFlags(&p.free_stream, cudaStreamNonBlocking));
  }
  return p;
}

void* rows_alloc(size_t bytes, cudaStream_t s, const char* what) {
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  void* p = nullptr;
  const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, rows_pool(dev).pool, s);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    throw OutOfMemory(std::string("eda: ") + what + " (" + std::to_string(bytes >> 20) +
                      " MiB) do not fit the device memory; set max_imf or decompose fewer elements per call");
  }
  EDAB_CUDA(e);
  return p;
}

Run::~Run() {
  if (!dev_rows && !dev_orient) return;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return;
  cudaSetDevice(device);
  const cudaStream_t fs = rows_pool(device).free_stream;
  if (dev_rows) cudaFreeAsync(dev_rows, fs);
  if (dev_orient) cudaFreeAsync(dev_orient, fs);
  cudaSetDevice(prev);
}

namespace {

// dst (B, P, count) from the rows (B, cap, src_count): src_count > count for an element of a 1-D
// batch of uneven lengths (its rows are laid out at the batch's longest length).
template <class T>
__global__ void collect_kernel(int64_t B, int32_t P, int32_t cap, int64_t count, int64_t src_count,
                               const int32_t* n_imfs, const int32_t* error, const T* __restrict__ src,
                               T* __restrict__ dst) {
  const int64_t total = B * P * count;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx % count;
    const int64_t bk = idx / count;
    const int64_t k = bk % P;
    const int64_t b = bk / P;
    T v;
    if (error[b] != 0) v = static_cast<T>(d_nan());
    else if (k <= n_imfs[b]) v = src[(b * cap + k) * src_count + i];
    else v = T(0);
    dst[idx] = v;
  }
}

// dir (B, K, D, count) and coh (B, K, count) from the orientation rows (B, rows, D + 1, count): rows
// k < n_imfs[b] of elements without an error, zero elsewhere.
template <class T>
__global__ void orient_collect_kernel(int64_t B, int32_t D, int64_t count, int32_t K, int32_t rows,
                                      const int32_t* n_imfs, const int32_t* error, const T* __restrict__ src,
                                      T* __restrict__ dir, T* __restrict__ coh) {
  const int64_t total = B * K * (D + 1) * count;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = idx % count;
    const int64_t q = idx / count;
    const int32_t a = static_cast<int32_t>(q % (D + 1));
    const int64_t bk = q / (D + 1);
    const int64_t k = bk % K;
    const int64_t b = bk / K;
    const T v = error[b] == 0 && k < n_imfs[b] ? src[((b * rows + k) * (D + 1) + a) * count + i] : T(0);
    if (a < D) dir[(bk * D + a) * count + i] = v;
    else coh[bk * count + i] = v;
  }
}

// The longest axis. 2-D and 3-D: the reference's limits (8192 float32, 4096 float64 samples; the
// passes stage whole lines in shared memory). 1-D signals: up to kMaxLine1D samples in either
// dtype (the reference stops at the 2-D limits); lines beyond the staged capacity fold in global
// memory (cube.cu, stats.cu).
constexpr int32_t kMaxLine1D = 65536;
int32_t max_axis(int dtype, int dim) { return dim == 1 ? kMaxLine1D : (dtype == 0 ? 8192 : 4096); }

}  // namespace

void Run::collect(void* dst, bool dst_on_device, cudaStream_t s) {
  if (!lens.empty()) throw std::logic_error("eda: a batch of uneven lengths is collected element by element");
  if (batch == 0 || rows == 0) return;
  const size_t es = dtype == 0 ? 4 : 8;
  const size_t elems = static_cast<size_t>(batch) * rows * count;
  int32_t* meta = nullptr;
  EDAB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&meta), sizeof(int32_t) * 2 * batch, s));
  EDAB_CUDA(cudaMemcpyAsync(meta, n_imfs.data(), sizeof(int32_t) * batch, cudaMemcpyHostToDevice, s));
  EDAB_CUDA(cudaMemcpyAsync(meta + batch, error.data(), sizeof(int32_t) * batch, cudaMemcpyHostToDevice, s));
  void* out = dst;
  if (!dst_on_device) EDAB_CUDA(cudaMallocAsync(&out, elems * es, s));
  const unsigned blocks = blocks_for(static_cast<int64_t>(elems) / 4 + 1);
  const unsigned grid = std::min<unsigned>(blocks, 1u << 20);
  if (dtype == 0) {
    collect_kernel<float><<<grid, kThreads, 0, s>>>(batch, rows, rows_cap, count, count, meta, meta + batch,
                                                    static_cast<const float*>(dev_rows), static_cast<float*>(out));
  } else {
    collect_kernel<double><<<grid, kThreads, 0, s>>>(batch, rows, rows_cap, count, count, meta, meta + batch,
                                                     static_cast<const double*>(dev_rows), static_cast<double*>(out));
  }
  EDAB_LAUNCH("collect_kernel");
  if (!dst_on_device) {
    copy_to_pageable(dst, out, elems * es, s);
    EDAB_CUDA(cudaFreeAsync(out, s));
  }
  EDAB_CUDA(cudaFreeAsync(meta, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
}

void Run::collect_orientation(void* dir, void* coh, bool dst_on_device, cudaStream_t s) {
  if (!dev_orient) throw std::invalid_argument("eda: the call kept no orientation (return_orientation)");
  const int32_t D = geom.dim;
  if (batch == 0 || K == 0) return;
  const size_t es = dtype == 0 ? 4 : 8;
  const size_t nd = static_cast<size_t>(batch) * K * D * static_cast<size_t>(count);
  const size_t nc = static_cast<size_t>(batch) * K * static_cast<size_t>(count);
  int32_t* meta = nullptr;
  EDAB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&meta), sizeof(int32_t) * 2 * batch, s));
  EDAB_CUDA(cudaMemcpyAsync(meta, n_imfs.data(), sizeof(int32_t) * batch, cudaMemcpyHostToDevice, s));
  EDAB_CUDA(cudaMemcpyAsync(meta + batch, error.data(), sizeof(int32_t) * batch, cudaMemcpyHostToDevice, s));
  void* d = dir;
  void* c = coh;
  if (!dst_on_device) {
    EDAB_CUDA(cudaMallocAsync(&d, nd * es, s));
    EDAB_CUDA(cudaMallocAsync(&c, nc * es, s));
  }
  const unsigned grid = std::min<unsigned>(blocks_for(static_cast<int64_t>(nd + nc) / 4 + 1), 1u << 20);
  if (dtype == 0) {
    orient_collect_kernel<float><<<grid, kThreads, 0, s>>>(batch, D, count, K, rows_cap - 1, meta, meta + batch,
                                                           static_cast<const float*>(dev_orient),
                                                           static_cast<float*>(d), static_cast<float*>(c));
  } else {
    orient_collect_kernel<double><<<grid, kThreads, 0, s>>>(batch, D, count, K, rows_cap - 1, meta, meta + batch,
                                                            static_cast<const double*>(dev_orient),
                                                            static_cast<double*>(d), static_cast<double*>(c));
  }
  EDAB_LAUNCH("orient_collect_kernel");
  if (!dst_on_device) {
    copy_to_pageable(dir, d, nd * es, s);
    copy_to_pageable(coh, c, nc * es, s);
    EDAB_CUDA(cudaFreeAsync(d, s));
    EDAB_CUDA(cudaFreeAsync(c, s));
  }
  EDAB_CUDA(cudaFreeAsync(meta, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
}

namespace {

// One element's rows of a ragged run's group, to be written at dst + dst_off.
struct CollectItem {
  int64_t src_off;   // (j cap) src_count: the element's first row in the group's rows
  int64_t dst_off;
  int64_t count;     // the element's samples per row
  int32_t P, n_imfs, error;
};

// Blocks over the items (y) and over each item's P count samples (x).
template <class T>
__global__ void collect_items(const CollectItem* items, int64_t n_items, int64_t src_count, const T* __restrict__ src,
                              T* __restrict__ dst) {
  for (int64_t it = blockIdx.y; it < n_items; it += gridDim.y) {
    const CollectItem c = items[it];
    const int64_t total = static_cast<int64_t>(c.P) * c.count;
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const int64_t k = idx / c.count, t = idx - k * c.count;
      T v;
      if (c.error != 0) v = static_cast<T>(d_nan());
      else if (k <= c.n_imfs) v = src[c.src_off + k * src_count + t];
      else v = T(0);
      dst[c.dst_off + idx] = v;
    }
  }
}

}  // namespace

void RaggedRun::collect_all(void* dst, bool dst_on_device, const int64_t* offsets, cudaStream_t s) {
  const int64_t count = static_cast<int64_t>(group.size());
  if (count == 0) return;
  if (!dst || !offsets) throw std::invalid_argument("eda: null argument");
  const size_t es = dtype == 0 ? 4 : 8;
  int prev = 0;
  EDAB_CUDA(cudaGetDevice(&prev));
  if (prev != device) EDAB_CUDA(cudaSetDevice(device));
  // the extent of the destination, and every element's item in its group
  int64_t total = 0;
  std::vector<std::vector<CollectItem>> items(groups.size());
  for (int64_t i = 0; i < count; ++i) {
    const Run& r = *groups[static_cast<size_t>(group[static_cast<size_t>(i)])];
    const int64_t j = index[static_cast<size_t>(i)];
    CollectItem c{};
    c.src_off = j * r.rows_cap * r.count;
    c.dst_off = offsets[i];
    c.count = r.count_of(j);
    c.P = r.rows_of(j);
    c.n_imfs = r.n_imfs[static_cast<size_t>(j)];
    c.error = r.error[static_cast<size_t>(j)];
    if (c.dst_off < 0) throw std::invalid_argument("eda: a negative destination offset");
    total = std::max(total, c.dst_off + static_cast<int64_t>(c.P) * c.count);
    items[static_cast<size_t>(group[static_cast<size_t>(i)])].push_back(c);
  }
  void* out = dst;
  if (!dst_on_device) EDAB_CUDA(cudaMallocAsync(&out, static_cast<size_t>(total) * es, s));
  std::vector<void*> tables;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    if (items[gi].empty()) continue;
    const Run& r = *groups[gi];
    void* tb = nullptr;
    EDAB_CUDA(cudaMallocAsync(&tb, items[gi].size() * sizeof(CollectItem), s));
    tables.push_back(tb);
    EDAB_CUDA(cudaMemcpyAsync(tb, items[gi].data(), items[gi].size() * sizeof(CollectItem), cudaMemcpyHostToDevice, s));
    const int64_t ni = static_cast<int64_t>(items[gi].size());
    int64_t longest = 1;
    for (const CollectItem& c : items[gi]) longest = std::max(longest, static_cast<int64_t>(c.P) * c.count);
    const dim3 grid(std::min<unsigned>(blocks_for(longest), 256u), static_cast<unsigned>(std::min<int64_t>(ni, 65535)));
    if (dtype == 0) {
      collect_items<float><<<grid, kThreads, 0, s>>>(static_cast<const CollectItem*>(tb), ni, r.count,
                                                     static_cast<const float*>(r.dev_rows), static_cast<float*>(out));
    } else {
      collect_items<double><<<grid, kThreads, 0, s>>>(static_cast<const CollectItem*>(tb), ni, r.count,
                                                      static_cast<const double*>(r.dev_rows), static_cast<double*>(out));
    }
    EDAB_LAUNCH("collect_items");
  }
  if (!dst_on_device) {
    copy_to_pageable(dst, out, static_cast<size_t>(total) * es, s);
    EDAB_CUDA(cudaFreeAsync(out, s));
  }
  for (void* tb : tables) EDAB_CUDA(cudaFreeAsync(tb, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
  if (prev != device) EDAB_CUDA(cudaSetDevice(prev));
}

void Run::collect_one(int64_t j, void* dst, bool dst_on_device, cudaStream_t s) {
  if (j < 0 || j >= batch) throw std::invalid_argument("eda: element index out of range");
  const size_t es = dtype == 0 ? 4 : 8;
  const int32_t P = rows_of(j);
  const int64_t cj = count_of(j);
  const size_t elems = static_cast<size_t>(P) * static_cast<size_t>(cj);
  int32_t* meta = nullptr;
  EDAB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&meta), sizeof(int32_t) * 2, s));
  EDAB_CUDA(cudaMemcpyAsync(meta, n_imfs.data() + j, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  EDAB_CUDA(cudaMemcpyAsync(meta + 1, error.data() + j, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  void* out = dst;
  if (!dst_on_device) EDAB_CUDA(cudaMallocAsync(&out, elems * es, s));
  const unsigned grid = std::min<unsigned>(blocks_for(static_cast<int64_t>(elems) / 4 + 1), 1u << 20);
  const size_t off = static_cast<size_t>(j) * static_cast<size_t>(rows_cap) * static_cast<size_t>(count);
  if (dtype == 0) {
    collect_kernel<float><<<grid, kThreads, 0, s>>>(1, P, rows_cap, cj, count, meta, meta + 1,
                                                    static_cast<const float*>(dev_rows) + off, static_cast<float*>(out));
  } else {
    collect_kernel<double><<<grid, kThreads, 0, s>>>(1, P, rows_cap, cj, count, meta, meta + 1,
                                                     static_cast<const double*>(dev_rows) + off,
                                                     static_cast<double*>(out));
  }
  EDAB_LAUNCH("collect_kernel");
  if (!dst_on_device) {
    copy_to_pageable(dst, out, elems * es, s);
    EDAB_CUDA(cudaFreeAsync(out, s));
  }
  EDAB_CUDA(cudaFreeAsync(meta, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
}

void validate(int dtype, int dim, int64_t batch, const int64_t* n, const Params& p) {
  if (dim < 1 || dim > kMaxDim) throw std::invalid_argument("eda: D must be 1, 2 or 3");
  if (dtype != 0 && dtype != 1) throw std::invalid_argument("eda: the input must be float32 or float64");
  const int32_t lim = max_axis(dtype, dim);
  for (int a = 0; a < dim; ++a) {
    if (n[a] < 1) throw std::invalid_argument("eda: every spatial extent must be >= 1");
    if (n[a] > lim) {
      throw std::invalid_argument("eda: axis extent " + std::to_string(n[a]) + " exceeds the limit " + std::to_string(lim) +
                                  (dtype == 0 ? " for float32" : " for float64"));
    }
  }
  for (int a = 0; a < dim; ++a) {
    if (n[a] < 2) {
      if (dim == 1) {
        throw std::invalid_argument(
            "eda: a 1D signal needs at least 2 samples, got 1 (one sample has no sample differences, so no noise "
            "level; it is its own residue)");
      }
      throw std::invalid_argument("eda: every spatial axis of a " + std::to_string(dim) +
                                  "D field needs extent >= 2, but spatial axis " + std::to_string(a) +
                                  " has extent 1; drop that axis (squeeze it, or leave it out of axes=) to decompose "
                                  "the field in " + std::to_string(dim - 1) + "D");
    }
  }
  if (batch < 1) throw std::invalid_argument("eda: the batch needs at least one element");
  if (!(p.tie_tolerance < 0) && !std::isfinite(p.tie_tolerance)) {
    throw std::invalid_argument("eda: tie_tolerance must be a finite value >= 0");
  }
  if (p.sifts < 1) throw std::invalid_argument("eda: sifts must be >= 1");
  if (p.max_chunk < 0) throw std::invalid_argument("eda: max_chunk must be >= 0");
}

namespace {

// decompose(), decompose_strided() and decompose_lengths(): src (device input only) gives the
// input's own layout and element type, converted chunk by chunk into the staging buffer; without it
// x is dense. lens (host, 1-D only): every element's length, n[0] their maximum.
std::unique_ptr<Run> decompose_impl(const void* x, bool on_device, const SourceView* src, int dtype, int dim,
                                    int64_t batch, const int64_t* n, const Params& p, cudaStream_t s,
                                    const int32_t* lens = nullptr) {
  validate(dtype, dim, batch, n, p);
  const bool f32 = dtype == 0;
  const size_t es = f32 ? 4 : 8;
  const Geom g = make_geom(dim, batch, n);
  // the lengths on the device, released with the call
  struct DeviceLens {
    int32_t* p = nullptr;
    cudaStream_t s = nullptr;
    ~DeviceLens() {
      if (p) cudaFreeAsync(p, s);
    }
  } dlens;
  if (lens) {
    if (dim != 1) throw std::invalid_argument("eda: uneven lengths are 1-D only");
    dlens.s = s;
    EDAB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dlens.p), sizeof(int32_t) * static_cast<size_t>(batch), s));
    EDAB_CUDA(cudaMemcpyAsync(dlens.p, lens, sizeof(int32_t) * static_cast<size_t>(batch), cudaMemcpyHostToDevice, s));
  }
  const double tau = p.tie_tolerance >= 0 ? p.tie_tolerance : (f32 ? std::ldexp(1.0, -14) : std::ldexp(1.0, -30));
  Ctl c = make_ctl(g, f32, p.sifts, tau, p.max_imf, p.check_finite, 0);
  const int32_t bound = mode_bound(c);
  const int32_t modes_max = p.max_imf > 0 ? std::min(bound, p.max_imf) : bound;
  const int32_t cap = modes_max + 2;
  c.rows_cap = cap;
  auto run = std::make_unique<Run>();
  run->dtype = dtype;
  EDAB_CUDA(cudaGetDevice(&run->device));
  run->geom = g;
  run->batch = batch;
  run->count = g.count;
  if (lens) run->lens.assign(lens, lens + batch);
  run->rows_cap = cap;
  const size_t row_bytes = static_cast<size_t>(batch) * cap * static_cast<size_t>(g.count) * es;
  const size_t he = static_cast<size_t>(batch) * static_cast<size_t>(cap - 1);
  run->dev_rows = rows_alloc(row_bytes, s, "the output rows");
  if (p.orientation && dim >= 2) {
    const size_t ob = static_cast<size_t>(batch) * (cap - 1) * (dim + 1) * static_cast<size_t>(g.count) * es;
    run->dev_orient = rows_alloc(ob, s, "the orientation rows");
    EDAB_CUDA(cudaMemsetAsync(run->dev_orient, 0, ob, s));
  }
  // the history: scale, sifts (int32), spacing, energy (double), [B, cap - 1] each
  int32_t* hist_i = nullptr;
  double* hist_d = nullptr;
  EDAB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&hist_i), sizeof(int32_t) * 2 * std::max<size_t>(he, 1), s));
  EDAB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&hist_d), sizeof(double) * 2 * std::max<size_t>(he, 1), s));
  EDAB_CUDA(cudaMemsetAsync(hist_i, 0, sizeof(int32_t) * 2 * std::max<size_t>(he, 1), s));
  EDAB_CUDA(cudaMemsetAsync(hist_d, 0, sizeof(double) * 2 * std::max<size_t>(he, 1), s));
  // the chunk: the largest batch whose workspace fits the free memory (halving)
  int64_t Bc = batch;
  if (p.max_chunk > 0) Bc = std::min(Bc, p.max_chunk);
  size_t free_b = 0, total_b = 0;
  EDAB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (p.mem_budget > 0) free_b = std::min(free_b, static_cast<size_t>(p.mem_budget));
  const size_t margin = std::max<size_t>(p.mem_budget > 0 ? size_t{64} << 20 : size_t{256} << 20, free_b / 20);
  const auto need = [&](int64_t nb) {
    const Geom gc = make_geom(dim, nb, n);
    const size_t stage = static_cast<size_t>(nb) * static_cast<size_t>(g.count) * es;
    return (f32 ? engine_bytes<float>(gc) : engine_bytes<double>(gc)) + stage + 4096;
  };
  Workspace& ws = thread_workspace();
  for (;;) {
    const size_t want = need(Bc);
    if (want + margin <= free_b + 0 || Bc == 1) {
      if (want + margin > free_b && Bc == 1) {
        // the workspace held by this thread counts as free for this call
        ws.release();
        EDAB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        if (want > free_b) {
          throw OutOfMemory("eda: one element needs a workspace of " + std::to_string(want >> 20) + " MiB and " +
                            std::to_string(free_b >> 20) + " MiB are free");
        }
      }
      break;
    }
    Bc = (Bc + 1) / 2;
  }
  run->chunk = Bc;
  ws.reserve(need(Bc), s);
  std::vector<Elem> elems(static_cast<size_t>(batch));
  std::vector<int32_t> exps(static_cast<size_t>(batch), 0);
  std::vector<Elem> part;
  for (int64_t b0 = 0; b0 < batch; b0 += Bc) {
    const int64_t nb = std::min(Bc, batch - b0);
    Geom gc = make_geom(dim, nb, n);
    if (lens) {
      gc.len = dlens.p + b0;
      gc.len_host = lens + b0;
    }
    ws.reset();
    // the chunk's dense input, staged at the head of the workspace
    void* staged = ws.take<unsigned char>(static_cast<size_t>(nb) * static_cast<size_t>(g.count) * es);
    if (src) {
      if (f32) convert_chunk<float>(s, *src, x, b0, nb, dim, n, static_cast<float*>(staged));
      else convert_chunk<double>(s, *src, x, b0, nb, dim, n, static_cast<double*>(staged));
    } else {
      const unsigned char* in = static_cast<const unsigned char*>(x) + static_cast<size_t>(b0) * g.count * es;
      const size_t bytes = static_cast<size_t>(nb) * g.count * es;
      EDAB_CUDA(cudaMemcpyAsync(staged, in, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    }
    const size_t ho = static_cast<size_t>(b0) * static_cast<size_t>(cap - 1);
    unsigned char* rows0 = static_cast<unsigned char*>(run->dev_rows) + static_cast<size_t>(b0) * cap * g.count * es;
    unsigned char* orient0 =
        run->dev_orient ? static_cast<unsigned char*>(run->dev_orient) +
                              static_cast<size_t>(b0) * (cap - 1) * (dim + 1) * static_cast<size_t>(g.count) * es
                        : nullptr;
    if (f32) {
      run_chunk<float>(gc, c, s, ws, static_cast<const float*>(staged), reinterpret_cast<float*>(rows0), hist_i + ho,
                       hist_i + he + ho, hist_d + ho, hist_d + he + ho, part, reinterpret_cast<float*>(orient0));
    } else {
      run_chunk<double>(gc, c, s, ws, static_cast<const double*>(staged), reinterpret_cast<double*>(rows0),
                        hist_i + ho, hist_i + he + ho, hist_d + ho, hist_d + he + ho, part,
                        reinterpret_cast<double*>(orient0));
    }
    for (int64_t b = 0; b < nb; ++b) elems[static_cast<size_t>(b0 + b)] = part[static_cast<size_t>(b)];
  }
  run->n_imfs.assign(static_cast<size_t>(batch), 0);
  run->error.assign(static_cast<size_t>(batch), 0);
  int32_t P = 0;
  bool any_error = false;
  for (int64_t b = 0; b < batch; ++b) {
    const Elem& e = elems[static_cast<size_t>(b)];
    exps[static_cast<size_t>(b)] = e.exp;
    int32_t err = 0, ni = 0;
    if (e.status == kError) err = e.error ? e.error : kErrInternal;
    else if (e.error == kErrNonFiniteResult) err = kErrNonFiniteResult;
    else if (e.status != kDone || e.n_imfs + 1 > cap) err = kErrInternal;
    else ni = e.n_imfs;
    run->error[static_cast<size_t>(b)] = err;
    run->n_imfs[static_cast<size_t>(b)] = ni;
    if (err) any_error = true;
    else P = std::max(P, ni + 1);
    run->K = std::max(run->K, ni);
  }
  if (any_error) P = std::max(P, 1);
  run->rows = P;
  run->hist_scale.resize(he);
  run->hist_sifts.resize(he);
  run->hist_spacing.resize(he);
  run->hist_energy.resize(he);
  if (he) {
    EDAB_CUDA(cudaMemcpyAsync(run->hist_scale.data(), hist_i, he * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaMemcpyAsync(run->hist_sifts.data(), hist_i + he, he * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaMemcpyAsync(run->hist_spacing.data(), hist_d, he * sizeof(double), cudaMemcpyDeviceToHost, s));
    EDAB_CUDA(cudaMemcpyAsync(run->hist_energy.data(), hist_d + he, he * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  EDAB_CUDA(cudaFreeAsync(hist_i, s));
  EDAB_CUDA(cudaFreeAsync(hist_d, s));
  EDAB_CUDA(cudaStreamSynchronize(s));
  // the energies in x's units: 4^k times the prescaled sums
  for (int64_t b = 0; b < batch && he; ++b) {
    const int32_t k = exps[static_cast<size_t>(b)];
    if (k == 0 || run->error[static_cast<size_t>(b)]) continue;
    double* e = run->hist_energy.data() + static_cast<size_t>(b) * static_cast<size_t>(cap - 1);
    for (int32_t j = 0; j < run->n_imfs[static_cast<size_t>(b)]; ++j) e[j] = std::ldexp(e[j], 2 * k);
  }
  return run;
}

}  // namespace

std::unique_ptr<Run> decompose(const void* x, bool on_device, int dtype, int dim, int64_t batch, const int64_t* n,
                               const Params& p, cudaStream_t s) {
  return decompose_impl(x, on_device, nullptr, dtype, dim, batch, n, p, s);
}

std::unique_ptr<Run> decompose_lengths(const void* x, bool on_device, int dtype, int64_t batch, const int32_t* lens,
                                       const Params& p, cudaStream_t s) {
  if (batch > 0 && (!x || !lens)) throw std::invalid_argument("eda: null argument");
  int64_t n_max = 1;
  for (int64_t b = 0; b < batch; ++b) {
    const int64_t nb = lens[b];
    validate(dtype, 1, 1, &nb, p);
    n_max = std::max(n_max, nb);
  }
  return decompose_impl(x, on_device, nullptr, dtype, 1, batch, &n_max, p, s, lens);
}

std::unique_ptr<Run> decompose_strided(const void* x, const SourceView& src, int dtype, int dim, const int64_t* n,
                                       const Params& p, cudaStream_t s) {
  (void)source_item_size(src.type);  // rejects an unknown element type
  if (src.batch_axes < 0 || src.batch_axes > kMaxBatchAxes) {
    throw std::invalid_argument("eda: at most " + std::to_string(kMaxBatchAxes) + " batch axes");
  }
  int64_t batch = 1;
  for (int k = 0; k < src.batch_axes; ++k) {
    if (src.batch_shape[k] < 0) throw std::invalid_argument("eda: a batch extent is negative");
    batch *= src.batch_shape[k];
  }
  if (batch > 0 && !x) throw std::invalid_argument("eda: null input");
  return decompose_impl(x, true, &src, dtype, dim, batch, n, p, s);
}

}  // namespace edab
