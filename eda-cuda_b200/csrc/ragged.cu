// SPDX-License-Identifier: Apache-2.0
// Ragged batches: elements of different shapes in one call. The reference's call takes one shape
// per call (cpp/src/decompose.hpp:106), so a ragged workload runs there as one call per shape, one
// after the other. Here the elements are grouped (an element's rows and information do not depend
// on the other elements of its batch): 1-D signals by length class, the lengths in [2^k, 2^(k+1))
// together, each class one engine run over a batch of uneven lengths (every kernel reads its
// element's own length); 2-D and 3-D fields, and 1-D signals with the classes switched off, by
// shape. The groups run on concurrent workers: host threads with their own CUDA stream and
// workspace, so that the launch latency and the per-mode host reads of small groups overlap on the
// GPU instead of adding up. Each worker gets an equal share of the free device memory as the budget
// of its calls (chunking a group that does not fit, as a single call does).
#include "driver.hpp"

#include <algorithm>
#include <array>
#include <atomic>
#include <exception>
#include <map>
#include <mutex>
#include <thread>

namespace edab {

namespace {

struct Group {
  std::array<int64_t, kMaxDim> n{};  // the shape (a length class: the longest length)
  std::vector<int64_t> members;  // element indices, in input order
  std::vector<int32_t> lens;     // a length class of uneven lengths: the members' lengths
  double work = 0;
};

std::atomic<int32_t> g_length_classes{1};

int32_t length_class(int64_t n) {
  int32_t k = 0;
  while ((int64_t{2} << k) <= n) ++k;
  return k;  // 2^k <= n < 2^(k+1)
}

// Runs group g on the calling worker: the group's elements gathered into one batch (an element
// alone is used in place), then one engine call on stream s.
std::unique_ptr<Run> run_group(const Group& g, const void* const* xs, bool on_device, int dtype, int dim,
                               const Params& p, cudaStream_t s) {
  const size_t es = dtype == 0 ? 4 : 8;
  size_t count = 1;
  for (int a = 0; a < dim; ++a) count *= static_cast<size_t>(g.n[a]);
  const int64_t nb = static_cast<int64_t>(g.members.size());
  const size_t bytes = count * es;
  if (!g.lens.empty()) {
    // one batch of uneven lengths: element j in the first lens[j] samples of row j
    if (on_device) {
      void* buf = nullptr;
      EDAB_CUDA(cudaMallocAsync(&buf, bytes * nb, s));
      for (int64_t j = 0; j < nb; ++j) {
        EDAB_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(buf) + bytes * j, xs[g.members[j]],
                                  static_cast<size_t>(g.lens[j]) * es, cudaMemcpyDeviceToDevice, s));
      }
      std::unique_ptr<Run> r;
      try {
        r = decompose_lengths(buf, true, dtype, nb, g.lens.data(), p, s);
      } catch (...) {
        cudaFreeAsync(buf, s);
        throw;
      }
      EDAB_CUDA(cudaFreeAsync(buf, s));
      return r;
    }
    std::vector<unsigned char> host(bytes * nb, 0);
    for (int64_t j = 0; j < nb; ++j) {
      std::memcpy(host.data() + bytes * j, xs[g.members[j]], static_cast<size_t>(g.lens[j]) * es);
    }
    return decompose_lengths(host.data(), false, dtype, nb, g.lens.data(), p, s);
  }
  if (nb == 1) return decompose(xs[g.members[0]], on_device, dtype, dim, 1, g.n.data(), p, s);
  if (on_device) {
    void* buf = nullptr;
    EDAB_CUDA(cudaMallocAsync(&buf, bytes * nb, s));
    for (int64_t j = 0; j < nb; ++j) {
      EDAB_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(buf) + bytes * j, xs[g.members[j]], bytes,
                                cudaMemcpyDeviceToDevice, s));
    }
    std::unique_ptr<Run> r;
    try {
      r = decompose(buf, true, dtype, dim, nb, g.n.data(), p, s);
    } catch (...) {
      cudaFreeAsync(buf, s);
      throw;
    }
    EDAB_CUDA(cudaFreeAsync(buf, s));
    return r;
  }
  std::vector<unsigned char> host(bytes * nb);
  for (int64_t j = 0; j < nb; ++j) std::memcpy(host.data() + bytes * j, xs[g.members[j]], bytes);
  return decompose(host.data(), false, dtype, dim, nb, g.n.data(), p, s);
}

}  // namespace

void set_length_classes(bool on) { g_length_classes.store(on ? 1 : 0); }
bool length_classes() { return g_length_classes.load() != 0; }

std::unique_ptr<RaggedRun> decompose_ragged(const void* const* xs, bool on_device, int dtype, int dim, int64_t count,
                                            const int64_t* n, const Params& p, int workers, cudaStream_t s) {
  if (count < 0) throw std::invalid_argument("eda: the number of elements must be >= 0");
  if (count > 0 && (!xs || !n)) throw std::invalid_argument("eda: null argument");
  if (workers < 1) throw std::invalid_argument("eda: workers must be >= 1");
  auto out = std::make_unique<RaggedRun>();
  out->dtype = dtype;
  out->dim = dim;
  out->group.assign(static_cast<size_t>(count), 0);
  out->index.assign(static_cast<size_t>(count), 0);
  // every element is checked before any work starts
  std::map<std::array<int64_t, kMaxDim>, int32_t> by_shape;
  std::vector<Group> groups;
  const bool classes = dim == 1 && g_length_classes.load() != 0;
  for (int64_t i = 0; i < count; ++i) {
    if (!xs[i]) throw std::invalid_argument("eda: element " + std::to_string(i) + " is a null pointer");
    validate(dtype, dim, 1, n + i * dim, p);
    std::array<int64_t, kMaxDim> key{1, 1, 1};
    for (int a = 0; a < dim; ++a) key[a] = n[i * dim + a];
    if (classes) key = {-1 - length_class(n[i]), 1, 1};  // (negative: no shape collides with it)
    auto it = by_shape.find(key);
    if (it == by_shape.end()) {
      it = by_shape.emplace(key, static_cast<int32_t>(groups.size())).first;
      Group g;
      g.n = key;
      groups.push_back(g);
    }
    Group& g = groups[static_cast<size_t>(it->second)];
    out->group[static_cast<size_t>(i)] = it->second;
    out->index[static_cast<size_t>(i)] = static_cast<int64_t>(g.members.size());
    g.members.push_back(i);
  }
  // a length class: its longest length, and the members' lengths unless they are all equal
  if (classes) {
    for (Group& g : groups) {
      int64_t lo = n[g.members[0]], hi = lo;
      for (const int64_t i : g.members) {
        lo = std::min(lo, n[i]);
        hi = std::max(hi, n[i]);
      }
      g.n = {hi, 1, 1};
      if (lo != hi) {
        g.lens.reserve(g.members.size());
        for (const int64_t i : g.members) g.lens.push_back(static_cast<int32_t>(n[i]));
      }
    }
  }
  EDAB_CUDA(cudaGetDevice(&out->device));
  out->groups.resize(groups.size());
  if (groups.empty()) return out;
  // the largest groups first (longest-processing-time order over the workers)
  std::vector<int32_t> order(groups.size());
  for (size_t k = 0; k < groups.size(); ++k) {
    double c = 0;
    if (!groups[k].lens.empty()) {
      for (const int32_t l : groups[k].lens) c += static_cast<double>(l);
    } else {
      c = 1;
      for (int a = 0; a < dim; ++a) c *= static_cast<double>(groups[k].n[a]);
      c *= static_cast<double>(groups[k].members.size());
    }
    groups[k].work = c;
    order[k] = static_cast<int32_t>(k);
  }
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return groups[a].work > groups[b].work; });
  const int nw = static_cast<int>(std::min<size_t>(static_cast<size_t>(workers), groups.size()));
  size_t free_b = 0, total_b = 0;
  EDAB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  Params pw = p;
  if (nw > 1) pw.mem_budget = static_cast<int64_t>(free_b / static_cast<size_t>(nw));
  // the workers' streams start after the work the caller queued on s (the inputs' producers)
  cudaEvent_t ready = nullptr;
  EDAB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  EDAB_CUDA(cudaEventRecord(ready, s));
  std::atomic<size_t> next{0};
  std::atomic<bool> stop{false};
  std::mutex err_mu;
  std::exception_ptr first_error;
  const int device = out->device;
  RaggedRun* res = out.get();
  auto work = [&] {
    cudaStream_t ws = nullptr;
    Workspace* leased = nw > 1 ? lease_workspace() : nullptr;  // one worker: the caller's own
    if (leased) set_thread_workspace(leased);
    try {
      EDAB_CUDA(cudaSetDevice(device));
      EDAB_CUDA(cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
      EDAB_CUDA(cudaStreamWaitEvent(ws, ready, 0));
      for (;;) {
        if (stop.load()) break;
        const size_t k = next.fetch_add(1);
        if (k >= order.size()) break;
        const int32_t gi = order[k];
        res->groups[static_cast<size_t>(gi)] = run_group(groups[static_cast<size_t>(gi)], xs, on_device, dtype, dim,
                                                         nw > 1 ? pw : p, ws);
      }
    } catch (...) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_error) first_error = std::current_exception();
      stop.store(true);
    }
    if (ws) {
      cudaStreamSynchronize(ws);
      cudaStreamDestroy(ws);
    }
    if (leased) {
      set_thread_workspace(nullptr);
      return_workspace(leased);
    }
  };
  if (nw == 1) {
    work();
  } else {
    std::vector<std::thread> pool;
    pool.reserve(static_cast<size_t>(nw));
    for (int w = 0; w < nw; ++w) pool.emplace_back(work);
    for (auto& t : pool) t.join();
  }
  cudaEventDestroy(ready);
  if (first_error) std::rethrow_exception(first_error);
  return out;
}

}  // namespace edab
