// SPDX-License-Identifier: Apache-2.0
// The cube passes' autotuner (no counterpart in the reference, whose launch shapes are fixed:
// vhgw_lines_per_cta, cpp/src/field/vhgw.cu:540-559). A pass's launch shape (lines per CTA, line
// groups per CTA, the segment share from which windows fold whole segments) changes no bit of any
// result, only its speed, and the best shape depends on the geometry: the axis lengths (line and
// segment counts per CTA), the batch (waves of CTAs) and the dtype. eda_autotune times every
// candidate shape on a synthetic field of the geometry, through a max+min and a box cube over a
// ladder of windows like the method's, and records the fastest for that geometry; the records
// live in a table of the process, can be saved to and loaded from a text file (the on-disk
// cache; the environment variable EDA_TUNING_CACHE names one that the first cube pass loads), and
// every later cube pass of a recorded geometry uses its shape.
#include "../../include/eda_b200.h"
#include "driver.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <random>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

namespace edab {
void set_last_error(const char* message);

namespace {

// a geometry: element size, dimension, extents, batch bucket (floor log2 of the batch)
struct TuneKey {
  int es, dim, n0, n1, n2, bucket;
  bool operator<(const TuneKey& o) const {
    return std::tie(es, dim, n0, n1, n2, bucket) < std::tie(o.es, o.dim, o.n0, o.n1, o.n2, o.bucket);
  }
};
struct TuneRecord {
  CubeTune tune;
  double us_default = 0, us_best = 0;
};

std::mutex g_mu;
std::map<TuneKey, TuneRecord> g_table;
bool g_env_loaded = false;
thread_local const CubeTune* t_override = nullptr;

int bucket_of(int64_t batch) {
  int b = 0;
  while ((int64_t{2} << b) <= batch && b < 62) ++b;
  return b;
}
TuneKey key_of(const Geom& g, size_t es) {
  return TuneKey{static_cast<int>(es), g.dim, g.n[0], g.n[1], g.n[2], bucket_of(g.batch)};
}

void load_file_locked(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::invalid_argument("eda: cannot read the tuning cache " + path);
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    TuneKey k{};
    TuneRecord r{};
    if (!(ls >> k.es >> k.dim >> k.n0 >> k.n1 >> k.n2 >> k.bucket >> r.tune.lines >> r.tune.groups >>
          r.tune.seq_share >> r.us_default >> r.us_best)) {
      throw std::invalid_argument("eda: malformed tuning cache line: " + line);
    }
    if ((k.es != 4 && k.es != 8) || k.dim < 1 || k.dim > kMaxDim || r.tune.lines < 0 || r.tune.lines > 8 ||
        r.tune.groups < 0 || r.tune.groups > 4 || r.tune.seq_share < 0 || r.tune.seq_share > 64) {
      throw std::invalid_argument("eda: out-of-range tuning cache line: " + line);
    }
    g_table[k] = r;
  }
}

std::string dump_locked() {
  std::ostringstream os;
  os << "# es dim n0 n1 n2 batch_log2 lines groups seq_share us_default us_best\n";
  for (const auto& [k, r] : g_table) {
    os << k.es << ' ' << k.dim << ' ' << k.n0 << ' ' << k.n1 << ' ' << k.n2 << ' ' << k.bucket << ' ' << r.tune.lines
       << ' ' << r.tune.groups << ' ' << r.tune.seq_share << ' ' << r.us_default << ' ' << r.us_best << '\n';
  }
  return os.str();
}

void load_env_once_locked() {
  if (g_env_loaded) return;
  g_env_loaded = true;
  const char* p = std::getenv("EDA_TUNING_CACHE");
  if (p && *p) {
    try {
      load_file_locked(p);
    } catch (const std::exception&) {
      // a missing or unreadable cache leaves the defaults
    }
  }
}

// The windows of a tuning run: one, then a ladder up to the longest axis's clamped window.
std::vector<int32_t> tuning_windows(const Geom& g) {
  std::vector<int32_t> w{1};
  for (double v = 3.0; v <= 2.0 * g.n_max - 1; v *= 2.0) w.push_back(odd_window(v));
  if (w.size() > static_cast<size_t>(kMaxRungs)) w.resize(kMaxRungs);
  return w;
}

template <class T>
__global__ void fill_noise(T* f, int64_t total, uint64_t seed) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t z = seed + static_cast<uint64_t>(i) * 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z ^= z >> 31;
    f[i] = static_cast<T>(static_cast<double>(z >> 11) * 0x1.0p-53 - 0.5);
  }
}

template <class T>
TuneRecord tune_geometry(const Geom& g, cudaStream_t s) {
  const std::vector<int32_t> wins = tuning_windows(g);
  const int32_t R = static_cast<int32_t>(wins.size());
  const int64_t fe = g.batch * g.field;
  T *in = nullptr, *o0 = nullptr, *o1 = nullptr;
  int32_t* dw = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<int32_t> hw(static_cast<size_t>(R) * g.batch);
  for (int32_t j = 0; j < R; ++j)
    for (int64_t b = 0; b < g.batch; ++b) hw[static_cast<size_t>(j * g.batch + b)] = wins[static_cast<size_t>(j)];
  TuneRecord best{};
  try {
    EDAB_CUDA(cudaMalloc(&in, fe * sizeof(T)));
    EDAB_CUDA(cudaMalloc(&o0, fe * R * sizeof(T)));
    EDAB_CUDA(cudaMalloc(&o1, fe * R * sizeof(T)));
    EDAB_CUDA(cudaMalloc(&dw, hw.size() * sizeof(int32_t)));
    EDAB_CUDA(cudaMemcpyAsync(dw, hw.data(), hw.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    fill_noise<T><<<blocks_for(std::min<int64_t>(fe, 1 << 24)), kThreads, 0, s>>>(in, fe, 12345);
    EDAB_LAUNCH("fill_noise");
    EDAB_CUDA(cudaEventCreate(&e0));
    EDAB_CUDA(cudaEventCreate(&e1));
    const auto time_shape = [&](const CubeTune* t) {
      cube_tune_override(t);
      double us = 1e300;
      for (int rep = 0; rep < 3; ++rep) {  // the first is a warm-up
        EDAB_CUDA(cudaEventRecord(e0, s));
        CubeArgs<T> a{};
        a.in = in;
        a.out0 = o0;
        a.out1 = o1;
        a.win = dw;
        a.rungs = R;
        a.out_stride = fe;
        a.epi = BoxEpi::kStore;
        cube<T>(s, g, CubeOp::kMaxMin, a);
        a.out1 = nullptr;
        cube<T>(s, g, CubeOp::kBox, a);
        EDAB_CUDA(cudaEventRecord(e1, s));
        EDAB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        EDAB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0) us = std::min(us, 1000.0 * ms);
      }
      cube_tune_override(nullptr);
      return us;
    };
    best.us_default = time_shape(nullptr);
    best.us_best = best.us_default;
    for (int lines : {8, 4, 2}) {
      for (int groups : {1, 2}) {
        for (int share : {2, 4, 8}) {
          const CubeTune t{lines, groups, share};
          const double us = time_shape(&t);
          if (us < best.us_best) {
            best.us_best = us;
            best.tune = t;
          }
        }
      }
    }
  } catch (...) {
    cube_tune_override(nullptr);
    cudaFree(in);
    cudaFree(o0);
    cudaFree(o1);
    cudaFree(dw);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    throw;
  }
  cudaFree(in);
  cudaFree(o0);
  cudaFree(o1);
  cudaFree(dw);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

void put(char* buf, size_t len, const std::string& s) {
  if (!buf || len == 0) return;
  const size_t k = std::min(len - 1, s.size());
  std::memcpy(buf, s.data(), k);
  buf[k] = '\0';
}

}  // namespace

CubeTune cube_tune_for(const Geom& g, int axis, size_t es) {
  (void)axis;  // one shape per geometry: every pass of its cubes
  if (t_override) return *t_override;
  std::lock_guard<std::mutex> lock(g_mu);
  load_env_once_locked();
  if (g_table.empty()) return CubeTune{};
  const auto it = g_table.find(key_of(g, es));
  return it == g_table.end() ? CubeTune{} : it->second.tune;
}

void cube_tune_override(const CubeTune* t) { t_override = t; }

}  // namespace edab

namespace {
template <class F>
int guarded_call(F f) {
  try {
    f();
    edab::set_last_error("");
    return EDA_OK;
  } catch (const std::invalid_argument& e) {
    edab::set_last_error(e.what());
    return EDA_INVALID_ARGUMENT;
  } catch (const edab::OutOfMemory& e) {
    edab::set_last_error(e.what());
    return EDA_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    edab::set_last_error(e.what());
    return EDA_CUDA_ERROR;
  }
}
}  // namespace

extern "C" {

EDA_API int eda_autotune(int dtype, int dim, int64_t batch, const int64_t* n, const char* cache_path, char* report,
                         size_t len) {
  return guarded_call([&] {
    if (!n) throw std::invalid_argument("eda: eda_autotune: null extents");
    edab::Params p;
    edab::validate(dtype, dim, batch, n, p);
    const edab::Geom g = edab::make_geom(dim, batch, n);
    cudaStream_t s = nullptr;
    EDAB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    edab::TuneRecord r;
    try {
      r = dtype == EDA_FLOAT32 ? edab::tune_geometry<float>(g, s) : edab::tune_geometry<double>(g, s);
    } catch (...) {
      cudaStreamDestroy(s);
      throw;
    }
    cudaStreamDestroy(s);
    std::lock_guard<std::mutex> lock(edab::g_mu);
    edab::load_env_once_locked();
    edab::g_table[edab::key_of(g, dtype == EDA_FLOAT32 ? 4 : 8)] = r;
    if (cache_path && *cache_path) {
      std::ofstream out(cache_path, std::ios::trunc);
      if (!out) throw std::invalid_argument(std::string("eda: cannot write the tuning cache ") + cache_path);
      out << edab::dump_locked();
    }
    char js[512];
    std::snprintf(js, sizeof js,
                  "{\"lines\": %d, \"groups\": %d, \"seq_share\": %d, \"us_default\": %.1f, \"us_best\": %.1f}",
                  r.tune.lines, r.tune.groups, r.tune.seq_share, r.us_default, r.us_best);
    edab::put(report, len, js);
  });
}

EDA_API int eda_tuning_load(const char* cache_path) {
  return guarded_call([&] {
    if (!cache_path) throw std::invalid_argument("eda: eda_tuning_load: null path");
    std::lock_guard<std::mutex> lock(edab::g_mu);
    edab::g_env_loaded = true;
    edab::load_file_locked(cache_path);
  });
}

EDA_API int eda_tuning_dump(char* buf, size_t len) {
  return guarded_call([&] {
    std::lock_guard<std::mutex> lock(edab::g_mu);
    edab::put(buf, len, edab::dump_locked());
  });
}

EDA_API int eda_tuning_clear(void) {
  return guarded_call([&] {
    std::lock_guard<std::mutex> lock(edab::g_mu);
    edab::g_table.clear();
    edab::g_env_loaded = true;
  });
}

}  // extern "C"
