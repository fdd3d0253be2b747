// SPDX-License-Identifier: Apache-2.0
// The statistics of a mode: canonical energies, exact selections, the noise levels, the local
// threshold field, the significant extrema, the raw local window, the scale field with its
// face-connected components and the per-voxel floor, G2's rung test and G3's coarse median.
// Semantics of eda-cuda (cpp/src/method/stats*.cu, cpp/src/field/common.cuh:133-259); every
// decision is an integer reduction or an exact order statistic, so nothing depends on the order
// of atomics or on the launch shape.
#include "engine.cuh"

#include <algorithm>
#include <cmath>

namespace edab {
namespace {

// ---------------------------------------------------------------------------------------------
// Canonical energies. A warp per row: sum v^2 in double over each 32-sample chunk (sequential),
// the pairwise tree over the chunks padded with zeros to a power of two (32 chunks per warp step
// by shuffles, the steps' sums by a binary-counter stack), and the exact max |v|.
struct RowPartial {
  double sum_sq;
  uint64_t amax;
};

__device__ __forceinline__ double warp_tree32(double v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double o = __shfl_down_sync(0xffffffffu, v, d);
    if ((lane & (2 * d - 1)) == 0) v = __dadd_rn(v, o);
  }
  return v;  // lane 0
}

template <class T>
__global__ void __launch_bounds__(kThreads) row_partials(const T* __restrict__ f, Geom g, RowPartial* rows,
                                                         uint64_t* nonfinite) {
  const int lane = threadIdx.x & 31;
  const int64_t total = g.batch * g.rows;
  const int32_t n = g.n_last;
  const int32_t nchunks = (n + 31) >> 5;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  for (int64_t q = blockIdx.x * static_cast<int64_t>(kThreads / 32) + (threadIdx.x >> 5); q < total; q += warps) {
    const T* row = f + q * g.pitch;
    uint64_t amax = 0;
    unsigned bad = 0;
    double stack[24];
    int level[24];
    int top = 0;
    for (int32_t c0 = 0; c0 < nchunks; c0 += 32) {
      const int32_t c = c0 + lane;
      double acc = 0.0;
      if (c < nchunks) {
        const int32_t e1 = min(c * 32 + 32, n);
        for (int32_t e = c * 32; e < e1; ++e) {
          const T v = row[e];
          const double d = static_cast<double>(v);
          acc = __dadd_rn(acc, __dmul_rn(d, d));
          const uint64_t ab = abs_bits(v);
          amax = ab > amax ? ab : amax;
          bad += isfinite(d) ? 0u : 1u;
        }
      }
      double v = warp_tree32(acc);
      if (lane == 0) {
        int l = 0;
        while (top > 0 && level[top - 1] == l) {
          v = __dadd_rn(stack[top - 1], v);
          --top;
          ++l;
        }
        stack[top] = v;
        level[top] = l;
        ++top;
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      const uint64_t o = __shfl_down_sync(0xffffffffu, amax, d);
      amax = o > amax ? o : amax;
      bad += __shfl_down_sync(0xffffffffu, bad, d);
    }
    if (lane == 0) {
      double v = stack[top - 1];
      for (int i = top - 2; i >= 0; --i) v = __dadd_rn(stack[i], v);
      rows[q] = RowPartial{v, amax};
      if (nonfinite && bad) atomicAdd(reinterpret_cast<unsigned long long*>(&nonfinite[q / g.rows]), bad);
    }
  }
}

// One CTA per element: the pairwise tree over the element's row sums (leaves of 1024 rows in
// shared memory, the leaves by a binary-counter stack), the max of the row maxima.
constexpr int kLeaf = 1024;
__global__ void __launch_bounds__(kThreads) element_totals(Geom g, const RowPartial* rows, double* energy,
                                                           double* amax_out) {
  __shared__ double leaf[kLeaf];
  __shared__ uint64_t am[kThreads / 32];
  const int tid = threadIdx.x;
  for (int64_t b = blockIdx.x; b < g.batch; b += gridDim.x) {
    const RowPartial* base = rows + b * g.rows;
    double stack[40];
    int level[40];
    int top = 0;
    uint64_t amax = 0;
    for (int64_t start = 0; start < g.rows; start += kLeaf) {
      for (int k = 0; k < kLeaf / kThreads; ++k) {
        const int i = tid + k * kThreads;
        double v = 0.0;
        if (start + i < g.rows) {
          const RowPartial p = base[start + i];
          v = p.sum_sq;
          amax = p.amax > amax ? p.amax : amax;
        }
        leaf[i] = v;
      }
      __syncthreads();
      for (int d = 1; d < kLeaf; d <<= 1) {
        for (int i = tid * 2 * d; i < kLeaf; i += kThreads * 2 * d) leaf[i] = __dadd_rn(leaf[i], leaf[i + d]);
        __syncthreads();
      }
      if (tid == 0) {
        double v = leaf[0];
        int l = 0;
        while (top > 0 && level[top - 1] == l) {
          v = __dadd_rn(stack[top - 1], v);
          --top;
          ++l;
        }
        stack[top] = v;
        level[top] = l;
        ++top;
      }
      __syncthreads();
    }
    for (int d = 16; d > 0; d >>= 1) {
      const uint64_t o = __shfl_down_sync(0xffffffffu, amax, d);
      amax = o > amax ? o : amax;
    }
    if ((tid & 31) == 0) am[tid >> 5] = amax;
    __syncthreads();
    if (tid == 0) {
      double v = 0.0;
      if (top > 0) {
        v = stack[top - 1];
        for (int i = top - 2; i >= 0; --i) v = __dadd_rn(stack[i], v);
      }
      uint64_t m = 0;
      for (int w = 0; w < kThreads / 32; ++w) m = am[w] > m ? am[w] : m;
      if (energy) energy[b] = v;
      if (amax_out) amax_out[b] = bits_d(m);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// Selections: MSD radix select over the 64-bit order keys of the values (as doubles), 11-bit
// digits (six passes: 11 x 5 + 9), two ranks at once (a median's middle pair, a quantile's
// neighbours). Histograms: shared-memory u32 bins flushed into u64 global bins.
constexpr int kSelBits = 11;
constexpr int kSelBins = 1 << kSelBits;
constexpr int kSelPasses = 6;

struct alignas(16) SelState {
  uint64_t prefix[2];
  uint64_t rank[2];
  int64_t count;
  double gamma;
  int32_t valid, same;
};

__device__ __forceinline__ uint64_t sel_key(double d) {
  uint64_t u = static_cast<uint64_t>(__double_as_longlong(d));
  if ((u << 1) == 0) u = 0;
  return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}
__device__ __forceinline__ double sel_value(uint64_t k) {
  const uint64_t u = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
  return bits_d(u);
}

template <class T>
struct SelView {
  Sel<T> sel;
  int32_t naxes;
  int32_t ax[kMaxDim];
  int64_t items;
};

template <class T>
__device__ __forceinline__ bool sel_item(const Geom& g, const SelView<T>& a, int64_t b, int64_t t, double* out) {
  double val;
  if (a.sel.src == SelSrc::kField) {
    if (is_pad(g, t)) return false;
    const int64_t i = b * g.field + t;
    if (a.sel.mask != nullptr && (a.sel.mask[i] & a.sel.bits) == 0) return false;
    val = static_cast<double>(a.sel.field[i]);
  } else {
#ifdef __CUDA_ARCH__
    const int64_t k = static_cast<int64_t>(__umul64hi(static_cast<uint64_t>(t), g.field_inv));  // t < 3 field
#else
    const int64_t k = t / g.field;
#endif
    const int64_t v = t - k * g.field;
    const int axis = k == 0 ? a.ax[0] : (k == 1 ? a.ax[1] : a.ax[2]);
    if (is_pad(g, v) || coord_of(g, v, axis) >= geom_n(g, axis) - 1) return false;
    const int64_t i = b * g.field + v;
    const int64_t st = axis == g.dim - 1 ? 1 : geom_stride(g, axis);
    val = static_cast<double>(sub_rn(a.sel.field[i + st], a.sel.field[i]));
  }
  if (a.sel.center != nullptr) val = fabs(__dsub_rn(val, a.sel.center[b]));
  *out = val;
  return true;
}

template <class T>
__global__ void __launch_bounds__(kThreads) sel_hist(Geom g, SelView<T> a, const int32_t* run, SelState* st,
                                                     uint64_t* hist, int32_t nblk, int32_t shift, int32_t width,
                                                     int32_t first) {
  __shared__ uint32_t h[2][kSelBins];
  const int64_t b = blockIdx.y;
  if (run && !run[b]) return;
  const SelState S = st[b];
  if (!first && !S.valid) return;
  const int nr = (first || S.same) ? 1 : 2;
  for (int i = threadIdx.x; i < 2 * kSelBins; i += blockDim.x) h[i / kSelBins][i % kSelBins] = 0u;
  __syncthreads();
  const int hi = shift + width;
  const uint64_t dmask = (1ULL << width) - 1ULL;
  const int64_t stride = static_cast<int64_t>(nblk) * blockDim.x;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < a.items; t += stride) {
    double v;
    if (!sel_item(g, a, b, t, &v)) continue;
    const uint64_t k = sel_key(v);
    const uint32_t bin = static_cast<uint32_t>((k >> shift) & dmask);
    if (first) {
      atomicAdd(&h[0][bin], 1u);
    } else {
      if ((k >> hi) == (S.prefix[0] >> hi)) atomicAdd(&h[0][bin], 1u);
      if (nr == 2 && (k >> hi) == (S.prefix[1] >> hi)) atomicAdd(&h[1][bin], 1u);
    }
  }
  __syncthreads();
  const int nb = 1 << width;
  for (int i = threadIdx.x; i < nr * nb; i += blockDim.x) {
    const int r = i / nb, bin = i % nb;
    const uint32_t c = h[r][bin];
    if (c) atomicAdd(reinterpret_cast<unsigned long long*>(&hist[(b * 2 + r) * kSelBins + bin]), static_cast<unsigned long long>(c));
  }
}

// NumPy's linear quantile index ((n - 1) q; ends clamped) and the end-exact lerp.
__device__ __forceinline__ void q_index(int64_t n, double q, int64_t* i, int64_t* j, double* gamma) {
  const double v = __dmul_rn(static_cast<double>(n - 1), q);
  if (v >= static_cast<double>(n - 1)) {
    *i = *j = n - 1;
    *gamma = __dadd_rn(v, 1.0);
  } else if (v < 0.0) {
    *i = *j = 0;
    *gamma = v;
  } else {
    const double fl = floor(v);
    *i = static_cast<int64_t>(fl);
    *j = *i + 1;
    *gamma = __dsub_rn(v, fl);
  }
}
__device__ __forceinline__ double q_lerp(double a, double b, double gamma) {
  const double diff = __dsub_rn(b, a);
  return gamma >= 0.5 ? __dsub_rn(b, __dmul_rn(diff, __dsub_rn(1.0, gamma))) : __dadd_rn(a, __dmul_rn(diff, gamma));
}

__global__ void __launch_bounds__(kThreads) sel_pick(const int32_t* run, SelState* st, uint64_t* hist, int32_t shift,
                                                     int32_t width, int32_t first, double q) {
  __shared__ uint64_t part[kThreads];
  __shared__ uint64_t base[kThreads];
  __shared__ SelState S;
  __shared__ int32_t found_bin;
  __shared__ uint64_t found_rank;
  const int64_t b = blockIdx.x;
  if (run && !run[b]) return;
  const int tid = threadIdx.x;
  if (tid == 0) S = st[b];
  __syncthreads();
  if (!first && !S.valid) return;
  const int nb = 1 << width;
  const int per = nb / kThreads;
  uint64_t* h0 = hist + (b * 2) * kSelBins;
  if (first) {
    uint64_t sum = 0;
    for (int j = 0; j < per; ++j) sum += h0[tid * per + j];
    part[tid] = sum;
    __syncthreads();
    if (tid == 0) {
      uint64_t n = 0;
      for (int t = 0; t < kThreads; ++t) n += part[t];
      S.count = static_cast<int64_t>(n);
      S.valid = n > 0;
      S.prefix[0] = S.prefix[1] = 0;
      S.same = 1;
      if (n > 0) {
        if (q < 0) {
          S.rank[0] = (n - 1) / 2;
          S.rank[1] = n / 2;
        } else {
          int64_t i = 0, j = 0;
          double gm = 0.0;
          q_index(static_cast<int64_t>(n), q, &i, &j, &gm);
          S.gamma = gm;
          S.rank[0] = static_cast<uint64_t>(i);
          S.rank[1] = static_cast<uint64_t>(j);
        }
      }
    }
    __syncthreads();
    if (!S.valid) {
      if (tid == 0) st[b] = S;
      return;
    }
  }
  for (int r = 0; r < 2; ++r) {
    const uint64_t* hr = hist + (b * 2 + (S.same ? 0 : r)) * kSelBins;
    uint64_t sum = 0;
    for (int j = 0; j < per; ++j) sum += hr[tid * per + j];
    part[tid] = sum;
    __syncthreads();
    if (tid == 0) {
      uint64_t acc = 0;
      for (int t = 0; t < kThreads; ++t) {
        base[t] = acc;
        acc += part[t];
      }
    }
    __syncthreads();
    const uint64_t rank = S.rank[r];
    if (rank >= base[tid] && rank < base[tid] + part[tid]) {
      uint64_t acc = base[tid];
      for (int j = 0; j < per; ++j) {
        const uint64_t c = hr[tid * per + j];
        if (rank < acc + c) {
          found_bin = tid * per + j;
          found_rank = rank - acc;
          break;
        }
        acc += c;
      }
    }
    __syncthreads();
    if (tid == 0) {
      S.prefix[r] |= static_cast<uint64_t>(found_bin) << shift;
      S.rank[r] = found_rank;
    }
    __syncthreads();
  }
  for (int i = tid; i < 2 * kSelBins; i += kThreads) h0[i] = 0;
  if (tid == 0) {
    S.same = S.prefix[0] == S.prefix[1];
    st[b] = S;
  }
}

// low: key bits below the last digit the passes resolved; every item sharing the resolved prefix
// has the same low bits (float values: zeros for keys of non-negative values, ones for negative).
__global__ void sel_final(int64_t B, const int32_t* run, const SelState* st, double q, double* out, int64_t* count,
                          int32_t low) {
  const int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= B || (run && !run[b])) return;
  const SelState S = st[b];
  if (count) count[b] = S.valid ? S.count : 0;
  if (!S.valid) {
    out[b] = d_nan();
    return;
  }
  const uint64_t lm = low > 0 ? (1ULL << low) - 1ULL : 0ULL;
  const double a = sel_value(S.prefix[0] | ((S.prefix[0] >> 63) ? 0ULL : lm));
  const double c = sel_value(S.prefix[1] | ((S.prefix[1] >> 63) ? 0ULL : lm));
  if (q < 0) out[b] = S.count % 2 ? a : (a + c) / 2.0;
  else out[b] = q_lerp(a, c, S.gamma);
}

__global__ void sel_init(int64_t B, const int32_t* run, SelState* st, uint64_t* hist) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= B * 2 * kSelBins) return;
  const int64_t b = i / (2 * kSelBins);
  if (run && !run[b]) return;
  hist[i] = 0;
  if (i % (2 * kSelBins) == 0) st[b] = SelState{};
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

size_t totals_scratch_bytes(const Geom& g) {
  return align256(static_cast<size_t>(g.batch * g.rows) * sizeof(RowPartial));
}

template <class T>
void field_totals(cudaStream_t s, const Geom& g, const T* f, double* energy, double* amax, uint64_t* nonfinite,
                  void* scratch) {
  auto* rows = static_cast<RowPartial*>(scratch);
  const int64_t total = g.batch * g.rows;
  int64_t blocks = (total + (kThreads / 32) - 1) / (kThreads / 32);
  blocks = std::clamp<int64_t>(blocks, 1, int64_t{1} << 20);
  row_partials<T><<<static_cast<unsigned>(blocks), kThreads, 0, s>>>(f, g, rows, nonfinite);
  EDAB_LAUNCH("row_partials");
  const unsigned eb = static_cast<unsigned>(std::clamp<int64_t>(g.batch, 1, 65535));
  element_totals<<<eb, kThreads, 0, s>>>(g, rows, energy, amax);
  EDAB_LAUNCH("element_totals");
}

size_t select_scratch_bytes(const Geom& g) {
  return align256(static_cast<size_t>(g.batch) * sizeof(SelState)) +
         align256(static_cast<size_t>(g.batch) * 2 * kSelBins * sizeof(uint64_t));
}

template <class T>
void select(cudaStream_t s, const Geom& g, const Sel<T>& sel, double q, const int32_t* run, double* out,
            int64_t* count, void* scratch) {
  SelView<T> a{};
  a.sel = sel;
  if (sel.src == SelSrc::kField) {
    a.naxes = 1;
    a.items = g.field;
  } else {
    for (int ax = 0; ax < g.dim; ++ax) {
      if (sel.axes & (1u << ax)) a.ax[a.naxes++] = ax;
    }
    a.items = static_cast<int64_t>(a.naxes) * g.field;
  }
  const int64_t B = g.batch;
  auto* st = static_cast<SelState*>(scratch);
  auto* hist = reinterpret_cast<uint64_t*>(static_cast<char*>(scratch) + align256(static_cast<size_t>(B) * sizeof(SelState)));
  sel_init<<<blocks_for(B * 2 * kSelBins), kThreads, 0, s>>>(B, run, st, hist);
  EDAB_LAUNCH("sel_init");
  int64_t nblk = (a.items + int64_t{kThreads} * 32 - 1) / (int64_t{kThreads} * 32);
  nblk = std::clamp<int64_t>(nblk, 1, 1024);
  if (B > 65535) throw std::invalid_argument("edab: select batch too large");
  // float items (a float32 field or its float32 differences, no centre) have double keys whose low
  // 29 bits depend only on the sign: four passes resolve every bit above bit 20
  const int passes = std::is_same_v<T, float> && sel.center == nullptr ? 4 : kSelPasses;
  int low = 0;
  for (int p = 0; p < passes; ++p) {
    const int top = 64 - kSelBits * p;
    const int shift = top - kSelBits > 0 ? top - kSelBits : 0;
    const int width = top - shift;
    sel_hist<T><<<dim3(static_cast<unsigned>(nblk), static_cast<unsigned>(B)), kThreads, 0, s>>>(
        g, a, run, st, hist, static_cast<int32_t>(nblk), shift, width, p == 0);
    EDAB_LAUNCH("sel_hist");
    sel_pick<<<static_cast<unsigned>(B), kThreads, 0, s>>>(run, st, hist, shift, width, p == 0, q);
    EDAB_LAUNCH("sel_pick");
    low = shift;
  }
  sel_final<<<blocks_for(B), kThreads, 0, s>>>(B, run, st, q, out, count, low);
  EDAB_LAUNCH("sel_final");
}

// ---------------------------------------------------------------------------------------------
// Significant extrema (cpp/src/method/stats_fields.cu:1-14, 182-331 of eda-cuda): the peaks of r
// and -r along every line as scipy.signal.find_peaks defines them, with topographic prominence
// >= tau at the peak. A CTA stages P lines in shared memory with their 32-sample block minima and
// maxima; the thread of a run start owns a peak and walks each side over samples, then whole
// blocks (entering a block only where it holds the side's end).
namespace {

constexpr int kBlk = 32;

// fl64(a - b) >= tau: for float the float difference decides except on a tie with tau.
template <class T>
__device__ __forceinline__ bool deep(T a, T b, T tau) {
  if constexpr (std::is_same_v<T, float>) {
    const float d = __fsub_rn(a, b);
    if (d != tau) return d > tau;
    return __dsub_rn(static_cast<double>(a), static_cast<double>(b)) >= static_cast<double>(tau);
  } else {
    return __dsub_rn(a, b) >= tau;
  }
}

template <bool Max, class T>
__device__ __forceinline__ int side_step(T u, T v, T tau) {
  if (Max ? !(u <= v) : !(u >= v)) return 2;
  return (Max ? deep<T>(v, u, tau) : deep<T>(u, v, tau)) ? 1 : 0;
}

// Sample k of a staged line: one pad word after every 32 samples (the lanes of a warp scanning
// consecutive blocks hit distinct banks).
template <class T>
__device__ __forceinline__ T xs(const T* x, int32_t k) {
  return x[k + (k >> 5)];
}

template <bool Max, int Dir, class T>
__device__ bool side_deep(const T* x, int32_t n, int32_t p, T v, T tau, const T* bmin, const T* bmax) {
  const int32_t cp = p / kBlk;
  const int32_t lim = Dir < 0 ? cp * kBlk : min(cp * kBlk + kBlk - 1, n - 1);
  for (int32_t k = p + Dir; Dir < 0 ? k >= lim : k <= lim; k += Dir) {
    const int st = side_step<Max>(xs(x, k), v, tau);
    if (st) return st == 1;
  }
  const int32_t nb = (n + kBlk - 1) / kBlk;
  for (int32_t c = cp + Dir; Dir < 0 ? c >= 0 : c < nb; c += Dir) {
    const T hi = Max ? bmax[c] : bmin[c];
    if (Max ? !(hi <= v) : !(hi >= v)) {
      const int32_t k0 = Dir < 0 ? c * kBlk + kBlk - 1 : c * kBlk;
      const int32_t k1 = Dir < 0 ? c * kBlk : min(c * kBlk + kBlk - 1, n - 1);
      for (int32_t k = k0; Dir < 0 ? k >= k1 : k <= k1; k += Dir) {
        const int st = side_step<Max>(xs(x, k), v, tau);
        if (st) return st == 1;
      }
      return false;
    }
    const T lo = Max ? bmin[c] : bmax[c];
    if (Max ? deep<T>(v, lo, tau) : deep<T>(lo, v, tau)) return true;
  }
  return false;
}

// Staged lines: P lines of LX words (sample k at k + k / 32; LX odd, so lanes on consecutive lines
// hit distinct banks), then the block minima and maxima. Rows: threads over the samples of a line;
// column panels: lanes over the panel's columns (coalesced tau reads and flag writes).
template <class T>
__global__ void __launch_bounds__(kThreads) flags_pass(Geom g, int axis, const T* __restrict__ r,
                                                       const T* __restrict__ tau, uint8_t* __restrict__ flags,
                                                       Elem* el, const int32_t* run, int P, int32_t LX) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int64_t b = blockIdx.y;
  if (run && !run[b]) return;
  const int32_t n = geom_n(g, axis);
  const bool contig = axis == g.dim - 1;
  const int32_t nb = (n + kBlk - 1) / kBlk;
  T* X = reinterpret_cast<T*>(smem_raw);
  T* bmin = X + static_cast<int64_t>(P) * LX;
  T* bmax = bmin + static_cast<int64_t>(P) * nb;
  __shared__ int64_t base_s[64];
  __shared__ int32_t ok_s[64];
  __shared__ int32_t count_s;
  const int64_t grp = blockIdx.x;
  if (threadIdx.x < P) {
    const int p = threadIdx.x;
    bool ok;
    int64_t base;
    if (contig) {
      const int64_t row = grp * P + p;
      ok = row < g.rows;
      base = row * g.pitch;
    } else {
      const int64_t inner = geom_stride(g, axis);
      const int64_t gpo = (inner + P - 1) / P;
      const int64_t o = grp / gpo;
      const int64_t c = (grp - o * gpo) * P + p;
      ok = c < inner && (c % g.pitch) < g.n_last;
      base = o * static_cast<int64_t>(n) * inner + c;
    }
    base_s[p] = base;
    ok_s[p] = ok ? 1 : 0;
  }
  if (threadIdx.x == 0) count_s = 0;
  const int64_t step = contig ? 1 : geom_stride(g, axis);
  const int64_t eoff = b * g.field;
  __syncthreads();
  if (contig) {
    // lines in turn, consecutive samples over the threads
    for (int p = 0; p < P; ++p) {
      if (!ok_s[p]) continue;
      const T* src = r + eoff + base_s[p];
      T* x = X + p * LX;
      for (int32_t i = threadIdx.x; i < n; i += blockDim.x) x[i + (i >> 5)] = src[i];
    }
  } else {
    // the P columns of a row over consecutive threads (whole sectors); one division per thread
    const int32_t rows_per = static_cast<int32_t>(blockDim.x) / P;
    const int p = static_cast<int>(threadIdx.x % P);
    const int32_t i0 = static_cast<int32_t>(threadIdx.x / P);
    if (i0 < rows_per && ok_s[p]) {
      const T* src = r + eoff + base_s[p];
      T* x = X + p * LX;
      for (int32_t i = i0; i < n; i += rows_per) x[i + (i >> 5)] = src[static_cast<int64_t>(i) * step];
    }
  }
  __syncthreads();
  for (int32_t t = threadIdx.x; t < P * nb; t += blockDim.x) {
    const int p = t / nb;
    const int32_t c = t - p * nb;
    if (!ok_s[p]) continue;
    const T* xb = X + p * LX + c * (kBlk + 1);  // block c, stored contiguously
    const int32_t len = min(kBlk, n - c * kBlk);
    T mn = xb[0], mx = mn;
    for (int32_t i = 1; i < len; ++i) {
      const T v = xb[i];
      mn = (v < mn || v != v) ? v : mn;
      mx = (v > mx || v != v) ? v : mx;
    }
    bmin[p * nb + c] = mn;
    bmax[p * nb + c] = mx;
  }
  __syncthreads();
  int mine = 0;
  // the run of samples equal to x[s] from s (s a run start): significant extremum -> flag its peak
  const auto visit = [&](int p, int32_t s) {
    const T* x = X + p * LX;
    // the threshold at s, read for every sample (coalesced over the warp) ahead of its use at a peak
    const T tp_s = tau[eoff + base_s[p] + s * step];
    const T cur = xs(x, s), prev = xs(x, s - 1);
    if (!(prev < cur || prev > cur)) return;
    const T* pmin = bmin + p * nb;
    const T* pmax = bmax + p * nb;
    int32_t e;
    {
      const int32_t lim = min((s / kBlk) * kBlk + kBlk - 1, n - 1);
      int32_t k = s + 1;
      while (k <= lim && xs(x, k) == cur) ++k;
      if (k <= lim || k >= n) {
        e = k - 1;
      } else {
        e = n - 1;
        for (int32_t c = k / kBlk; c < nb; ++c) {
          if (pmin[c] == cur && pmax[c] == cur) continue;
          k = c * kBlk;
          while (xs(x, k) == cur) ++k;
          e = k - 1;
          break;
        }
      }
    }
    if (e > n - 2) return;
    const T nxt = xs(x, e + 1);
    const bool is_max = prev < cur && nxt < cur;
    const bool is_min = prev > cur && nxt > cur;
    if (!is_max && !is_min) return;
    const int32_t pk = (s + e) / 2;
    const int64_t at = eoff + base_s[p] + pk * step;
    const T tp = pk == s ? tp_s : tau[at];
    const bool sig = is_max ? side_deep<true, -1>(x, n, pk, cur, tp, pmin, pmax) && side_deep<true, 1>(x, n, pk, cur, tp, pmin, pmax)
                            : side_deep<false, -1>(x, n, pk, cur, tp, pmin, pmax) && side_deep<false, 1>(x, n, pk, cur, tp, pmin, pmax);
    if (sig) {
      flags[at] |= static_cast<uint8_t>(1u << axis);
      ++mine;
    }
  };
  if (contig) {
    for (int p = 0; p < P; ++p) {
      if (!ok_s[p]) continue;
      for (int32_t s = 1 + threadIdx.x; s <= n - 2; s += blockDim.x) visit(p, s);
    }
  } else {
    // lanes over the panel's columns; a warp covers 32 / P rows (P a power of two <= 32)
    const int p = threadIdx.x & (P - 1);
    const int32_t rpw = 32 / P;
    const int32_t nrows = static_cast<int32_t>(blockDim.x >> 5) * rpw;
    if (ok_s[p]) {
      for (int32_t s = 1 + static_cast<int32_t>(threadIdx.x / P); s <= n - 2; s += nrows) visit(p, s);
    }
  }
  for (int d = 16; d > 0; d >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, d);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&count_s, mine);
  __syncthreads();
  if (threadIdx.x == 0 && count_s) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&el[b].ext[axis]), static_cast<unsigned long long>(count_s));
  }
}

// ---------------------------------------------------------------------------------------------
// Face-connected components: union-find over the padded in-element indices with atomicMin links
// (a parent is always smaller than its child), so the root of a component is its smallest index
// whatever the order of the atomics; a final pass writes every voxel's root.
__device__ __forceinline__ int32_t find_root(const int32_t* L, int32_t x) {
  const volatile int32_t* V = L;
  int32_t p = V[x];
  while (p != x) {
    x = p;
    p = V[x];
  }
  return x;
}
__device__ __forceinline__ void unite(int32_t* L, int32_t a, int32_t c) {
  for (;;) {
    a = find_root(L, a);
    c = find_root(L, c);
    if (a == c) return;
    if (a > c) {
      const int32_t t = a;
      a = c;
      c = t;
    }
    const int32_t old = atomicMin(L + c, a);
    if (old == c) return;
    c = old;
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
template <class T>
void sig_flags(cudaStream_t s, const Geom& g, const T* r, const T* tau, uint8_t* flags, Elem* el, const int32_t* run) {
  for_samples(s, g.batch * g.field, [=] __device__(int64_t i) {
    if (run == nullptr || run[elem_of(g, i)]) flags[i] = 0;
  });
  int optin = 0, dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  EDAB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t cap = static_cast<size_t>(optin) - 2048;
  static bool attr_set[2] = {false, false};
  if (!attr_set[sizeof(T) == 8]) {
    EDAB_CUDA(cudaFuncSetAttribute(flags_pass<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cap)));
    attr_set[sizeof(T) == 8] = true;
  }
  for (int a = 0; a < g.dim; ++a) {
    const int32_t n = g.n[a];
    if (n < 3) continue;
    const int32_t nb = (n + kBlk - 1) / kBlk;
    int P;
    if (a == g.dim - 1) P = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>({static_cast<int64_t>(8192 / n), g.rows, 64})));
    else P = static_cast<int>(std::min<int64_t>(16, g.stride[a]));  // a power of two (stride: a multiple of 32)
    const int32_t LX = (n + ((n - 1) >> 5) + 1) | 1;  // padded line words, odd
    const auto bytes = [&](int p) { return static_cast<size_t>(p) * (LX + 2 * nb) * sizeof(T); };
    while (P > 1 && bytes(P) > cap) P = a == g.dim - 1 ? P - 1 : P / 2;
    if (bytes(P) > cap) throw std::invalid_argument("edab: a line exceeds the shared memory of the extrema pass");
    int64_t groups;
    if (a == g.dim - 1) {
      groups = (g.rows + P - 1) / P;
    } else {
      int64_t outer = 1;
      for (int ax = 0; ax < a; ++ax) outer *= g.n[ax];
      groups = outer * ((g.stride[a] + P - 1) / P);
    }
    flags_pass<T><<<dim3(static_cast<unsigned>(groups), static_cast<unsigned>(g.batch)), kThreads, bytes(P), s>>>(
        g, a, r, tau, flags, el, run, P, LX);
    EDAB_LAUNCH("flags_pass");
  }
}

void ccl(cudaStream_t s, const Geom& g, const uint8_t* mask, uint8_t bits, int32_t* labels, const int32_t* run) {
  const int64_t total = g.batch * g.field;
  for_samples(s, total, [=] __device__(int64_t i) {
    const int64_t b = elem_of(g, i);
    if (run && !run[b]) return;
    const int64_t v = i - b * g.field;
    labels[i] = (!is_pad(g, v) && (mask[i] & bits) != 0) ? static_cast<int32_t>(v) : -1;
  });
  for_samples(s, total, [=] __device__(int64_t i) {
    const int64_t b = elem_of(g, i);
    if (run && !run[b]) return;
    int32_t* L = labels + b * g.field;
    const int32_t v = static_cast<int32_t>(i - b * g.field);
    if (L[v] < 0) return;
    for (int a = 0; a < g.dim; ++a) {
      if (coord_of(g, v, a) + 1 >= geom_n(g, a)) continue;
      const int32_t u = v + static_cast<int32_t>(a == g.dim - 1 ? 1 : geom_stride(g, a));
      if (L[u] < 0) continue;
      unite(L, v, u);
    }
  });
  for_samples(s, total, [=] __device__(int64_t i) {
    const int64_t b = elem_of(g, i);
    if (run && !run[b]) return;
    int32_t* L = labels + b * g.field;
    const int32_t v = static_cast<int32_t>(i - b * g.field);
    if (L[v] < 0) return;
    const int32_t root = find_root(L, v);
    reinterpret_cast<volatile int32_t*>(L)[v] = root;
  });
}

template void field_totals<float>(cudaStream_t, const Geom&, const float*, double*, double*, uint64_t*, void*);
template void field_totals<double>(cudaStream_t, const Geom&, const double*, double*, double*, uint64_t*, void*);
template void select<float>(cudaStream_t, const Geom&, const Sel<float>&, double, const int32_t*, double*, int64_t*, void*);
template void select<double>(cudaStream_t, const Geom&, const Sel<double>&, double, const int32_t*, double*, int64_t*, void*);
template void sig_flags<float>(cudaStream_t, const Geom&, const float*, const float*, uint8_t*, Elem*, const int32_t*);
template void sig_flags<double>(cudaStream_t, const Geom&, const double*, const double*, uint8_t*, Elem*, const int32_t*);

}  // namespace edab
