// SPDX-License-Identifier: Apache-2.0
// The statistics of a mode: canonical energies, exact selections, the noise levels, the local
// threshold field, the significant extrema, the raw local window, the scale field with its
// face-connected components and the per-voxel floor, G2's rung test and G3's coarse median.
// Semantics of eda-cuda (cpp/src/method/stats*.cu, cpp/src/field/common.cuh:133-259); every
// decision is an integer reduction or an exact order statistic, so nothing depends on the order
// of atomics or on the launch shape.
#include "engine.cuh"

#include <cooperative_groups.h>

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
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  for (int64_t q = blockIdx.x * static_cast<int64_t>(kThreads / 32) + (threadIdx.x >> 5); q < total; q += warps) {
    const int32_t n = g.len ? elem_len(g, q / g.rows) : g.n_last;
    const int32_t nchunks = (n + 31) >> 5;
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
// Exact selections (order statistics) by most-significant-digit radix selection on order keys,
// unsigned integers that sort as the values do (-0 counts as +0). Float32 items without a centre
// select on 32-bit keys of the float values (three digits: 11, 11 and 10 bits); every other
// selection on 64-bit keys of the values as doubles (six digits: five of 11 bits, one of 9).
//
// One thread-block cluster (up to 8 CTAs) serves one element, all digits in one launch: each CTA
// counts its share of the items per digit value in shared memory; the counts are added into the
// cluster leader's shared table through distributed shared memory; the leader's threads find the
// digit value that holds the wanted rank by a block-wide prefix sum and publish the extended prefix.
// Two ranks are followed at once (a median's middle pair, a quantile's neighbours); they share one
// table while their resolved digits agree.
namespace cg = cooperative_groups;

constexpr int kDigitBits = 11;
constexpr int kDigitBins = 1 << kDigitBits;
constexpr int kSelClusterMax = 8;
// The cluster form for batches that fill the GPU with clusters (1), or the grid-wide form always (0).
#ifndef EDAB_SEL_CLUSTERS
#define EDAB_SEL_CLUSTERS 1
#endif
constexpr bool kSelClusters = EDAB_SEL_CLUSTERS != 0;
constexpr size_t kSelSmem = 2 * kDigitBins * sizeof(unsigned long long) + 2 * kDigitBins * sizeof(uint32_t);

__device__ __forceinline__ uint32_t order_key(float v) {
  uint32_t u = __float_as_uint(v);
  if ((u & 0x7fffffffu) == 0u) u = 0u;
  return (u & 0x80000000u) ? ~u : (u ^ 0x80000000u);
}
__device__ __forceinline__ uint64_t order_key(double v) {
  uint64_t u = static_cast<uint64_t>(__double_as_longlong(v));
  if ((u & 0x7fffffffffffffffULL) == 0ULL) u = 0ULL;
  return (u >> 63) ? ~u : (u ^ 0x8000000000000000ULL);
}
__device__ __forceinline__ double key_value(uint32_t k) {
  return static_cast<double>(__uint_as_float((k & 0x80000000u) ? (k ^ 0x80000000u) : ~k));
}
__device__ __forceinline__ double key_value(uint64_t k) {
  return bits_d((k >> 63) ? (k ^ 0x8000000000000000ULL) : ~k);
}

template <class T>
struct SelView {
  Sel<T> sel;
  int32_t naxes;
  int32_t ax[kMaxDim];
  int64_t items;
};

// Item t of element b (a voxel, or a forward difference along one of the pooled axes) as a value of
// the element's dtype; false where t is a pad, masked out, or has no forward neighbour.
template <class T>
__device__ __forceinline__ bool sel_raw(const Geom& g, const SelView<T>& a, int64_t b, int64_t t, T* out) {
  if (a.sel.src == SelSrc::kField) {
    if (is_pad_b(g, b, t)) return false;
    const int64_t i = b * g.field + t;
    if (a.sel.mask != nullptr && (a.sel.mask[i] & a.sel.bits) == 0) return false;
    *out = a.sel.field[i];
    return true;
  }
  const int64_t k = static_cast<int64_t>(__umul64hi(static_cast<uint64_t>(t), g.field_inv));  // t < 3 field
  const int64_t v = t - k * g.field;
  const int axis = k == 0 ? a.ax[0] : (k == 1 ? a.ax[1] : a.ax[2]);
  if (is_pad_b(g, b, v) || coord_of(g, v, axis) >= elem_n(g, b, axis) - 1) return false;
  const int64_t i = b * g.field + v;
  const int64_t st = axis == g.dim - 1 ? 1 : geom_stride(g, axis);
  *out = sub_rn(a.sel.field[i + st], a.sel.field[i]);
  return true;
}
template <class T, class K>
__device__ __forceinline__ bool sel_key_of(const Geom& g, const SelView<T>& a, int64_t b, int64_t t, K* key) {
  T v;
  if (!sel_raw(g, a, b, t, &v)) return false;
  if constexpr (sizeof(K) == 4) {
    *key = order_key(static_cast<float>(v));
  } else {
    double d = static_cast<double>(v);
    if (a.sel.center != nullptr) d = fabs(__dsub_rn(d, a.sel.center[b]));
    *key = order_key(d);
  }
  return true;
}

// One shared-memory count per distinct digit among the warp's active lanes (the lanes holding the
// same digit add together through their lowest lane): a field's items crowd into few digit values
// (the sign and exponent bits lead every key), and per-lane atomics on one address serialize.
__device__ __forceinline__ void count_digit(uint32_t* hist, uint32_t digit, bool take) {
  const unsigned active = __ballot_sync(0xffffffffu, take);
  if (!take) return;
  const unsigned same = __match_any_sync(active, digit);
  if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&hist[digit], static_cast<uint32_t>(__popc(same)));
}

// The candidates of a selection: the keys that share the digits resolved before the candidates'
// pass (64-bit keys: two digits, the items within about 2^-10 of the statistic's binade position;
// 32-bit keys: one digit), written while that pass counts, which every later pass reads instead of
// the items. cap keys per element; a selection with more candidates reads the items in every pass
// (the count n keeps growing past cap, nothing is written there).
// The digit pass that writes the candidates (the later passes read them): the third for 64-bit
// keys; the second for 32-bit keys (after one digit: sign, exponent and two mantissa bits, a quarter
// binade of the values; measured 10 % faster on the 2-D benchmark's float32 selections). Building
// with EDAB_SEL_CAND32=0 leaves 32-bit selections without candidates.
#ifndef EDAB_SEL_CAND32
#define EDAB_SEL_CAND32 1
#endif
template <class K>
constexpr int kCandPass = sizeof(K) == 8 ? 2 : 1;

template <class K>
struct SelCand {
  K* keys;               // [B][cap]; nullptr: no candidates
  unsigned long long* n;  // [B]
  int64_t cap;
};
// Appends key k of the lanes with app set (the warp's 32 lanes call it together).
template <class K>
__device__ __forceinline__ void cand_append(const SelCand<K>& c, int64_t b, bool app, K k) {
  const unsigned m = __ballot_sync(0xffffffffu, app);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  const int first = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == first) base = atomicAdd(c.n + b, static_cast<unsigned long long>(__popc(m)));
  base = __shfl_sync(0xffffffffu, base, first);
  if (app) {
    const unsigned long long pos = base + static_cast<unsigned long long>(__popc(m & ((1u << lane) - 1u)));
    if (pos < static_cast<unsigned long long>(c.cap)) c.keys[b * c.cap + static_cast<int64_t>(pos)] = k;
  }
}

template <class K>
struct SelLeader {
  K prefix[2];
  unsigned long long rank[2];
  long long count;
  double gamma;
  int32_t live, same;
};

// The digit value of table tb (nb bins) that holds rank, and the rank inside it: one block-wide
// exclusive prefix sum over the bins (nb / kThreads consecutive bins per thread).
__device__ __forceinline__ void rank_digit(const unsigned long long* tb, int nb, unsigned long long rank,
                                           unsigned long long* warp_tot, int* bin_out,
                                           unsigned long long* rest_out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = nb / kThreads;
  unsigned long long mine = 0;
  for (int j = 0; j < per; ++j) mine += tb[tid * per + j];
  unsigned long long incl = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long o = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += o;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  unsigned long long before = incl - mine;
  for (int w = 0; w < warp; ++w) before += warp_tot[w];
  if (rank >= before && rank < before + mine) {
    unsigned long long acc = before;
    for (int j = 0; j < per; ++j) {
      const unsigned long long c = tb[tid * per + j];
      if (rank < acc + c) {
        *bin_out = tid * per + j;
        *rest_out = rank - acc;
        break;
      }
      acc += c;
    }
  }
  __syncthreads();
}

// NumPy's "linear" quantile: the index (n - 1) q, clamped at the ends, and its fraction.
__device__ __forceinline__ void linear_index(long long n, double q, long long* i, long long* j, double* frac) {
  const double pos = __dmul_rn(static_cast<double>(n - 1), q);
  if (pos >= static_cast<double>(n - 1)) {
    *i = *j = n - 1;
    *frac = __dadd_rn(pos, 1.0);
  } else if (pos < 0.0) {
    *i = *j = 0;
    *frac = pos;
  } else {
    const double whole = floor(pos);
    *i = static_cast<long long>(whole);
    *j = *i + 1;
    *frac = __dsub_rn(pos, whole);
  }
}
// NumPy's interpolation between neighbours: from the nearer end.
__device__ __forceinline__ double linear_between(double lo, double hi, double frac) {
  const double span = __dsub_rn(hi, lo);
  if (frac >= 0.5) return __dsub_rn(hi, __dmul_rn(span, __dsub_rn(1.0, frac)));
  return __dadd_rn(lo, __dmul_rn(span, frac));
}

template <class T, class K>
__global__ void __launch_bounds__(kThreads) select_cluster(Geom g, SelView<T> a, const int32_t* run, double q,
                                                          double* out, int64_t* count_out, SelCand<K> cand) {
  constexpr int kKeyBits = 8 * static_cast<int>(sizeof(K));
  constexpr int kDigits = (kKeyBits + kDigitBits - 1) / kDigitBits;
  extern __shared__ __align__(16) unsigned char sel_smem[];
  auto* table = reinterpret_cast<unsigned long long*>(sel_smem);                                  // leader: [2][bins]
  auto* local = reinterpret_cast<uint32_t*>(sel_smem + 2 * kDigitBins * sizeof(unsigned long long));  // [2][bins]
  __shared__ SelLeader<K> lead;
  __shared__ unsigned long long warp_tot[kThreads / 32];
  __shared__ int hit_bin;
  __shared__ unsigned long long hit_rest;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned me = cl.block_rank();
  const unsigned ctas = cl.num_blocks();
  const int64_t b = blockIdx.y;
  if (run && !run[b]) return;  // every CTA of the cluster leaves here
  const int tid = threadIdx.x;
  const bool leader = me == 0;
  SelLeader<K>* L = cl.map_shared_rank(&lead, 0);
  unsigned long long* T0 = cl.map_shared_rank(table, 0);
  if (leader) {
    for (int i = tid; i < 2 * kDigitBins; i += kThreads) table[i] = 0ULL;
    if (tid == 0) {
      lead.prefix[0] = lead.prefix[1] = K(0);
      lead.live = 1;
      lead.same = 1;
      if (cand.keys) cand.n[b] = 0ULL;
    }
  }
  bool from_cand = false;
  int64_t n_it = a.items;
  for (int pass = 0; pass < kDigits; ++pass) {
    const int hi = kKeyBits - kDigitBits * pass;  // key bits at and above hi are resolved
    const int shift = hi > kDigitBits ? hi - kDigitBits : 0;
    const int width = hi - shift;
    const K dmask = static_cast<K>((K(1) << width) - K(1));
    for (int i = tid; i < 2 * kDigitBins; i += kThreads) local[i] = 0u;
    cl.sync();  // the leader's prefixes and cleared table are visible to the cluster
    const int live = L->live;
    if (!live) break;
    const bool two = pass > 0 && !L->same;
    const K p0 = L->prefix[0], p1 = L->prefix[1];
    if (pass == kCandPass<K> + 1 && cand.keys) {  // the candidates are complete (the barrier above)
      const unsigned long long nc = *reinterpret_cast<volatile unsigned long long*>(cand.n + b);
      from_cand = nc <= static_cast<unsigned long long>(cand.cap);
      if (from_cand) n_it = static_cast<int64_t>(nc);
    }
    const int64_t stride = static_cast<int64_t>(ctas) * kThreads;
    // the warp steps through the items together (count_digit is warp-collective)
    const int64_t t_end = (n_it + 31) / 32 * 32;
    for (int64_t t = static_cast<int64_t>(me) * kThreads + tid; t < t_end + stride; t += stride) {
      if (t - tid % 32 >= n_it) break;  // the warp's first item is past the end: the whole warp leaves
      K k = K(0);
      bool have;
      if (from_cand) {
        have = t < n_it;
        if (have) k = cand.keys[b * cand.cap + t];
      } else {
        have = t < a.items && sel_key_of<T, K>(g, a, b, t, &k);
      }
      const uint32_t digit = static_cast<uint32_t>((k >> shift) & dmask);
      const K top = pass == 0 ? K(0) : (k >> hi);
      count_digit(local, digit, have && (pass == 0 || top == (p0 >> hi)));
      if (two) count_digit(local + kDigitBins, digit, have && top == (p1 >> hi));
      if (pass == kCandPass<K> && cand.keys) cand_append(cand, b, have && (top == (p0 >> hi) || (two && top == (p1 >> hi))), k);
    }
    __syncthreads();
    const int bins = 1 << width;
    for (int i = tid; i < (two ? 2 : 1) * bins; i += kThreads) {
      const int r = i >= bins ? 1 : 0;
      const uint32_t c = local[r * kDigitBins + (i - r * bins)];
      if (c) atomicAdd(&T0[r * kDigitBins + (i - r * bins)], static_cast<unsigned long long>(c));
    }
    cl.sync();  // the cluster's counts are complete in the leader's table
    if (!leader) continue;
    if (pass == 0) {
      // the item count and the ranks of the statistic
      unsigned long long n = 0;
      for (int i = tid; i < bins; i += kThreads) n += table[i];
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) n += __shfl_xor_sync(0xffffffffu, n, d);
      if ((tid & 31) == 0) warp_tot[tid >> 5] = n;
      __syncthreads();
      if (tid == 0) {
        unsigned long long total = 0;
        for (int w = 0; w < kThreads / 32; ++w) total += warp_tot[w];
        lead.count = static_cast<long long>(total);
        lead.live = total > 0;
        if (total > 0) {
          if (q < 0) {
            lead.rank[0] = (total - 1) / 2;
            lead.rank[1] = total / 2;
          } else {
            long long i = 0, j = 0;
            linear_index(static_cast<long long>(total), q, &i, &j, &lead.gamma);
            lead.rank[0] = static_cast<unsigned long long>(i);
            lead.rank[1] = static_cast<unsigned long long>(j);
          }
        }
      }
      __syncthreads();
    }
    if (lead.live) {
      for (int r = 0; r < 2; ++r) {
        rank_digit(table + (two ? r : 0) * kDigitBins, bins, lead.rank[r], warp_tot, &hit_bin, &hit_rest);
        if (tid == 0) {
          lead.prefix[r] |= static_cast<K>(hit_bin) << shift;
          lead.rank[r] = hit_rest;
        }
        __syncthreads();
      }
      if (tid == 0) lead.same = lead.prefix[0] == lead.prefix[1];
    }
    for (int i = tid; i < 2 * kDigitBins; i += kThreads) table[i] = 0ULL;
  }
  cl.sync();  // no CTA reads the leader's shared memory after this
  if (leader && tid == 0) {
    if (!lead.live) {
      out[b] = d_nan();
      if (count_out) count_out[b] = 0;
    } else {
      const double v0 = key_value(lead.prefix[0]), v1 = key_value(lead.prefix[1]);
      out[b] = q < 0 ? ((lead.count & 1) ? v0 : __dmul_rn(__dadd_rn(v0, v1), 0.5)) : linear_between(v0, v1, lead.gamma);
      if (count_out) count_out[b] = lead.count;
    }
  }
}

// The grid-wide form for batches too small to fill the GPU with clusters (few, large elements):
// per digit, a counting launch over many CTAs per element (warp-aggregated shared-memory counts,
// flushed with one global atomic per digit value and CTA) and a pick launch of one CTA per element
// (the same block-wide prefix sum), the element's state in global memory between launches.
template <class K>
struct SelGridState {
  K prefix[2];
  unsigned long long rank[2];
  long long count;
  double gamma;
  int32_t live, same;
};

template <int KeyBits>
__device__ __forceinline__ void digit_of_pass(int pass, int* hi, int* shift, int* width) {
  *hi = KeyBits - kDigitBits * pass;
  *shift = *hi > kDigitBits ? *hi - kDigitBits : 0;
  *width = *hi - *shift;
}

template <class T, class K>
__global__ void __launch_bounds__(kThreads) select_grid_count(Geom g, SelView<T> a, const int32_t* run,
                                                             const SelGridState<K>* st,
                                                             unsigned long long* table, int32_t pass,
                                                             SelCand<K> cand) {
  __shared__ uint32_t local[2 * kDigitBins];
  const int64_t b = blockIdx.y;
  if (run && !run[b]) return;
  bool two = false;
  K p0 = K(0), p1 = K(0);
  if (pass > 0) {
    if (!st[b].live) return;
    two = !st[b].same;
    p0 = st[b].prefix[0];
    p1 = st[b].prefix[1];
  }
  int hi, shift, width;
  digit_of_pass<8 * static_cast<int>(sizeof(K))>(pass, &hi, &shift, &width);
  const K dmask = static_cast<K>((K(1) << width) - K(1));
  const int tid = threadIdx.x;
  for (int i = tid; i < 2 * kDigitBins; i += kThreads) local[i] = 0u;
  __syncthreads();
  // after the candidates pass, its candidates (when they fit) instead of the items
  bool from_cand = false;
  int64_t n_it = a.items;
  if (pass > kCandPass<K> && cand.keys) {
    const unsigned long long nc = cand.n[b];
    from_cand = nc <= static_cast<unsigned long long>(cand.cap);
    if (from_cand) n_it = static_cast<int64_t>(nc);
  }
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kThreads;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kThreads + tid;; t += stride) {
    if (t - tid % 32 >= n_it) break;  // the warp's first item is past the end
    K k = K(0);
    bool have;
    if (from_cand) {
      have = t < n_it;
      if (have) k = cand.keys[b * cand.cap + t];
    } else {
      have = t < a.items && sel_key_of<T, K>(g, a, b, t, &k);
    }
    const uint32_t digit = static_cast<uint32_t>((k >> shift) & dmask);
    const K top = pass == 0 ? K(0) : (k >> hi);
    count_digit(local, digit, have && (pass == 0 || top == (p0 >> hi)));
    if (two) count_digit(local + kDigitBins, digit, have && top == (p1 >> hi));
    if (pass == kCandPass<K> && cand.keys) cand_append(cand, b, have && (top == (p0 >> hi) || (two && top == (p1 >> hi))), k);
  }
  __syncthreads();
  const int bins = 1 << width;
  unsigned long long* tb = table + static_cast<int64_t>(b) * 2 * kDigitBins;
  for (int i = tid; i < (two ? 2 : 1) * bins; i += kThreads) {
    const int r = i >= bins ? 1 : 0;
    const uint32_t c = local[r * kDigitBins + (i - r * bins)];
    if (c) atomicAdd(&tb[r * kDigitBins + (i - r * bins)], static_cast<unsigned long long>(c));
  }
}

template <class K>
__global__ void __launch_bounds__(kThreads) select_grid_pick(const int32_t* run, SelGridState<K>* st,
                                                            unsigned long long* table, int32_t pass, double q,
                                                            double* out, int64_t* count_out) {
  constexpr int kKeyBits = 8 * static_cast<int>(sizeof(K));
  constexpr int kDigits = (kKeyBits + kDigitBits - 1) / kDigitBits;
  __shared__ SelGridState<K> S;
  __shared__ unsigned long long warp_tot[kThreads / 32];
  __shared__ int hit_bin;
  __shared__ unsigned long long hit_rest;
  const int64_t b = blockIdx.x;
  if (run && !run[b]) return;
  const int tid = threadIdx.x;
  int hi, shift, width;
  digit_of_pass<kKeyBits>(pass, &hi, &shift, &width);
  const int bins = 1 << width;
  unsigned long long* tb = table + static_cast<int64_t>(b) * 2 * kDigitBins;
  if (pass == 0) {
    unsigned long long n = 0;
    for (int i = tid; i < bins; i += kThreads) n += tb[i];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) n += __shfl_xor_sync(0xffffffffu, n, d);
    if ((tid & 31) == 0) warp_tot[tid >> 5] = n;
    __syncthreads();
    if (tid == 0) {
      unsigned long long total = 0;
      for (int w = 0; w < kThreads / 32; ++w) total += warp_tot[w];
      S.prefix[0] = S.prefix[1] = K(0);
      S.same = 1;
      S.count = static_cast<long long>(total);
      S.live = total > 0;
      S.gamma = 0.0;
      if (q < 0) {
        S.rank[0] = total ? (total - 1) / 2 : 0;
        S.rank[1] = total / 2;
      } else if (total) {
        long long i = 0, j = 0;
        linear_index(static_cast<long long>(total), q, &i, &j, &S.gamma);
        S.rank[0] = static_cast<unsigned long long>(i);
        S.rank[1] = static_cast<unsigned long long>(j);
      }
    }
  } else if (tid == 0) {
    S = st[b];
  }
  __syncthreads();
  const bool two = pass > 0 && !S.same;
  if (S.live) {
    for (int r = 0; r < 2; ++r) {
      rank_digit(tb + (two ? r : 0) * kDigitBins, bins, S.rank[r], warp_tot, &hit_bin, &hit_rest);
      if (tid == 0) {
        S.prefix[r] |= static_cast<K>(hit_bin) << shift;
        S.rank[r] = hit_rest;
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < 2 * kDigitBins; i += kThreads) tb[i] = 0ULL;  // clean for the next digit
  if (tid == 0) {
    S.same = S.prefix[0] == S.prefix[1];
    st[b] = S;
    if (pass == kDigits - 1) {
      if (!S.live) {
        out[b] = d_nan();
        if (count_out) count_out[b] = 0;
      } else {
        const double v0 = key_value(S.prefix[0]), v1 = key_value(S.prefix[1]);
        out[b] = q < 0 ? ((S.count & 1) ? v0 : __dmul_rn(__dadd_rn(v0, v1), 0.5)) : linear_between(v0, v1, S.gamma);
        if (count_out) count_out[b] = S.count;
      }
    }
  }
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

// Candidate keys per element: a quarter of the largest selection's items (the differences along
// every axis), at least 64.
int64_t cand_cap(const Geom& g) { return std::max<int64_t>(64, static_cast<int64_t>(g.dim) * g.field / 4 / 32 * 32); }

// scratch: the grid form's states and count tables, then the candidates' counts and keys
size_t select_scratch_bytes(const Geom& g) {
  const size_t B = static_cast<size_t>(g.batch);
  return align256(B * sizeof(SelGridState<uint64_t>)) + align256(B * 2 * kDigitBins * sizeof(unsigned long long)) +
         align256(B * sizeof(unsigned long long)) + align256(B * static_cast<size_t>(cand_cap(g)) * sizeof(uint64_t));
}

template <class K>
SelCand<K> cand_of(const Geom& g, void* scratch) {
  const size_t B = static_cast<size_t>(g.batch);
  char* p = static_cast<char*>(scratch) + align256(B * sizeof(SelGridState<uint64_t>)) +
            align256(B * 2 * kDigitBins * sizeof(unsigned long long));
  SelCand<K> c;
  c.n = reinterpret_cast<unsigned long long*>(p);
  c.keys = reinterpret_cast<K*>(p + align256(B * sizeof(unsigned long long)));
  c.cap = cand_cap(g);
  return c;
}

// The grid-wide form: every digit a counting and a pick launch (scratch: the states, then the
// [B][2][bins] count tables, zeroed here and left zeroed by every pick).
template <class T, class K>
void select_grid(cudaStream_t s, const Geom& g, const SelView<T>& a, double q, const int32_t* run, double* out,
                 int64_t* count, void* scratch, int sms) {
  constexpr int kDigits = (8 * static_cast<int>(sizeof(K)) + kDigitBits - 1) / kDigitBits;
  auto* st = static_cast<SelGridState<K>*>(scratch);
  auto* table = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch) +
                                                       align256(static_cast<size_t>(g.batch) * sizeof(SelGridState<uint64_t>)));
  EDAB_CUDA(cudaMemsetAsync(table, 0, static_cast<size_t>(g.batch) * 2 * kDigitBins * sizeof(unsigned long long), s));
  // CTAs per element: 64 items per thread, and for small batches enough CTAs for 8 per SM (at
  // least 4 items per thread)
  const int64_t by_items = (a.items + int64_t{kThreads} * 64 - 1) / (int64_t{kThreads} * 64);
  const int64_t fill = std::min<int64_t>((int64_t{8} * sms + g.batch - 1) / g.batch,
                                         std::max<int64_t>(1, a.items / (int64_t{kThreads} * 4)));
  const unsigned ctas = static_cast<unsigned>(std::clamp<int64_t>(std::max(by_items, fill), 1, 1024));
  const SelCand<K> cand = (sizeof(K) == 8 || EDAB_SEL_CAND32) ? cand_of<K>(g, scratch) : SelCand<K>{};
  if (cand.keys) EDAB_CUDA(cudaMemsetAsync(cand.n, 0, static_cast<size_t>(g.batch) * sizeof(unsigned long long), s));
  for (int pass = 0; pass < kDigits; ++pass) {
    select_grid_count<T, K><<<dim3(ctas, static_cast<unsigned>(g.batch)), kThreads, 0, s>>>(g, a, run, st, table, pass,
                                                                                          cand);
    EDAB_LAUNCH("select_grid_count");
    select_grid_pick<K><<<static_cast<unsigned>(g.batch), kThreads, 0, s>>>(run, st, table, pass, q, out, count);
    EDAB_LAUNCH("select_grid_pick");
  }
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
  if (g.batch > 65535) throw std::invalid_argument("edab: select batch too large");
  // clusters (one launch) when the batch fills the GPU with them, else the grid-wide form
  int sms = 148;
  {
    int dev = 0;
    EDAB_CUDA(cudaGetDevice(&dev));
    EDAB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  if (!kSelClusters || g.batch * kSelClusterMax < 2 * static_cast<int64_t>(sms)) {
    if (!scratch) throw std::logic_error("edab: the grid-wide selection needs its scratch");
    if constexpr (std::is_same_v<T, float>) {
      if (sel.center == nullptr) {
        select_grid<T, uint32_t>(s, g, a, q, run, out, count, scratch, sms);
        return;
      }
    }
    select_grid<T, uint64_t>(s, g, a, q, run, out, count, scratch, sms);
    return;
  }
  // CTAs per element: about 16 items per thread, up to a cluster of 8
  const int64_t per_cta = int64_t{kThreads} * 16;
  const unsigned ctas = static_cast<unsigned>(std::clamp<int64_t>((a.items + per_cta - 1) / per_cta, 1, kSelClusterMax));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(ctas, static_cast<unsigned>(g.batch));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSelSmem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const auto launch = [&](auto kernel, auto cand) {
    once_on_device(reinterpret_cast<const void*>(kernel), [&] {
      EDAB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSelSmem)));
    });
    EDAB_CUDA(cudaLaunchKernelEx(&cfg, kernel, g, a, run, q, out, count, cand));
    EDAB_LAUNCH("select_cluster");
  };
  if constexpr (std::is_same_v<T, float>) {
    if (sel.center == nullptr) {
      launch(select_cluster<T, uint32_t>, (EDAB_SEL_CAND32 && scratch) ? cand_of<uint32_t>(g, scratch) : SelCand<uint32_t>{});
      return;
    }
  }
  launch(select_cluster<T, uint64_t>, scratch ? cand_of<uint64_t>(g, scratch) : SelCand<uint64_t>{});
}

// ---------------------------------------------------------------------------------------------
// Significant extrema (cpp/src/method/stats_fields.cu:1-14, 182-331 of eda-cuda): the peaks of r
// and -r along every line as scipy.signal.find_peaks defines them, with topographic prominence
// >= tau at the peak. A CTA stages P lines in shared memory with their 32-sample block minima and
// maxima; the thread of a run start owns a peak and walks each side over samples, then whole
// blocks (entering a block only where it holds the side's end).
namespace {

constexpr int kBlk = 32;

// A drop from hi to lo is significant when fl64(hi - lo) >= tau: the difference of the two samples
// in double, rounded once. (For float32 samples the float difference decides the same way except on
// an exact tie with tau; the double difference settles every case with one rule.)
template <class T>
__device__ __forceinline__ bool drops(T hi, T lo, T tau) {
  return __dsub_rn(static_cast<double>(hi), static_cast<double>(lo)) >= static_cast<double>(tau);
}

// Sample k of a staged line: one pad word after every 32 samples (the lanes of a warp scanning
// consecutive blocks hit distinct banks).
template <class T>
__device__ __forceinline__ T xs(const T* x, int32_t k) {
  return x[k + (k >> 5)];
}

// Samples k = from, from + Dir, .. to of a staged line against the peak value v: 1 when a sample
// lies a significant drop away from v before any sample lies beyond v (above a maximum, below a
// minimum, or NaN), 0 when a sample beyond v comes first, -1 when the range holds neither.
template <bool Max, int Dir, class T, class X>
__device__ __forceinline__ int walk_samples(const X& x, int32_t from, int32_t to, T v, T tau) {
  for (int32_t k = from; (to - k) * Dir >= 0; k += Dir) {
    const T u = x(k);
    if (Max ? !(u <= v) : !(u >= v)) return 0;
    if (Max ? drops(v, u, tau) : drops(u, v, tau)) return 1;
  }
  return -1;
}

// Whether the side of the peak at p (value v) in direction Dir falls by tau before it rises beyond
// v (the line end counts as no fall): SciPy's prominence base on that side is at least tau below
// the peak. The rest of the peak's 32-sample block is walked sample by sample; then every block is
// judged by its extremes (bext: the extreme towards "beyond", bnear: the other one): a block with
// nothing beyond v either holds a significant drop or is passed over; the first block with a sample
// beyond v is walked and decides.
template <bool Max, int Dir, class T, class X>
__device__ bool side_falls(const X& x, int32_t n, int32_t p, T v, T tau, const T* bext, const T* bnear) {
  const int32_t blocks = (n + kBlk - 1) / kBlk;
  int32_t c = p / kBlk;
  const int32_t edge = Dir > 0 ? min(c * kBlk + kBlk - 1, n - 1) : c * kBlk;
  if ((edge - p) * Dir > 0) {
    const int verdict = walk_samples<Max, Dir, T>(x, p + Dir, edge, v, tau);
    if (verdict >= 0) return verdict == 1;
  }
  for (c += Dir; c >= 0 && c < blocks; c += Dir) {
    const T e = bext[c];
    if (Max ? !(e <= v) : !(e >= v)) {
      const int32_t first = c * kBlk, last = min(first + kBlk - 1, n - 1);
      return walk_samples<Max, Dir, T>(x, Dir > 0 ? first : last, Dir > 0 ? last : first, v, tau) == 1;
    }
    if (Max ? drops(v, bnear[c], tau) : drops(bnear[c], v, tau)) return true;
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
  const int32_t n = elem_n(g, b, axis);
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
    const auto at_k = [x](int32_t k) { return xs(x, k); };
    const bool sig = is_max ? side_falls<true, -1>(at_k, n, pk, cur, tp, pmax, pmin) && side_falls<true, 1>(at_k, n, pk, cur, tp, pmax, pmin)
                            : side_falls<false, -1>(at_k, n, pk, cur, tp, pmin, pmax) && side_falls<false, 1>(at_k, n, pk, cur, tp, pmin, pmax);
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

// Lines too long to stage (1-D signals beyond the staged capacity): one CTA per line reads the
// samples from global memory (L1 / L2) and keeps only the 32-sample block extremes in shared
// memory; the peaks and their walks are those of the staged kernel.
template <class T>
__global__ void __launch_bounds__(kThreads) flags_long(Geom g, const T* __restrict__ r, const T* __restrict__ tau,
                                                       uint8_t* __restrict__ flags, Elem* el, const int32_t* run) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int32_t count_s;
  const int64_t b = blockIdx.y;
  if (run && !run[b]) return;
  const int64_t row = blockIdx.x;
  const int32_t n = elem_len(g, b);
  const int32_t nb = (n + kBlk - 1) / kBlk;
  T* bmin = reinterpret_cast<T*>(smem_raw);
  T* bmax = bmin + nb;
  const int64_t base = b * g.field + row * g.pitch;
  const T* line = r + base;
  if (threadIdx.x == 0) count_s = 0;
  for (int32_t c = threadIdx.x; c < nb; c += blockDim.x) {
    const int32_t len = min(kBlk, n - c * kBlk);
    const T* xb = line + c * kBlk;
    T mn = xb[0], mx = mn;
    for (int32_t i = 1; i < len; ++i) {
      const T v = xb[i];
      mn = (v < mn || v != v) ? v : mn;
      mx = (v > mx || v != v) ? v : mx;
    }
    bmin[c] = mn;
    bmax[c] = mx;
  }
  __syncthreads();
  const auto at_k = [line](int32_t k) { return line[k]; };
  int mine = 0;
  for (int32_t s = 1 + threadIdx.x; s <= n - 2; s += blockDim.x) {
    const T cur = line[s], prev = line[s - 1];
    if (!(prev < cur || prev > cur)) continue;
    // the run of samples equal to cur from s: samples of s's block, then whole blocks of cur
    int32_t e;
    {
      const int32_t lim = min((s / kBlk) * kBlk + kBlk - 1, n - 1);
      int32_t k = s + 1;
      while (k <= lim && line[k] == cur) ++k;
      if (k <= lim || k >= n) {
        e = k - 1;
      } else {
        e = n - 1;
        for (int32_t c = k / kBlk; c < nb; ++c) {
          if (bmin[c] == cur && bmax[c] == cur) continue;
          k = c * kBlk;
          while (line[k] == cur) ++k;
          e = k - 1;
          break;
        }
      }
    }
    if (e > n - 2) continue;
    const T nxt = line[e + 1];
    const bool is_max = prev < cur && nxt < cur;
    const bool is_min = prev > cur && nxt > cur;
    if (!is_max && !is_min) continue;
    const int32_t pk = (s + e) / 2;
    const T tp = tau[base + pk];
    const bool sig = is_max ? side_falls<true, -1>(at_k, n, pk, cur, tp, bmax, bmin) && side_falls<true, 1>(at_k, n, pk, cur, tp, bmax, bmin)
                            : side_falls<false, -1>(at_k, n, pk, cur, tp, bmin, bmax) && side_falls<false, 1>(at_k, n, pk, cur, tp, bmin, bmax);
    if (sig) {
      flags[base + pk] |= static_cast<uint8_t>(1u);
      ++mine;
    }
  }
  for (int d = 16; d > 0; d >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, d);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&count_s, mine);
  __syncthreads();
  if (threadIdx.x == 0 && count_s) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&el[b].ext[0]), static_cast<unsigned long long>(count_s));
  }
}

// ---------------------------------------------------------------------------------------------
// Face-connected components, labelled by the smallest padded index of the component. Parent links
// always point to a smaller index and a root is linked only by a compare-and-swap that finds it
// still a root, so every tree's root is its smallest member whatever the order of the threads.
// Phase 1 labels the components of every tile (consecutive rows of an element) in shared memory;
// phase 2 joins the trees across the tile borders in global memory; phase 3 points every voxel at
// its root.

// Root of x; parent reads bypass L1 (another SM may have relinked a root), shared memory is
// coherent inside the CTA and read volatile.
template <bool Global>
__device__ __forceinline__ int32_t uf_root(int32_t* P, int32_t x) {
  for (;;) {
    const int32_t up = Global ? __ldcg(P + x) : *reinterpret_cast<volatile int32_t*>(P + x);
    if (up == x) return x;
    x = up;
  }
}
template <bool Global>
__device__ __forceinline__ void uf_join(int32_t* P, int32_t x, int32_t y) {
  for (;;) {
    x = uf_root<Global>(P, x);
    y = uf_root<Global>(P, y);
    if (x == y) return;
    const int32_t big = x > y ? x : y, small = x > y ? y : x;
    if (atomicCAS(P + big, big, small) == big) return;  // big was still a root: now under small
    x = big;
    y = small;
  }
}

constexpr int32_t kTileWords = 8192;  // int32 parents per tile (32 KiB of shared memory)

__device__ __forceinline__ int64_t rows_between(const Geom& g, int a) { return geom_stride(g, a) / g.pitch; }

// A tile is tile_rows consecutive rows of an element, whole (tile_cols = pitch), or for rows longer
// than a tile (1-D lines beyond kTileWords samples) a run of tile_cols columns of one row.
__global__ void __launch_bounds__(kThreads) ccl_tiles(Geom g, const uint8_t* __restrict__ mask, uint8_t bits,
                                                     int32_t* __restrict__ labels, const int32_t* run, int32_t tile_rows,
                                                     int32_t tile_cols) {
  __shared__ int32_t P[kTileWords];
  const int64_t b = blockIdx.y;
  if (run && !run[b]) return;
  const int32_t pitch = static_cast<int32_t>(g.pitch), nl = elem_len(g, b);
  const int32_t col_tiles = (pitch + tile_cols - 1) / tile_cols;
  const int64_t row0 = static_cast<int64_t>(blockIdx.x / col_tiles) * tile_rows;
  const int32_t c0 = static_cast<int32_t>(blockIdx.x % col_tiles) * tile_cols;
  if (row0 >= g.rows) return;
  const int32_t rows = static_cast<int32_t>(min(static_cast<int64_t>(tile_rows), g.rows - row0));
  const int32_t cols = min(tile_cols, pitch - c0);
  const int32_t words = rows * cols;
  const int64_t v0 = row0 * g.pitch + c0;  // the tile's first padded offset in the element
  const int64_t eb = b * g.field;
  // local index k = r cols + c <-> padded offset v0 + r pitch + c
  for (int32_t k = threadIdx.x; k < words; k += blockDim.x) {
    const int32_t r = k / cols, c = k - r * cols;
    P[k] = (c0 + c < nl && (mask[eb + v0 + static_cast<int64_t>(r) * pitch + c] & bits) != 0) ? k : -1;
  }
  __syncthreads();
  for (int32_t k = threadIdx.x; k < words; k += blockDim.x) {
    if (P[k] < 0) continue;
    const int32_t r = k / cols, c = k - r * cols;
    if (c + 1 < cols && c0 + c + 1 < nl && P[k + 1] >= 0) uf_join<false>(P, k, k + 1);
    for (int a = 0; a + 1 < g.dim; ++a) {
      const int64_t rs = rows_between(g, a);
      if (r + rs >= rows || coord_of(g, v0 + static_cast<int64_t>(r) * pitch + c, a) + 1 >= geom_n(g, a)) continue;
      const int32_t u = k + static_cast<int32_t>(rs) * cols;
      if (P[u] >= 0) uf_join<false>(P, k, u);
    }
  }
  __syncthreads();
  for (int32_t k = threadIdx.x; k < words; k += blockDim.x) {
    const int32_t r = k / cols, c = k - r * cols;
    int32_t lab = -1;
    if (P[k] >= 0) {
      const int32_t root = uf_root<false>(P, k);  // the local root: the smallest local index, so the
      const int32_t rr = root / cols;             // smallest padded offset of the tile's component
      lab = static_cast<int32_t>(v0 + static_cast<int64_t>(rr) * pitch + (root - rr * cols));
    }
    labels[eb + v0 + static_cast<int64_t>(r) * pitch + c] = lab;
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
  once_on_device(reinterpret_cast<const void*>(flags_pass<T>), [&] {  // the limit is per device
    EDAB_CUDA(cudaFuncSetAttribute(flags_pass<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cap)));
  });
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
    if (bytes(P) > cap) {
      // a 1-D line beyond the staged capacity: samples from global memory, block extremes staged
      const size_t ext_bytes = static_cast<size_t>(2) * nb * sizeof(T);
      if (g.dim != 1 || ext_bytes > cap) throw std::invalid_argument("edab: a line exceeds the shared memory of the extrema pass");
      once_on_device(reinterpret_cast<const void*>(flags_long<T>), [&] {
        EDAB_CUDA(cudaFuncSetAttribute(flags_long<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(cap)));
      });
      flags_long<T><<<dim3(static_cast<unsigned>(g.rows), static_cast<unsigned>(g.batch)), kThreads, ext_bytes, s>>>(
          g, r, tau, flags, el, run);
      EDAB_LAUNCH("flags_long");
      continue;
    }
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
  const bool wide = g.pitch > kTileWords;
  const int32_t tile_rows = wide ? 1 : static_cast<int32_t>(kTileWords / g.pitch);
  const int32_t tile_cols = wide ? kTileWords : static_cast<int32_t>(g.pitch);
  const int64_t col_tiles = (g.pitch + tile_cols - 1) / tile_cols;
  const int64_t tiles = (g.rows + tile_rows - 1) / tile_rows * col_tiles;
  if (tiles > 0x7fffffffLL || g.batch > 65535) throw std::invalid_argument("edab: components: grid too large");
  ccl_tiles<<<dim3(static_cast<unsigned>(tiles), static_cast<unsigned>(g.batch)), kThreads, 0, s>>>(
      g, mask, bits, labels, run, tile_rows, tile_cols);
  EDAB_LAUNCH("ccl_tiles");
  // the edges between tiles
  for_voxels(s, g, [=] __device__(int64_t b) { return run == nullptr || run[b] != 0; },
             [=] __device__(int64_t b, int64_t v, int64_t i) {
               int32_t* L = labels + b * g.field;
               if (L[v] < 0) return;
               const int64_t row = pitch_row(g, v);
               const int64_t col = v - row * g.pitch;
               if (wide && (col + 1) % tile_cols == 0 && col + 1 < elem_len(g, b) && L[v + 1] >= 0) {
                 uf_join<true>(L, static_cast<int32_t>(v), static_cast<int32_t>(v + 1));
               }
               const int64_t tile = row / tile_rows;
               for (int a = 0; a + 1 < g.dim; ++a) {
                 const int64_t rs = geom_stride(g, a) / g.pitch;
                 if ((row + rs) / tile_rows == tile || coord_of(g, v, a) + 1 >= geom_n(g, a)) continue;
                 const int64_t u = v + geom_stride(g, a);
                 if (L[u] >= 0) uf_join<true>(L, static_cast<int32_t>(v), static_cast<int32_t>(u));
               }
             });
  // every voxel to its root
  for_voxels(s, g, [=] __device__(int64_t b) { return run == nullptr || run[b] != 0; },
             [=] __device__(int64_t b, int64_t v, int64_t i) {
               int32_t* L = labels + b * g.field;
               if (L[v] < 0) return;
               L[v] = uf_root<true>(L, static_cast<int32_t>(v));
             });
}

template void field_totals<float>(cudaStream_t, const Geom&, const float*, double*, double*, uint64_t*, void*);
template void field_totals<double>(cudaStream_t, const Geom&, const double*, double*, double*, uint64_t*, void*);
template void select<float>(cudaStream_t, const Geom&, const Sel<float>&, double, const int32_t*, double*, int64_t*, void*);
template void select<double>(cudaStream_t, const Geom&, const Sel<double>&, double, const int32_t*, double*, int64_t*, void*);
template void sig_flags<float>(cudaStream_t, const Geom&, const float*, const float*, uint8_t*, Elem*, const int32_t*);
template void sig_flags<double>(cudaStream_t, const Geom&, const double*, const double*, uint8_t*, Elem*, const int32_t*);

}  // namespace edab
