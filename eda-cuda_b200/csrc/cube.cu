// SPDX-License-Identifier: Apache-2.0
// The separable cube filter: along every axis a running max, min or box sum of odd width 2r + 1,
// r = min((w - 1) / 2, n_a - 1), with half-sample reflection, by the van Herk / Gil-Werman scheme
// with the reference's canonical fold structure (cpp/src/field/vhgw.cu:1-36 of eda-cuda), so
// that every output depends only on the line, its length and the window:
//   - the extended line e in [-r, n + r) reads the line through half-sample reflection; it is cut
//     into segments of wa = 2r + 1 samples starting at o + k wa, o = (n (wa + 1) / 2) mod wa;
//   - G (prefix fold of a segment): 32-sample chunks from the segment start, a sequential fold in
//     each chunk, a sequential carry over the chunk totals, G = carry op local; H (suffix fold) is
//     G of the reversed line;
//   - y(x) = op(H(x - r), G(x + r)); a box window aligned with a segment takes (H + G) * 0.5.
// Box sums run axis 0 first and the last pass multiplies by fl_T(1 / prod of the clamped sides);
// max and min fold the integer order keys of the values (the order of max_c / min_c).
//
// B200 design. A CTA runs a run of consecutive line groups of one element (and one rung, or every
// rung of a ladder that shares its input); a group is P lines: P rows of the contiguous axis, or a
// panel of P adjacent columns of an outer axis. Shared-memory layouts keep every global transfer a
// 16-byte copy: rows are stored line after line with a padded line stride (4 words modulo 32, so
// the P lanes of a worker reading one sample of P lines hit distinct banks); a column panel keeps
// its global row layout, sample i of line p at i P + p. The next group's input is copied with
// cp.async into the second of two buffers while the current group is folded; order keys (max /
// min) are formed in place by the threads that copied the samples. The window setup of every rung
// is made once per CTA. Lanes map to lines: P lanes of a warp ("a worker") run the same fold task
// on their P lines, so control flow is uniform. The fold tasks (one per direction, segment and
// 32-sample chunk) are spread over the CTA's workers: chunk totals, per-segment exclusive carries,
// then the H folds and the G folds combined with them. A whole 32-sample chunk inside the line runs
// as an unrolled fold with immediate shared-memory offsets; only the chunks that cross a line end,
// the window's first r samples or a segment end take the general path. A chunk without a carry
// folds from the operation's identity (-0 for sums, the extreme keys for max / min), which changes
// no bit of any result.
#include "engine.cuh"

#include <algorithm>
#include <climits>
#include <mutex>

namespace edab {
namespace {

constexpr int kOpMaxK = 0, kOpMinK = 1, kOpSum = 2;
// Threads of a cube CTA, and CTAs per SM the registers are bounded for (build-time choices; the
// lines, groups and segment share of a launch are chosen at run time).
#ifndef EDAB_CUBE_THREADS
#define EDAB_CUBE_THREADS 256
#endif
#ifndef EDAB_CUBE_CTAS
#define EDAB_CUBE_CTAS 4
#endif
constexpr int kCubeThreads = EDAB_CUBE_THREADS;
constexpr int kWarps = kCubeThreads / 32;
constexpr int kMaxGroupsPerCta = 4;  // line groups one CTA may run (the default launch shape runs one)
// A window folds whole segments per worker when its segments number at least workers / seq_share
// (the default, or the tuned value of the geometry).
constexpr int kSeqShare = 4;

__host__ __device__ constexpr int32_t tot_slots(int32_t n) { return n / 8 + 24; }
// Line stride of the row layout in elements: the padded row rounded up, plus 16 bytes (4 words
// modulo 32 for 4-byte samples, 2 elements modulo 16 for 8-byte samples).
template <class T>
__host__ __device__ constexpr int32_t row_stride(int32_t n) {
  return sizeof(T) == 4 ? ((n + 31) & ~31) + 4 : ((n + 15) & ~15) + 2;
}
// Elements of one line-group buffer (a multiple of 16 bytes).
template <class T>
__host__ __device__ constexpr int32_t group_elems(int32_t n, int P, bool rows) {
  return rows ? P * row_stride<T>(n) : ((n * P + 3) & ~3);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Order key of v as a T-sized integer (its own inverse): integer order = order of max_c/min_c.
__device__ __forceinline__ float okey(float v) {
  const int32_t b = __float_as_int(v);
  return __int_as_float(b ^ ((b >> 31) & 0x7fffffff));
}
__device__ __forceinline__ double okey(double v) {
  const long long b = __double_as_longlong(v);
  return __longlong_as_double(b ^ ((b >> 63) & 0x7fffffffffffffffLL));
}
template <int OP>
__device__ __forceinline__ float fop(float a, float b) {
  if constexpr (OP == kOpSum) {
    return __fadd_rn(a, b);
  } else {
    const int32_t x = __float_as_int(a), y = __float_as_int(b);
    return __int_as_float(OP == kOpMaxK ? max(x, y) : min(x, y));
  }
}
template <int OP>
__device__ __forceinline__ double fop(double a, double b) {
  if constexpr (OP == kOpSum) {
    return __dadd_rn(a, b);
  } else {
    const long long x = __double_as_longlong(a), y = __double_as_longlong(b);
    return __longlong_as_double(OP == kOpMaxK ? (x > y ? x : y) : (x < y ? x : y));
  }
}
// The identity of fop: fop(identity, x) == x bit for bit (-0 + x == x; the extreme integer keys).
template <class T, int OP>
__device__ __forceinline__ T fold_identity() {
  if constexpr (OP == kOpSum) {
    return T(-0.0);
  } else if constexpr (sizeof(T) == 4) {
    return __int_as_float(OP == kOpMaxK ? INT_MIN : INT_MAX);
  } else {
    return __longlong_as_double(OP == kOpMaxK ? LLONG_MIN : LLONG_MAX);
  }
}

struct Win {
  int32_t r, wa, o, k_lo, nseg, cps;
  // the segments a CTA folds, relative to k_lo: segments [hk0, hk0 + hn) of the reversed line for
  // H and [gk0, gk0 + gn) of the line for G (a whole line: 0 and nseg both; a tile of a long line:
  // the segments its outputs need)
  int32_t hk0, hn, gk0, gn;
};
// 32-bit arithmetic but for the offset's product (n (wa + 1) / 2 reaches 2^32 for the longest
// lines; one 64-bit modulo per window set-up): the 64-bit integer divisions of a general formula
// are long emulated sequences on the GPU.
__device__ __forceinline__ int32_t floor_div32(int32_t a, int32_t b) {  // b > 0
  const int32_t q = a / b;
  return (a % b != 0 && a < 0) ? q - 1 : q;
}
__device__ __forceinline__ Win make_win(int32_t n, int32_t w) {
  Win q;
  const int32_t half = (w - 1) >> 1;
  q.r = min(half, n - 1);
  q.wa = 2 * q.r + 1;
  q.o = static_cast<int32_t>((static_cast<uint64_t>(n) * static_cast<uint64_t>((q.wa + 1) >> 1)) %
                             static_cast<uint64_t>(q.wa));
  q.k_lo = floor_div32(q.r - q.o, q.wa);
  const int32_t k_hi = floor_div32(n - 1 + q.r - q.o, q.wa);
  q.nseg = k_hi - q.k_lo + 1;
  q.cps = (q.wa + 31) >> 5;
  q.hk0 = q.gk0 = 0;
  q.hn = q.gn = q.nseg;
  return q;
}

// Line-sample index of extended position e in direction dir (1: the reversed line).
__device__ __forceinline__ int32_t ext_index(int32_t e, int32_t n, int dir) {
  const int32_t i = reflect_index(e, n);
  return dir ? n - 1 - i : i;
}

// The general fold of a chunk [c0, c1] of direction dir into acc (first sample stored as is),
// calling f(e, local) after every sample: interior chunks index linearly, boundary chunks reflect.
template <class T, int OP, class F>
__device__ __forceinline__ T fold_chunk(const T* __restrict__ V, int32_t PP, int32_t n, int32_t c0, int32_t c1, int dir,
                                     F&& f) {
  T loc;
  if (c0 >= 0 && c1 <= n - 1) {
    int32_t i = dir ? n - 1 - c0 : c0;
    const int32_t di = dir ? -PP : PP;
    const T* ptr = V + i * PP;
    loc = *ptr;
    f(c0, loc);
    for (int32_t e = c0 + 1; e <= c1; ++e) {
      ptr += di;
      loc = fop<OP>(loc, *ptr);
      f(e, loc);
    }
  } else {
    loc = V[ext_index(c0, n, dir) * PP];
    f(c0, loc);
    for (int32_t e = c0 + 1; e <= c1; ++e) {
      loc = fop<OP>(loc, V[ext_index(e, n, dir) * PP]);
      f(e, loc);
    }
  }
  return loc;
}

// The unrolled folds of a whole 32-sample chunk inside the line (STEP: +PP forward, -PP reversed).
template <class T, int OP, int STEP>
__device__ __forceinline__ T chunk_total(const T* __restrict__ vp) {
  T loc = vp[0];
#pragma unroll
  for (int s = 1; s < 32; ++s) loc = fop<OP>(loc, vp[s * STEP]);
  return loc;
}
// H of the chunk into its output slots (one slot back per sample): carry op local.
// Every chunk fold returns its last fold value: the chunk's local total for sums, the fold from the
// carry for max / min (a segment folded chunk after chunk chains its carries from these).
template <class T, int OP, int PP>
__device__ __forceinline__ T chunk_h(const T* __restrict__ vp, T* __restrict__ rp, T cv) {
  if constexpr (OP == kOpSum) {
    T loc = vp[0];
    rp[0] = add_rn(cv, loc);
#pragma unroll
    for (int s = 1; s < 32; ++s) {
      loc = add_rn(loc, vp[-s * PP]);
      rp[-s * PP] = add_rn(cv, loc);
    }
    return loc;
  } else {
    T loc = cv;
#pragma unroll
    for (int s = 0; s < 32; ++s) {
      loc = fop<OP>(loc, vp[-s * PP]);
      rp[-s * PP] = loc;
    }
    return loc;
  }
}
// G of the chunk combined with the H already in its output slots; the segment's last sample of an
// aligned box window (aligned_end) takes (H + G) * 0.5.
template <class T, int OP, int PP>
__device__ __forceinline__ T chunk_g(const T* __restrict__ vp, T* __restrict__ rp, T cv, bool aligned_end) {
  if constexpr (OP == kOpSum) {
    T loc = vp[0];
#pragma unroll
    for (int s = 0; s < 32; ++s) {
      if (s) loc = add_rn(loc, vp[s * PP]);
      const T y = add_rn(rp[s * PP], add_rn(cv, loc));
      rp[s * PP] = (s == 31 && aligned_end) ? mul_rn(y, T(0.5)) : y;
    }
    return loc;
  } else {
    T loc = cv;
#pragma unroll
    for (int s = 0; s < 32; ++s) {
      loc = fop<OP>(loc, vp[s * PP]);
      rp[s * PP] = fop<OP>(rp[s * PP], loc);
    }
    return loc;
  }
}

// The partial folds of a chunk inside the line (fewer than 32 samples, or a chunk that starts
// before the first output). v: the chunk's first sample (STEP words per sample), r: the output slot
// of the chunk's first sample (STEP words per sample); only samples i >= skip have an output.
// Max / min fold from the carry (the operation's identity without one); sums fold locally and add
// the carry to every output (the canonical G = carry op local).
template <class T, int OP>
__device__ __forceinline__ T fold_init(T cv, T v0) {
  if constexpr (OP == kOpSum) return v0;
  else return fop<OP>(cv, v0);
}
template <class T, int OP>
__device__ __forceinline__ T fold_out(T cv, T loc) {
  if constexpr (OP == kOpSum) return add_rn(cv, loc);
  else return loc;
}
template <class T, int OP, int STEP>
__device__ __forceinline__ T partial_total(const T* __restrict__ v, int32_t len) {
  T loc = v[0];
  int32_t i = 1;
  for (; i + 3 < len; i += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) loc = fop<OP>(loc, v[(i + u) * STEP]);
  }
  for (; i < len; ++i) loc = fop<OP>(loc, v[i * STEP]);
  return loc;
}
// H: the output of sample i is stored (slots step back with the samples: STEP = -PP for both)
template <class T, int OP, int PP>
__device__ __forceinline__ T partial_h(const T* __restrict__ v, T* __restrict__ r, int32_t len, int32_t skip,
                                       T cv) {
  T loc = fold_init<T, OP>(cv, v[0]);
  if (skip == 0) r[0] = fold_out<T, OP>(cv, loc);
  int32_t i = 1;
  const int32_t pre = min(skip, len);
  for (; i < pre; ++i) loc = fop<OP>(loc, v[-i * PP]);
  for (; i + 3 < len; i += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      loc = fop<OP>(loc, v[-(i + u) * PP]);
      r[-(i + u) * PP] = fold_out<T, OP>(cv, loc);
    }
  }
  for (; i < len; ++i) {
    loc = fop<OP>(loc, v[-i * PP]);
    r[-i * PP] = fold_out<T, OP>(cv, loc);
  }
  return loc;
}
// G combined with the H in the slots (STEP = +PP); the chunk's last sample, when it ends an aligned
// box window (aligned_end), takes (H + G) * 0.5.
template <class T, int OP>
__device__ __forceinline__ void combine_g(T* __restrict__ slot, T cv, T loc, bool half) {
  if constexpr (OP == kOpSum) {
    const T y = add_rn(*slot, add_rn(cv, loc));
    *slot = half ? mul_rn(y, T(0.5)) : y;
  } else {
    *slot = fop<OP>(*slot, loc);
  }
}
template <class T, int OP, int PP>
__device__ __forceinline__ T partial_g(const T* __restrict__ v, T* __restrict__ r, int32_t len, int32_t skip,
                                       T cv, bool aligned_end) {
  const int32_t last = len - 1;
  T loc = fold_init<T, OP>(cv, v[0]);
  if (last == 0) {
    if (skip == 0) combine_g<T, OP>(r, cv, loc, aligned_end);
    return loc;
  }
  if (skip == 0) combine_g<T, OP>(r, cv, loc, false);
  int32_t i = 1;
  const int32_t pre = min(skip, last);
  for (; i < pre; ++i) loc = fop<OP>(loc, v[i * PP]);
  for (; i + 3 < last; i += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      loc = fop<OP>(loc, v[(i + u) * PP]);
      combine_g<T, OP>(r + (i + u) * PP, cv, loc, false);
    }
  }
  for (; i < last; ++i) {
    loc = fop<OP>(loc, v[i * PP]);
    combine_g<T, OP>(r + i * PP, cv, loc, false);
  }
  loc = fop<OP>(loc, v[last * PP]);
  if (last >= skip) combine_g<T, OP>(r + last * PP, cv, loc, aligned_end);
  return loc;
}

// The carry into the next chunk of a segment from this chunk's fold value (the canonical chunk
// carries: the first chunk's total, then carry op total; max / min values already hold the carry).
template <class T, int OP>
__device__ __forceinline__ T next_carry(T carry, T loc, bool first) {
  if constexpr (OP == kOpSum) return first ? loc : add_rn(carry, loc);
  else return fop<OP>(carry, loc);
}

// A whole segment [s, e_last] folded by one worker, chunk after chunk with the carries chained (no
// chunk totals pass, no carry pass): H of the reversed line into the output slots n - 1 + r - e,
// then (after the CTA's barrier) G combined with them.
template <class T, int OP, int PP>
__device__ __forceinline__ void seg_h(const T* __restrict__ Vp, T* __restrict__ Rp, int32_t n, const Win& q,
                                      int32_t s, int32_t e_last) {
  T carry = fold_identity<T, OP>();
  for (int32_t c = 0, c0 = s; c0 <= e_last; ++c, c0 += 32) {
    const int32_t c1 = min(c0 + 31, e_last);
    T loc;
    if (c0 >= 0 && c1 <= n - 1) {
      const T* vp = Vp + (n - 1 - c0) * PP;
      T* rp = Rp + (n - 1 + q.r - c0) * PP;
      if (c1 == c0 + 31 && c0 >= q.r) loc = chunk_h<T, OP, PP>(vp, rp, carry);
      else loc = partial_h<T, OP, PP>(vp, rp, c1 - c0 + 1, max(0, q.r - c0), carry);
    } else {
      const T cv = carry;
      loc = fold_chunk<T, OP>(Vp, PP, n, c0, c1, 1, [&](int32_t e, T l) {
        if (e >= q.r) Rp[(n - 1 + q.r - e) * PP] = fop<OP>(cv, l);
      });
    }
    carry = next_carry<T, OP>(carry, loc, c == 0);
  }
}
template <class T, int OP, int PP>
__device__ __forceinline__ void seg_g(const T* __restrict__ Vp, T* __restrict__ Rp, int32_t n, const Win& q,
                                      int32_t s, int32_t e_last) {
  const int32_t e_al = s + q.wa - 1;
  T carry = fold_identity<T, OP>();
  for (int32_t c = 0, c0 = s; c0 <= e_last; ++c, c0 += 32) {
    const int32_t c1 = min(c0 + 31, e_last);
    T loc;
    if (c0 >= 0 && c1 <= n - 1) {
      const T* vp = Vp + c0 * PP;
      T* rp = Rp + (c0 - q.r) * PP;
      if (c1 == c0 + 31 && c0 >= q.r) loc = chunk_g<T, OP, PP>(vp, rp, carry, c1 == e_al);
      else loc = partial_g<T, OP, PP>(vp, rp, c1 - c0 + 1, max(0, q.r - c0), carry, c1 == e_al);
    } else {
      const T cv = carry;
      loc = fold_chunk<T, OP>(Vp, PP, n, c0, c1, 0, [&](int32_t e, T l) {
        if (e < q.r) return;
        const T g = fop<OP>(cv, l);
        T* slot = Rp + (e - q.r) * PP;
        const T h = *slot;
        if constexpr (OP == kOpSum) {
          const T sum = add_rn(h, g);
          *slot = e == e_al ? mul_rn(sum, T(0.5)) : sum;
        } else {
          *slot = fop<OP>(h, g);
        }
      });
    }
    carry = next_carry<T, OP>(carry, loc, c == 0);
  }
}

// The fold tasks (segment k, chunk c) of one worker, chunk-major (u = c nseg + k, u = first,
// first + stride, ..): the workers of a warp take the same chunk of consecutive segments (wa
// samples apart, spreading their shared-memory banks). Advanced without divisions.
struct Tasks {
  int32_t k, c, dk, dc;
  __device__ __forceinline__ Tasks(int32_t first, int32_t stride, int32_t nseg) {
    if (nseg > stride) {  // first < stride: no division
      k = first;
      c = 0;
      dk = stride;
      dc = 0;
    } else {
      k = first % nseg;
      c = first / nseg;
      dk = stride % nseg;
      dc = stride / nseg;
    }
  }
  __device__ __forceinline__ void next(int32_t nseg) {
    k += dk;
    c += dc;
    if (k >= nseg) {
      k -= nseg;
      ++c;
    }
  }
};

// One stage on the staged lines of this CTA: V -> R (sample i of line p at p LS + i PP), tot: the
// chunk totals / carries [2][TS][P] (slot k cps + c). Workers: P lanes each (lane % P = the line).
// RANGE: fold the window's segment range (a long line's tile); else every segment of the line.
template <class T, int OP, int P, int PP, bool RANGE = false>
__device__ __forceinline__ void run_stage(const T* __restrict__ V, T* __restrict__ R, T* __restrict__ tot, int32_t n,
                                          int32_t TS, const Win& q, int32_t LS, int32_t seq_share) {
  const int32_t hn = RANGE ? q.hn : q.nseg, gn = RANGE ? q.gn : q.nseg;
  const int32_t hk0 = RANGE ? q.hk0 : 0, gk0 = RANGE ? q.gk0 : 0;
  constexpr int slots = 32 / P;
  constexpr int workers = kWarps * slots;
  const int lane = threadIdx.x & 31;
  const int p = lane & (P - 1);
  const int worker = (threadIdx.x >> 5) * slots + lane / P;
  const int32_t e_max = n - 1 + q.r;
  const T* Vp = V + p * LS;
  T* Rp = R + p * LS;
  const T idn = fold_identity<T, OP>();
  if (q.wa == 1) {
    // one-sample segments: H = G = the sample, so y = op(v, v): the sample for max / min, and for
    // sums the aligned mean (v + v) * 0.5 of the canonical path, rounded the same way. With r = 0
    // and o = 0 the G segments are the outputs themselves: the whole line, or a long line's tile.
    const int32_t i1 = q.o + q.k_lo + gk0 + gn;
    for (int32_t i = q.o + q.k_lo + gk0 + worker; i < i1; i += workers) {
      const T v = Vp[i * PP];
      Rp[i * PP] = OP == kOpSum ? mul_rn(add_rn(v, v), T(0.5)) : v;
    }
    __syncthreads();
    return;
  }
  // Windows of many segments per line: every worker folds whole segments (a run of `per` of them,
  // about one run per worker), chunk after chunk with chained carries, in two barrier-separated
  // phases. Windows of few, long segments (seq_share * nseg < workers) split their segments into
  // chunks over the workers instead: chunk totals, carries, then the H and G folds (four phases,
  // twice the folds, but every worker busy).
  if (q.cps == 1 || max(hn, gn) * seq_share >= workers) {
    const int32_t hper = (hn + workers - 1) / workers;
    const int32_t hk_end = min((worker + 1) * hper, hn);
    for (int32_t k = worker * hper; k < hk_end; ++k) {
      const int32_t s = q.o + (q.k_lo + hk0 + k) * q.wa;
      const int32_t c1 = min(s + q.wa - 1, e_max);
      if (q.cps > 1) {
        seg_h<T, OP, PP>(Vp, Rp, n, q, s, c1);
      } else if (s >= 0 && c1 <= n - 1) {  // a one-chunk segment inside the line
        partial_h<T, OP, PP>(Vp + (n - 1 - s) * PP, Rp + (n - 1 + q.r - s) * PP, c1 - s + 1, max(0, q.r - s), idn);
      } else {
        fold_chunk<T, OP>(Vp, PP, n, s, c1, 1, [&](int32_t e, T loc) {
          if (e >= q.r) Rp[(n - 1 + q.r - e) * PP] = fop<OP>(idn, loc);
        });
      }
    }
    __syncthreads();
    const int32_t gper = (gn + workers - 1) / workers;
    const int32_t gk_end = min((worker + 1) * gper, gn);
    for (int32_t k = worker * gper; k < gk_end; ++k) {
      const int32_t s = q.o + (q.k_lo + gk0 + k) * q.wa;
      const int32_t e_al = s + q.wa - 1;
      const int32_t c1 = min(e_al, e_max);
      if (q.cps > 1) {
        seg_g<T, OP, PP>(Vp, Rp, n, q, s, c1);
      } else if (s >= 0 && c1 <= n - 1) {
        partial_g<T, OP, PP>(Vp + s * PP, Rp + (s - q.r) * PP, c1 - s + 1, max(0, q.r - s), idn, c1 == e_al);
      } else {
        fold_chunk<T, OP>(Vp, PP, n, s, c1, 0, [&](int32_t e, T loc) {
          if (e < q.r) return;
          const T gv = fop<OP>(idn, loc);
          T* slot = Rp + (e - q.r) * PP;
          const T h = *slot;
          if constexpr (OP == kOpSum) {
            const T sum = add_rn(h, gv);
            *slot = e == e_al ? mul_rn(sum, T(0.5)) : sum;
          } else {
            *slot = fop<OP>(h, gv);
          }
        });
      }
    }
    __syncthreads();
    return;
  }
  if (q.cps > 1) {
    // phase 1: chunk totals; half of the workers take the line, half the reversed line
    constexpr int half = workers / 2;
    const int dir = worker >= half;
    const int32_t dn = dir ? hn : gn;
    const int32_t dk0 = q.k_lo + (dir ? hk0 : gk0);
    for (Tasks t(worker - dir * half, half, dn); t.c < q.cps; t.next(dn)) {
      const int32_t s = q.o + (dk0 + t.k) * q.wa;
      const int32_t e_last = min(s + q.wa - 1, e_max);
      const int32_t c0 = s + 32 * t.c;
      if (c0 > e_last) continue;
      const int32_t c1 = min(c0 + 31, e_last);
      T total;
      if (c0 >= 0 && c1 <= n - 1) {
        if (dir) {
          const T* vp = Vp + (n - 1 - c0) * PP;
          total = c1 == c0 + 31 ? chunk_total<T, OP, -PP>(vp) : partial_total<T, OP, -PP>(vp, c1 - c0 + 1);
        } else {
          const T* vp = Vp + c0 * PP;
          total = c1 == c0 + 31 ? chunk_total<T, OP, PP>(vp) : partial_total<T, OP, PP>(vp, c1 - c0 + 1);
        }
      } else {
        total = fold_chunk<T, OP>(Vp, PP, n, c0, c1, dir, [](int32_t, T) {});
      }
      tot[(dir * TS + t.k * q.cps + t.c) * P + p] = total;
    }
    __syncthreads();
    // phase 2: exclusive carries per segment, in place (slot c holds the carry of chunk c >= 1)
    for (int32_t t = worker; t < gn + hn; t += workers) {
      const int dir = t >= gn;
      const int32_t k = t - dir * gn;
      const int32_t s = q.o + (q.k_lo + (dir ? hk0 : gk0) + k) * q.wa;
      const int32_t e_last = min(s + q.wa - 1, e_max);
      const int32_t nch = (e_last - s) / 32 + 1;
      T* tl = tot + (dir * TS + k * q.cps) * P + p;
      T run = tl[0];
      for (int32_t c = 1; c < nch; ++c) {
        const T next = tl[c * P];
        tl[c * P] = run;
        run = fop<OP>(run, next);
      }
    }
    __syncthreads();
  }
  // phase 3: H (the reversed line's G) into R at the output slots n - 1 + r - e (e >= r)
  for (Tasks t(worker, workers, hn); t.c < q.cps; t.next(hn)) {
    const int32_t s = q.o + (q.k_lo + hk0 + t.k) * q.wa;
    const int32_t e_last = min(s + q.wa - 1, e_max);
    const int32_t c0 = s + 32 * t.c;
    if (c0 > e_last) continue;
    const int32_t c1 = min(c0 + 31, e_last);
    const T cv = t.c > 0 ? tot[(TS + t.k * q.cps + t.c) * P + p] : idn;
    if (c0 >= 0 && c1 <= n - 1) {
      const T* vp = Vp + (n - 1 - c0) * PP;
      T* rp = Rp + (n - 1 + q.r - c0) * PP;  // the slot of e = c0 (written only when c0 >= r)
      if (c1 == c0 + 31 && c0 >= q.r) chunk_h<T, OP, PP>(vp, rp, cv);
      else partial_h<T, OP, PP>(vp, rp, c1 - c0 + 1, max(0, q.r - c0), cv);
    } else {
      fold_chunk<T, OP>(Vp, PP, n, c0, c1, 1, [&](int32_t e, T loc) {
        if (e >= q.r) Rp[(n - 1 + q.r - e) * PP] = fop<OP>(cv, loc);
      });
    }
  }
  __syncthreads();
  // phase 4: G combined with H in place: y(x) = op(H(x - r), G(x + r)), slot x = e - r
  for (Tasks t(worker, workers, gn); t.c < q.cps; t.next(gn)) {
    const int32_t s = q.o + (q.k_lo + gk0 + t.k) * q.wa;
    const int32_t e_al = s + q.wa - 1;
    const int32_t e_last = min(e_al, e_max);
    const int32_t c0 = s + 32 * t.c;
    if (c0 > e_last) continue;
    const int32_t c1 = min(c0 + 31, e_last);
    const T cv = t.c > 0 ? tot[(t.k * q.cps + t.c) * P + p] : idn;
    if (c0 >= 0 && c1 <= n - 1) {
      const T* vp = Vp + c0 * PP;
      T* rp = Rp + (c0 - q.r) * PP;  // the slot of e = c0 (written only when c0 >= r)
      if (c1 == c0 + 31 && c0 >= q.r) chunk_g<T, OP, PP>(vp, rp, cv, c1 == e_al);
      else partial_g<T, OP, PP>(vp, rp, c1 - c0 + 1, max(0, q.r - c0), cv, c1 == e_al);
    } else {
      fold_chunk<T, OP>(Vp, PP, n, c0, c1, 0, [&](int32_t e, T loc) {
        if (e < q.r) return;
        const T g = fop<OP>(cv, loc);
        T* slot = Rp + (e - q.r) * PP;
        const T h = *slot;
        if constexpr (OP == kOpSum) {
          const T sum = add_rn(h, g);
          *slot = e == e_al ? mul_rn(sum, T(0.5)) : sum;
        } else {
          *slot = fop<OP>(h, g);
        }
      });
    }
  }
  __syncthreads();
}

template <class T>
struct PassArgs {
  const T* in0;           // input of field 0 (rung 0 when in_stride != 0)
  const T* in1;           // input of field 1 (maxmin later passes)
  const uint8_t* bits;    // box first pass: bit `bit` of this u8 field
  int32_t bit;
  T* out0;
  T* out1;
  const int32_t* win;     // [rungs * B]
  int32_t rungs;          // rungs of the launch
  int64_t in_stride;      // per-rung input offset (0: one input shared by every rung)
  int64_t out_stride;     // per-rung output offset
  int32_t op;             // CubeOp
  int32_t axis;
  int32_t last;           // the cube's last pass (box scale / epilogue)
  int32_t epi;            // BoxEpi on the last pass
  const T* aux;
  int32_t rung_loop;      // 1: the CTA loops over the rungs (shared input); else blockIdx.z is the rung
  int32_t vec;            // every pointer and stride allows 16-byte copies
  int64_t groups;         // line groups per element
  int32_t gpc;            // line groups per CTA (blockIdx.x runs groups [x gpc, x gpc + gpc))
  int32_t seq_share;      // windows of at least workers / seq_share segments fold whole segments
  int32_t dbuf;           // two staging buffers (a CTA that stages more than once copies ahead)
  unsigned long long* bytes;  // instrumentation: the pass's algorithmic bytes (nullptr: off)
};

// Where a line group lies inside its element: rows, line p at base + p pitch; column panels, line
// p at base + p (rows of the panel `step` apart). mask: bit p set for a line of the field (rows
// inside the element, columns left of the row padding).
struct GroupPos {
  int64_t base;
  uint32_t mask;
  int32_t o, c, cpos;  // rows: c is the first row; column panels: outer index, first column, first
                       // column modulo the pitch
};
template <int P, bool ROWS>
__device__ __forceinline__ GroupPos group_at(const Geom& g, int64_t grp, int32_t n, int64_t inner) {
  GroupPos s{};
  if constexpr (ROWS) {
    s.c = static_cast<int32_t>(grp * P);
  } else {
    // 32-bit divisions (an element holds fewer than 2^31 samples)
    const uint32_t gpo = static_cast<uint32_t>(inner) / P;
    s.o = static_cast<int32_t>(static_cast<uint32_t>(grp) / gpo);
    s.c = static_cast<int32_t>((static_cast<uint32_t>(grp) - static_cast<uint32_t>(s.o) * gpo) * P);
    s.cpos = static_cast<int32_t>(static_cast<uint32_t>(s.c) % static_cast<uint32_t>(g.pitch));
  }
  return s;
}
template <int P, bool ROWS>
__device__ __forceinline__ void group_next(GroupPos& s, const Geom& g, int32_t n, int64_t inner) {
  if constexpr (ROWS) {
    s.c += P;
  } else {
    s.c += P;
    s.cpos += P;
    if (s.cpos == g.pitch) s.cpos = 0;
    if (s.c == inner) {
      s.c = 0;
      ++s.o;
    }
  }
}
template <int P, bool ROWS>
__device__ __forceinline__ void group_finish(GroupPos& s, const Geom& g, int32_t n, int64_t inner) {
  if constexpr (ROWS) {
    s.base = static_cast<int64_t>(s.c) * g.pitch;
    const int64_t left = g.rows - s.c;
    s.mask = left >= P ? (1u << P) - 1u : (left > 0 ? (1u << left) - 1u : 0u);
  } else {
    s.base = static_cast<int64_t>(s.o) * n * inner + s.c;
    const int32_t room = g.n_last - s.cpos;  // columns of the panel left of the padding
    s.mask = room >= P ? (1u << P) - 1u : (room > 0 ? (1u << room) - 1u : 0u);
  }
}

template <class T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
};
template <>
struct Vec16<double> {
  using type = double2;
};

template <class T, int P, bool ROWS>
__global__ void __launch_bounds__(kCubeThreads, EDAB_CUBE_CTAS) cube_pass(Geom g, PassArgs<T> a) {
  constexpr int VW = 16 / static_cast<int>(sizeof(T));  // samples per 16-byte copy
  constexpr int PP = ROWS ? 1 : P;                        // sample stride in shared memory
  using V16 = typename Vec16<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Win win_s[kMaxRungs];
  __shared__ T fac_s[kMaxRungs];
  __shared__ int32_t any_s;
  const int64_t b = blockIdx.y;
  const int axis = a.axis;
  // (a kernel parameter indexed by a runtime value would be copied to local memory)
  const int32_t n = elem_n(g, b, axis);
  const int64_t inner = ROWS ? 1 : geom_stride(g, axis);  // column panels: the axis stride
  const int64_t step = ROWS ? 1 : inner;
  const int32_t TS = tot_slots(n);
  const int32_t LS = ROWS ? row_stride<T>(n) : 1;  // line stride in shared memory
  const int32_t gel = group_elems<T>(n, P, ROWS);
  T* V0 = reinterpret_cast<T*>(smem_raw);
  T* V1 = a.dbuf ? V0 + gel : V0;  // a CTA that stages once keeps one staging buffer
  T* R = V1 + gel;
  T* tot = R + gel;
  const int32_t j_begin = a.rung_loop ? 0 : static_cast<int32_t>(blockIdx.z);
  const int32_t nr = a.rung_loop ? a.rungs : 1;
  const bool box = a.op == static_cast<int>(CubeOp::kBox);
  const int nf = a.op == static_cast<int>(CubeOp::kMaxMin) ? 2 : 1;
  // the windows of this CTA's rungs, once
  if (threadIdx.x == 0) any_s = 0;
  __syncthreads();
  for (int32_t jj = threadIdx.x; jj < nr; jj += kCubeThreads) {
    const int32_t w = a.win[static_cast<int64_t>(j_begin + jj) * g.batch + b];
    Win q{};
    if (w >= 1) {
      q = make_win(n, w);
      any_s = 1;
      if (box && a.last) {
        double prod = 1.0;
#pragma unroll
        for (int ax = 0; ax < kMaxDim; ++ax) {
          if (ax < g.dim) prod *= static_cast<double>(2 * min((w - 1) / 2, (g.len ? n : g.n[ax]) - 1) + 1);
        }
        fac_s[jj] = static_cast<T>(1.0 / prod);
      }
    }
    win_s[jj] = q;  // wa == 0: the rung skips this element
  }
  __syncthreads();
  if (!any_s) return;
  const int64_t g0 = static_cast<int64_t>(blockIdx.x) * a.gpc;
  const int64_t ng = min(static_cast<int64_t>(a.gpc), a.groups - g0);
  if (ng <= 0) return;
  const int64_t eoff = b * g.field;
  // one staging per group when every rung and field reads the same input, else one per field
  const bool shared_in = a.in_stride == 0 && (nf == 1 || a.in1 == nullptr);
  const int nst = shared_in ? 1 : nf;
  const int64_t S = ng * nst;
  const bool async = a.vec && a.bits == nullptr && (ROWS || P >= VW);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // copy roles. Rows: kWpl warps per line, lanes over 16-byte units. Column panels: QP units per
  // panel row, threads over rows.
  constexpr int kWpl = P >= kWarps ? 1 : kWarps / P;
  constexpr int QP = P >= VW ? P / VW : 1;
  const int r_p = warp / kWpl;
  const int32_t r_u0 = lane + 32 * (warp % kWpl);
  const int32_t r_du = 32 * kWpl;
  const int c_q = threadIdx.x % QP;
  const int32_t c_i0 = threadIdx.x / QP;
  const int32_t c_di = kCubeThreads / QP;
  const auto src_of = [&](int f) -> const T* {
    const T* s = (f == 0 || a.in1 == nullptr) ? a.in0 : a.in1;
    return s + static_cast<int64_t>(j_begin) * a.in_stride + eoff;
  };
  // issue the 16-byte copies of one staging (async mode)
  const auto issue = [&](T* Vb, const GroupPos& s, const T* src) {
    if constexpr (ROWS) {
      if ((s.mask >> r_p) & 1u) {
        const int32_t units = (n + VW - 1) / VW;
        const T* line = src + s.base + static_cast<int64_t>(r_p) * g.pitch;
        T* dst = Vb + r_p * LS;
        for (int32_t u = r_u0; u < units; u += r_du) cp_async16(dst + u * VW, line + u * VW);
      }
    } else {
      if (s.mask) {
        const T* col = src + s.base + c_q * VW;
        for (int32_t i = c_i0; i < n; i += c_di) cp_async16(Vb + i * P + c_q * VW, col + static_cast<int64_t>(i) * step);
      }
    }
  };
  // order keys in place over the units this thread copied (async mode, max / min)
  const auto keys = [&](T* Vb, const GroupPos& s) {
    if constexpr (ROWS) {
      if ((s.mask >> r_p) & 1u) {
        const int32_t units = (n + VW - 1) / VW;
        T* line = Vb + r_p * LS;
        for (int32_t u = r_u0; u < units; u += r_du) {
          T* v = line + u * VW;
#pragma unroll
          for (int k = 0; k < VW; ++k) v[k] = okey(v[k]);
        }
      }
    } else {
      if (s.mask) {
        for (int32_t i = c_i0; i < n; i += c_di) {
          T* v = Vb + i * P + c_q * VW;
#pragma unroll
          for (int k = 0; k < VW; ++k) v[k] = okey(v[k]);
        }
      }
    }
  };
  // synchronous staging (bit-field input, unaligned pointers, narrow column panels)
  const auto stage_sync = [&](T* Vb, const GroupPos& s, int f) {
    const T* src = a.bits ? nullptr : src_of(f);
    const uint8_t* bits = a.bits ? a.bits + eoff : nullptr;
    if constexpr (ROWS) {
      if ((s.mask >> r_p) & 1u) {
        const int64_t line = s.base + static_cast<int64_t>(r_p) * g.pitch;
        for (int32_t i = r_u0; i < n; i += r_du) {
          const T v = bits ? (((bits[line + i] >> a.bit) & 1u) ? T(1) : T(0)) : src[line + i];
          Vb[r_p * LS + i] = box ? v : okey(v);
        }
      }
    } else {
      if (s.mask) {
        const int p = threadIdx.x % P;
        for (int32_t i = threadIdx.x / P; i < n; i += kCubeThreads / P) {
          const int64_t at = s.base + static_cast<int64_t>(i) * step + p;
          const T v = bits ? (((bits[at] >> a.bit) & 1u) ? T(1) : T(0)) : src[at];
          Vb[i * P + p] = box ? v : okey(v);
        }
      }
    }
  };
  const bool detsq = box && a.last && a.epi == static_cast<int>(BoxEpi::kDetSq);
  const auto epi = [&](T y, T fac, T auxv) -> T {
    if (!box) return okey(y);
    if (a.last) {
      y = mul_rn(y, fac);
      if (detsq) {
        const T d = sub_rn(auxv, y);
        y = mul_rn(d, d);
      }
    }
    return y;
  };
  // the store of R as field f of rung j (pads of the contiguous axis written as 0)
  const auto store = [&](const GroupPos& s, int32_t j, int f, T fac) {
    T* dst = (f == 0 ? a.out0 : a.out1) + static_cast<int64_t>(j) * a.out_stride + eoff;
    const T* aux = detsq ? a.aux + eoff : nullptr;
    if constexpr (ROWS) {
      if (!((s.mask >> r_p) & 1u)) return;
      const int64_t line = s.base + static_cast<int64_t>(r_p) * g.pitch;
      const T* rl = R + r_p * LS;
      if (a.vec) {
        const int32_t units = static_cast<int32_t>(g.pitch) / VW;
        for (int32_t u = r_u0; u < units; u += r_du) {
          const int32_t i0 = u * VW;
          V16 yv = *reinterpret_cast<const V16*>(rl + i0);
          V16 av{};
          if (detsq) av = *reinterpret_cast<const V16*>(aux + line + i0);
          T* y = reinterpret_cast<T*>(&yv);
          const T* ax = reinterpret_cast<const T*>(&av);
#pragma unroll
          for (int k = 0; k < VW; ++k) y[k] = i0 + k < n ? epi(y[k], fac, ax[k]) : T(0);
          *reinterpret_cast<V16*>(dst + line + i0) = yv;
        }
      } else {
        for (int32_t i = r_u0; i < static_cast<int32_t>(g.pitch); i += r_du) {
          dst[line + i] = i < n ? epi(rl[i], fac, detsq ? aux[line + i] : T(0)) : T(0);
        }
      }
    } else {
      if (!s.mask) return;
      if (a.vec && P >= VW) {
        uint32_t live = 0;  // this thread's columns left of the row padding
#pragma unroll
        for (int k = 0; k < VW; ++k) live |= ((s.mask >> (c_q * VW + k)) & 1u) << k;
        for (int32_t i = c_i0; i < n; i += c_di) {
          const int64_t at = s.base + static_cast<int64_t>(i) * step + c_q * VW;
          V16 yv = *reinterpret_cast<const V16*>(R + i * P + c_q * VW);
          V16 av{};
          if (detsq) av = *reinterpret_cast<const V16*>(aux + at);
          T* y = reinterpret_cast<T*>(&yv);
          const T* ax = reinterpret_cast<const T*>(&av);
#pragma unroll
          for (int k = 0; k < VW; ++k) y[k] = ((live >> k) & 1u) ? epi(y[k], fac, ax[k]) : T(0);
          *reinterpret_cast<V16*>(dst + at) = yv;
        }
      } else {
        const int p = threadIdx.x % P;
        if (!((s.mask >> p) & 1u)) return;
        for (int32_t i = threadIdx.x / P; i < n; i += kCubeThreads / P) {
          const int64_t at = s.base + static_cast<int64_t>(i) * step + p;
          dst[at] = epi(R[i * P + p], fac, detsq ? aux[at] : T(0));
        }
      }
    }
  };
  unsigned long long acct = 0;
  GroupPos cur = group_at<P, ROWS>(g, g0, n, inner);
  group_finish<P, ROWS>(cur, g, n, inner);
  GroupPos nxt = cur;  // the group of the staging in flight
  if (async) {
    issue(V0, cur, src_of(0));
    cp_async_commit();
  }
  for (int64_t st = 0; st < S; ++st) {
    T* Vb = (st & 1) ? V1 : V0;
    const int f_st = nst == 1 ? 0 : static_cast<int>(st & 1);
    if (async) {
      if (st + 1 < S) {
        const int f_next = nst == 1 ? 0 : static_cast<int>((st + 1) & 1);
        if (f_next == 0) {
          group_next<P, ROWS>(nxt, g, n, inner);
          group_finish<P, ROWS>(nxt, g, n, inner);
        }
        issue((st & 1) ? V0 : V1, nxt, src_of(f_next));
      }
      cp_async_commit();
      cp_async_wait_prior();
      if (!box) keys(Vb, cur);
    } else {
      stage_sync(Vb, cur, f_st);
    }
    __syncthreads();
    const int32_t valid = __popc(cur.mask);
    if (a.bytes && threadIdx.x == 0) acct += static_cast<unsigned long long>(valid) * n * (a.bits ? 1u : sizeof(T));
    if (cur.mask) {
      const int32_t jn = shared_in ? nr : 1;
      for (int32_t jj = 0; jj < jn; ++jj) {
        const Win q = win_s[jj];
        if (q.wa == 0) continue;
        const T fac = box && a.last ? fac_s[jj] : T(1);
        const int f_lo = shared_in ? 0 : f_st;
        const int f_hi = shared_in ? nf : f_st + 1;
        for (int f = f_lo; f < f_hi; ++f) {
          const bool is_min =
              a.op == static_cast<int>(CubeOp::kMin) || (a.op == static_cast<int>(CubeOp::kMaxMin) && f == 1);
          if (box) run_stage<T, kOpSum, P, PP>(Vb, R, tot, n, TS, q, LS, a.seq_share);
          else if (is_min) run_stage<T, kOpMinK, P, PP>(Vb, R, tot, n, TS, q, LS, a.seq_share);
          else run_stage<T, kOpMaxK, P, PP>(Vb, R, tot, n, TS, q, LS, a.seq_share);
          store(cur, j_begin + jj, f, fac);
          if (a.bytes && threadIdx.x == 0) acct += static_cast<unsigned long long>(valid) * n * sizeof(T);
          __syncthreads();  // the next stage rewrites R and tot
        }
      }
    }
    // the next staging: a new group after the last field of this one
    if (nst == 1 || (st & 1)) {
      group_next<P, ROWS>(cur, g, n, inner);
      group_finish<P, ROWS>(cur, g, n, inner);
    }
  }
  if (a.bytes && threadIdx.x == 0 && acct) atomicAdd(a.bytes, acct);
}

// ---------------------------------------------------------------------------------------------
// Lines too long to stage in shared memory (1-D signals beyond the staged capacity; the other
// axes stay within it). The line's fold input (order keys for max / min, the samples or the bit
// field's 0 / 1 for sums) is written once per element into a global scratch (long_line_input).
// Then the line is cut into tiles of kLongTile outputs, one CTA per tile, element and rung: the CTA
// stages the samples of the segments its outputs need (x - r lies in a segment of the reversed
// line, whose H it folds; x + r in a segment of the line, whose G it folds; every segment whole,
// from its start, so every fold is the canonical one) and runs the staged kernel's fold phases on
// them in shared memory. A window whose segments do not fit a tile's shared memory folds in the
// segment launches further down (chunk totals, carries, H and G folds over many CTAs, on global
// memory: the line and its output stay in L2). Every bit of the result is that of the staged
// kernel.
template <class T>
__global__ void __launch_bounds__(kThreads) long_line_input(Geom g, PassArgs<T> a, T* keys) {
  const int64_t total = g.batch * g.pitch;  // 1-D: one row per element
  const bool box = a.op == static_cast<int>(CubeOp::kBox);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    T v;
    if (a.bits) v = ((a.bits[i] >> a.bit) & 1u) ? T(1) : T(0);
    else v = a.in0[i];
    keys[i] = box ? v : okey(v);
  }
}

constexpr int32_t kLongTile = 4096;  // outputs per tile

// The bounding interval [lo, hi] of the line samples that the extended positions [u, v] read
// (reflect_index; -n <= u <= v < 2n).
__device__ __forceinline__ void reflect_span(int32_t u, int32_t v, int32_t n, int32_t* lo, int32_t* hi) {
  int32_t l = max(u, 0), h = min(v, n - 1);
  if (u < 0) {
    l = 0;
    h = max(h, min(-u - 1, n - 1));
  }
  if (v > n - 1) {
    h = n - 1;
    l = min(l, max(2 * n - 1 - v, 0));
  }
  *lo = l;
  *hi = h;
}

// Whether the tiles of a line fold window q in shared memory of smem_elems samples: by bounds of any
// tile's samples, slots and totals (nv, nx <= L + 2r + 2wa + 4, TS <= ((L + 2wa) / wa + 2) cps, checked
// against every tile's exact extents on the CPU), so that every tile of a line, and the kernels of
// the wider windows, decide alike.
// Windows of one-chunk segments (cps 1) fold without chunk totals and always fit.
__device__ __forceinline__ bool long_tiled(const Win& q, int32_t smem_elems) {
  const int32_t span16 = (kLongTile + 2 * q.r + 2 * q.wa + 4 + 3) & ~3;
  const int32_t ts_bound = q.cps == 1 ? 0 : ((kLongTile + 2 * q.wa) / q.wa + 2) * q.cps;
  return 2 * span16 + 2 * ts_bound <= smem_elems;
}

template <class T>
__global__ void __launch_bounds__(kCubeThreads) cube_long(Geom g, PassArgs<T> a, const T* __restrict__ keys,
                                                         int32_t smem_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ T fac_s;
  const int64_t b = blockIdx.y;
  const int32_t j = static_cast<int32_t>(blockIdx.z);
  const int32_t n = elem_len(g, b);
  const int32_t X0 = static_cast<int32_t>(blockIdx.x) * kLongTile;
  if (X0 >= n) return;
  const int32_t w = a.win[static_cast<int64_t>(j) * g.batch + b];
  if (w < 1) return;
  const int32_t X1 = min(X0 + kLongTile, n);
  const bool box = a.op == static_cast<int>(CubeOp::kBox);
  const int nf = a.op == static_cast<int>(CubeOp::kMaxMin) ? 2 : 1;
  const bool detsq = box && a.last && a.epi == static_cast<int>(BoxEpi::kDetSq);
  const Win q = make_win(n, w);
  if (threadIdx.x == 0 && box && a.last) fac_s = static_cast<T>(1.0 / static_cast<double>(q.wa));
  // the tile's segments: G of the line's segments holding x + r, H of the reversed line's holding
  // n - 1 - (x - r), for x in [X0, X1)
  const int32_t e_max = n - 1 + q.r;
  Win t = q;
  t.gk0 = floor_div32(X0 + q.r - q.o, q.wa) - q.k_lo;
  t.gn = floor_div32(X1 - 1 + q.r - q.o, q.wa) - q.k_lo - t.gk0 + 1;
  t.hk0 = floor_div32(n - X1 + q.r - q.o, q.wa) - q.k_lo;
  t.hn = floor_div32(n - 1 - X0 + q.r - q.o, q.wa) - q.k_lo - t.hk0 + 1;
  const int32_t gs = q.o + (q.k_lo + t.gk0) * q.wa, ge = min(gs + t.gn * q.wa - 1, e_max);
  const int32_t hs = q.o + (q.k_lo + t.hk0) * q.wa, he = min(hs + t.hn * q.wa - 1, e_max);
  // the samples they read, and the output slots they write (H: n - 1 + r - e for e >= r; G: e - r)
  int32_t glo, ghi, hlo, hhi;
  reflect_span(gs, ge, n, &glo, &ghi);
  reflect_span(hs, he, n, &hlo, &hhi);
  const int32_t vlo = min(glo, n - 1 - hhi), vhi = max(ghi, n - 1 - hlo);
  const int32_t xlo = min(max(gs, q.r) - q.r, n - 1 + q.r - he);
  const int32_t xhi = max(ge - q.r, n - 1 + q.r - max(hs, q.r));
  const int32_t nv = vhi - vlo + 1, nx = xhi - xlo + 1;
  const int32_t TS = q.cps == 1 ? 0 : max(t.gn, t.hn) * q.cps;  // one-chunk segments use no totals
  const int32_t nv16 = (nv + 3) & ~3, nx16 = (nx + 3) & ~3;  // 16-byte aligned regions
  // wider windows fold in the segment kernels below (every tile of the line decides alike); the
  // exact extents lie within the bounds (a tile past them would return, no access outside)
  if (!long_tiled(q, smem_elems) || nv16 + nx16 + 2 * TS > smem_elems) return;
  __syncthreads();
  const T* line = keys + b * g.pitch;
  unsigned long long acct = 0;
  T* Vs = reinterpret_cast<T*>(smem_raw);
  T* Rs = Vs + nv16;
  T* tot = Rs + nx16;
  for (int32_t i = threadIdx.x; i < nv; i += blockDim.x) Vs[i] = line[vlo + i];
  __syncthreads();
  for (int f = 0; f < nf; ++f) {
    const bool is_min = a.op == static_cast<int>(CubeOp::kMin) || (a.op == static_cast<int>(CubeOp::kMaxMin) && f == 1);
    // (the staged samples and slots at their line indices: only the staged ones are touched)
    if (box) run_stage<T, kOpSum, 1, 1, true>(Vs - vlo, Rs - xlo, tot, n, TS, t, 0, a.seq_share);
    else if (is_min) run_stage<T, kOpMinK, 1, 1, true>(Vs - vlo, Rs - xlo, tot, n, TS, t, 0, a.seq_share);
    else run_stage<T, kOpMaxK, 1, 1, true>(Vs - vlo, Rs - xlo, tot, n, TS, t, 0, a.seq_share);
    T* R = (f == 0 ? a.out0 : a.out1) + static_cast<int64_t>(j) * a.out_stride + b * g.field;
    const T* aux = detsq ? a.aux + b * g.field : nullptr;
    const int32_t end = X1 == n ? static_cast<int32_t>(g.pitch) : X1;  // the last tile writes the pads
    for (int32_t x = X0 + threadIdx.x; x < end; x += blockDim.x) {
      T y = T(0);
      if (x < n) {
        y = Rs[x - xlo];
        if (!box) {
          y = okey(y);
        } else if (a.last) {
          y = mul_rn(y, fac_s);
          if (detsq) {
            const T d = sub_rn(aux[x], y);
            y = mul_rn(d, d);
          }
        }
      }
      R[x] = y;
    }
    __syncthreads();  // the next field rewrites the slots and totals
  }
  acct = static_cast<unsigned long long>(X1 - X0) * sizeof(T) * (1 + nf);
  if (a.bytes && threadIdx.x == 0) atomicAdd(a.bytes, acct);
}

// The windows too wide for the tiles (their segments exceed a tile's shared memory) fold each line
// in four launches over many CTAs, with no CTA waiting for another: the chunk totals of both
// directions into a global table, the per-segment exclusive carries, the H folds into the output
// row, the G folds combined with them; then the pass's epilogue. The tasks and their arithmetic are
// those of the staged kernel's chunk schedule (one lane per chunk of a line), so every bit is the
// same. tot: per field, rung and element 2 x TSL samples (TSL = tot_slots of the longest line).
struct LongSeg {
  int64_t b;
  int32_t j, n, e_max;
  Win q;
  bool wide;  // the window folds here (not in the tiles)
};
template <class T>
__device__ __forceinline__ LongSeg long_seg(const Geom& g, const PassArgs<T>& a, int32_t smem_elems) {
  LongSeg L{};
  L.b = blockIdx.y;
  L.j = static_cast<int32_t>(blockIdx.z);
  L.n = elem_len(g, L.b);
  const int32_t w = a.win[static_cast<int64_t>(L.j) * g.batch + L.b];
  if (w < 1) return L;
  L.q = make_win(L.n, w);
  L.e_max = L.n - 1 + L.q.r;
  // (a wide window has segments of many chunks: nseg cps <= tot_slots(n) <= TSL, checked on the CPU
  // for every length and window; the kernels also leave any other window alone)
  L.wide = !long_tiled(L.q, smem_elems) && L.q.cps > 1 && L.q.nseg * L.q.cps <= tot_slots(L.n);
  return L;
}
template <class T>
__device__ __forceinline__ int op_of(const PassArgs<T>& a, int f) {
  if (a.op == static_cast<int>(CubeOp::kBox)) return kOpSum;
  return (a.op == static_cast<int>(CubeOp::kMin) || (a.op == static_cast<int>(CubeOp::kMaxMin) && f == 1)) ? kOpMinK
                                                                                                          : kOpMaxK;
}

// Chunk totals: task t < 2 nseg cps is (direction, segment, chunk), the line's G chunks first.
template <class T, int OP>
__device__ __forceinline__ void seg_totals(const LongSeg& L, const T* __restrict__ V, T* __restrict__ tot, int32_t TS) {
  const Win& q = L.q;
  const int32_t per_dir = q.nseg * q.cps;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < 2 * per_dir; t += stride) {
    const int dir = t >= per_dir;
    const int32_t kc = static_cast<int32_t>(t - dir * per_dir);
    const int32_t k = kc / q.cps, c = kc - k * q.cps;
    const int32_t s = q.o + (q.k_lo + k) * q.wa;
    const int32_t e_last = min(s + q.wa - 1, L.e_max);
    const int32_t c0 = s + 32 * c;
    if (c0 > e_last) continue;
    const int32_t c1 = min(c0 + 31, e_last);
    const int32_t n = L.n;
    T total;
    if (c0 >= 0 && c1 <= n - 1) {
      if (dir) {
        const T* vp = V + (n - 1 - c0);
        total = c1 == c0 + 31 ? chunk_total<T, OP, -1>(vp) : partial_total<T, OP, -1>(vp, c1 - c0 + 1);
      } else {
        const T* vp = V + c0;
        total = c1 == c0 + 31 ? chunk_total<T, OP, 1>(vp) : partial_total<T, OP, 1>(vp, c1 - c0 + 1);
      }
    } else {
      total = fold_chunk<T, OP>(V, 1, n, c0, c1, dir, [](int32_t, T) {});
    }
    tot[dir * TS + kc] = total;
  }
}

template <class T>
__global__ void __launch_bounds__(kThreads) long_totals(Geom g, PassArgs<T> a, const T* __restrict__ keys, int f,
                                                        T* tot_all, int32_t TSL, int32_t smem_elems) {
  const LongSeg L = long_seg(g, a, smem_elems);
  if (!L.wide) return;
  const T* V = keys + L.b * g.pitch;
  T* tot = tot_all + ((static_cast<int64_t>(L.j) * g.batch + L.b) * 2) * TSL;
  const int op = op_of(a, f);
  if (op == kOpSum) seg_totals<T, kOpSum>(L, V, tot, TSL);
  else if (op == kOpMinK) seg_totals<T, kOpMinK>(L, V, tot, TSL);
  else seg_totals<T, kOpMaxK>(L, V, tot, TSL);
}

// Exclusive carries per segment and direction, in place (slot c holds the carry of chunk c >= 1),
// sequential in chunk order (the canonical carries of sums), from shared memory.
template <class T>
__global__ void __launch_bounds__(kThreads) long_carries(Geom g, PassArgs<T> a, int f, T* tot_all, int32_t TSL,
                                                         int32_t smem_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const LongSeg L = long_seg(g, a, smem_elems);
  if (!L.wide) return;
  const Win& q = L.q;
  T* tot = tot_all + ((static_cast<int64_t>(L.j) * g.batch + L.b) * 2) * TSL;
  T* st = reinterpret_cast<T*>(smem_raw);  // [2][nseg cps]
  const int32_t per_dir = q.nseg * q.cps;
  for (int32_t i = threadIdx.x; i < 2 * per_dir; i += blockDim.x) {
    const int dir = i >= per_dir;
    st[i] = tot[dir * TSL + (i - dir * per_dir)];
  }
  __syncthreads();
  const int op = op_of(a, f);
  for (int32_t t = threadIdx.x; t < 2 * q.nseg; t += blockDim.x) {
    const int dir = t >= q.nseg;
    const int32_t k = t - dir * q.nseg;
    const int32_t s = q.o + (q.k_lo + k) * q.wa;
    const int32_t e_last = min(s + q.wa - 1, L.e_max);
    const int32_t nch = (e_last - s) / 32 + 1;
    T* tl = st + dir * per_dir + k * q.cps;
    T run = tl[0];
    for (int32_t c = 1; c < nch; ++c) {
      const T next = tl[c];
      tl[c] = run;
      run = op == kOpSum ? fop<kOpSum>(run, next) : (op == kOpMinK ? fop<kOpMinK>(run, next) : fop<kOpMaxK>(run, next));
    }
  }
  __syncthreads();
  for (int32_t i = threadIdx.x; i < 2 * per_dir; i += blockDim.x) {
    const int dir = i >= per_dir;
    tot[dir * TSL + (i - dir * per_dir)] = st[i];
  }
}

// H (the reversed line's G) of task t = (segment, chunk) into the output slots n - 1 + r - e (e >= r).
template <class T, int OP>
__device__ __forceinline__ void seg_fold_h(const LongSeg& L, const T* __restrict__ V, T* __restrict__ R,
                                           const T* __restrict__ tot, int32_t TS) {
  const Win& q = L.q;
  const int32_t n = L.n;
  const T idn = fold_identity<T, OP>();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < q.nseg * q.cps; t += stride) {
    const int32_t kc = static_cast<int32_t>(t);
    const int32_t k = kc / q.cps, c = kc - k * q.cps;
    const int32_t s = q.o + (q.k_lo + k) * q.wa;
    const int32_t e_last = min(s + q.wa - 1, L.e_max);
    const int32_t c0 = s + 32 * c;
    if (c0 > e_last) continue;
    const int32_t c1 = min(c0 + 31, e_last);
    const T cv = c > 0 ? tot[TS + kc] : idn;
    if (c0 >= 0 && c1 <= n - 1) {
      const T* vp = V + (n - 1 - c0);
      T* rp = R + (n - 1 + q.r - c0);
      if (c1 == c0 + 31 && c0 >= q.r) chunk_h<T, OP, 1>(vp, rp, cv);
      else partial_h<T, OP, 1>(vp, rp, c1 - c0 + 1, max(0, q.r - c0), cv);
    } else {
      fold_chunk<T, OP>(V, 1, n, c0, c1, 1, [&](int32_t e, T loc) {
        if (e >= q.r) R[n - 1 + q.r - e] = fop<OP>(cv, loc);
      });
    }
  }
}
// G of task t combined with the H in its slots: y(x) = op(H(x - r), G(x + r)), slot x = e - r.
template <class T, int OP>
__device__ __forceinline__ void seg_fold_g(const LongSeg& L, const T* __restrict__ V, T* __restrict__ R,
                                           const T* __restrict__ tot) {
  const Win& q = L.q;
  const int32_t n = L.n;
  const T idn = fold_identity<T, OP>();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < q.nseg * q.cps; t += stride) {
    const int32_t kc = static_cast<int32_t>(t);
    const int32_t k = kc / q.cps, c = kc - k * q.cps;
    const int32_t s = q.o + (q.k_lo + k) * q.wa;
    const int32_t e_al = s + q.wa - 1;
    const int32_t e_last = min(e_al, L.e_max);
    const int32_t c0 = s + 32 * c;
    if (c0 > e_last) continue;
    const int32_t c1 = min(c0 + 31, e_last);
    const T cv = c > 0 ? tot[kc] : idn;
    if (c0 >= 0 && c1 <= n - 1) {
      const T* vp = V + c0;
      T* rp = R + (c0 - q.r);
      if (c1 == c0 + 31 && c0 >= q.r) chunk_g<T, OP, 1>(vp, rp, cv, c1 == e_al);
      else partial_g<T, OP, 1>(vp, rp, c1 - c0 + 1, max(0, q.r - c0), cv, c1 == e_al);
    } else {
      fold_chunk<T, OP>(V, 1, n, c0, c1, 0, [&](int32_t e, T loc) {
        if (e < q.r) return;
        const T gv = fop<OP>(cv, loc);
        T* slot = R + (e - q.r);
        const T h = *slot;
        if constexpr (OP == kOpSum) {
          const T sum = add_rn(h, gv);
          *slot = e == e_al ? mul_rn(sum, T(0.5)) : sum;
        } else {
          *slot = fop<OP>(h, gv);
        }
      });
    }
  }
}

// pass H (G = false) or G (G = true) of field f over the wide windows
template <class T, bool G>
__global__ void __launch_bounds__(kThreads) long_folds(Geom g, PassArgs<T> a, const T* __restrict__ keys, int f,
                                                       const T* tot_all, int32_t TSL, int32_t smem_elems) {
  const LongSeg L = long_seg(g, a, smem_elems);
  if (!L.wide) return;
  const T* V = keys + L.b * g.pitch;
  T* R = (f == 0 ? a.out0 : a.out1) + static_cast<int64_t>(L.j) * a.out_stride + L.b * g.field;
  const T* tot = tot_all + ((static_cast<int64_t>(L.j) * g.batch + L.b) * 2) * TSL;
  const int op = op_of(a, f);
  if constexpr (G) {
    if (op == kOpSum) seg_fold_g<T, kOpSum>(L, V, R, tot);
    else if (op == kOpMinK) seg_fold_g<T, kOpMinK>(L, V, R, tot);
    else seg_fold_g<T, kOpMaxK>(L, V, R, tot);
  } else {
    if (op == kOpSum) seg_fold_h<T, kOpSum>(L, V, R, tot, TSL);
    else if (op == kOpMinK) seg_fold_h<T, kOpMinK>(L, V, R, tot, TSL);
    else seg_fold_h<T, kOpMaxK>(L, V, R, tot, TSL);
  }
}

// The pass's epilogue on the folded row of field f (order keys back to values; the box's scale and
// detail energy on its last pass); the pads are written 0.
template <class T>
__global__ void __launch_bounds__(kThreads) long_epilogue(Geom g, PassArgs<T> a, int f, int32_t smem_elems) {
  const LongSeg L = long_seg(g, a, smem_elems);
  if (!L.wide) return;
  const bool box = a.op == static_cast<int>(CubeOp::kBox);
  const bool detsq = box && a.last && a.epi == static_cast<int>(BoxEpi::kDetSq);
  const T fac = static_cast<T>(1.0 / static_cast<double>(L.q.wa));
  T* R = (f == 0 ? a.out0 : a.out1) + static_cast<int64_t>(L.j) * a.out_stride + L.b * g.field;
  const T* aux = detsq ? a.aux + L.b * g.field : nullptr;
  const int32_t pitch = static_cast<int32_t>(g.pitch);
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pitch; i += gridDim.x * blockDim.x) {
    T y = T(0);
    if (i < L.n) {
      y = R[i];
      if (!box) {
        y = okey(y);
      } else if (a.last) {
        y = mul_rn(y, fac);
        if (detsq) {
          const T d = sub_rn(aux[i], y);
          y = mul_rn(d, d);
        }
      }
    }
    R[i] = y;
  }
  if (a.bytes && f == 0 && blockIdx.x == 0 && threadIdx.x == 0) {
    const int nf = a.op == static_cast<int>(CubeOp::kMaxMin) ? 2 : 1;
    atomicAdd(a.bytes, static_cast<unsigned long long>(L.n) * sizeof(T) * (1 + nf));
  }
}

thread_local void* t_long_scratch = nullptr;
thread_local size_t t_long_bytes = 0;

// The long-line scratch: the lines' fold input (batch x pitch samples), then the wide windows' chunk
// totals (rungs x batch x 2 x tot_slots(longest line) samples).
size_t long_keys_bytes(const Geom& g, size_t es) {
  return (static_cast<size_t>(g.batch) * static_cast<size_t>(g.pitch) * es + 255) / 256 * 256;
}
size_t long_scratch_need(const Geom& g, size_t es) {
  return long_keys_bytes(g, es) +
         static_cast<size_t>(kMaxRungs) * static_cast<size_t>(g.batch) * 2 * static_cast<size_t>(tot_slots(g.n_last)) * es;
}

size_t smem_bytes(int32_t n, int P, bool rows, size_t es, bool dbuf = true) {
  const int32_t gel = es == 4 ? group_elems<float>(n, P, rows) : group_elems<double>(n, P, rows);
  return (static_cast<size_t>(dbuf ? 3 : 2) * gel + static_cast<size_t>(2) * tot_slots(n) * P) * es;
}

template <class T>
void allow_smem(int bytes) {
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

struct DevFacts {
  int sms = 148;
  size_t smem = 227 * 1024;  // dynamic shared memory a CTA may take
  size_t sm_smem = 228 * 1024;  // shared memory of an SM
};
DevFacts dev_facts() {
  static std::mutex mu;
  static DevFacts f[64];
  static bool have[64] = {};
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (!have[dev]) {
    int optin = 0, sms = 0, per_sm = 0;
    EDAB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    EDAB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EDAB_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    f[dev].sms = sms;
    f[dev].smem = static_cast<size_t>(optin) - 2048;  // the kernel's static shared memory
    f[dev].sm_smem = static_cast<size_t>(per_sm);
    allow_smem<float>(static_cast<int>(f[dev].smem));
    allow_smem<double>(static_cast<int>(f[dev].smem));
    have[dev] = true;
  }
  return f[dev];
}

// Lines per group (a power of two up to 8): 8 lines for column panels (whole sectors) and rows;
// fewer where the element's rows run out or the shared memory would hold fewer than two CTAs.
template <class T>
int lines_per_cta(const Geom& g, int axis, size_t cap) {
  const int32_t n = g.n[axis];
  const bool rows = axis == g.dim - 1;
  int P = 8;
  if (rows) {
    while (P > kWarps) P /= 2;  // rows: a warp (or more) stages and stores each line
    while (P > 1 && P / 2 >= g.rows) P /= 2;
  }
  while (P > 1 && smem_bytes(n, P, rows, sizeof(T)) > cap / 2) P /= 2;
  if (smem_bytes(n, P, rows, sizeof(T)) > cap) {
    throw std::invalid_argument("edab: an axis of " + std::to_string(n) + " samples exceeds the shared-memory line capacity");
  }
  return P;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <class T>
void launch_long(cudaStream_t s, const Geom& g, PassArgs<T> a) {
  if (g.dim != 1) throw std::invalid_argument("edab: lines beyond the shared-memory capacity are 1-D only");
  const size_t keys_bytes = long_keys_bytes(g, sizeof(T));
  const int32_t TSL = tot_slots(g.n_last);
  if (t_long_scratch == nullptr || t_long_bytes < long_scratch_need(g, sizeof(T))) {
    throw std::logic_error("edab: a long-line cube pass needs the thread's long-line scratch");
  }
  T* keys = static_cast<T*>(t_long_scratch);
  T* tot = reinterpret_cast<T*>(static_cast<unsigned char*>(t_long_scratch) + keys_bytes);
  long_line_input<T><<<blocks_for(g.batch * g.pitch), kThreads, 0, s>>>(g, a, keys);
  EDAB_LAUNCH("long_line_input");
  // shared memory: a line's chunk totals (the wide windows' carries), and at least half an SM's (two
  // tile CTAs per SM) for the tiles' samples, slots and totals
  const size_t whole = static_cast<size_t>(2) * TSL * sizeof(T);
  if (whole > dev_facts().smem) throw std::invalid_argument("edab: a line is too long for the long-line cube pass");
  const size_t half_sm = (dev_facts().sm_smem / 2 - 2048) / 16 * 16;
  const size_t smem = std::min(dev_facts().smem, std::max(whole, half_sm)) / 16 * 16;
  once_on_device(reinterpret_cast<const void*>(cube_long<T>), [] {
    EDAB_CUDA(cudaFuncSetAttribute(cube_long<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(dev_facts().smem)));
    EDAB_CUDA(cudaFuncSetAttribute(long_carries<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(dev_facts().smem)));
  });
  const int64_t tiles = (g.n_last + kLongTile - 1) / kLongTile;
  if (g.batch > 65535 || a.rungs > kMaxRungs) throw std::invalid_argument("edab: cube launch too large");
  a.bytes = cube_bytes_counter();
  profile_cube_launch(s, true);
  const dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(g.batch), static_cast<unsigned>(a.rungs));
  const int32_t smem_elems = static_cast<int32_t>(smem / sizeof(T));
  cube_long<T><<<grid, kCubeThreads, smem, s>>>(g, a, keys, smem_elems);
  EDAB_LAUNCH("cube_long");
  // the wide windows (the kernels return at once for the windows the tiles took)
  const int nf = a.op == static_cast<int>(CubeOp::kMaxMin) ? 2 : 1;
  const unsigned xt = static_cast<unsigned>(std::clamp<int64_t>((TSL + kThreads - 1) / kThreads, 1, 32));
  const unsigned xe = static_cast<unsigned>(std::clamp<int64_t>((g.pitch + 4 * kThreads - 1) / (4 * kThreads), 1, 16));
  const dim3 gt(xt, static_cast<unsigned>(g.batch), static_cast<unsigned>(a.rungs));
  const dim3 g1(1, static_cast<unsigned>(g.batch), static_cast<unsigned>(a.rungs));
  const dim3 ge(xe, static_cast<unsigned>(g.batch), static_cast<unsigned>(a.rungs));
  for (int f = 0; f < nf; ++f) {
    long_totals<T><<<gt, kThreads, 0, s>>>(g, a, keys, f, tot, TSL, smem_elems);
    EDAB_LAUNCH("long_totals");
    long_carries<T><<<g1, kThreads, whole, s>>>(g, a, f, tot, TSL, smem_elems);
    EDAB_LAUNCH("long_carries");
    long_folds<T, false><<<gt, kThreads, 0, s>>>(g, a, keys, f, tot, TSL, smem_elems);
    EDAB_LAUNCH("long_folds");
    long_folds<T, true><<<gt, kThreads, 0, s>>>(g, a, keys, f, tot, TSL, smem_elems);
    EDAB_LAUNCH("long_folds");
    long_epilogue<T><<<ge, kThreads, 0, s>>>(g, a, f, smem_elems);
    EDAB_LAUNCH("long_epilogue");
  }
  profile_cube_launch(s, false);
}

template <class T>
void launch_pass(cudaStream_t s, const Geom& g, PassArgs<T> a) {
  const DevFacts f = dev_facts();
  const bool rows = a.axis == g.dim - 1;
  const CubeTune tune = cube_tune_for(g, a.axis, sizeof(T));
  a.seq_share = tune.seq_share > 0 ? tune.seq_share : kSeqShare;
  if (rows && smem_bytes(g.n[a.axis], 1, true, sizeof(T)) > f.smem) {
    launch_long<T>(s, g, a);
    return;
  }
  int P = lines_per_cta<T>(g, a.axis, f.smem);
  if (tune.lines > 0 && tune.lines <= 8 && smem_bytes(g.n[a.axis], tune.lines, rows, sizeof(T)) <= f.smem &&
      (!rows || (tune.lines <= std::max<int64_t>(1, g.rows) && tune.lines <= kWarps))) {
    P = tune.lines;
  }
  if (a.rungs > kMaxRungs) throw std::invalid_argument("edab: more rungs than a cube launch holds");
  int64_t groups;
  if (rows) {
    groups = (g.rows + P - 1) / P;
  } else {
    int64_t outer = 1;
    for (int ax = 0; ax < a.axis; ++ax) outer *= g.n[ax];
    groups = outer * (g.stride[a.axis] / P);
  }
  // line groups per CTA: the tuned value, else one (measured fastest on the default shapes)
  int gpc = tune.groups > 0 ? std::min(tune.groups, kMaxGroupsPerCta) : 1;
  gpc = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(gpc, groups)));
  // a second staging buffer only for a CTA that stages more than once (several groups, or the two
  // fields of a max+min pass with separate inputs)
  const int nf = a.op == static_cast<int>(CubeOp::kMaxMin) ? 2 : 1;
  const bool shared_in = a.in_stride == 0 && (nf == 1 || a.in1 == nullptr);
  a.dbuf = (gpc > 1 || (shared_in ? 1 : nf) > 1) ? 1 : 0;
  const size_t smem = smem_bytes(g.n[a.axis], P, rows, sizeof(T), a.dbuf != 0);
  const int64_t gx = (groups + gpc - 1) / gpc;
  if (gx > 0x7fffffffLL || g.batch > 65535) throw std::invalid_argument("edab: cube launch too large");
  a.groups = groups;
  a.gpc = gpc;
  const int64_t es = static_cast<int64_t>(sizeof(T));
  a.vec = aligned16(a.in0) && aligned16(a.in1) && aligned16(a.out0) && aligned16(a.out1) && aligned16(a.aux) &&
          (a.in_stride * es) % 16 == 0 && (a.out_stride * es) % 16 == 0 && (g.field * es) % 16 == 0 &&
          (g.pitch * es) % 16 == 0 && (rows || (g.stride[a.axis] * es) % 16 == 0);
  const dim3 grid(static_cast<unsigned>(gx), static_cast<unsigned>(g.batch), a.rung_loop ? 1u : static_cast<unsigned>(a.rungs));
  a.bytes = cube_bytes_counter();
  profile_cube_launch(s, true);
#define EDAB_CUBE_LAUNCH(PV)                                                    \
  do {                                                                          \
    if (rows) cube_pass<T, PV, true><<<grid, kCubeThreads, smem, s>>>(g, a);        \
    else cube_pass<T, PV, false><<<grid, kCubeThreads, smem, s>>>(g, a);            \
  } while (0)
  switch (P) {
    case 1: EDAB_CUBE_LAUNCH(1); break;
    case 2: EDAB_CUBE_LAUNCH(2); break;
    case 4: EDAB_CUBE_LAUNCH(4); break;
    default: EDAB_CUBE_LAUNCH(8); break;
  }
#undef EDAB_CUBE_LAUNCH
  EDAB_LAUNCH("cube_pass");
  profile_cube_launch(s, false);
}

}  // namespace

template <class T>
void cube(cudaStream_t s, const Geom& g, CubeOp op, const CubeArgs<T>& c) {
  const int D = g.dim;
  const int32_t rungs = c.rungs < 1 ? 1 : c.rungs;
  PassArgs<T> base{};
  base.win = c.win;
  base.rungs = rungs;
  base.out_stride = c.out_stride;
  base.op = static_cast<int32_t>(op);
  base.aux = c.aux;
  if (op == CubeOp::kBox) {
    for (int ax = 0; ax < D; ++ax) {
      PassArgs<T> a = base;
      a.axis = ax;
      a.last = ax == D - 1;
      a.epi = a.last ? static_cast<int32_t>(c.epi) : 0;
      if (ax == 0) {
        a.in0 = c.in;
        a.bits = c.src_bits;
        a.bit = c.bit;
        a.in_stride = 0;
        a.rung_loop = 1;
      } else {
        a.in0 = c.out0;
        a.in_stride = c.out_stride;
        a.rung_loop = 0;
      }
      a.out0 = c.out0;
      launch_pass<T>(s, g, a);
    }
    return;
  }
  for (int ax = D - 1; ax >= 0; --ax) {
    PassArgs<T> a = base;
    a.axis = ax;
    const bool first = ax == D - 1;
    if (first) {
      a.in0 = c.in;
      a.in1 = nullptr;
      a.in_stride = 0;
      a.rung_loop = 1;
    } else {
      a.in0 = c.out0;
      a.in1 = op == CubeOp::kMaxMin ? c.out1 : nullptr;
      a.in_stride = c.out_stride;
      a.rung_loop = 0;
    }
    a.out0 = c.out0;
    a.out1 = c.out1;
    launch_pass<T>(s, g, a);
  }
}

void set_long_line_scratch(void* p, size_t bytes) {
  t_long_scratch = p;
  t_long_bytes = bytes;
}

size_t long_line_scratch_bytes(const Geom& g, size_t es) {
  if (g.dim != 1) return 0;
  const size_t staged = es == 4 ? smem_bytes(g.n_last, 1, true, 4) : smem_bytes(g.n_last, 1, true, 8);
  if (staged <= dev_facts().smem) return 0;
  return long_scratch_need(g, es);
}

template <class T>
void cube_simple(cudaStream_t s, const Geom& g, CubeOp op, const T* in, T* out0, T* out1, const int32_t* win) {
  CubeArgs<T> a{};
  a.in = in;
  a.out0 = out0;
  a.out1 = out1;
  a.win = win;
  a.rungs = 1;
  cube<T>(s, g, op, a);
}

template void cube<float>(cudaStream_t, const Geom&, CubeOp, const CubeArgs<float>&);
template void cube<double>(cudaStream_t, const Geom&, CubeOp, const CubeArgs<double>&);
template void cube_simple<float>(cudaStream_t, const Geom&, CubeOp, const float*, float*, float*, const int32_t*);
template void cube_simple<double>(cudaStream_t, const Geom&, CubeOp, const double*, double*, double*, const int32_t*);

}  // namespace edab
