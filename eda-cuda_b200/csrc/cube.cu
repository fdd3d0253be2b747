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
// B200 design. A CTA stages P lines of one element (rows of the contiguous axis, or a panel of P
// adjacent columns of an outer axis: whole 32-byte sectors) in shared memory, interleaved: sample i
// of line p at i * PP + p. Lanes map to lines: P lanes of a warp ("a worker") run the same fold
// task on their P lines, so control flow is uniform and a worker's shared-memory accesses are
// consecutive words. The fold tasks (one per direction, segment and 32-sample chunk) are spread over
// the CTA's workers: chunk totals, per-segment exclusive carries, then the H folds and the G folds
// combined with them. P is a compile-time constant, so a whole 32-sample chunk inside the line runs
// as an unrolled fold with immediate shared-memory offsets; only the chunks that cross a line end,
// the window's first r samples or a segment end take the general path. A chunk without a carry
// folds from the operation's identity (-0 for sums, the extreme keys for max / min), which changes
// no bit of any result. The first pass of a cube stages its input once and runs every rung of the
// ladder on it (the operators' rung group); later passes run one rung per CTA.
#include "engine.cuh"

#include <algorithm>
#include <climits>
#include <mutex>

namespace edab {
namespace {

constexpr int kOpMaxK = 0, kOpMinK = 1, kOpSum = 2;
constexpr int kWarps = kThreads / 32;
constexpr int kStageLoads = 8;  // global loads in flight per thread while staging lines

__host__ __device__ constexpr int32_t tot_slots(int32_t n) { return n / 8 + 24; }
// Words per staged sample row: P lines plus one (odd, so a transposed row staging of 32
// consecutive samples hits 32 distinct banks); one line is stored contiguously.
__host__ __device__ constexpr int32_t line_pitch(int P) { return P == 1 ? 1 : P + 1; }

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
};
// 32-bit arithmetic throughout (n <= 8192 and wa <= 2n - 1, so n (wa + 1) / 2 < 2^27): the 64-bit
// integer divisions of a general formula are long emulated sequences on the GPU.
__device__ __forceinline__ int32_t floor_div32(int32_t a, int32_t b) {  // b > 0
  const int32_t q = a / b;
  return (a % b != 0 && a < 0) ? q - 1 : q;
}
__device__ __forceinline__ Win make_win(int32_t n, int32_t w) {
  Win q;
  const int32_t half = (w - 1) >> 1;
  q.r = min(half, n - 1);
  q.wa = 2 * q.r + 1;
  q.o = static_cast<int32_t>((static_cast<uint32_t>(n) * static_cast<uint32_t>((q.wa + 1) >> 1)) %
                             static_cast<uint32_t>(q.wa));
  q.k_lo = floor_div32(q.r - q.o, q.wa);
  const int32_t k_hi = floor_div32(n - 1 + q.r - q.o, q.wa);
  q.nseg = k_hi - q.k_lo + 1;
  q.cps = (q.wa + 31) >> 5;
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
template <class T, int OP, int PP>
__device__ __forceinline__ void chunk_h(const T* __restrict__ vp, T* __restrict__ rp, T cv) {
  if constexpr (OP == kOpSum) {
    T loc = vp[0];
    rp[0] = add_rn(cv, loc);
#pragma unroll
    for (int s = 1; s < 32; ++s) {
      loc = add_rn(loc, vp[-s * PP]);
      rp[-s * PP] = add_rn(cv, loc);
    }
  } else {
    T loc = cv;
#pragma unroll
    for (int s = 0; s < 32; ++s) {
      loc = fop<OP>(loc, vp[-s * PP]);
      rp[-s * PP] = loc;
    }
  }
}
// G of the chunk combined with the H already in its output slots; the segment's last sample of an
// aligned box window (aligned_end) takes (H + G) * 0.5.
template <class T, int OP, int PP>
__device__ __forceinline__ void chunk_g(const T* __restrict__ vp, T* __restrict__ rp, T cv, bool aligned_end) {
  if constexpr (OP == kOpSum) {
    T loc = vp[0];
#pragma unroll
    for (int s = 0; s < 32; ++s) {
      if (s) loc = add_rn(loc, vp[s * PP]);
      const T y = add_rn(rp[s * PP], add_rn(cv, loc));
      rp[s * PP] = (s == 31 && aligned_end) ? mul_rn(y, T(0.5)) : y;
    }
  } else {
    T loc = cv;
#pragma unroll
    for (int s = 0; s < 32; ++s) {
      loc = fop<OP>(loc, vp[s * PP]);
      rp[s * PP] = fop<OP>(rp[s * PP], loc);
    }
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
__device__ __forceinline__ void partial_h(const T* __restrict__ v, T* __restrict__ r, int32_t len, int32_t skip,
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
__device__ __forceinline__ void partial_g(const T* __restrict__ v, T* __restrict__ r, int32_t len, int32_t skip,
                                          T cv, bool aligned_end) {
  const int32_t last = len - 1;
  T loc = fold_init<T, OP>(cv, v[0]);
  if (last == 0) {
    if (skip == 0) combine_g<T, OP>(r, cv, loc, aligned_end);
    return;
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
}

// The fold tasks (segment k, chunk c) of one worker, chunk-major (u = c nseg + k, u = first,
// first + stride, ..): the workers of a warp take the same chunk of consecutive segments (wa
// samples apart, spreading their shared-memory banks). Advanced without divisions.
struct Tasks {
  int32_t k, c, dk, dc;
  __device__ __forceinline__ Tasks(int32_t first, int32_t stride, int32_t nseg)
      : k(first % nseg), c(first / nseg), dk(stride % nseg), dc(stride / nseg) {}
  __device__ __forceinline__ void next(int32_t nseg) {
    k += dk;
    c += dc;
    if (k >= nseg) {
      k -= nseg;
      ++c;
    }
  }
};

// One stage on the staged lines of this CTA: V -> R (both n x PP, line p at column p), tot: the
// chunk totals / carries [2][TS][PP] (slot k cps + c). Workers: P lanes each (lane % P = the line).
template <class T, int OP, int P>
__device__ __forceinline__ void run_stage(const T* __restrict__ V, T* __restrict__ R, T* __restrict__ tot, int32_t n,
                                          int32_t TS, const Win& q) {
  constexpr int PP = line_pitch(P);
  constexpr int slots = 32 / P;
  constexpr int workers = kWarps * slots;
  const int lane = threadIdx.x & 31;
  const int p = lane & (P - 1);
  const int worker = (threadIdx.x >> 5) * slots + lane / P;
  const int32_t e_max = n - 1 + q.r;
  const T* Vp = V + p;
  T* Rp = R + p;
  const T idn = fold_identity<T, OP>();
  if (q.cps > 1) {
    // phase 1: chunk totals; half of the workers take the line, half the reversed line
    constexpr int half = workers / 2;
    const int dir = worker >= half;
    for (Tasks t(worker - dir * half, half, q.nseg); t.c < q.cps; t.next(q.nseg)) {
      const int32_t s = q.o + (q.k_lo + t.k) * q.wa;
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
      tot[(dir * TS + t.k * q.cps + t.c) * PP + p] = total;
    }
    __syncthreads();
    // phase 2: exclusive carries per segment, in place (slot c holds the carry of chunk c >= 1)
    for (int32_t t = worker; t < 2 * q.nseg; t += workers) {
      const int dir = t >= q.nseg;
      const int32_t k = t - dir * q.nseg;
      const int32_t s = q.o + (q.k_lo + k) * q.wa;
      const int32_t e_last = min(s + q.wa - 1, e_max);
      const int32_t nch = (e_last - s) / 32 + 1;
      T* tl = tot + (dir * TS + k * q.cps) * PP + p;
      T run = tl[0];
      for (int32_t c = 1; c < nch; ++c) {
        const T next = tl[c * PP];
        tl[c * PP] = run;
        run = fop<OP>(run, next);
      }
    }
    __syncthreads();
  }
  // phase 3: H (the reversed line's G) into R at the output slots n - 1 + r - e (e >= r)
  for (Tasks t(worker, workers, q.nseg); t.c < q.cps; t.next(q.nseg)) {
    const int32_t s = q.o + (q.k_lo + t.k) * q.wa;
    const int32_t e_last = min(s + q.wa - 1, e_max);
    const int32_t c0 = s + 32 * t.c;
    if (c0 > e_last) continue;
    const int32_t c1 = min(c0 + 31, e_last);
    const T cv = t.c > 0 ? tot[(TS + t.k * q.cps + t.c) * PP + p] : idn;
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
  for (Tasks t(worker, workers, q.nseg); t.c < q.cps; t.next(q.nseg)) {
    const int32_t s = q.o + (q.k_lo + t.k) * q.wa;
    const int32_t e_al = s + q.wa - 1;
    const int32_t e_last = min(e_al, e_max);
    const int32_t c0 = s + 32 * t.c;
    if (c0 > e_last) continue;
    const int32_t c1 = min(c0 + 31, e_last);
    const T cv = t.c > 0 ? tot[(t.k * q.cps + t.c) * PP + p] : idn;
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
  unsigned long long* bytes;  // instrumentation: the pass's algorithmic bytes (nullptr: off)
};

// Thread roles of the staging and the store of P lines of n samples. Rows (the contiguous axis):
// warps take lines (kWarps / P warps per line when P < kWarps), lanes consecutive samples. Column
// panels: thread t takes line t % P and samples t / P + k kThreads / P.
template <int P>
struct LineRoles {
  static constexpr int kWpl = P >= kWarps ? 1 : kWarps / P;  // warps per line (rows)
  static constexpr int kRowStride = 32 * kWpl;                 // sample stride of a thread (rows)
  static constexpr int kColStride = kThreads / P;              // sample stride of a thread (columns)
};

template <class T, int P>
__global__ void __launch_bounds__(kThreads, 5) cube_pass(Geom g, PassArgs<T> a) {
  constexpr int PP = line_pitch(P);
  using Roles = LineRoles<P>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int64_t b = blockIdx.y;
  const int axis = a.axis;
  // (a kernel parameter indexed by a runtime value would be copied to local memory)
  const int32_t n = geom_n(g, axis);
  const int64_t axis_stride = geom_stride(g, axis);
  const int32_t n_last = geom_n(g, g.dim - 1);
  const bool contig = axis == g.dim - 1;
  const int32_t TS = tot_slots(n);
  T* V = reinterpret_cast<T*>(smem_raw);
  T* R = V + static_cast<int64_t>(n) * PP;
  T* tot = R + static_cast<int64_t>(n) * PP;
  __shared__ int64_t base_s[32];
  __shared__ int32_t ok_s[32];
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
      // 32-bit divisions (an element holds fewer than 2^31 samples)
      const uint32_t inner = static_cast<uint32_t>(axis_stride);
      const uint32_t gpo = (inner + P - 1) / P;
      const uint32_t o = static_cast<uint32_t>(grp) / gpo;
      const uint32_t c = (static_cast<uint32_t>(grp) - o * gpo) * P + p;
      ok = c < inner && (c % static_cast<uint32_t>(g.pitch)) < static_cast<uint32_t>(n_last);
      base = static_cast<int64_t>(o) * n * inner + c;
    }
    base_s[p] = base;
    ok_s[p] = ok ? 1 : 0;
  }
  const int64_t step = contig ? 1 : axis_stride;
  __syncthreads();
  int32_t valid = 0;
  if (a.bytes && threadIdx.x == 0) {
    for (int p = 0; p < P; ++p) valid += ok_s[p];
  }
  unsigned long long acct = 0;
  const int64_t eoff = b * g.field;
  const int nf = a.op == static_cast<int>(CubeOp::kMaxMin) ? 2 : 1;
  const bool box = a.op == static_cast<int>(CubeOp::kBox);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this thread's line and first sample in the staging and the store
  const int my_p = contig ? warp / Roles::kWpl : (threadIdx.x & (P - 1));
  const int32_t my_i0 = contig ? lane + 32 * (warp % Roles::kWpl) : static_cast<int32_t>(threadIdx.x / P);
  const int32_t my_di = contig ? Roles::kRowStride : Roles::kColStride;
  const int my_dp = contig ? kWarps / Roles::kWpl : P;  // line stride of this thread (rows: P > kWarps)
  const int32_t nw = contig ? static_cast<int32_t>(g.pitch) : n;  // samples written per line
  const int32_t j_begin = a.rung_loop ? 0 : static_cast<int32_t>(blockIdx.z);
  const int32_t j_end = a.rung_loop ? a.rungs : j_begin + 1;
  bool staged = false;  // V holds the staged shared input (first pass with a rung loop)
  for (int32_t j = j_begin; j < j_end; ++j) {
    const int32_t w = a.win[static_cast<int64_t>(j) * g.batch + b];
    if (w < 1) continue;
    const Win q = make_win(n, w);
    double fac = 1.0;
    if (box && a.last) {
      double prod = 1.0;
#pragma unroll
      for (int ax = 0; ax < kMaxDim; ++ax) {
        if (ax < g.dim) prod *= static_cast<double>(2 * min((w - 1) / 2, g.n[ax] - 1) + 1);
      }
      fac = static_cast<double>(static_cast<T>(1.0 / prod));
    }
    for (int f = 0; f < nf; ++f) {
      // stage field f (the input of this rung) as values (box) or order keys (max / min)
      const bool shared_in = a.in_stride == 0 && (f == 0 || a.in1 == nullptr);
      if (!(staged && shared_in)) {
        const T* src = (f == 0 || a.in1 == nullptr) ? a.in0 : a.in1;
        if (src) src += static_cast<int64_t>(j) * a.in_stride + eoff;
        const uint8_t* bits = a.bits ? a.bits + eoff : nullptr;
        for (int p = my_p; p < P; p += my_dp) {
          if (!ok_s[p]) continue;
          const int64_t base = base_s[p];
          // kStageLoads independent loads in flight per thread before their shared-memory stores
          for (int32_t i0 = my_i0; i0 < n; i0 += kStageLoads * my_di) {
            T v[kStageLoads];
#pragma unroll
            for (int u = 0; u < kStageLoads; ++u) {
              const int32_t i = i0 + u * my_di;
              if (i < n) {
                const int64_t at = base + static_cast<int64_t>(i) * step;
                v[u] = bits ? (((bits[at] >> a.bit) & 1u) ? T(1) : T(0)) : src[at];
              }
            }
#pragma unroll
            for (int u = 0; u < kStageLoads; ++u) {
              const int32_t i = i0 + u * my_di;
              if (i < n) V[i * PP + p] = box ? v[u] : okey(v[u]);
            }
          }
        }
        __syncthreads();
        staged = shared_in;
        acct += static_cast<unsigned long long>(valid) * n * (bits ? 1u : sizeof(T));
      }
      const bool is_min = a.op == static_cast<int>(CubeOp::kMin) || (a.op == static_cast<int>(CubeOp::kMaxMin) && f == 1);
      if (box) run_stage<T, kOpSum, P>(V, R, tot, n, TS, q);
      else if (is_min) run_stage<T, kOpMinK, P>(V, R, tot, n, TS, q);
      else run_stage<T, kOpMaxK, P>(V, R, tot, n, TS, q);
      // store (pads of the contiguous axis written as 0)
      T* dst = (f == 0 ? a.out0 : a.out1) + static_cast<int64_t>(j) * a.out_stride + eoff;
      acct += static_cast<unsigned long long>(valid) * n * sizeof(T);
      const bool detsq = box && a.last && a.epi == static_cast<int>(BoxEpi::kDetSq);
      const T* aux = detsq ? a.aux + eoff : nullptr;
      for (int p = my_p; p < P; p += my_dp) {
        if (!ok_s[p]) continue;
        const int64_t base = base_s[p];
        for (int32_t i = my_i0; i < nw; i += my_di) {
          const int64_t at = base + static_cast<int64_t>(i) * step;
          if (i >= n) {
            dst[at] = T(0);
            continue;
          }
          T y = R[i * PP + p];
          if (!box) {
            y = okey(y);
          } else if (a.last) {
            y = mul_rn(y, static_cast<T>(fac));
            if (detsq) {
              const T d = sub_rn(aux[at], y);
              y = mul_rn(d, d);
            }
          }
          dst[at] = y;
        }
      }
      __syncthreads();  // the next stage rewrites R and tot
    }
  }
  if (a.bytes && threadIdx.x == 0 && acct) atomicAdd(a.bytes, acct);
}

size_t smem_bytes(int32_t n, int P, size_t es) {
  return (static_cast<size_t>(2) * n + static_cast<size_t>(2) * tot_slots(n)) * static_cast<size_t>(line_pitch(P)) * es;
}

template <class T>
void allow_smem(int bytes) {
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  EDAB_CUDA(cudaFuncSetAttribute(cube_pass<T, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

struct DevFacts {
  int sms = 148;
  size_t smem = 227 * 1024;
};
DevFacts dev_facts() {
  static std::mutex mu;
  static DevFacts f[64];
  static bool have[64] = {};
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (!have[dev]) {
    int optin = 0, sms = 0;
    EDAB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    EDAB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    f[dev].sms = sms;
    f[dev].smem = static_cast<size_t>(optin) - 1024;  // the kernel's static shared memory
    allow_smem<float>(static_cast<int>(f[dev].smem));
    allow_smem<double>(static_cast<int>(f[dev].smem));
    have[dev] = true;
  }
  return f[dev];
}

// Lines per CTA (a power of two up to 32): 8 lines for column panels (whole sectors, and shared
// memory for several CTAs per SM), rows up to 8 per CTA; fewer where the shared memory or the
// element's rows run out.
template <class T>
int lines_per_cta(const Geom& g, int axis, size_t cap) {
  const int32_t n = g.n[axis];
  int P = 8;
  if (axis == g.dim - 1) {
    while (P > 1 && P / 2 >= g.rows) P /= 2;
  } else {
    while (P > 1 && P / 2 >= g.stride[axis]) P /= 2;
  }
  while (P > 1 && smem_bytes(n, P, sizeof(T)) > cap / 2) P /= 2;
  if (smem_bytes(n, P, sizeof(T)) > cap) {
    throw std::invalid_argument("edab: an axis of " + std::to_string(n) + " samples exceeds the shared-memory line capacity");
  }
  return P;
}

template <class T>
void launch_pass(cudaStream_t s, const Geom& g, PassArgs<T> a) {
  const DevFacts f = dev_facts();
  const int P = lines_per_cta<T>(g, a.axis, f.smem);
  int64_t groups;
  if (a.axis == g.dim - 1) {
    groups = (g.rows + P - 1) / P;
  } else {
    int64_t outer = 1;
    for (int ax = 0; ax < a.axis; ++ax) outer *= g.n[ax];
    groups = outer * ((g.stride[a.axis] + P - 1) / P);
  }
  if (groups > 0x7fffffffLL || g.batch > 65535) throw std::invalid_argument("edab: cube launch too large");
  const dim3 grid(static_cast<unsigned>(groups), static_cast<unsigned>(g.batch), a.rung_loop ? 1u : static_cast<unsigned>(a.rungs));
  const size_t smem = smem_bytes(g.n[a.axis], P, sizeof(T));
  a.bytes = cube_bytes_counter();
  profile_cube_launch(s, true);
  switch (P) {
    case 1: cube_pass<T, 1><<<grid, kThreads, smem, s>>>(g, a); break;
    case 2: cube_pass<T, 2><<<grid, kThreads, smem, s>>>(g, a); break;
    case 4: cube_pass<T, 4><<<grid, kThreads, smem, s>>>(g, a); break;
    case 8: cube_pass<T, 8><<<grid, kThreads, smem, s>>>(g, a); break;
    case 16: cube_pass<T, 16><<<grid, kThreads, smem, s>>>(g, a); break;
    default: cube_pass<T, 32><<<grid, kThreads, smem, s>>>(g, a); break;
  }
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
