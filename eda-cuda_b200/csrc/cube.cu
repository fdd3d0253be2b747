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
// combined with them; reflection is evaluated only in the chunks that cross a line end. The first
// pass of a cube stages its input once and runs every rung of the ladder on it (the operators'
// rung group); later passes run one rung per CTA.
#include "engine.cuh"

#include <algorithm>
#include <mutex>

namespace edab {
namespace {

constexpr int kOpMaxK = 0, kOpMinK = 1, kOpSum = 2;
constexpr int kWarps = kThreads / 32;

__host__ __device__ inline int32_t tot_slots(int32_t n) { return n / 8 + 24; }
// Words per staged sample row: P lines plus one (odd, so a transposed row staging of 32
// consecutive samples hits 32 distinct banks); one line is stored contiguously.
__host__ __device__ inline int32_t line_pitch(int P) { return P == 1 ? 1 : P + 1; }

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

struct Win {
  int32_t r, wa, o, k_lo, nseg, cps;
};
__device__ __forceinline__ Win make_win(int32_t n, int32_t w) {
  Win q;
  const int32_t half = (w - 1) / 2;
  q.r = min(half, n - 1);
  q.wa = 2 * q.r + 1;
  q.o = static_cast<int32_t>((static_cast<int64_t>(n) * ((q.wa + 1) / 2)) % q.wa);
  q.k_lo = static_cast<int32_t>(floor_div(static_cast<int64_t>(q.r) - q.o, q.wa));
  const int32_t k_hi = static_cast<int32_t>(floor_div(static_cast<int64_t>(n) - 1 + q.r - q.o, q.wa));
  q.nseg = k_hi - q.k_lo + 1;
  q.cps = (q.wa + 31) >> 5;
  return q;
}

// Line-sample index of extended position e in direction dir (1: the reversed line).
__device__ __forceinline__ int32_t ext_index(int32_t e, int32_t n, int dir) {
  const int32_t i = reflect_index(e, n);
  return dir ? n - 1 - i : i;
}

// The fold of a chunk [c0, c1] of direction dir into acc (first sample stored as is), calling
// f(e, local) after every sample. Interior chunks index linearly; boundary chunks reflect.
template <class T, int OP, class F>
__device__ __forceinline__ T fold_chunk(const T* __restrict__ V, int32_t PP, int32_t n, int32_t c0, int32_t c1,
                                        int dir, F&& f) {
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

// One stage on the staged lines of this CTA: V -> R (both n x PP, line p at column p), tot: the
// chunk totals / carries [2][TS][PP]. Workers: P lanes each (lane % P = the line).
template <class T, int OP>
__device__ void run_stage(const T* __restrict__ V, T* __restrict__ R, T* __restrict__ tot, int P, int32_t PP,
                          int32_t n, int32_t TS, const Win& q) {
  const int lane = threadIdx.x & 31;
  const int slots = 32 / P;
  const int p = lane % P;
  const bool active_lane = lane < slots * P;
  const int worker = (threadIdx.x >> 5) * slots + lane / P;
  const int workers = kWarps * slots;
  const int32_t per_dir = q.nseg * q.cps;
  const int32_t e_max = n - 1 + q.r;
  const T* Vp = V + p;
  T* Rp = R + p;
  if (q.cps > 1) {
    // phase 1: chunk totals of both directions
    for (int32_t t = worker; active_lane && t < 2 * per_dir; t += workers) {
      const int dir = t >= per_dir;
      const int32_t u = t - dir * per_dir;
      const int32_t k = u / q.cps, c = u - k * q.cps;
      const int32_t s = q.o + (q.k_lo + k) * q.wa;
      const int32_t e_last = min(s + q.wa - 1, e_max);
      const int32_t c0 = s + 32 * c;
      if (c0 > e_last) continue;
      const T total = fold_chunk<T, OP>(Vp, PP, n, c0, min(c0 + 31, e_last), dir, [](int32_t, T) {});
      tot[(dir * TS + u) * PP + p] = total;
    }
    __syncthreads();
    // phase 2: exclusive carries per segment, in place (slot c holds the carry of chunk c >= 1)
    for (int32_t t = worker; active_lane && t < 2 * q.nseg; t += workers) {
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
  // phase 3: H (the reversed line's G) into R at the output slots
  for (int32_t u = worker; active_lane && u < per_dir; u += workers) {
    const int32_t k = u / q.cps, c = u - k * q.cps;
    const int32_t s = q.o + (q.k_lo + k) * q.wa;
    const int32_t e_last = min(s + q.wa - 1, e_max);
    const int32_t c0 = s + 32 * c;
    if (c0 > e_last) continue;
    const bool carry = c > 0;
    const T cv = carry ? tot[(TS + u) * PP + p] : T(0);
    fold_chunk<T, OP>(Vp, PP, n, c0, min(c0 + 31, e_last), 1, [&](int32_t e, T loc) {
      if (e >= q.r) Rp[(n - 1 + q.r - e) * PP] = carry ? fop<OP>(cv, loc) : loc;
    });
  }
  __syncthreads();
  // phase 4: G combined with H in place: y(x) = op(H(x - r), G(x + r))
  for (int32_t u = worker; active_lane && u < per_dir; u += workers) {
    const int32_t k = u / q.cps, c = u - k * q.cps;
    const int32_t s = q.o + (q.k_lo + k) * q.wa;
    const int32_t e_last = min(s + q.wa - 1, e_max);
    const int32_t c0 = s + 32 * c;
    if (c0 > e_last) continue;
    const bool carry = c > 0;
    const T cv = carry ? tot[u * PP + p] : T(0);
    const int32_t e_al = s + q.wa - 1;
    fold_chunk<T, OP>(Vp, PP, n, c0, min(c0 + 31, e_last), 0, [&](int32_t e, T loc) {
      if (e < q.r) return;
      const T g = carry ? fop<OP>(cv, loc) : loc;
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
  int32_t P;              // lines per CTA (1, 2, 4, 8, 16 or 32)
  int32_t rung_loop;      // 1: the CTA loops over the rungs (shared input); else blockIdx.z is the rung
  unsigned long long* bytes;  // instrumentation: the pass's algorithmic bytes (nullptr: off)
};

template <class T>
__global__ void __launch_bounds__(kThreads) cube_pass(Geom g, PassArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int64_t b = blockIdx.y;
  const int axis = a.axis;
  const int32_t n = g.n[axis];
  const bool contig = axis == g.dim - 1;
  const int P = a.P;
  const int32_t PP = line_pitch(P);
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
      const int64_t inner = g.stride[axis];
      const int64_t gpo = (inner + P - 1) / P;
      const int64_t o = grp / gpo;
      const int64_t c = (grp - o * gpo) * P + p;
      ok = c < inner && (c % g.pitch) < g.n[g.dim - 1];
      base = o * static_cast<int64_t>(n) * inner + c;
    }
    base_s[p] = base;
    ok_s[p] = ok ? 1 : 0;
  }
  const int64_t step = contig ? 1 : g.stride[axis];
  __syncthreads();
  int32_t valid = 0;
  if (a.bytes && threadIdx.x == 0) {
    for (int p = 0; p < P; ++p) valid += ok_s[p];
  }
  unsigned long long acct = 0;
  const int64_t eoff = b * g.field;
  const int nf = a.op == static_cast<int>(CubeOp::kMaxMin) ? 2 : 1;
  const bool box = a.op == static_cast<int>(CubeOp::kBox);
  const int32_t total = P * n;
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
      for (int ax = 0; ax < g.dim; ++ax) prod *= static_cast<double>(2 * min((w - 1) / 2, g.n[ax] - 1) + 1);
      fac = static_cast<double>(static_cast<T>(1.0 / prod));
    }
    for (int f = 0; f < nf; ++f) {
      // stage field f (the input of this rung) as values (box) or order keys (max / min)
      const bool shared_in = a.in_stride == 0 && (f == 0 || a.in1 == nullptr);
      if (!(staged && shared_in)) {
        const T* src = (f == 0 || a.in1 == nullptr) ? a.in0 : a.in1;
        if (src) src += static_cast<int64_t>(j) * a.in_stride + eoff;
        const uint8_t* bits = a.bits ? a.bits + eoff : nullptr;
        for (int32_t t = threadIdx.x; t < total; t += blockDim.x) {
          int p, i;
          if (contig) {
            p = t / n;
            i = t - p * n;
          } else {
            i = t / P;
            p = t - i * P;
          }
          if (!ok_s[p]) continue;
          const int64_t at = base_s[p] + static_cast<int64_t>(i) * step;
          T v;
          if (bits) v = ((bits[at] >> a.bit) & 1u) ? T(1) : T(0);
          else v = src[at];
          V[i * PP + p] = box ? v : okey(v);
        }
        __syncthreads();
        staged = shared_in;
        acct += static_cast<unsigned long long>(valid) * n * (bits ? 1u : sizeof(T));
      }
      const bool is_min = a.op == static_cast<int>(CubeOp::kMin) || (a.op == static_cast<int>(CubeOp::kMaxMin) && f == 1);
      if (box) run_stage<T, kOpSum>(V, R, tot, P, PP, n, TS, q);
      else if (is_min) run_stage<T, kOpMinK>(V, R, tot, P, PP, n, TS, q);
      else run_stage<T, kOpMaxK>(V, R, tot, P, PP, n, TS, q);
      // store (pads of the contiguous axis written as 0)
      T* dst = (f == 0 ? a.out0 : a.out1) + static_cast<int64_t>(j) * a.out_stride + eoff;
      acct += static_cast<unsigned long long>(valid) * n * sizeof(T);
      const int32_t nw = contig ? static_cast<int32_t>(g.pitch) : n;
      const int32_t tw = P * nw;
      for (int32_t t = threadIdx.x; t < tw; t += blockDim.x) {
        int p, i;
        if (contig) {
          p = t / nw;
          i = t - p * nw;
        } else {
          i = t / P;
          p = t - i * P;
        }
        if (!ok_s[p]) continue;
        const int64_t at = base_s[p] + static_cast<int64_t>(i) * step;
        if (i >= n) {
          dst[at] = T(0);
          continue;
        }
        T y = R[i * PP + p];
        if (!box) {
          y = okey(y);
        } else if (a.last) {
          y = mul_rn(y, static_cast<T>(fac));
          if (a.epi == static_cast<int>(BoxEpi::kDetSq)) {
            const T d = sub_rn(a.aux[eoff + at], y);
            y = mul_rn(d, d);
          }
        }
        dst[at] = y;
      }
      __syncthreads();  // the next stage rewrites R and tot
    }
  }
  if (a.bytes && threadIdx.x == 0 && acct) atomicAdd(a.bytes, acct);
}

size_t smem_bytes(int32_t n, int P, size_t es) {
  return (static_cast<size_t>(2) * n + static_cast<size_t>(2) * tot_slots(n)) * static_cast<size_t>(line_pitch(P)) * es;
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
    EDAB_CUDA(cudaFuncSetAttribute(cube_pass<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(f[dev].smem)));
    EDAB_CUDA(cudaFuncSetAttribute(cube_pass<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(f[dev].smem)));
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
  a.P = P;
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
  a.bytes = cube_bytes_counter();
  profile_cube_launch(s, true);
  cube_pass<T><<<grid, kThreads, smem_bytes(g.n[a.axis], P, sizeof(T)), s>>>(g, a);
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
