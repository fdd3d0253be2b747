// SPDX-License-Identifier: Apache-2.0
// The decomposition of one call on the B200 engine: the per-element control (the window rule,
// G2's rung machine, the growth floor, G3), the threshold field, the raw window, the scale field,
// the element with its ladder and weights, the operators Dil_B / Ero_B / Avg_B, the sifts with G1
// and the sup-norm guard, the commit, and the host driver that sequences them for a chunk of
// elements in lockstep. Semantics of eda-cuda's method (cpp/src/method/driver.cpp:393-700,
// mode.cu, sift.cu, element.cu, element_op.cuh, stats_fields.cu, stats_scale.cu,
// stats_rungs.cu); every kernel is this engine's own.
//
// Host synchronisations per mode: S1 after the window passes (who is active; G2's candidate
// rungs, which the reference computes with the host's pow), S4 after the element build (the
// ladders, from the host's log and pow, as the reference), S5 after the commit (whether another
// mode runs). G2's rung loop runs on device-resident machines without a synchronisation per rung.
#include "engine.cuh"
#include "orient.cuh"
#include "driver.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <set>
#include <vector>

namespace edab {

void cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  const char* base = std::strrchr(file, '/');
  throw CudaError(std::string("eda: CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " +
                      what + " at " + (base ? base + 1 : file) + ":" + std::to_string(line),
                  static_cast<int>(e));
}

Geom make_geom(int dim, int64_t batch, const int64_t* n) {
  if (dim < 1 || dim > kMaxDim) throw std::invalid_argument("eda: the number of spatial axes must be 1, 2 or 3");
  Geom g{};
  g.dim = dim;
  g.batch = batch;
  g.n_max = 1;
  for (int a = 0; a < kMaxDim; ++a) g.n[a] = 1;
  int64_t count = 1;
  for (int a = 0; a < dim; ++a) {
    if (n[a] < 1 || n[a] > (int64_t{1} << 31)) throw std::invalid_argument("eda: a spatial extent is out of range");
    g.n[a] = static_cast<int32_t>(n[a]);
    g.n_max = std::max(g.n_max, g.n[a]);
    count *= n[a];
  }
  g.count = count;
  g.pitch = (static_cast<int64_t>(g.n[dim - 1]) + 31) / 32 * 32;
  for (int a = 0; a < kMaxDim; ++a) g.stride[a] = 1;
  if (dim >= 2) g.stride[dim - 2] = g.pitch;
  for (int a = dim - 3; a >= 0; --a) g.stride[a] = static_cast<int64_t>(g.n[a + 1]) * g.stride[a + 1];
  g.field = dim == 1 ? g.pitch : static_cast<int64_t>(g.n[0]) * g.stride[0];
  if (g.field > (int64_t{1} << 31)) throw std::invalid_argument("eda: an element's padded field exceeds 2^31 samples");
  g.rows = g.field / g.pitch;
  g.n_last = g.n[dim - 1];
  g.pitch_inv = ~uint64_t{0} / static_cast<uint64_t>(g.pitch) + 1;
  g.field_inv = ~uint64_t{0} / static_cast<uint64_t>(g.field) + 1;
  // i < batch field <= 2^64 / field keeps umulhi(i, field_inv) exact
  const long double f = static_cast<long double>(g.field);
  g.field_fast = static_cast<long double>(batch) * f * f <= 18446744073709551616.0L ? 1 : 0;
  return g;
}

Ctl make_ctl(const Geom& g, bool f32, int32_t sifts, double tau, int32_t max_imf, bool check_finite, int32_t rows_cap) {
  Ctl c;
  std::memset(&c, 0, sizeof c);
  c.n_max = g.n_max;
  c.count = g.count;
  c.sifts = sifts;
  c.u = 2;
  c.s = 1;
  c.sig_passes = 2;
  c.growth_from = 2;
  c.anorm_smooth = 1;
  c.kappa = 1.0;
  c.beta = 2.0;
  c.c_lo = 1.5;
  c.c_hi = 2.0;
  c.reset = 2.0;
  c.q = 4.0;
  c.span = 1.0;
  c.growth = 2.0;
  c.sig_theta = 0.3;
  c.sig_rho = 2.0;
  c.sig_noise = 1.0;
  c.absent = 3.0;
  c.absent_jump = 2.0;
  c.absent_reach = 1.0;
  c.absent_lo = 1.2;
  c.t0 = 0.2;
  c.t1 = 0.5;
  c.anorm_floor = 0.1;
  c.ramp_k0 = 0.3;
  c.ramp_k1 = 0.6;
  c.fine_beta = 2.0;
  c.fine_theta = 1.0;
  c.fine_jump = 2.0;
  c.fine_lo = 1.5;
  c.fine_pop = 0.25;
  c.fine_core = 2.0;
  c.split = 1.0;
  c.tiny = f32 ? static_cast<double>(FLT_MIN) : 1e-300;
  c.tau = f32 ? static_cast<double>(static_cast<float>(tau)) : tau;
  c.log_absent = std::log(c.absent);
  {
    volatile double two = 2.0;
    const double l2 = std::log(static_cast<double>(two));
    const double s = l2 / (2.0 * std::sqrt(2.0 * l2));
    c.two_sigma2 = 2.0 * (s * s);
  }
  c.sqrt2 = std::sqrt(2.0);
  c.max_imf = max_imf;
  c.check_finite = check_finite ? 1 : 0;
  c.rows_cap = rows_cap;
  return c;
}

int32_t mode_bound(const Ctl& c) {
  int32_t w_prev = 1, count = 0;
  for (int32_t k = 0;; ++k) {
    int64_t w = std::max(3, w_prev + 2);
    if (c.growth > 1.0 && k >= c.growth_from) w = std::max<int64_t>(w, odd_window(c.growth * static_cast<double>(w_prev)));
    if (w > c.n_max) break;
    ++count;
    w_prev = static_cast<int32_t>(w);
  }
  return count;
}

// G2's candidate rungs (host pow, as the reference: cpp/src/method/driver.cpp:59-71).
std::vector<int32_t> g2_candidate_rungs(int32_t w, int32_t w_prev, double jump) {
  const int32_t s0 = std::max(3, w_prev + 2);
  std::vector<int32_t> out;
  for (int32_t j = 0;; ++j) {
    const int32_t s = odd_window(static_cast<double>(s0) * std::pow(kRungRatio, static_cast<double>(j)));
    if (static_cast<double>(s) * jump > static_cast<double>(w)) break;
    if (out.empty() || s != out.back()) out.push_back(s);
    if (static_cast<int32_t>(out.size()) > kMaxG2Rungs) throw std::length_error("eda: too many G2 rungs");
  }
  return out;
}

// The ladder (host log and pow, as the reference: cpp/src/method/element.cu:343-370).
std::vector<int32_t> rung_ladder(double d_min, double d_max, int32_t w, int32_t n_max) {
  if (!(std::isfinite(d_min) && std::isfinite(d_max)) || w < 1 || n_max < 1) {
    throw std::invalid_argument("eda: rung_ladder: d_min, d_max must be finite, w and n_max >= 1");
  }
  volatile double qv = kRungRatio;
  const double q = qv;
  const double lq = std::log(q);
  const double wd = static_cast<double>(w);
  const double jl = std::floor(std::log((d_min > 1.0 ? d_min : 1.0) / wd) / lq + 1e-9);
  const double jh = std::ceil(std::log((d_max > 1.0 ? d_max : 1.0) / wd) / lq - 1e-9);
  if (!(jh - jl <= 4096.0)) throw std::length_error("eda: rung_ladder: the ladder spans too many rungs");
  const int64_t cap = 2 * static_cast<int64_t>(n_max) + 1;
  std::set<int64_t> sides;
  for (int64_t j = static_cast<int64_t>(jl); j <= static_cast<int64_t>(jh); ++j) {
    const double v = wd * std::pow(q, static_cast<double>(j));
    const int64_t side = v >= static_cast<double>(cap) + 1.0 ? cap : std::min<int64_t>(odd_window(v), cap);
    sides.insert(side);
  }
  if (sides.size() > static_cast<size_t>(kMaxRungs)) throw std::length_error("eda: rung_ladder: too many rungs");
  return std::vector<int32_t>(sides.begin(), sides.end());
}

namespace {

// Window slots, [kSlots * B] int32: slot k of element b at k * B + b (0: the element is skipped).
enum Slot : int32_t {
  kWd = 0, kWl, kW, kNear, kFloor, kG2b, kG2core, kG2rq, kG3c, kG3r, kSlots
};
// Run masks, [kMasks * B] int32.
enum Mask : int32_t { kOn = 0, kOnG2, kOnFloor, kOnFine, kSrung, kOnG3, kMasks };

__device__ __forceinline__ void tau_windows(const Ctl& c, int32_t w, int32_t* wd, int32_t* wl) {
  const double wv = static_cast<double>(w);
  *wd = odd_window(__dmul_rn(c.sig_rho, wv));
  const double m = c.beta >= c.sig_rho ? c.beta : c.sig_rho;
  *wl = odd_window(__dmul_rn(m, wv));
}

__device__ __forceinline__ void leave(Elem& e, int32_t* win, int32_t* mask, int64_t B, int64_t b, int32_t status) {
  e.status = status;
  for (int k = 0; k < kSlots; ++k) win[k * B + b] = 0;
  mask[kOn * B + b] = 0;
  mask[kOnG2 * B + b] = 0;
  mask[kOnFloor * B + b] = 0;
  mask[kOnFine * B + b] = 0;
  mask[kOnG3 * B + b] = 0;
}
__device__ __forceinline__ void fail2(Elem& e, int32_t* win, int32_t* mask, int64_t B, int64_t b) {
  leave(e, win, mask, B, b, kError);
  e.error = kErrNonFiniteResult;
}

template <class T>
__device__ __forceinline__ T times_pow2(T v, int32_t k) {
  if constexpr (std::is_same_v<T, float>) return static_cast<float>(ldexp(static_cast<double>(v), k));
  else return ldexp(v, k);
}

template <class T>
__device__ __forceinline__ double tie_tol(double tau, double amax) {
  return static_cast<double>(mul_rn(static_cast<T>(tau), static_cast<T>(amax)));
}

// d, e of a voxel (cpp/src/method/element.cuh:238-254): the cube side shrinks with the coherence c
// and the segment half length takes up what the side gave away.
template <class T>
__device__ __forceinline__ void element_de(T L, T c, T q, T span_m1, T* d, T* e) {
  const T one = T(1);
  const T f = add_rn(sub_rn(one, c), div_rn(c, q));
  *d = mul_rn(L, f);
  const T len = mul_rn(L, add_rn(one, mul_rn(span_m1, c)));
  const T diff = sub_rn(len, *d);
  *e = mul_rn(T(0.5), diff > T(0) ? diff : T(0));
}

// The element's extent (cpp/src/method/element.cu:182-226): per voxel d and e, the segment
// offset o = e n (D >= 2), and the element's smallest and largest d (as double bits: d >= 0).
// The voxel keeps d in the weight field t and whether its segment reaches past a quarter sample
// (e > 1/4, the rungs that need segment points) in the rung field lo, so the rung pass that
// follows reads 5 bytes per voxel instead of recomputing d and e from L and c. Extremes: a warp
// folds its lanes' by shuffles, one atomic per warp.
template <class T, int D>
__global__ void __launch_bounds__(kThreads) element_extent(Geom g, Ctl c, const T* __restrict__ L,
                                                          const T* __restrict__ coh, const T* n0, const T* n1,
                                                          const T* n2, T* o0, T* o1, T* o2, T* d_out,
                                                          uint8_t* far_out, Elem* el, const int32_t* run) {
  const int64_t b = blockIdx.y;
  if (!run[b]) return;
  const T q = static_cast<T>(c.q), sm1 = static_cast<T>(c.span - 1.0);
  uint64_t lo_bits = ~0ULL, hi_bits = 0ULL;
  const int32_t nl = elem_len(g, b);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field; v += step) {
    if (pitch_col(g, v) >= nl) continue;
    const int64_t i = b * g.field + v;
    T d, e;
    element_de<T>(L[i], D == 1 ? T(0) : coh[i], q, sm1, &d, &e);
    if constexpr (D >= 2) {
      o0[i] = mul_rn(e, n0[i]);
      o1[i] = mul_rn(e, n1[i]);
      if constexpr (D == 3) o2[i] = mul_rn(e, n2[i]);
    }
    d_out[i] = d;
    far_out[i] = e > T(0.25) ? 1 : 0;
    const uint64_t bits = static_cast<uint64_t>(__double_as_longlong(static_cast<double>(d)));
    lo_bits = bits < lo_bits ? bits : lo_bits;
    hi_bits = bits > hi_bits ? bits : hi_bits;
  }
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    const uint64_t a = __shfl_xor_sync(0xffffffffu, lo_bits, m), z = __shfl_xor_sync(0xffffffffu, hi_bits, m);
    lo_bits = a < lo_bits ? a : lo_bits;
    hi_bits = z > hi_bits ? z : hi_bits;
  }
  if ((threadIdx.x & 31) == 0 && hi_bits >= lo_bits) {  // the warp saw a voxel
    atomicMin(reinterpret_cast<unsigned long long*>(&el[b].d_min_bits), static_cast<unsigned long long>(lo_bits));
    atomicMax(reinterpret_cast<unsigned long long*>(&el[b].d_max_bits), static_cast<unsigned long long>(hi_bits));
  }
}

// The voxel's place on the element's ladder (cpp/src/method/element.cu:228-292): with the ladder's
// logs lw_0 < .. < lw_{K-1}, the bracket j of log(clamp(d, w_0, w_{K-1})) (the last rung whose log
// is at most it, kept inside 0 .. K - 2, found by bisection) and the hat weight t of rung j + 1
// (rung j weighs 1 - t). The rung masks: rungs some voxel weighs (used) and those of voxels whose
// segment reaches past a quarter sample (pts); a warp ORs its lanes', one atomic per warp. Reads d
// from t and the reach bit from lo (element_extent), then overwrites both.
template <class T>
__global__ void __launch_bounds__(kThreads) element_rungs(Geom g, uint8_t* lo, T* t, Elem* el, const int32_t* run) {
  __shared__ double lw[kMaxRungs];
  const int64_t b = blockIdx.y;
  if (!run[b]) return;
  const int K = el[b].n_rungs;
  if (threadIdx.x < kMaxRungs) lw[threadIdx.x] = static_cast<int>(threadIdx.x) < K ? el[b].rung_lw[threadIdx.x] : 0.0;
  __syncthreads();
  const double w_first = static_cast<double>(el[b].rung_w[0]);
  const double w_last = static_cast<double>(el[b].rung_w[K > 0 ? K - 1 : 0]);
  unsigned used = 0u, pts = 0u;
  const int32_t nl = elem_len(g, b);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field; v += step) {
    if (pitch_col(g, v) >= nl) continue;
    const int64_t i = b * g.field + v;
    const bool far = lo[i] != 0;
    int j = 0;
    T w = T(0);
    if (K > 1) {
      const double x = log(fmin(fmax(static_cast<double>(t[i]), w_first), w_last));
      int lo_j = 0, hi_j = K;  // lw[lo_j - 1] <= x < lw[hi_j]
      while (lo_j < hi_j) {
        const int mid = (lo_j + hi_j) >> 1;
        if (lw[mid] <= x) lo_j = mid + 1;
        else hi_j = mid;
      }
      j = min(max(lo_j - 1, 0), K - 2);
      w = static_cast<T>(__ddiv_rn(__dsub_rn(x, lw[j]), __dsub_rn(lw[j + 1], lw[j])));
    }
    lo[i] = static_cast<uint8_t>(j);
    t[i] = w;
    const unsigned mine = (sub_rn(T(1), w) > T(0) ? 1u << j : 0u) | (w > T(0) ? 1u << (j + 1) : 0u);
    used |= mine;
    if (far) pts |= mine;
  }
  used = __reduce_or_sync(0xffffffffu, used);
  pts = __reduce_or_sync(0xffffffffu, pts);
  if ((threadIdx.x & 31) == 0) {
    if (used) atomicOr(&el[b].rung_used, used);
    if (pts) atomicOr(&el[b].rung_pts, pts);
  }
}

// The gather of the operators (cpp/src/method/element_op.cuh:38-154): a voxel's rung lo with
// weight 1 - t and rung lo + 1 with weight t, each read at x and, where the rung carries the
// segment points (D >= 2), at x +- (i / 2) o by D-linear interpolation of the reflected periodic
// extension. OP 0: max (Dil), 2: max and min (Dil, Ero), 3: box (Avg). The rung cubes of every rung
// lie in rung0 (rung1: the min cubes) at j * B * field.
// Segment point q of a voxel (q = 0..3: x + (1/2) o, x - (1/2) o, x + o, x - o): per axis the
// offsets (in the element, reflected) of the two interpolation neighbours and their weights.
// The gathers' launch shape: CTAs of 256 threads per SM (the register bound) and how many of a
// voxel's four segment points are read together (more loads in flight, more registers).
#ifndef EDAB_GATHER_CTAS
#define EDAB_GATHER_CTAS 6
#endif
#ifndef EDAB_GATHER_UNROLL
#define EDAB_GATHER_UNROLL 1
#endif
constexpr int kGatherUnroll = EDAB_GATHER_UNROLL;
template <class T, int D>
struct SegPoint {
  int32_t off0[D], off1[D];
  T w0[D], w1[D];
};
// reflect_any for 32-bit indices (|i| < 2^30, n <= 8192)
__device__ __forceinline__ int32_t reflect32(int32_t i, int32_t n) {
  if (i >= 0 && i < n) return i;
  if (i < 0 && i >= -n) return -i - 1;
  if (i >= n && i < 2 * n) return 2 * n - 1 - i;
  int32_t m = i % (2 * n);
  if (m < 0) m += 2 * n;
  return m < n ? m : 2 * n - 1 - m;
}
// xd: the voxel's coordinates as doubles (converted once per voxel).
template <class T, int D>
__device__ __forceinline__ SegPoint<T, D> seg_point(const Geom& g, const double* xd, const double* ov, int q) {
  SegPoint<T, D> P;
  const double s = (q >> 1) ? 1.0 : 0.5;  // (q / 2 + 1) / 2
  const int sg = q & 1;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double off = __dmul_rn(s, ov[a]);
    const double y = sg == 0 ? __dadd_rn(xd[a], off) : __dsub_rn(xd[a], off);
    const double fl = floor(y);
    const double tt = __dsub_rn(y, fl);
    const T t1 = static_cast<T>(tt);
    P.w1[a] = t1;
    P.w0[a] = sub_rn(T(1), t1);
    const int32_t st = a == D - 1 ? 1 : static_cast<int32_t>(g.stride[a]);  // offsets stay below 2^31
    if (fabs(fl) < 1073741824.0) {
      const int32_t i0 = static_cast<int32_t>(fl);
      P.off0[a] = reflect32(i0, g.n[a]) * st;
      P.off1[a] = reflect32(i0 + 1, g.n[a]) * st;
    } else {
      const int64_t i0 = static_cast<int64_t>(fl);
      P.off0[a] = static_cast<int32_t>(reflect_any(i0, g.n[a]) * st);
      P.off1[a] = static_cast<int32_t>(reflect_any(i0 + 1, g.n[a]) * st);
    }
  }
  return P;
}
// The D-linear interpolation of f at a segment point: corners in binary order (axis 0 the high
// bit), each corner's value times its axis weights in axis order, summed in corner order.
template <class T, int D>
__device__ __forceinline__ T interp_read(const T* __restrict__ f, const SegPoint<T, D>& P) {
  T acc = T(0);
#pragma unroll
  for (int corner = 0; corner < (1 << D); ++corner) {
    int32_t off = 0;
#pragma unroll
    for (int a = 0; a < D; ++a) off += ((corner >> (D - 1 - a)) & 1) ? P.off1[a] : P.off0[a];
    T term = __ldg(f + off);
#pragma unroll
    for (int a = 0; a < D; ++a) term = mul_rn(term, ((corner >> (D - 1 - a)) & 1) ? P.w1[a] : P.w0[a]);
    acc = add_rn(acc, term);
  }
  return acc;
}
template <int OP, class T>
__device__ __forceinline__ T gather_op(T acc, T v, bool second) {
  if constexpr (OP == 3) return add_rn(acc, v);
  else if constexpr (OP == 2) return second ? min_c(acc, v) : max_c(acc, v);
  else return max_c(acc, v);
}

template <class T, int D, int OP>
__global__ void __launch_bounds__(kThreads, EDAB_GATHER_CTAS) gather_kernel(Geom g, const Elem* __restrict__ el,
                                                         const int32_t* __restrict__ run, const uint8_t* __restrict__ lo,
                                                         const T* __restrict__ t, const T* __restrict__ o0,
                                                         const T* __restrict__ o1, const T* __restrict__ o2,
                                                         const T* __restrict__ rung0, const T* __restrict__ rung1,
                                                         T* __restrict__ out0, T* __restrict__ out1) {
  const int64_t fe = g.batch * g.field;
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    if (!run[b]) continue;
    const int32_t nl = elem_len(g, b);
    const uint32_t pts_mask = el[b].rung_pts;
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      int32_t x[kMaxDim];
      if (!voxel_coords_d<D>(g, v, nl, x)) continue;
      const int64_t at = b * g.field + v;
      const int l = __ldg(lo + at);
      const T tt = __ldg(t + at);
      const T wl = sub_rn(T(1), tt);
      // side 0: rung l with weight 1 - t, side 1: rung l + 1 with weight t (read only when weighted);
      // accumulators a<side><cube>: the value at x, then the segment points in order
      const bool use0 = wl > T(0), use1 = tt > T(0);
      const T* fa0 = rung0 + static_cast<int64_t>(l) * fe + b * g.field;
      const T* fb0 = fa0 + fe;
      const T* fa1 = OP == 2 ? rung1 + static_cast<int64_t>(l) * fe + b * g.field : nullptr;
      const T* fb1 = OP == 2 ? fa1 + fe : nullptr;
      T a00 = use0 ? __ldg(fa0 + v) : T(0), a10 = use1 ? __ldg(fb0 + v) : T(0);
      T a01 = T(0), a11 = T(0);
      if constexpr (OP == 2) {
        a01 = use0 ? __ldg(fa1 + v) : T(0);
        a11 = use1 ? __ldg(fb1 + v) : T(0);
      }
      if constexpr (D >= 2) {
        const bool pts0 = use0 && ((pts_mask >> l) & 1u);
        const bool pts1 = use1 && ((pts_mask >> (l + 1)) & 1u);
        if (pts0 || pts1) {
          double ov[D], xd[D];
          ov[0] = static_cast<double>(__ldg(o0 + at));
          ov[1] = static_cast<double>(__ldg(o1 + at));
          if constexpr (D >= 3) ov[2] = static_cast<double>(__ldg(o2 + at));
#pragma unroll
          for (int a = 0; a < D; ++a) xd[a] = static_cast<double>(x[a]);
#pragma unroll kGatherUnroll
          for (int q = 0; q < 4; ++q) {
            const SegPoint<T, D> P = seg_point<T, D>(g, xd, ov, q);
            if (pts0) {
              a00 = gather_op<OP>(a00, interp_read<T, D>(fa0, P), false);
              if constexpr (OP == 2) a01 = gather_op<OP>(a01, interp_read<T, D>(fa1, P), true);
            }
            if (pts1) {
              a10 = gather_op<OP>(a10, interp_read<T, D>(fb0, P), false);
              if constexpr (OP == 2) a11 = gather_op<OP>(a11, interp_read<T, D>(fb1, P), true);
            }
          }
          if constexpr (OP == 3) {
            if (pts0) a00 = div_rn(a00, T(5));
            if (pts1) a10 = div_rn(a10, T(5));
          }
        }
      }
      T r0 = T(0), r1 = T(0);
      if (use0) {
        r0 = mul_rn(wl, a00);
        if constexpr (OP == 2) r1 = mul_rn(wl, a01);
      }
      if (use1) {
        const T v0 = mul_rn(tt, a10);
        r0 = use0 ? add_rn(r0, v0) : v0;
        if constexpr (OP == 2) {
          const T v1 = mul_rn(tt, a11);
          r1 = use0 ? add_rn(r1, v1) : v1;
        }
      }
      out0[at] = r0;
      if constexpr (OP == 2) out1[at] = r1;
    }
  }
}

template <class T, int D>
__global__ void __launch_bounds__(kThreads) sift_step_kernel(Geom g, int32_t j, Elem* el, const T* __restrict__ r,
                                                            const T* __restrict__ h, const T* __restrict__ mh,
                                                            const T* __restrict__ a, T* __restrict__ hn) {
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    const Elem& e = el[b];
    if (e.status != kActive || !e.sifting) continue;
    const int32_t nl = elem_len(g, b);
    uint64_t m_res = 0, m_h = 0;
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      if (pitch_col(g, v) >= nl) continue;
      const int64_t i = b * g.field + v;
      T m = mh[i];
      if (j >= 1) m = mul_rn(a[i], m);
      const T x = sub_rn(h[i], m);
      hn[i] = x;
      if (j >= 1) {
        const uint64_t br = abs_bits(sub_rn(r[i], x));
        const uint64_t bh = abs_bits(x);
        m_res = br > m_res ? br : m_res;
        m_h = bh > m_h ? bh : m_h;
      }
    }
    if (j >= 1) {
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t u1 = __shfl_xor_sync(0xffffffffu, m_res, o);
        const uint64_t u2 = __shfl_xor_sync(0xffffffffu, m_h, o);
        m_res = u1 > m_res ? u1 : m_res;
        m_h = u2 > m_h ? u2 : m_h;
      }
      if ((threadIdx.x & 31) == 0) {
        if (m_res) atomicMax(reinterpret_cast<unsigned long long*>(&el[b].gmax_res_bits), static_cast<unsigned long long>(m_res));
        if (m_h) atomicMax(reinterpret_cast<unsigned long long*>(&el[b].gmax_h_bits), static_cast<unsigned long long>(m_h));
      }
    }
  }
}

__device__ __forceinline__ bool sift_accepted(const Elem& e) {
  return !(bits_d(e.gmax_res_bits) > e.r_inf) && !(bits_d(e.gmax_h_bits) > e.r_inf);
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// The engine of one chunk geometry.
template <class T>
class Engine {
 public:
  Engine(const Geom& g, const Ctl& c, cudaStream_t s, Workspace& ws) : g_(g), c_(c), s_(s) { bind(ws); }
  // return_orientation: rows (B, rows_cap - 1, D + 1, count) receiving n and c of every mode
  T* orient_out_ = nullptr;

  // x: the chunk's input, dense (B, count) on the device. Rows into rows_out (B, cap, count).
  void run(const T* x, T* rows_out, int32_t* hist_scale, int32_t* hist_sifts, double* hist_spacing,
           double* hist_energy, std::vector<Elem>& out);

  // (public: the stages launch extended device lambdas, which nvcc accepts only in public members)
  Geom g_;
  Ctl c_;
  cudaStream_t s_;
  int64_t B_ = 0;
  // fields
  T *r_, *L_, *Lp_, *h_, *t_, *tau_, *tmp_, *om_, *om2_, *tmp0_, *tmp1_;
  T *n_[kMaxDim], *coh_, *o_[kMaxDim];
  T *m_, *u_, *l_, *mid_, *R_, *U1_, *U2_, *gw_, *a_, *plain_, *up_, *lo_f_, *hd_, *e0_, *emax_, *emin_, *gk_, *e_,
      *q_, *Mn_, *u2_, *l2_, *hn_;
  T *rung0_, *rung1_;
  T* owork_;
  uint8_t *flags_, *ff_, *P_[2], *Pacc_, *A_, *lo_, *marks_, *selm_;
  int32_t* labels_;
  Elem* el_;
  int32_t *win_, *mask_, *rung_win_;
  double* dsc_;      // 8 [B] doubles
  int64_t* cnt_;     // [B]
  uint64_t* nonfin_; // [B]
  int32_t* any_;     // device flags: [0, 2) the mode loop's, [kTcErr] the orientation's pipeline error
  static constexpr int kTcErr = 4;
  void* sel_ws_;
  void* tot_ws_;
  const OrientPlan* plan_ = nullptr;
  int32_t* hist_scale_ = nullptr;
  int32_t* hist_sifts_ = nullptr;
  double* hist_spacing_ = nullptr;
  double* hist_energy_ = nullptr;
  T* rows_ = nullptr;
  std::vector<Elem> hel_;

  void bind(Workspace& ws);
  int32_t* win(int slot) const { return win_ + static_cast<int64_t>(slot) * B_; }
  int32_t* mask(int k) const { return mask_ + static_cast<int64_t>(k) * B_; }
  void read_el() {
    EDAB_CUDA(cudaMemcpyAsync(hel_.data(), el_, sizeof(Elem) * B_, cudaMemcpyDeviceToHost, s_));
    EDAB_CUDA(cudaStreamSynchronize(s_));
  }
  void write_el() { EDAB_CUDA(cudaMemcpyAsync(el_, hel_.data(), sizeof(Elem) * B_, cudaMemcpyHostToDevice, s_)); }

  void noise(const T* r, unsigned axes, const int32_t* run, double* out);
  void noise_per_axis(const T* r, const int32_t* run, double* out);
  void tau_field(const int32_t* run, bool floor2, T* tau);
  void raw_window(const uint8_t* flags, const int32_t* w, const int32_t* run, T* om, T* tmp);
  void scale_field();
  void local_floor();
  void g2();
  void g2_test(const uint8_t* ff, uint8_t* P);
  void orientation_and_build();
  void store_orientation();
  bool ladder_and_weights(int32_t* n_rungs_max);
  void op(int which, const T* in, T* out0, T* out1, int32_t n_rungs_max);
  void envelope_mean(const T* h, T* m, T* u, T* l, int32_t nrm);
  void sifts(int32_t nrm);
  bool commit();
};

template <class T>
void Engine<T>::bind(Workspace& ws) {
  B_ = g_.batch;
  const size_t F = static_cast<size_t>(B_ * g_.field);
  auto fld = [&]() { return ws.take<T>(F); };
  r_ = fld(); L_ = fld(); Lp_ = fld(); h_ = fld(); t_ = fld(); tau_ = fld(); tmp_ = fld(); om_ = fld(); om2_ = fld();
  tmp0_ = fld(); tmp1_ = fld();
  for (int a = 0; a < kMaxDim; ++a) {
    n_[a] = a < g_.dim && g_.dim >= 2 ? fld() : nullptr;
    o_[a] = a < g_.dim && g_.dim >= 2 ? fld() : nullptr;
  }
  coh_ = fld();
  m_ = fld(); u_ = fld(); l_ = fld(); mid_ = fld(); R_ = fld(); U1_ = fld(); U2_ = fld(); gw_ = fld(); a_ = fld();
  plain_ = fld(); up_ = fld(); lo_f_ = fld(); hd_ = fld(); e0_ = fld(); emax_ = fld(); emin_ = fld(); gk_ = fld();
  e_ = fld(); q_ = fld(); Mn_ = fld(); u2_ = fld(); l2_ = fld(); hn_ = fld();
  rung0_ = ws.take<T>(F * kMaxRungs);
  rung1_ = ws.take<T>(F * kMaxRungs);
  owork_ = g_.dim >= 2 ? ws.take<T>(static_cast<size_t>(orient_work_samples(g_))) : nullptr;
  flags_ = ws.take<uint8_t>(F); ff_ = ws.take<uint8_t>(F); P_[0] = ws.take<uint8_t>(F); P_[1] = ws.take<uint8_t>(F);
  Pacc_ = ws.take<uint8_t>(F); A_ = ws.take<uint8_t>(F); lo_ = ws.take<uint8_t>(F); marks_ = ws.take<uint8_t>(F);
  selm_ = ws.take<uint8_t>(F);
  labels_ = ws.take<int32_t>(F);
  el_ = ws.take<Elem>(static_cast<size_t>(B_));
  win_ = ws.take<int32_t>(static_cast<size_t>(kSlots * B_));
  mask_ = ws.take<int32_t>(static_cast<size_t>(kMasks * B_));
  rung_win_ = ws.take<int32_t>(static_cast<size_t>(kMaxRungs * B_));
  dsc_ = ws.take<double>(static_cast<size_t>(8 * B_));
  cnt_ = ws.take<int64_t>(static_cast<size_t>(B_));
  nonfin_ = ws.take<uint64_t>(static_cast<size_t>(B_));
  any_ = ws.take<int32_t>(8);
  sel_ws_ = ws.take<unsigned char>(select_scratch_bytes(g_));
  tot_ws_ = ws.take<unsigned char>(totals_scratch_bytes(g_));
  if (g_.dim >= 2) plan_ = &orient_plan(g_, std::is_same_v<T, double>);
  hel_.resize(static_cast<size_t>(B_));
}

// Noise level of r over the axes of `axes`, pooled: (1.4826 MAD) / sqrt 2 (cpp/src/method/stats.cu:261-334).
template <class T>
void Engine<T>::noise(const T* r, unsigned axes, const int32_t* run, double* out) {
  Sel<T> sel{};
  sel.src = SelSrc::kDiff;
  sel.field = r;
  sel.axes = static_cast<uint8_t>(axes);
  double* center = dsc_;
  double* mad = dsc_ + B_;
  select<T>(s_, g_, sel, -1.0, run, center, nullptr, sel_ws_);
  sel.center = center;
  select<T>(s_, g_, sel, -1.0, run, mad, nullptr, sel_ws_);
  const double sqrt2 = c_.sqrt2;
  for_elements(s_, B_, [=] __device__(int64_t b) {
    if (run[b]) out[b] = __ddiv_rn(__dmul_rn(1.4826, mad[b]), sqrt2);
  });
}

template <class T>
void Engine<T>::noise_per_axis(const T* r, const int32_t* run, double* out) {
  double* acc = dsc_ + 2 * B_;
  double* v = dsc_ + 3 * B_;
  for_elements(s_, B_, [=] __device__(int64_t b) { acc[b] = 0.0; });
  for (int a = 0; a < g_.dim; ++a) {
    if (g_.n[a] < 2) continue;
    noise(r, 1u << a, run, v);
    for_elements(s_, B_, [=] __device__(int64_t b) {
      if (run[b] && v[b] > acc[b]) acc[b] = v[b];
    });
  }
  for_elements(s_, B_, [=] __device__(int64_t b) {
    if (run[b]) out[b] = acc[b];
  });
}

// The threshold field (cpp/src/method/stats_fields.cu:25-69): det = r - Box_Wd r, lev =
// sqrt(max(Box_Wl det^2, 0)), tau = max(theta max(lev, k sigma_n), tol, floor2).
template <class T>
void Engine<T>::tau_field(const int32_t* run, bool floor2, T* tau) {
  CubeArgs<T> a{};
  a.in = r_;
  a.out0 = tmp_;
  a.win = win(kWd);
  a.rungs = 1;
  a.epi = BoxEpi::kDetSq;
  a.aux = r_;
  cube<T>(s_, g_, CubeOp::kBox, a);
  cube_simple<T>(s_, g_, CubeOp::kBox, tmp_, tau, nullptr, win(kWl));
  const Ctl c = c_;
  Elem* el = el_;
  const int32_t* wd = win(kWd);
  for_voxels(s_, g_, [=] __device__(int64_t b) { return run[b] && wd[b] >= 1; },
             [=] __device__(int64_t b, int64_t, int64_t i) {
               const T be = tau[i];
               const double sn = el[b].sigma_n;
               if (!(isfinite(be) && isfinite(sn))) el[b].nonfinite = 1;
               const T lev = sqrt_rn<T>(be > T(0) ? be : T(0));
               const double f = __dmul_rn(c.sig_noise, sn);
               const double fl = f > 0.0 ? f : 0.0;
               const double ld = static_cast<double>(lev);
               double t = __dmul_rn(c.sig_theta, ld > fl ? ld : fl);
               const double tl = el[b].tol;
               t = t > tl ? t : tl;
               if (floor2) {
                 const double f2 = __dmul_rn(c.fine_theta, el[b].sigma_x);
                 t = t > f2 ? t : f2;
               }
               tau[i] = static_cast<T>(t);
             });
}

// The raw window (cpp/src/method/stats_fields.cu:340-369): rho_a = Box_w (bit a of flags), om =
// 2 kappa / max(sqrt(sum rho_a^2), tiny) where the density is positive, +inf elsewhere.
template <class T>
void Engine<T>::raw_window(const uint8_t* flags, const int32_t* w, const int32_t* run, T* om, T* tmp) {
  const T two_kappa = static_cast<T>(2.0 * c_.kappa);
  const T tiny = static_cast<T>(c_.tiny);
  const int D = g_.dim;
  for (int a = 0; a < D; ++a) {
    CubeArgs<T> ca{};
    ca.src_bits = flags;
    ca.bit = a;
    ca.out0 = tmp;
    ca.win = w;
    ca.rungs = 1;
    cube<T>(s_, g_, CubeOp::kBox, ca);
    const bool last = a == D - 1;
    for_voxels(s_, g_, [=] __device__(int64_t b) { return run[b] && w[b] >= 1; },
               [=] __device__(int64_t, int64_t, int64_t i) {
                 const T rho = tmp[i];
                 const T sq = mul_rn(rho, rho);
                 const T acc = a == 0 ? sq : add_rn(om[i], sq);
                 if (!last) {
                   om[i] = acc;
                   return;
                 }
                 const T dens = sqrt_rn<T>(acc);
                 om[i] = dens > T(0) ? div_rn<T>(two_kappa, dens > tiny ? dens : tiny) : inf_t<T>();
               });
  }
}

// The scale field with the absence rule (cpp/src/method/stats_scale.cu:85-167, 222-246).
template <class T>
void Engine<T>::scale_field() {
  const Ctl c = c_;
  Elem* el = el_;
  const Geom g = g_;
  int32_t* wnear = win(kNear);
  const int32_t* wW = win(kW);
  const int32_t* on = mask(kOn);
  for_elements(s_, B_, [=] __device__(int64_t b) {
    const int32_t W = el[b].W;
    wnear[b] = (on[b] && wW[b] >= 1) ? odd_window(__dmul_rn(__dmul_rn(2.0, c.absent_reach), static_cast<double>(W))) : 0;
  });
  T* fine = tmp0_;
  uint8_t* A = A_;
  uint8_t* marks = marks_;
  const T* om = om_;
  const auto runW = [=] __device__(int64_t b) { return on[b] && wW[b] >= 1; };
  for_samples(s_, B_ * g_.field, [=] __device__(int64_t i) {
    const int64_t b = elem_of(g, i);
    if (on[b] && wW[b] >= 1) marks[i] = 0;
  });
  for_voxels(s_, g_, runW, [=] __device__(int64_t b, int64_t, int64_t i) {
    const double w = static_cast<double>(el[b].w);
    const double o = static_cast<double>(om[i]);
    const bool a0 = o > __dmul_rn(c.reset, w);
    const bool aw = o > __dmul_rn(c.absent_lo, w);
    const bool fn = o < __ddiv_rn(__dmul_rn(c.absent_lo, w), el[b].jump);
    A[i] = static_cast<uint8_t>((a0 ? 4u : 0u) | (aw ? 2u : 0u));
    fine[i] = fn ? T(1) : T(0);
  });
  cube_simple<T>(s_, g_, CubeOp::kMax, fine, fine, nullptr, wnear);
  ccl(s_, g_, A_, 2u, labels_, wW);
  const int32_t* labels = labels_;
  for_voxels(s_, g_, runW, [=] __device__(int64_t b, int64_t, int64_t i) {
    if ((A[i] & 2u) && fine[i] > T(0.5)) marks[b * g.field + labels[i]] = 1;
  });
  T* L = L_;
  for_voxels(s_, g_, runW, [=] __device__(int64_t b, int64_t, int64_t i) {
    const uint8_t m = A[i];
    const int32_t lab = labels[i];
    const bool a = (m & 4u) && lab >= 0 && marks[b * g.field + lab];
    A[i] = a ? 1 : 0;
    const double w = static_cast<double>(el[b].w);
    double v;
    if (a) {
      v = c.absent;
    } else {
      const double o = static_cast<double>(om[i]);
      const double ow = o > __dmul_rn(c.reset, w) ? w : o;
      const double lo = __ddiv_rn(w, c.c_lo);
      const double hi = __dmul_rn(c.c_hi, w);
      v = ow > lo ? ow : lo;
      v = v < hi ? v : hi;
    }
    L[i] = log_t<T>(static_cast<T>(v));
  });
  cube_simple<T>(s_, g_, CubeOp::kBox, L, L, nullptr, wW);
  for_voxels(s_, g_, runW, [=] __device__(int64_t, int64_t, int64_t i) { L[i] = exp_t<T>(L[i]); });
}

// The per-voxel floor of modes k >= 1 (cpp/src/method/stats_scale.cu:169-201, 249-268).
template <class T>
void Engine<T>::local_floor() {
  Elem* el = el_;
  int32_t* wf = win(kFloor);
  const int32_t* onf = mask(kOnFloor);
  for_elements(s_, B_, [=] __device__(int64_t b) { wf[b] = (onf[b] && el[b].W >= 1) ? el[b].W : 0; });
  CubeArgs<T> ca{};
  ca.src_bits = A_;
  ca.bit = 0;
  ca.out0 = tmp0_;
  ca.win = wf;
  ca.rungs = 1;
  cube<T>(s_, g_, CubeOp::kBox, ca);
  const Ctl c = c_;
  const T* Lp = Lp_;
  const T* chi = tmp0_;
  T* L = L_;
  for_voxels(s_, g_, [=] __device__(int64_t b) { return wf[b] >= 1; }, [=] __device__(int64_t b, int64_t, int64_t i) {
    const T lp = Lp[i];
    const bool grow = c.growth > 1.0 && el[b].k >= c.growth_from;
    T fl = grow ? mul_rn(static_cast<T>(c.growth), lp) : add_rn(lp, T(2));
    const T cap = static_cast<T>(__dmul_rn(c.c_hi, static_cast<double>(el[b].w)));
    fl = fl < cap ? fl : cap;
    const T x = chi[i];
    const T e = add_rn(mul_rn(sub_rn(T(1), x), log_t<T>(fl)), mul_rn(x, static_cast<T>(c.log_absent)));
    const T f = exp_t<T>(e);
    const T l = L[i];
    L[i] = l >= f ? l : f;
  });
}

// One G2 rung test of every element with srung > 0 (cpp/src/method/stats_rungs.cu:14-87).
template <class T>
void Engine<T>::g2_test(const uint8_t* ff, uint8_t* P) {
  const Ctl c = c_;
  Elem* el = el_;
  const int32_t* srung = mask(kSrung);
  int32_t* wb = win(kG2b);
  int32_t* wcore = win(kG2core);
  int32_t* wrq = win(kG2rq);
  for_elements(s_, B_, [=] __device__(int64_t b) {
    const int32_t s = srung[b];
    int32_t x = 0, y = 0, z = 0;
    if (s > 0) {
      const double sd = static_cast<double>(s);
      x = odd_window(__dmul_rn(c.fine_beta, sd));
      y = odd_window(__dmul_rn(c.fine_core, sd));
      z = odd_window(__dmul_rn(__dmul_rn(2.0, c.absent_reach), static_cast<double>(x)));
    }
    wb[b] = x;
    wcore[b] = y;
    wrq[b] = z;
    el[b].g2_any_core = 0;
    el[b].g2_any_jump = 0;
  });
  T* om = om2_;
  T* t1 = tmp1_;
  raw_window(ff, wb, srung, om, t1);
  const auto runS = [=] __device__(int64_t b) { return srung[b] > 0; };
  for_voxels(s_, g_, runS, [=] __device__(int64_t b, int64_t, int64_t i) {
    const bool in = static_cast<double>(om[i]) < __dmul_rn(c.fine_lo, static_cast<double>(srung[b]));
    P[i] = in ? 1 : 0;
    t1[i] = in ? T(1) : T(0);
  });
  cube_simple<T>(s_, g_, CubeOp::kMin, t1, t1, nullptr, wcore);
  for_voxels(s_, g_, runS, [=] __device__(int64_t b, int64_t, int64_t i) {
    if (t1[i] > T(0.5)) el[b].g2_any_core = 1;
    t1[i] = (P[i] & 1u) ? T(1) : T(0);
  });
  Sel<T> sel{};
  sel.src = SelSrc::kField;
  sel.field = om;
  sel.mask = P;
  sel.bits = 1;
  double* p = dsc_ + 4 * B_;
  int64_t* np = cnt_;
  select<T>(s_, g_, sel, c_.fine_pop, srung, p, np, sel_ws_);
  cube_simple<T>(s_, g_, CubeOp::kMax, t1, t1, nullptr, wrq);
  for_voxels(s_, g_, runS, [=] __device__(int64_t b, int64_t, int64_t i) {
    if (static_cast<double>(om[i]) > __dmul_rn(c.reset, p[b]) && t1[i] > T(0.5)) el[b].g2_any_jump = 1;
  });
  const Geom g = g_;
  for_elements(s_, B_, [=] __device__(int64_t b) {
    if (srung[b] <= 0) return;
    Elem& e = el[b];
    e.g2_res_np = np[b];
    e.g2_res_p = p[b];
    e.g2_res_cov = __ddiv_rn(static_cast<double>(np[b]), static_cast<double>(elem_count(g, b)));
    if (np[b] == 0 || !e.g2_any_core) e.g2_res_outcome = kG2None;
    else if (__dmul_rn(c.fine_jump, p[b]) > static_cast<double>(e.w)) e.g2_res_outcome = kG2Stop;
    else e.g2_res_outcome = e.g2_any_jump ? kG2Accepted : kG2None;
  });
}

// G2 and G3 (cpp/src/method/driver.cpp:445-509; the machine of driver.cpp:73-116 on the device).
template <class T>
void Engine<T>::g2() {
  // S1: the candidates of every G2-eligible element (host pow)
  read_el();
  int32_t steps = 0;
  bool any = false;
  for (int64_t b = 0; b < B_; ++b) {
    Elem& e = hel_[static_cast<size_t>(b)];
    e.g2_n = 0;
    e.g2_done = 1;
    e.g2_accepted = 0;
    if (e.status != kActive || !e.on_g2) continue;
    const std::vector<int32_t> rungs = g2_candidate_rungs(e.w, e.w_prev, c_.fine_jump);
    e.g2_n = static_cast<int32_t>(rungs.size());
    for (size_t i = 0; i < rungs.size(); ++i) e.g2_rungs[i] = rungs[i];
    e.g2_rungs[rungs.size()] = odd_window(static_cast<double>(rungs.back()) * kRungRatio + 1.0);
    e.g2_i = 0;
    e.g2_pending = 0;
    e.g2_done = rungs.empty() ? 1 : 0;
    e.g2_acc_index = -1;
    steps = std::max(steps, e.g2_n + 1);
    any = any || !rungs.empty();
  }
  write_el();
  if (!any) return;
  Elem* el = el_;
  int32_t* ong2 = mask(kOnG2);
  for_elements(s_, B_, [=] __device__(int64_t b) { ong2[b] = el[b].status == kActive && el[b].on_g2; });
  const uint8_t* ff = flags_;
  if (c_.fine_theta > 0) {
    tau_field(ong2, true, tau_);
    sig_flags<T>(s_, g_, r_, tau_, ff_, el_, ong2);
    ff = ff_;
  }
  int32_t* srung = mask(kSrung);
  for (int32_t step = 0; step < steps; ++step) {
    for_elements(s_, B_, [=] __device__(int64_t b) {
      const Elem& e = el[b];
      srung[b] = (e.status == kActive && e.on_g2 && !e.g2_done) ? e.g2_rungs[e.g2_i] : 0;
    });
    g2_test(ff, P_[step & 1]);
    for_elements(s_, B_, [=] __device__(int64_t b) {
      if (srung[b] <= 0) return;
      Elem& e = el[b];
      const int32_t o = e.g2_res_outcome;
      if (e.g2_pending) {
        if (o == kG2Accepted) {
          e.g2_done = 1;
          e.g2_accepted = 1;
          e.g2_acc_index = e.g2_i - 1;
          return;
        }
        if (o == kG2Stop) {
          e.g2_done = 1;
          return;
        }
        e.g2_pending = 0;
        ++e.g2_i;
      } else {
        if (o == kG2Stop) {
          e.g2_done = 1;
          return;
        }
        if (o == kG2Accepted) {
          e.g2_pending = 1;
          e.g2_cand_p = e.g2_res_p;
          e.g2_cand_cov = e.g2_res_cov;
          e.g2_cand_s = e.g2_rungs[e.g2_i];
        }
        ++e.g2_i;
      }
      if (e.g2_i >= e.g2_n && !e.g2_pending) e.g2_done = 1;
    });
  }
  // accepted: fine, p, the population of the accepted rung (step acc_index wrote P[acc_index & 1])
  int32_t* onfine = mask(kOnFine);
  for_elements(s_, B_, [=] __device__(int64_t b) {
    Elem& e = el[b];
    const bool acc = e.status == kActive && e.on_g2 && e.g2_accepted;
    onfine[b] = acc ? 1 : 0;
    if (!acc) return;
    e.fine = 1;
    e.p = e.g2_cand_p;
    e.p_odd = odd_window(e.g2_cand_p);
    e.cov = e.g2_cand_cov;
    e.g2_slot = e.g2_acc_index & 1;
  });
  uint8_t* P0 = P_[0];
  uint8_t* P1 = P_[1];
  uint8_t* Pacc = Pacc_;
  const Geom g = g_;
  for_samples(s_, B_ * g_.field, [=] __device__(int64_t i) {
    const int64_t b = elem_of(g, i);
    if (onfine[b]) Pacc[i] = el[b].g2_slot ? P1[i] : P0[i];
  });
  // G3: the coarse median of the raw window outside the population's reach
  // (cpp/src/method/stats_rungs.cu:89-121, 161-187)
  const Ctl c = c_;
  int32_t* w3c = win(kG3c);
  int32_t* w3r = win(kG3r);
  for_elements(s_, B_, [=] __device__(int64_t b) {
    const bool run = onfine[b] != 0;
    w3c[b] = run ? odd_window(__dmul_rn(c.beta, static_cast<double>(el[b].w))) : 0;
    const int32_t wf = odd_window(__dmul_rn(c.fine_beta, static_cast<double>(el[b].p_odd)));
    w3r[b] = run ? odd_window(__dmul_rn(__dmul_rn(2.0, c.absent_reach), static_cast<double>(wf))) : 0;
  });
  T* omc = om2_;
  T* t1 = tmp1_;
  raw_window(ff, w3c, onfine, omc, t1);
  for_voxels(s_, g_, [=] __device__(int64_t b) { return onfine[b] != 0; },
             [=] __device__(int64_t, int64_t, int64_t i) { t1[i] = (Pacc[i] & 1u) ? T(1) : T(0); });
  cube_simple<T>(s_, g_, CubeOp::kMax, t1, t1, nullptr, w3r);
  uint8_t* sel = selm_;
  for_samples(s_, B_ * g_.field, [=] __device__(int64_t i) {
    const int64_t b = elem_of(g, i);
    if (!onfine[b]) return;
    sel[i] = (!is_pad_b(g, b, i - b * g.field) && t1[i] < T(0.5) && omc[i] < inf_t<T>()) ? 1 : 0;
  });
  Sel<T> ss{};
  ss.src = SelSrc::kField;
  ss.field = omc;
  ss.mask = sel;
  ss.bits = 1;
  double* wc = dsc_ + 5 * B_;
  select<T>(s_, g_, ss, -1.0, onfine, wc, cnt_, sel_ws_);
  const int64_t* cnt = cnt_;
  for_elements(s_, B_, [=] __device__(int64_t b) {
    if (onfine[b]) el[b].wc = cnt[b] == 0 ? d_inf() : wc[b];
  });
}

// The orientation and the element build (cpp/src/method/element.cu:181-216).
template <class T>
void Engine<T>::orientation_and_build() {
  const int32_t* on = mask(kOn);
  Elem* el = el_;
  int32_t* win_s = win_;
  int32_t* mask_s = mask_;
  const int64_t B = B_;
  if (g_.dim >= 2) {
    orientation<T>(s_, g_, *plan_, r_, el_, on, n_, coh_, owork_, c_.two_sigma2, any_ + kTcErr);
    for_elements(s_, B_, [=] __device__(int64_t b) {
      if (el[b].status == kActive && el[b].nonfinite) fail2(el[b], win_s, mask_s, B, b);
    });
    if (orient_out_) store_orientation();
  }
  const dim3 grid = voxel_grid(g_);
  switch (g_.dim) {
    case 1: element_extent<T, 1><<<grid, kThreads, 0, s_>>>(g_, c_, L_, coh_, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, t_, lo_, el_, on); break;
    case 2: element_extent<T, 2><<<grid, kThreads, 0, s_>>>(g_, c_, L_, coh_, n_[0], n_[1], nullptr, o_[0], o_[1], nullptr, t_, lo_, el_, on); break;
    default: element_extent<T, 3><<<grid, kThreads, 0, s_>>>(g_, c_, L_, coh_, n_[0], n_[1], n_[2], o_[0], o_[1], o_[2], t_, lo_, el_, on); break;
  }
  EDAB_LAUNCH("element_extent");
}

// return_orientation: n with the canonical sign (the first component of magnitude above the dtype's
// default tie tolerance positive) and c at the row of this mode's IMF, unpadded, for every element
// still active (cpp/src/method/orientation.cu:412-418, 495-522; driver.cpp:553-559).
template <class T>
void Engine<T>::store_orientation() {
  const Elem* el = el_;
  const Geom g = g_;
  const int32_t D = g_.dim;
  const int32_t rows = c_.rows_cap - 1;
  const T zero = static_cast<T>(std::is_same_v<T, float> ? std::ldexp(1.0, -14) : std::ldexp(1.0, -30));
  const T* n0 = n_[0];
  const T* n1 = n_[1];
  const T* n2 = n_[2];
  const T* coh = coh_;
  T* out = orient_out_;
  const int32_t nl = g_.n_last;
  for_voxels(s_, g_, [=] __device__(int64_t b) { return el[b].status == kActive; },
             [=] __device__(int64_t b, int64_t v, int64_t i) {
               T nt[3] = {n0[i], n1[i], D >= 3 ? n2[i] : T(0)};
               int sg = 0;
               for (int a = 0; a < D; ++a) sg = sg == 0 && fabs(nt[a]) > zero ? (nt[a] > T(0) ? 1 : -1) : sg;
               const int64_t q = pitch_row(g, v);
               const int64_t t = v - q * g.pitch;
               T* o = out + ((b * rows + el[b].n_imfs) * (D + 1)) * g.count + q * nl + t;
               for (int a = 0; a < D; ++a) o[a * g.count] = sg < 0 ? -nt[a] : nt[a];
               o[D * g.count] = coh[i];
             });
}

// S4: the ladders (host), then the rung logs, the weights and the rung windows.
template <class T>
bool Engine<T>::ladder_and_weights(int32_t* n_rungs_max) {
  read_el();
  int32_t nrm = 0;
  bool any = false;
  for (int64_t b = 0; b < B_; ++b) {
    Elem& e = hel_[static_cast<size_t>(b)];
    e.rung_pts = 0;
    e.rung_used = 0;
    if (e.status != kActive) {
      e.n_rungs = 0;
      continue;
    }
    any = true;
    double d_min, d_max;
    std::memcpy(&d_min, &e.d_min_bits, sizeof d_min);
    std::memcpy(&d_max, &e.d_max_bits, sizeof d_max);
    const int32_t n_max = g_.len_host ? g_.len_host[b] : c_.n_max;
    const std::vector<int32_t> ladder = rung_ladder(d_min, d_max, e.w, n_max);
    if (ladder.empty() || static_cast<int32_t>(ladder.size()) > kMaxRungs) throw std::logic_error("eda: ladder size out of range");
    e.n_rungs = static_cast<int32_t>(ladder.size());
    for (int32_t j = 0; j < kMaxRungs; ++j) e.rung_w[j] = j < e.n_rungs ? ladder[static_cast<size_t>(j)] : 0;
    nrm = std::max(nrm, e.n_rungs);
  }
  write_el();
  *n_rungs_max = nrm;
  if (!any) return false;
  Elem* el = el_;
  const int32_t* on = mask(kOn);
  for_samples(s_, B_ * kMaxRungs, [=] __device__(int64_t i) {
    const int64_t b = i / kMaxRungs;
    const int j = static_cast<int>(i % kMaxRungs);
    if (on[b] && j < el[b].n_rungs) el[b].rung_lw[j] = log(static_cast<double>(el[b].rung_w[j]));
  });
  element_rungs<T><<<voxel_grid(g_), kThreads, 0, s_>>>(g_, lo_, t_, el_, on);
  EDAB_LAUNCH("element_rungs");
  int32_t* rw = rung_win_;
  const int64_t B = B_;
  for_samples(s_, B_ * kMaxRungs, [=] __device__(int64_t i) {
    const int j = static_cast<int>(i / B);
    const int64_t b = i - static_cast<int64_t>(j) * B;
    const Elem& e = el[b];
    const bool use = e.status == kActive && j < nrm && j < e.n_rungs && ((e.rung_used >> j) & 1u) != 0u;
    rw[i] = use ? e.rung_w[j] : 0;
  });
  return true;
}

// An operator over every used rung: the rung cubes (one launch per pass for all rungs; the first
// pass stages the input once), then one gather per voxel.
template <class T>
void Engine<T>::op(int which, const T* in, T* out0, T* out1, int32_t nrm) {
  CubeArgs<T> a{};
  a.in = in;
  a.out0 = rung0_;
  a.out1 = which == 2 ? rung1_ : nullptr;
  a.win = rung_win_;
  a.rungs = nrm;
  a.out_stride = B_ * g_.field;
  const CubeOp cop = which == 3 ? CubeOp::kBox : (which == 2 ? CubeOp::kMaxMin : CubeOp::kMax);
  // the gather's segment points index an element with 32-bit offsets
  if (g_.field > INT32_MAX) throw std::invalid_argument("eda: an element of more than 2^31 padded samples");
  cube<T>(s_, g_, cop, a);
  const dim3 grid = voxel_grid(g_);
  const int32_t* on = mask(kOn);
  const T* o0 = o_[0];
  const T* o1 = o_[1];
  const T* o2 = o_[2];
#define EDAB_GATHER(D, OP) \
  gather_kernel<T, D, OP><<<grid, kThreads, 0, s_>>>(g_, el_, on, lo_, t_, o0, o1, o2, rung0_, rung1_, out0, out1)
  if (g_.dim == 1) {
    if (which == 0) EDAB_GATHER(1, 0); else if (which == 2) EDAB_GATHER(1, 2); else EDAB_GATHER(1, 3);
  } else if (g_.dim == 2) {
    if (which == 0) EDAB_GATHER(2, 0); else if (which == 2) EDAB_GATHER(2, 2); else EDAB_GATHER(2, 3);
  } else {
    if (which == 0) EDAB_GATHER(3, 0); else if (which == 2) EDAB_GATHER(3, 2); else EDAB_GATHER(3, 3);
  }
#undef EDAB_GATHER
  EDAB_LAUNCH("gather_kernel");
}

template <class T>
void Engine<T>::envelope_mean(const T* h, T* m, T* u, T* l, int32_t nrm) {
  op(2, h, u, l, nrm);
  T* mid = mid_;
  const int32_t* on = mask(kOn);
  for_voxels(s_, g_, [=] __device__(int64_t b) { return on[b] != 0; },
             [=] __device__(int64_t, int64_t, int64_t i) { mid[i] = mul_rn(T(0.5), add_rn(u[i], l[i])); });
  op(3, mid, m, nullptr, nrm);
}

// Sift 1, the continuation weight, sifts 2..S with G1 and the guard
// (cpp/src/method/driver.cpp:606-680; cpp/src/method/sift.cu:54-232).
template <class T>
void Engine<T>::sifts(int32_t nrm) {
  const Ctl c = c_;
  Elem* el = el_;
  const int32_t* on = mask(kOn);
  const auto runOn = [=] __device__(int64_t b) { return on[b] != 0; };
  T* r = r_;
  T* h = h_;
  envelope_mean(r_, m_, u_, l_, nrm);
  {
    const T* m = m_;
    for_voxels(s_, g_, [=] __device__(int64_t b) { return el[b].status == kActive && el[b].sifting; },
               [=] __device__(int64_t, int64_t, int64_t i) { h[i] = sub_rn(r[i], m[i]); });
    for_elements(s_, B_, [=] __device__(int64_t b) {
      if (el[b].status == kActive && el[b].sifting) el[b].n_sifts += 1;
      el[b].gmax_res_bits = 0;
      el[b].gmax_h_bits = 0;
    });
  }
  if (c_.sifts <= 1) return;
  // the continuation weight: R = max(Dil r - Ero r, 0), U = Dil^u R, g = ramp(R / U), a = clip(Avg^s g)
  {
    T* R = R_;
    const T* u = u_;
    const T* l = l_;
    for_voxels(s_, g_, runOn, [=] __device__(int64_t, int64_t, int64_t i) { R[i] = np_max(sub_rn(u[i], l[i]), T(0)); });
  }
  const T* U = R_;
  T* pp[2] = {U1_, U2_};
  for (int32_t i = 0; i < c_.u; ++i) {
    op(0, U, pp[i & 1], nullptr, nrm);
    U = pp[i & 1];
  }
  {
    const T* R = R_;
    T* gw = gw_;
    const T t0 = static_cast<T>(c.t0);
    const double dd = c.t1 - c.t0;
    const T den = static_cast<T>(dd >= 1e-12 ? dd : 1e-12);
    for_voxels(s_, g_, runOn, [=] __device__(int64_t b, int64_t, int64_t i) {
      const double tol = el[b].tol;
      const T Uv = U[i];
      T rho = T(0);
      if (static_cast<double>(Uv) > tol) rho = clip(div_rn(R[i], Uv), T(0), T(1));
      gw[i] = clip(div_rn(sub_rn(rho, t0), den), T(0), T(1));
    });
  }
  const T* cur = gw_;
  for (int32_t i = 0; i < c_.s; ++i) {
    T* dst = (i + 1 < c_.s) ? (cur == U1_ ? U2_ : U1_) : a_;
    op(3, cur, dst, nullptr, nrm);
    cur = dst;
  }
  {
    T* a = a_;
    for_voxels(s_, g_, runOn, [=] __device__(int64_t, int64_t, int64_t i) { a[i] = clip(a[i], T(0), T(1)); });
  }
  // sifts 2..S
  const int32_t* wW = win(kW);
  for (int32_t j = 1; j < c_.sifts; ++j) {
    envelope_mean(h_, plain_, up_, lo_f_, nrm);
    {
      T* hd = hd_;
      const T* up = up_;
      const T* lo = lo_f_;
      for_voxels(s_, g_, runOn, [=] __device__(int64_t, int64_t, int64_t i) { hd[i] = mul_rn(T(0.5), sub_rn(up[i], lo[i])); });
    }
    op(3, hd_, e0_, nullptr, nrm);
    cube_simple<T>(s_, g_, CubeOp::kMaxMin, e0_, emax_, emin_, wW);
    {
      T* kr = emax_;
      const T* emin = emin_;
      const T k0 = static_cast<T>(c.ramp_k0);
      const double dk = c.ramp_k1 - c.ramp_k0;
      const T kden = static_cast<T>(dk >= 1e-12 ? dk : 1e-12);
      for_voxels(s_, g_, runOn, [=] __device__(int64_t b, int64_t, int64_t i) {
        const double tol = el[b].tol;
        const T fl = static_cast<T>(tol >= c.tiny ? tol : c.tiny);
        const T hi = kr[i], lo = emin[i];
        const T den = np_max(add_rn(hi, lo), fl);
        const T kap = div_rn(sub_rn(hi, lo), den);
        kr[i] = clip(div_rn(sub_rn(kap, k0), kden), T(0), T(1));
      });
    }
    cube_simple<T>(s_, g_, CubeOp::kBox, emax_, gk_, nullptr, wW);
    {
      T* gk = gk_;
      for_voxels(s_, g_, runOn, [=] __device__(int64_t, int64_t, int64_t i) { gk[i] = clip(gk[i], T(0), T(1)); });
    }
    const T* esrc = e0_;
    for (int32_t i = 0; i < c_.anorm_smooth; ++i) {
      cube_simple<T>(s_, g_, CubeOp::kBox, esrc, e_, nullptr, wW);
      esrc = e_;
    }
    Sel<T> sel{};
    sel.src = SelSrc::kField;
    sel.field = e_;
    double* emed = dsc_ + 6 * B_;
    select<T>(s_, g_, sel, -1.0, on, emed, nullptr, sel_ws_);
    {
      T* e = e_;
      const T* hh = h_;
      T* q = q_;
      for_voxels(s_, g_, runOn, [=] __device__(int64_t b, int64_t, int64_t i) {
        double thr = __dmul_rn(c.anorm_floor, emed[b]);
        const double tol = el[b].tol;
        thr = thr >= tol ? thr : tol;
        thr = thr >= c.tiny ? thr : c.tiny;
        const T ev = e[i];
        const T ef = static_cast<double>(ev) >= thr ? ev : static_cast<T>(thr);
        e[i] = ef;
        q[i] = div_rn(hh[i], ef);
      });
    }
    envelope_mean(q_, Mn_, u2_, l2_, nrm);
    {
      T* Mn = Mn_;
      const T* gk = gk_;
      const T* e = e_;
      const T* up = up_;
      const T* lo = lo_f_;
      const T* plain = plain_;
      for_voxels(s_, g_, runOn, [=] __device__(int64_t, int64_t, int64_t i) {
        const T w = gk[i];
        const T mA = clip(mul_rn(e[i], Mn[i]), lo[i], up[i]);
        Mn[i] = add_rn(mul_rn(w, mA), mul_rn(sub_rn(T(1), w), plain[i]));
      });
    }
    const dim3 grid = voxel_grid(g_);
    sift_step_kernel<T, 1><<<grid, kThreads, 0, s_>>>(g_, j, el_, r_, h_, Mn_, a_, hn_);
    EDAB_LAUNCH("sift_step_kernel");
    {
      T* hh = h_;
      const T* hn = hn_;
      for_voxels(s_, g_, [=] __device__(int64_t b) { return el[b].status == kActive && el[b].sifting && sift_accepted(el[b]); },
                 [=] __device__(int64_t, int64_t, int64_t i) { hh[i] = hn[i]; });
      for_elements(s_, B_, [=] __device__(int64_t b) {
        Elem& e = el[b];
        if (e.status != kActive || !e.sifting) return;
        if (sift_accepted(e)) e.n_sifts += 1;
        else e.sifting = 0;
        e.gmax_res_bits = 0;
        e.gmax_h_bits = 0;
      });
    }
  }
}

// The commit (cpp/src/method/mode.cu:304-348; cpp/src/field/field_ops.cu:151-203): the IMF row,
// r -= h, the canonical energies, the history, the next mode's state; true while any element runs.
template <class T>
bool Engine<T>::commit() {
  const Ctl c = c_;
  Elem* el = el_;
  T* rows = rows_;
  T* r = r_;
  const T* h = h_;
  const Geom g = g_;
  const int32_t nl = g_.n_last;
  for_voxels(s_, g_, [=] __device__(int64_t b) { return el[b].status == kActive; },
             [=] __device__(int64_t b, int64_t v, int64_t i) {
               const int64_t q = pitch_row(g, v);
               const int64_t t = v - q * g.pitch;
               const T hv = h[i];
               rows[(b * c.rows_cap + el[b].n_imfs) * g.count + q * nl + t] = hv;
               r[i] = sub_rn(r[i], hv);
             });
  double* eh = dsc_ + 0 * B_;
  double* er = dsc_ + 1 * B_;
  double* am = dsc_ + 2 * B_;
  field_totals<T>(s_, g_, h_, eh, nullptr, nullptr, tot_ws_);
  field_totals<T>(s_, g_, r_, er, am, nullptr, tot_ws_);
  int32_t* any = any_;
  EDAB_CUDA(cudaMemsetAsync(any_, 0, sizeof(int32_t) * 2, s_));
  int32_t* hs = hist_scale_;
  int32_t* hf = hist_sifts_;
  double* hp = hist_spacing_;
  double* he = hist_energy_;
  for_elements(s_, B_, [=] __device__(int64_t b) {
    Elem& e = el[b];
    if (e.status == kActive) {
      const int64_t hrow = b * (c.rows_cap - 1) + e.n_imfs;
      hs[hrow] = e.w;
      he[hrow] = eh[b];
      hp[hrow] = e.spacing;
      hf[hrow] = e.n_sifts;
      e.n_imfs += 1;
      e.amax = am[b];
      e.r_energy = er[b];
      e.tol = tie_tol<T>(c.tau, e.amax);
      e.w_prev = e.w;
      e.k += 1;
      if (!isfinite(e.amax)) {
        e.status = kError;
        e.error = kErrNonFiniteResult;
      } else if (c.max_imf > 0 && e.n_imfs >= c.max_imf) {
        e.status = kDone;
      } else if (e.n_imfs + 1 >= c.rows_cap) {
        e.status = kError;
        e.error = kErrInternal;
        atomicOr(any + 1, 1);
      }
    }
    if (e.status == kActive) atomicOr(any, 1);
  });
  int32_t flags[2] = {0, 0};
  EDAB_CUDA(cudaMemcpyAsync(flags, any_, sizeof flags, cudaMemcpyDeviceToHost, s_));
  EDAB_CUDA(cudaStreamSynchronize(s_));
  if (flags[1]) throw std::logic_error("eda: the output rows are full (mode bound violated)");
  return flags[0] != 0;
}

template <class T>
void Engine<T>::run(const T* x, T* rows_out, int32_t* hist_scale, int32_t* hist_sifts, double* hist_spacing,
                    double* hist_energy, std::vector<Elem>& out) {
  rows_ = rows_out;
  hist_scale_ = hist_scale;
  hist_sifts_ = hist_sifts;
  hist_spacing_ = hist_spacing;
  hist_energy_ = hist_energy;
  const Ctl c = c_;
  const Geom g = g_;
  const int64_t B = B_;
  Elem* el = el_;
  int32_t* winp = win_;
  int32_t* maskp = mask_;
  T* r = r_;
  // start (cpp/src/method/driver.cpp:393-420): the padded copy, the prescale by 2^-ilogb(max|x|)
  const int32_t nl = g_.n_last;
  for_samples(s_, B_ * g_.field, [=] __device__(int64_t i) {
    const int64_t b = elem_of(g, i);
    const int64_t v = i - b * g.field;
    const int64_t q = pitch_row(g, v);
    const int64_t t = v - q * g.pitch;
    r[i] = t < (g.len ? elem_len(g, b) : nl) ? x[b * g.count + q * nl + t] : T(0);
  });
  EDAB_CUDA(cudaMemsetAsync(nonfin_, 0, sizeof(uint64_t) * B_, s_));
  EDAB_CUDA(cudaMemsetAsync(el_, 0, sizeof(Elem) * B_, s_));
  EDAB_CUDA(cudaMemsetAsync(any_ + kTcErr, 0, sizeof(int32_t), s_));
  double* am = dsc_ + 2 * B_;
  double* en = dsc_ + 1 * B_;
  field_totals<T>(s_, g_, r_, en, am, nonfin_, tot_ws_);
  for_elements(s_, B_, [=] __device__(int64_t b) {
    const double a = am[b];
    el[b].exp = (a > 0.0 && isfinite(a)) ? static_cast<int32_t>(ilogb(a)) : 0;
  });
  for_voxels(s_, g_, [=] __device__(int64_t b) { return el[b].exp != 0; },
             [=] __device__(int64_t b, int64_t, int64_t i) { r[i] = times_pow2(r[i], -el[b].exp); });
  field_totals<T>(s_, g_, r_, en, am, nullptr, tot_ws_);
  const uint64_t* nf = nonfin_;
  for_elements(s_, B_, [=] __device__(int64_t b) {
    Elem& e = el[b];
    e.amax = am[b];
    e.r_energy = en[b];
    e.tol = tie_tol<T>(c.tau, e.amax);
    e.nonfinite_in = nf[b];
    e.w_prev = 1;
    e.k = 0;
    e.jump = 1.0;
    e.g3 = 1.0;
    e.wc = d_inf();
    if (nf[b] != 0 && c.check_finite) {
      e.status = kError;
      e.error = kErrNonFinite;
    } else {
      e.status = kActive;
      e.error = kErrNone;
    }
    maskp[kOn * B + b] = e.status == kActive ? 1 : 0;
  });
  double* sx = dsc_ + 7 * B_;
  noise_per_axis(r_, mask(kOn), sx);
  for_elements(s_, B_, [=] __device__(int64_t b) {
    if (maskp[kOn * B + b]) el[b].sigma_x = sx[b];
  });
  EDAB_CUDA(cudaMemsetAsync(Lp_, 0, sizeof(T) * B_ * g_.field, s_));

  for (;;) {
    // step 0: mode start (cpp/src/method/mode.cu:95-136)
    for_elements(s_, B_, [=] __device__(int64_t b) {
      Elem& e = el[b];
      if (e.status != kActive) {
        leave(e, winp, maskp, B, b, e.status);
        return;
      }
      e.r_inf = e.amax;
      for (int a = 0; a < kMaxDim; ++a) e.ext[a] = 0;
      e.fine = 0;
      e.jump = c.absent_jump;
      e.p_odd = 0;
      e.p = 0.0;
      e.cov = 0.0;
      e.wc = d_inf();
      e.g3 = 1.0;
      e.sifting = 1;
      e.n_sifts = 0;
      e.gmax_res_bits = 0;
      e.gmax_h_bits = 0;
      e.on_g2 = 0;
      const int32_t w0 = max(3, e.w_prev + 2);
      int32_t wd, wl;
      tau_windows(c, w0, &wd, &wl);
      for (int k = 0; k < kSlots; ++k) winp[k * B + b] = 0;
      winp[kWd * B + b] = wd;
      winp[kWl * B + b] = wl;
      maskp[kOn * B + b] = 1;
      maskp[kOnG2 * B + b] = 0;
      maskp[kOnFloor * B + b] = e.k >= 1 ? 1 : 0;
      maskp[kOnFine * B + b] = 0;
    });
    noise(r_, (1u << g_.dim) - 1u, mask(kOn), dsc_ + 7 * B_);
    {
      const double* sn = dsc_ + 7 * B_;
      const int32_t* on = mask(kOn);
      for_elements(s_, B_, [=] __device__(int64_t b) {
        if (on[b]) el[b].sigma_n = sn[b];
      });
    }
    // steps 1-2: the window passes
    for (int32_t pass = 0; pass < c_.sig_passes; ++pass) {
      tau_field(mask(kOn), false, tau_);
      for_elements(s_, B_, [=] __device__(int64_t b) {
        if (el[b].status == kActive && el[b].nonfinite) fail2(el[b], winp, maskp, B, b);
      });
      sig_flags<T>(s_, g_, r_, tau_, flags_, el_, mask(kOn));
      const int32_t ps = pass;
      for_elements(s_, B_, [=] __device__(int64_t b) {
        Elem& e = el[b];
        if (e.status != kActive) return;
        const uint64_t N = static_cast<uint64_t>(elem_count(g, b));
        uint64_t S2 = 0;
        bool enough = false;
        for (int a = 0; a < g.dim; ++a) {
          const uint64_t ea = e.ext[a];
          S2 += ea * ea;
          if (ea * static_cast<uint64_t>(elem_n(g, b, a)) >= 3 * N) enough = true;
        }
        for (int a = 0; a < kMaxDim; ++a) e.ext[a] = 0;
        if (!enough) {
          leave(e, winp, maskp, B, b, kDone);
          return;
        }
        const double sp = __ddiv_rn(static_cast<double>(N), __dsqrt_rn(static_cast<double>(S2)));
        const double v = __dmul_rn(__dmul_rn(2.0, c.kappa), sp);
        if (!(v < 1073741824.0)) {
          leave(e, winp, maskp, B, b, kDone);
          return;
        }
        int32_t w = 2 * static_cast<int32_t>(floor((v > 1.0 ? v : 1.0) / 2.0)) + 1;
        w = max(w, 3);
        w = max(w, e.w_prev + 2);
        if (w > (g.len ? elem_len(g, b) : c.n_max)) {
          leave(e, winp, maskp, B, b, kDone);
          return;
        }
        e.spacing = sp;
        int32_t wd, wl;
        tau_windows(c, w, &wd, &wl);
        winp[kWd * B + b] = wd;
        winp[kWl * B + b] = wl;
        if (ps == c.sig_passes - 1) {
          e.w = w;
          const int32_t s0 = max(3, e.w_prev + 2);
          e.on_g2 = (__dmul_rn(c.fine_jump, static_cast<double>(s0)) <= static_cast<double>(w)) ? 1 : 0;
        }
      });
    }
    // step 3: G2 (S1 inside)
    g2();
    bool any_active = false;
    for (const Elem& e : hel_) any_active = any_active || e.status == kActive;
    if (!any_active) break;
    // step 4: the guard, the window (cpp/src/method/mode.cu:189-223)
    for_elements(s_, B_, [=] __device__(int64_t b) {
      Elem& e = el[b];
      if (e.status == kActive && e.nonfinite) {
        fail2(e, winp, maskp, B, b);
        return;
      }
      if (e.status != kActive) return;
      int32_t w = e.w;
      if (e.fine) {
        w = max(max(e.p_odd, e.w_prev + 2), 3);
        e.jump = 1.0;
      }
      if (c.growth > 1.0 && e.k >= c.growth_from) {
        w = max(w, odd_window(__dmul_rn(c.growth, static_cast<double>(e.w_prev))));
        if (w > (g.len ? elem_len(g, b) : c.n_max)) {
          leave(e, winp, maskp, B, b, kDone);
          return;
        }
      }
      e.w = w;
      const int32_t W = odd_window(__dmul_rn(c.beta, static_cast<double>(w)));
      e.W = W;
      winp[kW * B + b] = W;
      if (e.fine) {
        double f = 1.0;
        if (isfinite(e.wc)) {
          const double qq = __dsqrt_rn(__ddiv_rn(e.wc, static_cast<double>(e.p_odd)));
          f = __ddiv_rn(__dmul_rn(c.split, qq), 2.0);
          f = f < 1.0 ? f : 1.0;
        }
        e.g3 = f;
      }
      e.d_min_bits = 0x7ff0000000000000ULL;
      e.d_max_bits = 0;
    });
    // step 5: the scale field, the floor, G3's scaling
    raw_window(flags_, win(kW), mask(kOn), om_, tmp_);
    scale_field();
    local_floor();
    {
      T* L = L_;
      for_voxels(s_, g_, [=] __device__(int64_t b) { return el[b].status == kActive && el[b].fine; },
                 [=] __device__(int64_t b, int64_t, int64_t i) {
                   const T v = mul_rn(static_cast<T>(el[b].g3), L[i]);
                   L[i] = v >= T(3) ? v : T(3);
                 });
    }
    // step 6: orientation and the element build
    orientation_and_build();
    // step 7: the ladders (S4), the weights
    int32_t nrm = 0;
    if (!ladder_and_weights(&nrm)) break;
    // steps 8-9: the sifts
    sifts(nrm);
    // step 10: the commit (S5); the next mode's L_prev is this L
    const bool more = commit();
    std::swap(L_, Lp_);
    if (!more) break;
  }
  // finish: the residue row, the rows scaled back
  {
    const int32_t nl2 = g_.n_last;
    T* rows = rows_;
    for_voxels(s_, g_, [=] __device__(int64_t b) { return el[b].status != kError; },
               [=] __device__(int64_t b, int64_t v, int64_t i) {
                 const int64_t q = pitch_row(g, v);
                 const int64_t t = v - q * g.pitch;
                 rows[(b * c.rows_cap + el[b].n_imfs) * g.count + q * nl2 + t] = r[i];
               });
    const int64_t per = static_cast<int64_t>(c.rows_cap) * g.count;
    for_samples(s_, B_ * per, [=] __device__(int64_t idx) {
      const int64_t b = idx / per;
      const int32_t k = el[b].exp;
      if (k == 0 || el[b].status == kError) return;
      const int64_t at = idx - b * per;
      if (at / g.count > el[b].n_imfs) return;
      if (g.len && at % g.count >= elem_len(g, b)) return;  // beyond the element's length: never written
      const T v = times_pow2(rows[idx], k);
      rows[idx] = v;
      if (!isfinite(v)) el[b].error = kErrNonFiniteResult;
    });
  }
  out.resize(static_cast<size_t>(B_));
  EDAB_CUDA(cudaMemcpyAsync(out.data(), el_, sizeof(Elem) * B_, cudaMemcpyDeviceToHost, s_));
  int32_t tc_err = 0;
  EDAB_CUDA(cudaMemcpyAsync(&tc_err, any_ + kTcErr, sizeof tc_err, cudaMemcpyDeviceToHost, s_));
  EDAB_CUDA(cudaStreamSynchronize(s_));
  if (tc_err) {
    throw CudaError("eda: a tensor-core transform of the orientation gave up waiting for its pipeline",
                    static_cast<int>(cudaErrorLaunchTimeout));
  }
}

// ---------------------------------------------------------------------------------------------
template <class T>
size_t engine_bytes(const Geom& g) {
  const size_t F = static_cast<size_t>(g.batch * g.field);
  const int D = g.dim;
  size_t fields = 11 + 1 + 24 + (D >= 2 ? 2 * D : 0);
  size_t b = fields * F * sizeof(T) + 2 * kMaxRungs * F * sizeof(T) + 9 * F + 4 * F;
  if (D >= 2) b += static_cast<size_t>(orient_work_samples(g)) * sizeof(T);
  b += static_cast<size_t>(g.batch) * (sizeof(Elem) + 4 * (kSlots + kMasks + kMaxRungs) + 8 * 10 + 64);
  b += select_scratch_bytes(g) + totals_scratch_bytes(g);
  b += long_line_scratch_bytes(g, sizeof(T));  // 1-D lines beyond the cube passes' staged capacity
  b += 160 * 256;  // every take is rounded up to 256 bytes
  return b;
}

namespace {
// The long-line scratch of the calling thread for the duration of one engine run.
struct LongLineScratch {
  LongLineScratch(void* p, size_t bytes) { set_long_line_scratch(p, bytes); }
  ~LongLineScratch() { set_long_line_scratch(nullptr, 0); }
};
}  // namespace

template <class T>
void run_chunk(const Geom& g, const Ctl& c, cudaStream_t s, Workspace& ws, const T* x, T* rows, int32_t* hs,
               int32_t* hf, double* hp, double* he, std::vector<Elem>& out, T* orient) {
  Engine<T> e(g, c, s, ws);
  e.orient_out_ = g.dim >= 2 ? orient : nullptr;
  const size_t lb = long_line_scratch_bytes(g, sizeof(T));
  const LongLineScratch scratch(lb ? ws.take<unsigned char>(lb) : nullptr, lb);
  e.run(x, rows, hs, hf, hp, he, out);
}

template size_t engine_bytes<float>(const Geom&);
template size_t engine_bytes<double>(const Geom&);
template void run_chunk<float>(const Geom&, const Ctl&, cudaStream_t, Workspace&, const float*, float*, int32_t*,
                               int32_t*, double*, double*, std::vector<Elem>&, float*);
template void run_chunk<double>(const Geom&, const Ctl&, cudaStream_t, Workspace&, const double*, double*,
                                int32_t*, int32_t*, double*, double*, std::vector<Elem>&, double*);

}  // namespace edab
