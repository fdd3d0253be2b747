// SPDX-License-Identifier: Apache-2.0
// The B200 engine of the sifting hot path: shared types, the padded field layout, canonical
// arithmetic and launch helpers. Every kernel of the engine includes this header.
//
// Arithmetic contract (the reference's, cpp/src/field/common.cuh:5-9): every floating-point
// operation that feeds a result is a round-to-nearest intrinsic in a fixed order, so an element's
// result depends only on its own samples (never on the batch, the launch shape or the order of
// atomics) and the CPU oracle restates it operation by operation. Decisions are integer
// reductions or exact order statistics.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace edab {

constexpr int kMaxDim = 3;
constexpr int kMaxRungs = 32;
constexpr int kMaxG2Rungs = 32;
constexpr int kThreads = 256;
constexpr double kRungRatio = 1.4142135623730951;

// ---------------------------------------------------------------------------------------------
// Errors: every CUDA failure becomes a CudaError carrying the code; argument errors are
// std::invalid_argument; device memory exhaustion is OutOfMemory.
struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& what, int c) : std::runtime_error(what), code(c) {}
};
struct OutOfMemory : std::runtime_error {
  using std::runtime_error::runtime_error;
};
void cuda_fail(cudaError_t e, const char* what, const char* file, int line);
#define EDAB_CUDA(call)                                                   \
  do {                                                                    \
    const cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) ::edab::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)
// Every kernel launch of the engine is followed by EDAB_LAUNCH: it checks the launch and counts it
// for the instrumentation (profile.cu).
void note_launch();
// Runs set(), which sets attributes of kernel `key` on the current device (such as its dynamic
// shared-memory limit: they are per device), on the first call for that kernel and device. Every
// other call, from any host thread, returns only once set() has completed, so no launch can
// overtake the attributes it needs; a set() that throws leaves the kernel to the next call.
void once_on_device(const void* key, const std::function<void()>& set);
#define EDAB_LAUNCH(name)            \
  do {                               \
    ::edab::note_launch();           \
    EDAB_CUDA(cudaGetLastError());   \
  } while (0)

// Instrumentation of the dominant kernel (the cube passes): when enabled, every pass launch is
// bracketed by CUDA events and its CTAs add the pass's algorithmic bytes (every distinct field
// sample read or written once, unpadded) into a device counter.
bool profiling();
unsigned long long* cube_bytes_counter();
void profile_cube_launch(cudaStream_t s, bool begin);

// ---------------------------------------------------------------------------------------------
// The padded field layout of a call: B elements of C-contiguous (n_0, .., n_{D-1}) samples, the
// innermost axis padded to `pitch` (a multiple of 32: every row starts on a 128-byte boundary for
// float, so rows load as whole sectors and as 16-byte vectors). Pad samples are zero and never
// enter a result.
//
// A 1-D batch of uneven lengths (len != nullptr) lays every element out at the longest length
// (n[0], pitch and count are the batch's longest) and gives element b its own length len[b]: every
// kernel reads the element's extent through elem_len / elem_count, so an element's samples from
// len[b] on are pads, and its results are those of a call on that element alone.
struct Geom {
  int32_t dim;
  int32_t n[kMaxDim];       // n[a] = 1 for a >= dim
  int64_t batch;
  int64_t pitch;
  int64_t stride[kMaxDim];  // padded strides inside an element; stride[dim - 1] = 1
  int64_t field;            // padded samples per element
  int64_t count;            // unpadded samples per element
  int64_t rows;             // rows of the innermost axis per element
  int32_t n_max;
  int32_t n_last;            // n[dim - 1] (device code reads this, not n[] at a run-time index)
  uint64_t pitch_inv;        // ceil(2^64 / pitch): v / pitch = umulhi(v, pitch_inv) for 0 <= v < 2^32
  uint64_t field_inv;        // ceil(2^64 / field): i / field = umulhi(i, field_inv) for 0 <= i < 2^64 / field
  int32_t field_fast;        // batch field^2 <= 2^64: every sample index of the batch divides by umulhi
  const int32_t* len;        // 1-D batches of uneven lengths: element lengths (device), else nullptr
  const int32_t* len_host;   // the same lengths in host memory (the host's per-element decisions)
};
Geom make_geom(int dim, int64_t batch, const int64_t* n);

// n[a] and stride[a] for a run-time axis a, by selects: a kernel parameter indexed at a run-time
// index would be copied to local memory.
__host__ __device__ inline int32_t geom_n(const Geom& g, int a) { return a == 0 ? g.n[0] : (a == 1 ? g.n[1] : g.n[2]); }
__host__ __device__ inline int64_t geom_stride(const Geom& g, int a) {
  return a == 0 ? g.stride[0] : (a == 1 ? g.stride[1] : g.stride[2]);
}
// The row and column of in-element offset v (0 <= v < 2^32) without a division on the device:
// umulhi(v, ceil(2^64 / pitch)) is exact since v / 2^64 < 1 / pitch.
__host__ __device__ inline int64_t pitch_row(const Geom& g, int64_t v) {
#ifdef __CUDA_ARCH__
  return static_cast<int64_t>(__umul64hi(static_cast<uint64_t>(v), g.pitch_inv));
#else
  return v / g.pitch;
#endif
}
__host__ __device__ inline int64_t pitch_col(const Geom& g, int64_t v) { return v - pitch_row(g, v) * g.pitch; }
__host__ __device__ inline bool is_pad(const Geom& g, int64_t v) { return pitch_col(g, v) >= g.n_last; }
// The extent of element b along the last axis (its length in 1-D), and its sample count.
__device__ __forceinline__ int32_t elem_len(const Geom& g, int64_t b) { return g.len ? __ldg(g.len + b) : g.n_last; }
__device__ __forceinline__ int64_t elem_count(const Geom& g, int64_t b) { return g.len ? __ldg(g.len + b) : g.count; }
// n[a] of element b (a ragged batch is 1-D: its only axis is the element's length).
__device__ __forceinline__ int32_t elem_n(const Geom& g, int64_t b, int a) {
  return g.len ? __ldg(g.len + b) : (a == 0 ? g.n[0] : (a == 1 ? g.n[1] : g.n[2]));
}
__device__ __forceinline__ bool is_pad_b(const Geom& g, int64_t b, int64_t v) { return pitch_col(g, v) >= elem_len(g, b); }
// Element of sample index i of the batch (i / field without a 64-bit division where exact).
__host__ __device__ inline int64_t elem_of(const Geom& g, int64_t i) {
#ifdef __CUDA_ARCH__
  if (g.field_fast) return static_cast<int64_t>(__umul64hi(static_cast<uint64_t>(i), g.field_inv));
#endif
  return i / g.field;
}
// Coordinate along axis a of padded offset v (v < field < 2^31: the row index fits 32 bits).
__host__ __device__ inline int32_t coord_of(const Geom& g, int64_t v, int a) {
  const int64_t row = pitch_row(g, v);
  if (a == g.dim - 1) return static_cast<int32_t>(v - row * g.pitch);
  const uint32_t r32 = static_cast<uint32_t>(row);
  if (g.dim == 2) return static_cast<int32_t>(r32);  // a == 0: rows are the axis-0 index
  const uint32_t n1 = static_cast<uint32_t>(g.n[1]);  // dim 3: row = x0 n1 + x1
  return static_cast<int32_t>(a == 1 ? r32 % n1 : r32 / n1);
}
// Coordinates of padded offset v; false for a pad.
__host__ __device__ inline bool voxel_coords(const Geom& g, int64_t v, int32_t* x) {
  const int64_t row = pitch_row(g, v);
  const int64_t col = v - row * g.pitch;
  if (col >= g.n_last) return false;
  x[g.dim - 1] = static_cast<int32_t>(col);
  uint32_t q = static_cast<uint32_t>(row);  // row < field < 2^31
  for (int a = g.dim - 2; a >= 1; --a) {
    x[a] = static_cast<int32_t>(q % static_cast<uint32_t>(g.n[a]));
    q /= static_cast<uint32_t>(g.n[a]);
  }
  if (g.dim >= 2) x[0] = static_cast<int32_t>(q);  // the outermost index needs no modulo
  return true;
}

// voxel_coords for a compile-time D (the Geom parameter and x stay in registers).
// nl: the element's extent along the last axis (elem_len).
template <int D>
__device__ __forceinline__ bool voxel_coords_d(const Geom& g, int64_t v, int32_t nl, int32_t* x) {
  const int64_t row = pitch_row(g, v);
  const int64_t col = v - row * g.pitch;
  if (col >= nl) return false;
  x[D - 1] = static_cast<int32_t>(col);
  uint32_t q = static_cast<uint32_t>(row);  // row < field < 2^31
#pragma unroll
  for (int a = D - 2; a >= 1; --a) {
    x[a] = static_cast<int32_t>(q % static_cast<uint32_t>(g.n[a]));
    q /= static_cast<uint32_t>(g.n[a]);
  }
  if constexpr (D >= 2) x[0] = static_cast<int32_t>(q);  // the outermost index needs no modulo
  return true;
}

// ---------------------------------------------------------------------------------------------
// The method's per-call constants (cpp/src/method/common.cpp:14-63 of the reference).
struct Ctl {
  int32_t n_max;
  int64_t count;
  int32_t sifts, u, s, sig_passes, growth_from, anorm_smooth;
  double kappa, beta, c_lo, c_hi, reset, q, span, growth;
  double sig_theta, sig_rho, sig_noise;
  double absent, absent_jump, absent_reach, absent_lo;
  double t0, t1;
  double anorm_floor, ramp_k0, ramp_k1;
  double fine_beta, fine_theta, fine_jump, fine_lo, fine_pop, fine_core, split;
  double tiny;
  double tau;         // relative tie tolerance, rounded to T
  double log_absent;  // log(absent), host C library
  double two_sigma2;  // the band's 2 sigma^2 (host C library)
  double lq;          // log(sqrt 2), host C library (the ladder)
  double sqrt2;       // sqrt(2) correctly rounded
  double powq[48];    // sqrt(2)^j for j = -8 .. 39 (host pow): ladder and G2 rungs, index j + 8
  int32_t max_imf, check_finite, rows_cap;
};
Ctl make_ctl(const Geom& g, bool f32, int32_t sifts, double tau, int32_t max_imf, bool check_finite,
             int32_t rows_cap);
int32_t mode_bound(const Ctl& c);

enum Status : int32_t { kActive = 0, kDone = 1, kError = 3 };
enum ErrCode : int32_t { kErrNone = 0, kErrNonFinite = 1, kErrNonFiniteResult = 2, kErrInternal = 255 };
enum G2Outcome : int32_t { kG2None = 0, kG2Accepted = 1, kG2Stop = 2 };

// Per-element state, device-resident (one per element).
struct alignas(16) Elem {
  int32_t status, error, k, n_imfs;
  int32_t w_prev, w, W, fine;
  int32_t wd, wl;                 // the boxes of the next threshold field
  int32_t exp;                    // prescale exponent
  int32_t p_odd;
  double amax, tol, r_inf, r_energy;
  double sigma_n, sigma_x, spacing, jump, p, cov, wc, g3;
  uint64_t nonfinite_in;          // inf / NaN samples of the input copy
  uint64_t ext[kMaxDim];          // significant extrema per axis
  int32_t nonfinite;              // a non-finite intermediate
  int32_t on_g2;
  // G2's rung machine
  int32_t g2_n, g2_i, g2_pending, g2_done, g2_accepted, g2_acc_index, g2_srung, g2_slot;
  int32_t g2_rungs[kMaxG2Rungs + 1];
  double g2_cand_p, g2_cand_cov;
  int32_t g2_cand_s, g2_res_outcome;
  double g2_res_p, g2_res_cov;
  int64_t g2_res_np;
  int32_t g2_any_core, g2_any_jump;
  // the element and its ladder
  uint64_t d_min_bits, d_max_bits;
  int32_t n_rungs;
  uint32_t rung_pts, rung_used;
  int32_t rung_w[kMaxRungs];
  double rung_lw[kMaxRungs];
  // the sifts
  int32_t sifting, n_sifts;
  uint64_t gmax_res_bits, gmax_h_bits;
  double e_med;
  // selection scratch results
  double sel_out;
  int64_t sel_count;
};

// ---------------------------------------------------------------------------------------------
// Canonical arithmetic (device): round-to-nearest intrinsics, never contracted.
template <class T>
__device__ __forceinline__ T add_rn(T a, T b) {
  if constexpr (std::is_same_v<T, float>) return __fadd_rn(a, b); else return __dadd_rn(a, b);
}
template <class T>
__device__ __forceinline__ T sub_rn(T a, T b) {
  if constexpr (std::is_same_v<T, float>) return __fsub_rn(a, b); else return __dsub_rn(a, b);
}
template <class T>
__device__ __forceinline__ T mul_rn(T a, T b) {
  if constexpr (std::is_same_v<T, float>) return __fmul_rn(a, b); else return __dmul_rn(a, b);
}
template <class T>
__device__ __forceinline__ T div_rn(T a, T b) {
  if constexpr (std::is_same_v<T, float>) return __fdiv_rn(a, b); else return __ddiv_rn(a, b);
}
template <class T>
__device__ __forceinline__ T sqrt_rn(T a) {
  if constexpr (std::is_same_v<T, float>) return __fsqrt_rn(a); else return __dsqrt_rn(a);
}
template <class T>
__device__ __forceinline__ T log_t(T v) {
  if constexpr (std::is_same_v<T, float>) return logf(v); else return log(v);
}
template <class T>
__device__ __forceinline__ T exp_t(T v) {
  if constexpr (std::is_same_v<T, float>) return expf(v); else return exp(v);
}
template <class T>
__device__ __forceinline__ T inf_t() {
  if constexpr (std::is_same_v<T, float>) return __int_as_float(0x7f800000);
  else return __longlong_as_double(0x7ff0000000000000LL);
}
__device__ __forceinline__ double d_inf() { return __longlong_as_double(0x7ff0000000000000LL); }
__device__ __forceinline__ double d_nan() { return __longlong_as_double(0x7ff8000000000000LL); }

// Commutative max / min, bitwise (+0 above -0).
template <class T>
__device__ __forceinline__ T max_c(T a, T b) { return (a > b || (a == b && !signbit(a))) ? a : b; }
template <class T>
__device__ __forceinline__ T min_c(T a, T b) { return (a < b || (a == b && signbit(a))) ? a : b; }
// NumPy's maximum / minimum on non-NaN values: the first operand on ties.
template <class T>
__device__ __forceinline__ T np_max(T a, T b) { return a >= b ? a : b; }
template <class T>
__device__ __forceinline__ T np_min(T a, T b) { return a <= b ? a : b; }
template <class T>
__device__ __forceinline__ T clip(T v, T lo, T hi) { return np_min(np_max(v, lo), hi); }

template <class T>
__device__ __forceinline__ uint64_t abs_bits(T v) {
  return static_cast<uint64_t>(__double_as_longlong(static_cast<double>(v))) & 0x7fffffffffffffffULL;
}
__device__ __forceinline__ double bits_d(uint64_t u) { return __longlong_as_double(static_cast<long long>(u)); }

__host__ __device__ inline int64_t floor_div(int64_t a, int64_t b) {
  const int64_t q = a / b;
  return (a % b != 0 && a < 0) ? q - 1 : q;
}
__host__ __device__ inline int64_t floor_mod(int64_t a, int64_t b) {
  const int64_t m = a % b;
  return m < 0 ? m + b : m;
}
__host__ __device__ inline int32_t reflect_index(int32_t e, int32_t n) {
  return e < 0 ? -e - 1 : (e >= n ? 2 * n - 1 - e : e);
}
__host__ __device__ inline int64_t reflect_any(int64_t i, int64_t n) {
  // within one reflection of the line (every segment point but those of windows longer than the
  // line) without the 64-bit modulo, which the GPU emulates in a long instruction sequence
  if (i >= 0 && i < n) return i;
  if (i < 0 && i >= -n) return -i - 1;
  if (i >= n && i < 2 * n) return 2 * n - 1 - i;
  const int64_t m = floor_mod(i, 2 * n);
  return m < n ? m : 2 * n - 1 - m;
}
__host__ __device__ inline int32_t odd_window(double v) {
  const double u = v > 1.0 ? v : 1.0;
  return 2 * static_cast<int32_t>(floor(u / 2.0)) + 1;
}

// ---------------------------------------------------------------------------------------------
// Launch helpers. Voxel kernels: grid (x over the element's padded field, y over elements).
inline dim3 voxel_grid(const Geom& g, int per_thread = 4) {
  int64_t x = (g.field + static_cast<int64_t>(kThreads) * per_thread - 1) / (static_cast<int64_t>(kThreads) * per_thread);
  x = x < 1 ? 1 : (x > 65535 ? 65535 : x);
  int64_t y = g.batch < 1 ? 1 : (g.batch > 65535 ? 65535 : g.batch);
  return dim3(static_cast<unsigned>(x), static_cast<unsigned>(y));
}
inline unsigned blocks_for(int64_t n, int threads = kThreads) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 0x7fffffffLL) throw std::length_error("edab: launch grid too large");
  return static_cast<unsigned>(b);
}

// Runs f(b, v, i) on every non-pad voxel v of every element b with (run == nullptr || run(b)),
// i = b * field + v.
template <class Run, class F>
__global__ void __launch_bounds__(kThreads) voxel_kernel(Geom g, Run run, F f) {
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    if (!run(b)) continue;
    const int32_t nl = elem_len(g, b);
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      if (pitch_col(g, v) >= nl) continue;
      f(b, v, b * g.field + v);
    }
  }
}
template <class Run, class F>
void for_voxels(cudaStream_t s, const Geom& g, Run run, F f) {
  voxel_kernel<<<voxel_grid(g), kThreads, 0, s>>>(g, run, f);
  EDAB_LAUNCH("voxel_kernel");
}
// Every padded sample (pads included).
template <class F>
__global__ void __launch_bounds__(kThreads) sample_kernel(int64_t total, F f) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    f(i);
  }
}
template <class F>
void for_samples(cudaStream_t s, int64_t total, F f) {
  int64_t blocks = (total + kThreads * 4 - 1) / (kThreads * 4);
  blocks = blocks < 1 ? 1 : (blocks > (1 << 20) ? (1 << 20) : blocks);
  sample_kernel<<<static_cast<unsigned>(blocks), kThreads, 0, s>>>(total, f);
  EDAB_LAUNCH("sample_kernel");
}
template <class F>
__global__ void element_kernel(int64_t B, F f) {
  const int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (b < B) f(b);
}
template <class F>
void for_elements(cudaStream_t s, int64_t B, F f) {
  element_kernel<<<blocks_for(B), kThreads, 0, s>>>(B, f);
  EDAB_LAUNCH("element_kernel");
}

// ---------------------------------------------------------------------------------------------
// Engine entry points (the host driver composes them; each file documents its part).
enum class CubeOp : int8_t { kMax = 0, kMin = 1, kMaxMin = 2, kBox = 3 };

// Pointwise hooks of a cube filter. The first pass of a box cube may read its input from a
// bit field (src_bits: bit `bit` of a u8 field, as 0 / 1); the last pass of a box cube may apply
// an epilogue instead of a plain store.
enum class BoxEpi : int8_t {
  kStore = 0,   // out = box
  kDetSq = 1,   // out = (aux - box)^2 (the detail energy of the threshold field; aux = r)
};
template <class T>
struct CubeArgs {
  const T* in;                // input field (nullptr with src_bits)
  const uint8_t* src_bits;    // box only: the input is bit `bit` of this u8 field
  int32_t bit;
  T* out0;                    // max (or the one output)
  T* out1;                    // min of kMaxMin
  const int32_t* win;         // [rungs * B] odd windows (< 1: skip the element)
  int32_t rungs;              // > 1: rung j reads win + j B and writes out + j * out_stride
  int64_t out_stride;
  BoxEpi epi;
  const T* aux;
};
template <class T>
void cube(cudaStream_t s, const Geom& g, CubeOp op, const CubeArgs<T>& a);
template <class T>
void cube_simple(cudaStream_t s, const Geom& g, CubeOp op, const T* in, T* out0, T* out1, const int32_t* win);
// The launch shape of a cube pass: lines per CTA (1, 2, 4 or 8), line groups per CTA, and the
// segment share from which a window folds whole segments per worker; 0 leaves the default. The
// shapes change no bit of any result (the folds are canonical): tune.cu times them per geometry
// and keeps the fastest (eda_autotune); cube_tune_for returns the recorded shape of a pass, or the
// calling thread's override while tuning.
struct CubeTune {
  int32_t lines = 0, groups = 0, seq_share = 0;
};
CubeTune cube_tune_for(const Geom& g, int axis, size_t es);
void cube_tune_override(const CubeTune* t);  // nullptr: none (per calling thread)

// 1-D lines too long for a pass to stage in shared memory fold in global memory: the calling host
// thread provides a scratch of long_line_scratch_bytes (batch x pitch samples; 0 when the lines
// fit) for the lines' fold input, before its cube calls.
size_t long_line_scratch_bytes(const Geom& g, size_t es);
void set_long_line_scratch(void* p, size_t bytes);

// Canonical reductions: per element sum v^2 (canonical tree) and max|v| of f.
template <class T>
void field_totals(cudaStream_t s, const Geom& g, const T* f, double* energy, double* amax, uint64_t* nonfinite,
                  void* scratch);
size_t totals_scratch_bytes(const Geom& g);

// Selections (exact order statistics, NumPy's median and linear quantile).
enum class SelSrc : int8_t { kField = 0, kDiff = 1 };
template <class T>
struct Sel {
  SelSrc src;
  const T* field;
  const uint8_t* mask;   // kField: (mask & bits) != 0 selects; nullptr: all voxels
  uint8_t bits;
  uint8_t axes;          // kDiff: bit a pools the differences along axis a
  const double* center;  // |value - center[b]| (double) when given
};
size_t select_scratch_bytes(const Geom& g);
// out[b] and count[b] (optional) for the elements with run[b] != 0; q < 0: the median.
template <class T>
void select(cudaStream_t s, const Geom& g, const Sel<T>& sel, double q, const int32_t* run, double* out,
            int64_t* count, void* scratch);

// Significant extrema of every line of every axis into bit a of flags (cleared first for the
// running elements), counts added to el[b].ext[a].
template <class T>
void sig_flags(cudaStream_t s, const Geom& g, const T* r, const T* tau, uint8_t* flags, Elem* el, const int32_t* run);
// Face-connected components of (mask & bits) != 0: labels = the smallest padded index of the
// component, -1 outside.
void ccl(cudaStream_t s, const Geom& g, const uint8_t* mask, uint8_t bits, int32_t* labels, const int32_t* run);

}  // namespace edab
