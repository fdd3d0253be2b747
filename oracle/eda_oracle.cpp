// SPDX-License-Identifier: Apache-2.0
// TEST INFRASTRUCTURE ONLY. The oracle: a CPU restatement of eda-cuda's decomposition (the sifting
// hot path behind eda.decompose), element by element, in the element's own dtype T (float or
// double) with the reference's canonical arithmetic: every operation rounds separately (this file
// is compiled with -ffp-contract=off and without fast-math), in the reference's order of
// operations. It is the checker of the CUDA path (tests/, __graft_entry__.smoke, bench.py's CPU
// baseline) and is never linked into the product library.
//
// Where it follows the reference (paths inside giorgioangel/eda-cuda):
//   constants                 cpp/src/method/common.cpp:14-63 (method_ctl)
//   mode loop, steps 0-10     cpp/src/method/driver.cpp:393-700 (Chunk::start, mode, finish)
//   mode bound, G2 machine    cpp/src/method/driver.cpp:59-140
//   vHGW cube filter          cpp/src/field/vhgw.cu:1-36, cpp/src/method/common.cpp:66-130
//   canonical energies        cpp/src/field/common.cuh:133-259
//   selections (NumPy rules)  cpp/src/method/stats.cu, cpp/src/method/stats_common.cuh:202-270
//   noise levels              cpp/src/method/stats.cu:261-334
//   threshold, extrema, raw   cpp/src/method/stats_fields.cu:25-69, 182-331, 340-369
//   scale field, CCL, floor   cpp/src/method/stats_scale.cu:20-201
//   G2 test, G3 median        cpp/src/method/stats_rungs.cu:14-187
//   mode control, commit      cpp/src/method/mode.cu:27-348
//   sift pointwise, guard     cpp/src/method/sift.cu:25-232
//   element, ladder, weights  cpp/src/method/element.cu:55-370, element.cuh:238-259
//   operators, interpolation  cpp/src/method/element_op.cuh:38-174
//   orientation               cpp/src/method/orientation.cu:1-127, 199-404 (restated with direct
//                             sums of the DCT-II basis instead of cuFFT: rows agree with the
//                             reference within rounding, not bit for bit, in 2-D and 3-D)
//
// The only other departure: log / exp are the host C library's (the reference's kernels call the
// CUDA device functions), so the scale field and the hat weights can differ in the last place;
// decisions match the reference's on stable inputs and rows agree within the stated tolerances.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

namespace oracle {

constexpr int kMaxDim = 3;
constexpr int kMaxRungs = 32;
constexpr int kMaxG2Rungs = 32;
constexpr double kRungRatio = 1.4142135623730951;
constexpr int kM = 2;  // segment points per side of the operators

// ---------------------------------------------------------------------------------------------
// Scalar helpers (cpp/src/field/common.cuh:71-125, cpp/src/method/method.hpp:143-150)

template <class T>
inline T max_c(T a, T b) { return (a > b || (a == b && !std::signbit(a))) ? a : b; }
template <class T>
inline T min_c(T a, T b) { return (a < b || (a == b && std::signbit(a))) ? a : b; }
template <class T>
inline T np_max(T a, T b) { return a >= b ? a : b; }
template <class T>
inline T np_min(T a, T b) { return a <= b ? a : b; }
template <class T>
inline T clip(T v, T lo, T hi) { return np_min(np_max(v, lo), hi); }

inline int64_t floor_div(int64_t a, int64_t b) {
  const int64_t q = a / b;
  return (a % b != 0 && a < 0) ? q - 1 : q;
}
inline int64_t floor_mod(int64_t a, int64_t b) {
  const int64_t m = a % b;
  return m < 0 ? m + b : m;
}
inline int32_t reflect_index(int32_t e, int32_t n) { return e < 0 ? -e - 1 : (e >= n ? 2 * n - 1 - e : e); }
inline int64_t reflect_any(int64_t i, int64_t n) {
  const int64_t m = floor_mod(i, 2 * n);
  return m < n ? m : 2 * n - 1 - m;
}
inline int32_t odd_window(double v) {
  const double u = v > 1.0 ? v : 1.0;
  return 2 * static_cast<int32_t>(std::floor(u / 2.0)) + 1;
}
inline uint64_t dbits(double d) {
  uint64_t u;
  std::memcpy(&u, &d, sizeof u);
  return u;
}
inline double bits_d(uint64_t u) {
  double d;
  std::memcpy(&d, &u, sizeof d);
  return d;
}
template <class T>
inline uint64_t abs_bits(T v) { return dbits(static_cast<double>(v)) & 0x7fffffffffffffffULL; }

template <class T>
inline T log_t(T v) { return std::log(v); }
template <class T>
inline T exp_t(T v) { return std::exp(v); }

// ---------------------------------------------------------------------------------------------
// Geometry of one element: C order (n_0, .., n_{D-1}), unpadded.
struct Shape {
  int dim = 1;
  int32_t n[kMaxDim] = {1, 1, 1};
  int64_t count = 1;
  int64_t st[kMaxDim] = {1, 1, 1};
  int32_t n_max = 1;
  Shape() = default;
  Shape(int d, const int64_t* ext) : dim(d) {
    count = 1;
    for (int a = 0; a < d; ++a) {
      n[a] = static_cast<int32_t>(ext[a]);
      count *= ext[a];
      n_max = std::max(n_max, n[a]);
    }
    int64_t s = 1;
    for (int a = d - 1; a >= 0; --a) {
      st[a] = s;
      s *= n[a];
    }
  }
  int64_t lines(int a) const { return count / n[a]; }
  // base offset of line l along axis a
  int64_t line_base(int a, int64_t l) const {
    const int64_t inner = st[a];
    const int64_t o = l / inner, j = l - o * inner;
    return o * n[a] * inner + j;
  }
  void coords(int64_t i, int32_t* x) const {
    for (int a = dim - 1; a >= 0; --a) {
      x[a] = static_cast<int32_t>(i % n[a]);
      i /= n[a];
    }
  }
};

// ---------------------------------------------------------------------------------------------
// The vHGW pass of one line (cpp/src/field/vhgw.cu:1-36): canonical segment folds.
enum Op { kMax = 0, kMin = 1, kSum = 2 };

template <class T>
inline T apply_op(Op op, T a, T b) {
  return op == kMax ? max_c(a, b) : (op == kMin ? min_c(a, b) : static_cast<T>(a + b));
}

// G of the line (rev: of the reversed line) at every e in [r, n - 1 + r], into g[e - r].
template <class T>
void g_folds(const T* v, int32_t n, int32_t r, int32_t wa, int32_t o, Op op, bool rev, T* g) {
  const auto ext = [&](int32_t e) {
    int32_t i = reflect_index(e, n);
    if (rev) i = n - 1 - i;
    return v[i];
  };
  const int64_t k_lo = floor_div(static_cast<int64_t>(r) - o, wa);
  const int64_t k_hi = floor_div(static_cast<int64_t>(n) - 1 + r - o, wa);
  const int32_t e_max = n - 1 + r;
  for (int64_t k = k_lo; k <= k_hi; ++k) {
    const int32_t s = static_cast<int32_t>(o + k * wa);
    const int32_t e_last = std::min(s + wa - 1, e_max);
    T carry = T(0);
    bool have = false;
    for (int32_t c0 = s; c0 <= e_last; c0 += 32) {
      const int32_t c1 = std::min(c0 + 31, e_last);
      T local = ext(c0);
      if (c0 >= r) g[c0 - r] = have ? apply_op(op, carry, local) : local;
      for (int32_t e = c0 + 1; e <= c1; ++e) {
        local = apply_op(op, local, ext(e));
        if (e >= r) g[e - r] = have ? apply_op(op, carry, local) : local;
      }
      carry = have ? apply_op(op, carry, local) : local;
      have = true;
    }
  }
}

// One line in place: y(x) = op(H(x - r), G(x + r)); box: (H + G) * 0.5 on aligned windows.
template <class T>
void vhgw_line(T* v, int32_t n, int32_t w, Op op, std::vector<T>& gf, std::vector<T>& gr) {
  const int32_t r = std::min((w - 1) / 2, n - 1);
  const int32_t wa = 2 * r + 1;
  const int32_t o = static_cast<int32_t>((static_cast<int64_t>(n) * ((wa + 1) / 2)) % wa);
  gf.resize(n);
  gr.resize(n);
  g_folds(v, n, r, wa, o, op, false, gf.data());
  g_folds(v, n, r, wa, o, op, true, gr.data());
  for (int32_t x = 0; x < n; ++x) {
    const T g = gf[x];                   // G(x + r)
    const T h = gr[(n - 1 - (x - r)) - r];  // H(x - r) = G_rev(n - 1 - (x - r))
    if (op == kSum) {
      const bool aligned = floor_mod(static_cast<int64_t>(x) - r - o, wa) == 0;
      const T s = h + g;
      v[x] = aligned ? static_cast<T>(s * T(0.5)) : s;
    } else {
      v[x] = apply_op(op, h, g);
    }
  }
}

template <class T>
void vhgw_axis(const Shape& sh, int a, int32_t w, Op op, std::vector<T>& f) {
  const int32_t n = sh.n[a];
  const int64_t st = sh.st[a];
  std::vector<T> line(n), gf, gr;
  for (int64_t l = 0; l < sh.lines(a); ++l) {
    const int64_t base = sh.line_base(a, l);
    for (int32_t i = 0; i < n; ++i) line[i] = f[base + i * st];
    vhgw_line<T>(line.data(), n, w, op, gf, gr);
    for (int32_t i = 0; i < n; ++i) f[base + i * st] = line[i];
  }
}

enum CubeOp { kCubeMax = 0, kCubeMin = 1, kCubeBox = 3 };

// The separable cube filter (cpp/src/method/common.cpp:66-130): box along axis 0 first, times
// fl_T(1 / prod of the clamped sides); max / min exact in any order.
template <class T>
std::vector<T> cube(const Shape& sh, CubeOp op, std::vector<T> f, int32_t w) {
  if (op == kCubeBox) {
    for (int a = 0; a < sh.dim; ++a) vhgw_axis<T>(sh, a, w, kSum, f);
    double prod = 1.0;
    const int32_t half = (w - 1) / 2;
    for (int a = 0; a < sh.dim; ++a) prod *= static_cast<double>(2 * std::min(half, sh.n[a] - 1) + 1);
    const T fac = static_cast<T>(1.0 / prod);
    for (T& v : f) v = v * fac;
    return f;
  }
  for (int a = sh.dim - 1; a >= 0; --a) vhgw_axis<T>(sh, a, w, op == kCubeMax ? kMax : kMin, f);
  return f;
}

// ---------------------------------------------------------------------------------------------
// Canonical energies (cpp/src/field/common.cuh:133-259): sum v^2 in double over 32-sample chunks
// of a row, the pairwise tree over the chunks, then the pairwise tree over the rows.
inline double pairwise(std::vector<double> s) {
  size_t m = 1;
  while (m < s.size()) m <<= 1;
  s.resize(std::max<size_t>(m, 1), 0.0);
  for (size_t d = 1; d < s.size(); d <<= 1) {
    for (size_t i = 0; i + d < s.size(); i += 2 * d) s[i] = s[i] + s[i + d];
  }
  return s[0];
}

template <class T>
double field_energy(const Shape& sh, const std::vector<T>& f) {
  const int64_t nl = sh.n[sh.dim - 1];
  std::vector<double> rows;
  std::vector<double> chunks;
  for (int64_t q = 0; q < sh.count / nl; ++q) {
    chunks.clear();
    const T* row = f.data() + q * nl;
    for (int64_t c = 0; c < nl; c += 32) {
      double acc = 0.0;
      for (int64_t e = c; e < std::min(c + 32, nl); ++e) {
        const double d = static_cast<double>(row[e]);
        acc = acc + d * d;
      }
      chunks.push_back(acc);
    }
    rows.push_back(pairwise(chunks));
  }
  return pairwise(rows);
}

template <class T>
double amax_of(const std::vector<T>& f) {
  uint64_t m = 0;
  for (T v : f) m = std::max(m, abs_bits(v));
  return bits_d(m);
}

// ---------------------------------------------------------------------------------------------
// Exact selections (cpp/src/method/stats.cu, stats_common.cuh:202-270)
inline uint64_t sel_key(double d) {
  uint64_t u = dbits(d);
  if ((u << 1) == 0) u = 0;
  return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}
inline double sel_value(uint64_t k) {
  const uint64_t u = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
  return bits_d(u);
}

inline void quantile_index(int64_t n, double q, int64_t* i, int64_t* j, double* gamma) {
  const double v = static_cast<double>(n - 1) * q;
  if (v >= static_cast<double>(n - 1)) {
    *i = *j = n - 1;
    *gamma = v + 1.0;
  } else if (v < 0.0) {
    *i = *j = 0;
    *gamma = v;
  } else {
    const double f = std::floor(v);
    *i = static_cast<int64_t>(f);
    *j = *i + 1;
    *gamma = v - f;
  }
}
inline double quantile_linear(double a, double b, double gamma) {
  const double diff = b - a;
  return gamma >= 0.5 ? b - diff * (1.0 - gamma) : a + diff * gamma;
}

// median (NaN for an empty set) and linear quantile of the doubles in v (reordered).
inline double select_median(std::vector<double>& v) {
  const int64_t n = static_cast<int64_t>(v.size());
  if (n == 0) return std::numeric_limits<double>::quiet_NaN();
  std::vector<uint64_t> k(v.size());
  for (size_t i = 0; i < v.size(); ++i) k[i] = sel_key(v[i]);
  const size_t r0 = static_cast<size_t>((n - 1) / 2), r1 = static_cast<size_t>(n / 2);
  std::nth_element(k.begin(), k.begin() + r0, k.end());
  const double a = sel_value(k[r0]);
  if (n % 2) return a;
  const uint64_t kb = *std::min_element(k.begin() + r1, k.end());
  return (a + sel_value(kb)) / 2.0;
}
inline double select_quantile(std::vector<double>& v, double q) {
  const int64_t n = static_cast<int64_t>(v.size());
  if (n == 0) return std::numeric_limits<double>::quiet_NaN();
  std::vector<uint64_t> k(v.size());
  for (size_t i = 0; i < v.size(); ++i) k[i] = sel_key(v[i]);
  std::sort(k.begin(), k.end());
  int64_t i = 0, j = 0;
  double g = 0.0;
  quantile_index(n, q, &i, &j, &g);
  return quantile_linear(sel_value(k[static_cast<size_t>(i)]), sel_value(k[static_cast<size_t>(j)]), g);
}

// ---------------------------------------------------------------------------------------------
// The method's constants (cpp/src/method/common.cpp:14-63)
struct Ctl {
  int32_t n_max;
  int64_t count;
  int32_t sifts = 3, u = 2, s = 1, sig_passes = 2, growth_from = 2, anorm_smooth = 1;
  double kappa = 1.0, beta = 2.0, c_lo = 1.5, c_hi = 2.0, reset = 2.0, q = 4.0, span = 1.0, growth = 2.0;
  double sig_theta = 0.3, sig_rho = 2.0, sig_noise = 1.0;
  double absent = 3.0, absent_jump = 2.0, absent_reach = 1.0, absent_lo = 1.2;
  double t0 = 0.2, t1 = 0.5;
  double anorm_floor = 0.1, ramp_k0 = 0.3, ramp_k1 = 0.6;
  double fine_beta = 2.0, fine_theta = 1.0, fine_jump = 2.0, fine_lo = 1.5, fine_pop = 0.25, fine_core = 2.0,
         split = 1.0;
  double tiny;
};

// The largest mode count (cpp/src/method/driver.cpp:128-140).
inline int32_t mode_bound(const Ctl& c) {
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

// G2's candidate rungs (cpp/src/method/driver.cpp:59-71)
inline std::vector<int32_t> g2_candidate_rungs(int32_t w, int32_t w_prev, double jump) {
  const int32_t s0 = std::max(3, w_prev + 2);
  std::vector<int32_t> out;
  for (int32_t j = 0;; ++j) {
    const int32_t s = odd_window(static_cast<double>(s0) * std::pow(kRungRatio, static_cast<double>(j)));
    if (static_cast<double>(s) * jump > static_cast<double>(w)) break;
    if (out.empty() || s != out.back()) out.push_back(s);
    if (static_cast<int32_t>(out.size()) > kMaxG2Rungs) throw std::length_error("oracle: too many G2 rungs");
  }
  return out;
}

// The ladder (cpp/src/method/element.cu:343-370)
inline std::vector<int32_t> rung_ladder(double d_min, double d_max, int32_t w, int32_t n_max) {
  if (!(std::isfinite(d_min) && std::isfinite(d_max)) || w < 1 || n_max < 1) {
    throw std::invalid_argument("oracle: rung_ladder arguments");
  }
  volatile double qv = kRungRatio;
  const double q = qv;
  const double lq = std::log(q);
  const double wd = static_cast<double>(w);
  const double jl = std::floor(std::log((d_min > 1.0 ? d_min : 1.0) / wd) / lq + 1e-9);
  const double jh = std::ceil(std::log((d_max > 1.0 ? d_max : 1.0) / wd) / lq - 1e-9);
  if (!(jh - jl <= 4096.0)) throw std::length_error("oracle: ladder span");
  const int64_t cap = 2 * static_cast<int64_t>(n_max) + 1;
  std::set<int64_t> sides;
  for (int64_t j = static_cast<int64_t>(jl); j <= static_cast<int64_t>(jh); ++j) {
    const double v = wd * std::pow(q, static_cast<double>(j));
    const int64_t side = v >= static_cast<double>(cap) + 1.0 ? cap : std::min<int64_t>(odd_window(v), cap);
    sides.insert(side);
  }
  if (sides.size() > static_cast<size_t>(kMaxRungs)) throw std::length_error("oracle: ladder too long");
  return std::vector<int32_t>(sides.begin(), sides.end());
}

// ---------------------------------------------------------------------------------------------
// The per-element method.
enum G2Outcome { kG2None = 0, kG2Accepted = 1, kG2Stop = 2 };
struct G2Result {
  int32_t outcome = kG2None;
  int32_t s = 0;
  int64_t n_p = 0;
  double p = 0.0, cov = 0.0;
};

struct Result {
  int32_t n_imfs = 0, error = 0, exp = 0;
  std::vector<int32_t> windows, sifts;
  std::vector<double> spacing, energy;
};

// The energy tensor T = R1 R1^T + R2 R2^T in T and its Jacobi eigen-decomposition in double
// (cpp/src/method/element.cu:49-164): nf[a] the top eigenvector, coh = (mu1 - mu2) / (mu1 + mu2)
// clipped to [0, 1]; *nonfinite set when a tensor entry is not finite.
template <class T>
void orientation_eigen(int D, int64_t N, const std::vector<T>* R1, const std::vector<T>* R2, std::vector<T>* nf,
                       std::vector<T>& coh, bool* nonfinite) {
  const auto pair = [D](int a, int b) {
    if (a > b) std::swap(a, b);
    return D == 2 ? (a == 0 ? b : 2) : (a == 0 ? b : (a == 1 ? 2 + b : 5));
  };
  for (int a = 0; a < D; ++a) nf[a].assign(static_cast<size_t>(N), T(0));
  coh.assign(static_cast<size_t>(N), T(0));
  for (int64_t i = 0; i < N; ++i) {
    // the tensor in T: v = R1_a R1_c, then + h(a, k) h(k, c) for k = 0..D-1
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    bool finite = true;
    for (int a = 0; a < D; ++a) {
      for (int c = a; c < D; ++c) {
        T v = R1[a][i] * R1[c][i];
        for (int k = 0; k < D; ++k) v = v + static_cast<T>(R2[pair(a, k)][i] * R2[pair(k, c)][i]);
        A[a][c] = A[c][a] = static_cast<double>(v);
        finite = finite && std::isfinite(A[a][c]);
      }
    }
    if (!finite) *nonfinite = true;
    // Jacobi (element.cu:49-164): one rotation in 2-D; 6 cyclic sweeps after a power-of-two
    // prescale in 3-D
    const auto rotate = [&](int pp, int q, int rr, int dim) {
      const double apq = A[pp][q];
      if (apq == 0.0) return;
      const double theta = (A[q][q] - A[pp][pp]) / (2.0 * apq);
      const double at = std::fabs(theta);
      const double t = std::copysign(1.0, theta) / (at + std::sqrt(theta * theta + 1.0));
      const double cc = 1.0 / std::sqrt(t * t + 1.0);
      const double s = t * cc;
      const double tau = s / (1.0 + cc);
      const double tapq = t * apq;
      A[pp][pp] = A[pp][pp] - tapq;
      A[q][q] = A[q][q] + tapq;
      A[pp][q] = A[q][pp] = 0.0;
      if (rr >= 0) {
        const double gg = A[rr][pp], hh = A[rr][q];
        const double np_ = gg - s * (hh + gg * tau);
        const double nq_ = hh + s * (gg - hh * tau);
        A[rr][pp] = A[pp][rr] = np_;
        A[rr][q] = A[q][rr] = nq_;
      }
      for (int k = 0; k < dim; ++k) {
        const double gg = V[k][pp], hh = V[k][q];
        V[k][pp] = gg - s * (hh + gg * tau);
        V[k][q] = hh + s * (gg - hh * tau);
      }
    };
    if (D == 2) {
      rotate(0, 1, -1, 2);
    } else {
      double am = 0.0;
      for (int a = 0; a < 3; ++a) {
        for (int c = a; c < 3; ++c) am = std::fmax(am, std::fabs(A[a][c]));
      }
      if (am > 0.0 && am < INFINITY) {
        const double sc = std::scalbn(1.0, -std::ilogb(am));
        for (int a = 0; a < 3; ++a) {
          for (int c = 0; c < 3; ++c) A[a][c] = A[a][c] * sc;
        }
      }
      for (int sweep = 0; sweep < 6; ++sweep) {
        rotate(0, 1, 2, 3);
        rotate(0, 2, 1, 3);
        rotate(1, 2, 0, 3);
      }
    }
    double mu[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < D; ++a) mu[a] = A[a][a];
    int top = 0;
    for (int a = 1; a < D; ++a) top = mu[a] > mu[top] ? a : top;
    double mu2 = -INFINITY;
    for (int a = 0; a < D; ++a) mu2 = (a != top && mu[a] > mu2) ? mu[a] : mu2;
    const double mu1 = mu[top];
    const double ssum = mu1 + mu2;
    double cv = ssum > 0.0 ? (mu1 - mu2) / ssum : 0.0;
    cv = cv < 0.0 ? 0.0 : (cv > 1.0 ? 1.0 : cv);
    coh[i] = static_cast<T>(cv);
    for (int a = 0; a < D; ++a) nf[a][i] = static_cast<T>(V[a][top]);
  }
}

template <class T>
void extrema_flags(const Shape& sh, const std::vector<T>& r, const std::vector<T>& tau, std::vector<uint8_t>& flags,
                   uint64_t* ext);

template <class T>
class Element {
 public:
  Element(const Shape& sh, const Ctl& c, double tau_rel, bool check_finite, int32_t max_imf, int32_t cap)
      : sh_(sh), c_(c), tau_(static_cast<double>(static_cast<T>(tau_rel))), check_finite_(check_finite),
        max_imf_(max_imf), cap_(cap) {}

  // Runs the decomposition of x (count samples) into rows (cap x count): IMFs, then the residue.
  Result run(const T* x, T* rows);
  // With return_orientation: rows (cap - 1, D + 1, count) receive n (canonical sign) and c of every
  // mode at the row of its IMF (cpp/src/method/driver.cpp:553-559; orientation.cu:495-522).
  void keep_orientation(T* orient) { orient_ = orient; }

 private:
  using F = std::vector<T>;
  const Shape sh_;
  const Ctl c_;
  const double tau_;
  const bool check_finite_;
  const int32_t max_imf_, cap_;
  T* orient_ = nullptr;
  // per-element record (cpp/src/method/method.hpp:94-132)
  int32_t k_ = 0, w_prev_ = 1, w_ = 0, W_ = 0, fine_ = 0, p_odd_ = 0, n_rungs_ = 0, n_sifts_ = 0;
  uint64_t ext_[kMaxDim] = {0, 0, 0};
  double tol_ = 0, r_inf_ = 0, sigma_n_ = 0, sigma_x_ = 0, jump_ = 1.0, spacing_ = 0, p_ = 0, wc_ = INFINITY,
         g3_ = 1.0;
  bool nonfinite_ = false;
  uint32_t rung_pts_ = 0, rung_used_ = 0;
  std::vector<int32_t> rung_w_;
  double amax_ = 0;
  // the element
  std::vector<uint8_t> lo_;
  F t_;
  F o_[kMaxDim];

  double noise_sigma(const F& r, bool per_axis) const;
  void tau_field(const F& r, int32_t wd, int32_t wl, const double* floor2, F& tau);
  void sig_flags(const F& r, const F& tau, std::vector<uint8_t>& flags, uint64_t* ext) const;
  F raw_window(const std::vector<uint8_t>& flags, int32_t win) const;
  bool rice(int pass, int32_t* wd, int32_t* wl);
  G2Result g2_test(const std::vector<uint8_t>& ff, int32_t s, std::vector<uint8_t>& P) const;
  double g3_coarse(const std::vector<uint8_t>& ff, const std::vector<uint8_t>& P) const;
  void scale_field(const F& om, std::vector<uint8_t>& A, F& L) const;
  void local_floor(const F& L_prev, const std::vector<uint8_t>& A, F& L) const;
  void orientation(const F& r, F* n, F& coh);
  void element_build(const F& L, const F& coh, const F* n, double* d_min, double* d_max);
  void element_weights(const F& L, const F& coh);
  F op(int which, const F& in, F* out1) const;  // 0 Dil, 2 Dil+Ero, 3 Avg
  void envelope_mean(const F& h, F& m, F& u, F& l) const;
};

template <class T>
double Element<T>::noise_sigma(const F& r, bool per_axis) const {
  // cpp/src/method/stats.cu:299-334: median of the forward differences (in T), the MAD, 1.4826 MAD / sqrt 2
  const double sqrt2 = std::sqrt(2.0);
  const auto level = [&](unsigned axes) {
    std::vector<double> d;
    for (int a = 0; a < sh_.dim; ++a) {
      if (!((axes >> a) & 1u)) continue;
      const int64_t st = sh_.st[a];
      for (int64_t i = 0; i < sh_.count; ++i) {
        int32_t x[kMaxDim];
        sh_.coords(i, x);
        if (x[a] >= sh_.n[a] - 1) continue;
        d.push_back(static_cast<double>(static_cast<T>(r[i + st] - r[i])));
      }
    }
    std::vector<double> dd = d;
    const double center = select_median(dd);
    for (double& v : d) v = std::fabs(v - center);
    const double mad = select_median(d);
    return (1.4826 * mad) / sqrt2;
  };
  if (!per_axis) return level((1u << sh_.dim) - 1u);
  double acc = 0.0;
  for (int a = 0; a < sh_.dim; ++a) {
    if (sh_.n[a] < 2) continue;
    const double v = level(1u << a);
    if (v > acc) acc = v;
  }
  return acc;
}

template <class T>
void Element<T>::tau_field(const F& r, int32_t wd, int32_t wl, const double* floor2, F& tau) {
  // cpp/src/method/stats_fields.cu:25-69, 375-389
  const F box = cube<T>(sh_, kCubeBox, r, wd);
  F e(r.size());
  for (int64_t i = 0; i < sh_.count; ++i) {
    const T det = r[i] - box[i];
    e[i] = det * det;
  }
  e = cube<T>(sh_, kCubeBox, e, wl);
  tau.resize(r.size());
  const double f = c_.sig_noise * sigma_n_;
  const double fl = f > 0.0 ? f : 0.0;
  for (int64_t i = 0; i < sh_.count; ++i) {
    const T be = e[i];
    if (!(std::isfinite(be) && std::isfinite(sigma_n_))) nonfinite_ = true;
    const T lev = std::sqrt(be > T(0) ? be : T(0));
    const double ld = static_cast<double>(lev);
    double t = c_.sig_theta * (ld > fl ? ld : fl);
    t = t > tol_ ? t : tol_;
    if (floor2) t = t > *floor2 ? t : *floor2;
    tau[i] = static_cast<T>(t);
  }
}

// fl64(a - b) >= tau (cpp/src/method/stats_fields.cu:182-205)
template <class T>
inline bool deep(T a, T b, T tau) {
  if constexpr (std::is_same_v<T, float>) {
    const float d = a - b;
    if (d != tau) return d > tau;
    return static_cast<double>(a) - static_cast<double>(b) >= static_cast<double>(tau);
  } else {
    return a - b >= tau;
  }
}

template <class T>
void Element<T>::sig_flags(const F& r, const F& tau, std::vector<uint8_t>& flags, uint64_t* ext) const {
  extrema_flags<T>(sh_, r, tau, flags, ext);
}

template <class T>
void extrema_flags(const Shape& sh_, const std::vector<T>& r, const std::vector<T>& tau, std::vector<uint8_t>& flags,
                   uint64_t* ext) {
  // scipy.signal.find_peaks + peak_prominences >= tau on every line of every axis
  // (cpp/src/method/stats_fields.cu:1-14, 207-331)
  flags.assign(static_cast<size_t>(sh_.count), 0);
  for (int a = 0; a < sh_.dim; ++a) {
    const int32_t n = sh_.n[a];
    if (n < 3) continue;
    const int64_t st = sh_.st[a];
    uint64_t count = 0;
    for (int64_t l = 0; l < sh_.lines(a); ++l) {
      const int64_t base = sh_.line_base(a, l);
      const auto X = [&](int32_t k) { return r[base + k * st]; };
      for (int32_t s = 1; s <= n - 2; ++s) {
        const T cur = X(s), prev = X(s - 1);
        if (!(prev < cur || prev > cur)) continue;
        int32_t e = s;
        while (e + 1 < n && X(e + 1) == cur) ++e;
        if (e > n - 2) continue;
        const T nxt = X(e + 1);
        const bool is_max = prev < cur && nxt < cur;
        const bool is_min = prev > cur && nxt > cur;
        if (!is_max && !is_min) continue;
        const int32_t p = (s + e) / 2;
        const T tp = tau[base + p * st];
        const auto side = [&](int dir) {
          for (int32_t k = p + dir; k >= 0 && k < n; k += dir) {
            const T u = X(k);
            if (is_max ? !(u <= cur) : !(u >= cur)) return false;
            if (is_max ? deep<T>(cur, u, tp) : deep<T>(u, cur, tp)) return true;
          }
          return false;
        };
        if (side(-1) && side(1)) {
          flags[base + p * st] |= static_cast<uint8_t>(1u << a);
          ++count;
        }
      }
    }
    ext[a] += count;
  }
}

template <class T>
typename Element<T>::F Element<T>::raw_window(const std::vector<uint8_t>& flags, int32_t win) const {
  // cpp/src/method/stats_fields.cu:340-369, 425-440
  F om(static_cast<size_t>(sh_.count));
  const T two_kappa = static_cast<T>(2.0 * c_.kappa);
  const T tiny = static_cast<T>(c_.tiny);
  for (int a = 0; a < sh_.dim; ++a) {
    F f(static_cast<size_t>(sh_.count));
    for (int64_t i = 0; i < sh_.count; ++i) f[i] = ((flags[i] >> a) & 1u) ? T(1) : T(0);
    f = cube<T>(sh_, kCubeBox, f, win);
    for (int64_t i = 0; i < sh_.count; ++i) {
      const T sq = f[i] * f[i];
      om[i] = a == 0 ? sq : static_cast<T>(om[i] + sq);
    }
  }
  for (int64_t i = 0; i < sh_.count; ++i) {
    const T dens = std::sqrt(om[i]);
    om[i] = dens > T(0) ? static_cast<T>(two_kappa / (dens > tiny ? dens : tiny)) : std::numeric_limits<T>::infinity();
  }
  return om;
}

// The window rule of one pass (cpp/src/method/mode.cu:138-187); false: the element is done.
template <class T>
bool Element<T>::rice(int pass, int32_t* wd, int32_t* wl) {
  const uint64_t N = static_cast<uint64_t>(sh_.count);
  uint64_t S2 = 0;
  bool enough = false;
  for (int a = 0; a < sh_.dim; ++a) {
    const uint64_t ea = ext_[a];
    S2 += ea * ea;
    if (ea * static_cast<uint64_t>(sh_.n[a]) >= 3 * N) enough = true;
  }
  for (int a = 0; a < kMaxDim; ++a) ext_[a] = 0;
  if (!enough) return false;
  const double sp = static_cast<double>(N) / std::sqrt(static_cast<double>(S2));
  const double v = (2.0 * c_.kappa) * sp;
  if (!(v < 1073741824.0)) return false;
  int32_t w = 2 * static_cast<int32_t>(std::floor((v > 1.0 ? v : 1.0) / 2.0)) + 1;
  w = std::max(w, 3);
  w = std::max(w, w_prev_ + 2);
  if (w > c_.n_max) return false;
  spacing_ = sp;
  *wd = odd_window(c_.sig_rho * static_cast<double>(w));
  *wl = odd_window(std::max(c_.beta, c_.sig_rho) * static_cast<double>(w));
  if (pass == c_.sig_passes - 1) w_ = w;
  return true;
}

template <class T>
G2Result Element<T>::g2_test(const std::vector<uint8_t>& ff, int32_t s, std::vector<uint8_t>& P) const {
  // cpp/src/method/stats_rungs.cu:14-87, 127-159
  const double sd = static_cast<double>(s);
  const int32_t wb = odd_window(c_.fine_beta * sd);
  const int32_t wcore = odd_window(c_.fine_core * sd);
  const int32_t wr = odd_window((2.0 * c_.absent_reach) * static_cast<double>(wb));
  const F om = raw_window(ff, wb);
  P.assign(static_cast<size_t>(sh_.count), 0);
  F t1(static_cast<size_t>(sh_.count));
  std::vector<double> pop;
  for (int64_t i = 0; i < sh_.count; ++i) {
    const bool in = static_cast<double>(om[i]) < c_.fine_lo * sd;
    P[i] = in ? 1 : 0;
    t1[i] = in ? T(1) : T(0);
    if (in) pop.push_back(static_cast<double>(om[i]));
  }
  const F core = cube<T>(sh_, kCubeMin, t1, wcore);
  bool any_core = false;
  for (int64_t i = 0; i < sh_.count; ++i) any_core = any_core || core[i] > T(0.5);
  G2Result res;
  res.s = s;
  res.n_p = static_cast<int64_t>(pop.size());
  res.p = select_quantile(pop, c_.fine_pop);
  res.cov = static_cast<double>(res.n_p) / static_cast<double>(c_.count);
  const F dil = cube<T>(sh_, kCubeMax, t1, wr);
  bool any_jump = false;
  for (int64_t i = 0; i < sh_.count; ++i) {
    any_jump = any_jump || (static_cast<double>(om[i]) > c_.reset * res.p && dil[i] > T(0.5));
  }
  if (res.n_p == 0 || !any_core) {
    res.outcome = kG2None;
  } else if (c_.fine_jump * res.p > static_cast<double>(w_)) {
    res.outcome = kG2Stop;
  } else {
    res.outcome = any_jump ? kG2Accepted : kG2None;
  }
  return res;
}

template <class T>
double Element<T>::g3_coarse(const std::vector<uint8_t>& ff, const std::vector<uint8_t>& P) const {
  // cpp/src/method/stats_rungs.cu:89-121, 161-187
  const int32_t wcw = odd_window(c_.beta * static_cast<double>(w_));
  const int32_t wf = odd_window(c_.fine_beta * static_cast<double>(p_odd_));
  const int32_t wr = odd_window((2.0 * c_.absent_reach) * static_cast<double>(wf));
  const F omc = raw_window(ff, wcw);
  F t1(static_cast<size_t>(sh_.count));
  for (int64_t i = 0; i < sh_.count; ++i) t1[i] = (P[i] & 1u) ? T(1) : T(0);
  const F dil = cube<T>(sh_, kCubeMax, t1, wr);
  std::vector<double> sel;
  for (int64_t i = 0; i < sh_.count; ++i) {
    if (dil[i] < T(0.5) && omc[i] < std::numeric_limits<T>::infinity()) sel.push_back(static_cast<double>(omc[i]));
  }
  if (sel.empty()) return INFINITY;
  return select_median(sel);
}

// Face-connected components of mask != 0: the label is the smallest index of the component.
inline std::vector<int64_t> components(const Shape& sh, const std::vector<uint8_t>& mask) {
  std::vector<int64_t> lab(static_cast<size_t>(sh.count), -1);
  std::vector<int64_t> stack;
  for (int64_t i = 0; i < sh.count; ++i) {
    if (!mask[i] || lab[i] >= 0) continue;
    lab[i] = i;  // i is the smallest index of its component (every smaller member would have claimed it)
    stack.push_back(i);
    while (!stack.empty()) {
      const int64_t v = stack.back();
      stack.pop_back();
      int32_t x[kMaxDim];
      sh.coords(v, x);
      for (int a = 0; a < sh.dim; ++a) {
        for (int dir = -1; dir <= 1; dir += 2) {
          const int32_t y = x[a] + dir;
          if (y < 0 || y >= sh.n[a]) continue;
          const int64_t u = v + dir * sh.st[a];
          if (mask[u] && lab[u] < 0) {
            lab[u] = i;
            stack.push_back(u);
          }
        }
      }
    }
  }
  return lab;
}

template <class T>
void Element<T>::scale_field(const F& om, std::vector<uint8_t>& A, F& L) const {
  // cpp/src/method/stats_scale.cu:85-167, 222-246
  const int32_t w_near = odd_window((2.0 * c_.absent_reach) * static_cast<double>(W_));
  const double w = static_cast<double>(w_);
  F fine(static_cast<size_t>(sh_.count));
  A.assign(static_cast<size_t>(sh_.count), 0);
  std::vector<uint8_t> aw(static_cast<size_t>(sh_.count));
  for (int64_t i = 0; i < sh_.count; ++i) {
    const double o = static_cast<double>(om[i]);
    const bool a0 = o > c_.reset * w;
    const bool awb = o > c_.absent_lo * w;
    const bool fn = o < (c_.absent_lo * w) / jump_;
    A[i] = static_cast<uint8_t>((a0 ? 4u : 0u) | (awb ? 2u : 0u));
    aw[i] = awb ? 1 : 0;
    fine[i] = fn ? T(1) : T(0);
  }
  const F near = cube<T>(sh_, kCubeMax, fine, w_near);
  const std::vector<int64_t> lab = components(sh_, aw);
  std::vector<uint8_t> marks(static_cast<size_t>(sh_.count), 0);
  for (int64_t i = 0; i < sh_.count; ++i) {
    if ((A[i] & 2u) && near[i] > T(0.5)) marks[lab[i]] = 1;
  }
  L.resize(static_cast<size_t>(sh_.count));
  for (int64_t i = 0; i < sh_.count; ++i) {
    const bool a = (A[i] & 4u) && lab[i] >= 0 && marks[lab[i]];
    A[i] = a ? 1 : 0;
    double v;
    if (a) {
      v = c_.absent;
    } else {
      const double o = static_cast<double>(om[i]);
      const double ow = o > c_.reset * w ? w : o;
      const double lo = w / c_.c_lo;
      const double hi = c_.c_hi * w;
      v = ow > lo ? ow : lo;
      v = v < hi ? v : hi;
    }
    L[i] = log_t<T>(static_cast<T>(v));
  }
  L = cube<T>(sh_, kCubeBox, L, W_);
  for (T& v : L) v = exp_t<T>(v);
}

template <class T>
void Element<T>::local_floor(const F& L_prev, const std::vector<uint8_t>& A, F& L) const {
  // cpp/src/method/stats_scale.cu:169-201, 249-268
  F chi(static_cast<size_t>(sh_.count));
  for (int64_t i = 0; i < sh_.count; ++i) chi[i] = (A[i] & 1u) ? T(1) : T(0);
  chi = cube<T>(sh_, kCubeBox, chi, W_);
  const double log_absent = std::log(c_.absent);
  const bool grow = c_.growth > 1.0 && k_ >= c_.growth_from;
  const T cap = static_cast<T>(c_.c_hi * static_cast<double>(w_));
  for (int64_t i = 0; i < sh_.count; ++i) {
    const T lp = L_prev[i];
    T fl = grow ? static_cast<T>(static_cast<T>(c_.growth) * lp) : static_cast<T>(lp + T(2));
    fl = fl < cap ? fl : cap;
    const T x = chi[i];
    const T e = static_cast<T>(static_cast<T>((T(1) - x) * log_t<T>(fl)) + static_cast<T>(x * static_cast<T>(log_absent)));
    const T f = exp_t<T>(e);
    L[i] = L[i] >= f ? L[i] : f;
  }
}

// ---------------------------------------------------------------------------------------------
// The orientation (cpp/src/method/orientation.cu:1-37, 98-127, 199-404; element.cu:55-164), with
// the DCT-II and its inverses as direct sums over the basis (in double).
template <class T>
void Element<T>::orientation(const F& r, F* nf, F& coh) {
  const int D = sh_.dim;
  const int64_t N = sh_.count;
  // mean in double
  double mean = 0.0;
  for (int64_t i = 0; i < N; ++i) mean += static_cast<double>(r[i]);
  mean = mean / static_cast<double>(N);
  std::vector<double> X(static_cast<size_t>(N));
  for (int64_t i = 0; i < N; ++i) X[i] = static_cast<double>(static_cast<T>(static_cast<double>(r[i]) - mean));
  // the per-axis matrices: kind 0 forward (row k, column x), 1 inverse cos (row x, column k), 2
  // inverse sin (row x, column k)
  const auto axis_matrix = [](int64_t n, int kind) {
    std::vector<double> m(static_cast<size_t>(n * n));
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int64_t i = 0; i < n; ++i) {
      for (int64_t j = 0; j < n; ++j) {
        const int64_t k = kind == 0 ? i : j, x = kind == 0 ? j : i;
        const long double c = std::sqrt((k ? 2.0L : 1.0L) / static_cast<long double>(n));
        const int64_t q = (k * (2 * x + 1)) % (4 * n);
        const long double ang = pi * static_cast<long double>(q) / static_cast<long double>(2 * n);
        m[static_cast<size_t>(i * n + j)] = static_cast<double>(c * (kind == 2 ? std::sin(ang) : std::cos(ang)));
      }
    }
    return m;
  };
  std::vector<double> M[kMaxDim][3];
  for (int a = 0; a < D; ++a) {
    for (int k = 0; k < 3; ++k) M[a][k] = axis_matrix(sh_.n[a], k);
  }
  const auto apply_axis = [&](int a, const std::vector<double>& m, std::vector<double>& f) {
    const int64_t n = sh_.n[a], st = sh_.st[a];
    std::vector<double> line(static_cast<size_t>(n));
    for (int64_t l = 0; l < sh_.lines(a); ++l) {
      const int64_t base = sh_.line_base(a, l);
      for (int64_t i = 0; i < n; ++i) line[i] = f[base + i * st];
      for (int64_t i = 0; i < n; ++i) {
        double acc = 0.0;
        const double* row = &m[static_cast<size_t>(i * n)];
        for (int64_t j = 0; j < n; ++j) acc += row[j] * line[j];
        f[base + i * st] = acc;
      }
    }
  };
  for (int a = 0; a < D; ++a) apply_axis(a, M[a][0], X);
  // the band (rounded to T, as the reference stores the spectrum in T)
  const double l2 = std::log(2.0);
  const double sg = l2 / (2.0 * std::sqrt(2.0 * l2));
  const double two_sigma2 = 2.0 * (sg * sg);
  std::vector<double> uk(static_cast<size_t>(D * N)), rad(static_cast<size_t>(N));
  for (int64_t i = 0; i < N; ++i) {
    int32_t k[kMaxDim];
    sh_.coords(i, k);
    double r2 = 0.0;
    for (int a = 0; a < D; ++a) {
      const double u = static_cast<double>(k[a]) * (1.0 / (2.0 * static_cast<double>(sh_.n[a])));
      uk[a * N + i] = u;
      r2 = r2 + u * u;
    }
    rad[i] = std::sqrt(r2);
    double G = 0.0;
    if (rad[i] > 0.0) {
      const double f0 = 1.0 / (1.0 * static_cast<double>(w_));
      const double l = std::log(rad[i] / f0);
      G = std::exp(-(l * l) / two_sigma2);
    }
    X[i] = static_cast<double>(static_cast<T>(static_cast<T>(X[i]) * G));
  }
  // components: R1_a (sin on a), then R2_ab (a <= b; sin on a and b when a != b)
  const auto component = [&](int kind, int a, int b) {
    std::vector<double> y(static_cast<size_t>(N), 0.0);
    for (int64_t i = 0; i < N; ++i) {
      if (!(rad[i] > 0.0)) continue;
      const double inv = 1.0 / rad[i];
      const double ua = uk[a * N + i] * inv;
      double m;
      if (kind == 0) m = ua;
      else if (a == b) m = -ua * ua;
      else m = ua * (uk[b * N + i] * inv);
      y[i] = static_cast<double>(static_cast<T>(m * X[i]));
    }
    const int odd = kind == 0 ? (1 << a) : (a == b ? 0 : ((1 << a) | (1 << b)));
    for (int ax = 0; ax < D; ++ax) apply_axis(ax, M[ax][((odd >> ax) & 1) ? 2 : 1], y);
    F out(static_cast<size_t>(N));
    for (int64_t i = 0; i < N; ++i) out[i] = static_cast<T>(y[i]);
    return out;
  };
  F R1[kMaxDim], R2[6];
  for (int a = 0; a < D; ++a) R1[a] = component(0, a, a);
  int p = 0;
  for (int a = 0; a < D; ++a) {
    for (int b = a; b < D; ++b, ++p) R2[p] = component(1, a, b);
  }
  bool nonfinite = false;
  orientation_eigen<T>(D, N, R1, R2, nf, coh, &nonfinite);
  if (nonfinite) nonfinite_ = true;
}

// d, e of a voxel (cpp/src/method/element.cuh:238-254)
template <class T>
inline void element_de(T L, T c, T q, T span_m1, T* d, T* e) {
  const T f = static_cast<T>(static_cast<T>(T(1) - c) + static_cast<T>(c / q));
  *d = L * f;
  const T len = L * static_cast<T>(T(1) + static_cast<T>(span_m1 * c));
  const T diff = len - *d;
  *e = T(0.5) * (diff > T(0) ? diff : T(0));
}

template <class T>
void Element<T>::element_build(const F& L, const F& coh, const F* n, double* d_min, double* d_max) {
  // cpp/src/method/element.cu:181-216
  const T q = static_cast<T>(c_.q), sm1 = static_cast<T>(c_.span - 1.0);
  uint64_t mn = 0x7ff0000000000000ULL, mx = 0;
  for (int a = 0; a < sh_.dim && sh_.dim >= 2; ++a) o_[a].assign(static_cast<size_t>(sh_.count), T(0));
  for (int64_t i = 0; i < sh_.count; ++i) {
    T d, e;
    element_de<T>(L[i], sh_.dim == 1 ? T(0) : coh[i], q, sm1, &d, &e);
    if (sh_.dim >= 2) {
      for (int a = 0; a < sh_.dim; ++a) o_[a][i] = e * n[a][i];
    }
    const uint64_t b = dbits(static_cast<double>(d));
    mn = std::min(mn, b);
    mx = std::max(mx, b);
  }
  *d_min = bits_d(mn);
  *d_max = bits_d(mx);
}

template <class T>
void Element<T>::element_weights(const F& L, const F& coh) {
  // cpp/src/method/element.cu:218-292
  const T q = static_cast<T>(c_.q), sm1 = static_cast<T>(c_.span - 1.0);
  const int K = n_rungs_;
  std::vector<double> lw(static_cast<size_t>(K));
  for (int j = 0; j < K; ++j) lw[j] = std::log(static_cast<double>(rung_w_[j]));
  const double w_lo = static_cast<double>(rung_w_[0]);
  const double w_hi = static_cast<double>(rung_w_[K - 1]);
  lo_.assign(static_cast<size_t>(sh_.count), 0);
  t_.assign(static_cast<size_t>(sh_.count), T(0));
  rung_pts_ = rung_used_ = 0;
  for (int64_t i = 0; i < sh_.count; ++i) {
    T d, e;
    element_de<T>(L[i], sh_.dim == 1 ? T(0) : coh[i], q, sm1, &d, &e);
    int idx = 0;
    T tt = T(0);
    if (K > 1) {
      double dc = static_cast<double>(d);
      dc = dc > w_lo ? dc : w_lo;
      dc = dc < w_hi ? dc : w_hi;
      const double lg = std::log(dc);
      int cnt = 0;
      for (int j = 0; j < K; ++j) cnt += lw[j] <= lg ? 1 : 0;
      idx = cnt - 1;
      idx = idx < 0 ? 0 : (idx > K - 2 ? K - 2 : idx);
      const double tv = (lg - lw[idx]) / (lw[idx + 1] - lw[idx]);
      tt = static_cast<T>(tv);
    }
    lo_[i] = static_cast<uint8_t>(idx);
    t_[i] = tt;
    const T wl = T(1) - tt;
    uint32_t bits = 0u;
    if (wl > T(0)) bits |= 1u << idx;
    if (tt > T(0)) bits |= 1u << (idx + 1);
    rung_used_ |= bits;
    if (e > T(0.25)) rung_pts_ |= bits;
  }
}

// The operators (cpp/src/method/element_op.cuh:38-154): which 0 Dil (max), 2 Dil into the result
// and Ero into out1, 3 Avg (box).
template <class T>
typename Element<T>::F Element<T>::op(int which, const F& in, F* out1) const {
  const int D = sh_.dim;
  F out0(static_cast<size_t>(sh_.count), T(0));
  if (which == 2) out1->assign(static_cast<size_t>(sh_.count), T(0));
  for (int j = 0; j < n_rungs_; ++j) {
    if (((rung_used_ >> j) & 1u) == 0u) continue;
    F f0, f1;
    if (which == 3) {
      f0 = cube<T>(sh_, kCubeBox, in, rung_w_[j]);
    } else {
      f0 = cube<T>(sh_, kCubeMax, in, rung_w_[j]);
      if (which == 2) f1 = cube<T>(sh_, kCubeMin, in, rung_w_[j]);
    }
    const bool pts = D >= 2 && ((rung_pts_ >> j) & 1u) != 0u;
    for (int64_t i = 0; i < sh_.count; ++i) {
      const int l = lo_[i];
      const T tt = t_[i];
      const T wl = T(1) - tt;
      T wgt;
      bool add;
      if (l == j && wl > T(0)) {
        wgt = wl;
        add = false;
      } else if (l + 1 == j && tt > T(0)) {
        wgt = tt;
        add = wl > T(0);
      } else {
        continue;
      }
      T acc0 = f0[i];
      T acc1 = which == 2 ? f1[i] : T(0);
      if (pts) {
        int32_t x[kMaxDim];
        sh_.coords(i, x);
        for (int k = 1; k <= kM; ++k) {
          const double s = static_cast<double>(k) / static_cast<double>(kM);
          for (int sg = 0; sg < 2; ++sg) {
            double y[kMaxDim];
            for (int a = 0; a < D; ++a) {
              const double off = s * static_cast<double>(o_[a][i]);
              const double xa = static_cast<double>(x[a]);
              y[a] = sg == 0 ? xa + off : xa - off;
            }
            // D-linear interpolation of the reflected periodic extension
            int64_t o0[kMaxDim], o1[kMaxDim];
            T w0[kMaxDim], w1[kMaxDim];
            for (int a = 0; a < D; ++a) {
              const double fl = std::floor(y[a]);
              const double tt2 = y[a] - fl;
              const int64_t i0 = static_cast<int64_t>(fl);
              w1[a] = static_cast<T>(tt2);
              w0[a] = T(1) - w1[a];
              o0[a] = reflect_any(i0, sh_.n[a]) * sh_.st[a];
              o1[a] = reflect_any(i0 + 1, sh_.n[a]) * sh_.st[a];
            }
            const auto read = [&](const F& f) {
              T acc = T(0);
              for (int corner = 0; corner < (1 << D); ++corner) {
                int64_t off = 0;
                for (int a = 0; a < D; ++a) off += ((corner >> (D - 1 - a)) & 1) ? o1[a] : o0[a];
                T term = f[off];
                for (int a = 0; a < D; ++a) term = term * (((corner >> (D - 1 - a)) & 1) ? w1[a] : w0[a]);
                acc = acc + term;
              }
              return acc;
            };
            if (which == 2) {
              acc0 = max_c(acc0, read(f0));
              acc1 = min_c(acc1, read(f1));
            } else if (which == 0) {
              acc0 = max_c(acc0, read(f0));
            } else {
              acc0 = acc0 + read(f0);
            }
          }
        }
        if (which == 3) acc0 = acc0 / static_cast<T>(2 * kM + 1);
      }
      const T v0 = wgt * acc0;
      out0[i] = add ? static_cast<T>(out0[i] + v0) : v0;
      if (which == 2) {
        const T v1 = wgt * acc1;
        (*out1)[i] = add ? static_cast<T>((*out1)[i] + v1) : v1;
      }
    }
  }
  return out0;
}

template <class T>
void Element<T>::envelope_mean(const F& h, F& m, F& u, F& l) const {
  // cpp/src/method/element_op.cuh:156-174, 265-282
  u = op(2, h, &l);
  F mid(static_cast<size_t>(sh_.count));
  for (int64_t i = 0; i < sh_.count; ++i) mid[i] = T(0.5) * static_cast<T>(u[i] + l[i]);
  m = op(3, mid, nullptr);
}

template <class T>
Result Element<T>::run(const T* x, T* rows) {
  const int64_t N = sh_.count;
  Result res;
  F r(x, x + N);
  // start (cpp/src/method/driver.cpp:393-420)
  uint64_t nonfinite = 0;
  for (T v : r) nonfinite += std::isfinite(static_cast<double>(v)) ? 0 : 1;
  amax_ = amax_of(r);
  const int32_t kexp = (amax_ > 0.0 && std::isfinite(amax_)) ? std::ilogb(amax_) : 0;
  res.exp = kexp;
  if (kexp != 0) {
    for (T& v : r) {
      if constexpr (std::is_same_v<T, float>) v = static_cast<float>(std::ldexp(static_cast<double>(v), -kexp));
      else v = std::ldexp(v, -kexp);
    }
  }
  amax_ = amax_of(r);
  tol_ = static_cast<double>(static_cast<T>(static_cast<T>(tau_) * static_cast<T>(amax_)));
  if (nonfinite != 0 && check_finite_) {
    res.error = 1;
    return res;
  }
  bool error = false;
  sigma_x_ = noise_sigma(r, true);
  F L, Lp(static_cast<size_t>(N), T(0)), h, tau, tmp;
  std::vector<uint8_t> flags, ff, A;
  int32_t n_imfs = 0;
  for (;;) {
    // step 0: mode start (cpp/src/method/mode.cu:95-136)
    r_inf_ = amax_;
    fine_ = 0;
    jump_ = c_.absent_jump;
    p_odd_ = 0;
    p_ = 0.0;
    wc_ = INFINITY;
    g3_ = 1.0;
    n_sifts_ = 0;
    for (int a = 0; a < kMaxDim; ++a) ext_[a] = 0;
    const double floor2 = c_.fine_theta * sigma_x_;
    int32_t wd = odd_window(c_.sig_rho * static_cast<double>(std::max(3, w_prev_ + 2)));
    int32_t wl = odd_window(std::max(c_.beta, c_.sig_rho) * static_cast<double>(std::max(3, w_prev_ + 2)));
    sigma_n_ = noise_sigma(r, false);
    // steps 1-2: the window passes
    bool done = false;
    for (int pass = 0; pass < c_.sig_passes; ++pass) {
      tau_field(r, wd, wl, nullptr, tau);
      if (nonfinite_) {
        error = true;
        break;
      }
      sig_flags(r, tau, flags, ext_);
      if (!rice(pass, &wd, &wl)) {
        done = true;
        break;
      }
    }
    if (error || done) break;
    // step 3: G2 (cpp/src/method/driver.cpp:445-509)
    const int32_t s0 = std::max(3, w_prev_ + 2);
    if (c_.fine_jump * static_cast<double>(s0) <= static_cast<double>(w_)) {
      const std::vector<int32_t> rungs = g2_candidate_rungs(w_, w_prev_, c_.fine_jump);
      if (!rungs.empty()) {
        const std::vector<uint8_t>* ffp = &flags;
        if (c_.fine_theta > 0) {
          tau_field(r, wd, wl, &floor2, tau);
          uint64_t scratch[kMaxDim] = {0, 0, 0};
          sig_flags(r, tau, ff, scratch);
          ffp = &ff;
        }
        // the rung machine (cpp/src/method/driver.cpp:73-109)
        int32_t i = 0;
        bool pending = false, accepted = false;
        G2Result cand;
        std::vector<uint8_t> P, Pcand, Pacc;
        for (;;) {
          const int32_t s = i < static_cast<int32_t>(rungs.size()) ? rungs[static_cast<size_t>(i)]
                                                                 : odd_window(static_cast<double>(rungs.back()) * kRungRatio + 1.0);
          const G2Result o = g2_test(*ffp, s, P);
          if (pending) {
            if (o.outcome == kG2Accepted) {
              accepted = true;
              Pacc = Pcand;
              break;
            }
            if (o.outcome == kG2Stop) break;
            pending = false;
            ++i;
          } else {
            if (o.outcome == kG2Stop) break;
            if (o.outcome == kG2Accepted) {
              pending = true;
              cand = o;
              Pcand = P;
            }
            ++i;
          }
          if (i >= static_cast<int32_t>(rungs.size()) && !pending) break;
        }
        if (accepted) {
          fine_ = 1;
          p_ = cand.p;
          p_odd_ = odd_window(cand.p);
          wc_ = g3_coarse(*ffp, Pacc);
        }
      }
    }
    // step 4: guard, the window (cpp/src/method/mode.cu:189-223)
    if (nonfinite_) {
      error = true;
      break;
    }
    int32_t w = w_;
    if (fine_) {
      w = std::max(std::max(p_odd_, w_prev_ + 2), 3);
      jump_ = 1.0;
    }
    if (c_.growth > 1.0 && k_ >= c_.growth_from) {
      w = std::max(w, odd_window(c_.growth * static_cast<double>(w_prev_)));
      if (w > c_.n_max) break;
    }
    w_ = w;
    W_ = odd_window(c_.beta * static_cast<double>(w));
    if (fine_) {
      double f = 1.0;
      if (std::isfinite(wc_)) {
        const double qq = std::sqrt(wc_ / static_cast<double>(p_odd_));
        f = (c_.split * qq) / 2.0;
        f = f < 1.0 ? f : 1.0;
      }
      g3_ = f;
    }
    // step 5: the scale field
    const F om = raw_window(flags, W_);
    scale_field(om, A, L);
    if (k_ >= 1) local_floor(Lp, A, L);
    if (fine_) {
      for (T& v : L) {
        const T s = static_cast<T>(g3_) * v;
        v = s >= T(3) ? s : T(3);
      }
    }
    // step 6: orientation, element build
    F nv[kMaxDim], coh(static_cast<size_t>(N), T(0));
    if (sh_.dim >= 2) {
      orientation(r, nv, coh);
      if (nonfinite_) {
        error = true;
        break;
      }
      if (orient_) {
        // the first component of magnitude above the dtype's default tie tolerance is positive
        // (orientation.cu:412-418)
        const T zero = static_cast<T>(std::is_same_v<T, float> ? std::ldexp(1.0, -14) : std::ldexp(1.0, -30));
        const int D = sh_.dim;
        T* o = orient_ + static_cast<int64_t>(k_) * (D + 1) * N;
        for (int64_t i = 0; i < N; ++i) {
          int sgn = 0;
          for (int a = 0; a < D; ++a) {
            const T v = nv[a][static_cast<size_t>(i)];
            if (sgn == 0 && std::fabs(v) > zero) sgn = v > T(0) ? 1 : -1;
          }
          for (int a = 0; a < D; ++a) {
            const T v = nv[a][static_cast<size_t>(i)];
            o[a * N + i] = sgn < 0 ? -v : v;
          }
          o[D * N + i] = coh[static_cast<size_t>(i)];
        }
      }
    }
    double d_min, d_max;
    element_build(L, coh, nv, &d_min, &d_max);
    // step 7: the ladder and the weights
    rung_w_ = rung_ladder(d_min, d_max, w_, c_.n_max);
    n_rungs_ = static_cast<int32_t>(rung_w_.size());
    element_weights(L, coh);
    // step 8: sift 1, the continuation weight
    F m, u, l;
    envelope_mean(r, m, u, l);
    h.resize(static_cast<size_t>(N));
    for (int64_t i = 0; i < N; ++i) h[i] = r[i] - m[i];
    n_sifts_ = 1;
    F a;
    if (c_.sifts > 1) {
      F R(static_cast<size_t>(N));
      for (int64_t i = 0; i < N; ++i) R[i] = np_max(static_cast<T>(u[i] - l[i]), T(0));
      F U = R;
      for (int32_t it = 0; it < c_.u; ++it) U = op(0, U, nullptr);
      const T t0 = static_cast<T>(c_.t0);
      const double dd = c_.t1 - c_.t0;
      const T den = static_cast<T>(dd >= 1e-12 ? dd : 1e-12);
      F gw(static_cast<size_t>(N));
      for (int64_t i = 0; i < N; ++i) {
        T rho = T(0);
        if (static_cast<double>(U[i]) > tol_) rho = clip(static_cast<T>(R[i] / U[i]), T(0), T(1));
        gw[i] = clip(static_cast<T>(static_cast<T>(rho - t0) / den), T(0), T(1));
      }
      a = gw;
      for (int32_t it = 0; it < c_.s; ++it) a = op(3, a, nullptr);
      for (T& v : a) v = clip(v, T(0), T(1));
    }
    // step 9: sifts 2..S with G1 and the guard
    for (int32_t j = 1; j < c_.sifts; ++j) {
      F plain, up, lo;
      envelope_mean(h, plain, up, lo);
      F hd(static_cast<size_t>(N));
      for (int64_t i = 0; i < N; ++i) hd[i] = T(0.5) * static_cast<T>(up[i] - lo[i]);
      const F e0 = op(3, hd, nullptr);
      const F emax = cube<T>(sh_, kCubeMax, e0, W_);
      const F emin = cube<T>(sh_, kCubeMin, e0, W_);
      const T k0 = static_cast<T>(c_.ramp_k0);
      const double dk = c_.ramp_k1 - c_.ramp_k0;
      const T kden = static_cast<T>(dk >= 1e-12 ? dk : 1e-12);
      const T flr = static_cast<T>(tol_ >= c_.tiny ? tol_ : c_.tiny);
      F kr(static_cast<size_t>(N));
      for (int64_t i = 0; i < N; ++i) {
        const T hi = emax[i], lw = emin[i];
        const T den2 = np_max(static_cast<T>(hi + lw), flr);
        const T kap = static_cast<T>(hi - lw) / den2;
        kr[i] = clip(static_cast<T>(static_cast<T>(kap - k0) / kden), T(0), T(1));
      }
      F gk = cube<T>(sh_, kCubeBox, kr, W_);
      for (T& v : gk) v = clip(v, T(0), T(1));
      F e = e0;
      for (int32_t it = 0; it < c_.anorm_smooth; ++it) e = cube<T>(sh_, kCubeBox, e, W_);
      std::vector<double> ev(e.begin(), e.end());
      const double e_med = select_median(ev);
      double thr = c_.anorm_floor * e_med;
      thr = thr >= tol_ ? thr : tol_;
      thr = thr >= c_.tiny ? thr : c_.tiny;
      for (T& v : e) v = static_cast<double>(v) >= thr ? v : static_cast<T>(thr);
      F q(static_cast<size_t>(N));
      for (int64_t i = 0; i < N; ++i) q[i] = h[i] / e[i];
      F Mn, u2, l2;
      envelope_mean(q, Mn, u2, l2);
      F hn(static_cast<size_t>(N));
      uint64_t m_res = 0, m_h = 0;
      for (int64_t i = 0; i < N; ++i) {
        const T wv = gk[i];
        const T mA = clip(static_cast<T>(e[i] * Mn[i]), lo[i], up[i]);
        const T mh = static_cast<T>(static_cast<T>(wv * mA) + static_cast<T>(static_cast<T>(T(1) - wv) * plain[i]));
        const T mm = a.empty() ? mh : static_cast<T>(a[i] * mh);
        const T xv = h[i] - mm;
        hn[i] = xv;
        m_res = std::max(m_res, abs_bits(static_cast<T>(r[i] - xv)));
        m_h = std::max(m_h, abs_bits(xv));
      }
      if (!(bits_d(m_res) > r_inf_) && !(bits_d(m_h) > r_inf_)) {
        h = hn;
        ++n_sifts_;
      } else {
        break;
      }
    }
    // step 10: commit (cpp/src/method/mode.cu:304-348; field_ops.cu:151-203)
    std::copy(h.begin(), h.end(), rows + static_cast<int64_t>(n_imfs) * N);
    for (int64_t i = 0; i < N; ++i) r[i] = r[i] - h[i];
    res.windows.push_back(w_);
    res.energy.push_back(field_energy(sh_, h));
    res.spacing.push_back(spacing_);
    res.sifts.push_back(n_sifts_);
    ++n_imfs;
    amax_ = amax_of(r);
    tol_ = static_cast<double>(static_cast<T>(static_cast<T>(tau_) * static_cast<T>(amax_)));
    w_prev_ = w_;
    ++k_;
    Lp = L;
    if (!std::isfinite(amax_)) {
      error = true;
      break;
    }
    if (max_imf_ > 0 && n_imfs >= max_imf_) break;
    if (n_imfs + 1 >= cap_) throw std::logic_error("oracle: rows full");
  }
  if (error) {
    res.error = 2;
    res.n_imfs = 0;
    res.windows.clear();
    res.sifts.clear();
    res.spacing.clear();
    res.energy.clear();
    return res;
  }
  // finish: the residue row, the rows scaled back, the energies in x's units
  std::copy(r.begin(), r.end(), rows + static_cast<int64_t>(n_imfs) * N);
  if (kexp != 0) {
    for (int64_t i = 0; i < static_cast<int64_t>(n_imfs + 1) * N; ++i) {
      T v;
      if constexpr (std::is_same_v<T, float>) v = static_cast<float>(std::ldexp(static_cast<double>(rows[i]), kexp));
      else v = std::ldexp(rows[i], kexp);
      rows[i] = v;
      if (!std::isfinite(v)) error = true;
    }
    for (double& e : res.energy) e = std::ldexp(e, 2 * kexp);
  }
  if (error) {
    res.error = 2;
    res.n_imfs = 0;
    res.windows.clear();
    res.sifts.clear();
    res.spacing.clear();
    res.energy.clear();
    return res;
  }
  res.n_imfs = n_imfs;
  return res;
}

template <class T>
Ctl make_ctl(const Shape& sh, int32_t sifts) {
  Ctl c;
  c.n_max = sh.n_max;
  c.count = sh.count;
  c.sifts = sifts;
  c.tiny = std::is_same_v<T, float> ? static_cast<double>(FLT_MIN) : 1e-300;
  return c;
}


// ---------------------------------------------------------------------------------------------
// eda.monogenic (cpp/src/method/monogenic.cpp:61-158; orientation.cu:420-493, 791-831): the
// monogenic signal of one field, with the transforms as direct sums over the DCT bases in double.
// Planes: amplitude, phase, frequency [count], then (D >= 2) direction [D][count] and coherence.
template <class T>
bool monogenic(const Shape& sh, const T* x, T* out) {
  const int D = sh.dim;
  const int64_t N = sh.count;
  // the exact prescale f = x 2^-k, max|f| in [1, 2) (the driver's)
  double amax = 0.0;
  bool finite = true;
  for (int64_t i = 0; i < N; ++i) {
    const double v = static_cast<double>(x[i]);
    if (!std::isfinite(v)) finite = false;
    else amax = std::fmax(amax, std::fabs(v));
  }
  const int k = amax > 0.0 ? std::ilogb(amax) : 0;
  std::vector<T> f(static_cast<size_t>(N));
  for (int64_t i = 0; i < N; ++i) f[i] = static_cast<T>(std::ldexp(static_cast<double>(x[i]), -k));
  double mean = 0.0;
  for (int64_t i = 0; i < N; ++i) mean += static_cast<double>(f[i]);
  mean = mean / static_cast<double>(N);
  std::vector<double> X(static_cast<size_t>(N));
  for (int64_t i = 0; i < N; ++i) X[i] = static_cast<double>(static_cast<T>(static_cast<double>(f[i]) - mean));
  const auto axis_matrix = [](int64_t n, int kind) {
    std::vector<double> m(static_cast<size_t>(n * n));
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int64_t i = 0; i < n; ++i) {
      for (int64_t j = 0; j < n; ++j) {
        const int64_t kk = kind == 0 ? i : j, xx = kind == 0 ? j : i;
        const long double c = std::sqrt((kk ? 2.0L : 1.0L) / static_cast<long double>(n));
        const int64_t q = (kk * (2 * xx + 1)) % (4 * n);
        const long double ang = pi * static_cast<long double>(q) / static_cast<long double>(2 * n);
        m[static_cast<size_t>(i * n + j)] = static_cast<double>(c * (kind == 2 ? std::sin(ang) : std::cos(ang)));
      }
    }
    return m;
  };
  std::vector<double> M[kMaxDim][3];
  for (int a = 0; a < D; ++a) {
    for (int kk = 0; kk < 3; ++kk) M[a][kk] = axis_matrix(sh.n[a], kk);
  }
  const auto apply_axis = [&](int a, const std::vector<double>& m, std::vector<double>& g) {
    const int64_t n = sh.n[a], st = sh.st[a];
    std::vector<double> line(static_cast<size_t>(n));
    for (int64_t l = 0; l < sh.lines(a); ++l) {
      const int64_t base = sh.line_base(a, l);
      for (int64_t i = 0; i < n; ++i) line[i] = g[base + i * st];
      for (int64_t i = 0; i < n; ++i) {
        double acc = 0.0;
        const double* row = &m[static_cast<size_t>(i * n)];
        for (int64_t j = 0; j < n; ++j) acc += row[j] * line[j];
        g[base + i * st] = acc;
      }
    }
  };
  for (int a = 0; a < D; ++a) apply_axis(a, M[a][0], X);
  std::vector<double> uk(static_cast<size_t>(D * N)), rad(static_cast<size_t>(N));
  for (int64_t i = 0; i < N; ++i) {
    int32_t kk[kMaxDim];
    sh.coords(i, kk);
    double r2 = 0.0;
    for (int a = 0; a < D; ++a) {
      const double u = static_cast<double>(kk[a]) * (1.0 / (2.0 * static_cast<double>(sh.n[a])));
      uk[a * N + i] = u;
      r2 = r2 + u * u;
    }
    rad[i] = std::sqrt(r2);
    X[i] = static_cast<double>(static_cast<T>(X[i]));  // the spectrum is held in T
  }
  // kinds (riesz_mult, orientation.cu:116-127): 0 R1_a, 1 R2_aa, 2 R2_ab, 3 D_a f, 4 D_b R_a
  const auto component = [&](int kind, int a, int b) {
    std::vector<double> y(static_cast<size_t>(N), 0.0);
    for (int64_t i = 0; i < N; ++i) {
      if (!(rad[i] > 0.0)) continue;
      const double inv = 1.0 / rad[i];
      const double ua = uk[a * N + i] * inv;
      double m;
      if (kind == 0) m = ua;
      else if (kind == 1) m = -ua * ua;
      else if (kind == 3) m = -uk[a * N + i];
      else if (kind == 4) m = a == b ? uk[a * N + i] * ua : -(uk[a * N + i] * (uk[b * N + i] * inv));
      else m = ua * (uk[b * N + i] * inv);
      y[i] = static_cast<double>(static_cast<T>(m * X[i]));
    }
    const int odd = (kind == 0 || kind == 3) ? (1 << a) : (a == b ? 0 : ((1 << a) | (1 << b)));
    for (int ax = 0; ax < D; ++ax) apply_axis(ax, M[ax][((odd >> ax) & 1) ? 2 : 1], y);
    std::vector<T> o(static_cast<size_t>(N));
    for (int64_t i = 0; i < N; ++i) o[i] = static_cast<T>(y[i]);
    return o;
  };
  std::vector<T> R1[kMaxDim], DF[kMaxDim], R2[6], DR[6];
  for (int a = 0; a < D; ++a) {
    R1[a] = component(0, a, a);
    DF[a] = component(3, a, a);
  }
  int np = 0;
  for (int a = 0; a < D; ++a) {
    for (int b = a; b < D; ++b, ++np) {
      if (D >= 2) R2[np] = component(a == b ? 1 : 2, a, b);
      DR[np] = component(4, a, b);
    }
  }
  std::vector<T> nv[kMaxDim], coh;
  if (D >= 2) {
    bool eig_nonfinite = false;
    orientation_eigen<T>(D, N, R1, R2, nv, coh, &eig_nonfinite);
  }
  const T zero = static_cast<T>(std::is_same_v<T, float> ? std::ldexp(1.0, -14) : std::ldexp(1.0, -30));
  const double tiny = std::is_same_v<T, float> ? static_cast<double>(FLT_MIN) : 1e-300;
  const double pi = 3.141592653589793238462643383279502884;
  for (int64_t i = 0; i < N; ++i) {
    T nt[kMaxDim] = {T(1), T(0), T(0)};
    if (D >= 2) {
      int s = 0;
      for (int a = 0; a < D; ++a) {
        nt[a] = nv[a][static_cast<size_t>(i)];
        if (s == 0 && std::fabs(nt[a]) > zero) s = nt[a] > T(0) ? 1 : -1;
      }
      for (int a = 0; a < D; ++a) nt[a] = s < 0 ? -nt[a] : nt[a];
    }
    const double fv = static_cast<double>(f[i]);
    double q = 0.0, a2 = fv * fv, dnf = 0.0, dnq = 0.0;
    for (int a = 0; a < D; ++a) {
      const double r = static_cast<double>(R1[a][i]);
      const double na = static_cast<double>(nt[a]);
      q = q + na * r;
      a2 = a2 + r * r;
      dnf = dnf + na * static_cast<double>(DF[a][i]);
    }
    int p = 0;
    for (int a = 0; a < D; ++a) {
      for (int c = a; c < D; ++c, ++p) {
        const double na = static_cast<double>(nt[a]), nc = static_cast<double>(nt[c]);
        const double m = a == c ? na * na : 2.0 * (na * nc);
        dnq = dnq + m * static_cast<double>(DR[p][i]);
      }
    }
    double phase = 0.0, freq = 0.0;
    if (a2 > tiny) {
      phase = std::atan2(q, fv);
      freq = (fv * dnq - q * dnf) / a2;
    }
    out[i] = static_cast<T>(std::ldexp(std::sqrt(a2), k));
    const T pt = static_cast<T>(phase);
    out[N + i] = pt == -static_cast<T>(pi) ? static_cast<T>(pi) : pt;
    out[2 * N + i] = static_cast<T>(freq);
    if (D >= 2) {
      for (int a = 0; a < D; ++a) out[(3 + a) * N + i] = nt[a];
      out[(3 + D) * N + i] = coh[static_cast<size_t>(i)];
    }
  }
  return finite;
}

}  // namespace oracle

// ---------------------------------------------------------------------------------------------
// C ABI (ctypes): one call decomposes `batch` elements of `dim` axes n[0..dim-1] (C-contiguous,
// float32 when dtype == 0, float64 when 1). rows: batch x cap x count of the dtype, cap from
// eda_oracle_rows_cap; info arrays batch x (cap - 1). Returns 0, or -1 with the message in err.
extern "C" {

int eda_oracle_rows_cap(int dim, const int64_t* n, int32_t max_imf) {
  const oracle::Shape sh(dim, n);
  oracle::Ctl c = oracle::make_ctl<double>(sh, 3);
  const int32_t bound = oracle::mode_bound(c);
  const int32_t modes_max = max_imf > 0 ? std::min(bound, max_imf) : bound;
  return modes_max + 2;
}

int eda_oracle_decompose_orientation(const void* x, int dtype, int dim, int64_t batch, const int64_t* n,
                                     int32_t max_imf, double tie, int32_t sifts, int32_t check_finite, int32_t threads,
                                     void* rows, int32_t* n_imfs, int32_t* error, int32_t* windows,
                                     int32_t* sifts_out, double* spacing, double* energy, int32_t* exps,
                                     void* orient, char* err, int64_t err_len);

int eda_oracle_decompose(const void* x, int dtype, int dim, int64_t batch, const int64_t* n, int32_t max_imf,
                         double tie, int32_t sifts, int32_t check_finite, int32_t threads, void* rows,
                         int32_t* n_imfs, int32_t* error, int32_t* windows, int32_t* sifts_out, double* spacing,
                         double* energy, int32_t* exps, char* err, int64_t err_len) {
  return eda_oracle_decompose_orientation(x, dtype, dim, batch, n, max_imf, tie, sifts, check_finite, threads, rows,
                                          n_imfs, error, windows, sifts_out, spacing, energy, exps, nullptr, err,
                                          err_len);
}

// eda_oracle_decompose that also keeps the orientation rows (B, cap - 1, D + 1, count) in orient
// (zero where no mode ran); orient NULL keeps none.
int eda_oracle_decompose_orientation(const void* x, int dtype, int dim, int64_t batch, const int64_t* n,
                                     int32_t max_imf, double tie, int32_t sifts, int32_t check_finite, int32_t threads,
                                     void* rows, int32_t* n_imfs, int32_t* error, int32_t* windows,
                                     int32_t* sifts_out, double* spacing, double* energy, int32_t* exps,
                                     void* orient, char* err, int64_t err_len) {
  try {
    const oracle::Shape sh(dim, n);
    const int32_t cap = eda_oracle_rows_cap(dim, n, max_imf);
    const int64_t N = sh.count;
    const int64_t he = cap - 1;
    const auto one = [&](int64_t b) {
      const auto body = [&](auto tag) {
        using T = decltype(tag);
        oracle::Ctl c = oracle::make_ctl<T>(sh, sifts);
        const double tau = tie >= 0 ? tie : (std::is_same_v<T, float> ? std::ldexp(1.0, -14) : std::ldexp(1.0, -30));
        oracle::Element<T> el(sh, c, tau, check_finite != 0, max_imf, cap);
        if (orient && dim >= 2) {
          T* o = static_cast<T*>(orient) + b * (cap - 1) * (dim + 1) * N;
          std::fill(o, o + (cap - 1) * (dim + 1) * N, T(0));
          el.keep_orientation(o);
        }
        T* out = static_cast<T*>(rows) + b * cap * N;
        std::fill(out, out + cap * N, T(0));
        const oracle::Result r = el.run(static_cast<const T*>(x) + b * N, out);
        n_imfs[b] = r.n_imfs;
        error[b] = r.error;
        exps[b] = r.exp;
        for (int64_t k = 0; k < he; ++k) {
          const bool have = k < static_cast<int64_t>(r.windows.size());
          windows[b * he + k] = have ? r.windows[k] : 0;
          sifts_out[b * he + k] = have ? r.sifts[k] : 0;
          spacing[b * he + k] = have ? r.spacing[k] : 0.0;
          energy[b * he + k] = have ? r.energy[k] : 0.0;
        }
        if (r.error) {
          const T nan = std::numeric_limits<T>::quiet_NaN();
          std::fill(out, out + cap * N, nan);
        }
      };
      if (dtype == 0) body(float{});
      else body(double{});
    };
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(threads, batch));
    if (nt <= 1) {
      for (int64_t b = 0; b < batch; ++b) one(b);
    } else {
      std::vector<std::thread> pool;
      std::vector<std::string> errs(static_cast<size_t>(nt));
      for (int64_t t = 0; t < nt; ++t) {
        pool.emplace_back([&, t] {
          try {
            for (int64_t b = t; b < batch; b += nt) one(b);
          } catch (const std::exception& e) {
            errs[static_cast<size_t>(t)] = e.what();
          }
        });
      }
      for (auto& th : pool) th.join();
      for (const auto& e : errs) {
        if (!e.empty()) throw std::runtime_error(e);
      }
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::strncpy(err, e.what(), static_cast<size_t>(err_len - 1));
      err[err_len - 1] = 0;
    }
    return -1;
  }
}

// eda.monogenic of batch fields of x (batch, n..): out (3 [+ D + 1 in 2-D / 3-D]) planes of
// batch x count in the reference's native layout (amplitude, phase, frequency, direction
// [batch][D][count], coherence); nonfinite[b] = 1 where field b holds inf or NaN.
int eda_oracle_monogenic(const void* x, int dtype, int dim, int64_t batch, const int64_t* n, void* out,
                         int32_t* nonfinite) {
  try {
    const oracle::Shape sh(dim, n);
    const int64_t N = sh.count;
    const int planes = dim == 1 ? 3 : 4 + dim;
    const auto body = [&](auto tag) {
      using T = decltype(tag);
      std::vector<T> one(static_cast<size_t>(planes * N));
      for (int64_t b = 0; b < batch; ++b) {
        nonfinite[b] = oracle::monogenic<T>(sh, static_cast<const T*>(x) + b * N, one.data()) ? 0 : 1;
        T* o = static_cast<T*>(out);
        for (int pl = 0; pl < 3; ++pl) std::copy(one.begin() + pl * N, one.begin() + (pl + 1) * N, o + (pl * batch + b) * N);
        if (dim >= 2) {
          std::copy(one.begin() + 3 * N, one.begin() + (3 + dim) * N, o + 3 * batch * N + b * dim * N);
          std::copy(one.begin() + (3 + dim) * N, one.begin() + (4 + dim) * N, o + (3 + dim) * batch * N + b * N);
        }
      }
    };
    if (dtype == 0) body(float{});
    else body(double{});
    return 0;
  } catch (...) {
    return -1;
  }
}

// The ladder alone (tests): out receives up to 32 rungs; returns their count or -1.
int eda_oracle_rung_ladder(double d_min, double d_max, int32_t w, int32_t n_max, int32_t* out) {
  try {
    const std::vector<int32_t> v = oracle::rung_ladder(d_min, d_max, w, n_max);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return static_cast<int>(v.size());
  } catch (...) {
    return -1;
  }
}

// One cube filter of one element (tests): op 0 max, 1 min, 3 box; f (count values) in place.
// Stage hooks for the stage-level tests: the exact selection of the doubles v (q < 0: the median;
// NaN for an empty set), the significant-extrema flags of one element (bit a: axis a) with the
// counts per axis, and the face-connected components of mask != 0 (label: the smallest index of
// the component, -1 outside).
int eda_oracle_select(const double* v, int64_t n, double q, double* out) {
  std::vector<double> w(v, v + n);
  *out = q < 0 ? oracle::select_median(w) : oracle::select_quantile(w, q);
  return 0;
}

int eda_oracle_flags(int dtype, int dim, const int64_t* n, const void* r, const void* tau, uint8_t* flags,
                     uint64_t* ext) {
  const oracle::Shape sh(dim, n);
  std::vector<uint8_t> f;
  for (int a = 0; a < 3; ++a) ext[a] = 0;
  if (dtype == 0) {
    const auto* rp = static_cast<const float*>(r);
    const auto* tp = static_cast<const float*>(tau);
    oracle::extrema_flags<float>(sh, std::vector<float>(rp, rp + sh.count), std::vector<float>(tp, tp + sh.count), f, ext);
  } else {
    const auto* rp = static_cast<const double*>(r);
    const auto* tp = static_cast<const double*>(tau);
    oracle::extrema_flags<double>(sh, std::vector<double>(rp, rp + sh.count), std::vector<double>(tp, tp + sh.count), f,
                                  ext);
  }
  std::copy(f.begin(), f.end(), flags);
  return 0;
}

int eda_oracle_components(int dim, const int64_t* n, const uint8_t* mask, int64_t* labels) {
  const oracle::Shape sh(dim, n);
  const std::vector<uint8_t> m(mask, mask + sh.count);
  const std::vector<int64_t> lab = oracle::components(sh, m);
  std::copy(lab.begin(), lab.end(), labels);
  return 0;
}

int eda_oracle_cube(int dtype, int dim, const int64_t* n, int op, int32_t w, void* f) {
  const oracle::Shape sh(dim, n);
  const auto body = [&](auto tag) {
    using T = decltype(tag);
    T* p = static_cast<T*>(f);
    std::vector<T> v(p, p + sh.count);
    v = oracle::cube<T>(sh, static_cast<oracle::CubeOp>(op), v, w);
    std::copy(v.begin(), v.end(), p);
  };
  if (dtype == 0) body(float{});
  else body(double{});
  return 0;
}

}  // extern "C"
