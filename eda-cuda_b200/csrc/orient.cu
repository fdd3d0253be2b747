// SPDX-License-Identifier: Apache-2.0
// The orientation (orient.cuh): mean, forward DCT-II along every axis, the log-Gabor band, the
// Riesz components by inverse cosine / sine transforms, the energy tensor and the Jacobi
// eigen-decomposition. Every axis transform is a rotated pass (RotPass): the contiguous axis of the
// current layout is transformed and becomes the slowest axis, so D passes return a field to the
// element layout and every pass reads K-major rows. Float32 passes run on the tensor cores
// (orient_tc.cu, 3xTF32); float64 passes run the SIMT product below (FP64 accumulation).
#include "orient.cuh"

#include <atomic>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

namespace edab {
namespace {

// C(i, j) = sum_k A(i, k) B(k, j) with strided operands; grid.z the batch of blocks.
struct GemmDesc {
  int64_t M, N, K;
  int64_t sAi, sAk, sBk, sBj, sCi, sCj;
  int64_t zA, zB, zC;       // batch strides of the blocks (A, B, C)
  int64_t outer;            // blocks per element (z = b * outer + o)
  int64_t eA, eB, eC;       // element strides
  int64_t oA, oB, oC;       // outer strides
};

constexpr int kBM = 64, kBN = 64, kBK = 16;

template <class T>
__global__ void __launch_bounds__(256) gemm_simt(GemmDesc d, const T* __restrict__ A, const T* __restrict__ Bm,
                                                 T* __restrict__ C, const int32_t* __restrict__ run) {
  __shared__ T As[kBK][kBM + 1];
  __shared__ T Bs[kBK][kBN + 1];
  const int64_t z = blockIdx.z;
  const int64_t b = z / d.outer, o = z - (z / d.outer) * d.outer;
  if (run && !run[b]) return;
  const T* pA = A + b * d.eA + o * d.oA;
  const T* pB = Bm + b * d.eB + o * d.oB;
  T* pC = C + b * d.eC + o * d.oC;
  const int64_t i0 = static_cast<int64_t>(blockIdx.y) * kBM, j0 = static_cast<int64_t>(blockIdx.x) * kBN;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = T(0);
  for (int64_t k0 = 0; k0 < d.K; k0 += kBK) {
    for (int t = threadIdx.x; t < kBK * kBM; t += 256) {
      const int kk = t / kBM, ii = t % kBM;
      const int64_t i = i0 + ii, k = k0 + kk;
      As[kk][ii] = (i < d.M && k < d.K) ? pA[i * d.sAi + k * d.sAk] : T(0);
    }
    for (int t = threadIdx.x; t < kBK * kBN; t += 256) {
      const int kk = t / kBN, jj = t % kBN;
      const int64_t j = j0 + jj, k = k0 + kk;
      Bs[kk][jj] = (j < d.N && k < d.K) ? pB[k * d.sBk + j * d.sBj] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      T a[4], bb[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = As[kk][ty + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; ++v) bb[v] = Bs[kk][tx + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], bb[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int64_t i = i0 + ty + 16 * u;
    if (i >= d.M) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int64_t j = j0 + tx + 16 * v;
      if (j < d.N) pC[i * d.sCi + j * d.sCj] = acc[u][v];
    }
  }
}

// The layout of an element's field during the orientation: axis order, the last contiguous (padded
// to a multiple of 32 samples).
struct Layout {
  int dim;
  int ax[kMaxDim];
};
inline int64_t pad32(int64_t n) { return (n + 31) / 32 * 32; }
Layout element_layout(const Geom& g) {
  Layout L{g.dim, {0, 1, 2}};
  return L;
}
Layout rotated(const Layout& L) {
  Layout R = L;
  R.ax[0] = L.ax[L.dim - 1];
  for (int i = 1; i < L.dim; ++i) R.ax[i] = L.ax[i - 1];
  return R;
}
int64_t layout_field(const Geom& g, const Layout& L) {
  int64_t rows = 1;
  for (int i = 0; i < L.dim - 1; ++i) rows *= g.n[L.ax[i]];
  return rows * pad32(g.n[L.ax[L.dim - 1]]);
}
RotPass make_pass(const Geom& g, const Layout& L) {
  const int D = L.dim;
  RotPass p{};
  p.K = g.n[L.ax[D - 1]];
  p.pitch_in = pad32(p.K);
  if (D == 1) {
    // one axis: every element is one row, stored in place (no rotation)
    p.rows = 1;
    p.f_in = p.pitch_in;
    p.n_lo = 1;
    p.pitch_out = 1;
    p.s_j = 1;
    p.f_out = p.pitch_in;
    p.M = g.batch;
    return p;
  }
  p.rows = 1;
  for (int i = 0; i < D - 1; ++i) p.rows *= g.n[L.ax[i]];
  p.f_in = p.rows * p.pitch_in;
  p.n_lo = g.n[L.ax[D - 2]];
  p.pitch_out = pad32(p.n_lo);
  p.s_j = (p.rows / p.n_lo) * p.pitch_out;
  p.f_out = static_cast<int64_t>(p.K) * p.s_j;
  p.M = g.batch * p.rows;
  return p;
}

// The rotated pass with the SIMT product: per element and outer block o (the rows above the
// fastest row axis), C(i, j) = sum_k A(i, k) B(k, j) with A the n_lo rows, B(k, j) = M[j][k].
template <class T>
void rot_pass_simt(cudaStream_t s, const RotPass& p, int32_t n, const T* M, const T* in, T* out, const int32_t* run) {
  GemmDesc d{};
  const int64_t outer = p.rows / p.n_lo;
  d.M = p.n_lo;
  d.N = p.K;
  d.K = p.K;
  d.sAi = p.pitch_in;
  d.sAk = 1;
  d.sBk = 1;
  d.sBj = n;
  d.sCi = 1;
  d.sCj = p.s_j;
  d.outer = outer;
  d.eA = p.f_in;
  d.oA = p.n_lo * p.pitch_in;
  d.eB = 0;
  d.oB = 0;
  d.eC = p.f_out;
  d.oC = p.pitch_out;
  const int64_t batch = p.M / p.rows;
  const dim3 grid(static_cast<unsigned>((d.N + kBN - 1) / kBN), static_cast<unsigned>((d.M + kBM - 1) / kBM),
                  static_cast<unsigned>(batch * outer));
  gemm_simt<T><<<grid, 256, 0, s>>>(d, in, M, out, run);
  EDAB_LAUNCH("gemm_simt");
}

// The element's mean in double, deterministic for a shape: fixed chunks of kMeanChunk padded
// samples, each summed by one CTA (a fixed per-thread order and a fixed tree), the chunk sums then
// added in chunk order.
constexpr int64_t kMeanChunk = 1 << 16;

template <class T>
__global__ void __launch_bounds__(256) mean_partial(Geom g, const T* __restrict__ r, const int32_t* run, double* part,
                                                    int64_t nchunks) {
  __shared__ double sh[256];
  const int64_t b = blockIdx.y, c = blockIdx.x;
  const int32_t nl = g.n_last;
  double acc = 0.0;
  if (run[b]) {
    const T* rb = r + b * g.field;
    const int64_t v1 = min(g.field, (c + 1) * kMeanChunk);
    for (int64_t v = c * kMeanChunk + threadIdx.x; v < v1; v += 256) {
      if (pitch_col(g, v) < nl) acc = __dadd_rn(acc, static_cast<double>(rb[v]));
    }
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[b * nchunks + c] = sh[0];
}

__global__ void mean_final(int64_t B, int64_t count, const int32_t* run, const double* part, int64_t nchunks,
                           double* mean) {
  const int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (b >= B) return;
  double s = 0.0;
  for (int64_t c = 0; c < nchunks; ++c) s = __dadd_rn(s, part[b * nchunks + c]);
  mean[b] = run[b] ? __ddiv_rn(s, static_cast<double>(count)) : 0.0;
}

// The frequencies of DCT index k in cycles per sample (u_a = k_a / (2 n_a)) and rad = |u|.
template <int D>
__device__ __forceinline__ double dct_freq(const Geom& g, const int32_t* k, double* u) {
  double r2 = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    u[a] = __dmul_rn(static_cast<double>(k[a]), __ddiv_rn(1.0, __dmul_rn(2.0, static_cast<double>(g.n[a]))));
    r2 = __dadd_rn(r2, __dmul_rn(u[a], u[a]));
  }
  return __dsqrt_rn(r2);
}

template <int D>
__host__ __device__ constexpr int tensor_pair(int a, int b) {
  return D == 2 ? (a == 0 ? b : 2) : (a == 0 ? b : (a == 1 ? 2 + b : 5));
}

// ---------------------------------------------------------------------------------------------
// The eigen step of the orientation: the top eigenvector n and the coherence c = (mu1 - mu2) /
// (mu1 + mu2) (clipped to [0, 1]) of the symmetric D x D energy tensor of every voxel
// (cpp/src/method/element.cu:49-164 computes the same quantities).
//
// Cyclic Jacobi with half-angle rotations: for a pair (p, q) with off-diagonal value b and half
// difference h = (A_qq - A_pp) / 2, r = hypot(h, b), the rotation J (cos t, sin t) with
// cos 2t = |h| / r that zeroes A_pq is applied as A <- J^T A J and V <- V J. A 2 x 2 tensor is
// diagonal after one rotation; a 3 x 3 one after a few sweeps (quadratic convergence), on the
// tensor prescaled by a power of two (exact) so that no product leaves the range.
//
// Precision: float32 fields solve in float (4 sweeps); where the gap (mu1 - mu2) / (mu1 + mu2) falls
// below kEigenGap the direction is ill-conditioned in float (its error grows as eps / gap) and the
// voxel is solved again in double (6 sweeps) from the same tensor. Float64 fields always solve in
// double. The direction's sign: its largest component (the first on a tie) is positive.
constexpr double kEigenGap = 1e-2;

template <class S, int D>
__device__ __forceinline__ void jacobi_pair(S (&A)[3][3], S (&V)[3][3], int p, int q) {
  const S b = A[p][q];
  if (b == S(0)) return;
  const S h = (A[q][q] - A[p][p]) * S(0.5);
  const S r = hypot(h, b);
  // cos t and sin t of the smaller rotation angle t (|t| <= pi / 4): tan 2t = b / h
  const S c = sqrt((S(1) + fabs(h) / r) * S(0.5));
  const S sn = (h < S(0) ? S(-1) : S(1)) * b / (S(2) * r * c);
  // columns p and q of A J, then rows p and q of J^T (A J)
  S AJ[3][3];
#pragma unroll
  for (int i = 0; i < D; ++i) {
#pragma unroll
    for (int j = 0; j < D; ++j) AJ[i][j] = A[i][j];
    AJ[i][p] = c * A[i][p] - sn * A[i][q];
    AJ[i][q] = sn * A[i][p] + c * A[i][q];
  }
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const S up = c * AJ[p][j] - sn * AJ[q][j];
    const S uq = sn * AJ[p][j] + c * AJ[q][j];
#pragma unroll
    for (int i = 0; i < D; ++i) A[i][j] = AJ[i][j];
    A[p][j] = up;
    A[q][j] = uq;
  }
  A[p][q] = A[q][p] = S(0);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const S vp = V[i][p], vq = V[i][q];
    V[i][p] = c * vp - sn * vq;
    V[i][q] = sn * vp + c * vq;
  }
}

// The eigen decomposition of the tensor A0 (double copies of the T entries) in precision S: the
// top eigenvector into nv, the coherence into *coh; returns the gap (mu1 - mu2) / (mu1 + mu2).
template <class S, int D>
__device__ __forceinline__ double eigen_top(const double (&A0)[3][3], double* nv, double* coh) {
  S A[3][3], V[3][3];
  double amax = 0.0;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) amax = fmax(amax, fabs(A0[i][j]));
  const double scale = (amax > 0.0 && amax < d_inf()) ? scalbn(1.0, -ilogb(amax)) : 1.0;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      A[i][j] = static_cast<S>(A0[i][j] * scale);
      V[i][j] = i == j ? S(1) : S(0);
    }
  if constexpr (D == 2) {
    jacobi_pair<S, 2>(A, V, 0, 1);
  } else {
    constexpr int kSweeps = sizeof(S) == 4 ? 4 : 6;
#pragma unroll 1
    for (int sweep = 0; sweep < kSweeps; ++sweep) {
      jacobi_pair<S, 3>(A, V, 0, 1);
      jacobi_pair<S, 3>(A, V, 0, 2);
      jacobi_pair<S, 3>(A, V, 1, 2);
    }
  }
  // the top eigenvalue (the first on a tie), the largest of the others, the top column of V; by
  // selects over compile-time indices (a run-time index would put A and V in local memory)
  int top = 0;
  S mu1 = A[0][0];
#pragma unroll
  for (int a = 1; a < D; ++a) {
    if (A[a][a] > mu1) {
      mu1 = A[a][a];
      top = a;
    }
  }
  S mu2 = -inf_t<S>();
  S col[3] = {S(0), S(0), S(0)};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    if (a != top && A[a][a] > mu2) mu2 = A[a][a];
#pragma unroll
    for (int j = 0; j < D; ++j) col[a] = j == top ? V[a][j] : col[a];
  }
  S lead = col[0];
#pragma unroll
  for (int a = 1; a < D; ++a) lead = fabs(col[a]) > fabs(lead) ? col[a] : lead;
  const S sgn = lead < S(0) ? S(-1) : S(1);
#pragma unroll
  for (int a = 0; a < D; ++a) nv[a] = static_cast<double>(sgn * col[a]);
  const S sum = mu1 + mu2;
  S cv = sum > S(0) ? (mu1 - mu2) / sum : S(0);
  cv = cv < S(0) ? S(0) : (cv > S(1) ? S(1) : cv);
  *coh = static_cast<double>(cv);
  return static_cast<double>(cv);
}

// The energy tensor T = R1 R1^T + R2 R2^T of every voxel in the field's dtype (the reference's
// rounding order: R1_a R1_c, then + R2_ak R2_kc for k = 0 .. D - 1), then its eigen step.
template <class T, int D>
__global__ void __launch_bounds__(256) tensor_eigen(Geom g, const int32_t* run, const T* __restrict__ work_r1,
                                                    const T* __restrict__ work_r2, T* n0, T* n1, T* n2, T* coh,
                                                    Elem* el) {
  constexpr int K = D * (D + 1) / 2;
  const int64_t F = g.batch * g.field;
  const int32_t nl = g.n[D - 1];
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    if (!run[b]) continue;
    bool bad = false;
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      if (pitch_col(g, v) >= nl) continue;
      const int64_t i = b * g.field + v;
      T R1[D], R2[K];
#pragma unroll
      for (int a = 0; a < D; ++a) R1[a] = work_r1[a * F + i];
#pragma unroll
      for (int p = 0; p < K; ++p) R2[p] = work_r2[p * F + i];
      double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      bool finite = true;
#pragma unroll
      for (int a = 0; a < D; ++a) {
#pragma unroll
        for (int c = a; c < D; ++c) {
          T acc = mul_rn(R1[a], R1[c]);
#pragma unroll
          for (int k = 0; k < D; ++k) {
            acc = add_rn(acc, mul_rn(R2[tensor_pair<D>(min(a, k), max(a, k))], R2[tensor_pair<D>(min(k, c), max(k, c))]));
          }
          A[a][c] = A[c][a] = static_cast<double>(acc);
          finite = finite && isfinite(A[a][c]);
        }
      }
      bad = bad || !finite;
      double nv[3] = {0, 0, 0}, cv = 0.0;
      if constexpr (std::is_same_v<T, float>) {
        if (eigen_top<float, D>(A, nv, &cv) < kEigenGap) eigen_top<double, D>(A, nv, &cv);
      } else {
        eigen_top<double, D>(A, nv, &cv);
      }
      coh[i] = static_cast<T>(cv);
      n0[i] = static_cast<T>(nv[0]);
      n1[i] = static_cast<T>(nv[1]);
      if constexpr (D == 3) n2[i] = static_cast<T>(nv[2]);
    }
    if (bad) el[b].nonfinite = 1;
  }
}

struct PlanKey {
  int dim, n0, n1, n2, f64, dev;
  bool operator<(const PlanKey& o) const {
    return std::tie(dim, n0, n1, n2, f64, dev) < std::tie(o.dim, o.n0, o.n1, o.n2, o.f64, o.dev);
  }
};

// tf32 round-to-nearest (ties away from zero) of a float32, on the host: the hi / lo split of the
// tensor-core bases (cvt.rna.tf32.f32 rounds the same way).
float tf32_rna(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// bfloat16 of a float32, round to nearest even (finite values), and back.
uint16_t bf16_rne(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  u += 0x7fffu + ((u >> 16) & 1u);
  return static_cast<uint16_t>(u >> 16);
}
float bf16_float(uint16_t b) {
  const uint32_t u = static_cast<uint32_t>(b) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

std::atomic<int> g_transform_precision{static_cast<int>(TransformPrecision::kTf32x3)};

template <class T>
void upload_axis(OrientPlan& p, int a, int32_t n) {
  // the bases in long double, rounded once to the dtype
  const long double pi = 3.141592653589793238462643383279502884L;
  const size_t nn = static_cast<size_t>(n) * n;
  std::vector<T> fwd(nn), ic(nn), is(nn);
  std::vector<long double> exact_c(nn), exact_s(nn);
  for (int32_t k = 0; k < n; ++k) {
    const long double ck = std::sqrt((k ? 2.0L : 1.0L) / static_cast<long double>(n));
    for (int32_t x = 0; x < n; ++x) {
      const int64_t q = (static_cast<int64_t>(k) * (2 * x + 1)) % (4 * static_cast<int64_t>(n));
      const long double ang = pi * static_cast<long double>(q) / static_cast<long double>(2 * n);
      const long double cv = ck * std::cos(ang), sv = ck * std::sin(ang);
      exact_c[static_cast<size_t>(k) * n + x] = cv;
      exact_s[static_cast<size_t>(k) * n + x] = sv;
      fwd[static_cast<size_t>(k) * n + x] = static_cast<T>(cv);
      ic[static_cast<size_t>(x) * n + k] = static_cast<T>(cv);
      is[static_cast<size_t>(x) * n + k] = static_cast<T>(sv);
    }
  }
  const size_t bytes = sizeof(T) * nn;
  EDAB_CUDA(cudaMalloc(&p.fwd[a], bytes));
  EDAB_CUDA(cudaMalloc(&p.icos[a], bytes));
  EDAB_CUDA(cudaMalloc(&p.isin[a], bytes));
  EDAB_CUDA(cudaMemcpy(p.fwd[a], fwd.data(), bytes, cudaMemcpyHostToDevice));
  EDAB_CUDA(cudaMemcpy(p.icos[a], ic.data(), bytes, cudaMemcpyHostToDevice));
  EDAB_CUDA(cudaMemcpy(p.isin[a], is.data(), bytes, cudaMemcpyHostToDevice));
  if constexpr (std::is_same_v<T, float>) {
    // [2][npad][kpad]: row j holds B(j, k) (hi), row npad + j its lo part
    const int32_t kpad = static_cast<int32_t>(pad32(n));
    const int32_t npad = (n + 127) / 128 * 128;
    p.kpad[a] = kpad;
    p.npad[a] = npad;
    const size_t tb = static_cast<size_t>(2) * npad * kpad;
    auto split = [&](auto&& value, void** dst) {
      std::vector<float> h(tb, 0.0f);
      for (int32_t j = 0; j < n; ++j) {
        for (int32_t k = 0; k < n; ++k) {
          const long double v = value(j, k);
          const float hi = tf32_rna(static_cast<float>(v));
          const float lo = tf32_rna(static_cast<float>(v - static_cast<long double>(hi)));
          h[static_cast<size_t>(j) * kpad + k] = hi;
          h[static_cast<size_t>(npad + j) * kpad + k] = lo;
        }
      }
      EDAB_CUDA(cudaMalloc(dst, tb * sizeof(float)));
      EDAB_CUDA(cudaMemcpy(*dst, h.data(), tb * sizeof(float), cudaMemcpyHostToDevice));
    };
    // the bfloat16 split: hi = bf16(v), lo = bf16(v - hi), round to nearest even
    const auto split16 = [&](auto&& value, void** dst) {
      std::vector<uint16_t> h(tb, 0);
      for (int32_t j = 0; j < n; ++j) {
        for (int32_t k = 0; k < n; ++k) {
          const long double v = value(j, k);
          const uint16_t hi = bf16_rne(static_cast<float>(v));
          const uint16_t lo = bf16_rne(static_cast<float>(v - static_cast<long double>(bf16_float(hi))));
          h[static_cast<size_t>(j) * kpad + k] = hi;
          h[static_cast<size_t>(npad + j) * kpad + k] = lo;
        }
      }
      EDAB_CUDA(cudaMalloc(dst, tb * sizeof(uint16_t)));
      EDAB_CUDA(cudaMemcpy(*dst, h.data(), tb * sizeof(uint16_t), cudaMemcpyHostToDevice));
    };
    // forward: output frequency j, input sample k; inverse: output sample j, input frequency k
    const auto fwd_v = [&](int32_t j, int32_t k) { return exact_c[static_cast<size_t>(j) * n + k]; };
    const auto icos_v = [&](int32_t j, int32_t k) { return exact_c[static_cast<size_t>(k) * n + j]; };
    const auto isin_v = [&](int32_t j, int32_t k) { return exact_s[static_cast<size_t>(k) * n + j]; };
    split(fwd_v, &p.tc_fwd[a]);
    split(icos_v, &p.tc_icos[a]);
    split(isin_v, &p.tc_isin[a]);
    split16(fwd_v, &p.bf_fwd[a]);
    split16(icos_v, &p.bf_icos[a]);
    split16(isin_v, &p.bf_isin[a]);
  }
}

}  // namespace

const OrientPlan& orient_plan(const Geom& g, bool f64) {
  static std::mutex mu;
  static std::map<PlanKey, std::unique_ptr<OrientPlan>> cache;
  int dev = 0;
  EDAB_CUDA(cudaGetDevice(&dev));
  const PlanKey key{g.dim, g.n[0], g.n[1], g.n[2], f64 ? 1 : 0, dev};
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return *it->second;
  auto p = std::make_unique<OrientPlan>();
  p->dim = g.dim;
  p->f64 = f64;
  p->device = dev;
  for (int a = 0; a < g.dim; ++a) {
    p->n[a] = g.n[a];
    if (f64) upload_axis<double>(*p, a, g.n[a]);
    else upload_axis<float>(*p, a, g.n[a]);
  }
  // the uploads above are legacy-stream copies from pageable memory, which may return before the
  // data lands: complete them before any stream (a non-blocking one included) reads the plan
  EDAB_CUDA(cudaStreamSynchronize(nullptr));
  const OrientPlan& ref = *p;
  cache.emplace(key, std::move(p));
  return ref;
}

template <class T>
void transform_axes(cudaStream_t s, const Geom& g, const OrientPlan& plan, const T* in, T* out, T* buf0, T* buf1,
                    const int* kinds, const int32_t* run, int32_t* err) {
  const int D = g.dim;
  Layout L = element_layout(g);
  const T* src = in;
  for (int step = 0; step < D; ++step) {
    const RotPass p = make_pass(g, L);
    const int a = L.ax[D - 1];
    T* dst = step == D - 1 ? out : (src == buf0 ? buf1 : buf0);
    const int which = kinds[a];
    if constexpr (std::is_same_v<T, float>) {
      const TransformPrecision mode = transform_precision();
      if (mode == TransformPrecision::kFp32) {
        const void* B = which == 0 ? plan.fwd[a] : (which == 1 ? plan.icos[a] : plan.isin[a]);
        rot_pass_simt<T>(s, p, g.n[a], static_cast<const T*>(B), src, dst, run);
      } else if (mode == TransformPrecision::kBf16x3) {
        const void* B = which == 0 ? plan.bf_fwd[a] : (which == 1 ? plan.bf_icos[a] : plan.bf_isin[a]);
        rot_pass_tc(s, p, B, true, plan.kpad[a], plan.npad[a], src, dst, run, err);
      } else {
        const void* B = which == 0 ? plan.tc_fwd[a] : (which == 1 ? plan.tc_icos[a] : plan.tc_isin[a]);
        rot_pass_tc(s, p, B, false, plan.kpad[a], plan.npad[a], src, dst, run, err);
      }
    } else {
      const void* B = which == 0 ? plan.fwd[a] : (which == 1 ? plan.icos[a] : plan.isin[a]);
      rot_pass_simt<T>(s, p, g.n[a], static_cast<const T*>(B), src, dst, run);
    }
    L = rotated(L);
    src = dst;
  }
}
TransformPrecision transform_precision() {
  return static_cast<TransformPrecision>(g_transform_precision.load(std::memory_order_relaxed));
}
void set_transform_precision(TransformPrecision p) {
  g_transform_precision.store(static_cast<int>(p), std::memory_order_relaxed);
}

template void transform_axes<float>(cudaStream_t, const Geom&, const OrientPlan&, const float*, float*, float*,
                                    float*, const int*, const int32_t*, int32_t*);
template void transform_axes<double>(cudaStream_t, const Geom&, const OrientPlan&, const double*, double*, double*,
                                     double*, const int*, const int32_t*, int32_t*);

int64_t orient_layout_samples(const Geom& g) {
  Layout L = element_layout(g);
  int64_t fmax = 0;
  for (int i = 0; i < g.dim; ++i) {
    fmax = std::max(fmax, layout_field(g, L));
    L = rotated(L);
  }
  return fmax;
}

int64_t orient_work_samples(const Geom& g) {
  const int D = g.dim;
  return g.batch * (3 * orient_layout_samples(g) + static_cast<int64_t>(D + D * (D + 1) / 2) * g.field);
}

template <class T>
void orientation(cudaStream_t s, const Geom& g, const OrientPlan& plan, const T* r, Elem* el, const int32_t* run,
                 T* const* n, T* coh, T* work, double two_sigma2, int32_t* err) {
  const int D = g.dim;
  const int64_t F = g.batch * g.field;
  const int64_t Fw = g.batch * orient_layout_samples(g);
  T* X = work;            // the band spectrum
  T* Y = work + Fw;       // a component spectrum (and a pass buffer)
  T* Z = work + 2 * Fw;   // pass buffer
  T* R1 = work + 3 * Fw;  // D fields
  T* R2 = R1 + D * F;     // D (D + 1) / 2 fields
  auto transform = [&](const T* in, T* out, auto&& mats) {
    int kinds[kMaxDim] = {0, 0, 0};
    for (int a = 0; a < D; ++a) kinds[a] = mats(a);
    transform_axes<T>(s, g, plan, in, out, Z, Y, kinds, run, err);
  };
  // mean, then f = r - mean (the difference in double, rounded to T)
  // the means and the chunk sums at the head of Z, consumed before Z is used
  const int64_t nchunks = (g.field + kMeanChunk - 1) / kMeanChunk;
  double* mean = reinterpret_cast<double*>(Z);
  double* part = mean + g.batch;
  mean_partial<T><<<dim3(static_cast<unsigned>(nchunks), static_cast<unsigned>(g.batch)), 256, 0, s>>>(g, r, run, part,
                                                                                                       nchunks);
  EDAB_LAUNCH("mean_partial");
  mean_final<<<blocks_for(g.batch), 256, 0, s>>>(g.batch, g.count, run, part, nchunks, mean);
  EDAB_LAUNCH("mean_final");
  for_voxels(s, g, [=] __device__(int64_t b) { return run[b] != 0; },
             [=] __device__(int64_t b, int64_t, int64_t i) {
               Y[i] = static_cast<T>(__dsub_rn(static_cast<double>(r[i]), mean[b]));
             });
  // forward DCT-II along every axis: Y -> X
  transform(Y, X, [](int) { return 0; });
  // the band: X *= G(rad), G the one-octave log-Gabor at f0 = 1 / w (G(0) = 0)
  const Geom gg = g;
  for_voxels(s, g, [=] __device__(int64_t b) { return run[b] != 0; },
             [=] __device__(int64_t b, int64_t v, int64_t i) {
               int32_t k[kMaxDim];
               voxel_coords(gg, v, k);
               double u[kMaxDim];
               double rad;
               if (gg.dim == 2) rad = dct_freq<2>(gg, k, u);
               else rad = dct_freq<3>(gg, k, u);
               double G = 0.0;
               if (rad > 0.0) {
                 const double f0 = __ddiv_rn(1.0, __dmul_rn(1.0, static_cast<double>(el[b].w)));
                 const double l = log(__ddiv_rn(rad, f0));
                 G = exp(__ddiv_rn(-__dmul_rn(l, l), two_sigma2));
               }
               X[i] = static_cast<T>(__dmul_rn(static_cast<double>(X[i]), G));
             });
  // the components: R1_a (sine on axis a), then R2_ab (a <= b; sine on a and b when a != b)
  int p = 0;
  for (int kind = 0; kind < 2; ++kind) {
    for (int a = 0; a < D; ++a) {
      for (int b2 = (kind == 0 ? a : a); b2 < (kind == 0 ? a + 1 : D); ++b2) {
        T* out = kind == 0 ? R1 + a * F : R2 + (p++) * F;
        const int ca = a, cb = b2, ck = kind;
        for_voxels(s, g, [=] __device__(int64_t bb) { return run[bb] != 0; },
                   [=] __device__(int64_t, int64_t v, int64_t i) {
                     int32_t k[kMaxDim];
                     voxel_coords(gg, v, k);
                     double u[kMaxDim];
                     const double rad = gg.dim == 2 ? dct_freq<2>(gg, k, u) : dct_freq<3>(gg, k, u);
                     double m = 0.0;
                     if (rad > 0.0) {
                       const double inv = __ddiv_rn(1.0, rad);
                       const double ua = __dmul_rn(u[ca], inv);
                       if (ck == 0) m = ua;
                       else if (ca == cb) m = __dmul_rn(-ua, ua);
                       else m = __dmul_rn(ua, __dmul_rn(u[cb], inv));
                     }
                     Y[i] = static_cast<T>(__dmul_rn(m, static_cast<double>(X[i])));
                   });
        const int odd = kind == 0 ? (1 << a) : (a == b2 ? 0 : ((1 << a) | (1 << b2)));
        transform(Y, out, [odd](int ax) { return ((odd >> ax) & 1) ? 2 : 1; });
      }
    }
  }
  const dim3 grid = voxel_grid(g);
  if (D == 2) tensor_eigen<T, 2><<<grid, 256, 0, s>>>(g, run, R1, R2, n[0], n[1], nullptr, coh, el);
  else tensor_eigen<T, 3><<<grid, 256, 0, s>>>(g, run, R1, R2, n[0], n[1], n[2], coh, el);
  EDAB_LAUNCH("tensor_eigen");
}

// ---------------------------------------------------------------------------------------------
// eda.monogenic (cpp/src/method/orientation.cu:420-493, 791-831 of eda-cuda): the Riesz components
// of the whole spectrum (no band) of the prescaled field f, the orientation's eigen step (D >= 2),
// then per sample, in double and in the reference's order: n canonical (1 in 1-D), q = sum n_a R1_a,
// A^2 = f^2 + sum R1_a^2, D_n f = sum n_b D_b f, D_n q = sum_{a <= b} m_ab D_b R_a (m_aa = n_a^2,
// m_ab = 2 n_a n_b); where A^2 > tiny: phase = atan2(q, f) (an angle that rounds to -pi is pi),
// frequency = (f D_n q - q D_n f) / A^2; amplitude = sqrt(A^2) 2^exp, rounded once.
namespace {

// The Riesz multiplier of component (kind, a, b) at the spectrum index k (riesz_mult, orientation.cu:
// 116-127): 0 R1_a, 1 R2_aa, 2 R2_ab, 3 D_a f, 4 D_b R_a; 0 at the DC.
template <int D>
__device__ __forceinline__ double riesz_mult(const Geom& g, int kind, int a, int b, const int32_t* k) {
  double u[kMaxDim];
  const double rad = dct_freq<D>(g, k, u);
  if (!(rad > 0.0)) return 0.0;
  const double inv = __ddiv_rn(1.0, rad);
  const double ua = __dmul_rn(u[a], inv);
  if (kind == 0) return ua;
  if (kind == 1) return __dmul_rn(-ua, ua);
  if (kind == 3) return -u[a];
  if (kind == 4) return a == b ? __dmul_rn(u[a], ua) : -__dmul_rn(u[a], __dmul_rn(u[b], inv));
  return __dmul_rn(ua, __dmul_rn(u[b], inv));
}

template <class T, int D>
__global__ void __launch_bounds__(256) riesz_spectrum(Geom g, int kind, int a, int b, const T* __restrict__ X,
                                                      T* __restrict__ Y) {
  for (int64_t e = blockIdx.y; e < g.batch; e += gridDim.y) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      int32_t k[kMaxDim];
      if (!voxel_coords_d<D>(g, v, g.n[D - 1], k)) continue;
      const int64_t i = e * g.field + v;
      Y[i] = static_cast<T>(__dmul_rn(riesz_mult<D>(g, kind, a, b, k), static_cast<double>(X[i])));
    }
  }
}

template <class T, int D>
__global__ void __launch_bounds__(256) monogenic_kernel(Geom g, const T* __restrict__ f, const T* r1,
                                                        const T* df, const T* dr, const T* n, const T* c,
                                                        const int32_t* __restrict__ exp, double tiny, T zero,
                                                        T* __restrict__ out, int64_t out_batch, int64_t b0) {
  constexpr int NP = D * (D + 1) / 2;
  const int64_t F = g.batch * g.field;
  const int64_t plane = out_batch * g.count;
  const double pi = 3.141592653589793238462643383279502884;
  for (int64_t b = blockIdx.y; b < g.batch; b += gridDim.y) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < g.field;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const int64_t row = pitch_row(g, v), col = v - row * g.pitch;
      if (col >= g.n_last) continue;
      const int64_t i = b * g.field + v;
      T nt[D];
#pragma unroll
      for (int a = 0; a < D; ++a) nt[a] = D == 1 ? T(1) : n[a * F + i];
      if constexpr (D >= 2) {
        int sg = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) sg = sg == 0 && fabs(nt[a]) > zero ? (nt[a] > T(0) ? 1 : -1) : sg;
#pragma unroll
        for (int a = 0; a < D; ++a) nt[a] = sg < 0 ? -nt[a] : nt[a];
      }
      const double fv = static_cast<double>(f[i]);
      double q = 0.0, a2 = __dmul_rn(fv, fv), dnf = 0.0, dnq = 0.0;
#pragma unroll
      for (int a = 0; a < D; ++a) {
        const double na = static_cast<double>(nt[a]);
        const double r = static_cast<double>(r1[a * F + i]);
        q = __dadd_rn(q, __dmul_rn(na, r));
        a2 = __dadd_rn(a2, __dmul_rn(r, r));
        dnf = __dadd_rn(dnf, __dmul_rn(na, static_cast<double>(df[a * F + i])));
      }
      int p = 0;
#pragma unroll
      for (int a = 0; a < D; ++a) {
#pragma unroll
        for (int cc = a; cc < D; ++cc, ++p) {
          const double na = static_cast<double>(nt[a]), nc = static_cast<double>(nt[cc]);
          const double m = a == cc ? __dmul_rn(na, na) : __dmul_rn(2.0, __dmul_rn(na, nc));
          dnq = __dadd_rn(dnq, __dmul_rn(m, static_cast<double>(dr[p * F + i])));
        }
      }
      (void)NP;
      double phase = 0.0, freq = 0.0;
      if (a2 > tiny) {
        phase = atan2(q, fv);
        freq = __ddiv_rn(__dsub_rn(__dmul_rn(fv, dnq), __dmul_rn(q, dnf)), a2);
      }
      const int64_t at = (b0 + b) * g.count + row * g.n_last + col;
      out[at] = static_cast<T>(ldexp(__dsqrt_rn(a2), exp[b]));
      const T pt = static_cast<T>(phase);
      out[plane + at] = pt == -static_cast<T>(pi) ? static_cast<T>(pi) : pt;
      out[2 * plane + at] = static_cast<T>(freq);
      if constexpr (D >= 2) {
        const int64_t e = (b0 + b) * D * g.count + row * g.n_last + col;
#pragma unroll
        for (int a = 0; a < D; ++a) out[3 * plane + e + a * g.count] = nt[a];
        out[(3 + D) * plane + at] = c[i];
      }
    }
  }
}

}  // namespace

int64_t monogenic_work_samples(const Geom& g) {
  const int D = g.dim;
  const int64_t P = D * (D + 1) / 2;
  return 3 * g.batch * orient_layout_samples(g) + (2 * D + (D >= 2 ? P : 0) + P + (D >= 2 ? D + 1 : 0)) * g.batch * g.field;
}

template <class T>
void monogenic_fields(cudaStream_t s, const Geom& g, const OrientPlan& plan, const T* f, const int32_t* run,
                      const int32_t* exp, Elem* el, T* work, T* out, int64_t out_batch, int64_t b0, int32_t* err) {
  const int D = g.dim;
  const int64_t F = g.batch * g.field;
  const int64_t Fw = g.batch * orient_layout_samples(g);
  const int P = D * (D + 1) / 2;
  T* X = work;
  T* Y = X + Fw;
  T* Z = Y + Fw;
  T* R1 = Z + Fw;      // D fields
  T* DF = R1 + D * F;  // D fields
  T* R2 = DF + D * F;  // P fields (D >= 2)
  T* DR = R2 + (D >= 2 ? P : 0) * F;  // P fields
  T* N = DR + P * F;   // D fields (D >= 2)
  T* C = N + D * F;    // 1 field (D >= 2)
  // the mean (double), then f - mean rounded to T, then the forward DCT-II of every axis
  const int64_t nchunks = (g.field + kMeanChunk - 1) / kMeanChunk;
  double* mean = reinterpret_cast<double*>(Z);
  double* part = mean + g.batch;
  mean_partial<T><<<dim3(static_cast<unsigned>(nchunks), static_cast<unsigned>(g.batch)), 256, 0, s>>>(g, f, run, part,
                                                                                                       nchunks);
  EDAB_LAUNCH("mean_partial");
  mean_final<<<blocks_for(g.batch), 256, 0, s>>>(g.batch, g.count, run, part, nchunks, mean);
  EDAB_LAUNCH("mean_final");
  for_voxels(s, g, [=] __device__(int64_t b) { return run[b] != 0; },
             [=] __device__(int64_t b, int64_t, int64_t i) {
               Y[i] = static_cast<T>(__dsub_rn(static_cast<double>(f[i]), mean[b]));
             });
  int kinds[kMaxDim] = {0, 0, 0};
  transform_axes<T>(s, g, plan, Y, X, Z, Y, kinds, run, err);
  const dim3 grid = voxel_grid(g);
  auto component = [&](int kind, int a, int b, T* dst) {
    switch (D) {
      case 1: riesz_spectrum<T, 1><<<grid, 256, 0, s>>>(g, kind, a, b, X, Y); break;
      case 2: riesz_spectrum<T, 2><<<grid, 256, 0, s>>>(g, kind, a, b, X, Y); break;
      default: riesz_spectrum<T, 3><<<grid, 256, 0, s>>>(g, kind, a, b, X, Y); break;
    }
    EDAB_LAUNCH("riesz_spectrum");
    const int odd = (kind == 0 || kind == 3) ? (1 << a) : (a == b ? 0 : ((1 << a) | (1 << b)));
    int kk[kMaxDim] = {1, 1, 1};
    for (int ax = 0; ax < D; ++ax) kk[ax] = ((odd >> ax) & 1) ? 2 : 1;
    transform_axes<T>(s, g, plan, Y, dst, Z, Y, kk, run, err);
  };
  for (int a = 0; a < D; ++a) {
    component(0, a, a, R1 + a * F);
    component(3, a, a, DF + a * F);
  }
  int p = 0;
  for (int a = 0; a < D; ++a) {
    for (int b = a; b < D; ++b, ++p) {
      if (D >= 2) component(a == b ? 1 : 2, a, b, R2 + p * F);
      component(4, a, b, DR + p * F);
    }
  }
  if (D == 2) tensor_eigen<T, 2><<<grid, 256, 0, s>>>(g, run, R1, R2, N, N + F, nullptr, C, el);
  else if (D == 3) tensor_eigen<T, 3><<<grid, 256, 0, s>>>(g, run, R1, R2, N, N + F, N + 2 * F, C, el);
  if (D >= 2) EDAB_LAUNCH("tensor_eigen");
  const double tiny = std::is_same_v<T, float> ? 1.17549435082228750797e-38 : 1e-300;
  const T zero = static_cast<T>(std::is_same_v<T, float> ? std::ldexp(1.0, -14) : std::ldexp(1.0, -30));
  switch (D) {
    case 1: monogenic_kernel<T, 1><<<grid, 256, 0, s>>>(g, f, R1, DF, DR, N, C, exp, tiny, zero, out, out_batch, b0); break;
    case 2: monogenic_kernel<T, 2><<<grid, 256, 0, s>>>(g, f, R1, DF, DR, N, C, exp, tiny, zero, out, out_batch, b0); break;
    default: monogenic_kernel<T, 3><<<grid, 256, 0, s>>>(g, f, R1, DF, DR, N, C, exp, tiny, zero, out, out_batch, b0); break;
  }
  EDAB_LAUNCH("monogenic_kernel");
}

template void monogenic_fields<float>(cudaStream_t, const Geom&, const OrientPlan&, const float*, const int32_t*,
                                      const int32_t*, Elem*, float*, float*, int64_t, int64_t, int32_t*);
template void monogenic_fields<double>(cudaStream_t, const Geom&, const OrientPlan&, const double*, const int32_t*,
                                       const int32_t*, Elem*, double*, double*, int64_t, int64_t, int32_t*);

template void orientation<float>(cudaStream_t, const Geom&, const OrientPlan&, const float*, Elem*, const int32_t*,
                                 float* const*, float*, float*, double, int32_t*);
template void orientation<double>(cudaStream_t, const Geom&, const OrientPlan&, const double*, Elem*, const int32_t*,
                                  double* const*, double*, double*, double, int32_t*);

}  // namespace edab
