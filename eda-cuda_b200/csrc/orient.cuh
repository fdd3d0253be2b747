// SPDX-License-Identifier: Apache-2.0
// The monogenic orientation of a mode (D >= 2): the band of the orthonormal N-D DCT-II of the
// residual, its first- and second-order Riesz components, the energy tensor and its
// eigen-decomposition into the dominant direction n and the coherence c
// (cpp/src/method/orientation.cu:1-37, 98-127, 199-404 and cpp/src/method/element.cu:49-164 of
// eda-cuda). The reference computes the transforms with cuFFT (Makhoul's permutation); here every
// transform is a dense matrix product along each axis: the forward DCT-II basis C, and for the
// inverse the cosine basis C^T on the even axes of a component and the sine basis S^T on its odd
// axes (S[k][x] = c_k sin(pi k (2x + 1) / 2n), the inverse DCT of the reversed spectrum times
// (-1)^x), so the whole orientation is GEMM-shaped work.
#pragma once

#include "engine.cuh"

namespace edab {

struct OrientPlan {
  int dim = 0;
  int32_t n[kMaxDim] = {1, 1, 1};
  bool f64 = false;
  int device = 0;
  // per axis, n x n row-major in the dtype: forward (row k, column x), inverse cosine (row x,
  // column k), inverse sine (row x, column k)
  void* fwd[kMaxDim] = {nullptr, nullptr, nullptr};
  void* icos[kMaxDim] = {nullptr, nullptr, nullptr};
  void* isin[kMaxDim] = {nullptr, nullptr, nullptr};
  // float32 only, for the tensor cores: the same bases split into tf32 hi and lo parts,
  // [2][npad][kpad] (hi rows, then lo rows; zero beyond n), kpad = n rounded up to 32, npad to 128
  void* tc_fwd[kMaxDim] = {nullptr, nullptr, nullptr};
  void* tc_icos[kMaxDim] = {nullptr, nullptr, nullptr};
  void* tc_isin[kMaxDim] = {nullptr, nullptr, nullptr};
  // the same split into bfloat16 hi and lo parts (BF16x3), [2][npad][kpad] bfloat16
  void* bf_fwd[kMaxDim] = {nullptr, nullptr, nullptr};
  void* bf_icos[kMaxDim] = {nullptr, nullptr, nullptr};
  void* bf_isin[kMaxDim] = {nullptr, nullptr, nullptr};
  int32_t kpad[kMaxDim] = {0, 0, 0};
  int32_t npad[kMaxDim] = {0, 0, 0};
};

// The product of the float32 transforms (process-wide; float64 always runs the FP64 product):
// 3xTF32 and BF16x3 split products on the tensor cores, or the plain float32 SIMT product.
enum class TransformPrecision : int { kTf32x3 = 0, kBf16x3 = 1, kFp32 = 2 };
TransformPrecision transform_precision();
void set_transform_precision(TransformPrecision p);
// The plan of a geometry and dtype on the current device (cached for the life of the process).
const OrientPlan& orient_plan(const Geom& g, bool f64);
// Samples of the orientation's work area: three ping-pong fields large enough for every rotated
// layout of an element (the spectrum, the component spectrum, a pass buffer), then R1 (D fields) and
// R2 (D (D + 1) / 2 fields) in the element layout.
int64_t orient_work_samples(const Geom& g);

// One axis pass of a rotated layout: the layout's contiguous axis (extent K, rows pitch_in apart,
// `rows` rows per element, element fields f_in apart) is transformed and stored with that axis
// first and the previous second-fastest axis (extent n_lo, padded to pitch_out) contiguous: row r =
// hi * n_lo + lo of element b stores column j at b * f_out + j * s_j + hi * pitch_out + lo.
struct RotPass {
  int64_t M;  // rows of the batch
  int32_t K;
  int64_t pitch_in, rows, f_in, n_lo, pitch_out, s_j, f_out;
};
// The pass on the tensor cores (float32 data): basis [2][npad][kpad] hi / lo parts, float32 tf32
// values (3xTF32) or bfloat16 (bf16: BF16x3); *err set when a bounded wait of the kernel expired.
void rot_pass_tc(cudaStream_t s, const RotPass& p, const void* basis, bool bf16, int32_t kpad, int32_t npad,
                 const float* in, float* out, const int32_t* run, int32_t* err);

// The separable transform of every element with run[b] along all axes (last axis first), kinds[a]
// = 0 forward DCT-II, 1 inverse cosine, 2 inverse sine basis on axis a: in (element layout) -> out
// (element layout) through D rotated passes, ping-ponging between buf0 and buf1 (each holding
// every rotated layout of the batch; in may be buf1, and is then overwritten).
template <class T>
void transform_axes(cudaStream_t s, const Geom& g, const OrientPlan& plan, const T* in, T* out, T* buf0, T* buf1,
                    const int* kinds, const int32_t* run, int32_t* err);
int64_t orient_layout_samples(const Geom& g);  // the largest rotated layout of one element

// n[0..D-1] and coh of every element with run[b]; el[b].w is the band's window; a non-finite
// tensor sets el[b].nonfinite.
template <class T>
void orientation(cudaStream_t s, const Geom& g, const OrientPlan& plan, const T* r, Elem* el, const int32_t* run,
                 T* const* n, T* coh, T* work, double two_sigma2, int32_t* err);

// eda.monogenic of the prescaled fields f (element layout; f = x 2^-exp[b]) of the elements with
// run[b]: the planes of out (out_batch elements; this chunk at b0): amplitude, phase, frequency
// [out_batch][count], then in 2-D / 3-D direction [out_batch][D][count] and coherence. work holds
// monogenic_work_samples(g) samples.
int64_t monogenic_work_samples(const Geom& g);
template <class T>
void monogenic_fields(cudaStream_t s, const Geom& g, const OrientPlan& plan, const T* f, const int32_t* run,
                      const int32_t* exp, Elem* el, T* work, T* out, int64_t out_batch, int64_t b0, int32_t* err);

}  // namespace edab
