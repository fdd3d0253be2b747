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
};
// The plan of a geometry and dtype on the current device (cached for the life of the process).
const OrientPlan& orient_plan(const Geom& g, bool f64);
// Work fields of the orientation: the spectrum, the component spectrum, a transpose buffer, R1 (D),
// R2 (D (D + 1) / 2).
inline int orient_work_fields(int D) { return 3 + D + D * (D + 1) / 2; }

// n[0..D-1] and coh of every element with run[b]; el[b].w is the band's window; a non-finite
// tensor sets el[b].nonfinite.
template <class T>
void orientation(cudaStream_t s, const Geom& g, const OrientPlan& plan, const T* r, Elem* el, const int32_t* run,
                 T* const* n, T* coh, T* work, double two_sigma2);

}  // namespace edab
