/* SPDX-License-Identifier: Apache-2.0
 *
 * eda_b200 testing hooks: single stages of the engine on a dense batch, for stage-level parity
 * tests against a CPU restatement. Not part of the decomposition interface (include/eda_b200.h);
 * the reference tests the same stages through C++ harnesses against host twins
 * (cpp/tests/test_cube.cu of giorgioangel/eda-cuda).
 */
#ifndef EDA_B200_TESTING_H_
#define EDA_B200_TESTING_H_

#include "eda_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The cube filter (op 0 max, 1 min, 2 max and min, 3 box mean) of every element of x_dev, a dense
 * C-contiguous (batch, n[0], .., n[dim-1]) array of float32 (dtype 0) or float64 (dtype 1) on the
 * current device, for `rungs` windows per element: win is a host array [rungs][batch] of odd
 * windows (< 1: the element is skipped and its output holds NaN). out0_dev (and out1_dev, the min
 * of op 2) receive dense (rungs, batch, n..) arrays. Rung 0 of every cube runs through the first
 * pass's rung loop and the later axes one rung per CTA, as the engine's operators run them. Replaces
 * the harness calls of enqueue_cube / enqueue_cube_rungs (cpp/src/method/method.hpp; tested in
 * cpp/tests/test_cube.cu:52-205). Synchronizes the stream. */
EDA_API int eda_testing_cube(const void* x_dev, int dtype, int dim, int64_t batch, const int64_t* n, int op,
                             const int32_t* win, int32_t rungs, void* out0_dev, void* out1_dev, void* stream);

/* The separable orthonormal transform of the orientation along every axis of every element of x_dev
 * (dense (batch, n[0], .., n[dim-1]), dim 2 or 3, on the current device): kinds[a] selects axis a's
 * basis, 0 the forward DCT-II C[k][x] = c_k cos(pi k (2x + 1) / 2n), 1 the inverse cosine C^T, 2
 * the inverse sine S^T with S[k][x] = c_k sin(pi k (2x + 1) / 2n); out_dev receives the dense result.
 * Float32 runs the tensor-core passes (3xTF32), float64 the FP64 product. Replaces the harness calls
 * of the reference's DCT stage (cpp/src/field/dct.*, tested in cpp/tests/test_orientation.cu).
 * Synchronizes the stream. */
EDA_API int eda_testing_transform(const void* x_dev, int dtype, int dim, int64_t batch, const int64_t* n,
                                  const int32_t* kinds, void* out_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EDA_B200_TESTING_H_ */
