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

/* The exact selection of every element of x_dev (dense (batch, n..), dtype 0 float32 / 1 float64,
 * on the current device): src 0 selects the samples (those with (mask & bits) != 0 when mask_dev, a
 * dense u8 array of the same shape, is given), src 1 the forward differences x[i + e_a] - x[i] in the
 * dtype along every axis a in the bit set `axes`; center (host, [batch], or NULL) selects
 * |value - center[b]| in double instead. q < 0: NumPy's median; 0 <= q <= 1: NumPy's "linear"
 * quantile; out (host, [batch]) receives it (NaN for an empty set), count (host, [batch], or NULL)
 * the number of items. Replaces the harness calls of enqueue_median / enqueue_quantile
 * (cpp/src/method/stats.cu:221-296; tested in cpp/tests/test_stats.cu:130-326). Synchronizes. */
EDA_API int eda_testing_select(const void* x_dev, int dtype, int dim, int64_t batch, const int64_t* n, int src,
                               int axes, const uint8_t* mask_dev, int bits, const double* center, double q,
                               double* out, int64_t* count, void* stream);

/* The significant extrema of every line of every axis of r_dev against the threshold field tau_dev
 * (both dense (batch, n..) of the dtype on the current device): flags_dev (dense u8) receives bit a
 * for an extremum of a line along axis a (SciPy's find_peaks with topographic prominence >= tau at
 * the peak), ext (host, [batch][dim]) their counts. Replaces the harness calls of enqueue_sig_flags
 * (cpp/src/method/stats_fields.cu:392-422; tested in cpp/tests/test_stats.cu:436-902). Synchronizes. */
EDA_API int eda_testing_flags(const void* r_dev, const void* tau_dev, int dtype, int dim, int64_t batch,
                              const int64_t* n, uint8_t* flags_dev, uint64_t* ext, void* stream);

/* The face-connected components of (mask & bits) != 0 of every element of mask_dev (dense u8
 * (batch, n..) on the current device): labels_dev (dense int32) receives the smallest dense index
 * of the sample's component inside its element, -1 outside. Replaces the harness calls of
 * enqueue_ccl (cpp/src/method/stats_scale.cu:208-220; tested in cpp/tests/test_stats.cu:966-1050).
 * Synchronizes. */
EDA_API int eda_testing_components(const uint8_t* mask_dev, int bits, int dim, int64_t batch, const int64_t* n,
                                   int32_t* labels_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EDA_B200_TESTING_H_ */
