// Preprocessing and output steps of BINDER's registration driver on the GPU:
//   - utils.bin_signal_robust / utils.bin_signal (BINDER/utils.py:12-82): intensity binning;
//   - the centre of mass of the non-zero bins (BINDER/FastRegistration.py:387-395, scipy's
//     center_of_mass of a boolean mask);
//   - utils.save_warped_image's resampling of the moving image through the final positions
//     (BINDER/utils.py:222-227: skimage.transform.warp, order 0, 1 or 3, constant zero outside).
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace binder {

// Robust min / max from a 1000-bin histogram of [min, max] (numpy's histogram arithmetic in the
// signal's own type T), then floor((x - lo) / width) clamped to [0, number_of_bins - 1].  signal
// and binned may be host or device memory; edges (number_of_bins + 1 values, in T widened to
// double) may be null.  T = float or double.
template <typename T>
void bin_signal_robust(const T *signal, long n, int number_of_bins, double lower_percentile,
                       double higher_percentile, int32_t *binned, double *edges);
// round-half-to-even((x - min) / ((max - min) / (number_of_bins - 1)))
template <typename T>
void bin_signal(const T *signal, long n, int number_of_bins, int32_t *binned);

// centre of mass (index space) of the voxels with bins > 0; false when there is none
bool center_of_mass_nonzero(const int32_t *bins, int nx, int ny, int nz, double out[3]);

// out[m] = image sampled at positions[m] (AoS [M][3], index space) with order 0 (nearest), 1
// (trilinear) or 3 (cubic B-spline, spline-prefiltered) interpolation, zero outside the image,
// clipped as skimage clips warp output.
// image [nx][ny][nz], out [M]; host or device memory.
void warp_image(const double *image, int nx, int ny, int nz, const double *positions, long M,
                int order, double *out);

}  // namespace binder
