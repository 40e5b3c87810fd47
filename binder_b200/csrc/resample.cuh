// Resampling of position / displacement fields between grid sizes (the multi-resolution step of
// BINDER/FastRegistration.py:550-650), FP64.
//
// Every resampling the reference performs there is separable and linear along each axis:
//   - NonLinearTransformation::up_sample (BINDER/src/cpu/NonLinearTransformation.cpp:366-430):
//     orthonormal DCT-II on the input grid, coefficients copied into the low corner of a zero
//     output spectrum, orthonormal DCT-III on the output grid -- per axis the m x n matrix
//     C_m^T[:, :n] C_n;
//   - skimage.transform.resize(order=1) as FastRegistration.py:562-564 calls it (mode 'reflect',
//     anti-aliasing on when any axis shrinks): a Gaussian pre-filter with sigma = (n/m - 1)/2 on
//     each shrinking axis (scipy.ndimage.gaussian_filter, truncate 4, 'mirror' boundary), then
//     scipy.ndimage.zoom(order=1, grid_mode=True, mode='mirror') -- per axis the m x n matrix
//     Z G.
// So one kernel applies a dense m x n matrix along one axis of an AoS field, and a resample is
// three such passes (z, y, x) with per-axis matrices built once on the host.
#pragma once

#include <vector>

#include "common.cuh"

namespace binder {

// m x n row-major: up-sampling by spectral zero padding (n <= m)
void dct_upsample_matrix(int n, int m, std::vector<double> &U);
// m x n row-major: order-1 resize along one axis with the anti-aliasing pre-filter when m < n
void linear_resize_matrix(int n, int m, std::vector<double> &R);

// Separable map of an AoS field [nx][ny][nz][N] (device, FP64) to [mx][my][mz][N]; Mx/My/Mz are
// device m_a x n_a matrices, or null where the axis keeps its length and the map is the
// identity.  tmp1 and tmp2 each hold nx*max(ny,my)*max(nz,mz)*N doubles.
void separable_apply(const double *in, int nx, int ny, int nz, int N, const double *Mx,
                     const double *My, const double *Mz, int mx, int my, int mz, double *out,
                     double *tmp1, double *tmp2, cudaStream_t s);

// Per-axis matrices of one resample kind, resident on the device for a fixed pair of grids.
class Resampler {
  public:
    enum Kind { kUpSample = 0, kLinear = 1 };
    Resampler(Kind kind, const int in[3], const int out[3], int N, cudaStream_t s);
    ~Resampler();
    Resampler(const Resampler &) = delete;
    Resampler &operator=(const Resampler &) = delete;
    // in [n][N] -> out [m][N] (AoS FP64, device); out may not alias in
    void apply(const double *in, double *out, cudaStream_t s);

  private:
    void release();
    int n_[3], m_[3], N_;
    double *M_[3] = {nullptr, nullptr, nullptr};
    double *tmp1_ = nullptr, *tmp2_ = nullptr;
    cudaStream_t s_;
};

// soa [N][nx*ny*nz] (FP32, device) += the order-1 resize (resize_linear, scale 1) of the AoS FP32
// displacement field [fx][fy][fz][N] (host or device memory) to the nx x ny x nz grid; stream s
// (synchronised before returning)
void add_resized_displacement(const float *field, int fx, int fy, int fz, int N, int nx, int ny,
                              int nz, float *soa, cudaStream_t s);

// Host-to-host entry points (own stream, device buffers from the pool).
// NonLinearTransformation.up_sample: N = 2 when mz == 1
void up_sample(const double *field, int nx, int ny, int nz, int mx, int my, int mz, double *out);
// skimage.transform.resize(field, (mx, my, mz), order=1) * scale on an AoS field with N components
void resize_linear(const double *field, int nx, int ny, int nz, int N, int mx, int my, int mz,
                   double scale, double *out);

}  // namespace binder
