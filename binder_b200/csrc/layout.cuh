// Device memory and host <-> device layout conversion shared by the engines.
//
// Allocation: every device buffer of the engines comes from the device's stream-ordered memory
// pool (cudaMallocAsync / cudaFreeAsync) with its release threshold raised once per device, so
// memory freed by one Registration is kept by the pool and handed to the next without a trip
// through the driver (a plain cudaFree also synchronises the whole device).
//
// Layout: the C ABI exchanges position fields as AoS [V][3] host arrays; the engines keep SoA
// [3][V] device arrays.  Inputs are copied to the device as they are (from the caller's memory,
// pinned or not) and rearranged there by the kernels below; outputs are rearranged on the device
// and copied back in one transfer.
#pragma once

#include "common.cuh"

namespace binder {

// stream-ordered allocation of `bytes` from the current device's pool (nullptr for 0 bytes)
void *dev_alloc(size_t bytes, cudaStream_t s);
// stream-ordered release into the pool (no-op for nullptr)
void dev_free(void *p, cudaStream_t s);

template <typename T>
T *dev_alloc_n(size_t n, cudaStream_t s) {
    return static_cast<T *>(dev_alloc(n * sizeof(T), s));
}
template <typename T>
void dev_free_p(T *&p, cudaStream_t s) {
    dev_free(p, s);
    p = nullptr;
}

// identity voxel grid of an nx x ny x nz volume with N components per voxel (N = 3; a 2D image
// nx x ny is described as nx x ny x 1 with N = 2): component c of voxel i is its c-th index
struct GridDims {
    int nx, ny, nz;
    int N;
};

// soa[c][i] = aos[i][c] (float, N components)
void launch_aos_to_soa(const float *aos, float *soa, long V, int N, cudaStream_t s);
// aos[i][c] = soa[c][i]
void launch_soa_to_aos(const float *soa, float *aos, long V, int N, cudaStream_t s);
// aos[i][c] = soa[c][i] + base[c][i], base = x (SoA) or, when x is null, the identity grid
void launch_soa_to_aos_plus(const float *soa, const float *x, GridDims g, float *aos,
                            cudaStream_t s);
// soa[c][i] = aos[i][c] - base[c][i] (base as above); `aos` may be null for an all-zero input
void launch_aos_minus_to_soa(const float *aos, const float *x, GridDims g, float *soa,
                             cudaStream_t s);
// *mismatch |= 1 unless aos[i][c] equals the identity grid coordinate exactly for every i, c
void launch_identity_check(const float *aos, GridDims g, unsigned *mismatch, cudaStream_t s);
// out[i] = in[i] as bytes for in[i] in [0, limit); *first_bad = min index with in[i] outside
void launch_bins_to_u8(const int *in, long n, int limit, uint8_t *out,
                       unsigned long long *first_bad, cudaStream_t s);
// bins of an nx x ny x nz node grid into the interior of the zero-padded byte volume
// vpad[(x + P) * pyn + (y + Py)][z + PZ] (row length zp); range check as above
void launch_bins_to_padded(const int *in, int nx, int ny, int nz, int limit, uint8_t *vpad, int P,
                           int Py, int PZ, int pyn, int zp, unsigned long long *first_bad,
                           cudaStream_t s);
// Welford outputs: mean_aos[i][c] = mean[c][i]; cov_aos[i][r][c] = m2[sym(r, c)][i] * scale, M2
// stored as its upper triangle (xx, xy, xz, yy, yz, zz for N = 3; xx, xy, yy for N = 2)
void launch_moments_to_aos(const double *mean, const double *m2, long V, int N, double scale,
                           double *mean_aos, double *cov_aos, cudaStream_t s);
// C chains' FP64 moments (mean [C][N][V], upper-triangle M2 [C][N (N + 1) / 2][V], n samples per
// chain) pooled into one mean [V][N] and covariance [V][N][N] (M2 / (C n - 1))
void launch_pool_moments(const double *mean, const double *m2, long V, int N, int C, double n,
                         double *mean_aos, double *cov_aos, cudaStream_t s);

}  // namespace binder
