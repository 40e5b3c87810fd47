// The whole DCT-prior M-step of a small 2D image in one launch (see mstep2d.cu).
#pragma once

#include "transform.cuh"

namespace binder {

// largest axis of the fused 2D M-step (the n x n matrix is staged in one CTA's shared memory)
constexpr int kM2dMaxN = 128;

// d = IDCT(DCT(r) / (1 + gamma sigma^2 D) [+ noise]) + x for both components of an nx x ny image
// (SoA [2][nx*ny]), costs into st: the pass sequence y, x (scaled), x^-1, y^-1 of the M-step.
// a: the spectral and positions fields of AxisArgs (D, st, sigma2, sample, want_raw, every,
// seed, chain, rho_p, eta2, xpos, skip, comp_stride = nx*ny); Fx, Fy: DCT-II matrices [k][j];
// Ix, Iy: their transposes.
void launch_mstep2d(const AxisArgs<float> &a, const float *r, float *d, int nx, int ny,
                    const float *Fx, const float *Ix, const float *Fy, const float *Iy,
                    cudaStream_t s);

}  // namespace binder
