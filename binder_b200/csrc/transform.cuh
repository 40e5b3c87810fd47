// Separable 3D transforms as mode-n products (one axis per pass) with fused epilogues.
//
// A pass multiplies every line of a volume along one axis by an n x n matrix M (rows = output
// index): y[.., k, ..] = sum_j M[k][j] x[.., j, ..].  The volume is C-order [nx][ny][nz]; an axis
// is described by (n, outer, s): element (o, j, t) sits at o*n*s + j*s + t.  The contiguous axis
// (s == 1) is tiled by rows, the strided axes by 64-wide column tiles; either way a CTA stages an
// n x 64 slab in shared memory and runs a register-blocked SIMT product over it.
#pragma once

#include "common.cuh"

namespace binder {

// device-side state of one registration/sampling run (FP64 accumulators, RNG-updated gammas)
struct DevState {
    double mll;            // -sum log normaliser (E-step)
    double lp_lik;         // Dirichlet prior cost of theta
    double lp_tr;          // deformation prior cost (spectral epilogue)
    double raw_reg;        // sum eta^2 rho D c^2 (sampling of nu)
    double mlp_old;        // previous min-log-posterior (EM convergence)
    double gamma[3];       // current per-component regularisation
    double nu;             // precision hyper-parameter (sampling)
    unsigned long long degenerate;  // voxels whose normaliser was <= 0
    int done;              // EM converged / iteration budget exhausted
    int iter;              // EM iterations completed
    unsigned flags;        // DeviceFlag bits
    int sweep;             // Gibbs sweep counter (Philox counter and Welford count)
};

enum EpilogueMode : int {
    kEpiNone = 0,       // plain store
    kEpiSpectral = 1,   // fused fwd -> DCT-prior scaling (+noise, costs) -> inverse (x axis)
    kEpiPositions = 2,  // store y + x_grid (final inverse pass) into the position field
    kEpiPoisson = 3,    // fused fwd -> -1/lambda (Hartley Poisson) -> inverse (x axis)
    kEpiTopoOut = 4,    // store u * scale + mean into a physical-position field (FP64)
    kEpiSpectralOut = 5,  // forward pass whose epilogue applies the prior scaling and stores it
    kEpiPoissonFwd = 6,   // forward pass whose epilogue applies -1/lambda and stores it (FP64)
};

template <typename T>
struct AxisArgs {
    const T *in;
    T *out;
    long comp_stride;  // elements between components (V)
    int comp0;         // component of blockIdx.z == 0 (the tensor-core passes run one per launch)
    const T *M;        // n x n, row-major
    const T *M2;       // second matrix of a fused pass (inverse), n x n
    int n;
    long outer, s;
    // spectral epilogue (DCT prior)
    const float *D;
    DevState *st;
    double sigma2;
    int sample;            // add prior-sampling noise (Philox counter sweep = st->sweep)
    // the noise precomputed by launch_prior_noise ([components][V], the launch's component
    // index), or null: the pass then draws it per element
    const float *noise;
    int want_raw;          // accumulate the raw regulariser when st->sweep % every == 0
    int every;
    uint64_t seed;
    uint32_t chain;
    double rho_p;
    double eta2[3];
    // positions epilogue
    const float *xpos;  // SoA voxel positions or null for the identity grid
    int ny, nz;
    int dims;           // 3, or 2 for an nx x ny image (nz = 1, components x, y)
    // Poisson epilogue: the periodic Laplacian symbol is 6 - 2cos_x - 2cos_y - 2cos_z
    const double *cos_x, *cos_y, *cos_z;  // cos(2 pi k / n) per axis
    double out_scale[3];   // kEpiTopoOut: per-component scale (voxel size / total)
    double out_offset[3];  // kEpiTopoOut: per-component offset (mean)
    const int *skip;       // when non-null and *skip != 0 the pass is a no-op
    // a batch of chains: components chain * chain_comps + n (n < chain_comps) with states
    // st[chain] and Philox chain indices chain + chain; 0 for one chain
    int chain_comps;
};

// The prior-sampling normals of every coefficient: noise[c * V + i] = dct_prior_normal(seed, i,
// st[c / chain_comps].sweep, chain + c / chain_comps, c % chain_comps) for the ncomp components
// of a launch (chain_comps 0: one chain, ncomp components); components 0 and 1 share one Philox
// draw (the cosine and the sine of one Box-Muller pair), as dct_prior_normal draws them.  A no-op
// when *skip.
void launch_prior_noise(float *noise, long V, int ncomp, int chain_comps, uint64_t seed,
                        uint32_t chain, const DevState *st, const int *skip, cudaStream_t s);

// Launch one pass over `ncomp` components (blockIdx.z = component).
template <typename T>
void launch_axis_pass(const AxisArgs<T> &a, int mode, int ncomp, cudaStream_t stream);

// host-built orthonormal DCT-II matrix (rows = frequency) in double precision
void dct2_matrix(int n, double *out);
// host-built Hartley matrix cas(2 pi jk / n)
void hartley_matrix(int n, double *out);

}  // namespace binder
