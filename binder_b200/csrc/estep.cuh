// E-step (EM and Gibbs), theta updates, prior-precision sampling, Welford moments.
#pragma once

#include "transform.cuh"

namespace binder {

// A 2D image nx x ny is passed as the volume nx x 1 x ny (ny, nyn = 1): its y axis is the packed
// (z) axis of the bin volume and positions have N = dim = 2 components (x, y).
struct SsdfState;

struct EStepArgs {
    const float *d;   // positions, SoA [dim][V] (node-grid coordinates)
    float *r;         // out: dream location minus voxel position, SoA [dim][V]
    const float *x;   // voxel positions SoA [dim][V], or null for the identity grid
    const uint8_t *u;     // fixed-image bins [V]
    const uint8_t *vpad;  // moving-image bins, zero-padded [nxn+2P][nyn+2P][zp bytes]
    const float *theta;   // [K*L]
    float *hist;          // EM: soft joint histogram [K*L] (accumulated)
    // the single-pass EM kernel's order-independent merge (all three null: FP32 atomics instead):
    // 64-bit fixed-point sums [K*L] (zero between launches), one log-likelihood partial per CTA
    // [kMaxEmCtas], and the count of CTAs done (zero between launches)
    unsigned long long *hfix;
    double *mpart;
    unsigned *hdone;
    unsigned *hcnt;       // Gibbs: joint counts [K*L] (accumulated)
    DevState *st;
    const int *skip;
    long V;
    int nx, ny, nz;
    int nxn, nyn, nzn;
    int P, PZ, pyn, zp;
    int K, L;
    int dim;    // 2 or 3
    int order;  // spline order 1, 2 or 3 (Spline.cpp:9-41), on the stencil of offsets -1 .. 2
    // log-space likelihood (the SSD likelihood): `theta` holds log2 likelihoods normalised per
    // voxel bin l by their maximum over k, whose natural log is colmax[l]
    int logt;
    const float *colmax;
    // the MI filter likelihood (M > 1 channels, or M == 1 with filter set): `u` and `vpad` hold
    // one volume per channel, uch / vch bytes apart; theta and hist are [M][K][L]
    int M;
    int filter;
    long uch, vch;
    // the SSD filter likelihood: voxel features [M][V] and node features [Fn][Vn] (FP64 SoA,
    // node index in the E-step's view), its state and the E-step's statistics
    int ssdf;
    int Fn;
    const double *fx;
    const double *fn;
    SsdfState *fstate;
    double *fstats;
    uint64_t seed;
    uint32_t chain;
    // the single-pass EM kernel of the MI likelihood (K <= 64): 1 = FP16 per-thread bin columns
    // (three CTAs per SM; each voxel's per-bin posterior mass rounded to FP16), 0 = FP32
    int halfcol;
    // set by launch_estep: fixed-point scale of the EM kernel's per-CTA histogram and its inverse
    // (FP64, so that the kernel multiplies: an FP64 division in the kernel's tail measured twice as
    // slow a whole launch)
    float hscale;
    double hinv;
};

// CTAs of the single-pass EM kernel at most when it merges in fixed order (EStepArgs::mpart)
constexpr int kMaxEmCtas = 2048;
// chains > 1: a batch of chains, the sampling E-step only (chain = blockIdx.y; buffers
// [chains][dim][V] positions / dream locations, [chains][K][L] theta / counts, [chains] states)
void launch_estep(const EStepArgs &a, bool sample, int grid, cudaStream_t s, int chains = 1);
// grid of one wave; half: for the FP16-column EM kernel (EStepArgs::halfcol)
int estep_grid(bool sample, int K, int L, long V, int dim, bool logt = false, bool half = false);
// largest number of bins of the log-space (SSD) E-step
constexpr int kLogMaxBins = 64;
// largest number of channels of the MI filter likelihood, and of M * K * L (its shared-memory
// theta and histograms)
constexpr int kMaxChannels = 8;
constexpr long kFilterMaxCells = 24576;
int estep_filter_grid(int K, int L, int M, long V, int dim, bool sample = false);
// whether the sampling E-step of the MI filter likelihood fits in shared memory (theta, counts
// and its per-thread draw table)
bool filter_sampling_fits(int K, int L, int M);

// State of the SSD filter likelihood (BINDER/src/cpu/SSDLikelihoodFilter.cpp): M fixed-image
// channels, F moving-image features (Fn = F, or M with reg_across_features, whose prediction of
// channel m at a node is its feature m: coefficients = identity), coeff [M][F], sigma [M], the
// inverse-gamma prior, and what the E-step reads.
constexpr int kSsdfMax = 8;
struct SsdfState {
    double coeff[kSsdfMax * kSsdfMax];
    double sigma[kSsdfMax];
    double alpha0, beta0;
    double lc;                        // sum_m -log(2 pi sigma_m) / 2
    double cf[kSsdfMax * kSsdfMax];   // prediction coefficients [M][Fn]
    double h[kSsdfMax];               // 1 / (2 sigma_m)
    int M, F, Fn, rfa;
};
// E-step statistics: A [Fn][Fn] = sum p n n^T, b [M][Fn] = sum p x_m n, S2 [M] = sum p x_m^2,
// eff = sum p (n the node's features, 0 outside the grid)
constexpr int kSsdfA = 0, kSsdfB = 64, kSsdfS2 = 128, kSsdfEff = 136, kSsdfStats = 137;
void ssdf_refresh_host(SsdfState &p);  // cf, h, lc from coeff, sigma
int estep_ssdf_grid(int M, int Fn, long V, int dim, bool sample = false);
// update_parameters (when update) and compute_cost of the SSD filter likelihood from stats,
// which it clears; the cost goes to st->lp_lik
void launch_ssdf_update(SsdfState *p, double *stats, int update, DevState *st, cudaStream_t s);
// the sampler's draw of the SSD filter likelihood's coefficients and sigmas
// (SSDLikelihoodFilter.cpp:459-463) from the sweep's statistics, which it clears; Philox ctr
// {index, st->sweep, 8 / 9, chain}; the prior cost into st->lp_lik.  One CTA.
void launch_ssdf_sample(SsdfState *p, double *stats, DevState *st, uint64_t seed,
                        uint32_t chain, cudaStream_t s);
// [n][C] features (device memory) to SoA [C][n]
void launch_features_to_soa(const double *in, long n, int C, double *out, cudaStream_t s);

// State of the SSD likelihood (BINDER/src/cpu/SSDLikelihood.cpp): sigma^2, shift, scale and the
// inverse-gamma prior (alpha0, beta0) of sigma^2
struct SsdState {
    double sigma2, shift, scale, alpha0, beta0;
    int shift_scale;
    int pad;
};
// SSDLikelihood::update_parameters from the joint histogram when `update` (:143-285), the cost
// of sigma^2 into st->lp_lik (:314-326), the log2 likelihood table [K][L] (normalised per column)
// and its column maxima rebuilt from the parameters, and the histogram cleared.  st may be null
// (table only, no histogram).  One CTA.
void launch_ssd_update(float *table, float *colmax, float *hist, int K, int L, int update,
                       SsdState *p, DevState *st, cudaStream_t s);

// the sampler's draw of the SSD likelihood's parameters (SSDLikelihood.cpp:284-302) from the
// sweep's counts hcnt [K][L] (Philox ctr {0, st->sweep, 6 / 7, chain}), the log2 table and its
// column maxima rebuilt, the counts cleared; the prior cost into st->lp_lik.  One CTA.
void launch_ssd_sample(float *table, float *colmax, unsigned *hcnt, int K, int L, SsdState *p,
                       DevState *st, uint64_t seed, uint32_t chain, cudaStream_t s);

// theta <- (hist + alpha - 1)/rowsum (if update), Dirichlet prior cost into st->lp_lik,
// hist zeroed for the next iteration.  One CTA.
void launch_theta_update(float *theta, float *hist, int K, int L, double alpha, int update,
                         DevState *st, cudaStream_t s);
// theta_k ~ Dirichlet(counts_k + alpha) with Philox gammas (tag 4, sweep = st->sweep); counts zeroed
void launch_dirichlet_sample(float *theta, unsigned *hcnt, int K, int L, double alpha,
                             uint64_t seed, uint32_t chain, DevState *st, cudaStream_t s,
                             int chains = 1);
// nu ~ Gamma(alpha0 + N V/2, beta0 + V/2 raw) when sample_gamma and sweep % every == 0;
// gammas refreshed from nu.  Also resets raw_reg.
void launch_nu_sample(DevState *st, int sample_gamma, int every, int N, long V, double rho_p,
                      const double eta2[3], uint64_t seed, uint32_t chain, cudaStream_t s,
                      int chains = 1);
// EM bookkeeping: min-log-posterior, per-iteration stats, convergence flag
void launch_em_finish(DevState *st, double *stats, int max_iter, double th, double nzv,
                      cudaStream_t s);
// Welford mean [N][V] / symmetric M2 [N (N + 1) / 2][V] update in FP64 when sweep >= N_b, then
// sweep += 1 (done once sweep reaches `total`)
void launch_sweep_end(const float *d, double *mean, double *m2, long V, int N, int N_b,
                      int total, DevState *st, cudaStream_t s, int chains = 1);
// sweep += 1 (done once sweep reaches `total`)
void launch_sweep_advance(DevState *st, int total, cudaStream_t s, int chains = 1);

}  // namespace binder
