/*
 * FP64 CPU oracle for the BINDER registration + Gibbs-sampling hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is compared against: only
 * tests/, __graft_entry__.smoke() and the cpu_baseline / reference leg of bench.py may load it.
 * The product (binder_b200) never links, loads or calls it.
 *
 * It restates, in plain C with double precision, the algorithms of the reference CPU backend
 * (ste93ste/BINDER, BINDER/src/cpu/...), each function citing the file:line it follows.  Where the
 * reference draws random numbers with std::mt19937, the oracle instead uses the Philox4x32-10
 * counter-based stream that the CUDA path uses (same counters, same keys), so sampler results are
 * reproducible draw-for-draw between oracle and GPU; parity with the reference's own sampler is
 * distributional (Monte-Carlo), as it is between the reference's CPU and GPU backends.
 *
 * Layouts follow the reference: position fields are [Nx][Ny][Nz][N] C-order interleaved (AoS),
 * N = 3 (or 2 when Nz == 1); bin volumes are int32 [Nx][Ny][Nz]; theta is [K][L] row-major with
 * K = moving (node) bins, L = fixed (voxel) bins.
 */
#ifndef BINDER_ORACLE_H
#define BINDER_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ---------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- cubic B-spline weights: BINDER/src/cpu/Spline.cpp:44-73 ---------------------------------- */
void orc_spline3(double d, double w[4]);
/* Spline::spline(d) of order 1, 2 or 3 (the reference's own four-weight layout) */
void orc_spline(int order, double d, double w[4]);
/* spline order (1, 2 or 3) of every E-step, EM and sampler call that follows */
void orc_set_spline_order(int order);
int  orc_get_spline_order(void);

/* ---- E-step (EM): BINDER/src/cpu/Registration.cpp:219-330 (sample == false branch) -------------
 * d      : positions [V*N] (node-grid coordinates)
 * u      : fixed-image bins [V];  v: moving-image bins [Vn];  theta: [K*L]
 * dream  : out [V*N], posterior-mean node coordinate per voxel
 * hist   : out [K*L], soft joint histogram (sum of normalised posteriors)
 * returns mll = -sum_i log(normaliser_i).  Voxels whose normaliser is <= 0 are counted in
 * *degenerate, keep dream = floor(d), and contribute nothing. */
double orc_estep(const double *d, const int *u, const int *v, const double *theta,
                 int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
                 double *dream, double *hist, long long *degenerate);
double orc_mi_filter_likelihood(const double *theta, const int *u, const int *v, int K, int L,
                                int M, int nxn, int nyn, int nzn, long voxel, int x, int y, int z);
double orc_estep_filter(const double *d, const int *u, const int *v, const double *theta,
                        int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L, int M,
                        double *dream, double *hist, long long *degenerate);

/* ---- sampled E-step (Gibbs block 1): Registration.cpp:278-307 (sample == true branch) ---------
 * Categorical draw over the 4x4x4 (4x4 in 2D) neighbours with the Philox stream
 * ctr = {voxel, sweep, 1, chain}, key = {seed_lo, seed_hi}.  hist receives counts. */
double orc_estep_sample(const double *d, const int *u, const int *v, const double *theta,
                        int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
                        uint64_t seed, uint32_t sweep, uint32_t chain,
                        double *dream, double *hist);

/* ---- MI likelihood: BINDER/src/cpu/MILikelihood.cpp ------------------------------------------- */
void   orc_theta_map(double *theta_inout_hist, int K, int L, double alpha);   /* :71-86  */
double orc_dirichlet_cost(const double *theta, int K, int L, double alpha);   /* :33-39, :183-206 */
/* :132-169 with Philox gammas; returns number of rows whose rejection sampler hit its cap */
int    orc_dirichlet_sample(double *theta_inout_hist, int K, int L, double alpha,
                            uint64_t seed, uint32_t sweep, uint32_t chain);
double orc_gamma_sample(double shape, uint64_t seed, uint32_t index, uint32_t sweep,
                        uint32_t tag, uint32_t chain, int *capped);

/* ---- orthonormal 3D DCT-II / DCT-III: BINDER/src/cpu/DCT.cpp:83-175 --------------------------- */
void orc_dct3(const double *in, double *out, int nx, int ny, int nz, int inverse);
/* NonLinearTransformation::up_sample: spectral zero-padding of an AoS field */
void orc_up_sample(const double *in, int nx, int ny, int nz, int nxo, int nyo, int nzo,
                   double *out);

/* ---- DCT-prior M-step: BINDER/src/cpu/NonLinearTransformation.cpp:58-76,128-137,173-223 -------
 * dream, voxel_pos: [V*N];  D: [V];  gamma[N];  out final [V*N].  Returns the prior cost.
 * When noise_seed_valid, adds the prior-sampling noise of :433-451 (Philox normals,
 * ctr = {coef, sweep, 2 or 3, chain}) and, if raw_reg != NULL, returns the raw regulariser
 * of :151-171 summed over components in *raw_reg. */
double orc_smooth(const double *dream, const double *voxel_pos, const double *D,
                  const double gamma[3], double sigma, int nx, int ny, int nz,
                  double *final_out,
                  int add_noise, uint64_t seed, uint32_t sweep, uint32_t chain,
                  const double rho[3], const double eta[3], double *raw_reg);

/* ---- prior sampling of a field: BINDER/src/cpu/NonLinearTransformation.cpp:280-341 ------------
 * n samples of IDCT(DCT(field)/(1+gamma sigma^2 D) + noise) with zero voxel positions, sample s
 * using sweep index sweep0 + s.  out [n*V*N]. */
void orc_sample_field(const double *field, const double *D, const double gamma[3], double sigma,
                      int nx, int ny, int nz, int n, uint64_t seed, uint32_t sweep0,
                      double *out);

/* ---- EM driver: BINDER/src/cpu/Registration.cpp:122-217 -------------------------------------- */
typedef struct {
    double mll, log_prior_likelihood, log_prior_transformation, mlp;
} orc_iter_stats;

int orc_em(double *final_locations, const double *voxel_pos, const int *u, const int *v,
           double *theta, double alpha, const double *D, const double gamma[3], double sigma,
           int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
           double non_zero_voxels, int max_iter, double convergence_th, int update_theta,
           orc_iter_stats *stats /* [max_iter] or NULL */);

/* ---- SSD likelihood: BINDER/src/cpu/SSDLikelihood.cpp ------------------------------------------ */
typedef struct {
    int shift_scale;
    double sigma2, shift, scale, alpha0, beta0;
} orc_ssd;
/* log-space E-step (Registration.cpp:331-470) with the SSD log-likelihood; hist[k][l] is the
 * posterior mass of node bin k at voxel bin l (bins >= 0; outside nodes count as bin 0) */
double orc_ssd_estep(const double *d, const int *u, const int *v, const orc_ssd *p, int nx,
                     int ny, int nz, int nxn, int nyn, int nzn, int K, int L, double *dream,
                     double *hist);
/* update_parameters (:143-285) from the joint histogram, then compute_cost (:314-326) */
double orc_ssd_update(const double *hist, int K, int L, orc_ssd *p, int update);
/* sample_parameters (:284-302) from the sweep's counts, Philox-driven; 1 if the gamma draw hit
 * its attempt cap */
int orc_ssd_sample(const double *hist, int K, int L, orc_ssd *p, uint64_t seed, uint32_t sweep,
                   uint32_t chain);
int orc_ssd_em(double *final_locations, const double *voxel_pos, const int *u, const int *v,
               orc_ssd *p, const double *D, const double gamma[3], double sigma, int nx, int ny,
               int nz, int nxn, int nyn, int nzn, int K, int L, double non_zero_voxels,
               int max_iter, double convergence_th, int update, orc_iter_stats *stats);

/* ---- SSD filter likelihood: BINDER/src/cpu/SSDLikelihoodFilter.cpp ----------------------------
 * M fixed-image channels (voxels [V][M]), F moving-image features (nodes [Vn][F], or [Vn][M] with
 * reg_across_features), coeff [M][F], sigma [M]; M, F <= 8 */
typedef struct {
    int M, F, rfa;
    double alpha0, beta0;
    double coeff[64];
    double sigma[8];
} orc_ssdf;
double orc_ssdf_loglik(const orc_ssdf *p, const double *nodes, const double *voxels, int nxn,
                       int nyn, int nzn, long voxel, int x, int y, int z);
double orc_ssdf_estep(const double *d, const double *nodes, const double *voxels,
                      const orc_ssdf *p, int nx, int ny, int nz, int nxn, int nyn, int nzn,
                      double *dream, double *gamma, double *s1, double *s2, double *outside);
double orc_ssdf_update(orc_ssdf *p, const double *nodes, int nxn, int nyn, int nzn,
                       const double *gamma, const double *s1, const double *s2,
                       const double *outside, int update);
/* sample_parameters (:459-463), Philox-driven; 1 if a gamma draw hit its attempt cap */
int orc_ssdf_sample(orc_ssdf *p, const double *nodes, int nxn, int nyn, int nzn,
                    const double *gamma, const double *s1, const double *s2,
                    const double *outside, uint64_t seed, uint32_t sweep, uint32_t chain);

/* ---- Gibbs sampler driver: BINDER/src/cpu/Registration.cpp:515-642 ----------------------------
 * mean_out [V*N], cov_out [V*N*N] (M2 / (N_s - 1)).  dream is the working dream-location buffer
 * (set by the caller when sample_posteriors == 0). */
int orc_sampler(double *final_locations, double *dream, const double *voxel_pos, const int *u,
                const int *v, double *theta, double alpha, const double *D, double gamma[3],
                double sigma, const double rho[3], const double eta[3],
                int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
                uint64_t seed, uint32_t chain, int N_b, int N_s, int sample_gamma,
                int sample_gamma_every, int sample_posteriors, int sample_likelihood_parameters,
                int sample_transformation_parameters, double *mean_out, double *cov_out);

/* ---- Jacobian determinant: BINDER/src/cpu/utils.cpp:100-345 (3D), :10-98 (2D) --------------- */
void orc_jacobian3d(const double *field, int nx, int ny, int nz, double vx, double vy, double vz,
                    double *J);
void orc_jacobian2d(const double *field, int nx, int ny, double vx, double vy, double *J);

/* ---- topology correction: BINDER/src/cpu/topology_correction_3D.cpp:17-607 ------------------ */
void orc_corner_jacobians3d(const double *pos, int nx, int ny, int nz, const double vs[3],
                            double e1, double e2, double *J_corner, int *n_below, int *n_above);
void orc_gradients3d(const double *pos, int nx, int ny, int nz, const double vs[3], double *grad);
int  orc_limit_gradients3d(double *grad, const double *J_corner, int nx, int ny, int nz,
                           double e1, double e2);
void orc_integrate3d(double *pos, const double *grad, int nx, int ny, int nz, const double vs[3],
                     const double mean[3]);
/* full driver; field in/out [V*3] grid units.  Returns the outer iterations run. */
int  orc_topology3d(double *field, double e1, double e2, int max_outer, int max_inner,
                    const double vs[3], int nx, int ny, int nz);
/* 2D topology correction (topology_correction_2D.cpp) on AoS [nx][ny][2] fields */
void orc_corner_jacobians2d(const double *pos, int nx, int ny, const double vs[2], double e1,
                            double e2, double *Jc, int *n_below, int *n_above);
void orc_gradients2d(const double *pos, int nx, int ny, const double vs[2], double *g);
int  orc_limit_gradients2d(double *g, const double *Jc, int nx, int ny, double e1, double e2);
void orc_integrate2d(double *pos, const double *g, int nx, int ny, const double vs[2],
                     const double mean[2]);
int  orc_topology2d(double *field, double e1, double e2, int max_outer, int max_inner,
                    const double vs[2], int nx, int ny);

/* ---- mutual information of a joint histogram [K*L] (FP64) ----------------------------------- */
double orc_mutual_information(const double *hist, int K, int L);

/* ---- threads used by the OpenMP loops (0 = OpenMP default) ---------------------------------- */
void orc_set_threads(int n);
int  orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
