/*
 * binder_b200 -- C ABI of the B200 (sm_100a) engine for BINDER's registration and Gibbs-sampling
 * hot path.
 *
 * Every entry point replaces one method of the reference's pybind11 module `BINDER._core`
 * (ste93ste/BINDER, BINDER/src/gpu/bindings.cpp for the CUDA backend, BINDER/src/cpu/bindings.cpp
 * for the CPU backend); the citation beside each declaration names the binding it stands in for.
 * Conventions:
 *   - plain host pointers and sizes; the library copies inputs and writes caller-owned outputs
 *     (the reference CPU backend instead keeps pointers into caller arrays);
 *   - position fields are [Nx][Ny][Nz][3] C-order, components interleaved; bins are int32;
 *     theta is [K][L] row-major (K = moving/node bins, L = fixed/voxel bins);
 *   - every function returns 0 on success or a BINDER_STATUS_* code; binder_last_error() then
 *     holds a message (thread-local).  Nothing here throws across the boundary.
 * All work runs on the calling thread's current CUDA device, on a stream owned by the object.
 */
#ifndef BINDER_B200_H
#define BINDER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BINDER_STATUS_OK 0
#define BINDER_STATUS_INVALID_ARGUMENT 1
#define BINDER_STATUS_CUDA_ERROR 2
#define BINDER_STATUS_UNSUPPORTED 3
#define BINDER_STATUS_NOT_READY 4
#define BINDER_STATUS_DEVICE_FAULT 5

/* device status bits reported by binder_registration_get_state */
#define BINDER_FLAG_GAMMA_CAPPED 1u   /* a Marsaglia-Tsang gamma sampler hit its attempt cap */
#define BINDER_FLAG_LIMITER_CAPPED 2u /* a topology limiter blend loop hit its step cap */
#define BINDER_FLAG_NON_FINITE 4u     /* the min-log-posterior became non-finite */

typedef struct binder_registration binder_registration;
typedef struct binder_transform binder_transform;
typedef struct binder_pyramid binder_pyramid;
typedef struct binder_initnet binder_initnet;
typedef struct binder_batch binder_batch;

/* last error message of this thread ("" when none) */
const char *binder_last_error(void);
/* "b200" -- stands in for `_core.backend` ("cuda" / "cpu"), bindings.cpp:16 (gpu), :20 (cpu) */
const char *binder_backend(void);
/* 1: topology correction is built -- `_core.has_topology_correction`, probed at
 * BINDER/FastRegistration.py:118-119 */
int binder_has_topology_correction(void);

/* ---- _core.Registration -------------------------------------------------------------------- */

/* Registration(final_locations, threads, voxel_pos, node_pos, Nx_v, Ny_v, Nz_v, Nx_n, Ny_n, Nz_n,
 *              spline_order, non_zero_voxels)                    gpu/bindings.cpp:18-47
 * final_locations, voxel_pos, node_pos: [Nx_v*Ny_v*Nz_v*3] floats.  `threads` is accepted for
 * interface parity and unused.  node_pos may be NULL (the reference never reads it).
 * spline_order 1, 2 or 3 with the CPU backend's offsets and sigma_spline (Spline.cpp:9-41; the
 * reference GPU backend builds only 3). */
int binder_registration_create(binder_registration **out, const float *final_locations,
                               int threads, const float *voxel_pos, const float *node_pos,
                               int Nx_v, int Ny_v, int Nz_v, int Nx_n, int Ny_n, int Nz_n,
                               int spline_order, double non_zero_voxels);
int binder_registration_destroy(binder_registration *h);

/* setMILikelihood(alpha, theta, K, L, threads, binned_nodes, binned_voxels)   gpu/bindings.cpp:49-70
 * theta [K*L]; binned_nodes [Nx_n*Ny_n*Nz_n] in [0, K); binned_voxels [Nx_v*Ny_v*Nz_v] in [0, L) */
int binder_registration_set_mi_likelihood(binder_registration *h, double alpha, const float *theta,
                                          int K, int L, int threads, const int32_t *binned_nodes,
                                          const int32_t *binned_voxels);

/* setMILikelihoodFilter(alpha, theta, threads, binned_nodes, binned_voxels, K, L, M)
 *                                                                  cpu/bindings.cpp:90-115
 * The CPU backend's multi-channel MI likelihood (MILikelihoodFilter.cpp): theta [M][K][L]; the
 * bins of channel m are read at [index + m] as the reference reads them, so binned_nodes holds
 * at least Nx_n*Ny_n*Nz_n + M - 1 bins in [0, K) and binned_voxels Nx_v*Ny_v*Nz_v + M - 1 in
 * [0, L).  1 <= M <= 8, M*K*L <= 24576.  EM and the sampler (M*K*L up to about 22000 there);
 * get_likelihood_parameters then returns M*K*L values. */
int binder_registration_set_mi_likelihood_filter(binder_registration *h, double alpha,
                                                 const float *theta, int threads,
                                                 const int32_t *binned_nodes,
                                                 const int32_t *binned_voxels, int K, int L,
                                                 int M);

/* setSSDLikelihood(bins, threads, sigma_sq, scale_shift, scale, shift, binned_nodes,
 *                  binned_voxels, alpha_0, beta_0)                  cpu/bindings.cpp:120-152
 * The CPU backend's SSD likelihood (SSDLikelihood.cpp): the bins are the intensities, bins <= 64;
 * scale_shift 0 fits sigma^2 only, 1 also shift and scale.  EM and the sampler (its draws of
 * sigma^2, shift and scale: SSDLikelihood.cpp:167-302 with sample = 1; not in sampler_chains).
 * get_likelihood_parameters then returns (scale, shift). */
int binder_registration_set_ssd_likelihood(binder_registration *h, int bins, int threads,
                                           double sigma_sq, int scale_shift, double scale,
                                           double shift, const int32_t *binned_nodes,
                                           const int32_t *binned_voxels, double alpha_0,
                                           double beta_0);
/* No counterpart in the reference (it prints sigmaSq): the SSD parameters sigma^2, shift, scale */
int binder_registration_get_ssd_parameters(const binder_registration *h, double out[3]);

/* setSSDLikelihoodFilter(coeff, threads, sigma, features_nodes, features_voxels,
 *                        reg_across_features, alpha_0, beta_0, M, F)   cpu/bindings.cpp:154-189
 * The CPU backend's feature SSD likelihood (SSDLikelihoodFilter.cpp): M fixed-image channels
 * (features_voxels [Nx_v*Ny_v*Nz_v][M]), F moving-image features (features_nodes
 * [Nx_n*Ny_n*Nz_n][F], or [..][M] with reg_across_features, which then predicts channel m by
 * feature m and fits no coefficients), coeff [M][F] and sigma [M] in host memory; 1 <= M, F <= 8.
 * EM in log space and the sampler (its draws of the coefficients and sigmas, :459-463, with
 * sample_multivariate_normal and sample_inverse_gamma as written; not in sampler_chains);
 * get_likelihood_parameters then returns the M*F coefficients. */
int binder_registration_set_ssd_likelihood_filter(binder_registration *h, const double *coeff,
                                                  int threads, const double *sigma,
                                                  const double *features_nodes,
                                                  const double *features_voxels,
                                                  int reg_across_features, double alpha_0,
                                                  double beta_0, int M, int F);
/* coeff [M][F] and sigma [M] of the SSD filter likelihood (either may be null) */
int binder_registration_get_ssd_filter_parameters(const binder_registration *h, double *coeff,
                                                  double *sigma);

/* setNonLinearTransformation(gamma_x..z, voxels_size_x..z, nodes_size_x..z, D)
 *                                                               gpu/bindings.cpp:72-95; D [V] */
int binder_registration_set_nonlinear_transformation(binder_registration *h, double gamma_x,
                                                     double gamma_y, double gamma_z,
                                                     double voxels_size_x, double voxels_size_y,
                                                     double voxels_size_z, double nodes_size_x,
                                                     double nodes_size_y, double nodes_size_z,
                                                     const float *D);

/* EM(max_EM_iterations, convergence_th, update_likelihood_parameters, debug)
 *                                                               gpu/bindings.cpp:99-103
 * *iterations_out (optional) receives the number of EM iterations run. */
int binder_registration_em(binder_registration *h, int max_iterations, double convergence_th,
                           int update_likelihood_parameters, int debug, int *iterations_out);

/* sampler(seed, N_b, N_s, sample_gamma, sample_gamma_every, sample_posteriors,
 *         sample_likelihood_parameters, sample_transformation_parameters) -> (mean, cov)
 *                                                               gpu/bindings.cpp:105-131
 * mean_out [V*3] and cov_out [V*3*3] (M2 / (N_s - 1)) in FP64 (FP64 Welford accumulators).
 * Every likelihood: MI, SSD, MI filter and SSD filter (cpu/Registration.cpp:515-642 drives
 * each through its sample_parameters). */
int binder_registration_sampler(binder_registration *h, uint64_t seed, int N_b, int N_s,
                                int sample_gamma, int sample_gamma_every, int sample_posteriors,
                                int sample_likelihood_parameters,
                                int sample_transformation_parameters, double *mean_out,
                                double *cov_out);

/* No counterpart in the reference (it runs one chain per Registration object,
 * gpu/Registration.cu:917-1026, cpu/Registration.cpp:515-642): `chains` independent chains of
 * the sampler above, every kernel of a sweep launched once for all of them.  Chain c draws with
 * Philox chain index (the object's chain index + c), so it equals, draw for draw, sampler() after
 * binder_registration_set_chain(chain index + c) from the same state.  Every chain starts from the
 * object's current positions, dream locations, theta and gammas, which the call leaves as they
 * are.  MI likelihood only.  Outputs (FP64, each optional / NULL): mean_out [chains*V*N] and
 * cov_out [chains*V*N*N] per chain (M2 / (N_s - 1)); pooled_mean_out [V*N] and pooled_cov_out
 * [V*N*N], the chains' samples pooled (M2 / (chains * N_s - 1)). */
int binder_registration_sampler_chains(binder_registration *h, uint64_t seed, int chains,
                                       int N_b, int N_s, int sample_gamma,
                                       int sample_gamma_every, int sample_posteriors,
                                       int sample_likelihood_parameters,
                                       int sample_transformation_parameters, double *mean_out,
                                       double *cov_out, double *pooled_mean_out,
                                       double *pooled_cov_out);

/* get_final_locations_as_numpy_array() -> [Nx,Ny,Nz,3]          gpu/bindings.cpp:142-157 */
int binder_registration_get_final_locations(const binder_registration *h, float *out);
/* get_dream_locations() / set_dream_locations(arr)              gpu/bindings.cpp:133-140 */
int binder_registration_get_dream_locations(const binder_registration *h, float *out);
int binder_registration_set_dream_locations(binder_registration *h, const float *in);
/* No counterpart in the reference: adds to the current positions a displacement field given on
 * an Nx_f x Ny_f x Nz_f grid (AoS FP32 [Nx_f][Ny_f][Nz_f][N], host or device memory), resampled
 * to the voxel grid by the order-1 resize of binder_resize_linear (Nz_f == 1 for a 2D
 * registration).  Theta, the likelihood and prior state are kept, so EM continues from the
 * moved positions (the learned initialiser's coarse prediction; reset() still restores the
 * creation-time positions). */
int binder_registration_add_displacement(binder_registration *h, const float *field, int Nx_f,
                                         int Ny_f, int Nz_f);
/* get_likelihood_parameters() -> K*L (M*K*L with the filter likelihood, (scale, shift) with
 * SSD)                                                                 gpu/bindings.cpp:97 */
int binder_registration_get_likelihood_parameters(const binder_registration *h, float *out);
/* get_shape() -> (Nx, Ny, Nz, N)                                cpu/bindings.cpp:294 */
int binder_registration_get_shape(const binder_registration *h, int out[4]);

/* Per-iteration statistics of the last EM call, [n][4] = (min-log-likelihood, Dirichlet prior,
 * deformation prior, min-log-posterior) in FP64 -- the values the reference prints at
 * Registration.cpp:197-202.  Returns n (<= max_n) through *n_out. */
int binder_registration_get_iteration_stats(const binder_registration *h, double *out, int max_n,
                                            int *n_out);
/* current gammas, nu, degenerate-voxel count and BINDER_FLAG_* bits; any pointer may be NULL */
int binder_registration_get_state(const binder_registration *h, double gamma_out[3],
                                  double *nu_out, unsigned long long *degenerate_out,
                                  unsigned *flags_out);
/* device time of the last EM / sampler call in milliseconds */
int binder_registration_last_elapsed_ms(const binder_registration *h, double *ms_out);
/* run the object's work on a caller stream (a cudaStream_t; NULL restores the object's own) */
int binder_registration_set_stream(binder_registration *h, void *cuda_stream);
/* Philox chain index, so independent chains with one seed draw disjoint streams */
int binder_registration_set_chain(binder_registration *h, uint32_t chain);

/* No counterpart in the reference: restore the positions given at creation, the theta given to
 * set_mi_likelihood, the gammas given to set_nonlinear_transformation (the sampler keeps the
 * gammas it draws) and a fresh iteration state, device to device (re-runs without host I/O). */
int binder_registration_reset(binder_registration *h);

/* Topology correction of the object's own current positions, on the device, in place.  Same
 * algorithm and arguments as binder_topology_correct_3d below (binder_topology_correct_2d for a
 * 2D registration; voxel_sizes[2] is then unused); it replaces the round trip
 * get_final_locations -> topology_correction_3D/2D().correct_topology -> next Registration that
 * BINDER/FastRegistration.py:515,527-546 performs.  stats_out as for binder_topology_correct_3d. */
int binder_registration_correct_topology(binder_registration *h, double e1, double e2,
                                         int max_outer_it, int max_it,
                                         const double voxel_sizes[3], long long *stats_out);

/* No counterpart in the reference (its GPU backend is FP32 cuFFT only): arithmetic of the DCT
 * passes.  BINDER_PRECISION_FP32 = FP32 FMA on the CUDA cores; _TF32X3 = tensor cores (tcgen05)
 * with hi/lo TF32 operand splitting, FP32-level accuracy; _TF32 = one TF32 tensor-core product;
 * _BF16X3 = BF16 hi/lo operand splitting, three kind::f16 products (about 16 mantissa bits);
 * _BF16 = one BF16 product.  All accumulate in FP32.  The default comes from the
 * BINDER_B200_PRECISION environment variable (0 to 4), else BF16X3. */
#define BINDER_PRECISION_FP32 0
#define BINDER_PRECISION_TF32X3 1
#define BINDER_PRECISION_TF32 2
#define BINDER_PRECISION_BF16X3 3
#define BINDER_PRECISION_BF16 4
int binder_registration_set_precision(binder_registration *h, int precision);
int binder_transform_set_precision(binder_transform *h, int precision);

/* No counterpart in the reference (its E-step accumulates the joint histogram in FP32): the
 * per-thread bin columns of the MI likelihood's EM E-step (K <= 64), where each voxel's posterior
 * mass is summed per moving bin before it enters the histogram.  BINDER_HISTOGRAM_FP32 (the
 * default) or BINDER_HISTOGRAM_FP16: FP16 columns use half the shared memory, so three CTAs fit
 * on an SM instead of two; each voxel's per-bin mass is rounded to FP16 (about 11 bits), while
 * the normaliser, the dream location, the log-likelihood and the histogram itself stay FP32 /
 * fixed point.  Other likelihoods and the sampler ignore the setting. */
#define BINDER_HISTOGRAM_FP32 0
#define BINDER_HISTOGRAM_FP16 1
int binder_registration_set_histogram_precision(binder_registration *h, int precision);

/* No counterpart in the reference: the cudaStream_t the object's work runs on (for events). */
int binder_registration_get_stream(const binder_registration *h, void **stream_out);

/* No counterpart in the reference: average device time in ms of one launch of a pipeline stage,
 * timed with CUDA events over `n` back-to-back eager launches on the object's stream.
 * stage 0 = EM E-step kernel, 1 = DCT-prior M-step (all passes), 2 = theta update.  The object's
 * positions, dream locations and histogram are left unspecified: call binder_registration_reset
 * before further use. */
int binder_registration_profile_stage(binder_registration *h, int stage, int n, double *avg_ms_out);

/* No counterpart in the reference: number of kernels this library has launched in this process
 * (each replay of a captured CUDA graph counts all of its kernels). */
long long binder_kernel_launch_count(void);
/* No counterpart in the reference: page-locked host memory for output arrays, cached by size
 * (a later alloc of the same size reuses a freed buffer).  binder_pinned_free takes the size
 * given to binder_pinned_alloc. */
int binder_pinned_alloc(size_t bytes, void **out);
int binder_pinned_free(void *p, size_t bytes);

/* ---- _core.NonLinearTransformation --------------------------------------------------------- */

/* NonLinearTransformation(gamma_x..z, voxels_size_x..z, nodes_size_x..z, D, Nx_v, Ny_v, Nz_v,
 *                         threads, sigma_spline, spline_offset)   gpu/bindings.cpp:160-198 */
int binder_transform_create(binder_transform **out, double gamma_x, double gamma_y,
                            double gamma_z, double voxels_size_x, double voxels_size_y,
                            double voxels_size_z, double nodes_size_x, double nodes_size_y,
                            double nodes_size_z, const float *D, int Nx_v, int Ny_v, int Nz_v,
                            int threads, double sigma_spline, double spline_offset);
int binder_transform_destroy(binder_transform *h);
/* smooth_deformation(field) -> (log_prior_deformation, field')  gpu/bindings.cpp:201-224 */
int binder_transform_smooth_deformation(binder_transform *h, const float *field, float *out,
                                        double *log_prior_out);
/* sampleDeformationField(field, n) -> [n, Nx, Ny, Nz, 3]        gpu/bindings.cpp:226-255 */
int binder_transform_sample_deformation_field(binder_transform *h, const float *field,
                                              int number_of_samples, float *out);
int binder_transform_get_shape(const binder_transform *h, int out[4]);
/* NonLinearTransformation.up_sample(field, N_x, N_y, N_z, N_x_o, N_y_o, N_z_o, threads)
 *   -> [N_x_o, N_y_o, N_z_o, N]                                  cpu/bindings.cpp:408-434
 * static: spectral zero-padding of an AoS field (N = 2 when N_z_o == 1), FP64; every output axis
 * at least as long as its input axis.  `threads` is accepted for interface parity. */
int binder_transform_up_sample(const double *field, int Nx, int Ny, int Nz, int Nx_o, int Ny_o,
                               int Nz_o, int threads, double *out);

/* No counterpart in the reference's module: skimage.transform.resize(field, (Nx_o, Ny_o, Nz_o),
 * order=1) * scale on an AoS [Nx][Ny][Nz][N] FP64 field, as BINDER/FastRegistration.py:562-564
 * resamples the deformation between resolutions (Gaussian anti-aliasing on shrinking axes, then
 * pixel-centre-aligned linear interpolation, mirror boundaries). */
int binder_resize_linear(const double *field, int Nx, int Ny, int Nz, int N, int Nx_o, int Ny_o,
                         int Nz_o, double scale, double *out);
/* ---- preprocessing and output of the registration driver ----------------------------------
 * No counterparts in the reference's module: the numpy / scipy / skimage steps that
 * BINDER/FastRegistration.py runs around it, on the GPU.  Pointers may be host or device memory.
 *
 * utils.bin_signal_robust(signal, number_of_bins, lower, higher)   BINDER/utils.py:20-82
 * signal: n values, float32 (is_double 0) or float64 (1), computed in that type with numpy's
 * operation order (bit-identical bins); binned_out int32[n]; bin_edges_out (optional) the
 * number_of_bins + 1 returned edges.  A constant signal is rejected. */
int binder_bin_signal_robust(const void *signal, int is_double, long long n, int number_of_bins,
                             double lower_percentile, double higher_percentile,
                             int32_t *binned_out, double *bin_edges_out);
/* utils.bin_signal(signal, number_of_bins)                          BINDER/utils.py:12-17 */
int binder_bin_signal(const void *signal, int is_double, long long n, int number_of_bins,
                      int32_t *binned_out);
/* scipy.ndimage.center_of_mass(bins > 0) as FastRegistration.py:387-395 computes it; index
 * space, exact (integer sums, one division).  No non-zero voxel: INVALID_ARGUMENT. */
int binder_center_of_mass(const int32_t *bins, int Nx, int Ny, int Nz, double out[3]);
/* the resampling of utils.save_warped_image (BINDER/utils.py:222-227): skimage.transform.warp of
 * the moving image [Nx][Ny][Nz] (FP64) at positions [M][3] (index space) with order 0, 1 or 3
 * (cubic B-spline with the spline prefilter, as run_BINDER.py's default --output-interpolation),
 * zero outside, clipped to the input range as skimage clips; out [M] FP64. */
int binder_warp_image(const double *image, int Nx, int Ny, int Nz, const double *positions,
                      long long M, int order, double *out);

/* ---- the multi-resolution step on the device ------------------------------------------------
 * No counterpart in the reference's module: FastRegistration.move_resolution
 * (BINDER/FastRegistration.py:550-650) plus the Registration set-up of run() (:443-486) for the
 * MI metric, done on the device from full-resolution data the pyramid keeps.
 *
 * binder_pyramid_create: full-resolution bins (int32, fixed image [V], moving image [Vn]) and the
 * voxel positions in node space (AoS [V*N] FP64, N = 2 when Nz_v == 1; NULL for the identity
 * grid), the two images' voxel sizes, and the options of FastRegistration of the same names
 * (`gamma` is its gamma_init).  The `smooth` option (Smoothing_Spline) is not built. */
int binder_pyramid_create(binder_pyramid **out, const int32_t *binned_voxels,
                          const int32_t *binned_nodes, const double *voxel_pos, int Nx_v, int Ny_v,
                          int Nz_v, int Nx_n, int Ny_n, int Nz_n,
                          const double voxels_voxel_size[3], const double nodes_voxel_size[3],
                          double gamma, int finite_difference_order,
                          int increase_gamma_at_DS_resolution, int upsample_in_frequency_domain,
                          int spline_order);
int binder_pyramid_destroy(binder_pyramid *p);
/* move_resolution(resolution) and a new registration for that level (*out; destroy it with
 * binder_registration_destroy), with setNonLinearTransformation and setMILikelihood applied.
 * The deformation comes from `prev`, a registration of this pyramid at prev_resolution, or from
 * the full-resolution voxel positions when prev is NULL (FastRegistration starts at resolution
 * 1).  theta [K*L] (host or device memory) or NULL to carry prev's over.  info_out (optional):
 * voxels_shape[3], nodes_shape[3], gamma_x/y/z, current voxel sizes[3], current node sizes[3],
 * non_zero_voxels. */
int binder_pyramid_level(binder_pyramid *p, int resolution, const binder_registration *prev,
                         int prev_resolution, double alpha, const float *theta, int K, int L,
                         binder_registration **out, double info_out[16]);

/* The per-axis m x n matrix (row-major, host memory, no device work) that the two resamplers
 * above apply along an axis of length n -> m: kind 0 spectral up-sampling, 1 linear resize. */
int binder_resample_matrix(int kind, int n, int m, double *out);

/* ---- Jacobian determinant and topology correction ----------------------------------------- */

/* compute_jacobian_determinant_3D(field, Nx, Ny, Nz, vx, vy, vz) -> [Nx,Ny,Nz]
 *                                                               cpu/bindings.cpp:564-593
 * FP64 in and out; evaluated on the GPU with the reference's arithmetic (bit-identical). */
int binder_jacobian_determinant_3d(const double *field, int Nx, int Ny, int Nz, double voxel_size_x,
                                   double voxel_size_y, double voxel_size_z, double *J_out);

/* compute_jacobian_determinant_2D(field, Nx, Ny, vx, vy) -> [Nx,Ny]   cpu/bindings.cpp:535-560
 * field AoS [Nx*Ny*2]; FP64, the reference's arithmetic (bit-identical). */
int binder_jacobian_determinant_2d(const double *field, int Nx, int Ny, double voxel_size_x,
                                   double voxel_size_y, double *J_out);

/* No counterpart in the reference: binder_jacobian_determinant_3d without any device allocation.
 * The call above allocates device buffers for the field and the determinants (cudaMalloc) and
 * frees them (cudaFree) every time.  Some callers cannot do that: a framework whose caching
 * allocator already holds most of the GPU's memory gets out-of-memory from a fresh cudaMalloc
 * even though its own pool has room, and a caller that keeps other streams busy cannot afford the
 * device-wide synchronisation cudaFree implies.  This variant stages the field, the determinants
 * and its summary in one fixed array inside the library's device image (16 MiB), so it handles
 * grids of at most binder_jacobian_noalloc_max_voxels() voxels (524288; e.g. 80x80x80) and
 * rejects larger ones with BINDER_STATUS_INVALID_ARGUMENT.  The summary is reset on every call.
 *   - The first call on each device looks up the array's device address (with that device
 *     current) and keeps it; make that first call before any stream capture begins.  A
 *     cudaDeviceReset after that first call is not supported (the address kept may be stale).
 *   - Work runs on the per-thread default stream (cudaStreamPerThread) of the calling thread's
 *     current device, which does not synchronise with the caller's other streams; the call
 *     returns when J_out is filled.
 *   - Calls that overlap in time on the same device share the array and race: serialise them.
 * J_out as for binder_jacobian_determinant_3d (bit-identical values).  minmax_out (optional, 2
 * values) receives min and max of J; negative_out (optional) the number of voxels with J < 0. */
int binder_jacobian_determinant_3d_noalloc(const double *field, int Nx, int Ny, int Nz,
                                           double voxel_size_x, double voxel_size_y,
                                           double voxel_size_z, double *J_out,
                                           double minmax_out[2], long long *negative_out);
/* largest voxel count binder_jacobian_determinant_3d_noalloc accepts */
long long binder_jacobian_noalloc_max_voxels(void);

/* topology_correction_3D().correct_topology(h, e1, e2, max_outer_it, max_it, threads,
 *                                           voxel_sizes, Nx, Ny, Nz) -> [Nx,Ny,Nz,3]
 *                                                               gpu/bindings.cpp:259-287
 * FP64 throughout.  stats_out (optional, 6 values): outer iterations, inner iterations,
 * voxels with J < e1 before and after, voxels with J > e2 before and after. */
int binder_topology_correct_3d(const double *field, double e1, double e2, int max_outer_it,
                               int max_it, int threads, const double voxel_sizes[3], int Nx,
                               int Ny, int Nz, double *out, long long *stats_out);

/* topology_correction_2D().correct_topology(h, e1, e2, max_outer_it, max_it, threads,
 *                                           voxel_sizes, Nx, Ny) -> [Nx,Ny,2]
 *                                                               cpu/bindings.cpp:447-480
 * field / out AoS [Nx*Ny*2], voxel_sizes [2]; FP64; stats_out as for the 3D entry point. */
int binder_topology_correct_2d(const double *field, double e1, double e2, int max_outer_it,
                               int max_it, int threads, const double voxel_sizes[2], int Nx,
                               int Ny, double *out, long long *stats_out);

/* ---- batches of registrations: no counterpart in the reference, which runs one pair per
 * Registration object (FastRegistration.py:443-486) ---------------------------------------------
 * Many registrations, image pairs of any sizes each set up as usual, run as one: every chunk of
 * EM iterations is one CUDA graph holding each pair's kernels on a branch of its own, so the
 * pairs' kernels overlap on the GPU and the whole batch advances with one graph launch per chunk.
 * Each pair keeps its own convergence test.  The registrations must outlive the batch; a
 * registration's own calls must not run while the batch runs. */
int binder_batch_create(binder_registration *const *regs, int n, binder_batch **out);
int binder_batch_destroy(binder_batch *h);
/* EM(max_iterations, convergence_th, update_likelihood_parameters) of every pair;
 * iterations_out [n] receives each pair's iteration count, ms_out (optional) the device time */
int binder_batch_em(binder_batch *h, int max_iterations, double convergence_th,
                    int update_likelihood_parameters, int *iterations_out, double *ms_out);
/* No counterpart in the reference: CTAs of the EM E-step launch (0 restores the default, every SM
 * times its occupancy); smaller grids let the pairs of a batch share the GPU */
int binder_registration_set_estep_grid(binder_registration *h, int ctas);

/* ---- learned initialiser: no counterpart in the reference -----------------------------------
 * A 3D convolutional encoder-decoder (channels 16-32-64-128, 3x3x3 convolutions with leaky ReLU,
 * 2x2x2 average pooling, a skip connection at the 4-voxel level) whose prediction seeds the
 * positions a registration starts from (the reference's hook is the final_locations argument of
 * Registration, FastRegistration.py:443-450).  Input: batch x S^3 voxels x in_channels channels
 * (moving and fixed intensities in [0, 1], optionally followed by a displacement field), FP32,
 * channels last; S a multiple of 8.  Output: the displacement
 * on the grid of every 4th voxel, batch x (S/4)^3 x 3, FP32, in voxels.  Every layer runs on
 * hand-written sm_100a kernels: im2col gathers into BF16 operands, a tcgen05 BF16 GEMM with FP32
 * accumulation in TMEM, FP32 master weights and Adam.  Pointers may be host or device memory. */
/* The network's matrix product on host arrays: C [M][N] (FP32) = A [M][K] . B [N][K]^T with
 * BF16 operands (raw bits, row-major, K contiguous), K a multiple of 64, on the tcgen05 kernel
 * every convolution runs on (FP32 accumulation in TMEM; K split over CTAs above 4096). */
int binder_gemm_bf16(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K);
int binder_initnet_create(binder_initnet **out, int batch, int size, int in_channels,
                          uint64_t seed);
int binder_initnet_destroy(binder_initnet *h);
int binder_initnet_parameter_count(const binder_initnet *h, long long *out);
/* FP32 parameters layer by layer: W [Cout][27 Cin] (tap-major: tap = (dx*3+dy)*3+dz, then Cin),
 * then b [Cout]; layers in forward order */
int binder_initnet_get_parameters(const binder_initnet *h, float *out);
int binder_initnet_set_parameters(binder_initnet *h, const float *in);
int binder_initnet_predict(binder_initnet *h, const float *in, float *out);
/* one Adam step (beta 0.9 / 0.999) on the mean squared error against target; loss_out (optional)
 * receives the loss before the step, grads_out (optional) its gradient */
int binder_initnet_train_step(binder_initnet *h, const float *in, const float *target, double lr,
                              double *loss_out, float *grads_out);
/* the loss and its gradient without a step */
int binder_initnet_gradients(binder_initnet *h, const float *in, const float *target,
                             double *loss_out, float *grads_out);

#ifdef __cplusplus
}
#endif
#endif /* BINDER_B200_H */
