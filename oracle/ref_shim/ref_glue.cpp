// extern "C" entry points over the reference's own CPU classes, compiled from the unmodified
// reference sources into oracle/_ref/libbinder_ref.so (test infrastructure: a checker only).
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

#include "MILikelihood.h"
#include "MILikelihoodFilter.h"
#include "SSDLikelihoodFilter.h"
#include "NonLinearTransformation.h"
#include "Registration.h"
#include "Spline.h"
#include "topology_correction_2D.h"
#include "topology_correction_3D.h"
#include "utils.h"

extern "C" {

// Spline::spline (BINDER/src/cpu/Spline.cpp:44-109)
void ref_spline(int order, double d, double out[4]) {
    Spline s(order, false);
    const auto w = s.spline(d);
    for (int i = 0; i < 4; ++i) out[i] = w[i];
}

// compute_jacobian_determinant_3D / _2D (BINDER/src/cpu/utils.cpp:10-345)
void ref_jacobian3d(const double *field, int nx, int ny, int nz, double vx, double vy, double vz,
                    double *J) {
    const auto r = compute_jacobian_determinant_3D(field, nx, ny, nz, vx, vy, vz);
    std::memcpy(J, r.data(), sizeof(double) * r.size());
}

void ref_jacobian2d(const double *field, int nx, int ny, double vx, double vy, double *J) {
    const auto r = compute_jacobian_determinant_2D(field, nx, ny, vx, vy);
    std::memcpy(J, r.data(), sizeof(double) * r.size());
}

// topology_correction_3D::correct_topology (BINDER/src/cpu/topology_correction_3D.cpp:17-143)
void ref_topology3d(const double *field, double e1, double e2, int max_outer, int max_inner,
                    const double *vs, int nx, int ny, int nz, double *out) {
    topology_correction_3D tc;
    const double *r = tc.correct_topology(field, e1, e2, max_outer, max_inner, 1, vs, nx, ny, nz);
    std::memcpy(out, r, sizeof(double) * (size_t)nx * ny * nz * 3);
}

// the same on `threads` threads (the FFT plans' thread count), with the wall seconds of the call
void ref_topology3d_mt(const double *field, double e1, double e2, int max_outer, int max_inner,
                       const double *vs, int nx, int ny, int nz, double *out, int threads,
                       double *seconds) {
    topology_correction_3D tc;
    const auto t0 = std::chrono::steady_clock::now();
    const double *r =
        tc.correct_topology(field, e1, e2, max_outer, max_inner, threads, vs, nx, ny, nz);
    if (seconds)
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::memcpy(out, r, sizeof(double) * (size_t)nx * ny * nz * 3);
}

// topology_correction_2D::correct_topology (BINDER/src/cpu/topology_correction_2D.cpp:17-163)
void ref_topology2d(const double *field, double e1, double e2, int max_outer, int max_inner,
                    const double *vs, int nx, int ny, double *out) {
    topology_correction_2D tc;
    const double *r = tc.correct_topology(field, e1, e2, max_outer, max_inner, 1, vs, nx, ny);
    std::memcpy(out, r, sizeof(double) * (size_t)nx * ny * 2);
}

// NonLinearTransformation::up_sample (BINDER/src/cpu/NonLinearTransformation.cpp:366-430)
void ref_up_sample(const double *field, int nx, int ny, int nz, int nxo, int nyo, int nzo,
                   double *out) {
    const auto r = NonLinearTransformation::up_sample(field, nx, ny, nz, nxo, nyo, nzo, 1);
    std::memcpy(out, r.data(), sizeof(double) * r.size());
}

// NonLinearTransformation::smooth_deformation (BINDER/src/cpu/NonLinearTransformation.cpp:226-278)
double ref_smooth_deformation(const double gamma[3], const double rho[3], const double eta[3],
                              const double *D, int nx, int ny, int nz, double sigma, double offset,
                              const double *field, double *out) {
    NonLinearTransformation t(gamma[0], gamma[1], gamma[2], rho[0], rho[1], rho[2], eta[0], eta[1],
                              eta[2], D, nx, ny, nz, 1, sigma, offset);
    auto [cost, ptr] = t.smooth_deformation(field);
    const int N = nz == 1 ? 2 : 3;
    std::memcpy(out, ptr, sizeof(double) * (size_t)nx * ny * nz * N);
    delete[] ptr;
    return cost;
}

// MILikelihood::update_parameters and compute_cost (BINDER/src/cpu/MILikelihood.cpp:33-124):
// the histogram is fed through accumulate_info with a 1-D node grid of K nodes (node k has bin k)
// and L voxels (voxel l has bin l).
double ref_mi_update(double alpha, const double *theta_in, const double *hist, int K, int L,
                     double *theta_out) {
    std::vector<int> nodes(K), voxels(L);
    for (int k = 0; k < K; ++k) nodes[k] = k;
    for (int l = 0; l < L; ++l) voxels[l] = l;
    MILikelihood mi(alpha, theta_in, 1, nodes.data(), voxels.data(), K, L, K, 1, 1, L, 1, 1);
    mi.initialize_parameters();
    for (int k = 0; k < K; ++k)
        for (int l = 0; l < L; ++l) mi.accumulate_info(0, l, k, 0, 0, hist[k * L + l]);
    mi.update_parameters();
    const auto th = mi.get_parameters();
    std::memcpy(theta_out, th.data(), sizeof(double) * K * L);
    return mi.compute_cost();
}

double ref_dirichlet_cost(double alpha, const double *theta, int K, int L) {
    std::vector<int> nodes(K, 0), voxels(L, 0);
    MILikelihood mi(alpha, theta, 1, nodes.data(), voxels.data(), K, L, K, 1, 1, L, 1, 1);
    return mi.compute_cost();
}

// MILikelihoodFilter::compute_likelihood (BINDER/src/cpu/MILikelihoodFilter.cpp:53-68) for one
// (voxel, node) pair; theta [M][K][L], bins read by the class at [index + m]
double ref_mi_filter_likelihood(const double *theta, const int *voxels, const int *nodes, int K,
                                int L, int M, int nxn, int nyn, int nzn, int nxv, int nyv, int nzv,
                                int voxel, int x, int y, int z) {
    MILikelihoodFilter f(2.0, theta, 1, nodes, voxels, K, L, M, nxn, nyn, nzn, nxv, nyv, nzv);
    return f.compute_likelihood(voxel, x, y, z);
}

// accumulate_info over n (voxel, node, posterior) triples, then update_parameters and
// compute_cost (MILikelihoodFilter.cpp:87-124 and :38-51); theta_out [M][K][L]
double ref_mi_filter_update(double alpha, const double *theta, const int *voxels, const int *nodes,
                            int K, int L, int M, int nxn, int nyn, int nzn, int nxv, int nyv,
                            int nzv, int n, const int *vxyz, const double *post,
                            double *theta_out) {
    MILikelihoodFilter f(alpha, theta, 1, nodes, voxels, K, L, M, nxn, nyn, nzn, nxv, nyv, nzv);
    for (int t = 0; t < n; ++t)
        f.accumulate_info(0, vxyz[4 * t], vxyz[4 * t + 1], vxyz[4 * t + 2], vxyz[4 * t + 3],
                          post[t]);
    f.update_parameters();
    const auto th = f.get_parameters();
    std::memcpy(theta_out, th.data(), sizeof(double) * th.size());
    return f.compute_cost();
}

// SSDLikelihoodFilter::compute_log_likelihood (BINDER/src/cpu/SSDLikelihoodFilter.cpp:123-158)
double ref_ssdf_loglik(const double *coeff, const double *sigma, const double *nodes,
                       const double *voxels, int rfa, double alpha0, double beta0, int M, int F,
                       int nxn, int nyn, int nzn, int nxv, int nyv, int nzv, int voxel, int x,
                       int y, int z) {
    SSDLikelihoodFilter f(coeff, 1, sigma, nodes, voxels, rfa, alpha0, beta0, M, F, nxn, nyn, nzn,
                          nxv, nyv, nzv);
    return f.compute_log_likelihood(voxel, x, y, z);
}

// accumulate_info over n (voxel, node, posterior) triples, update_parameters, compute_cost
// (:160-346, :72-89); coeff_out [M][F], sigma_out [M]
double ref_ssdf_update(const double *coeff, const double *sigma, const double *nodes,
                       const double *voxels, int rfa, double alpha0, double beta0, int M, int F,
                       int nxn, int nyn, int nzn, int nxv, int nyv, int nzv, int n,
                       const int *vxyz, const double *post, double *coeff_out,
                       double *sigma_out) {
    // the class keeps a pointer to the voxel features: give it a copy that can be probed below
    std::vector<double> vox(voxels, voxels + (size_t)nxv * nyv * nzv * M);
    SSDLikelihoodFilter f(coeff, 1, sigma, nodes, vox.data(), rfa, alpha0, beta0, M, F, nxn, nyn,
                          nzn, nxv, nyv, nzv);
    for (int t = 0; t < n; ++t)
        f.accumulate_info(0, vxyz[4 * t], vxyz[4 * t + 1], vxyz[4 * t + 2], vxyz[4 * t + 3],
                          post[t]);
    f.update_parameters();
    const auto c = f.get_parameters();
    std::memcpy(coeff_out, c.data(), sizeof(double) * c.size());
    const double cost = f.compute_cost();
    // sigma is private: read it back through compute_log_likelihood at a node outside the grid,
    // where the log-likelihood of voxel 0 is sum_m (x_m^2 / (-2 sigma_m) + c_m).  With x = 0 that
    // is sum_m c_m; with x = X in channel m alone it adds -X^2 / (2 sigma_m).
    const double X = 1.0e4;
    for (int m = 0; m < M; ++m) vox[m] = 0.0;
    const double base = f.compute_log_likelihood(0, -1, -1, -1);
    for (int m = 0; m < M; ++m) {
        vox[m] = X;
        const double lm = f.compute_log_likelihood(0, -1, -1, -1);
        vox[m] = 0.0;
        sigma_out[m] = -(X * X) / (2.0 * (lm - base));
    }
    return cost;
}

// The reference's own EM driver (Registration.cpp:122-217) on `threads` threads: construction,
// setNonLinearTransformation, the MI likelihood (lk 0: theta [K][L]) or the SSD likelihood (lk 1:
// ssd = {sigmaSq, shiftScale, scale, shift, alpha_0, beta_0}), EM(max_iter, th, update); returns
// the final locations [V*N], get_likelihood_parameters (theta [K*L], or {scale, shift}) and the
// wall seconds of the EM call alone.
void ref_em(const double *final_locations, const double *voxel_pos, const double *node_pos,
            int nx, int ny, int nz, int nxn, int nyn, int nzn, int spline_order,
            double non_zero_voxels, const double gamma[3], const double rho[3],
            const double eta[3], const double *D, int lk, double alpha, const double *theta,
            int K, int L, const double *ssd, const int *nodes, const int *voxels, int max_iter,
            double th, int update, double *final_out, double *params_out, int threads,
            double *seconds) {
    Registration r(final_locations, threads, voxel_pos, node_pos, nx, ny, nz, nxn, nyn, nzn,
                   spline_order, non_zero_voxels);
    r.setNonLinearTransformation(gamma[0], gamma[1], gamma[2], rho[0], rho[1], rho[2], eta[0],
                                 eta[1], eta[2], D);
    if (lk == 0)
        r.setMILikelihood(alpha, theta, K, L, threads, nodes, voxels);
    else
        r.setSSDLikelihood(K, threads, ssd[0], (int)ssd[1], ssd[2], ssd[3], nodes, voxels, ssd[4],
                           ssd[5]);
    const auto t0 = std::chrono::steady_clock::now();
    r.EM(max_iter, th, update != 0, false);
    if (seconds)
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const auto f = r.get_final_locations();
    std::memcpy(final_out, f.data(), sizeof(double) * f.size());
    const auto p = r.get_likelihood_parameters();
    std::memcpy(params_out, p.data(), sizeof(double) * p.size());
}

// Registration::EM with a filter likelihood: lk 2 = setMILikelihoodFilter(alpha, theta [M][K][L],
// nodes, voxels (int bins), K, L, M); lk 3 = setSSDLikelihoodFilter(coeff [M][F], sigma [M],
// fnodes, fvoxels (features), rfa, alpha_0, beta_0, M, F).  params_out: theta or coeff.
void ref_em_filter(const double *final_locations, const double *voxel_pos, int nx, int ny, int nz,
                   int nxn, int nyn, int nzn, int spline_order, double non_zero_voxels,
                   const double gamma[3], const double *D, int lk, double alpha,
                   const double *theta, int K, int L, int M, const int *nodes, const int *voxels,
                   const double *coeff, const double *sigma, const double *fnodes,
                   const double *fvoxels, int rfa, double alpha0, double beta0, int F,
                   int max_iter, double th, int update, double *final_out, double *params_out) {
    Registration r(final_locations, 1, voxel_pos, voxel_pos, nx, ny, nz, nxn, nyn, nzn,
                   spline_order, non_zero_voxels);
    r.setNonLinearTransformation(gamma[0], gamma[1], gamma[2], 1, 1, 1, 1, 1, 1, D);
    if (lk == 2)
        r.setMILikelihoodFilter(alpha, theta, 1, nodes, voxels, K, L, M);
    else
        r.setSSDLikelihoodFilter(coeff, 1, sigma, fnodes, fvoxels, rfa, alpha0, beta0, M, F);
    r.EM(max_iter, th, update != 0, false);
    const auto f = r.get_final_locations();
    std::memcpy(final_out, f.data(), sizeof(double) * f.size());
    const auto p = r.get_likelihood_parameters();
    std::memcpy(params_out, p.data(), sizeof(double) * p.size());
}

// Registration::sampler (Registration.cpp:515-642) with the MI likelihood on `threads` threads:
// N_b + N_s sweeps with the given switches from the given positions and theta; mean_out [V*N]
// and cov_out [V*N*N] receive the sampler's moments (mean, M2 / (N_s - 1)); returns the wall
// seconds of the sampler call
double ref_sampler(const double *final_locations, const double *voxel_pos, int nx, int ny, int nz,
                   const double gamma[3], const double *D, double alpha, const double *theta,
                   int K, int L, const int *nodes, const int *voxels, int seed, int N_b, int N_s,
                   int sample_gamma, int every, int posteriors, int lik_params,
                   int transf_params, int threads, double *mean_out, double *cov_out) {
    Registration r(final_locations, threads, voxel_pos, voxel_pos, nx, ny, nz, nx, ny, nz, 3,
                   (double)nx * ny * nz);
    r.setNonLinearTransformation(gamma[0], gamma[1], gamma[2], 1, 1, 1, 1, 1, 1, D);
    r.setMILikelihood(alpha, theta, K, L, threads, nodes, voxels);
    const auto t0 = std::chrono::steady_clock::now();
    const auto res = r.sampler(seed, N_b, N_s, sample_gamma, every, posteriors, lik_params,
                               transf_params);
    const double sec =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (mean_out) std::memcpy(mean_out, res.first.data(), sizeof(double) * res.first.size());
    if (cov_out) std::memcpy(cov_out, res.second.data(), sizeof(double) * res.second.size());
    return sec;
}

// Registration::sampler with the SSD likelihood (setSSDLikelihood(bins, threads, sigmaSq,
// shiftScale, scale, shift, nodes, voxels, alpha_0, beta_0), ssd = {sigmaSq, shiftScale, scale,
// shift, alpha_0, beta_0}); mean_out / cov_out as ref_sampler; params_out = {scale, shift} after
// the last sweep (get_likelihood_parameters); returns the wall seconds of the sampler call.
double ref_sampler_ssd(const double *final_locations, const double *voxel_pos, int nx, int ny,
                       int nz, const double gamma[3], const double *D, int bins,
                       const double *ssd, const int *nodes, const int *voxels, int seed, int N_b,
                       int N_s, int sample_gamma, int every, int posteriors, int lik_params,
                       int transf_params, int threads, double *mean_out, double *cov_out,
                       double *params_out) {
    Registration r(final_locations, threads, voxel_pos, voxel_pos, nx, ny, nz, nx, ny, nz, 3,
                   (double)nx * ny * nz);
    r.setNonLinearTransformation(gamma[0], gamma[1], gamma[2], 1, 1, 1, 1, 1, 1, D);
    r.setSSDLikelihood(bins, threads, ssd[0], (int)ssd[1], ssd[2], ssd[3], nodes, voxels, ssd[4],
                       ssd[5]);
    const auto t0 = std::chrono::steady_clock::now();
    const auto res = r.sampler(seed, N_b, N_s, sample_gamma, every, posteriors, lik_params,
                               transf_params);
    const double sec =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (mean_out) std::memcpy(mean_out, res.first.data(), sizeof(double) * res.first.size());
    if (cov_out) std::memcpy(cov_out, res.second.data(), sizeof(double) * res.second.size());
    if (params_out) {
        const auto p = r.get_likelihood_parameters();
        std::memcpy(params_out, p.data(), sizeof(double) * p.size());
    }
    return sec;
}

// Registration::sampler with a filter likelihood, set up as ref_em_filter does (lk 2: the MI
// filter likelihood, lk 3: the SSD filter likelihood); mean_out / cov_out as ref_sampler;
// params_out receives get_likelihood_parameters after the last sweep (theta [M][K][L] or
// coeff [M][F]).
void ref_sampler_filter(const double *final_locations, const double *voxel_pos, int nx, int ny,
                        int nz, const double gamma[3], const double *D, int lk, double alpha,
                        const double *theta, int K, int L, int M, const int *nodes,
                        const int *voxels, const double *coeff, const double *sigma,
                        const double *fnodes, const double *fvoxels, int rfa, double alpha0,
                        double beta0, int F, int seed, int N_b, int N_s, int sample_gamma,
                        int every, int posteriors, int lik_params, int transf_params,
                        double *mean_out, double *cov_out, double *params_out) {
    Registration r(final_locations, 1, voxel_pos, voxel_pos, nx, ny, nz, nx, ny, nz, 3,
                   (double)nx * ny * nz);
    r.setNonLinearTransformation(gamma[0], gamma[1], gamma[2], 1, 1, 1, 1, 1, 1, D);
    if (lk == 2)
        r.setMILikelihoodFilter(alpha, theta, 1, nodes, voxels, K, L, M);
    else
        r.setSSDLikelihoodFilter(coeff, 1, sigma, fnodes, fvoxels, rfa, alpha0, beta0, M, F);
    const auto res = r.sampler(seed, N_b, N_s, sample_gamma, every, posteriors, lik_params,
                               transf_params);
    if (mean_out) std::memcpy(mean_out, res.first.data(), sizeof(double) * res.first.size());
    if (cov_out) std::memcpy(cov_out, res.second.data(), sizeof(double) * res.second.size());
    if (params_out) {
        const auto p = r.get_likelihood_parameters();
        std::memcpy(params_out, p.data(), sizeof(double) * p.size());
    }
}

// the same, the wall seconds alone
double ref_sampler_seconds(const double *final_locations, const double *voxel_pos, int nx, int ny,
                           int nz, const double gamma[3], const double *D, double alpha,
                           const double *theta, int K, int L, const int *nodes, const int *voxels,
                           int seed, int N_b, int N_s, int sample_gamma, int every,
                           int posteriors, int lik_params, int transf_params, int threads) {
    Registration r(final_locations, threads, voxel_pos, voxel_pos, nx, ny, nz, nx, ny, nz, 3,
                   (double)nx * ny * nz);
    r.setNonLinearTransformation(gamma[0], gamma[1], gamma[2], 1, 1, 1, 1, 1, 1, D);
    r.setMILikelihood(alpha, theta, K, L, threads, nodes, voxels);
    const auto t0 = std::chrono::steady_clock::now();
    const auto res = r.sampler(seed, N_b, N_s, sample_gamma, every, posteriors, lik_params,
                               transf_params);
    (void)res;
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"
