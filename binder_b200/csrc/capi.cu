// extern "C" boundary: status codes instead of exceptions, thread-local error text.
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/binder_b200.h"
#include "engine.cuh"
#include "initnet.cuh"
#include "multires.cuh"
#include "preprocess.cuh"
#include "resample.cuh"

struct binder_registration {
    binder::Registration *impl;
};
struct binder_transform {
    binder::PriorTransform *impl;
};
struct binder_pyramid {
    binder::Pyramid *impl;
};
struct binder_initnet {
    binder::InitNet *impl;
};
struct binder_batch {
    binder::RegistrationBatch *impl;
};

namespace {
thread_local std::string g_err;

template <typename F>
int guard(F &&f) {
    try {
        g_err.clear();
        f();
        return BINDER_STATUS_OK;
    } catch (const binder::Error &e) {
        g_err = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        g_err = "host allocation failed";
        return BINDER_STATUS_CUDA_ERROR;
    } catch (const std::exception &e) {
        g_err = e.what();
        return BINDER_STATUS_CUDA_ERROR;
    } catch (...) {
        g_err = "unknown error";
        return BINDER_STATUS_CUDA_ERROR;
    }
}

#define NEED(p)                                                                              \
    do {                                                                                     \
        if (!(p)) throw binder::Error(BINDER_STATUS_INVALID_ARGUMENT, #p " must not be NULL"); \
    } while (0)
}  // namespace

extern "C" {

const char *binder_last_error(void) { return g_err.c_str(); }
const char *binder_backend(void) { return "b200"; }
int binder_has_topology_correction(void) { return 1; }

int binder_registration_create(binder_registration **out, const float *final_locations,
                               int threads, const float *voxel_pos, const float *node_pos,
                               int Nx_v, int Ny_v, int Nz_v, int Nx_n, int Ny_n, int Nz_n,
                               int spline_order, double non_zero_voxels) {
    (void)threads;
    (void)node_pos;
    return guard([&] {
        NEED(out);
        NEED(final_locations);
        NEED(voxel_pos);
        *out = nullptr;
        auto *impl = new binder::Registration(final_locations, voxel_pos, Nx_v, Ny_v, Nz_v, Nx_n,
                                              Ny_n, Nz_n, spline_order, non_zero_voxels);
        *out = new binder_registration{impl};
    });
}

int binder_registration_destroy(binder_registration *h) {
    return guard([&] {
        if (!h) return;
        delete h->impl;
        delete h;
    });
}

int binder_registration_set_mi_likelihood(binder_registration *h, double alpha, const float *theta,
                                          int K, int L, int threads, const int32_t *binned_nodes,
                                          const int32_t *binned_voxels) {
    (void)threads;
    return guard([&] {
        NEED(h);
        NEED(theta);
        NEED(binned_nodes);
        NEED(binned_voxels);
        h->impl->set_mi_likelihood(alpha, theta, K, L, binned_nodes, binned_voxels);
    });
}

int binder_registration_set_mi_likelihood_filter(binder_registration *h, double alpha,
                                                 const float *theta, int threads,
                                                 const int32_t *binned_nodes,
                                                 const int32_t *binned_voxels, int K, int L,
                                                 int M) {
    (void)threads;
    return guard([&] {
        NEED(h);
        NEED(theta);
        NEED(binned_nodes);
        NEED(binned_voxels);
        h->impl->set_mi_filter_likelihood(alpha, theta, K, L, M, binned_nodes, binned_voxels);
    });
}

int binder_registration_set_ssd_likelihood(binder_registration *h, int bins, int threads,
                                           double sigma_sq, int scale_shift, double scale,
                                           double shift, const int32_t *binned_nodes,
                                           const int32_t *binned_voxels, double alpha_0,
                                           double beta_0) {
    (void)threads;
    return guard([&] {
        NEED(h);
        NEED(binned_nodes);
        NEED(binned_voxels);
        h->impl->set_ssd_likelihood(bins, sigma_sq, scale_shift, scale, shift, binned_nodes,
                                    binned_voxels, alpha_0, beta_0);
    });
}

int binder_registration_set_ssd_likelihood_filter(binder_registration *h, const double *coeff,
                                                  int threads, const double *sigma,
                                                  const double *features_nodes,
                                                  const double *features_voxels,
                                                  int reg_across_features, double alpha_0,
                                                  double beta_0, int M, int F) {
    (void)threads;
    return guard([&] {
        NEED(h);
        NEED(coeff);
        NEED(sigma);
        NEED(features_nodes);
        NEED(features_voxels);
        h->impl->set_ssd_filter_likelihood(coeff, sigma, features_nodes, features_voxels,
                                           reg_across_features, alpha_0, beta_0, M, F);
    });
}

int binder_registration_get_ssd_filter_parameters(const binder_registration *h, double *coeff,
                                                  double *sigma) {
    return guard([&] {
        NEED(h);
        h->impl->get_ssd_filter_parameters(coeff, sigma);
    });
}

int binder_registration_get_ssd_parameters(const binder_registration *h, double out[3]) {
    return guard([&] {
        NEED(h);
        NEED(out);
        h->impl->get_ssd_parameters(out);
    });
}

int binder_registration_set_nonlinear_transformation(binder_registration *h, double gamma_x,
                                                     double gamma_y, double gamma_z,
                                                     double voxels_size_x, double voxels_size_y,
                                                     double voxels_size_z, double nodes_size_x,
                                                     double nodes_size_y, double nodes_size_z,
                                                     const float *D) {
    return guard([&] {
        NEED(h);
        NEED(D);
        const double g[3] = {gamma_x, gamma_y, gamma_z};
        const double rho[3] = {voxels_size_x, voxels_size_y, voxels_size_z};
        const double eta[3] = {nodes_size_x, nodes_size_y, nodes_size_z};
        h->impl->set_nonlinear_transformation(g, rho, eta, D);
    });
}

int binder_registration_em(binder_registration *h, int max_iterations, double convergence_th,
                           int update_likelihood_parameters, int debug, int *iterations_out) {
    return guard([&] {
        NEED(h);
        const int it = h->impl->em(max_iterations, convergence_th, update_likelihood_parameters, debug);
        if (iterations_out) *iterations_out = it;
    });
}

int binder_registration_sampler(binder_registration *h, uint64_t seed, int N_b, int N_s,
                                int sample_gamma, int sample_gamma_every, int sample_posteriors,
                                int sample_likelihood_parameters,
                                int sample_transformation_parameters, double *mean_out,
                                double *cov_out) {
    return guard([&] {
        NEED(h);
        NEED(mean_out);
        NEED(cov_out);
        h->impl->sampler(seed, N_b, N_s, sample_gamma, sample_gamma_every, sample_posteriors,
                         sample_likelihood_parameters, sample_transformation_parameters, mean_out,
                         cov_out);
    });
}

int binder_registration_sampler_chains(binder_registration *h, uint64_t seed, int chains,
                                       int N_b, int N_s, int sample_gamma,
                                       int sample_gamma_every, int sample_posteriors,
                                       int sample_likelihood_parameters,
                                       int sample_transformation_parameters, double *mean_out,
                                       double *cov_out, double *pooled_mean_out,
                                       double *pooled_cov_out) {
    return guard([&] {
        NEED(h);
        h->impl->sampler_chains(seed, chains, N_b, N_s, sample_gamma, sample_gamma_every,
                                sample_posteriors, sample_likelihood_parameters,
                                sample_transformation_parameters, mean_out, cov_out,
                                pooled_mean_out, pooled_cov_out);
    });
}

int binder_registration_get_final_locations(const binder_registration *h, float *out) {
    return guard([&] {
        NEED(h);
        NEED(out);
        h->impl->get_final_locations(out);
    });
}

int binder_registration_get_dream_locations(const binder_registration *h, float *out) {
    return guard([&] {
        NEED(h);
        NEED(out);
        h->impl->get_dream_locations(out);
    });
}

int binder_registration_set_dream_locations(binder_registration *h, const float *in) {
    return guard([&] {
        NEED(h);
        NEED(in);
        h->impl->set_dream_locations(in);
    });
}

int binder_registration_add_displacement(binder_registration *h, const float *field, int Nx_f,
                                         int Ny_f, int Nz_f) {
    return guard([&] {
        NEED(h);
        NEED(field);
        h->impl->add_displacement(field, Nx_f, Ny_f, Nz_f);
    });
}

int binder_registration_get_likelihood_parameters(const binder_registration *h, float *out) {
    return guard([&] {
        NEED(h);
        NEED(out);
        h->impl->get_likelihood_parameters(out);
    });
}

int binder_registration_get_shape(const binder_registration *h, int out[4]) {
    return guard([&] {
        NEED(h);
        NEED(out);
        h->impl->get_shape(out);
    });
}

int binder_registration_get_iteration_stats(const binder_registration *h, double *out, int max_n,
                                            int *n_out) {
    return guard([&] {
        NEED(h);
        NEED(out);
        const int n = h->impl->get_iteration_stats(out, max_n);
        if (n_out) *n_out = n;
    });
}

int binder_registration_get_state(const binder_registration *h, double gamma_out[3],
                                  double *nu_out, unsigned long long *degenerate_out,
                                  unsigned *flags_out) {
    return guard([&] {
        NEED(h);
        h->impl->get_state(gamma_out, nu_out, degenerate_out, flags_out);
    });
}

int binder_registration_last_elapsed_ms(const binder_registration *h, double *ms_out) {
    return guard([&] {
        NEED(h);
        NEED(ms_out);
        *ms_out = h->impl->last_elapsed_ms();
    });
}

int binder_registration_set_stream(binder_registration *h, void *cuda_stream) {
    return guard([&] {
        NEED(h);
        h->impl->set_stream(reinterpret_cast<cudaStream_t>(cuda_stream));
    });
}

int binder_registration_set_chain(binder_registration *h, uint32_t chain) {
    return guard([&] {
        NEED(h);
        h->impl->set_chain(chain);
    });
}

int binder_registration_reset(binder_registration *h) {
    return guard([&] {
        NEED(h);
        h->impl->reset();
    });
}

int binder_registration_correct_topology(binder_registration *h, double e1, double e2,
                                         int max_outer_it, int max_it,
                                         const double voxel_sizes[3], long long *stats_out) {
    return guard([&] {
        NEED(h);
        NEED(voxel_sizes);
        const auto r = h->impl->correct_topology(e1, e2, max_outer_it, max_it, voxel_sizes);
        if (stats_out) {
            stats_out[0] = r.outer_iterations;
            stats_out[1] = r.inner_iterations;
            stats_out[2] = r.below_before;
            stats_out[3] = r.below_after;
            stats_out[4] = r.above_before;
            stats_out[5] = r.above_after;
        }
    });
}

int binder_registration_set_precision(binder_registration *h, int precision) {
    return guard([&] {
        NEED(h);
        h->impl->set_precision(precision);
    });
}

int binder_registration_set_histogram_precision(binder_registration *h, int precision) {
    return guard([&] {
        NEED(h);
        h->impl->set_histogram_precision(precision);
    });
}

int binder_transform_set_precision(binder_transform *h, int precision) {
    return guard([&] {
        NEED(h);
        h->impl->set_precision(precision);
    });
}

int binder_registration_get_stream(const binder_registration *h, void **stream_out) {
    return guard([&] {
        NEED(h);
        NEED(stream_out);
        *stream_out = reinterpret_cast<void *>(h->impl->stream());
    });
}

int binder_registration_profile_stage(binder_registration *h, int stage, int n, double *avg_ms_out) {
    return guard([&] {
        NEED(h);
        NEED(avg_ms_out);
        *avg_ms_out = h->impl->profile_stage(stage, n);
    });
}

long long binder_kernel_launch_count(void) { return binder::launch_counter(); }

// Page-locked host buffers for outputs, cached by size: a device-to-host copy into pinned memory
// runs at PCIe/C2C speed, one into fresh pageable memory pays the driver's staging and the first
// touch of every page.  Freed buffers are kept for reuse up to kPinnedCacheBytes in total.
namespace {
constexpr size_t kPinnedCacheBytes = size_t(8) << 30;
std::mutex g_pinned_mu;
std::multimap<size_t, void *> g_pinned_free;
size_t g_pinned_cached = 0;
}  // namespace

int binder_pinned_alloc(size_t bytes, void **out) {
    return guard([&] {
        NEED(out);
        *out = nullptr;
        BINDER_CHECK(bytes > 0, "size must be positive");
        {
            std::lock_guard<std::mutex> lock(g_pinned_mu);
            auto it = g_pinned_free.find(bytes);
            if (it != g_pinned_free.end()) {
                *out = it->second;
                g_pinned_cached -= bytes;
                g_pinned_free.erase(it);
                return;
            }
        }
        BINDER_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocDefault));
    });
}

int binder_pinned_free(void *p, size_t bytes) {
    return guard([&] {
        if (!p) return;
        {
            std::lock_guard<std::mutex> lock(g_pinned_mu);
            if (g_pinned_cached + bytes <= kPinnedCacheBytes) {
                g_pinned_free.emplace(bytes, p);
                g_pinned_cached += bytes;
                return;
            }
        }
        BINDER_CUDA(cudaFreeHost(p));
    });
}

int binder_transform_create(binder_transform **out, double gamma_x, double gamma_y,
                            double gamma_z, double voxels_size_x, double voxels_size_y,
                            double voxels_size_z, double nodes_size_x, double nodes_size_y,
                            double nodes_size_z, const float *D, int Nx_v, int Ny_v, int Nz_v,
                            int threads, double sigma_spline, double spline_offset) {
    (void)threads;
    (void)spline_offset;
    return guard([&] {
        NEED(out);
        NEED(D);
        *out = nullptr;
        const double g[3] = {gamma_x, gamma_y, gamma_z};
        const double rho[3] = {voxels_size_x, voxels_size_y, voxels_size_z};
        const double eta[3] = {nodes_size_x, nodes_size_y, nodes_size_z};
        auto *impl = new binder::PriorTransform(g, rho, eta, D, Nx_v, Ny_v, Nz_v, sigma_spline);
        *out = new binder_transform{impl};
    });
}

int binder_transform_destroy(binder_transform *h) {
    return guard([&] {
        if (!h) return;
        delete h->impl;
        delete h;
    });
}

int binder_transform_smooth_deformation(binder_transform *h, const float *field, float *out,
                                        double *log_prior_out) {
    return guard([&] {
        NEED(h);
        NEED(field);
        NEED(out);
        const double c = h->impl->smooth(field, out);
        if (log_prior_out) *log_prior_out = c;
    });
}

int binder_transform_sample_deformation_field(binder_transform *h, const float *field,
                                              int number_of_samples, float *out) {
    return guard([&] {
        NEED(h);
        NEED(field);
        NEED(out);
        h->impl->sample(field, number_of_samples, out);
    });
}

int binder_transform_get_shape(const binder_transform *h, int out[4]) {
    return guard([&] {
        NEED(h);
        NEED(out);
        h->impl->get_shape(out);
    });
}

int binder_pyramid_create(binder_pyramid **out, const int32_t *binned_voxels,
                          const int32_t *binned_nodes, const double *voxel_pos, int Nx_v, int Ny_v,
                          int Nz_v, int Nx_n, int Ny_n, int Nz_n,
                          const double voxels_voxel_size[3], const double nodes_voxel_size[3],
                          double gamma, int finite_difference_order,
                          int increase_gamma_at_DS_resolution, int upsample_in_frequency_domain,
                          int spline_order) {
    return guard([&] {
        NEED(out);
        NEED(binned_voxels);
        NEED(binned_nodes);
        NEED(voxels_voxel_size);
        NEED(nodes_voxel_size);
        *out = nullptr;
        binder::PyramidConfig c{};
        c.nx = Nx_v; c.ny = Ny_v; c.nz = Nz_v;
        c.nxn = Nx_n; c.nyn = Ny_n; c.nzn = Nz_n;
        for (int a = 0; a < 3; ++a) {
            c.voxel_size[a] = voxels_voxel_size[a];
            c.node_size[a] = nodes_voxel_size[a];
        }
        c.gamma_init = gamma;
        c.finite_difference_order = finite_difference_order;
        c.increase_gamma_at_ds = increase_gamma_at_DS_resolution;
        c.upsample_in_frequency_domain = upsample_in_frequency_domain;
        c.spline_order = spline_order;
        auto *impl = new binder::Pyramid(c, binned_voxels, binned_nodes, voxel_pos);
        *out = new binder_pyramid{impl};
    });
}

int binder_pyramid_destroy(binder_pyramid *p) {
    return guard([&] {
        if (!p) return;
        delete p->impl;
        delete p;
    });
}

int binder_pyramid_level(binder_pyramid *p, int resolution, const binder_registration *prev,
                         int prev_resolution, double alpha, const float *theta, int K, int L,
                         binder_registration **out, double info_out[16]) {
    return guard([&] {
        NEED(p);
        NEED(out);
        *out = nullptr;
        binder::LevelInfo li{};
        binder::Registration *r = p->impl->level(resolution, prev ? prev->impl : nullptr,
                                                 prev_resolution, alpha, theta, K, L, &li);
        *out = new binder_registration{r};
        if (info_out) {
            for (int a = 0; a < 3; ++a) {
                info_out[a] = li.voxels_shape[a];
                info_out[3 + a] = li.nodes_shape[a];
                info_out[6 + a] = li.gamma[a];
                info_out[9 + a] = li.voxel_size[a];
                info_out[12 + a] = li.node_size[a];
            }
            info_out[15] = li.non_zero_voxels;
        }
    });
}

int binder_bin_signal_robust(const void *signal, int is_double, long long n, int number_of_bins,
                             double lower_percentile, double higher_percentile,
                             int32_t *binned_out, double *bin_edges_out) {
    return guard([&] {
        NEED(signal);
        NEED(binned_out);
        if (is_double)
            binder::bin_signal_robust(static_cast<const double *>(signal), (long)n,
                                      number_of_bins, lower_percentile, higher_percentile,
                                      binned_out, bin_edges_out);
        else
            binder::bin_signal_robust(static_cast<const float *>(signal), (long)n,
                                      number_of_bins, lower_percentile, higher_percentile,
                                      binned_out, bin_edges_out);
    });
}

int binder_bin_signal(const void *signal, int is_double, long long n, int number_of_bins,
                      int32_t *binned_out) {
    return guard([&] {
        NEED(signal);
        NEED(binned_out);
        if (is_double)
            binder::bin_signal(static_cast<const double *>(signal), (long)n, number_of_bins,
                               binned_out);
        else
            binder::bin_signal(static_cast<const float *>(signal), (long)n, number_of_bins,
                               binned_out);
    });
}

int binder_center_of_mass(const int32_t *bins, int Nx, int Ny, int Nz, double out[3]) {
    return guard([&] {
        NEED(bins);
        NEED(out);
        if (!binder::center_of_mass_nonzero(bins, Nx, Ny, Nz, out))
            throw binder::Error(BINDER_STATUS_INVALID_ARGUMENT, "no voxel has a non-zero bin");
    });
}

int binder_warp_image(const double *image, int Nx, int Ny, int Nz, const double *positions,
                      long long M, int order, double *out) {
    return guard([&] {
        NEED(image);
        NEED(positions);
        NEED(out);
        binder::warp_image(image, Nx, Ny, Nz, positions, (long)M, order, out);
    });
}

int binder_transform_up_sample(const double *field, int Nx, int Ny, int Nz, int Nx_o, int Ny_o,
                               int Nz_o, int threads, double *out) {
    (void)threads;
    return guard([&] {
        NEED(field);
        NEED(out);
        binder::up_sample(field, Nx, Ny, Nz, Nx_o, Ny_o, Nz_o, out);
    });
}

int binder_resample_matrix(int kind, int n, int m, double *out) {
    return guard([&] {
        NEED(out);
        std::vector<double> M;
        if (kind == 0)
            binder::dct_upsample_matrix(n, m, M);
        else if (kind == 1)
            binder::linear_resize_matrix(n, m, M);
        else
            throw binder::Error(BINDER_STATUS_INVALID_ARGUMENT, "kind must be 0 or 1");
        std::memcpy(out, M.data(), sizeof(double) * M.size());
    });
}

int binder_resize_linear(const double *field, int Nx, int Ny, int Nz, int N, int Nx_o, int Ny_o,
                         int Nz_o, double scale, double *out) {
    return guard([&] {
        NEED(field);
        NEED(out);
        binder::resize_linear(field, Nx, Ny, Nz, N, Nx_o, Ny_o, Nz_o, scale, out);
    });
}

int binder_jacobian_determinant_3d(const double *field, int Nx, int Ny, int Nz, double voxel_size_x,
                                   double voxel_size_y, double voxel_size_z, double *J_out) {
    return guard([&] {
        NEED(field);
        NEED(J_out);
        BINDER_CHECK(Nx > 0 && Ny > 0 && Nz > 0, "dimensions must be positive");
        const long V = (long)Nx * Ny * Nz;
        double *df = nullptr, *dj = nullptr;
        BINDER_CUDA(cudaMalloc(&df, sizeof(double) * V * 3));
        try {
            BINDER_CUDA(cudaMalloc(&dj, sizeof(double) * V));
            BINDER_CUDA(cudaMemcpy(df, field, sizeof(double) * V * 3, cudaMemcpyHostToDevice));
            const double vs[3] = {voxel_size_x, voxel_size_y, voxel_size_z};
            binder::jacobian3d_device(df, Nx, Ny, Nz, vs, dj, 0);
            BINDER_CUDA(cudaMemcpy(J_out, dj, sizeof(double) * V, cudaMemcpyDeviceToHost));
        } catch (...) {
            cudaFree(df);
            cudaFree(dj);
            throw;
        }
        cudaFree(df);
        cudaFree(dj);
    });
}

int binder_jacobian_determinant_3d_noalloc(const double *field, int Nx, int Ny, int Nz,
                                           double voxel_size_x, double voxel_size_y,
                                           double voxel_size_z, double *J_out,
                                           double minmax_out[2], long long *negative_out) {
    return guard([&] {
        NEED(field);
        NEED(J_out);
        const double vs[3] = {voxel_size_x, voxel_size_y, voxel_size_z};
        binder::JacStats st{};
        binder::jacobian3d_noalloc(field, Nx, Ny, Nz, vs, J_out, &st);
        if (minmax_out) {
            minmax_out[0] = st.jmin;
            minmax_out[1] = st.jmax;
        }
        if (negative_out) *negative_out = st.negative;
    });
}

long long binder_jacobian_noalloc_max_voxels(void) { return binder::kJacobianNoAllocMaxVoxels; }

int binder_jacobian_determinant_2d(const double *field, int Nx, int Ny, double voxel_size_x,
                                   double voxel_size_y, double *J_out) {
    return guard([&] {
        NEED(field);
        NEED(J_out);
        const double vs[2] = {voxel_size_x, voxel_size_y};
        binder::jacobian2d(field, Nx, Ny, vs, J_out);
    });
}

int binder_topology_correct_2d(const double *field, double e1, double e2, int max_outer_it,
                               int max_it, int threads, const double voxel_sizes[2], int Nx,
                               int Ny, double *out, long long *stats_out) {
    (void)threads;
    return guard([&] {
        NEED(field);
        NEED(voxel_sizes);
        NEED(out);
        BINDER_CHECK(e1 <= 1.0 && e2 >= 1.0 && e1 < e2,
                     "topology correction needs e1 <= 1 <= e2 (the identity must be admissible)");
        const long V = (long)Nx * Ny;
        if (out != field) std::memcpy(out, field, sizeof(double) * V * 2);
        const auto r = binder::topology_correct_2d(out, e1, e2, max_outer_it, max_it, voxel_sizes,
                                                   Nx, Ny, 0);
        if (stats_out) {
            stats_out[0] = r.outer_iterations;
            stats_out[1] = r.inner_iterations;
            stats_out[2] = r.below_before;
            stats_out[3] = r.below_after;
            stats_out[4] = r.above_before;
            stats_out[5] = r.above_after;
        }
    });
}

int binder_topology_correct_3d(const double *field, double e1, double e2, int max_outer_it,
                               int max_it, int threads, const double voxel_sizes[3], int Nx,
                               int Ny, int Nz, double *out, long long *stats_out) {
    (void)threads;
    return guard([&] {
        NEED(field);
        NEED(voxel_sizes);
        NEED(out);
        BINDER_CHECK(e1 <= 1.0 && e2 >= 1.0 && e1 < e2,
                     "topology correction needs e1 <= 1 <= e2 (the identity must be admissible)");
        const long V = (long)Nx * Ny * Nz;
        if (out != field) std::memcpy(out, field, sizeof(double) * V * 3);
        const auto r = binder::topology_correct_3d(out, e1, e2, max_outer_it, max_it, voxel_sizes,
                                                   Nx, Ny, Nz, 0);
        if (stats_out) {
            stats_out[0] = r.outer_iterations;
            stats_out[1] = r.inner_iterations;
            stats_out[2] = r.below_before;
            stats_out[3] = r.below_after;
            stats_out[4] = r.above_before;
            stats_out[5] = r.above_after;
        }
    });
}

// ---- batches of registrations ----------------------------------------------------------------
int binder_batch_create(binder_registration *const *regs, int n, binder_batch **out) {
    return guard([&] {
        NEED(regs);
        NEED(out);
        *out = nullptr;
        BINDER_CHECK(n >= 1, "a batch needs at least one registration");
        std::vector<binder::Registration *> v;
        for (int i = 0; i < n; ++i) {
            NEED(regs[i]);
            v.push_back(regs[i]->impl);
        }
        auto *h = new binder_batch{nullptr};
        try {
            h->impl = new binder::RegistrationBatch(v);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int binder_batch_destroy(binder_batch *h) {
    return guard([&] {
        if (!h) return;
        delete h->impl;
        delete h;
    });
}

int binder_batch_em(binder_batch *h, int max_iterations, double convergence_th,
                    int update_likelihood_parameters, int *iterations_out, double *ms_out) {
    return guard([&] {
        NEED(h);
        NEED(iterations_out);
        h->impl->em(max_iterations, convergence_th, update_likelihood_parameters,
                    iterations_out);
        if (ms_out) *ms_out = h->impl->last_elapsed_ms();
    });
}

int binder_registration_set_estep_grid(binder_registration *h, int ctas) {
    return guard([&] {
        NEED(h);
        h->impl->set_estep_grid(ctas);
    });
}

// ---- learned initialiser ----------------------------------------------------------------------
int binder_gemm_bf16(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K) {
    return guard([&] {
        NEED(A);
        NEED(B);
        NEED(C);
        binder::gemm_bf16_host(A, B, C, M, N, K);
    });
}

int binder_initnet_create(binder_initnet **out, int batch, int size, int in_channels,
                          uint64_t seed) {
    return guard([&] {
        NEED(out);
        *out = nullptr;
        auto *h = new binder_initnet{nullptr};
        try {
            h->impl = new binder::InitNet(batch, size, seed, in_channels);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int binder_initnet_destroy(binder_initnet *h) {
    return guard([&] {
        if (!h) return;
        delete h->impl;
        delete h;
    });
}

int binder_initnet_parameter_count(const binder_initnet *h, long long *out) {
    return guard([&] {
        NEED(h);
        NEED(out);
        *out = h->impl->parameter_count();
    });
}

int binder_initnet_get_parameters(const binder_initnet *h, float *out) {
    return guard([&] {
        NEED(h);
        NEED(out);
        h->impl->get_parameters(out);
    });
}

int binder_initnet_set_parameters(binder_initnet *h, const float *in) {
    return guard([&] {
        NEED(h);
        NEED(in);
        h->impl->set_parameters(in);
    });
}

int binder_initnet_predict(binder_initnet *h, const float *in, float *out) {
    return guard([&] {
        NEED(h);
        NEED(in);
        NEED(out);
        h->impl->predict(in, out);
    });
}

int binder_initnet_train_step(binder_initnet *h, const float *in, const float *target, double lr,
                              double *loss_out, float *grads_out) {
    return guard([&] {
        NEED(h);
        NEED(in);
        NEED(target);
        const double l = h->impl->train_step(in, target, lr, grads_out);
        if (loss_out) *loss_out = l;
    });
}

int binder_initnet_gradients(binder_initnet *h, const float *in, const float *target,
                             double *loss_out, float *grads_out) {
    return guard([&] {
        NEED(h);
        NEED(in);
        NEED(target);
        const double l = h->impl->gradients(in, target, grads_out);
        if (loss_out) *loss_out = l;
    });
}

}  // extern "C"
