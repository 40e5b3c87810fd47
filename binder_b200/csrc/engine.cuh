// Registration and prior-transformation engines behind the C-ABI (one object per image pair).
#pragma once

#include <vector>

#include "estep.cuh"
#include "layout.cuh"
#include "topology.cuh"
#include "umma_transform.cuh"

namespace binder {

// device DCT matrices of one grid (forward C and inverse C^T per axis)
struct DctSet {
    int n[3] = {0, 0, 0};
    float *fwd[3] = {nullptr, nullptr, nullptr};
    float *inv[3] = {nullptr, nullptr, nullptr};
    UmmaMatrix ufwd[3], uinv[3];  // the same matrices preformatted for the tensor cores
    void init(int nx, int ny, int nz, cudaStream_t s);
    void release(cudaStream_t s);
};

// The DCT-prior M-step of BINDER/src/cpu/NonLinearTransformation.cpp:58-126 on SoA buffers:
// out = IDCT( DCT(r) / (1 + gamma sigma^2 D) [+ noise] ) + x, costs into st.
struct MStep {
    int nx = 0, ny = 0, nz = 0;
    long V = 0;
    DctSet dct;
    float *t1 = nullptr, *t2 = nullptr;
    int precision = kPrecFP32Simt;  // TransformPrecision
    // tensor-core passes: one CTA per 128-line tile with the components on their own streams, or
    // persistent (all components per launch, one CTA per SM; measured slower on B200)
    bool persistent = false;
    // 2D images up to 128 x 128: the whole M-step in one launch (mstep2d.cu)
    bool fused2d = false;
    // the tensor-core passes of components 1 and 2 run on their own streams (graph branches), so
    // one component's last partial wave of tiles overlaps the other components' passes
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    // a batch of chains: every pass runs over chains x components in one launch (per-tile
    // tensor-core passes or the SIMT passes), the scratch holds [chains][3][V]
    int chains = 1;
    // the sampler's prior noise of every coefficient, [chains][3][V] (prepare_sampling; null
    // until a sampler call needs it): drawn by one fully occupied kernel before the passes, so
    // the tensor-core epilogue only reads it
    float *noise = nullptr;
    // buffers from the stream-ordered pool on stream s
    void init(int nx, int ny, int nz, cudaStream_t s, int chains = 1);
    void prepare_sampling(cudaStream_t s);
    void release(cudaStream_t s);
    void enqueue(const float *r, float *d, const float *xpos, const float *D, DevState *st,
                 double sigma2, int sample, int want_raw, int every, uint64_t seed, uint32_t chain,
                 double rho_p, const double eta2[3], const int *skip, cudaStream_t s);
    void run_chain(AxisArgs<float> a, int c0, int nc, cudaStream_t s, const float *r, float *d,
                   const float *xpos, bool tc, int planes);
};

// A captured chunk of EM iterations, replayed by later EM calls while the parameters it was
// captured with (and every buffer it names) stay the same; the setters that change either clear it.
struct EmGraphCache {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    long long kernels = 0;
    int chunk = 0, max_iter = 0, update = 0;
    double th = 0.0;
    cudaStream_t stream = nullptr;
    const double *stats = nullptr;
    void clear();
};

class Registration {
  public:
    Registration(const float *final_locations, const float *voxel_pos, int nx, int ny, int nz,
                 int nxn, int nyn, int nzn, int spline_order, double non_zero_voxels);
    ~Registration();

    void set_mi_likelihood(double alpha, const float *theta, int K, int L, const int *binned_nodes,
                           const int *binned_voxels);
    // the SSD filter likelihood (BINDER/src/cpu/Registration.cpp:481-487): coeff [M][F] and sigma
    // [M] host memory, features_nodes [Vn][F] ([Vn][M] with reg_across_features) and
    // features_voxels [V][M] host or device memory; EM only
    void set_ssd_filter_likelihood(const double *coeff, const double *sigma,
                                   const double *features_nodes, const double *features_voxels,
                                   int reg_across_features, double alpha0, double beta0, int M,
                                   int F);
    // coeff [M][F], sigma [M]
    void get_ssd_filter_parameters(double *coeff, double *sigma) const;
    int ssd_filter_channels(int *F) const {
        if (F) *F = fF_;
        return fM_;
    }
    // the MI filter likelihood (BINDER/src/cpu/Registration.cpp:466-470): M channels, theta
    // [M][K][L], bins of channel m read at [index + m]; EM only
    void set_mi_filter_likelihood(double alpha, const float *theta, int K, int L, int M,
                                  const int *binned_nodes, const int *binned_voxels);
    void set_nonlinear_transformation(const double gamma[3], const double rho[3],
                                      const double eta[3], const float *D);
    // the SSD likelihood instead of MI (BINDER/src/cpu/Registration.cpp:472-479), EM only
    void set_ssd_likelihood(int bins, double sigma2, int shift_scale, double scale, double shift,
                            const int *binned_nodes, const int *binned_voxels, double alpha0,
                            double beta0);
    void get_ssd_parameters(double out[3]) const;  // sigma^2, shift, scale
    int em(int max_iterations, double convergence_th, int update_likelihood_parameters, int debug);
    void sampler(uint64_t seed, int N_b, int N_s, int sample_gamma, int sample_gamma_every,
                 int sample_posteriors, int sample_likelihood_parameters,
                 int sample_transformation_parameters, double *mean_out, double *cov_out);
    // `chains` independent chains of the sampler in one pass per step: chain c draws Philox chain
    // index chain_ + c (what sampler() draws after set_chain(chain_ + c)) and starts from the
    // object's current positions, theta and gammas, which stay as they are.  Per-chain moments
    // mean_out [chains][V][N] / cov_out [chains][V][N][N], and / or the chains' pooled moments
    // pooled_mean [V][N] / pooled_cov [V][N][N]; any output may be null.
    void sampler_chains(uint64_t seed, int chains, int N_b, int N_s, int sample_gamma,
                        int sample_gamma_every, int sample_posteriors,
                        int sample_likelihood_parameters, int sample_transformation_parameters,
                        double *mean_out, double *cov_out, double *pooled_mean,
                        double *pooled_cov);

    // em() in pieces, for running many registrations in one graph (RegistrationBatch): a fresh
    // state and statistics buffer (host-synchronising), n iterations enqueued on stream s (each
    // a no-op once the convergence rule has fired), and the iteration count afterwards
    void em_prepare(int max_iterations);
    void enqueue_em(int n, int max_iterations, double th, int update, cudaStream_t s);
    int em_finish(double ms);
    bool em_done() const;
    // CTAs of the EM E-step launch (0: every SM times its occupancy, the default)
    void set_estep_grid(int g);
    long voxels() const { return V_; }

    // restore the positions given at construction, the theta given to set_mi_likelihood, the
    // gammas given to set_nonlinear_transformation and a fresh device state (device-to-device,
    // no host transfer)
    void reset();
    // topology correction of the object's own positions on the device (FP64), in place
    TopologyResult correct_topology(double e1, double e2, int max_outer, int max_inner,
                                    const double vs[3]);

    void get_final_locations(float *out) const;      // AoS [V][3]
    void set_final_locations(const float *in);
    void get_dream_locations(float *out) const;      // AoS [V][3]
    void set_dream_locations(const float *in);
    // positions += the order-1 resize of a displacement field on an fx x fy x fz grid (AoS FP32
    // [fx][fy][fz][N], host or device memory); theta and the other state are kept
    void add_displacement(const float *field, int fx, int fy, int fz);
    void get_likelihood_parameters(float *out) const;  // [K*L]
    void get_shape(int out[4]) const;
    int get_iteration_stats(double *out, int max_n) const;  // [n][4]: mll, lp_lik, lp_tr, mlp
    void get_state(double *gamma_out, double *nu_out, unsigned long long *degenerate,
                   unsigned *flags) const;
    void set_stream(cudaStream_t s);
    void set_chain(uint32_t c);
    void set_precision(int p);
    // E-step bin columns of the MI likelihood: 0 FP32 (the default), 1 FP16
    void set_histogram_precision(int h);
    int histogram_precision() const { return hist_prec_; }
    double last_elapsed_ms() const { return last_ms_; }
    cudaStream_t stream() const { return stream_; }
    // the device flag the EM bookkeeping sets once this object's convergence rule fires
    const int *done_flag() const { return &st_->done; }
    // average ms per launch of stage 0 (E-step), 1 (M-step) or 2 (theta update), n eager launches
    double profile_stage(int stage, int n);

    int K() const { return K_; }
    int L() const { return L_; }
    // device views for the multi-resolution step; valid while no call on this object runs
    const float *positions_device() const { return d_; }  // SoA [N][V], grid units
    const float *theta_device() const { return theta_; }  // [K][L] or null before set-up
    int components() const { return N_; }
    void dims(int out[3]) const { out[0] = nx_; out[1] = ny_; out[2] = nz_; }

  private:
    // grid dimensions as the E-step sees them (a 2D image nx x ny is the volume nx x 1 x ny)
    struct View {
        int nx, ny, nz, nxn, nyn, nzn;
    };
    View estep_view() const;
    GridDims grid_dims() const;
    EStepArgs estep_args(const int *skip) const;
    void enqueue_em_iteration(int max_iter, double th, int update, cudaStream_t s);
    void reset_state(bool for_sampler);
    void require_ready() const;
    // bins, theta and histogram buffers of an M-channel MI-type likelihood
    void load_bins(double alpha, const float *theta, int K, int L, int M, const int *binned_nodes,
                   const int *binned_voxels);

    int nx_, ny_, nz_, nxn_, nyn_, nzn_, N_;
    long V_, Vn_;
    double nzv_;
    // own_stream_ owns the buffers (pool allocations and frees); stream_ (own_stream_ unless the
    // caller set one) carries the copies and kernels
    cudaStream_t stream_ = 0, own_stream_ = 0;
    // the likelihood update of an EM iteration runs on lk_stream_, beside the M-step
    cudaStream_t lk_stream_ = nullptr;
    cudaEvent_t lk_fork_ = nullptr, lk_join_ = nullptr;
    uint32_t chain_ = 0;
    // device buffers
    float *d_ = nullptr, *x_ = nullptr, *r_ = nullptr, *D_ = nullptr, *theta_ = nullptr,
          *hist_ = nullptr, *d0_ = nullptr, *theta0_ = nullptr;
    TopologyWorkspace *topo_ = nullptr;
    unsigned *hcnt_ = nullptr;
    uint8_t *u_ = nullptr, *vpad_ = nullptr;
    unsigned long long *hfix_ = nullptr;  // order-independent EM histogram merge (EStepArgs)
    double *mpart_ = nullptr;
    unsigned *hdone_ = nullptr;
    double *mean_ = nullptr, *m2_ = nullptr, *stats_ = nullptr;
    int stats_cap_ = 0;
    DevState *st_ = nullptr;
    MStep mstep_;
    EmGraphCache em_graph_;
    // buffers of the last batch of chains (kept for the next call with the same count)
    struct ChainBatch {
        int chains = 0;
        float *d = nullptr, *r = nullptr, *theta = nullptr;
        unsigned *hcnt = nullptr;
        DevState *st = nullptr;
        double *mean = nullptr, *m2 = nullptr;
        MStep mstep;
    };
    ChainBatch *cb_ = nullptr;
    void release_chains();
    int estep_grid_override_ = 0;
    // likelihood / prior parameters
    bool have_mi_ = false, have_tr_ = false;
    int K_ = 0, L_ = 0;
    int M_ = 1;      // channels of the MI filter likelihood (1 otherwise)
    long vch_ = 0;   // bytes between the channels' padded bin volumes
    double alpha_ = 2.0;
    double gamma0_[3] = {0, 0, 0}, rho_[3] = {1, 1, 1}, eta_[3] = {1, 1, 1};
    double gamma_set_[3] = {0, 0, 0};  // as given to set_nonlinear_transformation (reset restores)
    double sigma2_ = 0.0;
    int P_ = 8, PZ_ = 8, pyn_ = 0, zp_ = 0;
    int egrid_e_ = 0, egrid_s_ = 0;
    int hist_prec_ = 0;  // set_histogram_precision
    uint64_t seed_ = 12345;
    int iters_done_ = 0;
    int order_ = 3;  // B-spline order of the E-step
    int lk_ = 0;     // likelihood: 0 MI (theta_ is theta), 1 SSD (theta_ is its log2 table),
                     // 2 MI filter (theta_ is [M][K][L]), 3 SSD filter (the f* buffers)
    double *fx_ = nullptr, *fn_ = nullptr;          // SSD filter: voxel / node features (SoA)
    SsdfState *fst_ = nullptr, *fst0_ = nullptr;    // SSD filter parameters, and as set
    double *fstats_ = nullptr;                      // SSD filter E-step statistics
    int fM_ = 0, fF_ = 0, fFn_ = 0;
    SsdState *ssd_ = nullptr, *ssd0_ = nullptr;  // SSD parameters, and as set
    float *colmax_ = nullptr, *colmax0_ = nullptr;  // SSD table column maxima, and as set
    double last_ms_ = 0.0;
};

// Many registrations -- image pairs of any sizes, each its own Registration -- run as one: every
// chunk of EM iterations is one CUDA graph holding each pair's kernels on a branch of its own, so
// the pairs' kernels overlap on the GPU and the whole batch advances with one graph launch per
// chunk.  Each pair keeps its own convergence test (its kernels become no-ops once it fires).
class RegistrationBatch {
  public:
    explicit RegistrationBatch(const std::vector<Registration *> &regs);
    ~RegistrationBatch();
    // Registration::em for every pair; its_out[i] receives pair i's iteration count
    void em(int max_iterations, double convergence_th, int update, int *its_out);
    double last_elapsed_ms() const { return last_ms_; }
    int size() const { return (int)regs_.size(); }

  private:
    std::vector<Registration *> regs_;
    cudaStream_t master_ = nullptr;
    std::vector<cudaStream_t> branch_;
    cudaEvent_t fork_ = nullptr;
    std::vector<cudaEvent_t> join_;
    int *done_host_ = nullptr;  // page-locked copies of the pairs' done flags
    double last_ms_ = 0.0;
};

// _core.NonLinearTransformation: smoothing and prior sampling of a displacement field
class PriorTransform {
  public:
    PriorTransform(const double gamma[3], const double rho[3], const double eta[3], const float *D,
                   int nx, int ny, int nz, double sigma_spline);
    ~PriorTransform();
    double smooth(const float *field_aos, float *out_aos);
    void sample(const float *field_aos, int n, float *out_aos);
    void get_shape(int out[4]) const;
    void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
    void set_precision(int p);

  private:
    int nx_, ny_, nz_;
    long V_;
    int N_ = 3;  // displacement components (2 for an image)
    double gamma_[3], rho_[3], eta_[3], sigma2_;
    float *D_ = nullptr, *r_ = nullptr, *d_ = nullptr, *zeros_ = nullptr, *chunk_ = nullptr;
    DevState *st_ = nullptr;
    MStep mstep_;
    cudaStream_t stream_ = 0, own_stream_ = 0;
    uint64_t seed_ = 1234;
    int sweep_ = 0;
};

// default transform precision: BINDER_B200_PRECISION (0 FP32 SIMT, 1 3xTF32, 2 TF32) or 3xTF32
int default_precision();
// default tensor-core pass kind: BINDER_B200_PERSISTENT (0 per-tile CTAs, 1 persistent) or 0
bool default_persistent();


}  // namespace binder
