// Registration / sampling engines: device buffers, CUDA-graph-captured iteration chunks and the
// device-side convergence test of the EM loop (BINDER/src/cpu/Registration.cpp:122-217,
// :515-642; BINDER/src/gpu/Registration.cu:839-1026).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "engine.cuh"
#include "layout.cuh"
#include "mstep2d.cuh"
#include "resample.cuh"

namespace binder {

namespace {

// device buffers come from the stream-ordered pool (layout.cuh)
template <typename T>
T *dalloc(size_t n, cudaStream_t s) {
    return dev_alloc_n<T>(n, s);
}
template <typename T>
void dfree(T *&p, cudaStream_t s) {
    dev_free_p(p, s);
}

bool verbose() {
    const char *v = std::getenv("BINDER_B200_VERBOSE");
    return v && v[0] && v[0] != '0';
}

// the B-spline prior's standard deviation for cubic splines, sqrt(9 / (8 pi))
// (BINDER/src/cpu/Spline.cpp:22)
// sigma_spline^2 of the Gaussian approximating the B-spline of each order
// (BINDER/src/cpu/Spline.cpp:19-41): sqrt(9 / (8 pi)), sqrt(8 / (9 pi)), 0.4
double spline_sigma2(int order) {
    const double pi = 3.14159265358979323846;
    if (order == 2) return 8.0 / (9.0 * pi);
    if (order == 1) return 0.4 * 0.4;
    return 9.0 / (8.0 * pi);
}

struct Graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~Graph() {
        if (e) cudaGraphExecDestroy(e);
        if (g) cudaGraphDestroy(g);
    }
};

// Capture `enqueue` into `graph` on stream s.  Kernels counted while capturing are taken back out
// of the launch counter and returned, so each replay can add them again.
template <typename F>
long long capture_graph(cudaStream_t s, Graph &graph, F &&enqueue) {
    const long long before = launch_counter();
    BINDER_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    try {
        enqueue();
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        launch_counter() = before;
        throw;
    }
    BINDER_CUDA(cudaStreamEndCapture(s, &graph.g));
    BINDER_CUDA(cudaGraphInstantiate(&graph.e, graph.g, 0));
    const long long captured = launch_counter() - before;
    launch_counter() = before;
    return captured;
}

void replay(const Graph &graph, long long kernels, cudaStream_t s) {
    BINDER_CUDA(cudaGraphLaunch(graph.e, s));
    count_launch(kernels);
}

}  // namespace

void EmGraphCache::clear() {
    if (e) cudaGraphExecDestroy(e);
    if (g) cudaGraphDestroy(g);
    e = nullptr;
    g = nullptr;
    kernels = 0;
}

long long &launch_counter() {
    static long long counter = 0;
    return counter;
}

// ------------------------------------------------------------------------------------------
void DctSet::init(int nx, int ny, int nz, cudaStream_t s) {
    const int dims[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        const int m = dims[a];
        n[a] = m;
        // the unit z axis of a 2D image has no transform; a unit axis of the image itself has
        // the 1 x 1 identity
        if (a == 2 && nz == 1) continue;
        std::vector<double> C((size_t)m * m);
        dct2_matrix(m, C.data());
        std::vector<float> F((size_t)m * m), I((size_t)m * m);
        for (int k = 0; k < m; ++k)
            for (int j = 0; j < m; ++j) {
                F[(size_t)k * m + j] = (float)C[(size_t)k * m + j];
                I[(size_t)j * m + k] = (float)C[(size_t)k * m + j];
            }
        fwd[a] = dalloc<float>((size_t)m * m, s);
        inv[a] = dalloc<float>((size_t)m * m, s);
        std::vector<double> CT((size_t)m * m);
        for (int k = 0; k < m; ++k)
            for (int j = 0; j < m; ++j) CT[(size_t)j * m + k] = C[(size_t)k * m + j];
        ufwd[a].init(C.data(), m, s);
        uinv[a].init(CT.data(), m, s);
        BINDER_CUDA(cudaMemcpyAsync(fwd[a], F.data(), sizeof(float) * m * m,
                                    cudaMemcpyHostToDevice, s));
        BINDER_CUDA(cudaMemcpyAsync(inv[a], I.data(), sizeof(float) * m * m,
                                    cudaMemcpyHostToDevice, s));
        BINDER_CUDA(cudaStreamSynchronize(s));  // F and I go out of scope
    }
}

void DctSet::release(cudaStream_t s) {
    for (int a = 0; a < 3; ++a) {
        dfree(fwd[a], s);
        dfree(inv[a], s);
        ufwd[a].release(s);
        uinv[a].release(s);
    }
}

void MStep::init(int x, int y, int z, cudaStream_t s, int nchains) {
    nx = x; ny = y; nz = z;
    V = (long)x * y * z;
    chains = nchains < 1 ? 1 : nchains;
    dct.init(x, y, z, s);
    t1 = dalloc<float>((size_t)V * 3 * chains, s);
    t2 = dalloc<float>((size_t)V * 3 * chains, s);
    precision = default_precision();
    // a persistent CTA's tiles span components (its cost sums could mix chains), and the fused 2D
    // M-step runs one chain
    persistent = chains == 1 && default_persistent();
    {
        const char *e = std::getenv("BINDER_B200_FUSED2D");
        const bool off = e && e[0] == '0' && e[1] == 0;
        fused2d = chains == 1 && !off && z == 1 && x <= kM2dMaxN && y <= kM2dMaxN;
    }
    for (int i = 0; i < 2; ++i) {
        BINDER_CUDA(cudaStreamCreate(&side[i]));
        BINDER_CUDA(cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming));
    }
    BINDER_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
}

bool default_persistent() {
    const char *e = std::getenv("BINDER_B200_PERSISTENT");
    return e && e[0] == '1' && e[1] == 0;
}

int default_precision() {
    const char *e = std::getenv("BINDER_B200_PRECISION");
    if (e && e[0] >= '0' && e[0] <= '4' && e[1] == 0) return e[0] - '0';
    // the BF16 split: FP32-level error at the full size (its FP64 error table is in the tests)
    // and fewer shared-memory bytes per pass than the TF32 split
    return kPrecBF16x3;
}

void MStep::prepare_sampling(cudaStream_t s) {
    if (!noise) noise = dalloc<float>((size_t)V * 3 * chains, s);
}

void MStep::release(cudaStream_t s) {
    dct.release(s);
    dfree(t1, s);
    dfree(t2, s);
    dfree(noise, s);
    for (int i = 0; i < 2; ++i) {
        if (side[i]) cudaStreamSynchronize(side[i]), cudaStreamDestroy(side[i]);
        if (join[i]) cudaEventDestroy(join[i]);
        side[i] = nullptr;
        join[i] = nullptr;
    }
    if (fork) cudaEventDestroy(fork);
    fork = nullptr;
}

void MStep::enqueue(const float *r, float *d, const float *xpos, const float *D, DevState *st,
                    double sigma2, int sample, int want_raw, int every, uint64_t seed,
                    uint32_t chain, double rho_p, const double eta2[3], const int *skip,
                    cudaStream_t s) {
    AxisArgs<float> a{};
    a.comp_stride = V;
    a.st = st;
    a.skip = skip;
    a.ny = ny;
    a.nz = nz;
    const int ncomp = nz == 1 ? 2 : 3;
    a.dims = ncomp;
    if (fused2d) {
        a.comp0 = 0;
        a.xpos = xpos;
        a.D = D; a.sigma2 = sigma2; a.sample = sample; a.want_raw = want_raw;
        a.every = every < 1 ? 1 : every; a.seed = seed; a.chain = chain; a.rho_p = rho_p;
        for (int n = 0; n < 3; ++n) a.eta2[n] = eta2[n];
        launch_mstep2d(a, r, d, nx, ny, dct.fwd[0], dct.inv[0], dct.fwd[1], dct.inv[1], s);
        return;
    }
    a.D = D; a.sigma2 = sigma2; a.sample = sample; a.want_raw = want_raw;
    a.every = every < 1 ? 1 : every; a.seed = seed; a.chain = chain; a.rho_p = rho_p;
    for (int n = 0; n < 3; ++n) a.eta2[n] = eta2[n];
    const bool tc = precision != kPrecFP32Simt;
    const int planes = (precision == kPrecTF32 || precision == kPrecBF16) ? 1 : 2;
    const bool bf16 = precision == kPrecBF16x3 || precision == kPrecBF16;
    // the per-tile tensor-core passes read the prior noise drawn beforehand by one fully occupied
    // kernel (the persistent and CUDA-core passes draw it per element)
    if (sample && tc && !(persistent && !bf16)) {
        BINDER_CHECK(noise, "sampling on the tensor-core passes needs MStep::prepare_sampling first");
        launch_prior_noise(noise, V, ncomp * chains, chains > 1 ? ncomp : 0, seed, chain, st, skip,
                           s);
        a.noise = noise;
    }
    if (chains > 1) {
        // chains x components per launch: enough tiles to fill the GPU without stream branches
        a.chain_comps = ncomp;
        run_chain(a, 0, ncomp * chains, s, r, d, xpos, tc, planes);
        return;
    }
    // the tensor-core path runs one chain of passes per component, each on its own stream
    const bool branches = tc && !persistent && side[0] && side[1];
    if (branches) {
        BINDER_CUDA(cudaEventRecord(fork, s));
        for (int c = 1; c < ncomp; ++c) BINDER_CUDA(cudaStreamWaitEvent(side[c - 1], fork, 0));
        for (int c = 0; c < ncomp; ++c)
            run_chain(a, c, 1, c == 0 ? s : side[c - 1], r, d, xpos, tc, planes);
        for (int c = 1; c < ncomp; ++c) {
            BINDER_CUDA(cudaEventRecord(join[c - 1], side[c - 1]));
            BINDER_CUDA(cudaStreamWaitEvent(s, join[c - 1], 0));
        }
    } else {
        run_chain(a, 0, ncomp, s, r, d, xpos, tc, planes);
    }
}

// the pass sequence of one M-step for components [c0, c0 + nc) on stream s
void MStep::run_chain(AxisArgs<float> a, int c0, int nc, cudaStream_t s, const float *r, float *d,
                  const float *xpos, bool tc, int planes) {
    a.comp0 = c0;
    const bool two_d = nz == 1;
    const bool bf16 = precision == kPrecBF16x3 || precision == kPrecBF16;
    auto pass = [&](int axis, bool inverse, int mode) {
        if (tc)
            launch_axis_pass_tc(a, inverse ? dct.uinv[axis] : dct.ufwd[axis],
                                mode == kEpiSpectral ? &dct.uinv[axis] : nullptr, mode, nc,
                                planes, s, persistent && !bf16, bf16);
        else
            launch_axis_pass(a, mode, nc, s);
    };
    if (two_d) {
        // an nx x ny image, components (x, y): forward along y, then x with the prior scaling,
        // inverse along x, and the inverse along y adds the pixel positions
        a.in = r; a.out = t1; a.M = dct.fwd[1]; a.n = ny; a.outer = nx; a.s = 1;
        pass(1, false, kEpiNone);
        a.in = t1; a.out = t2; a.M = dct.fwd[0]; a.M2 = dct.inv[0]; a.n = nx; a.outer = 1; a.s = ny;
        const float *yin = t2;
        if (tc) {
            pass(0, false, kEpiSpectralOut);
            a.in = t2; a.out = t1; a.M2 = nullptr;
            pass(0, true, kEpiNone);
            yin = t1;
        } else {
            pass(0, false, kEpiSpectral);
        }
        a.in = yin; a.out = d; a.M = dct.inv[1]; a.M2 = nullptr; a.n = ny; a.outer = nx; a.s = 1;
        a.xpos = xpos;
        pass(1, true, kEpiPositions);
        return;
    }
    // forward DCT-II along z, y
    a.in = r; a.out = t1; a.M = dct.fwd[2]; a.n = nz; a.outer = (long)nx * ny; a.s = 1;
    pass(2, false, kEpiNone);
    a.in = t1; a.out = t2; a.M = dct.fwd[1]; a.n = ny; a.outer = nx; a.s = nz;
    pass(1, false, kEpiNone);
    // x: forward, prior scaling (+ noise, costs), inverse.  The CUDA-core path fuses the three in
    // one pass; the tensor-core path stores the scaled coefficients and runs the inverse as its
    // own pass, so neither needs more than half of an SM's TMEM (two CTAs per SM).
    a.in = t2; a.out = t1; a.M = dct.fwd[0]; a.M2 = dct.inv[0]; a.n = nx; a.outer = 1;
    a.s = (long)ny * nz;
    const float *yin = t1;
    float *yout = t2;
    if (tc) {
        pass(0, false, kEpiSpectralOut);
        a.in = t1; a.out = t2; a.M2 = nullptr;
        pass(0, true, kEpiNone);
        yin = t2;
        yout = t1;
    } else {
        pass(0, false, kEpiSpectral);
    }
    // inverse DCT-III along y, z; the last pass adds the voxel positions
    a.in = yin; a.out = yout; a.M = dct.inv[1]; a.M2 = nullptr; a.n = ny; a.outer = nx; a.s = nz;
    pass(1, true, kEpiNone);
    a.in = yout; a.out = d; a.M = dct.inv[2]; a.n = nz; a.outer = (long)nx * ny; a.s = 1;
    a.xpos = xpos;
    pass(2, true, kEpiPositions);
}

// ------------------------------------------------------------------------------------------
Registration::Registration(const float *final_locations, const float *voxel_pos, int nx, int ny,
                           int nz, int nxn, int nyn, int nzn, int spline_order,
                           double non_zero_voxels)
    : nx_(nx), ny_(ny), nz_(nz), nxn_(nxn), nyn_(nyn), nzn_(nzn) {
    BINDER_CHECK(nx > 0 && ny > 0 && nz > 0 && nxn > 0 && nyn > 0 && nzn > 0,
                 "grid dimensions must be positive");
    if (spline_order < 1 || spline_order > 3)
        throw Error(kUnsupported, "spline_order must be 1, 2 or 3");
    order_ = spline_order;
    BINDER_CHECK((long)nx * ny * nz < (1L << 31), "volume too large");
    BINDER_CHECK(nz > 1 || nzn == 1, "a 2D image (Nz_v == 1) needs a 2D node grid (Nz_n == 1)");
    N_ = nz == 1 ? 2 : 3;  // a 2D image has two displacement components
    V_ = (long)nx * ny * nz;
    Vn_ = (long)nxn * nyn * nzn;
    nzv_ = non_zero_voxels;
    BINDER_CUDA(cudaStreamCreate(&own_stream_));
    stream_ = own_stream_;
    const cudaStream_t s = own_stream_;
    const GridDims g = grid_dims();
    const size_t VN = (size_t)V_ * N_;
    d_ = dalloc<float>(VN, s);
    r_ = dalloc<float>(VN, s);
    d0_ = dalloc<float>(VN, s);
    st_ = dalloc<DevState>(1, s);
    BINDER_CUDA(cudaMemsetAsync(st_, 0, sizeof(DevState), s));
    // the caller's AoS arrays go to the device as they are (r_ is the staging buffer) and are
    // rearranged there
    // inputs may be host or device memory (the multi-resolution step passes device arrays)
    BINDER_CUDA(cudaMemcpyAsync(r_, final_locations, sizeof(float) * VN, cudaMemcpyDefault, s));
    launch_aos_to_soa(r_, d_, V_, N_, s);
    BINDER_CUDA(cudaMemcpyAsync(d0_, d_, sizeof(float) * VN, cudaMemcpyDeviceToDevice, s));
    // the identity voxel grid (the common case) is recomputed in the kernels instead of read
    if (voxel_pos != final_locations)
        BINDER_CUDA(cudaMemcpyAsync(r_, voxel_pos, sizeof(float) * VN, cudaMemcpyDefault, s));
    launch_identity_check(r_, g, &st_->flags, s);
    unsigned mismatch = 0;
    BINDER_CUDA(cudaMemcpyAsync(&mismatch, &st_->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    if (mismatch) {
        x_ = dalloc<float>(VN, s);
        launch_aos_to_soa(r_, x_, V_, N_, s);
    }
    BINDER_CUDA(cudaMemsetAsync(st_, 0, sizeof(DevState), s));
    // dream locations start at zero: r = 0 - x
    launch_aos_minus_to_soa(nullptr, x_, g, r_, s);
    mstep_.init(nx, ny, nz, s);
    BINDER_CUDA(cudaStreamCreate(&lk_stream_));
    BINDER_CUDA(cudaEventCreateWithFlags(&lk_fork_, cudaEventDisableTiming));
    BINDER_CUDA(cudaEventCreateWithFlags(&lk_join_, cudaEventDisableTiming));
    BINDER_CUDA(cudaStreamSynchronize(s));
}

Registration::~Registration() {
    // nothing of this object may still run when its buffers go back to the pool
    if (stream_ != own_stream_) cudaStreamSynchronize(stream_);
    cudaStreamSynchronize(own_stream_);
    if (lk_stream_) cudaStreamSynchronize(lk_stream_), cudaStreamDestroy(lk_stream_);
    if (lk_fork_) cudaEventDestroy(lk_fork_);
    if (lk_join_) cudaEventDestroy(lk_join_);
    em_graph_.clear();
    const cudaStream_t s = own_stream_;
    dfree(d_, s); dfree(x_, s); dfree(r_, s); dfree(D_, s); dfree(theta_, s); dfree(hist_, s);
    dfree(hcnt_, s); dfree(u_, s); dfree(vpad_, s); dfree(mean_, s);
    dfree(m2_, s); dfree(hfix_, s); dfree(mpart_, s); dfree(hdone_, s);
    dfree(stats_, s); dfree(st_, s); dfree(d0_, s); dfree(theta0_, s);
    dfree(ssd_, s); dfree(ssd0_, s); dfree(colmax_, s); dfree(colmax0_, s);
    dfree(fx_, s); dfree(fn_, s); dfree(fst_, s); dfree(fst0_, s); dfree(fstats_, s);
    release_chains();
    delete topo_;
    mstep_.release(s);
    cudaStreamSynchronize(s);  // the frees complete, so the next object can reuse the memory
    cudaStreamDestroy(s);
}

void Registration::set_mi_likelihood(double alpha, const float *theta, int K, int L,
                                     const int *binned_nodes, const int *binned_voxels) {
    BINDER_CHECK((long)K * L <= 24576, "K * L must be at most 24576 (shared-memory histogram)");
    load_bins(alpha, theta, K, L, 1, binned_nodes, binned_voxels);
    lk_ = 0;
    egrid_e_ = estep_grid(false, K, L, V_, N_, false, hist_prec_ == 1);
    egrid_s_ = estep_grid(true, K, L, V_, N_);
    have_mi_ = true;
}

void Registration::set_histogram_precision(int h) {
    BINDER_CHECK(h == 0 || h == 1,
                 "histogram precision must be 0 (FP32 bin columns) or 1 (FP16 bin columns)");
    hist_prec_ = h;
    if (lk_ == 0 && K_ > 0) egrid_e_ = estep_grid(false, K_, L_, V_, N_, false, h == 1);
    em_graph_.clear();
}

// The MI filter likelihood (BINDER/src/cpu/Registration.cpp:466-470, MILikelihoodFilter.cpp):
// M channels of bins, channel m of voxel i at binned_voxels[i + m] and of node j at
// binned_nodes[j + m] (so the arrays hold at least V + M - 1 and Vn + M - 1 bins); theta
// [M][K][L].  Its theta update and cost are the MI ones over M * K rows.
void Registration::set_mi_filter_likelihood(double alpha, const float *theta, int K, int L,
                                            int M, const int *binned_nodes,
                                            const int *binned_voxels) {
    BINDER_CHECK(M >= 1 && M <= kMaxChannels, "the number of channels M must be in [1, 8]");
    BINDER_CHECK((long)M * K * L <= kFilterMaxCells,
                 "M * K * L must be at most 24576 (shared-memory theta and histograms)");
    load_bins(alpha, theta, K, L, M, binned_nodes, binned_voxels);
    lk_ = 2;
    egrid_e_ = estep_filter_grid(K, L, M, V_, N_);
    // the sampler's draw keeps a running-sum table per thread next to theta and the counts
    egrid_s_ = filter_sampling_fits(K, L, M) ? estep_filter_grid(K, L, M, V_, N_, true) : 0;
    have_mi_ = true;
}

void Registration::load_bins(double alpha, const float *theta, int K, int L, int M,
                             const int *binned_nodes, const int *binned_voxels) {
    have_mi_ = false;
    BINDER_CHECK(K >= 1 && K <= 256 && L >= 1 && L <= 256,
                 "numbers of bins K and L must be in [1, 256]");
    BINDER_CUDA(cudaStreamSynchronize(stream_));  // buffers below may be in use
    em_graph_.clear();
    release_chains();  // their theta and count buffers have the old K x L
    const cudaStream_t s = own_stream_;
    // zero-padded byte volume of the node bins, in the E-step's view (a 2D node grid nxn x nyn
    // is the volume nxn x 1 x nyn: its y axis is the packed axis and has no padded y rows); one
    // per channel.  The voxel bins of channel m are the byte array shifted by m.
    const View w = estep_view();
    P_ = 8;
    PZ_ = 8;
    const int Py = N_ == 3 ? P_ : 0;
    pyn_ = w.nyn + 2 * Py;
    zp_ = ((w.nzn + 2 * PZ_ + 3) / 4) * 4 + 4;
    const size_t padded = (size_t)(w.nxn + 2 * P_) * pyn_ * zp_;
    const long nv = V_ + M - 1, nn = Vn_ + M - 1;  // bins read: [index + m], m < M
    const long cells = (long)M * K * L;
    dfree(u_, s); dfree(vpad_, s); dfree(theta_, s); dfree(hist_, s);
    dfree(hcnt_, s); dfree(hfix_, s); dfree(mpart_, s); dfree(hdone_, s);
    dfree(theta0_, s);
    u_ = dalloc<uint8_t>((size_t)nv, s);
    theta0_ = dalloc<float>((size_t)cells, s);
    vpad_ = dalloc<uint8_t>(padded * M, s);
    theta_ = dalloc<float>((size_t)cells, s);
    hist_ = dalloc<float>((size_t)cells, s);
    hcnt_ = dalloc<unsigned>((size_t)cells, s);
    // int32 bins to the device as they are, narrowed to bytes (and range-checked) there
    int *bins = dalloc<int>((size_t)(nv + nn), s);
    uint8_t *nodes8 = M > 1 ? dalloc<uint8_t>((size_t)nn, s) : nullptr;
    unsigned long long *bad = dalloc<unsigned long long>(3, s);
    BINDER_CUDA(cudaMemsetAsync(bad, 0xff, 3 * sizeof(unsigned long long), s));
    BINDER_CUDA(cudaMemcpyAsync(bins, binned_voxels, sizeof(int) * nv, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaMemcpyAsync(bins + nv, binned_nodes, sizeof(int) * nn, cudaMemcpyDefault, s));
    launch_bins_to_u8(bins, nv, L, u_, bad, s);
    // every node bin is checked once here; the padded volumes below check their windows again
    if (nodes8) launch_bins_to_u8(bins + nv, nn, K, nodes8, bad + 1, s);
    BINDER_CUDA(cudaMemsetAsync(vpad_, 0, padded * M, s));
    for (int m = 0; m < M; ++m)
        launch_bins_to_padded(bins + nv + m, w.nxn, w.nyn, w.nzn, K, vpad_ + padded * m, P_, Py,
                              PZ_, pyn_, zp_, M > 1 ? bad + 2 : bad + 1, s);
    // the buffers of the order-independent histogram merge of the single-pass EM kernel (one
    // channel, K <= 64)
    if (M == 1 && K <= 64) {
        hfix_ = dalloc<unsigned long long>((size_t)K * L, s);
        mpart_ = dalloc<double>(kMaxEmCtas, s);
        hdone_ = dalloc<unsigned>(1, s);
        BINDER_CUDA(cudaMemsetAsync(hfix_, 0, sizeof(unsigned long long) * K * L, s));
        BINDER_CUDA(cudaMemsetAsync(hdone_, 0, sizeof(unsigned), s));
    }
    BINDER_CUDA(cudaMemcpyAsync(theta_, theta, sizeof(float) * cells, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaMemcpyAsync(theta0_, theta_, sizeof(float) * cells, cudaMemcpyDeviceToDevice, s));
    BINDER_CUDA(cudaMemsetAsync(hist_, 0, sizeof(float) * cells, s));
    BINDER_CUDA(cudaMemsetAsync(hcnt_, 0, sizeof(unsigned) * cells, s));
    unsigned long long hbad[2];
    BINDER_CUDA(cudaMemcpyAsync(hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    dfree(bad, s);
    dfree(bins, s);
    if (nodes8) dfree(nodes8, s);
    if (hbad[0] != ~0ull || hbad[1] != ~0ull) {
        // the offending value, read through a copy (the arrays may be device memory)
        auto value_at = [](const int *a, unsigned long long i) {
            int v = 0;
            BINDER_CUDA(cudaMemcpy(&v, a + i, sizeof(int), cudaMemcpyDefault));
            return v;
        };
        if (hbad[0] != ~0ull)
            throw Error(kInvalidArgument, "binned_voxels value " +
                                              std::to_string(value_at(binned_voxels, hbad[0])) +
                                              " outside [0, L) at voxel " + std::to_string(hbad[0]));
        throw Error(kInvalidArgument, "binned_nodes value " +
                                          std::to_string(value_at(binned_nodes, hbad[1])) +
                                          " outside [0, K) at node " + std::to_string(hbad[1]));
    }
    K_ = K;
    L_ = L;
    M_ = M;
    vch_ = (long)padded;
    alpha_ = alpha;
}

// The SSD likelihood is a K x L table over (node bin, voxel bin) -- outside nodes count as bin
// 0, whose value is 0 -- so the bins, histogram and E-step of the MI path carry it; the table
// lives in log2 (per voxel bin relative to its best node bin) and the E-step runs in log space,
// and its parameters follow from moments of the joint histogram.
void Registration::set_ssd_likelihood(int bins, double sigma2, int shift_scale, double scale,
                                      double shift, const int *binned_nodes,
                                      const int *binned_voxels, double alpha0, double beta0) {
    BINDER_CHECK(bins >= 1 && bins <= kLogMaxBins, "SSD bins must be in [1, 64]");
    BINDER_CHECK(sigma2 > 0.0, "sigma_sq must be positive");
    BINDER_CHECK(alpha0 > 0.0 && beta0 > 0.0, "alpha_0 and beta_0 must be positive");
    const std::vector<float> flat((size_t)bins * bins, 1.0f / bins);
    set_mi_likelihood(2.0, flat.data(), bins, bins, binned_nodes, binned_voxels);
    const cudaStream_t s = own_stream_;
    dfree(ssd_, s); dfree(ssd0_, s); dfree(colmax_, s); dfree(colmax0_, s);
    ssd_ = dalloc<SsdState>(1, s);
    ssd0_ = dalloc<SsdState>(1, s);
    colmax_ = dalloc<float>((size_t)bins, s);
    colmax0_ = dalloc<float>((size_t)bins, s);
    SsdState h{};
    h.sigma2 = sigma2;
    // kept as given with shiftScale 0 too: the likelihood then ignores them, and
    // get_likelihood_parameters reports them (SSDLikelihood.cpp:328-334)
    h.shift = shift;
    h.scale = scale;
    h.alpha0 = alpha0;
    h.beta0 = beta0;
    h.shift_scale = shift_scale ? 1 : 0;
    BINDER_CUDA(cudaMemcpyAsync(ssd_, &h, sizeof h, cudaMemcpyHostToDevice, s));
    BINDER_CUDA(cudaMemcpyAsync(ssd0_, &h, sizeof h, cudaMemcpyHostToDevice, s));
    launch_ssd_update(theta_, colmax_, nullptr, bins, bins, 0, ssd_, nullptr, s);
    BINDER_CUDA(cudaMemcpyAsync(theta0_, theta_, sizeof(float) * bins * bins,
                                cudaMemcpyDeviceToDevice, s));
    BINDER_CUDA(cudaMemcpyAsync(colmax0_, colmax_, sizeof(float) * bins, cudaMemcpyDeviceToDevice,
                                s));
    BINDER_CUDA(cudaStreamSynchronize(s));  // `h` goes out of scope
    lk_ = 1;
    egrid_e_ = estep_grid(false, bins, bins, V_, N_, true);
    egrid_s_ = estep_grid(true, bins, bins, V_, N_, true);
}

// The SSD filter likelihood (SSDLikelihoodFilter.cpp): continuous features, EM in log space.
// The features go to the device as FP64 SoA; the parameters stay FP64 in an SsdfState.
void Registration::set_ssd_filter_likelihood(const double *coeff, const double *sigma,
                                             const double *features_nodes,
                                             const double *features_voxels,
                                             int reg_across_features, double alpha0,
                                             double beta0, int M, int F) {
    BINDER_CHECK(M >= 1 && M <= kSsdfMax && F >= 1 && F <= kSsdfMax,
                 "the SSD filter likelihood needs 1 <= M, F <= 8");
    BINDER_CHECK(alpha0 > 0.0 && beta0 > 0.0, "alpha_0 and beta_0 must be positive");
    for (int m = 0; m < M; ++m)
        BINDER_CHECK(sigma[m] > 0.0 && std::isfinite(sigma[m]), "sigma must be positive");
    const int Fn = reg_across_features ? M : F;
    have_mi_ = false;
    BINDER_CUDA(cudaStreamSynchronize(stream_));  // buffers below may be in use
    em_graph_.clear();
    const cudaStream_t s = own_stream_;
    dfree(fx_, s); dfree(fn_, s); dfree(fst_, s); dfree(fst0_, s); dfree(fstats_, s);
    fx_ = dalloc<double>((size_t)V_ * M, s);
    fn_ = dalloc<double>((size_t)Vn_ * Fn, s);
    fst_ = dalloc<SsdfState>(1, s);
    fst0_ = dalloc<SsdfState>(1, s);
    fstats_ = dalloc<double>(kSsdfStats, s);
    const long nmax = (long)V_ * M > (long)Vn_ * Fn ? (long)V_ * M : (long)Vn_ * Fn;
    double *stage = dalloc<double>((size_t)nmax, s);
    BINDER_CUDA(cudaMemcpyAsync(stage, features_voxels, sizeof(double) * V_ * M,
                                cudaMemcpyDefault, s));
    launch_features_to_soa(stage, V_, M, fx_, s);
    BINDER_CUDA(cudaMemcpyAsync(stage, features_nodes, sizeof(double) * Vn_ * Fn,
                                cudaMemcpyDefault, s));
    launch_features_to_soa(stage, Vn_, Fn, fn_, s);
    dfree(stage, s);
    SsdfState h{};
    h.M = M;
    h.F = F;
    h.Fn = Fn;
    h.rfa = reg_across_features ? 1 : 0;
    h.alpha0 = alpha0;
    h.beta0 = beta0;
    for (int q = 0; q < M * F; ++q) h.coeff[q] = coeff[q];
    for (int m = 0; m < M; ++m) h.sigma[m] = sigma[m];
    ssdf_refresh_host(h);
    BINDER_CUDA(cudaMemcpyAsync(fst_, &h, sizeof h, cudaMemcpyHostToDevice, s));
    BINDER_CUDA(cudaMemcpyAsync(fst0_, &h, sizeof h, cudaMemcpyHostToDevice, s));
    BINDER_CUDA(cudaMemsetAsync(fstats_, 0, sizeof(double) * kSsdfStats, s));
    BINDER_CUDA(cudaStreamSynchronize(s));  // `h` goes out of scope
    fM_ = M;
    fF_ = F;
    fFn_ = Fn;
    lk_ = 3;
    egrid_e_ = estep_ssdf_grid(M, Fn, V_, N_);
    egrid_s_ = estep_ssdf_grid(M, Fn, V_, N_, true);
    have_mi_ = true;
}

void Registration::get_ssd_filter_parameters(double *coeff, double *sigma) const {
    if (lk_ != 3) throw Error(kNotReady, "setSSDLikelihoodFilter has not been called");
    SsdfState h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, fst_, sizeof h, cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    if (coeff)
        for (int q = 0; q < h.M * h.F; ++q) coeff[q] = h.coeff[q];
    if (sigma)
        for (int m = 0; m < h.M; ++m) sigma[m] = h.sigma[m];
}

void Registration::get_ssd_parameters(double out[3]) const {
    if (lk_ != 1) throw Error(kNotReady, "setSSDLikelihood has not been called");
    SsdState h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, ssd_, sizeof h, cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    out[0] = h.sigma2;
    out[1] = h.shift;
    out[2] = h.scale;
}

void Registration::set_nonlinear_transformation(const double gamma[3], const double rho[3],
                                                const double eta[3], const float *D) {
    for (int n = 0; n < 3; ++n) {
        gamma0_[n] = gamma_set_[n] = gamma[n];
        rho_[n] = rho[n];
        eta_[n] = eta[n];
    }
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    em_graph_.clear();
    dfree(D_, own_stream_);
    D_ = dalloc<float>((size_t)V_, own_stream_);
    BINDER_CUDA(cudaMemcpyAsync(D_, D, sizeof(float) * V_, cudaMemcpyDefault, own_stream_));
    BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    sigma2_ = spline_sigma2(order_);
    have_tr_ = true;
}

void Registration::require_ready() const {
    if (!have_mi_) throw Error(kNotReady, "setMILikelihood has not been called");
    if (!have_tr_) throw Error(kNotReady, "setNonLinearTransformation has not been called");
}

void Registration::reset_state(bool for_sampler) {
    DevState h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, st_, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    h.mll = h.lp_lik = h.lp_tr = h.raw_reg = 0.0;
    h.mlp_old = 1e100;
    for (int n = 0; n < 3; ++n) h.gamma[n] = gamma0_[n];
    const double rp = rho_[0] * rho_[1] * rho_[2];
    h.nu = gamma0_[0] / (rp * eta_[0] * eta_[0] * (double)V_);  // NonLinearTransformation.cpp:43
    h.degenerate = 0;
    h.done = 0;
    h.iter = 0;
    h.flags = 0;
    h.sweep = 0;
    (void)for_sampler;
    BINDER_CUDA(cudaMemcpyAsync(st_, &h, sizeof(DevState), cudaMemcpyHostToDevice, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));  // `h` goes out of scope
}

// grid dimensions as the E-step sees them: a 2D image nx x ny (nz = 1) is the volume nx x 1 x ny
Registration::View Registration::estep_view() const {
    if (N_ == 3) return View{nx_, ny_, nz_, nxn_, nyn_, nzn_};
    return View{nx_, 1, ny_, nxn_, 1, nyn_};
}

GridDims Registration::grid_dims() const { return GridDims{nx_, ny_, nz_, N_}; }

EStepArgs Registration::estep_args(const int *skip) const {
    const View w = estep_view();
    EStepArgs e{};
    e.d = d_; e.r = r_; e.x = x_; e.u = u_; e.vpad = vpad_; e.theta = theta_; e.hist = hist_;
    e.hfix = hfix_; e.mpart = mpart_; e.hdone = hdone_;
    e.hcnt = hcnt_; e.st = st_; e.skip = skip; e.V = V_;
    e.nx = w.nx; e.ny = w.ny; e.nz = w.nz; e.nxn = w.nxn; e.nyn = w.nyn; e.nzn = w.nzn;
    e.P = P_; e.PZ = PZ_; e.pyn = pyn_; e.zp = zp_; e.K = K_; e.L = L_; e.dim = N_;
    e.seed = seed_; e.chain = chain_; e.order = order_;
    e.logt = lk_ == 1; e.colmax = colmax_;
    e.halfcol = lk_ == 0 ? hist_prec_ : 0;
    e.M = lk_ == 3 ? fM_ : M_; e.filter = lk_ == 2; e.uch = 1; e.vch = vch_;
    e.ssdf = lk_ == 3; e.Fn = fFn_; e.fx = fx_; e.fn = fn_; e.fstate = fst_; e.fstats = fstats_;
    return e;
}

void Registration::enqueue_em_iteration(int max_iter, double th, int update, cudaStream_t s) {
    const int grid = estep_grid_override_ > 0 ? estep_grid_override_ : egrid_e_;
    launch_estep(estep_args(&st_->done), false, grid, s);
    // the likelihood update (one CTA) reads the E-step's histogram or statistics and the M-step
    // the dream locations: the two run side by side and join before the bookkeeping
    BINDER_CUDA(cudaEventRecord(lk_fork_, s));
    BINDER_CUDA(cudaStreamWaitEvent(lk_stream_, lk_fork_, 0));
    if (lk_ == 1)
        launch_ssd_update(theta_, colmax_, hist_, K_, L_, update, ssd_, st_, lk_stream_);
    else if (lk_ == 3)
        launch_ssdf_update(fst_, fstats_, update, st_, lk_stream_);
    else
        launch_theta_update(theta_, hist_, M_ * K_, L_, alpha_, update, st_, lk_stream_);
    BINDER_CUDA(cudaEventRecord(lk_join_, lk_stream_));
    const double eta2[3] = {eta_[0] * eta_[0], eta_[1] * eta_[1], eta_[2] * eta_[2]};
    mstep_.enqueue(r_, d_, x_, D_, st_, sigma2_, 0, 0, 1, seed_, chain_,
                   rho_[0] * rho_[1] * rho_[2], eta2, &st_->done, s);
    BINDER_CUDA(cudaStreamWaitEvent(s, lk_join_, 0));
    launch_em_finish(st_, stats_, max_iter, th, nzv_, s);
}

void Registration::em_prepare(int max_iterations) {
    require_ready();
    BINDER_CHECK(max_iterations >= 1, "max_iterations must be >= 1");
    if (stats_cap_ < max_iterations) {
        BINDER_CUDA(cudaStreamSynchronize(stream_));
        dfree(stats_, own_stream_);
        stats_ = dalloc<double>((size_t)max_iterations * 4, own_stream_);
        stats_cap_ = max_iterations;
        BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    }
    BINDER_CUDA(cudaMemsetAsync(stats_, 0, sizeof(double) * 4 * max_iterations, stream_));
    reset_state(false);
    em_graph_.clear();
}

void Registration::enqueue_em(int n, int max_iterations, double th, int update, cudaStream_t s) {
    for (int i = 0; i < n; ++i) enqueue_em_iteration(max_iterations, th, update, s);
}

int Registration::em_finish(double ms) {
    DevState h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, st_, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    iters_done_ = h.iter;
    last_ms_ = ms;
    return h.iter;
}

bool Registration::em_done() const {
    int done = 0;
    BINDER_CUDA(cudaMemcpyAsync(&done, &st_->done, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    return done != 0;
}

void Registration::set_estep_grid(int g) {
    BINDER_CHECK(g >= 0, "the E-step grid must be >= 0 (0: the default)");
    estep_grid_override_ = g;
    em_graph_.clear();
}

int Registration::em(int max_iterations, double convergence_th, int update, int debug) {
    require_ready();
    if (max_iterations <= 0) return 0;
    if (stats_cap_ < max_iterations) {
        BINDER_CUDA(cudaStreamSynchronize(stream_));
        dfree(stats_, own_stream_);
        stats_ = dalloc<double>((size_t)max_iterations * 4, own_stream_);
        stats_cap_ = max_iterations;
        BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    }
    BINDER_CUDA(cudaMemsetAsync(stats_, 0, sizeof(double) * 4 * max_iterations, stream_));
    reset_state(false);

    cudaEvent_t t0, t1;
    BINDER_CUDA(cudaEventCreate(&t0));
    BINDER_CUDA(cudaEventCreate(&t1));
    // iterations between two reads of the device state; the graph holds ONE iteration, replayed
    // chunk times (capturing and instantiating costs host time per node, and a new object's
    // first EM call pays it), and is kept for the next call with the same parameters and buffers
    const int chunk = max_iterations < 8 ? max_iterations : 8;
    EmGraphCache &gc = em_graph_;
    if (!gc.e || gc.max_iter != max_iterations || gc.update != update ||
        gc.th != convergence_th || gc.stream != stream_ || gc.stats != stats_) {
        gc.clear();
        Graph graph;
        gc.kernels = capture_graph(stream_, graph, [&] {
            enqueue_em_iteration(max_iterations, convergence_th, update, stream_);
        });
        gc.g = graph.g;
        gc.e = graph.e;
        graph.g = nullptr;
        graph.e = nullptr;
        gc.chunk = chunk;
        gc.max_iter = max_iterations;
        gc.update = update;
        gc.th = convergence_th;
        gc.stream = stream_;
        gc.stats = stats_;
    }
    const long long kernels = gc.kernels;

    BINDER_CUDA(cudaEventRecord(t0, stream_));
    DevState h{};
    int launched = 0;
    while (true) {
        const int n = max_iterations - launched < chunk ? max_iterations - launched : chunk;
        for (int c = 0; c < n; ++c) {
            BINDER_CUDA(cudaGraphLaunch(gc.e, stream_));
            count_launch(kernels);
        }
        launched += n;
        BINDER_CUDA(cudaMemcpyAsync(&h, st_, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
        BINDER_CUDA(cudaStreamSynchronize(stream_));
        if (h.done || launched >= max_iterations) break;
    }
    BINDER_CUDA(cudaEventRecord(t1, stream_));
    BINDER_CUDA(cudaEventSynchronize(t1));
    float ms = 0.0f;
    BINDER_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    last_ms_ = ms;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    iters_done_ = h.iter;
    if (debug || verbose()) {
        std::vector<double> s((size_t)h.iter * 4);
        if (h.iter) {
            BINDER_CUDA(cudaMemcpyAsync(s.data(), stats_, sizeof(double) * 4 * h.iter,
                                        cudaMemcpyDeviceToHost, stream_));
            BINDER_CUDA(cudaStreamSynchronize(stream_));
        }
        for (int it = 0; it < h.iter; ++it)
            std::printf("Iteration %d: mll %.8f  prior(theta) %.8f  prior(T) %.8f  mlp %.8f  "
                        "mlp/voxel %.8f\n",
                        it + 1, s[it * 4 + 0], s[it * 4 + 1], s[it * 4 + 2], s[it * 4 + 3],
                        s[it * 4 + 3] / nzv_);
        std::printf("EM: %d iterations in %.3f ms\n", h.iter, ms);
    }
    return h.iter;
}

void Registration::sampler(uint64_t seed, int N_b, int N_s, int sample_gamma,
                           int sample_gamma_every, int sample_posteriors,
                           int sample_likelihood_parameters, int sample_transformation_parameters,
                           double *mean_out, double *cov_out) {
    if (sample_posteriors || sample_likelihood_parameters) {
        if (!have_mi_) throw Error(kNotReady, "setMILikelihood has not been called");
    }
    if (lk_ == 2 && sample_posteriors && egrid_s_ == 0)
        throw Error(kUnsupported,
                    "the sampler with the MI filter likelihood needs M * K * L small enough for "
                    "its theta, counts and draw table in shared memory (about 22000 cells)");
    if (!have_tr_) throw Error(kNotReady, "setNonLinearTransformation has not been called");
    BINDER_CHECK(N_b >= 0 && N_s >= 0, "N_b and N_s must be non-negative");
    BINDER_CHECK(sample_gamma_every >= 1 || !sample_gamma, "sample_gamma_every must be >= 1");
    seed_ = seed;
    em_graph_.clear();
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    const int NM2 = N_ * (N_ + 1) / 2;  // upper triangle of the covariance
    if (!mean_) {
        mean_ = dalloc<double>((size_t)V_ * N_, own_stream_);
        m2_ = dalloc<double>((size_t)V_ * NM2, own_stream_);
        BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    }
    BINDER_CUDA(cudaMemsetAsync(mean_, 0, sizeof(double) * V_ * N_, stream_));
    BINDER_CUDA(cudaMemsetAsync(m2_, 0, sizeof(double) * V_ * NM2, stream_));
    reset_state(true);
    const int total = N_b + N_s;
    if (total > 0 && sample_transformation_parameters) {
        mstep_.prepare_sampling(own_stream_);
        BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    }
    if (total > 0) {
        const double eta2[3] = {eta_[0] * eta_[0], eta_[1] * eta_[1], eta_[2] * eta_[2]};
        const double rho_p = rho_[0] * rho_[1] * rho_[2];
        const int every = sample_gamma_every < 1 ? 1 : sample_gamma_every;
        // one sweep per graph, replayed `total` times (capture costs host time per node)
        const int chunk = 1;
        Graph graph;
        const long long kernels = capture_graph(stream_, graph, [&] {
            for (int c = 0; c < chunk; ++c) {
                if (sample_posteriors) {
                    launch_estep(estep_args(&st_->done), true, egrid_s_, stream_);
                }
                if (sample_likelihood_parameters) {
                    if (lk_ == 1)  // SSDLikelihood::sample_parameters from the sweep's counts
                        launch_ssd_sample(theta_, colmax_, hcnt_, K_, L_, ssd_, st_, seed_,
                                          chain_, stream_);
                    else if (lk_ == 3)  // SSDLikelihoodFilter::sample_parameters
                        launch_ssdf_sample(fst_, fstats_, st_, seed_, chain_, stream_);
                    else  // MI: K rows; MI filter: M * K rows (MILikelihoodFilter.cpp:152-175)
                        launch_dirichlet_sample(theta_, hcnt_, M_ * K_, L_, alpha_, seed_, chain_,
                                                st_, stream_);
                }
                if (sample_transformation_parameters) {
                    mstep_.enqueue(r_, d_, x_, D_, st_, sigma2_, 1, sample_gamma, every, seed_,
                                   chain_, rho_p, eta2, &st_->done, stream_);
                    if (sample_gamma)
                        launch_nu_sample(st_, sample_gamma, every, N_, V_, rho_p, eta2, seed_,
                                         chain_, stream_);
                }
                launch_sweep_end(d_, mean_, m2_, V_, N_, N_b, total, st_, stream_);
            }
        });
        cudaEvent_t t0, t1;
        BINDER_CUDA(cudaEventCreate(&t0));
        BINDER_CUDA(cudaEventCreate(&t1));
        BINDER_CUDA(cudaEventRecord(t0, stream_));
        for (int done = 0; done < total; done += chunk) replay(graph, kernels, stream_);
        BINDER_CUDA(cudaEventRecord(t1, stream_));
        BINDER_CUDA(cudaEventSynchronize(t1));
        float ms = 0.0f;
        BINDER_CUDA(cudaEventElapsedTime(&ms, t0, t1));
        last_ms_ = ms;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (verbose()) std::printf("sampler: %d sweeps in %.3f ms\n", total, ms);
    }
    DevState h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, st_, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
    // moments rearranged to AoS on the device, then one transfer each
    double *mean_aos = dalloc<double>((size_t)V_ * N_, stream_);
    double *cov_aos = dalloc<double>((size_t)V_ * N_ * N_, stream_);
    launch_moments_to_aos(mean_, m2_, V_, N_, 1.0 / (double)(N_s - 1), mean_aos, cov_aos, stream_);
    BINDER_CUDA(cudaMemcpyAsync(mean_out, mean_aos, sizeof(double) * V_ * N_,
                                cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaMemcpyAsync(cov_out, cov_aos, sizeof(double) * V_ * N_ * N_,
                                cudaMemcpyDeviceToHost, stream_));
    dfree(mean_aos, stream_);
    dfree(cov_aos, stream_);
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    for (int n = 0; n < 3; ++n) gamma0_[n] = h.gamma[n];  // the prior keeps sampled gammas
}

void Registration::release_chains() {
    if (!cb_) return;
    const cudaStream_t s = own_stream_;
    dfree(cb_->d, s); dfree(cb_->r, s); dfree(cb_->theta, s); dfree(cb_->hcnt, s);
    dfree(cb_->st, s); dfree(cb_->mean, s); dfree(cb_->m2, s);
    cb_->mstep.release(s);
    delete cb_;
    cb_ = nullptr;
}

// The sweep of sampler() (BINDER/src/cpu/Registration.cpp:545-625) for a batch of independent
// chains: each kernel of a sweep runs once for all chains (chain = blockIdx.y of the E-step,
// Dirichlet and Welford kernels; chains x components of every DCT pass), so a sweep of C chains is
// one graph of the same length as a sweep of one chain.
void Registration::sampler_chains(uint64_t seed, int chains, int N_b, int N_s, int sample_gamma,
                                  int sample_gamma_every, int sample_posteriors,
                                  int sample_likelihood_parameters,
                                  int sample_transformation_parameters, double *mean_out,
                                  double *cov_out, double *pooled_mean, double *pooled_cov) {
    if (lk_ != 0 && (sample_posteriors || sample_likelihood_parameters))
        throw Error(kUnsupported, "a batch of chains samples with the MI likelihood only");
    if (sample_posteriors || sample_likelihood_parameters) {
        if (!have_mi_) throw Error(kNotReady, "setMILikelihood has not been called");
    }
    if (!have_tr_) throw Error(kNotReady, "setNonLinearTransformation has not been called");
    BINDER_CHECK(chains >= 1 && chains <= 1024, "chains must be in [1, 1024]");
    BINDER_CHECK(N_b >= 0 && N_s >= 0, "N_b and N_s must be non-negative");
    BINDER_CHECK(sample_gamma_every >= 1 || !sample_gamma, "sample_gamma_every must be >= 1");
    BINDER_CHECK(!(pooled_mean || pooled_cov) || N_s >= 1,
                 "pooled moments need at least one sample per chain");
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    const cudaStream_t so = own_stream_;
    const int C = chains, N = N_, NM2 = N_ * (N_ + 1) / 2;
    const size_t VN = (size_t)V_ * N, KL = (size_t)(K_ > 0 ? K_ : 1) * (L_ > 0 ? L_ : 1);
    if (!cb_ || cb_->chains != C) {
        release_chains();
        cb_ = new ChainBatch();
        cb_->chains = C;
        cb_->d = dalloc<float>(VN * C, so);
        cb_->r = dalloc<float>(VN * C, so);
        cb_->theta = dalloc<float>(KL * C, so);
        cb_->hcnt = dalloc<unsigned>(KL * C, so);
        cb_->st = dalloc<DevState>((size_t)C, so);
        cb_->mean = dalloc<double>(VN * C, so);
        cb_->m2 = dalloc<double>((size_t)V_ * NM2 * C, so);
        cb_->mstep.init(nx_, ny_, nz_, so, C);
        BINDER_CUDA(cudaStreamSynchronize(so));
    }
    cb_->mstep.precision = mstep_.precision;
    if (sample_transformation_parameters) {
        cb_->mstep.prepare_sampling(own_stream_);
        BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    }
    ChainBatch &b = *cb_;
    // every chain starts from the object's positions, dream locations, theta and gammas
    for (int c = 0; c < C; ++c) {
        BINDER_CUDA(cudaMemcpyAsync(b.d + VN * c, d_, sizeof(float) * VN,
                                    cudaMemcpyDeviceToDevice, stream_));
        BINDER_CUDA(cudaMemcpyAsync(b.r + VN * c, r_, sizeof(float) * VN,
                                    cudaMemcpyDeviceToDevice, stream_));
        if (have_mi_)
            BINDER_CUDA(cudaMemcpyAsync(b.theta + KL * c, theta_, sizeof(float) * KL,
                                        cudaMemcpyDeviceToDevice, stream_));
    }
    BINDER_CUDA(cudaMemsetAsync(b.hcnt, 0, sizeof(unsigned) * KL * C, stream_));
    BINDER_CUDA(cudaMemsetAsync(b.mean, 0, sizeof(double) * VN * C, stream_));
    BINDER_CUDA(cudaMemsetAsync(b.m2, 0, sizeof(double) * V_ * NM2 * C, stream_));
    {
        DevState h{};
        for (int n = 0; n < 3; ++n) h.gamma[n] = gamma0_[n];
        h.mlp_old = 1e100;
        const double rp = rho_[0] * rho_[1] * rho_[2];
        h.nu = gamma0_[0] / (rp * eta_[0] * eta_[0] * (double)V_);  // NonLinearTransformation.cpp:43
        std::vector<DevState> hs((size_t)C, h);
        BINDER_CUDA(cudaMemcpyAsync(b.st, hs.data(), sizeof(DevState) * C,
                                    cudaMemcpyHostToDevice, stream_));
        BINDER_CUDA(cudaStreamSynchronize(stream_));  // `hs` goes out of scope
    }
    const int total = N_b + N_s;
    if (total > 0) {
        const double eta2[3] = {eta_[0] * eta_[0], eta_[1] * eta_[1], eta_[2] * eta_[2]};
        const double rho_p = rho_[0] * rho_[1] * rho_[2];
        const int every = sample_gamma_every < 1 ? 1 : sample_gamma_every;
        const int chunk = 1;  // one sweep of every chain per graph, replayed `total` times
        EStepArgs e = estep_args(&b.st->done);
        e.d = b.d; e.r = b.r; e.theta = b.theta; e.hcnt = b.hcnt; e.st = b.st; e.seed = seed;
        Graph graph;
        const long long kernels = capture_graph(stream_, graph, [&] {
            for (int c = 0; c < chunk; ++c) {
                if (sample_posteriors) launch_estep(e, true, egrid_s_, stream_, C);
                if (sample_likelihood_parameters)
                    launch_dirichlet_sample(b.theta, b.hcnt, K_, L_, alpha_, seed, chain_, b.st,
                                            stream_, C);
                if (sample_transformation_parameters) {
                    b.mstep.enqueue(b.r, b.d, x_, D_, b.st, sigma2_, 1, sample_gamma, every, seed,
                                    chain_, rho_p, eta2, &b.st->done, stream_);
                    if (sample_gamma)
                        launch_nu_sample(b.st, sample_gamma, every, N_, V_, rho_p, eta2, seed,
                                         chain_, stream_, C);
                }
                launch_sweep_end(b.d, b.mean, b.m2, V_, N_, N_b, total, b.st, stream_, C);
            }
        });
        cudaEvent_t t0, t1;
        BINDER_CUDA(cudaEventCreate(&t0));
        BINDER_CUDA(cudaEventCreate(&t1));
        BINDER_CUDA(cudaEventRecord(t0, stream_));
        for (int done = 0; done < total; done += chunk) replay(graph, kernels, stream_);
        BINDER_CUDA(cudaEventRecord(t1, stream_));
        BINDER_CUDA(cudaEventSynchronize(t1));
        float ms = 0.0f;
        BINDER_CUDA(cudaEventElapsedTime(&ms, t0, t1));
        last_ms_ = ms;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (verbose())
            std::printf("sampler: %d chains x %d sweeps in %.3f ms\n", C, total, ms);
    }
    // moments: per chain rearranged to AoS on the device and read back in one copy each, and / or
    // pooled over the chains
    const double scale = 1.0 / (double)(N_s - 1);
    double *mstage = (mean_out || pooled_mean) ? dalloc<double>(VN * (mean_out ? C : 1), stream_)
                                               : nullptr;
    double *cstage = (cov_out || pooled_cov)
                         ? dalloc<double>(VN * N * (cov_out ? C : 1), stream_)
                         : nullptr;
    if (mean_out || cov_out) {
        for (int c = 0; c < C; ++c)
            launch_moments_to_aos(b.mean + VN * c, b.m2 + (size_t)V_ * NM2 * c, V_, N, scale,
                                  mean_out ? mstage + VN * c : nullptr,
                                  cov_out ? cstage + VN * N * c : nullptr, stream_);
        if (mean_out)
            BINDER_CUDA(cudaMemcpyAsync(mean_out, mstage, sizeof(double) * VN * C,
                                        cudaMemcpyDeviceToHost, stream_));
        if (cov_out)
            BINDER_CUDA(cudaMemcpyAsync(cov_out, cstage, sizeof(double) * VN * N * C,
                                        cudaMemcpyDeviceToHost, stream_));
    }
    if (pooled_mean || pooled_cov) {
        // after the per-chain copies above (same stream), the staging buffers are reused
        launch_pool_moments(b.mean, b.m2, V_, N, C, (double)N_s, pooled_mean ? mstage : nullptr,
                            pooled_cov ? cstage : nullptr, stream_);
        if (pooled_mean)
            BINDER_CUDA(cudaMemcpyAsync(pooled_mean, mstage, sizeof(double) * VN,
                                        cudaMemcpyDeviceToHost, stream_));
        if (pooled_cov)
            BINDER_CUDA(cudaMemcpyAsync(pooled_cov, cstage, sizeof(double) * VN * N,
                                        cudaMemcpyDeviceToHost, stream_));
    }
    dfree(mstage, stream_);
    dfree(cstage, stream_);
    BINDER_CUDA(cudaStreamSynchronize(stream_));
}

double Registration::profile_stage(int stage, int n) {
    require_ready();
    BINDER_CHECK(stage >= 0 && stage <= 2, "stage must be 0 (E-step), 1 (M-step) or 2 (theta)");
    BINDER_CHECK(n >= 1, "n must be >= 1");
    reset_state(false);
    const EStepArgs e = estep_args(nullptr);
    const double eta2[3] = {eta_[0] * eta_[0], eta_[1] * eta_[1], eta_[2] * eta_[2]};
    auto one = [&] {
        if (stage == 0) launch_estep(e, false, egrid_e_, stream_);
        else if (stage == 1)
            mstep_.enqueue(r_, d_, x_, D_, st_, sigma2_, 0, 0, 1, seed_, chain_,
                           rho_[0] * rho_[1] * rho_[2], eta2, nullptr, stream_);
        else if (lk_ == 1)
            launch_ssd_update(theta_, colmax_, hist_, K_, L_, 0, ssd_, st_, stream_);
        else if (lk_ == 3)
            launch_ssdf_update(fst_, fstats_, 0, st_, stream_);
        else launch_theta_update(theta_, hist_, M_ * K_, L_, alpha_, 1, st_, stream_);
    };
    one();  // warm-up
    cudaEvent_t t0, t1;
    BINDER_CUDA(cudaEventCreate(&t0));
    BINDER_CUDA(cudaEventCreate(&t1));
    BINDER_CUDA(cudaEventRecord(t0, stream_));
    for (int i = 0; i < n; ++i) one();
    BINDER_CUDA(cudaEventRecord(t1, stream_));
    BINDER_CUDA(cudaEventSynchronize(t1));
    float ms = 0.0f;
    BINDER_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    BINDER_CUDA(cudaMemsetAsync(hist_, 0, sizeof(float) * M_ * K_ * L_, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    return ms / n;
}

void Registration::set_precision(int p) {
    BINDER_CHECK(p >= 0 && p <= 4,
                 "precision must be 0 (FP32), 1 (3xTF32), 2 (TF32), 3 (BF16x3) or 4 (BF16)");
    mstep_.precision = p;
    em_graph_.clear();
}

void Registration::set_stream(cudaStream_t s) {
    stream_ = s ? s : own_stream_;
    em_graph_.clear();
}

void Registration::set_chain(uint32_t c) {
    chain_ = c;
    em_graph_.clear();
}

void PriorTransform::set_precision(int p) {
    BINDER_CHECK(p >= 0 && p <= 4,
                 "precision must be 0 (FP32), 1 (3xTF32), 2 (TF32), 3 (BF16x3) or 4 (BF16)");
    mstep_.precision = p;
}

void Registration::reset() {
    for (int n = 0; n < 3; ++n) gamma0_[n] = gamma_set_[n];  // the sampler keeps sampled gammas
    BINDER_CUDA(cudaMemcpyAsync(d_, d0_, sizeof(float) * V_ * N_, cudaMemcpyDeviceToDevice, stream_));
    if (lk_ == 3) {
        BINDER_CUDA(cudaMemcpyAsync(fst_, fst0_, sizeof(SsdfState), cudaMemcpyDeviceToDevice,
                                    stream_));
        BINDER_CUDA(cudaMemsetAsync(fstats_, 0, sizeof(double) * kSsdfStats, stream_));
    } else if (have_mi_) {
        BINDER_CUDA(cudaMemcpyAsync(theta_, theta0_, sizeof(float) * M_ * K_ * L_,
                                    cudaMemcpyDeviceToDevice, stream_));
        BINDER_CUDA(cudaMemsetAsync(hist_, 0, sizeof(float) * M_ * K_ * L_, stream_));
        BINDER_CUDA(cudaMemsetAsync(hcnt_, 0, sizeof(unsigned) * M_ * K_ * L_, stream_));
    }
    if (lk_ == 1) {
        BINDER_CUDA(cudaMemcpyAsync(ssd_, ssd0_, sizeof(SsdState), cudaMemcpyDeviceToDevice,
                                    stream_));
        BINDER_CUDA(cudaMemcpyAsync(colmax_, colmax0_, sizeof(float) * L_,
                                    cudaMemcpyDeviceToDevice, stream_));
    }
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    reset_state(false);
}

TopologyResult Registration::correct_topology(double e1, double e2, int max_outer, int max_inner,
                                              const double vs[3]) {
    BINDER_CHECK(e1 <= 1.0 && e2 >= 1.0 && e1 < e2,
                 "topology correction needs e1 <= 1 <= e2 (the identity must be admissible)");
    if (!topo_) topo_ = new TopologyWorkspace(nx_, ny_, nz_, own_stream_);
    topo_->load_float_grid(d_, vs, stream_);
    TopologyResult r = topo_->run(e1, e2, max_outer, max_inner, vs, stream_);
    topo_->store_float_grid(d_, vs, stream_);
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    return r;
}

// AoS host arrays <-> device state, rearranged on the device with the M-step's scratch t1 (idle
// between calls) as the staging buffer
void Registration::get_final_locations(float *out) const {
    launch_soa_to_aos(d_, mstep_.t1, V_, N_, stream_);
    BINDER_CUDA(cudaMemcpyAsync(out, mstep_.t1, sizeof(float) * V_ * N_, cudaMemcpyDeviceToHost,
                                stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
}

void Registration::set_final_locations(const float *in) {
    BINDER_CUDA(cudaMemcpyAsync(mstep_.t1, in, sizeof(float) * V_ * N_, cudaMemcpyHostToDevice,
                                stream_));
    launch_aos_to_soa(mstep_.t1, d_, V_, N_, stream_);
    BINDER_CUDA(cudaStreamSynchronize(stream_));
}

void Registration::get_dream_locations(float *out) const {
    launch_soa_to_aos_plus(r_, x_, grid_dims(), mstep_.t1, stream_);
    BINDER_CUDA(cudaMemcpyAsync(out, mstep_.t1, sizeof(float) * V_ * N_, cudaMemcpyDeviceToHost,
                                stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
}

void Registration::set_dream_locations(const float *in) {
    BINDER_CUDA(cudaMemcpyAsync(mstep_.t1, in, sizeof(float) * V_ * N_, cudaMemcpyHostToDevice,
                                stream_));
    launch_aos_minus_to_soa(mstep_.t1, x_, grid_dims(), r_, stream_);
    BINDER_CUDA(cudaStreamSynchronize(stream_));
}

void Registration::add_displacement(const float *field, int fx, int fy, int fz) {
    BINDER_CHECK((N_ == 2) == (fz == 1), "a 2D registration takes a 2D field (fz == 1)");
    add_resized_displacement(field, fx, fy, fz, N_, nx_, ny_, nz_, d_, stream_);
}

void Registration::get_likelihood_parameters(float *out) const {
    if (!have_mi_) throw Error(kNotReady, "setMILikelihood has not been called");
    if (lk_ == 3) {  // SSDLikelihoodFilter::get_parameters (:457-466): the coefficients
        std::vector<double> c((size_t)fM_ * fF_);
        get_ssd_filter_parameters(c.data(), nullptr);
        for (size_t q = 0; q < c.size(); ++q) out[q] = (float)c[q];
        return;
    }
    if (lk_ == 1) {  // SSDLikelihood::get_parameters (SSDLikelihood.cpp:328-334): scale, shift
        double p[3];
        get_ssd_parameters(p);
        out[0] = (float)p[2];
        out[1] = (float)p[1];
        return;
    }
    BINDER_CUDA(cudaMemcpyAsync(out, theta_, sizeof(float) * M_ * K_ * L_, cudaMemcpyDeviceToHost,
                                stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
}

void Registration::get_shape(int out[4]) const {
    out[0] = nx_; out[1] = ny_; out[2] = nz_; out[3] = N_;
}

int Registration::get_iteration_stats(double *out, int max_n) const {
    const int n = iters_done_ < max_n ? iters_done_ : max_n;
    if (n > 0 && stats_) {
        BINDER_CUDA(cudaMemcpyAsync(out, stats_, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost,
                                    stream_));
        BINDER_CUDA(cudaStreamSynchronize(stream_));
    }
    return n;
}

void Registration::get_state(double *gamma_out, double *nu_out, unsigned long long *degenerate,
                             unsigned *flags) const {
    DevState h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, st_, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    if (gamma_out)
        for (int n = 0; n < 3; ++n) gamma_out[n] = h.gamma[n];
    if (nu_out) *nu_out = h.nu;
    if (degenerate) *degenerate = h.degenerate;
    if (flags) *flags = h.flags;
}

// ------------------------------------------------------------------------------------------
RegistrationBatch::RegistrationBatch(const std::vector<Registration *> &regs) : regs_(regs) {
    BINDER_CHECK(!regs.empty(), "a batch needs at least one registration");
    for (auto *r : regs) BINDER_CHECK(r != nullptr, "a batch member is null");
    BINDER_CUDA(cudaStreamCreateWithFlags(&master_, cudaStreamNonBlocking));
    BINDER_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    branch_.resize(regs.size(), nullptr);
    join_.resize(regs.size(), nullptr);
    BINDER_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&done_host_), sizeof(int) * regs.size(),
                              cudaHostAllocDefault));
    for (size_t i = 0; i < regs.size(); ++i) {
        BINDER_CUDA(cudaStreamCreateWithFlags(&branch_[i], cudaStreamNonBlocking));
        BINDER_CUDA(cudaEventCreateWithFlags(&join_[i], cudaEventDisableTiming));
    }
}

RegistrationBatch::~RegistrationBatch() {
    if (master_) cudaStreamSynchronize(master_);
    for (size_t i = 0; i < branch_.size(); ++i) {
        if (branch_[i]) cudaStreamSynchronize(branch_[i]), cudaStreamDestroy(branch_[i]);
        if (join_[i]) cudaEventDestroy(join_[i]);
    }
    if (fork_) cudaEventDestroy(fork_);
    if (master_) cudaStreamDestroy(master_);
    if (done_host_) cudaFreeHost(done_host_);
}

void RegistrationBatch::em(int max_iterations, double th, int update, int *its_out) {
    if (max_iterations <= 0) {
        for (size_t i = 0; i < regs_.size(); ++i) its_out[i] = 0;
        return;
    }
    for (auto *r : regs_) r->em_prepare(max_iterations);
    // the graph holds ONE iteration of every pair (capturing and instantiating costs host time
    // per node), replayed up to 8 times between two reads of the pairs' done flags; a pair whose
    // rule has fired turns its remaining kernels into no-ops
    const int chunk = 8;
    std::vector<size_t> active(regs_.size());
    for (size_t i = 0; i < active.size(); ++i) active[i] = i;
    Graph graph;
    const long long kernels = capture_graph(master_, graph, [&] {
        BINDER_CUDA(cudaEventRecord(fork_, master_));
        for (size_t i = 0; i < regs_.size(); ++i) {
            BINDER_CUDA(cudaStreamWaitEvent(branch_[i], fork_, 0));
            regs_[i]->enqueue_em(1, max_iterations, th, update, branch_[i]);
            BINDER_CUDA(cudaEventRecord(join_[i], branch_[i]));
            BINDER_CUDA(cudaStreamWaitEvent(master_, join_[i], 0));
        }
    });
    cudaEvent_t t0, t1;
    BINDER_CUDA(cudaEventCreate(&t0));
    BINDER_CUDA(cudaEventCreate(&t1));
    BINDER_CUDA(cudaEventRecord(t0, master_));
    int launched = 0;
    while (true) {
        const int n = max_iterations - launched < chunk ? max_iterations - launched : chunk;
        for (int c = 0; c < n; ++c) replay(graph, kernels, master_);
        launched += n;
        if (launched >= max_iterations) break;
        // the done flags of the pairs still iterating, in one round trip
        for (size_t i : active)
            BINDER_CUDA(cudaMemcpyAsync(&done_host_[i], regs_[i]->done_flag(), sizeof(int),
                                        cudaMemcpyDeviceToHost, master_));
        BINDER_CUDA(cudaStreamSynchronize(master_));
        std::vector<size_t> left;
        for (size_t i : active)
            if (!done_host_[i]) left.push_back(i);
        if (left.empty()) break;
        active.swap(left);
    }
    BINDER_CUDA(cudaEventRecord(t1, master_));
    BINDER_CUDA(cudaEventSynchronize(t1));
    float ms = 0.0f;
    BINDER_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    last_ms_ = ms;
    for (size_t i = 0; i < regs_.size(); ++i) its_out[i] = regs_[i]->em_finish(ms);
}

// ------------------------------------------------------------------------------------------
PriorTransform::PriorTransform(const double gamma[3], const double rho[3], const double eta[3],
                               const float *D, int nx, int ny, int nz, double sigma_spline)
    : nx_(nx), ny_(ny), nz_(nz) {
    BINDER_CHECK(nx > 0 && ny > 0 && nz > 0, "grid dimensions must be positive");
    V_ = (long)nx * ny * nz;
    N_ = nz == 1 ? 2 : 3;
    for (int n = 0; n < 3; ++n) {
        gamma_[n] = gamma[n];
        rho_[n] = rho[n];
        eta_[n] = eta[n];
    }
    sigma2_ = sigma_spline * sigma_spline;
    BINDER_CUDA(cudaStreamCreate(&own_stream_));
    stream_ = own_stream_;
    const cudaStream_t s = own_stream_;
    D_ = dalloc<float>((size_t)V_, s);
    BINDER_CUDA(cudaMemcpyAsync(D_, D, sizeof(float) * V_, cudaMemcpyHostToDevice, s));
    r_ = dalloc<float>((size_t)V_ * N_, s);
    d_ = dalloc<float>((size_t)V_ * N_, s);
    zeros_ = dalloc<float>((size_t)V_ * N_, s);
    BINDER_CUDA(cudaMemsetAsync(zeros_, 0, sizeof(float) * V_ * N_, s));
    st_ = dalloc<DevState>(1, s);
    BINDER_CUDA(cudaMemsetAsync(st_, 0, sizeof(DevState), s));
    mstep_.init(nx, ny, nz, s);
    BINDER_CUDA(cudaStreamSynchronize(s));
}

PriorTransform::~PriorTransform() {
    if (stream_ != own_stream_) cudaStreamSynchronize(stream_);
    cudaStreamSynchronize(own_stream_);
    const cudaStream_t s = own_stream_;
    dfree(D_, s); dfree(r_, s); dfree(d_, s); dfree(zeros_, s); dfree(chunk_, s); dfree(st_, s);
    mstep_.release(s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
}

// BINDER/src/cpu/NonLinearTransformation.cpp:226-278: voxel positions are zero, so the result
// is the smoothed field itself
double PriorTransform::smooth(const float *field, float *out) {
    BINDER_CUDA(cudaMemcpyAsync(mstep_.t1, field, sizeof(float) * V_ * N_,
                                cudaMemcpyHostToDevice, stream_));
    launch_aos_to_soa(mstep_.t1, r_, V_, N_, stream_);
    DevState h{};
    for (int n = 0; n < 3; ++n) h.gamma[n] = gamma_[n];
    BINDER_CUDA(cudaMemcpyAsync(st_, &h, sizeof(DevState), cudaMemcpyHostToDevice, stream_));
    const double eta2[3] = {eta_[0] * eta_[0], eta_[1] * eta_[1], eta_[2] * eta_[2]};
    mstep_.enqueue(r_, d_, zeros_, D_, st_, sigma2_, 0, 0, 1, seed_, 0,
                   rho_[0] * rho_[1] * rho_[2], eta2, nullptr, stream_);
    launch_soa_to_aos(d_, mstep_.t1, V_, N_, stream_);
    BINDER_CUDA(cudaMemcpyAsync(out, mstep_.t1, sizeof(float) * V_ * N_, cudaMemcpyDeviceToHost,
                                stream_));
    BINDER_CUDA(cudaMemcpyAsync(&h, st_, sizeof(DevState), cudaMemcpyDeviceToHost, stream_));
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    return h.lp_tr;
}

// NonLinearTransformation.cpp:280-341: independent prior samples around the given field.  The
// Philox sweep counter continues across calls, so repeated calls give fresh samples.
void PriorTransform::sample(const float *field, int n, float *out) {
    BINDER_CHECK(n >= 0, "number_of_samples must be non-negative");
    if (n == 0) return;
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    mstep_.prepare_sampling(own_stream_);
    BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    BINDER_CUDA(cudaMemcpyAsync(mstep_.t1, field, sizeof(float) * V_ * N_,
                                cudaMemcpyHostToDevice, stream_));
    launch_aos_to_soa(mstep_.t1, r_, V_, N_, stream_);
    DevState h{};
    for (int c = 0; c < 3; ++c) h.gamma[c] = gamma_[c];
    h.sweep = sweep_;
    BINDER_CUDA(cudaMemcpyAsync(st_, &h, sizeof(DevState), cudaMemcpyHostToDevice, stream_));
    const int B = n < 64 ? n : 64;
    dfree(chunk_, own_stream_);
    chunk_ = dalloc<float>((size_t)B * V_ * N_, own_stream_);
    BINDER_CUDA(cudaStreamSynchronize(own_stream_));
    const double eta2[3] = {eta_[0] * eta_[0], eta_[1] * eta_[1], eta_[2] * eta_[2]};
    const double rho_p = rho_[0] * rho_[1] * rho_[2];
    // each sample is rearranged to AoS straight into the chunk, which then goes to the caller's
    // output in one transfer
    auto enqueue = [&](int count) {
        for (int j = 0; j < count; ++j) {
            mstep_.enqueue(r_, d_, zeros_, D_, st_, sigma2_, 1, 0, 1, seed_, 0, rho_p, eta2,
                           nullptr, stream_);
            launch_soa_to_aos(d_, chunk_ + (size_t)j * V_ * N_, V_, N_, stream_);
            launch_sweep_advance(st_, 0x7fffffff, stream_);
        }
    };
    BINDER_CUDA(cudaStreamSynchronize(stream_));
    Graph full, tail;
    const long long k_full = capture_graph(stream_, full, [&] { enqueue(B); });
    const int rem = n % B;
    long long k_tail = 0;
    if (rem) k_tail = capture_graph(stream_, tail, [&] { enqueue(rem); });
    int done = 0;
    while (done < n) {
        const int cnt = (n - done) >= B ? B : rem;
        if (cnt == B) replay(full, k_full, stream_); else replay(tail, k_tail, stream_);
        BINDER_CUDA(cudaMemcpyAsync(out + (size_t)done * V_ * N_, chunk_,
                                    sizeof(float) * (size_t)cnt * V_ * N_, cudaMemcpyDeviceToHost,
                                    stream_));
        BINDER_CUDA(cudaStreamSynchronize(stream_));
        done += cnt;
    }
    sweep_ += n;
}

void PriorTransform::get_shape(int out[4]) const {
    out[0] = nx_; out[1] = ny_; out[2] = nz_; out[3] = N_;
}

}  // namespace binder
