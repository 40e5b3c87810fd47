// Separable FP64 resampling of AoS fields (the multi-resolution step); see resample.cuh.
#include <cmath>
#include <vector>

#include "layout.cuh"
#include "resample.cuh"
#include "transform.cuh"

namespace binder {

namespace {

// out[(o*no + ko)*s + t] = sum_ki M[ko*ni + ki] * in[(o*ni + ki)*s + t]
__global__ void rect_axis_kernel(const double *__restrict__ in, double *__restrict__ out,
                                 const double *__restrict__ M, int ni, int no, long outer, long s,
                                 double scale) {
    const long total = outer * no * s;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long)gridDim.x * blockDim.x) {
        const long t = q % s;
        const long r = q / s;
        const int ko = (int)(r % no);
        const long o = r / no;
        const double *src = in + o * ni * s + t;
        const double *row = M + (long)ko * ni;
        double acc = 0.0;
        for (int ki = 0; ki < ni; ++ki) acc += row[ki] * src[ki * s];
        out[q] = acc * scale;
    }
}

__global__ void scale_copy_kernel(const double *in, double *out, long n, double scale) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x)
        out[q] = in[q] * scale;
}

int blocks_for(long work) {
    int dev = 0, sms = 148;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long need = (work + 255) / 256;
    const long cap = (long)sms * 8;
    return (int)(need < 1 ? 1 : (need < cap ? need : cap));
}

// whole-sample symmetric ('mirror') extension of index i on a line of n samples
int mirror_index(long i, int n) {
    if (n <= 1) return 0;
    const long p = 2L * n - 2;
    i %= p;
    if (i < 0) i += p;
    return (int)(i >= n ? p - i : i);
}

// the same extension applied to a coordinate, as scipy.ndimage maps one before interpolating
double mirror_coordinate(double c, int n) {
    if (n <= 1) return 0.0;
    const double p = 2.0 * n - 2.0;
    if (c < 0) {
        c = p * (double)(long)(-c / p) + c;
        c = c <= 1 - n ? c + p : -c;
    } else if (c > n - 1) {
        c -= p * (double)(long)(c / p);
        if (c >= n) c = p - c;
    }
    return c;
}

template <typename T>
struct DBuf {
    T *p = nullptr;
    cudaStream_t s = 0;
    DBuf(size_t n, cudaStream_t stream) : s(stream) { p = dev_alloc_n<T>(n, s); }
    ~DBuf() { dev_free(p, s); }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
};

}  // namespace

void dct_upsample_matrix(int n, int m, std::vector<double> &U) {
    BINDER_CHECK(n >= 1 && m >= n, "spectral up-sampling needs an output axis at least as long");
    std::vector<double> Cn((size_t)n * n), Cm((size_t)m * m);
    dct2_matrix(n, Cn.data());  // Cn[k*n + j]: basis k at sample j
    dct2_matrix(m, Cm.data());
    U.assign((size_t)m * n, 0.0);
    for (int jo = 0; jo < m; ++jo)
        for (int j = 0; j < n; ++j) {
            double acc = 0.0;
            for (int k = 0; k < n; ++k) acc += Cm[(size_t)k * m + jo] * Cn[(size_t)k * n + j];
            U[(size_t)jo * n + j] = acc;
        }
}

void linear_resize_matrix(int n, int m, std::vector<double> &R) {
    BINDER_CHECK(n >= 1 && m >= 1, "axis lengths must be positive");
    const double factor = (double)n / (double)m;
    // Gaussian pre-filter (correlation with mirror extension) on a shrinking axis
    std::vector<double> G((size_t)n * n, 0.0);
    const double sigma = factor > 1.0 ? (factor - 1.0) / 2.0 : 0.0;
    if (sigma > 1e-15) {
        const int r = (int)(4.0 * sigma + 0.5);
        std::vector<double> w(2 * r + 1);
        double tot = 0.0;
        for (int j = -r; j <= r; ++j) {
            w[j + r] = std::exp(-0.5 / (sigma * sigma) * (double)j * (double)j);
            tot += w[j + r];
        }
        for (double &v : w) v /= tot;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j <= 2 * r; ++j)
                G[(size_t)i * n + mirror_index((long)i + j - r, n)] += w[j];
    } else {
        for (int i = 0; i < n; ++i) G[(size_t)i * n + i] = 1.0;
    }
    // linear interpolation at the pixel-centre-aligned coordinates (ko + 0.5) n/m - 0.5
    R.assign((size_t)m * n, 0.0);
    std::vector<double> z(n);
    for (int ko = 0; ko < m; ++ko) {
        std::fill(z.begin(), z.end(), 0.0);
        const double c = mirror_coordinate(((double)ko + 0.5) * factor - 0.5, n);
        const double f = std::floor(c);
        const double t = c - f;
        const int i0 = (int)f;
        z[mirror_index(i0, n)] += 1.0 - t;
        z[mirror_index((long)i0 + 1, n)] += t;
        for (int i = 0; i < n; ++i) {
            if (z[i] == 0.0) continue;
            for (int j = 0; j < n; ++j) R[(size_t)ko * n + j] += z[i] * G[(size_t)i * n + j];
        }
    }
}

void separable_apply(const double *in, int nx, int ny, int nz, int N, const double *Mx,
                     const double *My, const double *Mz, int mx, int my, int mz, double *out,
                     double *tmp1, double *tmp2, cudaStream_t s) {
    // z: [nx*ny][nz][N] -> [nx*ny][mz][N]
    const double *cur = in;
    auto pass = [&](const double *M, int ni, int no, long outer, long stride, double *dst) {
        const long total = outer * no * stride;
        count_launch(), rect_axis_kernel<<<blocks_for(total), 256, 0, s>>>(cur, dst, M, ni, no,
                                                                          outer, stride, 1.0);
        BINDER_CUDA(cudaGetLastError());
        cur = dst;
    };
    if (Mz) pass(Mz, nz, mz, (long)nx * ny, N, tmp1);
    if (My) pass(My, ny, my, nx, (long)mz * N, cur == tmp1 ? tmp2 : tmp1);
    if (Mx) {
        pass(Mx, nx, mx, 1, (long)my * mz * N, out);
    } else {
        const long total = (long)mx * my * mz * N;
        count_launch(), scale_copy_kernel<<<blocks_for(total), 256, 0, s>>>(cur, out, total, 1.0);
        BINDER_CUDA(cudaGetLastError());
    }
}

Resampler::Resampler(Kind kind, const int in[3], const int out[3], int N, cudaStream_t s)
    : N_(N), s_(s) {
    for (int a = 0; a < 3; ++a) {
        BINDER_CHECK(in[a] >= 1 && out[a] >= 1, "grid dimensions must be positive");
        n_[a] = in[a];
        m_[a] = out[a];
    }
    try {
        for (int a = 0; a < 3; ++a) {
            if (n_[a] == m_[a]) continue;  // both kinds are the identity on an unchanged axis
            std::vector<double> M;
            if (kind == kUpSample)
                dct_upsample_matrix(n_[a], m_[a], M);
            else
                linear_resize_matrix(n_[a], m_[a], M);
            M_[a] = dev_alloc_n<double>(M.size(), s);
            BINDER_CUDA(cudaMemcpyAsync(M_[a], M.data(), sizeof(double) * M.size(),
                                        cudaMemcpyHostToDevice, s));
            BINDER_CUDA(cudaStreamSynchronize(s));  // M goes out of scope
        }
        const long mz = m_[2] > n_[2] ? m_[2] : n_[2];
        const long my = m_[1] > n_[1] ? m_[1] : n_[1];
        tmp1_ = dev_alloc_n<double>((size_t)n_[0] * my * mz * N, s);
        tmp2_ = dev_alloc_n<double>((size_t)n_[0] * my * mz * N, s);
    } catch (...) {
        release();
        throw;
    }
}

Resampler::~Resampler() { release(); }

void Resampler::release() {
    for (auto &p : M_) dev_free_p(p, s_);
    dev_free_p(tmp1_, s_);
    dev_free_p(tmp2_, s_);
}

void Resampler::apply(const double *in, double *out, cudaStream_t s) {
    separable_apply(in, n_[0], n_[1], n_[2], N_, M_[0], M_[1], M_[2], m_[0], m_[1], m_[2], out,
                    tmp1_, tmp2_, s);
}

namespace {
void host_resample(Resampler::Kind kind, const double *field, const int in[3], const int out[3],
                   int N, double scale, double *host_out) {
    cudaStream_t s = nullptr;
    BINDER_CUDA(cudaStreamCreate(&s));
    try {
        const long V = (long)in[0] * in[1] * in[2], Vo = (long)out[0] * out[1] * out[2];
        {
            Resampler rs(kind, in, out, N, s);
            DBuf<double> a(V * N, s), b(Vo * N, s);
            BINDER_CUDA(cudaMemcpyAsync(a.p, field, sizeof(double) * V * N,
                                        cudaMemcpyHostToDevice, s));
            rs.apply(a.p, b.p, s);
            if (scale != 1.0) {
                count_launch(), scale_copy_kernel<<<blocks_for(Vo * N), 256, 0, s>>>(
                                    b.p, b.p, Vo * N, scale);
                BINDER_CUDA(cudaGetLastError());
            }
            BINDER_CUDA(cudaMemcpyAsync(host_out, b.p, sizeof(double) * Vo * N,
                                        cudaMemcpyDeviceToHost, s));
            BINDER_CUDA(cudaStreamSynchronize(s));
        }
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamSynchronize(s);  // the buffers' stream-ordered frees
    cudaStreamDestroy(s);
}
}  // namespace

namespace {
__global__ void f32_to_f64_kernel(const float *in, double *out, long n) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x)
        out[q] = (double)in[q];
}

__global__ void add_aos_to_soa_kernel(const double *aos, long V, int N, float *soa) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < N; ++c) soa[c * V + i] += (float)aos[i * N + c];
}
}  // namespace

void add_resized_displacement(const float *field, int fx, int fy, int fz, int N, int nx, int ny,
                              int nz, float *soa, cudaStream_t s) {
    BINDER_CHECK(fx >= 1 && fy >= 1 && fz >= 1, "the field's dimensions must be positive");
    BINDER_CHECK(N >= 1 && N <= 3, "fields have 1 to 3 components");
    const long Vf = (long)fx * fy * fz, V = (long)nx * ny * nz;
    const int in[3] = {fx, fy, fz}, o[3] = {nx, ny, nz};
    DBuf<float> f32(Vf * N, s);
    DBuf<double> f64(Vf * N, s), up(V * N, s);
    BINDER_CUDA(cudaMemcpyAsync(f32.p, field, sizeof(float) * Vf * N, cudaMemcpyDefault, s));
    count_launch(), f32_to_f64_kernel<<<blocks_for(Vf * N), 256, 0, s>>>(f32.p, f64.p, Vf * N);
    BINDER_CUDA(cudaGetLastError());
    {
        Resampler rs(Resampler::kLinear, in, o, N, s);
        rs.apply(f64.p, up.p, s);
        count_launch(), add_aos_to_soa_kernel<<<blocks_for(V), 256, 0, s>>>(up.p, V, N, soa);
        BINDER_CUDA(cudaGetLastError());
        BINDER_CUDA(cudaStreamSynchronize(s));  // the resampler's matrices go with it
    }
}

void up_sample(const double *field, int nx, int ny, int nz, int mx, int my, int mz, double *out) {
    BINDER_CHECK(nx >= 1 && ny >= 1 && nz >= 1, "input dimensions must be positive");
    BINDER_CHECK(mx >= nx && my >= ny && mz >= nz,
                 "up_sample needs every output axis at least as long as the input axis");
    BINDER_CHECK((nz == 1) == (mz == 1), "a 2D field (nz == 1) up-samples to a 2D field");
    const int in[3] = {nx, ny, nz}, o[3] = {mx, my, mz};
    host_resample(Resampler::kUpSample, field, in, o, mz == 1 ? 2 : 3, 1.0, out);
}

void resize_linear(const double *field, int nx, int ny, int nz, int N, int mx, int my, int mz,
                   double scale, double *out) {
    BINDER_CHECK(N >= 1 && N <= 3, "fields have 1 to 3 components");
    const int in[3] = {nx, ny, nz}, o[3] = {mx, my, mz};
    host_resample(Resampler::kLinear, field, in, o, N, scale, out);
}

}  // namespace binder
