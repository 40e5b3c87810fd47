// Stream-ordered device allocation and the AoS <-> SoA / bin-volume conversion kernels.
#include <cstdint>
#include <mutex>

#include "layout.cuh"

namespace binder {

namespace {

constexpr int kMaxDevices = 64;

// raise the release threshold of the current device's default pool once, so freed blocks stay
// cached in the process instead of going back to the driver at each synchronisation
void configure_pool() {
    static std::mutex mu;
    static bool done[kMaxDevices] = {};
    int dev = -1;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CHECK(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    BINDER_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t threshold = UINT64_MAX;
    BINDER_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    done[dev] = true;
}

int blocks_for(long work) {
    const long b = (work + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148L * 16 ? 148L * 16 : b));
}

// index c of voxel i of the identity grid (a 2D image nx x ny x 1: c = 0 -> x, c = 1 -> y)
__device__ __forceinline__ float grid_coord(long i, int c, const GridDims &g) {
    const long yz = (long)g.ny * g.nz;
    if (c == 0) return (float)(i / yz);
    if (g.N == 2) return (float)(i % yz);
    return c == 1 ? (float)((i / g.nz) % g.ny) : (float)(i % g.nz);
}

__global__ void aos_to_soa_kernel(const float *aos, float *soa, long V, int N) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < N; ++c) soa[c * V + i] = aos[N * i + c];
}

__global__ void soa_to_aos_kernel(const float *soa, float *aos, long V, int N) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < N; ++c) aos[N * i + c] = soa[c * V + i];
}

__global__ void soa_to_aos_plus_kernel(const float *soa, const float *x, GridDims g, float *aos) {
    const long V = (long)g.nx * g.ny * g.nz;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < g.N; ++c) {
            const float b = x ? x[c * V + i] : grid_coord(i, c, g);
            aos[g.N * i + c] = soa[c * V + i] + b;
        }
}

__global__ void aos_minus_to_soa_kernel(const float *aos, const float *x, GridDims g, float *soa) {
    const long V = (long)g.nx * g.ny * g.nz;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < g.N; ++c) {
            const float b = x ? x[c * V + i] : grid_coord(i, c, g);
            soa[c * V + i] = (aos ? aos[g.N * i + c] : 0.0f) - b;
        }
}

__global__ void identity_check_kernel(const float *aos, GridDims g, unsigned *mismatch) {
    const long V = (long)g.nx * g.ny * g.nz;
    bool bad = false;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < g.N; ++c) bad |= aos[g.N * i + c] != grid_coord(i, c, g);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(mismatch, 1u);
}

__global__ void bins_to_u8_kernel(const int *in, long n, int limit, uint8_t *out,
                                  unsigned long long *first_bad) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int b = in[i];
        if (b < 0 || b >= limit) {
            atomicMin(first_bad, (unsigned long long)i);
            out[i] = 0;
        } else {
            out[i] = (uint8_t)b;
        }
    }
}

__global__ void bins_to_padded_kernel(const int *in, int nx, int ny, int nz, int limit,
                                      uint8_t *vpad, int P, int Py, int PZ, int pyn, int zp,
                                      unsigned long long *first_bad) {
    const long n = (long)nx * ny * nz;
    for (long j = (long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (long)gridDim.x * blockDim.x) {
        const int z = (int)(j % nz), y = (int)((j / nz) % ny), x = (int)(j / ((long)ny * nz));
        int b = in[j];
        if (b < 0 || b >= limit) {
            atomicMin(first_bad, (unsigned long long)j);
            b = 0;
        }
        vpad[((long)(x + P) * pyn + (y + Py)) * zp + (z + PZ)] = (uint8_t)b;
    }
}

__global__ void moments_to_aos_kernel(const double *mean, const double *m2, long V, int N,
                                      double scale, double *mean_aos, double *cov_aos) {
    // symmetric M2 stored as its upper triangle: xx, xy, xz, yy, yz, zz (N = 3) or xx, xy, yy
    const int sym3[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    const int sym2[4] = {0, 1, 1, 2};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x) {
        if (mean_aos)
            for (int c = 0; c < N; ++c) mean_aos[N * i + c] = mean[c * V + i];
        if (cov_aos)
            for (int e = 0; e < N * N; ++e)
                cov_aos[N * N * i + e] = m2[(N == 3 ? sym3[e] : sym2[e]) * V + i] * scale;
    }
}

// moments of C chains of n samples each pooled (Chan et al.'s pairwise combination with equal
// counts): mean = the average of the chain means, M2 = sum_c M2_c + n sum_c (m_c - m)(m_c - m)^T,
// cov = M2 / (C n - 1); AoS outputs
__global__ void pool_moments_kernel(const double *mean, const double *m2, long V, int N, int C,
                                    double n, double *mean_aos, double *cov_aos) {
    const int sym3[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    const int sym2[4] = {0, 1, 1, 2};
    const int NM2 = N * (N + 1) / 2;
    const double scale = 1.0 / ((double)C * n - 1.0);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
         i += (long)gridDim.x * blockDim.x) {
        double m[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < C; ++c)
            for (int a = 0; a < N; ++a) m[a] += mean[((long)c * N + a) * V + i];
        for (int a = 0; a < N; ++a) m[a] /= (double)C;
        double q[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int c = 0; c < C; ++c) {
            double dm[3];
            for (int a = 0; a < N; ++a) dm[a] = mean[((long)c * N + a) * V + i] - m[a];
            int e = 0;
            for (int r = 0; r < N; ++r)
                for (int t = r; t < N; ++t, ++e)
                    q[e] += m2[((long)c * NM2 + e) * V + i] + n * dm[r] * dm[t];
        }
        if (mean_aos)
            for (int a = 0; a < N; ++a) mean_aos[N * i + a] = m[a];
        if (cov_aos)
            for (int e = 0; e < N * N; ++e)
                cov_aos[N * N * i + e] = q[N == 3 ? sym3[e] : sym2[e]] * scale;
    }
}

}  // namespace

void launch_pool_moments(const double *mean, const double *m2, long V, int N, int C, double n,
                         double *mean_aos, double *cov_aos, cudaStream_t s) {
    count_launch(), pool_moments_kernel<<<blocks_for(V), 256, 0, s>>>(mean, m2, V, N, C, n,
                                                                       mean_aos, cov_aos);
    BINDER_CUDA(cudaGetLastError());
}

void *dev_alloc(size_t bytes, cudaStream_t s) {
    if (!bytes) return nullptr;
    configure_pool();
    void *p = nullptr;
    BINDER_CUDA(cudaMallocAsync(&p, bytes, s));
    return p;
}

void dev_free(void *p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

void launch_aos_to_soa(const float *aos, float *soa, long V, int N, cudaStream_t s) {
    count_launch(), aos_to_soa_kernel<<<blocks_for(V), 256, 0, s>>>(aos, soa, V, N);
    BINDER_CUDA(cudaGetLastError());
}

void launch_soa_to_aos(const float *soa, float *aos, long V, int N, cudaStream_t s) {
    count_launch(), soa_to_aos_kernel<<<blocks_for(V), 256, 0, s>>>(soa, aos, V, N);
    BINDER_CUDA(cudaGetLastError());
}

void launch_soa_to_aos_plus(const float *soa, const float *x, GridDims g, float *aos,
                            cudaStream_t s) {
    const long V = (long)g.nx * g.ny * g.nz;
    count_launch(), soa_to_aos_plus_kernel<<<blocks_for(V), 256, 0, s>>>(soa, x, g, aos);
    BINDER_CUDA(cudaGetLastError());
}

void launch_aos_minus_to_soa(const float *aos, const float *x, GridDims g, float *soa,
                             cudaStream_t s) {
    const long V = (long)g.nx * g.ny * g.nz;
    count_launch(), aos_minus_to_soa_kernel<<<blocks_for(V), 256, 0, s>>>(aos, x, g, soa);
    BINDER_CUDA(cudaGetLastError());
}

void launch_identity_check(const float *aos, GridDims g, unsigned *mismatch, cudaStream_t s) {
    const long V = (long)g.nx * g.ny * g.nz;
    count_launch(), identity_check_kernel<<<blocks_for(V), 256, 0, s>>>(aos, g, mismatch);
    BINDER_CUDA(cudaGetLastError());
}

void launch_bins_to_u8(const int *in, long n, int limit, uint8_t *out,
                       unsigned long long *first_bad, cudaStream_t s) {
    count_launch(), bins_to_u8_kernel<<<blocks_for(n), 256, 0, s>>>(in, n, limit, out, first_bad);
    BINDER_CUDA(cudaGetLastError());
}

void launch_bins_to_padded(const int *in, int nx, int ny, int nz, int limit, uint8_t *vpad, int P,
                           int Py, int PZ, int pyn, int zp, unsigned long long *first_bad,
                           cudaStream_t s) {
    const long n = (long)nx * ny * nz;
    count_launch(), bins_to_padded_kernel<<<blocks_for(n), 256, 0, s>>>(
        in, nx, ny, nz, limit, vpad, P, Py, PZ, pyn, zp, first_bad);
    BINDER_CUDA(cudaGetLastError());
}

void launch_moments_to_aos(const double *mean, const double *m2, long V, int N, double scale,
                           double *mean_aos, double *cov_aos, cudaStream_t s) {
    count_launch(), moments_to_aos_kernel<<<blocks_for(V), 256, 0, s>>>(mean, m2, V, N, scale,
                                                                         mean_aos, cov_aos);
    BINDER_CUDA(cudaGetLastError());
}

}  // namespace binder
