// The multi-resolution step on the device; see multires.cuh.
#include <cmath>
#include <vector>

#include "layout.cuh"
#include "multires.cuh"
#include "resample.cuh"

namespace binder {

namespace {

int blocks(long work) {
    int dev = 0, sms = 148;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long need = (work + 255) / 256;
    const long cap = (long)sms * 8;
    return (int)(need < 1 ? 1 : (need < cap ? need : cap));
}

struct Dims {
    int x, y, z;
    __host__ __device__ long count() const { return (long)x * y * z; }
};

// full_voxels_pos[::r, ::r, ::r, :] / r as AoS FP64 [V][N] of the level grid `o`; the full grid
// `f` is the identity when pos is null.  In 2D (f.z == 1) the components are (x, y).
__global__ void strided_positions_kernel(const double *pos, Dims f, int r, Dims o, int N,
                                         double *out) {
    const long V = o.count();
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ((long)o.y * o.z)), y = (int)((p / o.z) % o.y),
                  z = (int)(p % o.z);
        const long q = ((long)x * r * f.y + (long)y * r) * f.z + (long)z * r;
        for (int n = 0; n < N; ++n) {
            double v;
            if (pos) {
                v = pos[q * N + n];
            } else {
                const int c = n == 0 ? x * r : (n == 1 ? y * r : z * r);
                v = (double)c;
            }
            out[p * N + n] = v / (double)r;
        }
    }
}

// registration positions (FP32 SoA [N][V]) -> FP64 AoS [V][N]
__global__ void soa_f32_to_aos_f64_kernel(const float *soa, long V, int N, double *aos) {
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x)
        for (int n = 0; n < N; ++n) aos[p * N + n] = (double)soa[n * V + p];
}

// a[i] = a[i] * s + b[i] (b may be null), over n values
__global__ void axpy_kernel(double *a, const double *b, double s, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        a[i] = b ? a[i] * s + b[i] : a[i] * s;
}

__global__ void sub_kernel(double *a, const double *b, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        a[i] = a[i] - b[i];
}

__global__ void to_f32_kernel(const double *in, float *out, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// full[::r, ::r, ::r] of an int32 volume, and the count of non-zero entries
__global__ void strided_bins_kernel(const int *full, Dims f, int r, Dims o, int *out,
                                    unsigned long long *nonzero) {
    const long V = o.count();
    unsigned long long nz = 0;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ((long)o.y * o.z)), y = (int)((p / o.z) % o.y),
                  z = (int)(p % o.z);
        const int b = full[((long)x * r * f.y + (long)y * r) * f.z + (long)z * r];
        out[p] = b;
        nz += b != 0;
    }
    if (nonzero) {
        for (int o2 = 16; o2 > 0; o2 >>= 1) nz += __shfl_xor_sync(0xffffffffu, nz, o2);
        if ((threadIdx.x & 31) == 0 && nz) atomicAdd(nonzero, nz);
    }
}

// D[k] = (t_x[kx] + t_y[ky] (+ t_z[kz])) ^ order in FP64, stored FP32
__global__ void prior_eigen_kernel(const double *tx, const double *ty, const double *tz, Dims o,
                                   int order, float *D) {
    const long V = o.count();
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ((long)o.y * o.z)), y = (int)((p / o.z) % o.y),
                  z = (int)(p % o.z);
        double d = tx[x] + ty[y];
        if (tz) d = d + tz[z];
        double v;
        if (order == 1)
            v = d;
        else if (order == 2)
            v = d * d;
        else
            v = pow(d, (double)order);
        D[p] = (float)v;
    }
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

int ceil_div(int n, int r) { return (n + r - 1) / r; }

}  // namespace

Pyramid::Pyramid(const PyramidConfig &c, const int *binned_voxels, const int *binned_nodes,
                 const double *voxel_pos)
    : c_(c) {
    BINDER_CHECK(c.nx > 0 && c.ny > 0 && c.nz > 0 && c.nxn > 0 && c.nyn > 0 && c.nzn > 0,
                 "grid dimensions must be positive");
    BINDER_CHECK(c.nz > 1 || c.nzn == 1, "a 2D image (Nz_v == 1) needs a 2D node grid");
    BINDER_CHECK(c.finite_difference_order >= 1, "finite_difference_order must be >= 1");
    for (int a = 0; a < 3; ++a)
        BINDER_CHECK(c.voxel_size[a] > 0 && c.node_size[a] > 0, "voxel sizes must be positive");
    N_ = c.nz == 1 ? 2 : 3;
    BINDER_CUDA(cudaStreamCreate(&s_));
    const long V = (long)c.nx * c.ny * c.nz, Vn = (long)c.nxn * c.nyn * c.nzn;
    try {
        u_ = dev_alloc_n<int>((size_t)V, s_);
        v_ = dev_alloc_n<int>((size_t)Vn, s_);
        BINDER_CUDA(cudaMemcpyAsync(u_, binned_voxels, sizeof(int) * V, cudaMemcpyDefault, s_));
        BINDER_CUDA(cudaMemcpyAsync(v_, binned_nodes, sizeof(int) * Vn, cudaMemcpyDefault, s_));
        if (voxel_pos) {
            pos_ = dev_alloc_n<double>((size_t)V * N_, s_);
            BINDER_CUDA(cudaMemcpyAsync(pos_, voxel_pos, sizeof(double) * V * N_,
                                        cudaMemcpyDefault, s_));
        }
        BINDER_CUDA(cudaStreamSynchronize(s_));
    } catch (...) {
        dev_free_p(u_, s_);
        dev_free_p(v_, s_);
        dev_free_p(pos_, s_);
        cudaStreamSynchronize(s_);
        cudaStreamDestroy(s_);
        throw;
    }
}

Pyramid::~Pyramid() {
    dev_free_p(u_, s_);
    dev_free_p(v_, s_);
    dev_free_p(pos_, s_);
    cudaStreamSynchronize(s_);
    cudaStreamDestroy(s_);
}

Registration *Pyramid::level(int res, const Registration *prev, int prev_res, double alpha,
                             const float *theta, int K, int L, LevelInfo *info) {
    BINDER_CHECK(res >= 1, "resolution must be >= 1");
    const int cur = prev ? prev_res : 1;
    BINDER_CHECK(cur >= 1, "previous resolution must be >= 1");
    BINDER_CHECK(theta || (prev && prev->theta_device()),
                 "theta must be given when there is no previous level to carry it over");
    BINDER_CHECK(theta || (prev->K() == K && prev->L() == L),
                 "the previous level's theta has other numbers of bins");
    const cudaStream_t s = s_;
    const int N = N_;
    const Dims full{c_.nx, c_.ny, c_.nz};
    const Dims fulln{c_.nxn, c_.nyn, c_.nzn};
    // FastRegistration.py:552-559: current sizes and shapes, ceil(shape / res)
    LevelInfo li{};
    const int vsh[3] = {ceil_div(c_.nx, res), ceil_div(c_.ny, res), ceil_div(c_.nz, res)};
    const int nsh[3] = {ceil_div(c_.nxn, res), ceil_div(c_.nyn, res), ceil_div(c_.nzn, res)};
    for (int a = 0; a < 3; ++a) {
        li.voxels_shape[a] = vsh[a];
        li.nodes_shape[a] = nsh[a];
        li.voxel_size[a] = c_.voxel_size[a] * res;
        li.node_size[a] = c_.node_size[a] * res;
    }
    const Dims lv{vsh[0], vsh[1], vsh[2]}, ln{nsh[0], nsh[1], nsh[2]};
    const Dims cd{ceil_div(c_.nx, cur), ceil_div(c_.ny, cur), ceil_div(c_.nz, cur)};
    if (prev) {
        int pd[3];
        prev->dims(pd);
        BINDER_CHECK(pd[0] == cd.x && pd[1] == cd.y && pd[2] == cd.z && prev->components() == N,
                     "the previous registration's grid is not this pyramid's grid at its "
                     "resolution");
        BINDER_CUDA(cudaStreamSynchronize(prev->stream()));  // its positions are final
    }
    const long Vl = lv.count(), Vc = cd.count();

    // voxels_pos = full_voxels_pos[::res] / res
    DBuf<double> lpos(Vl * N, s);
    count_launch(), strided_positions_kernel<<<blocks(Vl), 256, 0, s>>>(pos_, full, res, lv, N,
                                                                       lpos.p);
    BINDER_CUDA(cudaGetLastError());

    // the deformation at the current resolution, FP64 AoS
    DBuf<double> src(Vc * N, s);
    if (prev) {
        count_launch(), soa_f32_to_aos_f64_kernel<<<blocks(Vc), 256, 0, s>>>(
                            prev->positions_device(), Vc, N, src.p);
    } else {
        count_launch(), strided_positions_kernel<<<blocks(Vc), 256, 0, s>>>(pos_, full, 1, cd, N,
                                                                           src.p);
    }
    BINDER_CUDA(cudaGetLastError());

    // FastRegistration.py:562-577
    DBuf<double> fld(Vl * N, s);
    const int in_dims[3] = {cd.x, cd.y, cd.z};
    const double ratio = (double)cur / (double)res;
    if (!c_.upsample_in_frequency_domain || cur - res < 0) {
        Resampler rs(Resampler::kLinear, in_dims, vsh, N, s);
        rs.apply(src.p, fld.p, s);
        count_launch(), axpy_kernel<<<blocks(Vl * N), 256, 0, s>>>(fld.p, nullptr, ratio, Vl * N);
    } else if (res != cur) {
        // delta = deformation - full_voxels_pos[::cur] / cur, up-sampled, rescaled, + voxels_pos
        DBuf<double> cpos(Vc * N, s);
        count_launch(), strided_positions_kernel<<<blocks(Vc), 256, 0, s>>>(pos_, full, cur, cd,
                                                                            N, cpos.p);
        count_launch(), sub_kernel<<<blocks(Vc * N), 256, 0, s>>>(src.p, cpos.p, Vc * N);
        Resampler rs(Resampler::kUpSample, in_dims, vsh, N, s);
        rs.apply(src.p, fld.p, s);
        count_launch(), axpy_kernel<<<blocks(Vl * N), 256, 0, s>>>(fld.p, lpos.p, ratio, Vl * N);
    } else {
        BINDER_CUDA(cudaMemcpyAsync(fld.p, src.p, sizeof(double) * Vl * N,
                                    cudaMemcpyDeviceToDevice, s));
    }
    BINDER_CUDA(cudaGetLastError());

    // binned_voxels / binned_nodes = full[::res]; non_zero_voxels = count_nonzero(binned_voxels)
    DBuf<int> lu(Vl, s), lvb(ln.count(), s);
    DBuf<unsigned long long> nzc(1, s);
    BINDER_CUDA(cudaMemsetAsync(nzc.p, 0, sizeof(unsigned long long), s));
    count_launch(), strided_bins_kernel<<<blocks(Vl), 256, 0, s>>>(u_, full, res, lv, lu.p, nzc.p);
    count_launch(), strided_bins_kernel<<<blocks(ln.count()), 256, 0, s>>>(v_, fulln, res, ln,
                                                                          lvb.p, nullptr);
    BINDER_CUDA(cudaGetLastError());

    // D = initialize_fourier_domain_smoothing(voxels_shape, True, order, ndims, current size)
    // (BINDER/utils.py:270-365): per-axis terms (2 - 2 cos(pi k / n)) / h^2
    const int ndims = N;
    std::vector<double> t[3];
    DBuf<double> tx(vsh[0], s), ty(vsh[1], s), tz(vsh[2], s);
    double *tdev[3] = {tx.p, ty.p, tz.p};
    for (int a = 0; a < ndims; ++a) {
        // 2D: the axes are x and y (the unit z axis carries no term)
        const int n = vsh[a];
        const double h = li.voxel_size[a];
        t[a].resize(n);
        for (int k = 0; k < n; ++k)
            t[a][k] = (2.0 - 2.0 * std::cos(3.14159265358979323846 * k / n)) / (h * h);
        BINDER_CUDA(cudaMemcpyAsync(tdev[a], t[a].data(), sizeof(double) * n,
                                    cudaMemcpyHostToDevice, s));
    }
    DBuf<float> D(Vl, s);
    count_launch(), prior_eigen_kernel<<<blocks(Vl), 256, 0, s>>>(
                        tx.p, ty.p, ndims == 3 ? tz.p : nullptr, lv, c_.finite_difference_order,
                        D.p);
    BINDER_CUDA(cudaGetLastError());

    // FP32 arrays for the registration (its own precision)
    DBuf<float> fl32(Vl * N, s), pos32(Vl * N, s);
    count_launch(), to_f32_kernel<<<blocks(Vl * N), 256, 0, s>>>(fld.p, fl32.p, Vl * N);
    count_launch(), to_f32_kernel<<<blocks(Vl * N), 256, 0, s>>>(lpos.p, pos32.p, Vl * N);
    BINDER_CUDA(cudaGetLastError());
    unsigned long long nonzero = 0;
    BINDER_CUDA(cudaMemcpyAsync(&nonzero, nzc.p, sizeof(nonzero), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));  // tables, counts and arrays are complete
    li.non_zero_voxels = (double)nonzero;

    // FastRegistration.py:617-630: gamma per axis scaled by the current sizes and voxel count
    const double vprod = li.voxel_size[0] * li.voxel_size[1] * li.voxel_size[2];
    const double count = c_.increase_gamma_at_ds ? (double)c_.nx * c_.ny * c_.nz
                                                 : (double)vsh[0] * vsh[1] * vsh[2];
    for (int a = 0; a < 3; ++a)
        li.gamma[a] = c_.gamma_init * vprod * count * (li.node_size[a] * li.node_size[a]);

    // FastRegistration.py:452-486
    Registration *r = new Registration(fl32.p, pos32.p, vsh[0], vsh[1], vsh[2], nsh[0], nsh[1],
                                       nsh[2], c_.spline_order, li.non_zero_voxels);
    try {
        r->set_nonlinear_transformation(li.gamma, li.voxel_size, li.node_size, D.p);
        const float *th = theta ? theta : prev->theta_device();
        r->set_mi_likelihood(alpha, th, K, L, lvb.p, lu.p);
    } catch (...) {
        delete r;
        throw;
    }
    if (info) *info = li;
    return r;
}

}  // namespace binder
