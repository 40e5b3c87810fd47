// Separable transform passes (DCT prior smoothing, Hartley Poisson solve) -- see transform.cuh.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "transform.cuh"

namespace binder {

namespace {

constexpr int kThreads = 256;
constexpr int TC = 64;  // columns (lines) per CTA tile
constexpr int JC = 32;  // staged chunk of the matrix's inner dimension

template <typename T>
struct Pitch;
template <>
struct Pitch<float> {
    static constexpr int v = 68;  // 16-byte aligned rows
};
template <>
struct Pitch<double> {
    static constexpr int v = 66;
};

__device__ __forceinline__ void load4(const float *p, float v[4]) {
    const float4 q = *reinterpret_cast<const float4 *>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void load4(const double *p, double v[4]) {
    const double2 a = *reinterpret_cast<const double2 *>(p);
    const double2 b = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// acc[r][q] = sum_j M[k][j] * Xs[j][c] for rows k = k0 + ty + 16 r and columns c = 4 tx + q
template <typename T, int R>
__device__ __forceinline__ void gemm_tile(const T *__restrict__ M, int n, const T *Xs, T *Ms,
                                          T (&acc)[R][4], int tx, int ty, int k0) {
    constexpr int P = Pitch<T>::v;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[r][q] = T(0);
    for (int j0 = 0; j0 < n; j0 += JC) {
        __syncthreads();
        for (int f = threadIdx.x; f < 16 * R * JC; f += kThreads) {
            const int k = f / JC, jj = f - k * JC, j = j0 + jj;
            Ms[k * (JC + 1) + jj] = (k0 + k < n && j < n) ? M[(long)(k0 + k) * n + j] : T(0);
        }
        __syncthreads();
        const int jn = min(JC, n - j0);
        for (int jj = 0; jj < jn; ++jj) {
            T xv[4];
            load4(Xs + (j0 + jj) * P + tx * 4, xv);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const T m = Ms[(ty + 16 * r) * (JC + 1) + jj];
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[r][q] = fma(m, xv[q], acc[r][q]);
            }
        }
    }
}

// prior-sampling normal for DCT coefficient i of component comp (matches the oracle's stream)
__device__ __forceinline__ float prior_normal(uint64_t seed, uint32_t i, uint32_t sweep,
                                              uint32_t chain, int comp) {
    return dct_prior_normal(seed, i, sweep, chain, comp);
}

// Hartley Poisson step of an x-axis pass (outer == 1, s == ny*nz) on rows k = k0 + ty + 16 r:
// c <- -c / (lambda * V), lambda = 6 - 2cos z - 2cos x - 2cos y
template <typename T, int R>
__device__ __forceinline__ void poisson_scale(const AxisArgs<T> &a, T (&acc)[R][4], int k0,
                                              long t0, int ncol, int tx, int ty) {
    const int n = a.n, nz = a.nz;
    const double inv_total = 1.0 / ((double)n * (double)a.s);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = k0 + ty + 16 * r;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = tx * 4 + q;
            if (k < n && c < ncol) {
                const long t = t0 + c;
                const int ky = (int)(t / nz), kz = (int)(t - (long)ky * nz);
                const double lam =
                    6.0 - 2.0 * a.cos_z[kz] - 2.0 * a.cos_x[k] - 2.0 * a.cos_y[ky];
                acc[r][q] = fabs(lam) > 1e-10 ? (T)(-(double)acc[r][q] / lam * inv_total) : T(0);
            }
        }
    }
}

template <typename T, int R, int MODE>
__global__ void __launch_bounds__(kThreads) axis_kernel(const AxisArgs<T> a) {
    if (a.skip && *a.skip) return;
    constexpr int P = Pitch<T>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Xs = reinterpret_cast<T *>(smem_raw);
    T *Ms = Xs + (size_t)a.n * P;  // the slab holds all n rows
    __shared__ double red[32];

    const int comp = blockIdx.z;
    // components of a batch of chains are numbered chain * chain_comps + component: the chain
    // picks the state and the Philox chain index, the component within it everything else
    const int bch = a.chain_comps ? comp / a.chain_comps : 0;
    const int cn = comp - bch * a.chain_comps;
    DevState *const st = a.st ? a.st + bch : nullptr;
    const uint32_t chain = a.chain + (uint32_t)bch;
    const T *in = a.in + comp * a.comp_stride;
    T *out = a.out + comp * a.comp_stride;
    const int n = a.n;
    const bool contig = (a.s == 1);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    // output rows of this CTA: k0 .. k0 + 16R - 1 (one row block, k0 = 0, unless the launch splits
    // the rows of a plain or position-storing pass over blockIdx.y)
    const int k0 = blockIdx.y * 16 * R;

    long o, t0 = 0;
    int ncol;
    if (contig) {
        o = (long)blockIdx.x * TC;
        ncol = (int)min((long)TC, a.outer - o);
    } else {
        const long tiles = (a.s + TC - 1) / TC;
        o = blockIdx.x / tiles;
        t0 = (blockIdx.x % tiles) * TC;
        ncol = (int)min((long)TC, a.s - t0);
    }

    // ---- stage the n x TC slab ----
    if (contig) {
        const T *src = in + o * n;
        for (int f = threadIdx.x; f < ncol * n; f += kThreads) {
            const int c = f / n, j = f - c * n;
            Xs[j * P + c] = src[f];
        }
        if (ncol < TC)
            for (int f = threadIdx.x; f < n * TC; f += kThreads) {
                const int j = f / TC, c = f - j * TC;
                if (c >= ncol) Xs[j * P + c] = T(0);
            }
    } else {
        const T *src = in + o * n * a.s + t0;
        for (int f = threadIdx.x; f < n * TC; f += kThreads) {
            const int j = f / TC, c = f - j * TC;
            Xs[j * P + c] = (c < ncol) ? src[(long)j * a.s + c] : T(0);
        }
    }

    T acc[R][4];
    gemm_tile<T, R>(a.M, n, Xs, Ms, acc, tx, ty, k0);
    if constexpr (MODE == kEpiPoissonFwd) poisson_scale<T, R>(a, acc, k0, t0, ncol, tx, ty);

    if constexpr (MODE == kEpiSpectral || MODE == kEpiPoisson) {
        // x-axis pass (outer == 1, s == ny*nz): coefficient (k, t) has flat index k*s + t
        double part_cost = 0.0, part_raw = 0.0;
        if constexpr (MODE == kEpiSpectral) {
            const double g = st->gamma[cn];
            const float gs2 = (float)(g * a.sigma2);
            const uint32_t sweep = (uint32_t)st->sweep;
            const bool want_raw = a.want_raw && (st->sweep % a.every == 0);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int k = ty + 16 * r;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int c = tx * 4 + q;
                    if (k < n && c < ncol) {
                        const long i = (long)k * a.s + t0 + c;
                        const float Dv = a.D[i];
                        const float f = 1.0f / (1.0f + gs2 * Dv);
                        float v = (float)acc[r][q] * f;
                        if (a.sample)
                            v += sqrtf((float)a.sigma2 * f) *
                                 prior_normal(a.seed, (uint32_t)i, sweep, chain, cn);
                        const double v2 = (double)v * (double)v;
                        part_cost += 0.5 * g * (double)Dv * v2;
                        if (want_raw) part_raw += a.eta2[cn] * a.rho_p * (double)Dv * v2;
                        acc[r][q] = (T)v;
                    }
                }
            }
        } else {
            poisson_scale<T, R>(a, acc, 0, t0, ncol, tx, ty);
        }
        if constexpr (MODE == kEpiSpectral) {
            const double sc = block_sum(part_cost, red);
            if (threadIdx.x == 0) atomicAdd(&st->lp_tr, sc);
            if (a.want_raw) {  // uniform across the block: every thread takes the same branch
                const double sr = block_sum(part_raw, red);
                if (threadIdx.x == 0) atomicAdd(&st->raw_reg, sr);
            }
        }
        __syncthreads();  // everyone is done reading Xs
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = ty + 16 * r;
            if (k < n)
#pragma unroll
                for (int q = 0; q < 4; ++q) Xs[k * P + tx * 4 + q] = acc[r][q];
        }
        gemm_tile<T, R>(a.M2, n, Xs, Ms, acc, tx, ty, 0);
    }

    // ---- store ----
    if (contig) {
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = k0 + ty + 16 * r;
            if (k < n)
#pragma unroll
                for (int q = 0; q < 4; ++q) Xs[k * P + tx * 4 + q] = acc[r][q];
        }
        __syncthreads();
        T *dst = out + o * n;
        const long base = o * n;
        const int nr = min(16 * R, n - k0);  // rows of this CTA
        for (int f = threadIdx.x; f < ncol * nr; f += kThreads) {
            const int c = f / nr, j = k0 + (f - c * nr);
            const int e = c * n + j;  // element of the tile's lines
            T val = Xs[j * P + c];
            if constexpr (MODE == kEpiPositions) {
                const long i = base + e;
                float xv;
                if (a.xpos) {
                    xv = a.xpos[cn * a.comp_stride + i];
                } else {
                    const long yz = (long)a.ny * a.nz;
                    xv = cn == 0 ? (float)(i / yz)
                                   : (cn == 1 ? (float)((i / a.nz) % a.ny) : (float)(i % a.nz));
                }
                val = (T)((float)val + xv);
            } else if constexpr (MODE == kEpiTopoOut) {
                val = (T)((double)val * a.out_scale[cn] + a.out_offset[cn]);
            }
            dst[e] = val;
        }
    } else {
        T *dst = out + o * n * a.s + t0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = k0 + ty + 16 * r;
            if (k < n)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int c = tx * 4 + q;
                    if (c < ncol) dst[(long)k * a.s + c] = acc[r][q];
                }
        }
    }
}

template <typename T, int R, int MODE>
void launch_r(const AxisArgs<T> &a, int ncomp, cudaStream_t stream) {
    constexpr int P = Pitch<T>::v;
    const size_t smem = ((size_t)a.n * P + (size_t)16 * R * (JC + 1)) * sizeof(T);
    static bool configured = false;  // per instantiation; attribute is per-function
    if (!configured) {  // room for the longest axis, 256
        const size_t most = ((size_t)256 * P + (size_t)16 * R * (JC + 1)) * sizeof(T);
        BINDER_CUDA(cudaFuncSetAttribute(axis_kernel<T, R, MODE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most));
        configured = true;
    }
    const bool contig = (a.s == 1);
    const long gx = contig ? (a.outer + TC - 1) / TC : a.outer * ((a.s + TC - 1) / TC);
    BINDER_CHECK(gx < (1L << 31), "transform grid too large");
    dim3 grid((unsigned)gx, (unsigned)((a.n + 16 * R - 1) / (16 * R)), (unsigned)ncomp);
    count_launch(), axis_kernel<T, R, MODE><<<grid, kThreads, smem, stream>>>(a);
    BINDER_CUDA(cudaGetLastError());
}

template <typename T, int MODE>
void launch_mode(const AxisArgs<T> &a, int ncomp, cudaStream_t stream) {
    const int n = a.n;
    if constexpr (std::is_same<T, double>::value &&
                  (MODE == kEpiNone || MODE == kEpiTopoOut || MODE == kEpiPoissonFwd)) {
        // FP64 passes of a small image fill a few CTAs: split the rows into 16-row blocks
        const long gx = a.s == 1 ? (a.outer + TC - 1) / TC : a.outer * ((a.s + TC - 1) / TC);
        if (n > 16 && gx * ncomp < 148) return launch_r<T, 1, MODE>(a, ncomp, stream);
    }
    if (n <= 32)
        launch_r<T, 2, MODE>(a, ncomp, stream);
    else if (n <= 64)
        launch_r<T, 4, MODE>(a, ncomp, stream);
    else if (n <= 128)
        launch_r<T, 8, MODE>(a, ncomp, stream);
    else if (n <= 192)
        launch_r<T, 12, MODE>(a, ncomp, stream);
    else
        launch_r<T, 16, MODE>(a, ncomp, stream);
}

}  // namespace

template <typename T>
void launch_axis_pass(const AxisArgs<T> &a, int mode, int ncomp, cudaStream_t stream) {
    BINDER_CHECK(a.n >= 1 && a.n <= 256, "transform axis length must be in [1, 256]");
    switch (mode) {
        case kEpiNone: launch_mode<T, kEpiNone>(a, ncomp, stream); break;
        case kEpiSpectral:
            if constexpr (std::is_same<T, float>::value) launch_mode<T, kEpiSpectral>(a, ncomp, stream);
            break;
        case kEpiPositions:
            if constexpr (std::is_same<T, float>::value) launch_mode<T, kEpiPositions>(a, ncomp, stream);
            break;
        case kEpiPoisson:
            if constexpr (std::is_same<T, double>::value) launch_mode<T, kEpiPoisson>(a, ncomp, stream);
            break;
        case kEpiTopoOut:
            if constexpr (std::is_same<T, double>::value) launch_mode<T, kEpiTopoOut>(a, ncomp, stream);
            break;
        case kEpiPoissonFwd:
            if constexpr (std::is_same<T, double>::value)
                launch_mode<T, kEpiPoissonFwd>(a, ncomp, stream);
            break;
        default: BINDER_CHECK(false, "unknown transform epilogue");
    }
}

template void launch_axis_pass<float>(const AxisArgs<float> &, int, int, cudaStream_t);
template void launch_axis_pass<double>(const AxisArgs<double> &, int, int, cudaStream_t);

void dct2_matrix(int n, double *out) {
    // each size is built once per process (n^2 cosines: about 1.4 ms for the three axes of a
    // 160 x 192 x 160 grid, paid by every new registration otherwise) and copied from then on
    static std::mutex mu;
    static std::map<int, std::vector<double>> built;
    std::lock_guard<std::mutex> lock(mu);
    std::vector<double> &C = built[n];
    if (C.empty()) {
        C.resize((size_t)n * n);
        const double pi = 3.14159265358979323846;
        for (int k = 0; k < n; ++k) {
            const double s = (k == 0) ? std::sqrt(1.0 / n) : std::sqrt(2.0 / n);
            for (int j = 0; j < n; ++j) {
                const long m = ((long)(2 * j + 1) * k) % (4L * n);
                C[(size_t)k * n + j] = s * std::cos(pi * (double)m / (2.0 * n));
            }
        }
    }
    std::copy(C.begin(), C.end(), out);
}

void hartley_matrix(int n, double *out) {
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j) {
            const long m = ((long)j * k) % n;
            const double ang = 2.0 * pi * (double)m / n;
            out[(long)k * n + j] = std::cos(ang) + std::sin(ang);
        }
}

namespace {
__global__ void prior_noise_kernel(float *noise, long V, int ncomp, int chain_comps,
                                   uint64_t seed, uint32_t chain0, const DevState *st,
                                   const int *skip) {
    if (skip && *skip) return;
    const int per = chain_comps ? chain_comps : ncomp;  // components per chain
    const int chains = ncomp / per;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < V * chains;
         q += (long)gridDim.x * blockDim.x) {
        const int ch = (int)(q / V);
        const uint32_t i = (uint32_t)(q - (long)ch * V);
        const uint32_t sweep = (uint32_t)st[chain_comps ? ch : 0].sweep;
        const uint32_t chain = chain0 + (uint32_t)(chain_comps ? ch : 0);
        float *out = noise + (long)ch * per * V + i;
        // components 0 and 1: the cosine and the sine of one Box-Muller pair (tag 2)
        const u32x4 r = philox_draw(seed, i, sweep, 2u, chain);
        const float u1 = u01_f24(r.x), u2 = u01_f24(r.y);
        const float rad = sqrtf(-2.0f * logf(u1));
        float sn, cs;
        sincospif(2.0f * u2, &sn, &cs);
        out[0] = rad * cs;
        if (per > 1) out[V] = rad * sn;
        if (per > 2) out[2 * V] = dct_prior_normal(seed, i, sweep, chain, 2);
    }
}
}  // namespace

void launch_prior_noise(float *noise, long V, int ncomp, int chain_comps, uint64_t seed,
                        uint32_t chain, const DevState *st, const int *skip, cudaStream_t s) {
    const int per = chain_comps ? chain_comps : ncomp;
    BINDER_CHECK(per >= 1 && per <= 3 && ncomp % per == 0, "noise components");
    long b = (V * (ncomp / per) + 255) / 256;
    b = b < 1 ? 1 : (b > 148L * 16 ? 148L * 16 : b);
    count_launch(), prior_noise_kernel<<<(int)b, 256, 0, s>>>(noise, V, ncomp, chain_comps, seed,
                                                             chain, st, skip);
    BINDER_CUDA(cudaGetLastError());
}

}  // namespace binder
