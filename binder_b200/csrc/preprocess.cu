// Preprocessing and output steps on the GPU; see preprocess.cuh.
//
// The binning reproduces numpy's arithmetic operation by operation in the signal's type: the
// histogram's edges (np.linspace in T), its bin index ((x - first) / (last - first) * 1000,
// truncated, then corrected against the edges), the cumulative distribution (host, sequential,
// as np.cumsum), and the final floor((x - lo) / width).  The kernels use explicitly rounded
// intrinsics so no contraction changes a result.
#include <cmath>
#include <cstring>
#include <vector>

#include "layout.cuh"
#include "preprocess.cuh"

namespace binder {

namespace {

constexpr int kHistBins = 1000;  // the internal histogram of bin_signal_robust

int blocks(long work) {
    int dev = 0, sms = 148;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long need = (work + 255) / 256;
    const long cap = (long)sms * 8;
    return (int)(need < 1 ? 1 : (need < cap ? need : cap));
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

// exactly rounded arithmetic in T
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// order-preserving integer keys of floating-point values (for atomic min / max)
__device__ __forceinline__ unsigned long long okey(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double from_okey(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    double v;
    std::memcpy(&v, &b, sizeof v);
    return v;
}

struct MinMax {
    unsigned long long mn, mx;
};

// min and max of the signal (each value widened to double exactly, so the order is T's order)
template <typename T>
__global__ void minmax_kernel(const T *x, long n, MinMax *r) {
    double lo = INFINITY, hi = -INFINITY;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const double v = (double)x[i];
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&r->mn, okey(lo));
        atomicMax(&r->mx, okey(hi));
    }
}

// numpy.histogram(x, 1000) counts with its uniform-bin index computation and edge corrections
template <typename T>
__global__ void hist_kernel(const T *x, long n, const T *edges, T first, T denom,
                            unsigned long long *counts) {
    __shared__ unsigned int h[kHistBins];
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) h[i] = 0u;
    __syncthreads();
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const T v = x[i];
        const T f = mul_rn(div_rn(sub_rn(v, first), denom), (T)kHistBins);
        long idx = (long)f;
        if (idx == kHistBins) idx -= 1;
        if (idx < 0) idx = 0;                        // v is never below `first`
        if (idx > kHistBins - 1) idx = kHistBins - 1;
        if (v < edges[idx]) idx -= 1;
        if (idx < kHistBins - 1 && v >= edges[idx + 1]) idx += 1;
        if (idx >= 0) atomicAdd(&h[idx], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
        if (h[i]) atomicAdd(&counts[i], (unsigned long long)h[i]);
}

template <typename T>
__global__ void robust_bin_kernel(const T *x, long n, T lo, T hi, T width, int nb, int32_t *out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const T v = x[i];
        int32_t b;
        if (v < lo)
            b = 0;
        else if (v > hi)
            b = nb - 1;
        else
            b = (int32_t)floor(div_rn(sub_rn(v, lo), width));
        out[i] = b;
    }
}

template <typename T>
__global__ void plain_bin_kernel(const T *x, long n, T mn, T width, int32_t *out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        out[i] = (int32_t)rint(div_rn(sub_rn(x[i], mn), width));  // half to even, as np.round
}

// np.linspace(start, stop, num) computed in T: i * ((stop - start) / (num - 1)) + start, last
// value = stop
template <typename T>
std::vector<T> linspace_t(T start, T stop, int num) {
    std::vector<T> y(num);
    const T div = (T)(num - 1);
    const T step = (T)(stop - start) / div;
    for (int i = 0; i < num; ++i) {
        volatile T prod = (T)i * step;  // two roundings, as numpy's y * step then y += start
        y[i] = (T)(prod + start);
    }
    if (num > 1) y[num - 1] = stop;
    return y;
}

template <typename T>
void minmax(const T *dx, long n, cudaStream_t s, T *mn, T *mx) {
    DBuf<MinMax> r(1, s);
    MinMax h{~0ull, 0ull};
    BINDER_CUDA(cudaMemcpyAsync(r.p, &h, sizeof h, cudaMemcpyHostToDevice, s));
    count_launch(), minmax_kernel<T><<<blocks(n), 256, 0, s>>>(dx, n, r.p);
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaMemcpyAsync(&h, r.p, sizeof h, cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    *mn = (T)from_okey(h.mn);
    *mx = (T)from_okey(h.mx);
}

// run f(stream) with the signal on the device (copied when it is host memory) and the binned
// output written through `binned` (host or device)
struct Stream {
    cudaStream_t s = nullptr;
    Stream() { BINDER_CUDA(cudaStreamCreate(&s)); }
    ~Stream() {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
};

}  // namespace

template <typename T>
void bin_signal_robust(const T *signal, long n, int number_of_bins, double lower_percentile,
                       double higher_percentile, int32_t *binned, double *edges) {
    BINDER_CHECK(n > 0, "the signal is empty");
    BINDER_CHECK(number_of_bins >= 2, "number_of_bins must be at least 2");
    Stream st;
    const cudaStream_t s = st.s;
    DBuf<T> dx(n, s);
    DBuf<int32_t> db(n, s);
    BINDER_CUDA(cudaMemcpyAsync(dx.p, signal, sizeof(T) * n, cudaMemcpyDefault, s));
    T first, last;
    minmax(dx.p, n, s, &first, &last);
    BINDER_CHECK(std::isfinite((double)first) && std::isfinite((double)last),
                 "the signal holds non-finite values");
    if (first == last) {  // numpy widens an empty range by 0.5 each side
        first = (T)(first - (T)0.5);
        last = (T)(last + (T)0.5);
    }
    const std::vector<T> he = linspace_t<T>(first, last, kHistBins + 1);
    DBuf<T> de(kHistBins + 1, s);
    DBuf<unsigned long long> dc(kHistBins, s);
    BINDER_CUDA(cudaMemcpyAsync(de.p, he.data(), sizeof(T) * (kHistBins + 1),
                                cudaMemcpyHostToDevice, s));
    BINDER_CUDA(cudaMemsetAsync(dc.p, 0, sizeof(unsigned long long) * kHistBins, s));
    const T denom = (T)(last - first);
    count_launch(), hist_kernel<T><<<blocks(n), 256, 0, s>>>(dx.p, n, de.p, first, denom, dc.p);
    BINDER_CUDA(cudaGetLastError());
    std::vector<unsigned long long> counts(kHistBins);
    BINDER_CUDA(cudaMemcpyAsync(counts.data(), dc.p, sizeof(unsigned long long) * kHistBins,
                                cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    // cumsum(histogram / sum(histogram)) in FP64, sequentially
    double total = 0.0;
    for (unsigned long long c : counts) total += (double)c;
    std::vector<double> cdf(kHistBins);
    double acc = 0.0;
    for (int i = 0; i < kHistBins; ++i) {
        acc += (double)counts[i] / total;
        cdf[i] = acc;
    }
    // the last internal edge whose cumulative share is <= the percentile (raised by 0.01 steps
    // while none is)
    auto robust = [&](double p) {
        double add = 0.01, lim = p;
        for (int guard = 0; guard < 100000; ++guard) {
            int idx = -1;
            for (int i = 0; i < kHistBins; ++i)
                if (cdf[i] <= lim) idx = i;
            if (idx >= 0) return he[idx];
            lim = p + add;
            add = add + 0.01;
        }
        throw Error(kInvalidArgument, "no histogram bin reaches the percentile");
    };
    const T lo = robust(lower_percentile);
    const T hi = robust(higher_percentile);
    BINDER_CHECK(hi > lo, "the robust range of the signal is empty (a constant image?)");
    const T width = (T)((T)(hi - lo) / (T)(number_of_bins - 1));
    count_launch(), robust_bin_kernel<T><<<blocks(n), 256, 0, s>>>(dx.p, n, lo, hi, width,
                                                                   number_of_bins, db.p);
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaMemcpyAsync(binned, db.p, sizeof(int32_t) * n, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    if (edges) {
        const std::vector<T> e = linspace_t<T>(lo, hi, number_of_bins + 1);
        for (int i = 0; i <= number_of_bins; ++i) edges[i] = (double)e[i];
    }
}

template <typename T>
void bin_signal(const T *signal, long n, int number_of_bins, int32_t *binned) {
    BINDER_CHECK(n > 0, "the signal is empty");
    BINDER_CHECK(number_of_bins >= 2, "number_of_bins must be at least 2");
    Stream st;
    const cudaStream_t s = st.s;
    DBuf<T> dx(n, s);
    DBuf<int32_t> db(n, s);
    BINDER_CUDA(cudaMemcpyAsync(dx.p, signal, sizeof(T) * n, cudaMemcpyDefault, s));
    T mn, mx;
    minmax(dx.p, n, s, &mn, &mx);
    BINDER_CHECK(std::isfinite((double)mn) && std::isfinite((double)mx),
                 "the signal holds non-finite values");
    BINDER_CHECK(mx > mn, "the signal is constant");
    const T width = (T)((T)(mx - mn) / (T)(number_of_bins - 1));
    count_launch(), plain_bin_kernel<T><<<blocks(n), 256, 0, s>>>(dx.p, n, mn, width, db.p);
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaMemcpyAsync(binned, db.p, sizeof(int32_t) * n, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
}

template void bin_signal_robust<float>(const float *, long, int, double, double, int32_t *,
                                       double *);
template void bin_signal_robust<double>(const double *, long, int, double, double, int32_t *,
                                        double *);
template void bin_signal<float>(const float *, long, int, int32_t *);
template void bin_signal<double>(const double *, long, int, int32_t *);

// ---- centre of mass ------------------------------------------------------------------------
namespace {
struct ComSums {
    unsigned long long count, sx, sy, sz;
};
__global__ void com_kernel(const int32_t *b, int nx, int ny, int nz, ComSums *r) {
    const long V = (long)nx * ny * nz;
    unsigned long long c = 0, sx = 0, sy = 0, sz = 0;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        if (b[p] > 0) {
            const long x = p / ((long)ny * nz), y = (p / nz) % ny, z = p % nz;
            c += 1;
            sx += (unsigned long long)x;
            sy += (unsigned long long)y;
            sz += (unsigned long long)z;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(0xffffffffu, c, o);
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sz += __shfl_xor_sync(0xffffffffu, sz, o);
    }
    if ((threadIdx.x & 31) == 0 && c) {
        atomicAdd(&r->count, c);
        atomicAdd(&r->sx, sx);
        atomicAdd(&r->sy, sy);
        atomicAdd(&r->sz, sz);
    }
}
}  // namespace

bool center_of_mass_nonzero(const int32_t *bins, int nx, int ny, int nz, double out[3]) {
    BINDER_CHECK(nx > 0 && ny > 0 && nz > 0, "grid dimensions must be positive");
    const long V = (long)nx * ny * nz;
    Stream st;
    const cudaStream_t s = st.s;
    DBuf<int32_t> db(V, s);
    DBuf<ComSums> dr(1, s);
    BINDER_CUDA(cudaMemcpyAsync(db.p, bins, sizeof(int32_t) * V, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaMemsetAsync(dr.p, 0, sizeof(ComSums), s));
    count_launch(), com_kernel<<<blocks(V), 256, 0, s>>>(db.p, nx, ny, nz, dr.p);
    BINDER_CUDA(cudaGetLastError());
    ComSums h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, dr.p, sizeof h, cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    if (h.count == 0) return false;
    // the integer sums are exact, so each coordinate is one correctly rounded division
    out[0] = (double)h.sx / (double)h.count;
    out[1] = (double)h.sy / (double)h.count;
    out[2] = (double)h.sz / (double)h.count;
    return true;
}

// ---- output warping ------------------------------------------------------------------------
namespace {
__device__ __forceinline__ double at(const double *im, int nx, int ny, int nz, long x, long y,
                                     long z) {
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0.0;  // constant 0
    return im[(x * ny + y) * nz + z];
}

__global__ void warp_kernel(const double *im, int nx, int ny, int nz, const double *pos, long M,
                            int order, double *out) {
    for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < M;
         m += (long)gridDim.x * blockDim.x) {
        const double cx = pos[m * 3], cy = pos[m * 3 + 1], cz = pos[m * 3 + 2];
        double v = 0.0;
        if (!(isfinite(cx) && isfinite(cy) && isfinite(cz))) {
            v = 0.0;
        } else if (order == 0) {
            v = at(im, nx, ny, nz, (long)floor(cx + 0.5), (long)floor(cy + 0.5),
                   (long)floor(cz + 0.5));
        } else {
            const double fx = floor(cx), fy = floor(cy), fz = floor(cz);
            const double tx = cx - fx, ty = cy - fy, tz = cz - fz;
            const long x0 = (long)fx, y0 = (long)fy, z0 = (long)fz;
            const double wx[2] = {1.0 - tx, tx}, wy[2] = {1.0 - ty, ty}, wz[2] = {1.0 - tz, tz};
            double acc = 0.0;
            for (int i = 0; i < 2; ++i) {
                double ay = 0.0;
                for (int j = 0; j < 2; ++j) {
                    double az = 0.0;
                    for (int k = 0; k < 2; ++k)
                        az = fma(wz[k], at(im, nx, ny, nz, x0 + i, y0 + j, z0 + k), az);
                    ay = fma(wy[j], az, ay);
                }
                acc = fma(wx[i], ay, acc);
            }
            v = acc;
        }
        out[m] = v;
    }
}

// ---- order 3: cubic B-spline interpolation (scipy.ndimage.map_coordinates, order 3, mode
// 'grid-constant', prefilter on).  The image is padded by kSplinePad zero samples on every side,
// the padded array is converted to cubic B-spline coefficients by the recursive filter of Unser,
// Aldroubi and Eden ("B-spline signal processing", IEEE Trans. Signal Process. 41, 1993): per
// line, gain 6, a causal pass from a truncated mirror-symmetric start, an anti-causal pass from
// the mirror-symmetric end condition, pole z = sqrt(3) - 2.  An output sample is the 64-tap
// cubic B-spline sum of the coefficients around its position; taps outside the padded array
// read 0.  Zero padding makes the boundary condition of the filter immaterial to FP64 precision
// (its influence decays as |z|^12 before reaching the image and again before returning).
constexpr int kSplinePad = 12;
constexpr double kPole3 = -0.267949192431122706472553658494127633;  // sqrt(3) - 2

__global__ void pad_kernel(const double *im, int nx, int ny, int nz, double *c, int qx, int qy,
                           int qz) {
    const long n = (long)qx * qy * qz;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const long Z = i % qz, r = i / qz, Y = r % qy, X = r / qy;
        const long x = X - kSplinePad, y = Y - kSplinePad, z = Z - kSplinePad;
        c[i] = (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz)
                   ? im[(x * ny + y) * nz + z]
                   : 0.0;
    }
}

// one thread per line of length n (n >= 3) and element stride s: lines (o, t), o < outer, t < s,
// element k at o * n * s + t + k * s; in place
__global__ void spline_line_kernel(double *c, long outer, int n, long s) {
    const long nlines = outer * s;
    for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < nlines;
         l += (long)gridDim.x * blockDim.x) {
        const long o = l / s, t = l - o * s;
        double *p = c + o * (long)n * s + t;
        const double z = kPole3;
        // causal start: sum_k z^k c[k] over the terms above double precision
        const int h = n < 40 ? n : 40;
        double acc = 0.0, zk = 1.0;
        for (int k = 0; k < h; ++k) {
            acc = fma(zk, 6.0 * p[(long)k * s], acc);
            zk *= z;
        }
        double prev = acc;
        p[0] = prev;
        for (int k = 1; k < n; ++k) {
            prev = fma(z, prev, 6.0 * p[(long)k * s]);
            p[(long)k * s] = prev;
        }
        // anti-causal start from the last two causal values, then backwards in place
        double next = (z / (z * z - 1.0)) * (prev + z * p[(long)(n - 2) * s]);
        p[(long)(n - 1) * s] = next;
        for (int k = n - 2; k >= 0; --k) {
            next = z * (next - p[(long)k * s]);
            p[(long)k * s] = next;
        }
    }
}

__device__ __forceinline__ void bspline3_d(double t, double w[4]) {
    const double e = 1.0 - t;
    w[0] = e * e * e * (1.0 / 6.0);
    w[1] = (2.0 / 3.0) - t * t + 0.5 * t * t * t;
    w[2] = (2.0 / 3.0) - e * e + 0.5 * e * e * e;
    w[3] = t * t * t * (1.0 / 6.0);
}

__global__ void warp3_kernel(const double *c, int qx, int qy, int qz, const double *pos, long M,
                             double *out) {
    for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < M;
         m += (long)gridDim.x * blockDim.x) {
        const double cx = pos[m * 3] + kSplinePad, cy = pos[m * 3 + 1] + kSplinePad,
                     cz = pos[m * 3 + 2] + kSplinePad;
        double v = 0.0;
        // non-finite, or every tap outside the padded array: the fill value
        const bool near = cx > -3.0 && cy > -3.0 && cz > -3.0 && cx < qx + 2.0 &&
                          cy < qy + 2.0 && cz < qz + 2.0;
        if (near) {
            const double fx = floor(cx), fy = floor(cy), fz = floor(cz);
            double wx[4], wy[4], wz[4];
            bspline3_d(cx - fx, wx);
            bspline3_d(cy - fy, wy);
            bspline3_d(cz - fz, wz);
            const int bx = (int)fx - 1, by = (int)fy - 1, bz = (int)fz - 1;
            for (int i = 0; i < 4; ++i) {
                const int X = bx + i;
                if (X < 0 || X >= qx) continue;
                double ay = 0.0;
                for (int j = 0; j < 4; ++j) {
                    const int Y = by + j;
                    if (Y < 0 || Y >= qy) continue;
                    const double *row = c + ((long)X * qy + Y) * qz;
                    double az = 0.0;
                    for (int k = 0; k < 4; ++k) {
                        const int Zi = bz + k;
                        if (Zi >= 0 && Zi < qz) az = fma(wz[k], row[Zi], az);
                    }
                    ay = fma(wy[j], az, ay);
                }
                v = fma(wx[i], ay, v);
            }
        }
        out[m] = v;
    }
}

__global__ void clip_kernel(double *out, long M, double lo, double hi) {
    for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < M;
         m += (long)gridDim.x * blockDim.x)
        out[m] = fmin(fmax(out[m], lo), hi);
}
}  // namespace

void warp_image(const double *image, int nx, int ny, int nz, const double *positions, long M,
                int order, double *out) {
    BINDER_CHECK(nx > 0 && ny > 0 && nz > 0 && M > 0, "sizes must be positive");
    BINDER_CHECK(order == 0 || order == 1 || order == 3, "interpolation order must be 0, 1 or 3");
    const long V = (long)nx * ny * nz;
    Stream st;
    const cudaStream_t s = st.s;
    DBuf<double> di(V, s), dp(M * 3, s), dout(M, s);
    BINDER_CUDA(cudaMemcpyAsync(di.p, image, sizeof(double) * V, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaMemcpyAsync(dp.p, positions, sizeof(double) * M * 3, cudaMemcpyDefault, s));
    if (order == 3) {
        const int qx = nx + 2 * kSplinePad, qy = ny + 2 * kSplinePad, qz = nz + 2 * kSplinePad;
        const long Q = (long)qx * qy * qz;
        DBuf<double> dc(Q, s);
        count_launch(), pad_kernel<<<blocks(Q), 256, 0, s>>>(di.p, nx, ny, nz, dc.p, qx, qy, qz);
        BINDER_CUDA(cudaGetLastError());
        // x and y lines: neighbouring threads take neighbouring z, so every access is coalesced;
        // z lines are contiguous per thread
        count_launch(), spline_line_kernel<<<blocks((long)qy * qz), 256, 0, s>>>(
            dc.p, 1, qx, (long)qy * qz);
        count_launch(), spline_line_kernel<<<blocks((long)qx * qz), 256, 0, s>>>(dc.p, qx, qy,
                                                                                   qz);
        count_launch(), spline_line_kernel<<<blocks((long)qx * qy), 256, 0, s>>>(
            dc.p, (long)qx * qy, qz, 1);
        count_launch(), warp3_kernel<<<blocks(M), 256, 0, s>>>(dc.p, qx, qy, qz, dp.p, M,
                                                               dout.p);
        BINDER_CUDA(cudaGetLastError());
        // dc is released on s after the interpolation
    } else {
        count_launch(), warp_kernel<<<blocks(M), 256, 0, s>>>(di.p, nx, ny, nz, dp.p, M, order,
                                                              dout.p);
        BINDER_CUDA(cudaGetLastError());
    }
    // skimage clips the output to the input's range, widened to the fill value 0 when 0 lies
    // outside that range but inside the output's
    double imn, imx, omn, omx;
    minmax(di.p, V, s, &imn, &imx);
    minmax(dout.p, M, s, &omn, &omx);
    double lo = imn, hi = imx;
    const bool preserve_cval = !(imn <= 0.0 && 0.0 <= imx) && omn <= 0.0 && 0.0 <= omx;
    if (preserve_cval) {
        lo = lo < 0.0 ? lo : 0.0;
        hi = hi > 0.0 ? hi : 0.0;
    }
    count_launch(), clip_kernel<<<blocks(M), 256, 0, s>>>(dout.p, M, lo, hi);
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaMemcpyAsync(out, dout.p, sizeof(double) * M, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
}

}  // namespace binder
