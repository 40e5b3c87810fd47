// E-step kernels (EM soft assignment and Gibbs categorical draw), theta updates, Dirichlet and
// gamma-prior sampling, EM bookkeeping and FP64 Welford moments.
#include <cuda_fp16.h>

#include <cmath>
#include <type_traits>

#include "estep.cuh"

namespace binder {

namespace {

constexpr int kEThreads = 256;

// cubic B-spline weights for node offsets -1, 0, 1, 2 at fraction t in [0,1)
// (BINDER/src/cpu/Spline.cpp:44-73; Registration.cu:20-31 evaluates the same polynomial)
__device__ __forceinline__ void bspline3(float t, float w[4]) {
    const float t2 = t * t, t3 = t2 * t;
    const float e = 1.0f - t, e2 = e * e, e3 = e2 * e;
    w[0] = e3 * (1.0f / 6.0f);
    w[1] = (2.0f / 3.0f) - t2 + 0.5f * t3;
    w[2] = (2.0f / 3.0f) - e2 + 0.5f * e3;
    w[3] = t3 * (1.0f / 6.0f);
}

// base node index of position p and its four weights on the node offsets -1, 0, 1, 2 for spline
// order 1, 2 or 3 (BINDER/src/cpu/Spline.cpp:9-41 and :44-123): order 3 around floor(p); order
// 2 around floor(p + 0.5) on the offsets -1, 0, 1; order 1 around floor(p) on the offsets 0, 1.
// The unused taps carry weight 0, so they add nothing to the posterior, the histogram or the
// dream location.
__device__ __forceinline__ int spline_setup(float p, int order, float w[4]) {
    if (order == 2) {
        const float f = floorf(p + 0.5f), d = p - f;
        const float a = -2.0f * d + 1.0f, b = -2.0f * d - 1.0f;
        w[0] = 0.125f * (a * a);
        w[1] = 0.75f - d * d;
        w[2] = 0.125f * (b * b);
        w[3] = 0.0f;
        return (int)f;
    }
    const float f = floorf(p), d = p - f;
    if (order == 1) {
        w[0] = 0.0f;
        w[1] = 1.0f - d;
        w[2] = d;
        w[3] = 0.0f;
    } else {
        bspline3(d, w);
    }
    return (int)f;
}

// Bins of the 4 x 4 x 4 (3D) or 4 x 4 (2D) neighbourhood, packed 4 per word along the last axis.
// A 2D image is handled as an nx x 1 x ny volume: its y axis plays the packed (z) role and there
// is a single node row per x, so DIM == 2 gathers 4 words (x rows) and DIM == 3 gathers 16
// ((x, y) rows).  Fast path: two aligned 32-bit loads per row from the zero-padded bin volume and
// a funnel shift; the padding is bin 0, which is the reference's value for nodes outside the
// moving grid (MILikelihood.cpp:46-48).  Slow path (neighbourhood leaves the padded volume):
// per-node test.
template <int DIM>
__device__ __forceinline__ void gather_bins(const EStepArgs &a, int ix, int iy, int iz,
                                            uint32_t (&pk)[DIM == 3 ? 16 : 4]) {
    constexpr int Q = DIM == 3 ? 4 : 1;
    const int zz0 = iz - 1 + a.PZ;
    const int Py = DIM == 3 ? a.P : 0;
    const int y0 = DIM == 3 ? iy - 1 : 0;
    const bool fast = (ix - 1 + a.P >= 0) && (ix + 2 + a.P < a.nxn + 2 * a.P) &&
                      (DIM == 2 || ((iy - 1 + a.P >= 0) && (iy + 2 + a.P < a.nyn + 2 * a.P))) &&
                      (zz0 >= 0) && ((zz0 >> 2) + 2 <= (a.zp >> 2));
    if (fast) {
        const int w = zz0 >> 2, sh = (zz0 & 3) * 8;
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const uint32_t *row = reinterpret_cast<const uint32_t *>(
                    a.vpad + ((long)(ix - 1 + p + a.P) * a.pyn + (y0 + q + Py)) * a.zp);
                const uint32_t lo = __ldg(row + w), hi = __ldg(row + w + 1);
                pk[p * Q + q] = __funnelshift_r(lo, hi, sh);
            }
    } else {
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                uint32_t word = 0;
                const int X = ix - 1 + p, Y = y0 + q;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int Z = iz - 1 + c;
                    uint32_t b = 0;
                    if (X >= 0 && Y >= 0 && Z >= 0 && X < a.nxn && Y < a.nyn && Z < a.nzn)
                        b = a.vpad[((long)(X + a.P) * a.pyn + (Y + Py)) * a.zp + (Z + a.PZ)];
                    word |= b << (8 * c);
                }
                pk[p * Q + q] = word;
            }
    }
}

// word (p, q) of gather_bins alone: bins of nodes (ix-1+p, iy-1+q, iz-1 .. iz+2) (q = 0 in 2D),
// from the padded bin volume vpad (a.vpad, or one channel's volume of the filter likelihood)
template <int DIM>
__device__ __forceinline__ uint32_t gather_word(const EStepArgs &a, const uint8_t *vpad, int ix,
                                                int iy, int iz, int p, int q) {
    const int zz0 = iz - 1 + a.PZ;
    const int Py = DIM == 3 ? a.P : 0;
    const int X = ix - 1 + p, Y = DIM == 3 ? iy - 1 + q : 0;
    const bool fast = (X + a.P >= 0) && (X + a.P < a.nxn + 2 * a.P) &&
                      (DIM == 2 || ((Y + a.P >= 0) && (Y + a.P < a.nyn + 2 * a.P))) &&
                      (zz0 >= 0) && ((zz0 >> 2) + 2 <= (a.zp >> 2));
    if (fast) {
        const uint32_t *rowp = reinterpret_cast<const uint32_t *>(
            vpad + ((long)(X + a.P) * a.pyn + (Y + Py)) * a.zp);
        const int w = zz0 >> 2, sh = (zz0 & 3) * 8;
        return __funnelshift_r(__ldg(rowp + w), __ldg(rowp + w + 1), sh);
    }
    uint32_t word = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int Z = iz - 1 + c;
        uint32_t b = 0;
        if (X >= 0 && Y >= 0 && Z >= 0 && X < a.nxn && Y < a.nyn && Z < a.nzn)
            b = vpad[((long)(X + a.P) * a.pyn + (Y + Py)) * a.zp + (Z + a.PZ)];
        word |= b << (8 * c);
    }
    return word;
}

// One voxel's position and spline setup, shared by the E-step kernels.  Positions are SoA [N][V]
// (N = DIM); in 2D the second component is the packed-axis position (z role) and y is absent.
// Returns false for a degenerate position (outside any grid or not finite).
template <int DIM>
struct VoxelPos {
    float px, py, pz;     // position (py = 0 in 2D)
    float x0, x1, x2;     // voxel grid position
    // pos_off: elements from a.d to this chain's positions (a batch of chains; 0 otherwise)
    __device__ __forceinline__ bool load(const EStepArgs &a, unsigned i, unsigned V, unsigned ny,
                                         unsigned nz, long pos_off = 0) {
        const float *d = a.d + pos_off;
        px = d[i];
        py = DIM == 3 ? d[V + i] : 0.0f;
        pz = d[(size_t)(DIM - 1) * V + i];
        if (a.x) {
            x0 = a.x[i];
            x1 = DIM == 3 ? a.x[V + i] : 0.0f;
            x2 = a.x[(size_t)(DIM - 1) * V + i];
        } else {
            const unsigned row = i / nz;
            x2 = (float)(i - row * nz);
            const unsigned xi = row / ny;
            x1 = (float)(row - xi * ny);
            x0 = (float)xi;
        }
        return fabsf(px) < 1.0e6f && (DIM == 2 || fabsf(py) < 1.0e6f) && fabsf(pz) < 1.0e6f;
    }
    // r = dream location - voxel position, components (x, [y,] z-role)
    __device__ __forceinline__ void store_r(const EStepArgs &a, unsigned i, unsigned V, float vx,
                                            float vy, float vz, long pos_off = 0) const {
        float *r = a.r + pos_off;
        r[i] = vx - x0;
        if (DIM == 3) r[V + i] = vy - x1;
        r[(size_t)(DIM - 1) * V + i] = vz - x2;
    }
};

// row pitch (floats) of the shared theta / histogram tables: >= n and 9 banks apart row to row
__host__ __device__ constexpr int theta_pitch(int K) { return K + ((9 - K % 32) + 32) % 32; }

constexpr int kSmallK = 64;  // the single-pass EM kernel keeps a K-bin column per thread
constexpr int kFastThreads = 256;
// the single-pass EM kernel's wide form: one CTA of 24 warps per SM (FP32 columns for 768 threads
// and the tables fill the SM's shared memory, with the tables' rows 5 banks apart so they fit)
constexpr int kWideThreads = 768;
__host__ __device__ constexpr int wide_pitch(int K) { return K + ((5 - K % 32) + 32) % 32; }
template <int TPB>
__host__ __device__ constexpr int fast_pitch(int K) {
    return TPB > kFastThreads ? wide_pitch(K) : theta_pitch(K);
}

// FP16 bin columns (EStepArgs::halfcol): [K][TPB] halves, the thread's entry for bin k at
// col[k * TPB], the same indexing as the FP32 columns (one shift and add per neighbour).  Lanes 2j
// and 2j + 1 share a 32-bit word, so two such lanes updating different bins in one instruction
// meet in a bank (a two-way conflict); a layout pairing bins 2j, 2j + 1 of one thread in a word
// avoids that but costs more integer instructions per neighbour than the conflicts cost.  Each
// mass is rounded to FP16 before it is added, and the sum is held in FP16.
template <int TPB>
__device__ __forceinline__ __half *half_slot(__half *col, int k) {
    return col + k * TPB;
}
// masses w.x, w.y of two neighbours with bins ka, kb (one FP32 to FP16 pair conversion)
template <int TPB>
__device__ __forceinline__ void col_add2(float *__restrict__ col, int ka, int kb, float2 w) {
    col[ka * TPB] += w.x;
    col[kb * TPB] += w.y;
}
template <int TPB>
__device__ __forceinline__ void col_add2(__half *__restrict__ col, int ka, int kb, float2 w) {
    const __half2 h = __float22half2_rn(w);
    __half *p = half_slot<TPB>(col, ka);
    *p = __hadd(*p, __low2half(h));
    __half *q = half_slot<TPB>(col, kb);
    *q = __hadd(*q, __high2half(h));
}
template <int TPB>
__device__ __forceinline__ float col_get(const float *col, int k) { return col[k * TPB]; }
template <int TPB>
__device__ __forceinline__ float col_get(__half *col, int k) {
    return __half2float(*half_slot<TPB>(col, k));
}
template <int TPB>
__device__ __forceinline__ void col_clear(float *col, int k) { col[k * TPB] = 0.0f; }
template <int TPB>
__device__ __forceinline__ void col_clear(__half *col, int k) {
    *half_slot<TPB>(col, k) = __float2half_rn(0.0f);
}

// The node pass of one EM voxel (4 x Q rows of 4 packed nodes; Q = 4 in 3D, 1 in 2D): weights
// w = bx[p] by[q] bz[c] theta[k] added to the thread's private bin column col[k * TPB], their sum
// S, their first moments along each axis (node offset -1 .. 2 times w) and the range of bins
// touched.  theta and the column are disjoint regions of shared memory; the __restrict__
// qualifiers let the compiler hoist the theta loads of later nodes above earlier column updates.
// Products and sums run on paired FP32 lanes (nodes c = 0,1 and c = 2,3 of each packed word).
template <int TPB, int Q, typename CT>
__device__ __forceinline__ void em_accumulate(const float *__restrict__ thu,
                                              CT *__restrict__ col, const uint32_t (&pk)[4 * Q],
                                              const float (&bx)[4], const float (&by)[4],
                                              const float (&bz)[4], float &S, float &Sx, float &Sy,
                                              float &Sz, int &kmin, int &kmax) {
    const float2 bz01 = make_float2(bz[0], bz[1]), bz23 = make_float2(bz[2], bz[3]);
    const float2 m1 = make_float2(-1.0f, -1.0f), p2 = make_float2(2.0f, 2.0f);
    float2 a01 = make_float2(0.f, 0.f), a23 = a01;  // sum of w
    float2 x01 = a01, x23 = a01;                    // sum of (p - 1) w
    float2 y01 = a01, y23 = a01;                    // sum of (q - 1) w
    int lo = 255, hi = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float bxy = Q == 4 ? bx[p] * by[q] : bx[p];
            const float2 bb = make_float2(bxy, bxy);
            const float2 b01 = __fmul2_rn(bb, bz01), b23 = __fmul2_rn(bb, bz23);
            const uint32_t word = pk[p * Q + q];
            const int k0 = word & 0xff, k1 = (word >> 8) & 0xff, k2 = (word >> 16) & 0xff,
                      k3 = word >> 24;
            const float2 w01 = __fmul2_rn(b01, make_float2(thu[k0], thu[k1]));
            const float2 w23 = __fmul2_rn(b23, make_float2(thu[k2], thu[k3]));
            col_add2<TPB>(col, k0, k1, w01);
            col_add2<TPB>(col, k2, k3, w23);
            a01 = __fadd2_rn(a01, w01);
            a23 = __fadd2_rn(a23, w23);
            if (p == 0) { x01 = __ffma2_rn(m1, w01, x01); x23 = __ffma2_rn(m1, w23, x23); }
            if (p == 2) { x01 = __fadd2_rn(x01, w01); x23 = __fadd2_rn(x23, w23); }
            if (p == 3) { x01 = __ffma2_rn(p2, w01, x01); x23 = __ffma2_rn(p2, w23, x23); }
            if (Q == 4) {
                if (q == 0) { y01 = __ffma2_rn(m1, w01, y01); y23 = __ffma2_rn(m1, w23, y23); }
                if (q == 2) { y01 = __fadd2_rn(y01, w01); y23 = __fadd2_rn(y23, w23); }
                if (q == 3) { y01 = __ffma2_rn(p2, w01, y01); y23 = __ffma2_rn(p2, w23, y23); }
            }
            lo = min(min(lo, min(k0, k1)), min(k2, k3));
            hi = max(max(hi, max(k0, k1)), max(k2, k3));
        }
    S = (a01.x + a01.y) + (a23.x + a23.y);
    Sx = (x01.x + x01.y) + (x23.x + x23.y);
    Sy = (y01.x + y01.y) + (y23.x + y23.y);
    Sz = (a23.x - a01.x) + 2.0f * a23.y;  // offsets -1, 0, 1, 2 along the packed axis
    kmin = lo;
    kmax = hi;
}

// em_accumulate in log space (Registration.cpp:331-470): the table entries are log2 likelihoods,
// the spline weights enter as log2 too, and every term is exponentiated relative to the voxel's
// largest term, so no neighbourhood underflows.  mlog returns that largest term (log2).
template <int TPB, int Q>
__device__ __forceinline__ void em_accumulate_log(const float *__restrict__ thu,
                                                  float *__restrict__ col,
                                                  const uint32_t (&pk)[4 * Q],
                                                  const float (&bx)[4], const float (&by)[4],
                                                  const float (&bz)[4], float &S, float &Sx,
                                                  float &Sy, float &Sz, int &kmin, int &kmax,
                                                  float &mlog) {
    float lx[4], ly[4], lz[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        lx[t] = log2f(bx[t]);  // -inf for a zero tap, whose term then vanishes
        ly[t] = Q == 4 ? log2f(by[t]) : 0.0f;
        lz[t] = log2f(bz[t]);
    }
    float m = -INFINITY;
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float lxy = lx[p] + ly[q];
            const uint32_t word = pk[p * Q + q];
#pragma unroll
            for (int c = 0; c < 4; ++c)
                m = fmaxf(m, lxy + lz[c] + thu[(word >> (8 * c)) & 0xff]);
        }
    float a = 0.f, x = 0.f, y = 0.f, z = 0.f;
    int lo = 255, hi = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float lxy = lx[p] + ly[q] - m;
            const uint32_t word = pk[p * Q + q];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int k = (word >> (8 * c)) & 0xff;
                const float w = exp2f(lxy + lz[c] + thu[k]);
                col[k * TPB] += w;
                a += w;
                x = fmaf((float)(p - 1), w, x);
                if (Q == 4) y = fmaf((float)(q - 1), w, y);
                z = fmaf((float)(c - 1), w, z);
                lo = min(lo, k);
                hi = max(hi, k);
            }
        }
    S = a;
    Sx = x;
    Sy = y;
    Sz = z;
    kmin = lo;
    kmax = hi;
    mlog = m;
}

// EM E-step for K <= 64 (BINDER/src/cpu/Registration.cpp:219-330, sample == false), one pass over
// the 64 (3D) or 16 (2D) neighbours.  The posterior mass of a voxel is collected per moving bin k
// in a private shared-memory column hk[k][thread] (bank = thread % 32, so never a conflict and
// never an atomic), while the smallest and largest bin touched are tracked; once the normaliser S
// is known the columns in [kmin, kmax] that hold mass are flushed as hist[k][u] += hk[k] / S --
// one shared atomic per distinct bin instead of one per neighbour (the bin range of a
// neighbourhood is a handful of bins in smooth images).  The CTA histogram is 32-bit fixed point
// (scale a.hscale, chosen by the host so that a cell cannot overflow), which makes every flush a
// native integer shared atomic, and is converted to FP32 once per CTA.  Each contribution is
// rounded to within 0.5 / hscale (3.9e-6 at 127,097, the wide form's scale at 160 x 192 x 160);
// FP32 accumulation of the same sums would round each addition relative to the running sum
// instead.  theta is staged transposed (thT[u][k]); it and the histogram use a row pitch of 9
// (mod 32) banks (5 in the wide form), so lanes whose (u, k) pairs differ by small amounts hit
// different banks.  Voxel indices are 32-bit (V < 2^31 is checked by the host).
//
// HC (EStepArgs::halfcol): the columns hold FP16 (half the shared memory, so three CTAs fit on an SM
// instead of two), theta is staged multiplied by kHalfColScale so that the masses stay well inside
// FP16's normal range, and the log-likelihood takes the scale back out.  S, the moments and the CTA
// histogram stay FP32 / fixed point; only the per-voxel bin sums are rounded to FP16.
constexpr float kHalfColScale = 4096.0f;
constexpr double kLnHalfColScale = 8.317766166719343;  // ln 4096

template <int TPB, int DIM, bool LOGT, bool HC = false>
__global__ void __launch_bounds__(TPB, HC ? 3 : (TPB > kFastThreads ? 1 : 2))
    estep_em_fast_kernel(const EStepArgs a) {
    constexpr int Q = DIM == 3 ? 4 : 1;
    using CT = typename std::conditional<HC, __half, float>::type;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) float sm[];
    const int K = a.K, L = a.L, KL = K * L;
    const int KP = fast_pitch<TPB>(K), LP = fast_pitch<TPB>(L);
    float *thT = sm;                                             // [L][KP]
    unsigned *hs = reinterpret_cast<unsigned *>(sm + L * KP);    // [K][LP] CTA histogram (fixed)
    float *hkw = sm + L * KP + K * LP;  // per-thread bin masses: [K][TPB] FP32 or FP16
    const int hk_words = HC ? ((K + 1) / 2) * TPB : K * TPB;
    float *cmx = hkw + hk_words;                                 // [L] log-space column maxima
    __shared__ double red[32];
    if (LOGT)
        for (int l = threadIdx.x; l < L; l += TPB) cmx[l] = a.colmax[l];
    const float tscale = HC ? kHalfColScale : 1.0f;
    for (int q = threadIdx.x; q < KL; q += TPB) {
        const int k = q / L, l = q - k * L;
        thT[l * KP + k] = a.theta[q] * tscale;
        hs[k * LP + l] = 0u;
    }
    for (int q = threadIdx.x; q < hk_words; q += TPB) hkw[q] = 0.0f;
    __syncthreads();

    CT *my = reinterpret_cast<CT *>(hkw) + threadIdx.x;  // my[k * TPB]
    double mll = 0.0;
    unsigned deg = 0;
    // unsigned: i + stride stays below 2^32 for any V < 2^31
    const unsigned V = (unsigned)a.V, nz = (unsigned)a.nz, ny = (unsigned)a.ny;
    for (unsigned i = blockIdx.x * TPB + threadIdx.x; i < V; i += gridDim.x * TPB) {
        VoxelPos<DIM> vp;
        if (!vp.load(a, i, V, ny, nz)) {
            vp.store_r(a, i, V, vp.px, vp.py, vp.pz);
            ++deg;
            continue;
        }
        float bx[4], by[4] = {1.f, 1.f, 1.f, 1.f}, bz[4];
        const int ix = spline_setup(vp.px, a.order, bx);
        const int iy = DIM == 3 ? spline_setup(vp.py, a.order, by) : 0;
        const int iz = spline_setup(vp.pz, a.order, bz);
        const float fx = (float)ix, fy = (float)iy, fz = (float)iz;
        uint32_t pk[4 * Q];
        gather_bins<DIM>(a, ix, iy, iz, pk);
        const int ui = a.u[i];
        float S, Sx, Sy, Sz;
        int kmin, kmax;
        float mlog = 0.0f;
        if constexpr (LOGT)
            em_accumulate_log<TPB, Q>(thT + ui * KP, my, pk, bx, by, bz, S, Sx, Sy, Sz, kmin,
                                      kmax, mlog);
        else
            em_accumulate<TPB, Q>(thT + ui * KP, my, pk, bx, by, bz, S, Sx, Sy, Sz, kmin, kmax);
        const bool ok = S > 0.0f;
        const float inv = ok ? 1.0f / S : 0.0f;
        const float invs = inv * a.hscale;
        unsigned *hcol = hs + ui;  // hcol[k * LP]
        for (int k = kmin; k <= kmax; ++k) {
            const float m = col_get<TPB>(my, k);
            if (m != 0.0f) {
                if (ok) atomicAdd(&hcol[k * LP], __float2uint_rn(m * invs));
                col_clear<TPB>(my, k);
            }
        }
        if (!ok) {
            vp.store_r(a, i, V, fx, fy, fz);
            ++deg;
            continue;
        }
        mll -= (double)logf(S);  // FP32 log, FP64 accumulation
        if (HC) mll += kLnHalfColScale;
        if (LOGT) mll -= (double)mlog * 0.6931471805599453 + (double)cmx[ui];
        vp.store_r(a, i, V, fx + Sx * inv, fy + Sy * inv, fz + Sz * inv);
    }
    __syncthreads();
    const double m = block_sum(mll, red);
    const double dg = block_sum((double)deg, red);
    if (threadIdx.x == 0 && dg > 0.0) atomicAdd(&a.st->degenerate, (unsigned long long)dg);
    if (!a.hfix) {
        for (int q = threadIdx.x; q < KL; q += TPB) {
            const int k = q / L;
            const unsigned v = hs[k * LP + (q - k * L)];
            if (v) atomicAdd(&a.hist[q], (float)((double)v * a.hinv));
        }
        if (threadIdx.x == 0) atomicAdd(&a.st->mll, m);
        return;
    }
    // Order-independent merge, so that EM is bitwise repeatable: the CTA histograms are integers
    // and their 64-bit global sums are exact whatever order the CTAs arrive in; the last CTA to
    // finish converts the sums to the FP32 histogram (one rounding per cell) and adds the CTAs'
    // log-likelihood partials in CTA order.
    for (int q = threadIdx.x; q < KL; q += TPB) {
        const int k = q / L;
        const unsigned v = hs[k * LP + (q - k * L)];
        if (v) atomicAdd(&a.hfix[q], (unsigned long long)v);
    }
    if (threadIdx.x == 0) a.mpart[blockIdx.x] = m;
    __threadfence();
    __syncthreads();
    __shared__ unsigned last;
    if (threadIdx.x == 0) last = atomicAdd(a.hdone, 1u) == gridDim.x - 1 ? 1u : 0u;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double hinv = a.hinv;
    for (int q = threadIdx.x; q < KL; q += TPB) {
        const unsigned long long v = __ldcg(a.hfix + q);
        if (v) {
            a.hist[q] += (float)((double)v * hinv);
            a.hfix[q] = 0ull;
        }
    }
    double part = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += TPB) part += __ldcg(a.mpart + b);
    const double tot = block_sum(part, red);
    if (threadIdx.x == 0) {
        a.st->mll += tot;
        *a.hdone = 0u;
    }
}

// EM E-step with the MI filter likelihood (BINDER/src/cpu/MILikelihoodFilter.cpp:53-68 and
// :110-124 inside Registration.cpp:219-330): the weight of a neighbour is its spline weight times
// prod_m theta[m][k_m][u_m], the bins of channel m being read at [index + m] -- which the host has
// resolved into one shifted bin volume per channel -- and the posterior mass goes to every
// channel's histogram.  theta [M][L][KP] (transposed per channel) and the histograms [M][K][LP]
// live in shared memory; the second pass recomputes the weights and adds p = w / S with one
// shared atomic per channel and neighbour.
template <int DIM, bool SAMPLE = false>
__global__ void __launch_bounds__(kEThreads, 2) estep_filter_kernel(const EStepArgs a) {
    constexpr int Q = DIM == 3 ? 4 : 1;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) float sm[];
    const int K = a.K, L = a.L, M = a.M;
    const int KP = theta_pitch(K), LP = theta_pitch(L);
    const int KL = K * L;
    float *thT = sm;                        // [M][L][KP]
    float *hs = sm + (size_t)M * L * KP;    // [M][K][LP] EM histogram
    unsigned *hc = reinterpret_cast<unsigned *>(hs);  // sampling: counts
    // sampling: the running sum at the end of node row r, cps[r * kEThreads]
    float *cps = hs + (size_t)M * K * LP + threadIdx.x;
    for (int q = threadIdx.x; q < M * KL; q += blockDim.x) {
        const int m = q / KL, r = q - m * KL, k = r / L, l = r - k * L;
        thT[(m * L + l) * KP + k] = a.theta[q];
        if (SAMPLE) hc[(m * K + k) * LP + l] = 0u; else hs[(m * K + k) * LP + l] = 0.0f;
    }
    __syncthreads();

    const uint32_t sweep = SAMPLE ? (uint32_t)a.st->sweep : 0u;
    double mll = 0.0;
    unsigned deg = 0;
    const unsigned V = (unsigned)a.V, nz = (unsigned)a.nz, ny = (unsigned)a.ny;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        VoxelPos<DIM> vp;
        if (!vp.load(a, i, V, ny, nz)) {
            vp.store_r(a, i, V, vp.px, vp.py, vp.pz);
            ++deg;
            continue;
        }
        float bx[4], by[4] = {1.f, 1.f, 1.f, 1.f}, bz[4];
        const int ix = spline_setup(vp.px, a.order, bx);
        const int iy = DIM == 3 ? spline_setup(vp.py, a.order, by) : 0;
        const int iz = spline_setup(vp.pz, a.order, bz);
        const float fx = (float)ix, fy = (float)iy, fz = (float)iz;
        int um[kMaxChannels];
#pragma unroll
        for (int m = 0; m < kMaxChannels; ++m) um[m] = m < M ? a.u[m * a.uch + i] : 0;
        // pass 1: normaliser and first moments
        float S = 0.0f, Sx = 0.0f, Sy = 0.0f, Sz = 0.0f;
#pragma unroll 1
        for (int p = 0; p < 4; ++p)
#pragma unroll 1
            for (int q = 0; q < Q; ++q) {
                const float bxy = Q == 4 ? bx[p] * by[q] : bx[p];
                float t[4] = {bxy * bz[0], bxy * bz[1], bxy * bz[2], bxy * bz[3]};
#pragma unroll
                for (int m = 0; m < kMaxChannels; ++m) {
                    if (m >= M) break;
                    const uint32_t w = gather_word<DIM>(a, a.vpad + m * a.vch, ix, iy, iz, p, q);
                    const float *th = thT + (m * L + um[m]) * KP;
#pragma unroll
                    for (int c = 0; c < 4; ++c) t[c] *= th[(w >> (8 * c)) & 0xff];
                }
                if (SAMPLE) {
                    // node by node, so the draw below can re-add one row in the same order
#pragma unroll
                    for (int c = 0; c < 4; ++c) S = __fadd_rn(S, t[c]);
                    cps[(p * Q + q) * kEThreads] = S;
                    continue;
                }
                const float s4 = (t[0] + t[1]) + (t[2] + t[3]);
                S += s4;
                Sx += (float)(p - 1) * s4;
                if (Q == 4) Sy += (float)(q - 1) * s4;
                Sz += (t[2] - t[0]) + 2.0f * t[3];
            }
        if (!(S > 0.0f)) {
            vp.store_r(a, i, V, fx, fy, fz);
            ++deg;
            continue;
        }
        if (SAMPLE) {
            // categorical draw of one neighbour (Registration.cpp:219-330 with sample): the first
            // whose running sum reaches u * S; every channel counts the drawn node's bin
            // (MILikelihoodFilter.cpp:102-115 with posterior 1)
            const u32x4 rr = philox_draw(a.seed, i, sweep, 1u, a.chain);
            const float tgt = u01_f24(rr.x) * S;
            int row = 4 * Q - 1;
            float cdf = 0.0f;
            for (int r = 0; r < 4 * Q; ++r) {
                const float e = cps[r * kEThreads];
                if (e >= tgt) {
                    row = r;
                    break;
                }
                cdf = e;
            }
            const int p = row / Q, q = row % Q;
            const float bxp = p == 0 ? bx[0] : (p == 1 ? bx[1] : (p == 2 ? bx[2] : bx[3]));
            const float byq = q == 0 ? by[0] : (q == 1 ? by[1] : (q == 2 ? by[2] : by[3]));
            const float bxy = Q == 4 ? bxp * byq : bxp;
            float t[4] = {bxy * bz[0], bxy * bz[1], bxy * bz[2], bxy * bz[3]};
            uint32_t wd[kMaxChannels];
#pragma unroll
            for (int m = 0; m < kMaxChannels; ++m) {
                if (m >= M) break;
                wd[m] = gather_word<DIM>(a, a.vpad + m * a.vch, ix, iy, iz, p, q);
                const float *th = thT + (m * L + um[m]) * KP;
#pragma unroll
                for (int c = 0; c < 4; ++c) t[c] *= th[(wd[m] >> (8 * c)) & 0xff];
            }
            int pc = 3;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                cdf = __fadd_rn(cdf, t[c]);
                if (cdf >= tgt) {
                    pc = c;
                    break;
                }
            }
#pragma unroll
            for (int m = 0; m < kMaxChannels; ++m) {
                if (m >= M) break;
                const int k = (wd[m] >> (8 * pc)) & 0xff;
                atomicAdd(&hc[(m * K + k) * LP + um[m]], 1u);
            }
            vp.store_r(a, i, V, fx + (float)(p - 1), fy + (float)(q - 1), fz + (float)(pc - 1));
            continue;
        }
        const float inv = 1.0f / S;
        // pass 2: the posterior of every neighbour into every channel's histogram
#pragma unroll 1
        for (int p = 0; p < 4; ++p)
#pragma unroll 1
            for (int q = 0; q < Q; ++q) {
                const float bxy = Q == 4 ? bx[p] * by[q] : bx[p];
                float t[4] = {bxy * bz[0], bxy * bz[1], bxy * bz[2], bxy * bz[3]};
                uint32_t wd[kMaxChannels];
#pragma unroll
                for (int m = 0; m < kMaxChannels; ++m) {
                    if (m >= M) break;
                    wd[m] = gather_word<DIM>(a, a.vpad + m * a.vch, ix, iy, iz, p, q);
                    const float *th = thT + (m * L + um[m]) * KP;
#pragma unroll
                    for (int c = 0; c < 4; ++c) t[c] *= th[(wd[m] >> (8 * c)) & 0xff];
                }
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float pc = t[c] * inv;
                    if (pc == 0.0f) continue;
#pragma unroll
                    for (int m = 0; m < kMaxChannels; ++m) {
                        if (m >= M) break;
                        const int k = (wd[m] >> (8 * c)) & 0xff;
                        atomicAdd(&hs[(m * K + k) * LP + um[m]], pc);
                    }
                }
            }
        mll -= (double)logf(S);
        vp.store_r(a, i, V, fx + Sx * inv, fy + Sy * inv, fz + Sz * inv);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < M * KL; q += blockDim.x) {
        const int m = q / KL, r = q - m * KL, k = r / L, l = r - k * L;
        if (SAMPLE) {
            const unsigned v = hc[(m * K + k) * LP + l];
            if (v) atomicAdd(&a.hcnt[q], v);
            continue;
        }
        const float v = hs[(m * K + k) * LP + l];
        if (v != 0.0f) atomicAdd(&a.hist[q], v);
    }
    __shared__ double red[32];
    const double ms = block_sum(mll, red);
    if (threadIdx.x == 0 && !SAMPLE) atomicAdd(&a.st->mll, ms);
    const double dg = block_sum((double)deg, red);
    if (threadIdx.x == 0 && dg > 0.0) atomicAdd(&a.st->degenerate, (unsigned long long)dg);
}

// ---- the SSD filter likelihood (BINDER/src/cpu/SSDLikelihoodFilter.cpp) -------------------
constexpr int kSsdfThreads = 128;

// number of per-thread statistics: packed A (Fn (Fn + 1) / 2), b (M Fn), S2 (M), eff
__host__ __device__ constexpr int ssdf_nstats(int M, int Fn) {
    return Fn * (Fn + 1) / 2 + M * Fn + M + 1;
}

// Log-space EM E-step (Registration.cpp:331-470) with compute_log_likelihood (:123-158) written
// as sum_m -(x_m - t_m(j))^2 / (2 sigma_m) + log_constant_m, where t_m(j) = sum_f cf[m][f] n_f(j)
// is channel m's prediction from the node's features (0 outside the grid).  accumulate_info's
// per-node sums (:160-198) are only ever used through A = sum p n n^T, b_m = sum p x_m n,
// S2_m = sum p x_m^2 and eff = sum p (update_coefficients :205-290 and update_sigma :292-346,
// whose sigma numerator is S2_m - 2 c_m . b_m + c_m^T A c_m for the new coefficients c_m), so
// each voxel adds its posterior moments of n to per-thread FP64 columns in shared memory, reduced
// once per CTA.  Two passes over the neighbours: the largest term, then exp(term - max).
template <int DIM, int FM, bool SAMPLE = false>
__global__ void __launch_bounds__(kSsdfThreads) estep_ssdf_kernel(const EStepArgs a) {
    constexpr int Q = DIM == 3 ? 4 : 1;
    constexpr int NA = FM * (FM + 1) / 2;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) double cols[];  // [nstats][kSsdfThreads]
    __shared__ double cf[kSsdfMax * kSsdfMax], hh[kSsdfMax];
    __shared__ double red[32];
    const SsdfState *ps = a.fstate;
    const int M = ps->M, Fn = ps->Fn;
    const int nst = ssdf_nstats(M, Fn);
    for (int q = threadIdx.x; q < kSsdfMax * kSsdfMax; q += blockDim.x) cf[q] = ps->cf[q];
    if (threadIdx.x < kSsdfMax) hh[threadIdx.x] = ps->h[threadIdx.x];
    const double lc = ps->lc;
    double *my = cols + threadIdx.x;  // my[s * kSsdfThreads]
    for (int s = 0; s < nst; ++s) my[s * kSsdfThreads] = 0.0;
    // sampling: the running sum at the end of node row r, cps[r * kSsdfThreads]
    float *cps = reinterpret_cast<float *>(cols + (size_t)nst * kSsdfThreads) + threadIdx.x;
    const uint32_t sweep = SAMPLE ? (uint32_t)a.st->sweep : 0u;
    __syncthreads();

    const long Vn = (long)a.nxn * a.nyn * a.nzn;
    double mll = 0.0;
    unsigned deg = 0;
    const unsigned V = (unsigned)a.V, nz = (unsigned)a.nz, ny = (unsigned)a.ny;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        VoxelPos<DIM> vp;
        if (!vp.load(a, i, V, ny, nz)) {
            vp.store_r(a, i, V, vp.px, vp.py, vp.pz);
            ++deg;
            continue;
        }
        float bx[4], by[4] = {1.f, 1.f, 1.f, 1.f}, bz[4];
        const int ix = spline_setup(vp.px, a.order, bx);
        const int iy = DIM == 3 ? spline_setup(vp.py, a.order, by) : 0;
        const int iz = spline_setup(vp.pz, a.order, bz);
        float lx[4], ly[4], lz[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            lx[t] = logf(bx[t]);  // -inf for a zero tap, whose term then vanishes
            ly[t] = DIM == 3 ? logf(by[t]) : 0.0f;
            lz[t] = logf(bz[t]);
        }
        double xv[kSsdfMax];
#pragma unroll
        for (int m = 0; m < kSsdfMax; ++m) xv[m] = m < M ? a.fx[(long)m * V + i] : 0.0;
        // the log term of neighbour (p, q, c) and the node's features, in FP64: with poor
        // coefficients the residual sums reach the hundreds, where FP32 would shift posteriors
        auto term_of = [&](int p, int q, int c, double (&n)[FM]) -> double {
            const int X = ix - 1 + p, Y = DIM == 3 ? iy - 1 + q : 0, Z = iz - 1 + c;
            const bool in = X >= 0 && Y >= 0 && Z >= 0 && X < a.nxn && Y < a.nyn && Z < a.nzn;
            const long j = in ? ((long)X * a.nyn + Y) * a.nzn + Z : 0;
#pragma unroll
            for (int f = 0; f < FM; ++f) n[f] = (in && f < Fn) ? __ldg(a.fn + f * Vn + j) : 0.0;
            double qs = 0.0;
#pragma unroll
            for (int m = 0; m < kSsdfMax; ++m) {
                if (m >= M) break;
                double t = 0.0;
#pragma unroll
                for (int f = 0; f < FM; ++f)
                    if (f < Fn) t = fma(cf[m * Fn + f], n[f], t);
                const double r = xv[m] - t;
                qs = fma(r * r, hh[m], qs);
            }
            return (double)((lx[p] + ly[q]) + lz[c]) - qs;
        };
        double mx = -INFINITY;
#pragma unroll 1
        for (int p = 0; p < 4; ++p)
#pragma unroll 1
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    double n[FM];
                    mx = fmax(mx, term_of(p, q, c, n));
                }
        if (SAMPLE) {
            // categorical draw of one neighbour (Registration.cpp:331-470 with sample): the
            // first whose running sum of exp(term - max) reaches u * S; its statistics enter
            // with posterior 1 (SSDLikelihoodFilter.cpp:168-198)
            float S = 0.0f;
#pragma unroll 1
            for (int p = 0; p < 4; ++p)
#pragma unroll 1
                for (int q = 0; q < Q; ++q) {
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        double nd[FM];
                        S = __fadd_rn(S, expf((float)(term_of(p, q, c, nd) - mx)));
                    }
                    cps[(p * Q + q) * kSsdfThreads] = S;
                }
            if (!(S > 0.0f)) {
                vp.store_r(a, i, V, (float)ix, (float)iy, (float)iz);
                ++deg;
                continue;
            }
            const u32x4 rr = philox_draw(a.seed, i, sweep, 1u, a.chain);
            const float tgt = u01_f24(rr.x) * S;
            int row = 4 * Q - 1;
            float cdf = 0.0f;
            for (int r = 0; r < 4 * Q; ++r) {
                const float e = cps[r * kSsdfThreads];
                if (e >= tgt) {
                    row = r;
                    break;
                }
                cdf = e;
            }
            const int p = row / Q, q = row % Q;
            int pc = 3;
            double nd[FM], pick[FM];
#pragma unroll
            for (int f = 0; f < FM; ++f) pick[f] = 0.0;
#pragma unroll 1
            for (int c = 0; c < 4; ++c) {
                cdf = __fadd_rn(cdf, expf((float)(term_of(p, q, c, nd) - mx)));
                pc = c;
#pragma unroll
                for (int f = 0; f < FM; ++f) pick[f] = nd[f];
                if (cdf >= tgt) break;
            }
            int s = 0;
#pragma unroll
            for (int f = 0; f < FM; ++f)
#pragma unroll
                for (int g = f; g < FM; ++g)
                    if (g < Fn) my[(s++) * kSsdfThreads] += pick[f] * pick[g];
#pragma unroll
            for (int m = 0; m < kSsdfMax; ++m) {
                if (m >= M) break;
#pragma unroll
                for (int f = 0; f < FM; ++f)
                    if (f < Fn) my[(s++) * kSsdfThreads] += xv[m] * pick[f];
            }
#pragma unroll
            for (int m = 0; m < kSsdfMax; ++m) {
                if (m >= M) break;
                my[(s++) * kSsdfThreads] += xv[m] * xv[m];
            }
            my[s * kSsdfThreads] += 1.0;
            vp.store_r(a, i, V, (float)(ix - 1 + p), (float)(DIM == 3 ? iy - 1 + q : 0),
                       (float)(iz - 1 + pc));
            continue;
        }
        float S = 0.0f, Sx = 0.0f, Sy = 0.0f, Sz = 0.0f, Bn[FM], A[NA];
#pragma unroll
        for (int f = 0; f < FM; ++f) Bn[f] = 0.0f;
#pragma unroll
        for (int k = 0; k < NA; ++k) A[k] = 0.0f;
#pragma unroll 1
        for (int p = 0; p < 4; ++p)
#pragma unroll 1
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    double nd[FM];
                    const float e = expf((float)(term_of(p, q, c, nd) - mx));
                    float n[FM];
#pragma unroll
                    for (int f = 0; f < FM; ++f) n[f] = (float)nd[f];
                    S += e;
                    Sx = fmaf((float)(p - 1), e, Sx);
                    if (Q == 4) Sy = fmaf((float)(q - 1), e, Sy);
                    Sz = fmaf((float)(c - 1), e, Sz);
                    int k = 0;
#pragma unroll
                    for (int f = 0; f < FM; ++f) {
                        Bn[f] = fmaf(e, n[f], Bn[f]);
                        const float en = e * n[f];
#pragma unroll
                        for (int g = f; g < FM; ++g, ++k) A[k] = fmaf(en, n[g], A[k]);
                    }
                }
        const float inv = 1.0f / S;
        mll -= mx + log((double)S) + lc;
        vp.store_r(a, i, V, (float)ix + Sx * inv, (float)iy + Sy * inv, (float)iz + Sz * inv);
        // this voxel's statistics: A (packed f <= g), b [m][f], S2 [m], eff
        int s = 0;
#pragma unroll
        for (int f = 0; f < FM; ++f)
#pragma unroll
            for (int g = f; g < FM; ++g)
                if (g < Fn) my[(s++) * kSsdfThreads] += (double)A[f * FM - f * (f - 1) / 2 + (g - f)] * inv;
#pragma unroll
        for (int m = 0; m < kSsdfMax; ++m) {
            if (m >= M) break;
#pragma unroll
            for (int f = 0; f < FM; ++f)
                if (f < Fn) my[(s++) * kSsdfThreads] += xv[m] * ((double)Bn[f] * inv);
        }
#pragma unroll
        for (int m = 0; m < kSsdfMax; ++m) {
            if (m >= M) break;
            my[(s++) * kSsdfThreads] += xv[m] * xv[m];
        }
        my[s * kSsdfThreads] += 1.0;
    }
    __syncthreads();
    // column s: thread s sums it and adds it at its place in the full layout of fstats
    if ((int)threadIdx.x < nst) {
        const int s = threadIdx.x;
        double v = 0.0;
        for (int t = 0; t < kSsdfThreads; ++t) v += cols[s * kSsdfThreads + t];
        const int na = Fn * (Fn + 1) / 2;
        if (s < na) {
            int f = 0, r = s;
            while (r >= Fn - f) r -= Fn - f++;
            const int g = f + r;
            atomicAdd(&a.fstats[kSsdfA + f * Fn + g], v);
            if (g != f) atomicAdd(&a.fstats[kSsdfA + g * Fn + f], v);
        } else if (s < na + M * Fn) {
            atomicAdd(&a.fstats[kSsdfB + (s - na)], v);
        } else if (s < na + M * Fn + M) {
            atomicAdd(&a.fstats[kSsdfS2 + (s - na - M * Fn)], v);
        } else {
            atomicAdd(&a.fstats[kSsdfEff], v);
        }
    }
    const double ms = block_sum(mll, red);
    if (threadIdx.x == 0 && !SAMPLE) atomicAdd(&a.st->mll, ms);
    const double dg = block_sum((double)deg, red);
    if (threadIdx.x == 0 && dg > 0.0) atomicAdd(&a.st->degenerate, (unsigned long long)dg);
}

__host__ __device__ void ssdf_refresh(SsdfState &p) {
    const double pi = 3.14159265358979323846;
    double lc = 0.0;
    for (int m = 0; m < p.M; ++m) {
        for (int f = 0; f < p.Fn; ++f)
            p.cf[m * p.Fn + f] = p.rfa ? (m == f ? 1.0 : 0.0) : p.coeff[m * p.F + f];
        p.h[m] = 0.5 / p.sigma[m];
        lc += -0.5 * log(2.0 * pi * p.sigma[m]);
    }
    p.lc = lc;
}

// SSDLikelihoodFilter::solve_linear_system (:348-389): Gaussian elimination with partial pivoting
__device__ void ssdf_solve(int n, const double *A, const double *b, double *x) {
    double aug[kSsdfMax][kSsdfMax + 1];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) aug[i][j] = A[i * n + j];
        aug[i][n] = b[i];
    }
    for (int i = 0; i < n; ++i) {
        int piv = i;
        for (int j = i + 1; j < n; ++j)
            if (fabs(aug[j][i]) > fabs(aug[piv][i])) piv = j;
        if (piv != i)
            for (int k = 0; k <= n; ++k) {
                const double t = aug[i][k];
                aug[i][k] = aug[piv][k];
                aug[piv][k] = t;
            }
        for (int j = i + 1; j < n; ++j) {
            const double f = aug[j][i] / aug[i][i];
            for (int k = i; k <= n; ++k) aug[j][k] -= f * aug[i][k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = 0.0;
        for (int j = i + 1; j < n; ++j) s += aug[i][j] * x[j];
        x[i] = (aug[i][n] - s) / aug[i][i];
    }
}

// update_parameters (:200-346) from the statistics, compute_cost (:72-89); one thread
__global__ void ssdf_update_kernel(SsdfState *ps, double *stats, int update, DevState *st) {
    if (st && st->done) return;
    if (threadIdx.x == 0) {
        SsdfState &p = *ps;
        const int M = p.M, Fn = p.Fn;
        if (update) {
            const double *A = stats + kSsdfA, *b = stats + kSsdfB;
            double c[kSsdfMax * kSsdfMax];
            for (int m = 0; m < M; ++m) {
                if (p.rfa) {
                    for (int f = 0; f < Fn; ++f) c[m * Fn + f] = m == f ? 1.0 : 0.0;
                } else {
                    ssdf_solve(Fn, A, b + m * Fn, c + m * Fn);
                    for (int f = 0; f < Fn; ++f) p.coeff[m * p.F + f] = c[m * Fn + f];
                }
            }
            const double den = stats[kSsdfEff] + 2.0 * p.alpha0;
            for (int m = 0; m < M; ++m) {
                const double *cm = c + m * Fn;
                double cb = 0.0, cac = 0.0;
                for (int f = 0; f < Fn; ++f) {
                    cb += cm[f] * b[m * Fn + f];
                    double af = 0.0;
                    for (int g = 0; g < Fn; ++g) af += A[f * Fn + g] * cm[g];
                    cac += cm[f] * af;
                }
                const double num =
                    stats[kSsdfS2 + m] - 2.0 * cb + cac + 2.0 * p.alpha0 * p.beta0;
                p.sigma[m] = num / den;
                if (!isfinite(p.sigma[m]) || !(p.sigma[m] > 0.0) || !isfinite(p.coeff[0]))
                    atomicOr(&st->flags, (unsigned)kFlagNonFinite);
            }
            ssdf_refresh(p);
        }
        const double a = p.alpha0, bb = p.alpha0 * p.beta0;
        double cost = 0.0;
        for (int m = 0; m < M; ++m) {
            const double x = p.sigma[m];
            cost += -(a * log(bb) - lgamma(a) + (-a - 1.0) * log(x) - bb / x);
        }
        if (st) st->lp_lik = cost;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kSsdfStats; q += blockDim.x) stats[q] = 0.0;
}

// SSDLikelihoodFilter::sample_parameters (:459-463): update_coefficients and update_sigma with
// sample = true, from the sweep's statistics (the drawn nodes, posterior 1).  Coefficients
// (reg_across_features 0): x = solve(A, b_m), then sample_multivariate_normal(x, A) as written
// (:392-427): L = chol(A) -- A itself as the covariance -- and coefficient i = x_i + sum_{j<=i}
// L_ij z_ij with a fresh standard normal z_ij per term (Philox ctr {(m * 8 + i) * 8 + j, sweep,
// 8, chain}, Box-Muller on words 0 and 1).  sigma_m = 1 / g, g ~ Gamma(shape den / 2, scale
// 2 / num_m) (sample_inverse_gamma(den / 2, num_m / 2), :429-432; tag 9, index m) with num_m from
// the drawn coefficients.  One thread.
__device__ double gamma_mt(double shape, uint64_t seed, uint32_t index, uint32_t sweep,
                           uint32_t tag, uint32_t chain, bool *capped);

__global__ void ssdf_sample_kernel(SsdfState *ps, double *stats, DevState *st, uint64_t seed,
                                   uint32_t chain) {
    if (st->done) return;
    if (threadIdx.x == 0) {
        SsdfState &p = *ps;
        const int M = p.M, Fn = p.Fn;
        const uint32_t sweep = (uint32_t)st->sweep;
        const double *A = stats + kSsdfA, *b = stats + kSsdfB;
        double c[kSsdfMax * kSsdfMax];
        if (p.rfa) {
            for (int m = 0; m < M; ++m)
                for (int f = 0; f < Fn; ++f) c[m * Fn + f] = m == f ? 1.0 : 0.0;
        } else {
            double Lc[kSsdfMax * kSsdfMax];
            for (int i = 0; i < Fn; ++i)
                for (int j = 0; j <= i; ++j) {
                    double sum = 0.0;
                    for (int k = 0; k < j; ++k) sum += Lc[i * Fn + k] * Lc[j * Fn + k];
                    Lc[i * Fn + j] = i == j ? sqrt(A[j * Fn + j] - sum)
                                            : (A[i * Fn + j] - sum) / Lc[j * Fn + j];
                }
            for (int m = 0; m < M; ++m) {
                double x[kSsdfMax];
                ssdf_solve(Fn, A, b + m * Fn, x);
                for (int i = 0; i < Fn; ++i) {
                    double v = x[i];
                    for (int j = 0; j <= i; ++j) {
                        const u32x4 r = philox_draw(seed, (uint32_t)((m * 8 + i) * 8 + j), sweep,
                                                    8u, chain);
                        const double z = sqrt(-2.0 * log(u01_d32(r.x))) * cospi(2.0 * u01_d32(r.y));
                        v += Lc[i * Fn + j] * z;
                    }
                    c[m * Fn + i] = v;
                    p.coeff[m * p.F + i] = v;
                }
            }
        }
        const double den = stats[kSsdfEff] + 2.0 * p.alpha0;
        bool capped = false;
        for (int m = 0; m < M; ++m) {
            const double *cm = c + m * Fn;
            double cb = 0.0, cac = 0.0;
            for (int f = 0; f < Fn; ++f) {
                cb += cm[f] * b[m * Fn + f];
                double af = 0.0;
                for (int g = 0; g < Fn; ++g) af += A[f * Fn + g] * cm[g];
                cac += cm[f] * af;
            }
            const double num = stats[kSsdfS2 + m] - 2.0 * cb + cac + 2.0 * p.alpha0 * p.beta0;
            const double g = gamma_mt(0.5 * den, seed, (uint32_t)m, sweep, 9u, chain, &capped) *
                             (2.0 / num);
            p.sigma[m] = 1.0 / g;
            if (!isfinite(p.sigma[m]) || !(p.sigma[m] > 0.0))
                atomicOr(&st->flags, (unsigned)kFlagNonFinite);
        }
        if (capped) atomicOr(&st->flags, (unsigned)kFlagGammaCapped);
        ssdf_refresh(p);
        const double a = p.alpha0, bb = p.alpha0 * p.beta0;
        double cost = 0.0;
        for (int m = 0; m < M; ++m) {
            const double x = p.sigma[m];
            cost += -(a * log(bb) - lgamma(a) + (-a - 1.0) * log(x) - bb / x);
        }
        st->lp_lik = cost;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kSsdfStats; q += blockDim.x) stats[q] = 0.0;
}

__global__ void features_to_soa_kernel(const double *in, long n, int C, double *out) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n * C;
         q += (long)gridDim.x * blockDim.x) {
        const long i = q / C;
        const int c = (int)(q - i * C);
        out[(long)c * n + i] = in[q];
    }
}

// BINDER/src/cpu/Registration.cpp:219-330 (EM and sampling branches), restated per voxel with the
// histogram kept in shared memory and neighbouring equal bins combined before the atomics.  Used
// for the Gibbs draw and for EM with K > 64.  The MI draw fits in 80 registers (three CTAs, 24
// warps per SM); the log-space draw and EM keep 128 (two CTAs).
template <bool SAMPLE, int DIM, bool LOGT = false>
__global__ void __launch_bounds__(kEThreads, (SAMPLE && !LOGT) ? 3 : 2)
    estep_kernel(const EStepArgs args) {
    constexpr int Q = DIM == 3 ? 4 : 1;
    constexpr int R = 4 * Q;  // node rows of 4 packed nodes
    if (args.skip && *args.skip) return;
    // a batch of chains (gridDim.y > 1, sampling only): chain blockIdx.y has its own positions
    // and dream locations [dim][V], theta and counts [K][L] and state, one chain after another,
    // and Philox chain index chain + blockIdx.y; the bins are shared
    const EStepArgs &a = args;
    const long cs = SAMPLE ? (long)blockIdx.y * a.dim * a.V : 0;  // positions / dream offset
    const long ks = SAMPLE ? (long)blockIdx.y * a.K * a.L : 0;    // theta / counts offset
    DevState *const st = SAMPLE ? a.st + blockIdx.y : a.st;
    const uint32_t chain = SAMPLE ? a.chain + blockIdx.y : a.chain;
    extern __shared__ __align__(16) float sm[];
    const int KL = a.K * a.L;
    float *th = sm;
    float *hs = sm + KL;                                 // EM histogram
    unsigned *hc = reinterpret_cast<unsigned *>(sm + KL);  // Gibbs counts
    float *cps = sm + 2 * KL + threadIdx.x;  // Gibbs: cdf at the end of node row r, cps[r * kEThreads]
    __shared__ double red[32];
    for (int q = threadIdx.x; q < KL; q += blockDim.x) {
        th[q] = a.theta[ks + q];
        if (SAMPLE) hc[q] = 0u; else hs[q] = 0.0f;
    }
    __syncthreads();

    const uint32_t sweep = SAMPLE ? (uint32_t)st->sweep : 0u;
    double mll = 0.0;
    unsigned long long deg = 0;
    const unsigned V = (unsigned)a.V, nz = (unsigned)a.nz, ny = (unsigned)a.ny;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        VoxelPos<DIM> vp;
        // positions far outside any grid (or non-finite) are degenerate: keep them as they are
        if (!vp.load(a, i, V, ny, nz, cs)) {
            vp.store_r(a, i, V, vp.px, vp.py, vp.pz, cs);
            ++deg;
            continue;
        }
        float bx[4], by[4] = {1.f, 1.f, 1.f, 1.f}, bz[4];
        const int ix = spline_setup(vp.px, a.order, bx);
        const int iy = DIM == 3 ? spline_setup(vp.py, a.order, by) : 0;
        const int iz = spline_setup(vp.pz, a.order, bz);
        const float fx = (float)ix, fy = (float)iy, fz = (float)iz;
        uint32_t pk[R];
        gather_bins<DIM>(a, ix, iy, iz, pk);
        const float *thc = th + a.u[i];  // theta column of this voxel's bin: thc[k * L]
        const int L = a.L;
        // LOGT (the SSD likelihood, sampling): thc holds log2 likelihoods, the spline weights
        // enter as log2 (-inf for a zero tap) and every neighbour's weight is exp2 of its term
        // minus the voxel's largest term (Registration.cpp:331-470)
        float lx[4], ly[4] = {0.f, 0.f, 0.f, 0.f}, lz[4], lm = 0.0f;
        if (LOGT) {
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                lx[t] = log2f(bx[t]);
                if (DIM == 3) ly[t] = log2f(by[t]);
                lz[t] = log2f(bz[t]);
            }
            lm = -INFINITY;
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const uint32_t word = pk[p * Q + q];
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        lm = fmaxf(lm, __fadd_rn(__fadd_rn(__fadd_rn(lx[p], ly[q]), lz[c]),
                                                 thc[((word >> (8 * c)) & 0xff) * L]));
                }
        }

        // pass 1: normaliser and the posterior-weighted node offsets
        float S = 0.0f, Sx = 0.0f, Sy = 0.0f, Sz = 0.0f;
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float bxy = DIM == 3 ? __fmul_rn(bx[p], by[q]) : bx[p];
                const uint32_t word = pk[p * Q + q];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int k = (word >> (8 * c)) & 0xff;
                    const float w =
                        LOGT ? exp2f(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(lx[p], ly[q]),
                                                                   lz[c]), thc[k * L]), -lm))
                             : __fmul_rn(__fmul_rn(bxy, bz[c]), thc[k * L]);
                    S = __fadd_rn(S, w);
                    Sx = fmaf((float)(p - 1), w, Sx);
                    if (DIM == 3) Sy = fmaf((float)(q - 1), w, Sy);
                    Sz = fmaf((float)(c - 1), w, Sz);
                }
                if (SAMPLE) cps[(p * Q + q) * kEThreads] = S;
            }
        if (!(S > 0.0f)) {
            vp.store_r(a, i, V, fx, fy, fz, cs);
            ++deg;
            continue;
        }
        if (!SAMPLE) {
            const float inv = 1.0f / S;
            mll -= log((double)S);
            vp.store_r(a, i, V, fx + Sx * inv, fy + Sy * inv, fz + Sz * inv, cs);
            // pass 2: normalised posteriors into the histogram column u_i, runs of equal bins
            // combined in a register before each shared-memory atomic
            const int ui = a.u[i];
            int ck = -1;
            float cacc = 0.0f;
#pragma unroll
            for (int p = 0; p < 4; ++p)
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const float bxy = DIM == 3 ? __fmul_rn(bx[p], by[q]) : bx[p];
                    const uint32_t word = pk[p * Q + q];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int k = (word >> (8 * c)) & 0xff;
                        const float w = __fmul_rn(__fmul_rn(bxy, bz[c]), thc[k * L]) * inv;
                        if (k == ck) {
                            cacc += w;
                        } else {
                            if (ck >= 0) atomicAdd(&hs[ck * L + ui], cacc);
                            ck = k;
                            cacc = w;
                        }
                    }
                }
            atomicAdd(&hs[ck * L + ui], cacc);
        } else {
            // categorical draw: first neighbour whose running sum reaches u * S.  The running sum
            // is the same sequence of FP32 additions as S above and never decreases (w >= 0), so
            // the first node row whose end value reaches the target holds the pick; only that
            // row's four nodes are summed again, from the previous row's end value.
            const u32x4 rr = philox_draw(a.seed, i, sweep, 1u, chain);
            const float t = u01_f24(rr.x) * S;
            int row = R - 1;
            float cdf = 0.0f;
            for (int r = 0; r < R; ++r) {
                const float e = cps[r * kEThreads];
                if (e >= t) {
                    row = r;
                    break;
                }
                cdf = e;
            }
            const int p = row / Q, q = row % Q;
            const float bxp = p == 0 ? bx[0] : (p == 1 ? bx[1] : (p == 2 ? bx[2] : bx[3]));
            const float byq = q == 0 ? by[0] : (q == 1 ? by[1] : (q == 2 ? by[2] : by[3]));
            const float bxy = DIM == 3 ? __fmul_rn(bxp, byq) : bxp;
            float lxy = 0.0f;
            if (LOGT) {
                const float lxp = p == 0 ? lx[0] : (p == 1 ? lx[1] : (p == 2 ? lx[2] : lx[3]));
                const float lyq = q == 0 ? ly[0] : (q == 1 ? ly[1] : (q == 2 ? ly[2] : ly[3]));
                lxy = __fadd_rn(lxp, lyq);
            }
            const uint32_t word = gather_word<DIM>(a, a.vpad, ix, iy, iz, p, q);
            int pick = -1, kp = 0;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int k = (word >> (8 * c)) & 0xff;
                const float w =
                    LOGT ? exp2f(__fadd_rn(__fadd_rn(__fadd_rn(lxy, lz[c]), thc[k * L]), -lm))
                         : __fmul_rn(__fmul_rn(bxy, bz[c]), thc[k * L]);
                cdf = __fadd_rn(cdf, w);
                if (pick < 0 && cdf >= t) {
                    pick = row * 4 + c;
                    kp = k;
                }
            }
            if (pick < 0) {  // unreachable (cdf ends at S >= t); keep the last neighbour
                pick = 4 * R - 1;
                kp = (gather_word<DIM>(a, a.vpad, ix, iy, iz, 3, Q - 1) >> 24) & 0xff;
            }
            atomicAdd(&hc[kp * L + a.u[i]], 1u);
            const int ox = pick / (4 * Q) - 1, oy = (pick / 4) % Q - 1, oz = pick % 4 - 1;
            vp.store_r(a, i, V, fx + (float)ox, fy + (float)oy, fz + (float)oz, cs);
        }
    }

    // merge: histogram entries this CTA touched, and the FP64 mll / degenerate partials
    __syncthreads();
    for (int q = threadIdx.x; q < KL; q += blockDim.x) {
        if (SAMPLE) {
            const unsigned v = hc[q];
            if (v) atomicAdd(&a.hcnt[ks + q], v);
        } else {
            const float v = hs[q];
            if (v != 0.0f) atomicAdd(&a.hist[q], v);
        }
    }
    const double m = block_sum(mll, red);
    if (threadIdx.x == 0 && !SAMPLE) atomicAdd(&st->mll, m);
    const double dg = block_sum((double)deg, red);
    if (threadIdx.x == 0 && dg > 0.0) atomicAdd(&st->degenerate, (unsigned long long)dg);
}

// MILikelihood.cpp:71-86 (update) and :33-39, :183-206 (cost), one CTA
__global__ void theta_update_kernel(float *theta, float *hist, int K, int L, double alpha,
                                    int update, DevState *st) {
    if (st->done) return;
    __shared__ double rowlp[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double lp_total = 0.0;
    // the log-normaliser terms are the same for every row: lgamma(sum alpha) - L lgamma(alpha)
    double sum_alpha = 0.0;
    for (int l = 0; l < L; ++l) sum_alpha += alpha;
    double lnorm = lgamma(sum_alpha);
    const double lga = lgamma(alpha);
    for (int l = 0; l < L; ++l) lnorm -= lga;
    for (int k = wid; k < K; k += nw) {
        if (update) {
            double s = 0.0;
            for (int l = lane; l < L; l += 32) s += (double)hist[k * L + l] + alpha - 1.0;
            s = warp_sum(s);
            for (int l = lane; l < L; l += 32)
                theta[k * L + l] = (float)(((double)hist[k * L + l] + alpha - 1.0) / s);
            __syncwarp();
        }
        double sl = 0.0;
        for (int l = lane; l < L; l += 32) sl += (alpha - 1.0) * log((double)theta[k * L + l]);
        sl = warp_sum(sl);
        if (lane == 0) lp_total += -(lnorm + sl);
    }
    __syncthreads();  // every row has been read before the histogram is cleared
    for (int q = threadIdx.x; q < K * L; q += blockDim.x) hist[q] = 0.0f;
    if (lane == 0) rowlp[wid] = lp_total;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += rowlp[w];
        st->lp_lik = t;
    }
}

// Gamma(shape, 1) by Marsaglia & Tsang (ACM TOMS 26(3), 2000) in FP64, with the shape < 1 boost;
// attempt j uses Philox ctr = {index, sweep, tag | j << 8, chain}: words 0,1 Box-Muller normal,
// word 2 acceptance uniform, word 3 boost uniform.  At most 64 attempts; *capped set beyond.
__device__ double gamma_mt(double shape, uint64_t seed, uint32_t index, uint32_t sweep,
                           uint32_t tag, uint32_t chain, bool *capped) {
    const bool small = shape < 1.0;
    const double a = small ? shape + 1.0 : shape;
    const double dd = a - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * dd);
    for (uint32_t att = 0; att < 64; ++att) {
        const u32x4 r = philox_draw(seed, index, sweep, tag | (att << 8), chain);
        const double u1 = u01_d32(r.x), u2 = u01_d32(r.y);
        const double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        double v = 1.0 + c * z;
        if (v <= 0.0) continue;
        v = v * v * v;
        const double uu = u01_d32(r.z);
        if (uu < 1.0 - 0.0331 * (z * z) * (z * z) || log(uu) < 0.5 * z * z + dd * (1.0 - v + log(v))) {
            double g = dd * v;
            if (small) g *= pow(u01_d32(r.w), 1.0 / shape);
            return g;
        }
    }
    *capped = true;
    return dd;
}

// MILikelihood.cpp:132-169 (Registration.cu:426-442 on the GPU): one CTA per row k
__global__ void dirichlet_sample_kernel(float *theta, unsigned *hcnt, int K, int L, double alpha,
                                        uint64_t seed, uint32_t chain, DevState *st) {
    // chain blockIdx.y of a batch: its own theta, counts and state
    theta += (long)blockIdx.y * K * L;
    hcnt += (long)blockIdx.y * K * L;
    st += blockIdx.y;
    chain += blockIdx.y;
    if (st->done) return;
    __shared__ double red[32];
    const int k = blockIdx.x;
    const uint32_t sweep = (uint32_t)st->sweep;
    double g = 0.0;
    bool capped = false;
    const int l = threadIdx.x;
    if (l < L) {
        const double shape = (double)hcnt[k * L + l] + alpha;
        g = gamma_mt(shape, seed, (uint32_t)(k * L + l), sweep, 4u, chain, &capped);
        hcnt[k * L + l] = 0u;
    }
    const double s = block_sum(g, red);
    __shared__ double tot;
    if (threadIdx.x == 0) tot = s;
    __syncthreads();
    if (l < L) theta[k * L + l] = (float)(g / tot);
    if (capped) atomicOr(&st->flags, (unsigned)kFlagGammaCapped);
}

// NonLinearTransformation.cpp:115-124 and :140-148
__global__ void nu_sample_kernel(DevState *st, int sample_gamma, int every, int N, long V,
                                 double rho_p, double e0, double e1, double e2, uint64_t seed,
                                 uint32_t chain) {
    st += blockIdx.x;  // chain blockIdx.x of a batch
    chain += blockIdx.x;
    if (st->done) return;
    const int sweep = st->sweep;
    if (sample_gamma && (sweep % every == 0)) {
        const double alpha_0 = 1.0, beta_0 = 10000.0;
        const double a_post = alpha_0 + 0.5 * (double)N * (double)V;
        const double b_post = beta_0 + 0.5 * (double)V * st->raw_reg;
        bool capped = false;
        const double nu = gamma_mt(a_post, seed, 0u, (uint32_t)sweep, 5u, chain, &capped) / b_post;
        if (capped) st->flags |= kFlagGammaCapped;
        st->nu = nu;
        st->gamma[0] = nu * rho_p * e0 * (double)V;
        st->gamma[1] = nu * rho_p * e1 * (double)V;
        st->gamma[2] = nu * rho_p * e2 * (double)V;
    }
    st->raw_reg = 0.0;
}

// Registration.cpp:195-214
__global__ void em_finish_kernel(DevState *st, double *stats, int max_iter, double th, double nzv) {
    if (st->done) return;
    const double mlp = st->mll + st->lp_tr + st->lp_lik;
    const int it = st->iter;
    if (it < max_iter) {
        stats[it * 4 + 0] = st->mll;
        stats[it * 4 + 1] = st->lp_lik;
        stats[it * 4 + 2] = st->lp_tr;
        stats[it * 4 + 3] = mlp;
    }
    if (!isfinite(mlp)) st->flags |= kFlagNonFinite;
    st->iter = it + 1;
    if ((st->mlp_old - mlp) / nzv < th || it + 1 >= max_iter) st->done = 1;
    st->mlp_old = mlp;
    st->mll = 0.0;
    st->lp_tr = 0.0;
}

// Registration.cpp:593-623 in FP64 with the symmetric M2 (xx, xy, xz, yy, yz, zz)
// N components: mean [N][V], M2 as its upper triangle [N (N + 1) / 2][V] (row-major: xx, xy, xz,
// yy, yz, zz or xx, xy, yy)
template <int N>
__global__ void sweep_end_kernel(const float *d, double *mean, double *m2, long V, int N_b,
                                 DevState *st) {
    // chain blockIdx.y of a batch: positions [N][V], mean [N][V], M2 [N (N + 1) / 2][V] per chain
    d += (long)blockIdx.y * N * V;
    mean += (long)blockIdx.y * N * V;
    m2 += (long)blockIdx.y * (N * (N + 1) / 2) * V;
    st += blockIdx.y;
    if (st->done) return;
    const int sweep = st->sweep;
    if (sweep >= N_b) {
        const double inv_n = 1.0 / ((double)(sweep - N_b) + 1.0);
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < V;
             i += (long)gridDim.x * blockDim.x) {
            double d1[N], d2[N];
#pragma unroll
            for (int n = 0; n < N; ++n) {
                const double val = (double)d[n * V + i];
                const double mo = mean[n * V + i];
                d1[n] = val - mo;
                const double mn = mo + d1[n] * inv_n;
                mean[n * V + i] = mn;
                d2[n] = val - mn;
            }
            int e = 0;
#pragma unroll
            for (int r = 0; r < N; ++r)
#pragma unroll
                for (int c = r; c < N; ++c, ++e) m2[e * V + i] += d1[r] * d2[c];
        }
    }
}

__global__ void sweep_advance_kernel(DevState *st, int total) {
    st += blockIdx.x;  // chain blockIdx.x of a batch
    if (st->done) return;
    st->sweep += 1;
    if (st->sweep >= total) st->done = 1;
}

}  // namespace

namespace {
// shared memory of the single-pass EM kernel with tpb threads
size_t fast_smem(int K, int L, int tpb, bool logt, bool half) {
    const bool w = tpb > kFastThreads;
    const int KP = w ? wide_pitch(K) : theta_pitch(K), LP = w ? wide_pitch(L) : theta_pitch(L);
    return (size_t)(L * KP + K * LP + (half ? ((K + 1) / 2) * tpb : K * tpb) + (logt ? L : 0)) *
           sizeof(float);
}

int device_sms() {
    int dev = 0, sms = 148;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

// threads per CTA of the single-pass EM kernel (MI likelihood, FP32 columns): the wide form when
// its tables fit and one wave of it gives every thread 8 voxels at least, else 256 (two CTAs/SM).
// With fewer voxels per thread the last pass over the grid leaves more of the wide CTAs idle, and
// registrations run side by side (a batch) overlap better in the smaller CTAs.
constexpr int kWideMinVoxelsPerThread = 8;
int fast_threads(long V, int K, int L, bool logt, bool half) {
    if (logt || half || K > kSmallK) return kFastThreads;
    if (fast_smem(K, L, kWideThreads, false, false) + 512 > 227 * 1024) return kFastThreads;
    if (V < (long)device_sms() * kWideThreads * kWideMinVoxelsPerThread) return kFastThreads;
    return kWideThreads;
}

size_t estep_smem(bool sample, int K, int L, bool logt = false, bool half = false,
                  int tpb = kFastThreads) {
    if (!sample && K <= kSmallK) return fast_smem(K, L, tpb, logt, half);
    return (size_t)(2 * K * L + (sample ? 16 * kEThreads : 0)) * sizeof(float);
}
}  // namespace

namespace {
template <int DIM>
const void *estep_fn(bool sample, int K, bool logt, bool half, bool wide) {
    if (logt && sample) return (const void *)estep_kernel<true, DIM, true>;
    if (logt) return (const void *)estep_em_fast_kernel<kFastThreads, DIM, true>;
    if (half && !sample && K <= kSmallK)
        return (const void *)estep_em_fast_kernel<kFastThreads, DIM, false, true>;
    if (wide && !sample && K <= kSmallK)
        return (const void *)estep_em_fast_kernel<kWideThreads, DIM, false>;
    return sample ? (const void *)estep_kernel<true, DIM>
                  : (K <= kSmallK ? (const void *)estep_em_fast_kernel<kFastThreads, DIM, false>
                                  : (const void *)estep_kernel<false, DIM>);
}

size_t filter_smem(int K, int L, int M, bool sample = false) {
    return ((size_t)M * (L * theta_pitch(K) + K * theta_pitch(L)) + (sample ? 16 * kEThreads : 0)) *
           sizeof(float);
}

// the per-thread statistics columns, and for sampling the per-thread draw table (16 rows)
size_t ssdf_smem(int M, int Fn, bool sample = false) {
    return (size_t)ssdf_nstats(M, Fn) * kSsdfThreads * 8 + (sample ? 16 * kSsdfThreads * 4 : 0);
}

template <int DIM, bool SAMPLE>
const void *ssdf_fn_s(int Fn) {
    if (Fn <= 2) return (const void *)estep_ssdf_kernel<DIM, 2, SAMPLE>;
    if (Fn <= 4) return (const void *)estep_ssdf_kernel<DIM, 4, SAMPLE>;
    return (const void *)estep_ssdf_kernel<DIM, 8, SAMPLE>;
}

template <int DIM>
const void *ssdf_fn(int Fn, bool sample = false) {
    return sample ? ssdf_fn_s<DIM, true>(Fn) : ssdf_fn_s<DIM, false>(Fn);
}

template <int DIM, bool SAMPLE>
void launch_ssdf_dim_s(const EStepArgs &a, int grid, size_t smem, cudaStream_t s) {
    if (a.Fn <= 2)
        count_launch(), estep_ssdf_kernel<DIM, 2, SAMPLE><<<grid, kSsdfThreads, smem, s>>>(a);
    else if (a.Fn <= 4)
        count_launch(), estep_ssdf_kernel<DIM, 4, SAMPLE><<<grid, kSsdfThreads, smem, s>>>(a);
    else
        count_launch(), estep_ssdf_kernel<DIM, 8, SAMPLE><<<grid, kSsdfThreads, smem, s>>>(a);
}

template <int DIM>
void launch_ssdf_dim(const EStepArgs &a, bool sample, int grid, size_t smem, cudaStream_t s) {
    if (sample)
        launch_ssdf_dim_s<DIM, true>(a, grid, smem, s);
    else
        launch_ssdf_dim_s<DIM, false>(a, grid, smem, s);
}

template <int DIM>
void launch_estep_dim(const EStepArgs &a, bool sample, int grid, size_t smem, cudaStream_t s,
                      int ftpb) {
    if (a.ssdf)
        launch_ssdf_dim<DIM>(a, sample, grid, smem, s);
    else if (a.filter && sample)
        count_launch(), estep_filter_kernel<DIM, true><<<grid, kEThreads, smem, s>>>(a);
    else if (a.filter)
        count_launch(), estep_filter_kernel<DIM><<<grid, kEThreads, smem, s>>>(a);
    else if (a.logt && sample)
        count_launch(), estep_kernel<true, DIM, true><<<grid, kEThreads, smem, s>>>(a);
    else if (a.logt)
        count_launch(), estep_em_fast_kernel<kFastThreads, DIM, true>
                            <<<grid, kFastThreads, smem, s>>>(a);
    else if (sample)
        count_launch(), estep_kernel<true, DIM><<<grid, kEThreads, smem, s>>>(a);
    else if (a.K <= kSmallK && a.halfcol)
        count_launch(), estep_em_fast_kernel<kFastThreads, DIM, false, true>
                            <<<grid, kFastThreads, smem, s>>>(a);
    else if (a.K <= kSmallK && ftpb == kWideThreads)
        count_launch(), estep_em_fast_kernel<kWideThreads, DIM, false>
                            <<<grid, kWideThreads, smem, s>>>(a);
    else if (a.K <= kSmallK)
        count_launch(), estep_em_fast_kernel<kFastThreads, DIM, false>
                            <<<grid, kFastThreads, smem, s>>>(a);
    else
        count_launch(), estep_kernel<false, DIM><<<grid, kEThreads, smem, s>>>(a);
}
}  // namespace

int estep_grid(bool sample, int K, int L, long V, int dim, bool logt, bool half) {
    BINDER_CHECK(dim == 2 || dim == 3, "dimension must be 2 or 3");
    BINDER_CHECK(!logt || (K <= kSmallK && K <= kLogMaxBins),
                 "the log-space E-step supports at most 64 bins");
    int per_sm = 1;
    const int sms = device_sms();
    const bool hc = half && !sample && !logt && K <= kSmallK;
    const int ftpb = sample ? kFastThreads : fast_threads(V, K, L, logt, hc);
    const bool wide = ftpb == kWideThreads;
    const size_t smem = estep_smem(sample, K, L, logt, hc, ftpb);
    const void *fn = dim == 3 ? estep_fn<3>(sample, K, logt, hc, wide)
                              : estep_fn<2>(sample, K, logt, hc, wide);
    const int tpb = (!sample && (logt || K <= kSmallK)) ? ftpb : kEThreads;
    BINDER_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // all of the unified L1 / shared array as shared memory, so the CTAs the occupancy query
    // counts are the CTAs that become resident (the default carveout may be smaller)
    BINDER_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    BINDER_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, tpb, smem));
    per_sm = per_sm < 1 ? 1 : per_sm;
    const long need = (V + tpb - 1) / tpb;
    long g = (long)sms * per_sm;
    if (need < g) g = need < 1 ? 1 : need;
    return (int)g;
}

bool filter_sampling_fits(int K, int L, int M) {
    return filter_smem(K, L, M, true) <= 227 * 1024;
}

int estep_filter_grid(int K, int L, int M, long V, int dim, bool sample) {
    BINDER_CHECK(dim == 2 || dim == 3, "dimension must be 2 or 3");
    BINDER_CHECK(M >= 1 && M <= kMaxChannels && (long)M * K * L <= kFilterMaxCells,
                 "the MI filter likelihood needs 1 <= M <= 8 and M * K * L <= 24576");
    int dev = 0, sms = 148, per_sm = 1;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t smem = filter_smem(K, L, M, sample);
    BINDER_CHECK(smem <= 227 * 1024,
                 sample ? "the MI filter likelihood's theta, counts and draw table do not fit in "
                          "shared memory (the sampler needs M * K * L below about 22000)"
                        : "the MI filter likelihood's theta and histograms do not fit in shared "
                          "memory");
    const void *fn = sample ? (dim == 3 ? (const void *)estep_filter_kernel<3, true>
                                        : (const void *)estep_filter_kernel<2, true>)
                            : (dim == 3 ? (const void *)estep_filter_kernel<3>
                                        : (const void *)estep_filter_kernel<2>);
    BINDER_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BINDER_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    BINDER_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kEThreads, smem));
    per_sm = per_sm < 1 ? 1 : per_sm;
    const long need = (V + kEThreads - 1) / kEThreads;
    long g = (long)sms * per_sm;
    if (need < g) g = need < 1 ? 1 : need;
    return (int)g;
}

int estep_ssdf_grid(int M, int Fn, long V, int dim, bool sample) {
    BINDER_CHECK(dim == 2 || dim == 3, "dimension must be 2 or 3");
    BINDER_CHECK(M >= 1 && M <= kSsdfMax && Fn >= 1 && Fn <= kSsdfMax,
                 "the SSD filter likelihood needs 1 <= M, F <= 8");
    int dev = 0, sms = 148, per_sm = 1;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t smem = ssdf_smem(M, Fn, sample);
    // both dimensions' kernels for this feature count
    const void *fns[2] = {ssdf_fn<2>(Fn, sample), ssdf_fn<3>(Fn, sample)};
    for (const void *f : fns) {
        BINDER_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
        BINDER_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared));
    }
    BINDER_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fns[dim - 2], kSsdfThreads,
                                                              smem));
    per_sm = per_sm < 1 ? 1 : per_sm;
    const long need = (V + kSsdfThreads - 1) / kSsdfThreads;
    long g = (long)sms * per_sm;
    if (need < g) g = need < 1 ? 1 : need;
    return (int)g;
}

void ssdf_refresh_host(SsdfState &p) { ssdf_refresh(p); }

void launch_ssdf_sample(SsdfState *p, double *stats, DevState *st, uint64_t seed,
                        uint32_t chain, cudaStream_t s) {
    count_launch(), ssdf_sample_kernel<<<1, 160, 0, s>>>(p, stats, st, seed, chain);
    BINDER_CUDA(cudaGetLastError());
}

void launch_ssdf_update(SsdfState *p, double *stats, int update, DevState *st, cudaStream_t s) {
    count_launch(), ssdf_update_kernel<<<1, 160, 0, s>>>(p, stats, update, st);
    BINDER_CUDA(cudaGetLastError());
}

void launch_features_to_soa(const double *in, long n, int C, double *out, cudaStream_t s) {
    long b = (n * C + 255) / 256;
    b = b < 1 ? 1 : (b > 148L * 16 ? 148L * 16 : b);
    count_launch(), features_to_soa_kernel<<<(int)b, 256, 0, s>>>(in, n, C, out);
    BINDER_CUDA(cudaGetLastError());
}

void launch_estep(const EStepArgs &args, bool sample, int grid, cudaStream_t s, int chains) {
    BINDER_CHECK(!args.logt || (args.K <= kSmallK && (sample || args.colmax)),
                 "the log-space E-step supports at most 64 bins");
    BINDER_CHECK(!args.filter || (!args.logt && args.M >= 1 &&
                                  args.M <= kMaxChannels &&
                                  (long)args.M * args.K * args.L <= kFilterMaxCells),
                 "the MI filter E-step needs 1 <= M <= 8 and M * K * L <= 24576");
    BINDER_CHECK(!args.ssdf || (args.fstate && args.fstats && args.M >= 1 &&
                                args.M <= kSsdfMax && args.Fn >= 1 && args.Fn <= kSsdfMax),
                 "the SSD filter E-step needs 1 <= M, F <= 8");
    EStepArgs a = args;
    if (sample || a.logt || a.filter || a.ssdf) a.halfcol = 0;  // FP32 columns only there
    // threads per CTA of the single-pass EM kernel (the same choice as estep_grid's)
    const int ftpb = (sample || a.filter || a.ssdf)
                         ? kFastThreads
                         : fast_threads(a.V, a.K, a.L, a.logt != 0, a.halfcol != 0);
    const size_t smem = a.ssdf     ? ssdf_smem(a.M, a.Fn, sample)
                        : a.filter ? filter_smem(a.K, a.L, a.M, sample)
                                   : estep_smem(sample, a.K, a.L, a.logt != 0, a.halfcol != 0,
                                                ftpb);
    // the order-independent merge of the single-pass EM kernel keeps one partial per CTA
    if (a.hfix && grid > kMaxEmCtas) grid = kMaxEmCtas;
    // fixed-point scale of the EM histogram: the largest scale (at most 2^30, exact in FP32) for
    // which the voxels one CTA visits, each adding at most scale + 1/2 (a posterior of 1, rounded;
    // FP32 rounding of m / S can exceed 1 by a few ulps, covered by the factor 1 + 2^-16) to a
    // cell, fit in 32 bits
    const long per_cta = ((a.V + (long)grid * ftpb - 1) / ((long)grid * ftpb)) * ftpb;
    double sc = std::floor(4294967295.0 / ((double)per_cta * (1.0 + 1.0 / 65536.0)) - 1.0);
    sc = sc < 1.0 ? 1.0 : (sc > 1073741824.0 ? 1073741824.0 : sc);
    float fsc = (float)sc;
    if ((double)fsc > sc) fsc = std::nextafter(fsc, 0.0f);  // round down into FP32
    a.hscale = fsc;
    a.hinv = 1.0 / (double)fsc;
    BINDER_CHECK(a.dim == 2 || a.dim == 3, "dimension must be 2 or 3");
    BINDER_CHECK(chains >= 1 && chains <= 65535 && (chains == 1 || (sample && !a.logt)),
                 "a batch of chains runs the sampling E-step of the MI likelihood only");
    if (chains > 1) {
        // the single-chain grid (one wave of CTAs) shared out over the chains, rounded down so all
        // of them are resident at once (every CTA loops over its chain's voxels)
        const int gx = grid / chains > 0 ? grid / chains : 1;
        const dim3 g2((unsigned)gx, (unsigned)chains, 1);
        if (a.dim == 3)
            count_launch(), estep_kernel<true, 3><<<g2, kEThreads, smem, s>>>(a);
        else
            count_launch(), estep_kernel<true, 2><<<g2, kEThreads, smem, s>>>(a);
    } else if (a.dim == 3) {
        launch_estep_dim<3>(a, sample, grid, smem, s, ftpb);
    } else {
        launch_estep_dim<2>(a, sample, grid, smem, s, ftpb);
    }
    BINDER_CUDA(cudaGetLastError());
}

void launch_theta_update(float *theta, float *hist, int K, int L, double alpha, int update,
                         DevState *st, cudaStream_t s) {
    count_launch(), theta_update_kernel<<<1, 1024, 0, s>>>(theta, hist, K, L, alpha, update, st);
    BINDER_CUDA(cudaGetLastError());
}

namespace {
// SSDLikelihood.cpp:58-82 in natural log: log N(l; shift + scale k, sigma^2) (shift_scale 0:
// shift 0, scale 1); bin 0 also stands for the nodes outside the grid, whose value is 0
__device__ __forceinline__ double ssd_loglik(int k, int l, const SsdState &p) {
    const double adj = p.shift_scale ? (double)l - p.shift - p.scale * (double)k
                                     : (double)l - (double)k;
    return (adj * adj) / (-2.0 * p.sigma2) - log(sqrt(2.0 * 3.14159265358979323846 * p.sigma2));
}

__global__ void ssd_update_kernel(float *table, float *colmax, float *hist, int K, int L,
                                  int update, SsdState *ps, DevState *st) {
    if (st && st->done) return;
    __shared__ double G[kLogMaxBins], S1[kLogMaxBins], S2[kLogMaxBins], D2[kLogMaxBins];
    __shared__ SsdState p;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) p = *ps;
    __syncthreads();
    if (update && hist) {
        // per node bin k: posterior mass, its first and second moments in the voxel bin, and
        // the squared differences for the shiftScale-0 update (SSDLikelihood.cpp:111-141)
        for (int k = wid; k < K; k += nw) {
            double g = 0.0, s1 = 0.0, s2 = 0.0, d2 = 0.0;
            for (int l = lane; l < L; l += 32) {
                const double h = (double)hist[k * L + l], df = (double)l - (double)k;
                g += h;
                s1 += h * (double)l;
                s2 += h * (double)l * (double)l;
                d2 += h * df * df;
            }
            g = warp_sum(g);
            s1 = warp_sum(s1);
            s2 = warp_sum(s2);
            d2 = warp_sum(d2);
            if (lane == 0) {
                G[k] = g;
                S1[k] = s1;
                S2[k] = s2;
                D2[k] = d2;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double den = 0.0, num = 0.0;
            if (!p.shift_scale) {  // :147-163
                for (int k = 0; k < K; ++k) {
                    num += D2[k];
                    den += G[k];
                }
            } else {  // :167-285, the 2x2 normal equations in closed form
                double A00 = 0.0, A01 = 0.0, A11 = 0.0, b0 = 0.0, b1 = 0.0;
                for (int k = 0; k < K; ++k) {
                    A00 += G[k];
                    A01 += G[k] * (double)k;
                    A11 += G[k] * (double)k * (double)k;
                    b0 += S1[k];
                    b1 += S1[k] * (double)k;
                }
                const double det = A00 * A11 - A01 * A01;
                if (det != 0.0 && isfinite(det)) {
                    p.shift = (b0 * A11 - A01 * b1) / det;
                    p.scale = (A00 * b1 - A01 * b0) / det;
                }
                for (int k = 0; k < K; ++k) {
                    const double t1 = p.shift + p.scale * (double)k;
                    num += S2[k] + -2.0 * S1[k] * t1 + G[k] * (t1 * t1);
                    den += G[k];
                }
            }
            num += p.alpha0 * p.beta0;
            den += p.alpha0;
            p.sigma2 = num / den;
            *ps = p;
        }
        __syncthreads();
    }
    if (st && threadIdx.x == 0) {  // compute_cost (:314-326): -log InvGamma(sigma^2; a, a beta0)
        const double a = p.alpha0, b = p.alpha0 * p.beta0, x = p.sigma2;
        st->lp_lik = -(a * log(b) - lgamma(a) + (-a - 1.0) * log(x) - b / x);
        if (!isfinite(p.sigma2) || !(p.sigma2 > 0.0)) atomicOr(&st->flags, (unsigned)kFlagNonFinite);
    }
    // the next E-step's table: log2 likelihoods minus their maximum over k per voxel bin l
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        double m = -INFINITY;
        for (int k = 0; k < K; ++k) m = fmax(m, ssd_loglik(k, l, p));
        colmax[l] = (float)m;
        for (int k = 0; k < K; ++k)
            table[k * L + l] = (float)((ssd_loglik(k, l, p) - m) * 1.4426950408889634);
    }
    if (st && hist) {
        __syncthreads();  // every row was read before the histogram is cleared
        for (int q = threadIdx.x; q < K * L; q += blockDim.x) hist[q] = 0.0f;
    }
}

// SSDLikelihood::sample_parameters (:284-302) with update_shift_and_scale / update_sigma run with
// sample = 1 (:167-285), from the sweep's counts hcnt[k][l] (the drawn node's bin k at voxel bin
// l; bin 0 also holds the nodes outside the grid): shiftScale 0: sigmaSq = 1 / g with g ~
// Gamma(shape den / 2, scale 2 den / num), the reference's parameterisation as written;
// shiftScale 1: (shift, scale) = A^-1 b + chol(A^-1) z with z two standard normals, then sigmaSq
// the same way from the drawn shift and scale.  Philox ctr {0, sweep, 6, chain} gives z by
// Box-Muller on words 0 and 1; the gamma uses tag 7.  Then the next sweep's log2 table, and the
// counts cleared.  One CTA.
__global__ void ssd_sample_kernel(float *table, float *colmax, unsigned *hcnt, int K, int L,
                                  SsdState *ps, DevState *st, uint64_t seed, uint32_t chain) {
    if (st->done) return;
    __shared__ double G[kLogMaxBins], S1[kLogMaxBins], S2[kLogMaxBins], D2[kLogMaxBins];
    __shared__ SsdState p;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) p = *ps;
    for (int k = wid; k < K; k += nw) {
        double g = 0.0, s1 = 0.0, s2 = 0.0, d2 = 0.0;
        for (int l = lane; l < L; l += 32) {
            const double h = (double)hcnt[k * L + l], df = (double)l - (double)k;
            g += h;
            s1 += h * (double)l;
            s2 += h * (double)l * (double)l;
            d2 += h * df * df;
        }
        g = warp_sum(g);
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        d2 = warp_sum(d2);
        if (lane == 0) {
            G[k] = g;
            S1[k] = s1;
            S2[k] = s2;
            D2[k] = d2;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t sweep = (uint32_t)st->sweep;
        double num = 0.0, den = 0.0;
        if (!p.shift_scale) {
            for (int k = 0; k < K; ++k) {
                num += D2[k];
                den += G[k];
            }
        } else {
            double A00 = 0.0, A01 = 0.0, A11 = 0.0, b0 = 0.0, b1 = 0.0;
            for (int k = 0; k < K; ++k) {
                A00 += G[k];
                A01 += G[k] * (double)k;
                A11 += G[k] * (double)k * (double)k;
                b0 += S1[k];
                b1 += S1[k] * (double)k;
            }
            const double det = A00 * A11 - A01 * A01;
            if (det > 0.0 && isfinite(det)) {
                const double x0 = (b0 * A11 - A01 * b1) / det, x1 = (A00 * b1 - A01 * b0) / det;
                const double c00 = A11 / det, c01 = -A01 / det, c11 = A00 / det;
                const double l00 = sqrt(c00), l10 = c01 / l00, l11 = sqrt(c11 - l10 * l10);
                const u32x4 r = philox_draw(seed, 0u, sweep, 6u, chain);
                const double rad = sqrt(-2.0 * log(u01_d32(r.x))), t = 2.0 * u01_d32(r.y);
                const double z0 = rad * cospi(t), z1 = rad * sinpi(t);
                p.shift = x0 + l00 * z0;
                p.scale = x1 + l10 * z0 + l11 * z1;
            }
            for (int k = 0; k < K; ++k) {
                const double t1 = p.shift + p.scale * (double)k;
                num += S2[k] + -2.0 * S1[k] * t1 + G[k] * (t1 * t1);
                den += G[k];
            }
        }
        num += p.alpha0 * p.beta0;
        den += p.alpha0;
        bool capped = false;
        const double g = gamma_mt(den * 0.5, seed, 0u, sweep, 7u, chain, &capped) *
                         (2.0 * den / num);
        p.sigma2 = 1.0 / g;
        if (capped) atomicOr(&st->flags, (unsigned)kFlagGammaCapped);
        if (!isfinite(p.sigma2) || !(p.sigma2 > 0.0)) atomicOr(&st->flags, (unsigned)kFlagNonFinite);
        *ps = p;
        const double a = p.alpha0, b = p.alpha0 * p.beta0, x = p.sigma2;
        st->lp_lik = -(a * log(b) - lgamma(a) + (-a - 1.0) * log(x) - b / x);
    }
    __syncthreads();
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        double m = -INFINITY;
        for (int k = 0; k < K; ++k) m = fmax(m, ssd_loglik(k, l, p));
        colmax[l] = (float)m;
        for (int k = 0; k < K; ++k)
            table[k * L + l] = (float)((ssd_loglik(k, l, p) - m) * 1.4426950408889634);
    }
    for (int q = threadIdx.x; q < K * L; q += blockDim.x) hcnt[q] = 0u;
}
}  // namespace

void launch_ssd_update(float *table, float *colmax, float *hist, int K, int L, int update,
                       SsdState *p, DevState *st, cudaStream_t s) {
    BINDER_CHECK(K >= 1 && K <= kLogMaxBins && L >= 1, "SSD bins must be in [1, 64]");
    count_launch(), ssd_update_kernel<<<1, 256, 0, s>>>(table, colmax, hist, K, L, update, p, st);
    BINDER_CUDA(cudaGetLastError());
}

void launch_ssd_sample(float *table, float *colmax, unsigned *hcnt, int K, int L, SsdState *p,
                       DevState *st, uint64_t seed, uint32_t chain, cudaStream_t s) {
    BINDER_CHECK(K >= 1 && K <= kLogMaxBins && L >= 1, "SSD bins must be in [1, 64]");
    count_launch(), ssd_sample_kernel<<<1, 256, 0, s>>>(table, colmax, hcnt, K, L, p, st, seed,
                                                        chain);
    BINDER_CUDA(cudaGetLastError());
}

void launch_dirichlet_sample(float *theta, unsigned *hcnt, int K, int L, double alpha,
                             uint64_t seed, uint32_t chain, DevState *st, cudaStream_t s,
                             int chains) {
    const int threads = ((L + 31) / 32) * 32;
    count_launch(), dirichlet_sample_kernel<<<dim3((unsigned)K, (unsigned)chains), threads, 0, s>>>(
                        theta, hcnt, K, L, alpha, seed, chain, st);
    BINDER_CUDA(cudaGetLastError());
}

void launch_nu_sample(DevState *st, int sample_gamma, int every, int N, long V, double rho_p,
                      const double eta2[3], uint64_t seed, uint32_t chain, cudaStream_t s,
                      int chains) {
    count_launch(), nu_sample_kernel<<<chains, 1, 0, s>>>(st, sample_gamma, every, N, V, rho_p, eta2[0], eta2[1],
                                     eta2[2], seed, chain);
    BINDER_CUDA(cudaGetLastError());
}

void launch_em_finish(DevState *st, double *stats, int max_iter, double th, double nzv,
                      cudaStream_t s) {
    count_launch(), em_finish_kernel<<<1, 1, 0, s>>>(st, stats, max_iter, th, nzv);
    BINDER_CUDA(cudaGetLastError());
}

void launch_sweep_end(const float *d, double *mean, double *m2, long V, int N, int N_b,
                      int total, DevState *st, cudaStream_t s, int chains) {
    int dev = 0, sms = 148;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    long need = (V + 255) / 256;
    long g = need < (long)sms * 8 ? (need < 1 ? 1 : need) : (long)sms * 8;
    if (chains > 1) g = (g + chains - 1) / chains;  // the same total CTAs over the chains
    const dim3 grid((unsigned)g, (unsigned)chains);
    BINDER_CHECK(N == 2 || N == 3, "Welford moments need N = 2 or 3");
    if (N == 3) count_launch(), sweep_end_kernel<3><<<grid, 256, 0, s>>>(d, mean, m2, V, N_b, st);
    else count_launch(), sweep_end_kernel<2><<<grid, 256, 0, s>>>(d, mean, m2, V, N_b, st);
    BINDER_CUDA(cudaGetLastError());
    launch_sweep_advance(st, total, s, chains);
}

void launch_sweep_advance(DevState *st, int total, cudaStream_t s, int chains) {
    count_launch(), sweep_advance_kernel<<<chains, 1, 0, s>>>(st, total);
    BINDER_CUDA(cudaGetLastError());
}

}  // namespace binder
