// Jacobian determinants and topology correction in FP64.
//
// This file is compiled with -fmad=false: every determinant is evaluated with the reference's
// expression grouping and without fused multiply-adds, so the per-voxel Jacobians (and therefore
// the negative / out-of-range counts and the set of corners the limiter touches) equal the
// reference CPU backend's bit for bit on the same FP64 input.
#include <cmath>
#include <mutex>
#include <vector>

#include "layout.cuh"
#include "topology.cuh"
#include "transform.cuh"

namespace binder {

namespace {

// cofactor expansion along the first row with the reference's grouping
// (BINDER/src/cpu/utils.cpp:156-160, topology_correction_3D.cpp:286-288)
__device__ __forceinline__ double det3(double a00, double a01, double a02, double a10, double a11,
                                       double a12, double a20, double a21, double a22) {
    return a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) +
           a02 * (a10 * a21 - a11 * a20);
}

__device__ __forceinline__ unsigned long long ordered(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double unordered(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    double v;
    memcpy(&v, &b, sizeof(v));
    return v;
}

struct Red {
    unsigned long long mn, mx;
    unsigned long long below, above, negative;
    double sum[3];
    int count;  // flagged cells (limiter list length)
    int pad;
};

// BINDER/src/cpu/utils.cpp:100-345.  Element (p, m) of the field is f[p*ps + m*cs].
__global__ void jacobian_kernel(const double *f, long ps, long cs, int nx, int ny, int nz,
                                double vol, double *J, double e1, double e2, Red *red) {
    const long V = (long)nx * ny * nz;
    const long yz = (long)ny * nz;
    // corner order of the reference: fff, bff, fbf, ffb, bbf, bfb, fbb, bbb
    const int dir[8][3] = {{1, 1, 1},  {-1, 1, 1},  {1, -1, 1},  {1, 1, -1},
                           {-1, -1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1}};
    double lmin = 1e300, lmax = -1e300;
    unsigned long long lb = 0, la = 0, ln = 0;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / yz), y = (int)((p / nz) % ny), z = (int)(p % nz);
        double w0[3];
        for (int m = 0; m < 3; ++m) w0[m] = f[p * ps + m * cs];
        double tot = 0.0;
        int valid = 0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int sx = dir[c][0], sy = dir[c][1], sz = dir[c][2];
            if ((sx > 0 && x >= nx - 1) || (sx < 0 && x <= 0)) continue;
            if ((sy > 0 && y >= ny - 1) || (sy < 0 && y <= 0)) continue;
            if ((sz > 0 && z >= nz - 1) || (sz < 0 && z <= 0)) continue;
            const long qx = p + sx * yz, qy = p + sy * nz, qz = p + sz;
            double col[3][3];  // [axis][component]
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                const double ax = f[qx * ps + m * cs], ay = f[qy * ps + m * cs],
                             az = f[qz * ps + m * cs];
                col[0][m] = sx > 0 ? ax - w0[m] : w0[m] - ax;
                col[1][m] = sy > 0 ? ay - w0[m] : w0[m] - ay;
                col[2][m] = sz > 0 ? az - w0[m] : w0[m] - az;
            }
            const double jc = det3(col[0][0], col[1][0], col[2][0], col[0][1], col[1][1], col[2][1],
                                   col[0][2], col[1][2], col[2][2]) * vol;
            tot += jc;
            valid++;
        }
        const double jv = valid > 0 ? tot / valid : 1.0;
        if (J) J[p] = jv;
        lmin = fmin(lmin, jv);
        lmax = fmax(lmax, jv);
        lb += jv < e1;
        la += jv > e2;
        ln += jv < 0.0;
    }
    if (red) {
        // warp-level first, then one atomic per warp
        for (int o = 16; o > 0; o >>= 1) {
            lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
            lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
            lb += __shfl_xor_sync(0xffffffffu, lb, o);
            la += __shfl_xor_sync(0xffffffffu, la, o);
            ln += __shfl_xor_sync(0xffffffffu, ln, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&red->mn, ordered(lmin));
            atomicMax(&red->mx, ordered(lmax));
            if (lb) atomicAdd(&red->below, lb);
            if (la) atomicAdd(&red->above, la);
            if (ln) atomicAdd(&red->negative, ln);
        }
    }
}

// BINDER/src/cpu/utils.cpp:10-98: the 2D Jacobian averaged over the 4 one-sided corners (orders
// fxfy, bxfy, fxby, bxby), each the determinant of the forward / backward differences, with the
// reference's expression grouping.  Element (p, m) of the field is f[p*ps + m*cs]; J and red are
// optional, as in jacobian_kernel.
__global__ void jacobian2d_kernel(const double *f, long ps, long cs, int nx, int ny, double vol,
                                  double *J, double e1, double e2, Red *red) {
    const long V = (long)nx * ny;
    const int dir[4][2] = {{1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    double lmin = 1e300, lmax = -1e300;
    unsigned long long lb = 0, la = 0, ln = 0;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ny), y = (int)(p % ny);
        const double w0 = f[p * ps], w1 = f[p * ps + cs];
        double tot = 0.0;
        int valid = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int sx = dir[c][0], sy = dir[c][1];
            if ((sx > 0 && x >= nx - 1) || (sx < 0 && x <= 0)) continue;
            if ((sy > 0 && y >= ny - 1) || (sy < 0 && y <= 0)) continue;
            const long qx = p + (long)sx * ny, qy = p + sy;
            const double bx0 = f[qx * ps], bx1 = f[qx * ps + cs];
            const double by0 = f[qy * ps], by1 = f[qy * ps + cs];
            const double ax0 = sx > 0 ? bx0 - w0 : w0 - bx0;
            const double ax1 = sx > 0 ? bx1 - w1 : w1 - bx1;
            const double ay0 = sy > 0 ? by0 - w0 : w0 - by0;
            const double ay1 = sy > 0 ? by1 - w1 : w1 - by1;
            tot += (ax0 * ay1 - ay0 * ax1) * vol;
            valid++;
        }
        const double jv = valid > 0 ? tot / valid : 1.0;
        if (J) J[p] = jv;
        lmin = fmin(lmin, jv);
        lmax = fmax(lmax, jv);
        lb += jv < e1;
        la += jv > e2;
        ln += jv < 0.0;
    }
    if (red) {
        for (int o = 16; o > 0; o >>= 1) {
            lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
            lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
            lb += __shfl_xor_sync(0xffffffffu, lb, o);
            la += __shfl_xor_sync(0xffffffffu, la, o);
            ln += __shfl_xor_sync(0xffffffffu, ln, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&red->mn, ordered(lmin));
            atomicMax(&red->mx, ordered(lmax));
            if (lb) atomicAdd(&red->below, lb);
            if (la) atomicAdd(&red->above, la);
            if (ln) atomicAdd(&red->negative, ln);
        }
    }
}

// topology_correction_3D.cpp:488-607: the 8 vertex Jacobians of every cell, in the vertex order
// 000, 100, 010, 001, 011, 101, 110, 111, each from the three cell edges through its vertex.
// Positions are SoA [3][V].
__global__ void corner_kernel(const double *pos, int nx, int ny, int nz, double vol, double e1,
                              double e2, double *Jc, Red *red) {
    const long V = (long)nx * ny * nz;
    const long cy = ny - 1, cz = nz - 1;
    const long cells = (long)(nx - 1) * cy * cz;
    const int vert[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                            {0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
    unsigned long long lb = 0, la = 0;
    for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < cells;
         cell += (long)gridDim.x * blockDim.x) {
        const int x = (int)(cell / (cy * cz)), y = (int)((cell / cz) % cy), z = (int)(cell % cz);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int vx = vert[c][0], vy = vert[c][1], vz = vert[c][2];
            const long pw = ((long)(x + vx) * ny + (y + vy)) * nz + (z + vz);
            const long pxn = ((long)(x + 1 - vx) * ny + (y + vy)) * nz + (z + vz);
            const long pyn = ((long)(x + vx) * ny + (y + 1 - vy)) * nz + (z + vz);
            const long pzn = ((long)(x + vx) * ny + (y + vy)) * nz + (z + 1 - vz);
            double col[3][3];
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                const double w = pos[m * V + pw];
                const double a = pos[m * V + pxn], b = pos[m * V + pyn], d = pos[m * V + pzn];
                col[0][m] = vx ? w - a : a - w;
                col[1][m] = vy ? w - b : b - w;
                col[2][m] = vz ? w - d : d - w;
            }
            double j = det3(col[0][0], col[1][0], col[2][0], col[0][1], col[1][1], col[2][1],
                            col[0][2], col[1][2], col[2][2]);
            j *= vol;
            Jc[cell * 8 + c] = j;
            lb += j < e1;
            la += j > e2;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        lb += __shfl_xor_sync(0xffffffffu, lb, o);
        la += __shfl_xor_sync(0xffffffffu, la, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (lb) atomicAdd(&red->below, lb);
        if (la) atomicAdd(&red->above, la);
    }
}

// topology_correction_3D.cpp:172-245: periodic forward differences, g[(n1*3+n2)][p] =
// (pos_n1(p + e_n2) - pos_n1(p)) / vs[n1]
__global__ void gradient_kernel(const double *pos, int nx, int ny, int nz, double v0, double v1,
                                double v2, double *g) {
    const long V = (long)nx * ny * nz;
    const double vs[3] = {v0, v1, v2};
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ((long)ny * nz)), y = (int)((p / nz) % ny), z = (int)(p % nz);
        const int x2 = x + 1 > nx - 1 ? x + 1 - nx : x + 1;
        const int y2 = y + 1 > ny - 1 ? y + 1 - ny : y + 1;
        const int z2 = z + 1 > nz - 1 ? z + 1 - nz : z + 1;
        const long px = ((long)x2 * ny + y) * nz + z, py = ((long)x * ny + y2) * nz + z,
                   pz = ((long)x * ny + y) * nz + z2;
#pragma unroll
        for (int n1 = 0; n1 < 3; ++n1) {
            const double c = pos[n1 * V + p];
            g[(n1 * 3 + 0) * V + p] = (pos[n1 * V + px] - c) / vs[n1];
            g[(n1 * 3 + 1) * V + p] = (pos[n1 * V + py] - c) / vs[n1];
            g[(n1 * 3 + 2) * V + p] = (pos[n1 * V + pz] - c) / vs[n1];
        }
    }
}

__global__ void flag_cells_kernel(const double *Jc, int nx, int ny, int nz, double e1, double e2,
                                  int *list, Red *red) {
    const long cells = (long)(nx - 1) * (ny - 1) * (nz - 1);
    for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < cells;
         cell += (long)gridDim.x * blockDim.x) {
        bool any = false;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const double j = Jc[cell * 8 + c];
            any |= (j < e1 || j > e2);
        }
        if (any) list[atomicAdd(&red->count, 1)] = (int)cell;
    }
}

// the limiter step of one flagged corner (topology_correction_3D.cpp:279-345,
// topology_correction_2D.cpp:257-309): J the corner's N x N gradient matrix (column n2 read at
// vertex n2), replaced by (1 - a) J + a I.  The reference steps
// alpha by 0.1 (capped at 1) until det((1 - alpha) J + alpha I) lies in [e1, e2], at most 11
// steps, then takes one step more.  The alphas are constants, so the trial determinants are
// evaluated independently, a group at a time (the same expressions the loop evaluates), and the
// first one in range picks the step: the walk, one corner after another, gains the ILP.
template <int N>
__device__ __forceinline__ double detn(const double (&J)[N][N]) {
    if constexpr (N == 2)
        return J[0][0] * J[1][1] - J[0][1] * J[1][0];
    else
        return det3(J[0][0], J[0][1], J[0][2], J[1][0], J[1][1], J[1][2], J[2][0], J[2][1], J[2][2]);
}

template <int N>
__device__ __forceinline__ void limit_corner(double (&J)[N][N], double e1, double e2,
                                             bool &capped) {
    constexpr int kSteps = 11;
    double al[kSteps + 2];  // al[k]: alpha after k steps (constant-folded)
    al[0] = 0.0;
#pragma unroll
    for (int k = 1; k < kSteps + 2; ++k) {
        al[k] = al[k - 1] + 0.1;
        if (al[k] > 1.0) al[k] = 1.0;
    }
    const double det0 = detn<N>(J);
    // k steps taken (the first k whose determinant lies in [e1, e2]): the final alpha is al[k + 1]
    double alpha = al[1];
    if (det0 > e2 || det0 < e1) {
        bool none = true;  // alpha == 1 (identity) tried as well: [e1, e2] misses 1
        alpha = al[kSteps + 1];
        // trials in groups of kGroup (independent within a group), stopping at the first group
        // with a determinant in range
        constexpr int kGroup = 4;
#pragma unroll
        for (int t0 = 1; t0 <= kSteps; t0 += kGroup) {
            const int t1 = t0 + kGroup - 1 < kSteps ? t0 + kGroup - 1 : kSteps;
#pragma unroll
            for (int t = t1; t >= t0; --t) {
                const double a = al[t];
                double Jn[N][N];
                for (int n1 = 0; n1 < N; ++n1)
                    for (int n2 = 0; n2 < N; ++n2)
                        Jn[n1][n2] = (1 - a) * J[n1][n2] + a * (n1 == n2 ? 1.0 : 0.0);
                const double det = detn<N>(Jn);
                if (!(det > e2 || det < e1)) {
                    alpha = al[t + 1];
                    none = false;
                }
            }
            if (!none) break;
        }
        if (none) capped = true;
    }
    for (int n1 = 0; n1 < N; ++n1)
        for (int n2 = 0; n2 < N; ++n2)
            J[n1][n2] = (1 - alpha) * J[n1][n2] + alpha * (n1 == n2 ? 1.0 : 0.0);
}

// limit_corner by a group of 16 lanes holding the same J: lane t (1 <= t <= 11) evaluates trial
// t, and the lowest lane whose determinant lies in [e1, e2] picks the step.  The same expressions
// and the same choice as limit_corner; every lane of the group ends with the new J.  gmask names
// the group's lanes, which all take this call together.
__device__ __forceinline__ void limit_corner_lanes(double (&J)[2][2], double e1, double e2,
                                                   bool &capped, int gl, unsigned gmask,
                                                   double at, double an) {
    const double det0 = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    double alpha = 0.1;  // one step from 0
    if (det0 > e2 || det0 < e1) {  // uniform across the group
        bool in = false;
        if (gl >= 1 && gl <= 11) {
            double Jn[2][2];
            for (int n1 = 0; n1 < 2; ++n1)
                for (int n2 = 0; n2 < 2; ++n2)
                    Jn[n1][n2] = (1 - at) * J[n1][n2] + at * (n1 == n2 ? 1.0 : 0.0);
            const double det = Jn[0][0] * Jn[1][1] - Jn[0][1] * Jn[1][0];
            in = !(det > e2 || det < e1);
        }
        const unsigned b = __ballot_sync(gmask, in) & gmask;
        const int k = b ? __ffs((int)b) - 1 : -1;  // lane of the warp
        alpha = __shfl_sync(gmask, an, k < 0 ? 11 : (k & 15), 16);  // al[k + 1], or al[12] = 1
        if (k < 0) capped = true;
    }
    for (int n1 = 0; n1 < 2; ++n1)
        for (int n2 = 0; n2 < 2; ++n2)
            J[n1][n2] = (1 - alpha) * J[n1][n2] + alpha * (n1 == n2 ? 1.0 : 0.0);
}

// topology_correction_3D.cpp:247-332.  The reference visits cells in lexicographic order and a
// cell's 8 corners in order; a cell reads and writes gradients only inside its 2x2x2 footprint,
// so two cells interact only if they differ by at most 1 along every axis.  Level 4x + 2y + z
// orders every such pair exactly as the lexicographic walk does and never puts two of them on
// the same level, so processing levels in increasing order (cells of one level in parallel)
// reproduces the sequential result exactly.  One CTA of 256 threads; levels are separated by
// __syncthreads.
__global__ void __launch_bounds__(256) limiter_kernel(const int *list, int *sorted, const double *Jc,
                                                       double *g, int nx, int ny, int nz,
                                                       double e1, double e2, int nlev, Red *red,
                                                       unsigned *flags) {
    extern __shared__ int sh[];
    int *off = sh;             // nlev + 1
    int *cur = sh + nlev + 1;  // nlev
    const long V = (long)nx * ny * nz;
    const long cy = ny - 1, cz = nz - 1;
    const int n = red->count;
    for (int l = threadIdx.x; l < nlev + 1; l += blockDim.x) off[l] = 0;
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const long cell = list[q];
        const int x = (int)(cell / (cy * cz)), y = (int)((cell / cz) % cy), z = (int)(cell % cz);
        atomicAdd(&off[4 * x + 2 * y + z + 1], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int l = 0; l < nlev; ++l) off[l + 1] += off[l];
    __syncthreads();
    for (int l = threadIdx.x; l < nlev; l += blockDim.x) cur[l] = off[l];
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const long cell = list[q];
        const int x = (int)(cell / (cy * cz)), y = (int)((cell / cz) % cy), z = (int)(cell % cz);
        sorted[atomicAdd(&cur[4 * x + 2 * y + z], 1)] = (int)cell;
    }
    __syncthreads();
    const int vert[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                            {0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
    bool capped = false;
    for (int l = 0; l < nlev; ++l) {
        const int beg = off[l], end = off[l + 1];
        if (beg == end) continue;  // uniform: every thread reads the same shared value
        for (int q = beg + threadIdx.x; q < end; q += blockDim.x) {
            const long cell = sorted[q];
            const int x = (int)(cell / (cy * cz)), y = (int)((cell / cz) % cy), z = (int)(cell % cz);
            for (int c = 0; c < 8; ++c) {
                const double jv = Jc[cell * 8 + c];
                if (!(jv < e1 || jv > e2)) continue;
                long gp[3];
                for (int n2 = 0; n2 < 3; ++n2) {
                    int o[3] = {vert[c][0], vert[c][1], vert[c][2]};
                    o[n2] = 0;
                    gp[n2] = ((long)(x + o[0]) * ny + (y + o[1])) * nz + (z + o[2]);
                }
                double J[3][3];
                for (int n1 = 0; n1 < 3; ++n1)
                    for (int n2 = 0; n2 < 3; ++n2) J[n1][n2] = g[(n1 * 3 + n2) * V + gp[n2]];
                limit_corner<3>(J, e1, e2, capped);
                for (int n1 = 0; n1 < 3; ++n1)
                    for (int n2 = 0; n2 < 3; ++n2) g[(n1 * 3 + n2) * V + gp[n2]] = J[n1][n2];
            }
        }
        __syncthreads();
    }
    if (capped) atomicOr(flags, (unsigned)kFlagLimiterCapped);
}

// backward-difference divergence (periodic) of each component's gradient row; the reference's
// Fourier factor (e^{-i theta} - 1) applied to the gradient spectra is minus its transform
__global__ void divergence_kernel(const double *g, int nx, int ny, int nz, double *div) {
    const long V = (long)nx * ny * nz;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ((long)ny * nz)), y = (int)((p / nz) % ny), z = (int)(p % nz);
        const int xm = x == 0 ? nx - 1 : x - 1, ym = y == 0 ? ny - 1 : y - 1,
                  zm = z == 0 ? nz - 1 : z - 1;
        const long px = ((long)xm * ny + y) * nz + z, py = ((long)x * ny + ym) * nz + z,
                   pz = ((long)x * ny + y) * nz + zm;
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const double *gx = g + (n * 3 + 0) * V, *gy = g + (n * 3 + 1) * V,
                         *gz = g + (n * 3 + 2) * V;
            div[n * V + p] = (gx[p] - gx[px]) + (gy[p] - gy[py]) + (gz[p] - gz[pz]);
        }
    }
}

// topology_correction_2D.cpp:165-207: the 4 corner Jacobians of every cell in the vertex order
// 00, 10, 01, 11 (the reference's Jff, Jbf, Jfb, Jbb).  Corner (vx, vy) pairs the x edge at
// y + vy with the y edge at x + vx (hi - lo each).  `below` / `above` count cells with a corner
// out of range, as the reference's counters do.  Positions are SoA [2][V].
__global__ void corner2d_kernel(const double *pos, int nx, int ny, double vol, double e1,
                                double e2, double *Jc, Red *red) {
    const long V = (long)nx * ny;
    const long cy = ny - 1;
    const long cells = (long)(nx - 1) * cy;
    unsigned long long lb = 0, la = 0;
    for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < cells;
         cell += (long)gridDim.x * blockDim.x) {
        const int x = (int)(cell / cy), y = (int)(cell % cy);
        const long p00 = (long)x * ny + y, p10 = p00 + ny;
        const double X00 = pos[p00], X01 = pos[p00 + 1], X10 = pos[p10], X11 = pos[p10 + 1];
        const double Y00 = pos[V + p00], Y01 = pos[V + p00 + 1], Y10 = pos[V + p10],
                     Y11 = pos[V + p10 + 1];
        bool lo = false, hi = false;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int vx = c & 1, vy = c >> 1;
            // x edge at y + vy, y edge at x + vx
            const double ex0 = vy ? X11 - X01 : X10 - X00, ex1 = vy ? Y11 - Y01 : Y10 - Y00;
            const double ey0 = vx ? X11 - X10 : X01 - X00, ey1 = vx ? Y11 - Y10 : Y01 - Y00;
            const double j = (ex0 * ey1 - ey0 * ex1) * vol;
            Jc[cell * 4 + c] = j;
            lo |= j < e1;
            hi |= j > e2;
        }
        lb += lo;
        la += hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        lb += __shfl_xor_sync(0xffffffffu, lb, o);
        la += __shfl_xor_sync(0xffffffffu, la, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (lb) atomicAdd(&red->below, lb);
        if (la) atomicAdd(&red->above, la);
    }
}

// topology_correction_2D.cpp:209-246: periodic forward differences, g[(n1*2+n2)][p] =
// (pos_n1(p + e_n2) - pos_n1(p)) / vs[n1]
__global__ void gradient2d_kernel(const double *pos, int nx, int ny, double v0, double v1,
                                  double *g) {
    const long V = (long)nx * ny;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ny), y = (int)(p % ny);
        const long px = (long)(x + 1 > nx - 1 ? x + 1 - nx : x + 1) * ny + y;
        const long py = (long)x * ny + (y + 1 > ny - 1 ? y + 1 - ny : y + 1);
        const double c0 = pos[p], c1 = pos[V + p];
        g[0 * V + p] = (pos[px] - c0) / v0;
        g[1 * V + p] = (pos[py] - c0) / v0;
        g[2 * V + p] = (pos[V + px] - c1) / v1;
        g[3 * V + p] = (pos[V + py] - c1) / v1;
    }
}

__global__ void flag_cells2d_kernel(const double *Jc, int nx, int ny, double e1, double e2,
                                    int *list, Red *red) {
    const long cells = (long)(nx - 1) * (ny - 1);
    for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < cells;
         cell += (long)gridDim.x * blockDim.x) {
        bool any = false;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double j = Jc[cell * 4 + c];
            any |= (j < e1 || j > e2);
        }
        if (any) list[atomicAdd(&red->count, 1)] = (int)cell;
    }
}

// topology_correction_2D.cpp:248-313.  Cells are visited in lexicographic order and a cell's 4
// corners in order; a cell touches gradients only at its own 2x2 nodes, so two cells interact
// only if they differ by at most 1 along both axes.  Level 2x + y orders every such pair as the
// lexicographic walk does and never puts two of them on one level, so levels in increasing order
// (cells of one level in parallel) reproduce the sequential result exactly.  Column n2 of a
// corner's matrix is read at the corner's vertex with its n2 bit cleared, so a corner reads
// nodes (0, vy) and (vx, 0) of its cell and node (1, 1) is never read.
//
// The walk is a chain of some 3 max(nx, ny) short levels, so its time is the chain's length times
// the latency of one level.  One warp walks (a warp barrier per level), on shared-memory copies:
// the block first gives every node a flagged corner reads a slot (a V-sized map, -1 between
// calls), gathers those nodes' gradients and the cells' flagged-corner masks, and afterwards
// scatters the gradients back.  More than kStageCells cells or kStageNodes nodes: the warp walks
// global memory.  Either way the arithmetic and its order are those of the sequential walk.
constexpr int kLimiterThreads = 1024;
constexpr int kStageCells = 4096;
constexpr int kStageNodes = 6016;
// shared bytes of the staged walk: per node 4 gradients, per cell 3 slots and the corner mask
// (16 bits each)
constexpr size_t kStageBytes =
    kStageNodes * 4 * sizeof(double) + kStageCells * 4 * sizeof(unsigned short);
constexpr unsigned short kNoSlot = 0xffff;
static_assert(kStageNodes < kNoSlot, "slots are 16-bit");

__global__ void __launch_bounds__(kLimiterThreads) limiter2d_kernel(const int *list, int *sorted,
                                                                    const double *Jc, double *g,
                                                                    int nx, int ny, double e1,
                                                                    double e2, int nlev, Red *red,
                                                                    unsigned *flags, int *slot) {
    extern __shared__ __align__(16) unsigned char lsm[];
    int *off = reinterpret_cast<int *>(lsm);  // nlev + 1
    int *cur = off + nlev + 1;                // nlev
    const size_t o = ((size_t)(2 * nlev + 1) * sizeof(int) + 15) & ~(size_t)15;
    double *gs = reinterpret_cast<double *>(lsm + o);  // [kStageNodes][4]
    // [kStageCells][4]: slots of nodes (0, 0), (1, 0), (0, 1), then the flagged-corner mask
    unsigned short *cs = reinterpret_cast<unsigned short *>(gs + (size_t)kStageNodes * 4);
    __shared__ int nslot;
    const long V = (long)nx * ny;
    const long cy = ny - 1;
    const int n = red->count;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int l = tid; l < nlev + 1; l += blockDim.x) off[l] = 0;
    if (tid == 0) nslot = 0;
    __syncthreads();
    for (int q = tid; q < n; q += blockDim.x) {
        const long cell = list[q];
        atomicAdd(&off[2 * (int)(cell / cy) + (int)(cell % cy) + 1], 1);
    }
    __syncthreads();
    if (tid == 0)
        for (int l = 0; l < nlev; ++l) off[l + 1] += off[l];
    __syncthreads();
    for (int l = tid; l < nlev; l += blockDim.x) cur[l] = off[l];
    __syncthreads();
    for (int q = tid; q < n; q += blockDim.x) {
        const long cell = list[q];
        sorted[atomicAdd(&cur[2 * (int)(cell / cy) + (int)(cell % cy)], 1)] = (int)cell;
    }
    __syncthreads();
    bool staged = false;
    if (n <= kStageCells) {
        // claim a slot for every node (0, 0), (1, 0), (0, 1) a flagged corner reads
        for (int q = tid; q < n; q += blockDim.x) {
            const long cell = sorted[q];
            const int x = (int)(cell / cy), y = (int)(cell % cy);
            unsigned m = 0;
            for (int c = 0; c < 4; ++c) {
                const double jv = Jc[cell * 4 + c];
                m |= (jv < e1 || jv > e2) ? 1u << c : 0u;
            }
            cs[q * 4 + 3] = (unsigned short)m;
            const unsigned need = ((m & 1u) ? 1u : 0u) | ((m & 2u) ? 3u : 0u) |
                                  ((m & 4u) ? 5u : 0u) | ((m & 8u) ? 6u : 0u);  // bit d: node d
            int old[3];
            long p[3];
            for (int d = 0; d < 3; ++d) {
                p[d] = (long)(x + (d & 1)) * ny + (y + (d >> 1));
                old[d] = (need >> d & 1u) ? atomicCAS(&slot[p[d]], -1, -2) : 0;
            }
            for (int d = 0; d < 3; ++d)
                if ((need >> d & 1u) && old[d] == -1) {
                    slot[p[d]] = atomicAdd(&nslot, 1);
                }
        }
        __syncthreads();  // every claimed node holds its slot number
        const int ns = nslot;
        if (ns <= kStageNodes) {
            staged = true;
            // slots of the cells and the nodes' gradients (a node shared by cells is gathered
            // once per cell, the same values into the same slot)
            for (int q = tid; q < n; q += blockDim.x) {
                const long cell = sorted[q];
                const int x = (int)(cell / cy), y = (int)(cell % cy);
                const unsigned m = cs[q * 4 + 3];
                const unsigned need = ((m & 1u) ? 1u : 0u) | ((m & 2u) ? 3u : 0u) |
                                      ((m & 4u) ? 5u : 0u) | ((m & 8u) ? 6u : 0u);
                for (int d = 0; d < 3; ++d) {
                    unsigned short sl = kNoSlot;
                    if (need >> d & 1u) {
                        const long p = (long)(x + (d & 1)) * ny + (y + (d >> 1));
                        sl = (unsigned short)slot[p];
                        for (int k = 0; k < 4; ++k) gs[sl * 4 + k] = g[k * V + p];
                    }
                    cs[q * 4 + d] = sl;
                }
            }
        } else {
            // too many nodes: release the map and walk global memory
            for (int q = tid; q < n; q += blockDim.x) {
                const long cell = sorted[q];
                const int x = (int)(cell / cy), y = (int)(cell % cy);
                for (int d = 0; d < 3; ++d) slot[(long)(x + (d & 1)) * ny + (y + (d >> 1))] = -1;
            }
        }
        __syncthreads();
    }
    bool capped = false;
    if (tid < 32) {
        // lane gl of a 16-lane group: alpha of trial gl and of the step after it
        const int grp = lane >> 4, gl = lane & 15;
        const unsigned gmask = grp ? 0xffff0000u : 0x0000ffffu;
        double at = 0.0, an = 0.0, a = 0.0;
        for (int t = 0; t <= 11; ++t) {
            const double a1 = fmin(a + 0.1, 1.0);  // alpha += 0.1, capped at 1
            if (t == gl) {
                at = a;
                an = a1;
            }
            a = a1;
        }
        for (int l = 0; l < nlev; ++l) {
            const int beg = off[l], end = off[l + 1];
            if (beg == end) continue;  // uniform: every lane reads the same shared value
            if (staged && end - beg <= 2) {
                // one or two cells: a group of 16 lanes per cell, the trials across the lanes
                const int q = beg + grp;
                if (q < end) {  // uniform across the group
                    const unsigned m = cs[q * 4 + 3];
                    for (int c = 0; c < 4; ++c) {
                        if (!(m >> c & 1u)) continue;
                        const int vx = c & 1, vy = c >> 1;
                        const int sv[2] = {cs[q * 4 + 2 * vy], cs[q * 4 + vx]};
                        double J[2][2];
                        for (int n1 = 0; n1 < 2; ++n1)
                            for (int n2 = 0; n2 < 2; ++n2)
                                J[n1][n2] = gs[sv[n2] * 4 + n1 * 2 + n2];
                        limit_corner_lanes(J, e1, e2, capped, gl, gmask, at, an);
                        // every lane stores the same values; each reads its own store back
                        for (int n1 = 0; n1 < 2; ++n1)
                            for (int n2 = 0; n2 < 2; ++n2)
                                gs[sv[n2] * 4 + n1 * 2 + n2] = J[n1][n2];
                    }
                }
                __syncwarp();
                continue;
            }
            for (int q = beg + lane; q < end; q += 32) {
                if (staged) {
                    const unsigned m = cs[q * 4 + 3];
                    for (int c = 0; c < 4; ++c) {
                        if (!(m >> c & 1u)) continue;
                        const int vx = c & 1, vy = c >> 1;
                        const int sv[2] = {cs[q * 4 + 2 * vy], cs[q * 4 + vx]};
                        double J[2][2];
                        for (int n1 = 0; n1 < 2; ++n1)
                            for (int n2 = 0; n2 < 2; ++n2)
                                J[n1][n2] = gs[sv[n2] * 4 + n1 * 2 + n2];
                        limit_corner<2>(J, e1, e2, capped);
                        for (int n1 = 0; n1 < 2; ++n1)
                            for (int n2 = 0; n2 < 2; ++n2)
                                gs[sv[n2] * 4 + n1 * 2 + n2] = J[n1][n2];
                    }
                } else {
                    const long cell = sorted[q];
                    const int x = (int)(cell / cy), y = (int)(cell % cy);
                    for (int c = 0; c < 4; ++c) {
                        const double jv = Jc[cell * 4 + c];
                        if (!(jv < e1 || jv > e2)) continue;
                        const int vx = c & 1, vy = c >> 1;
                        const long gp[2] = {(long)x * ny + (y + vy), (long)(x + vx) * ny + y};
                        double J[2][2];
                        for (int n1 = 0; n1 < 2; ++n1)
                            for (int n2 = 0; n2 < 2; ++n2)
                                J[n1][n2] = g[(n1 * 2 + n2) * V + gp[n2]];
                        limit_corner<2>(J, e1, e2, capped);
                        for (int n1 = 0; n1 < 2; ++n1)
                            for (int n2 = 0; n2 < 2; ++n2)
                                g[(n1 * 2 + n2) * V + gp[n2]] = J[n1][n2];
                    }
                }
            }
            __syncwarp();
        }
    }
    if (staged) {
        __syncthreads();
        // scatter back (a shared node once per cell, the same values) and release the map
        for (int q = tid; q < n; q += blockDim.x) {
            const long cell = sorted[q];
            const int x = (int)(cell / cy), y = (int)(cell % cy);
            for (int d = 0; d < 3; ++d) {
                const unsigned short sl = cs[q * 4 + d];
                if (sl == kNoSlot) continue;
                const long p = (long)(x + (d & 1)) * ny + (y + (d >> 1));
                for (int k = 0; k < 4; ++k) g[k * V + p] = gs[sl * 4 + k];
                slot[p] = -1;
            }
        }
    }
    if (capped) atomicOr(flags, (unsigned)kFlagLimiterCapped);
}

// backward-difference divergence (periodic) of each component's 2D gradient row
__global__ void divergence2d_kernel(const double *g, int nx, int ny, double *div) {
    const long V = (long)nx * ny;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x) {
        const int x = (int)(p / ny), y = (int)(p % ny);
        const long px = (long)(x == 0 ? nx - 1 : x - 1) * ny + y;
        const long py = (long)x * ny + (y == 0 ? ny - 1 : y - 1);
#pragma unroll
        for (int n = 0; n < 2; ++n) {
            const double *gx = g + (n * 2 + 0) * V, *gy = g + (n * 2 + 1) * V;
            div[n * V + p] = (gx[p] - gx[px]) + (gy[p] - gy[py]);
        }
    }
}

__global__ void sum_kernel(const double *pos, long V, int N, Red *red) {
    double s[3] = {0.0, 0.0, 0.0};
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x)
        for (int n = 0; n < N; ++n) s[n] += pos[n * V + p];
    for (int n = 0; n < N; ++n) {
        double v = warp_sum(s[n]);
        if ((threadIdx.x & 31) == 0) atomicAdd(&red->sum[n], v);
    }
}

// AoS grid-unit field [V][N] -> SoA physical [N][V] (times the voxel size) and back
struct Scale {
    double v[3];
};
__global__ void aos_to_soa_kernel(const double *aos, long V, int N, Scale sc, double *soa) {
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x)
        for (int n = 0; n < N; ++n) soa[n * V + p] = aos[p * N + n] * sc.v[n];
}
__global__ void soa_to_aos_kernel(const double *soa, long V, int N, Scale sc, double *aos) {
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x)
        for (int n = 0; n < N; ++n) aos[p * N + n] = soa[n * V + p] / sc.v[n];
}

int grid_for(long work) {
    int dev = 0, sms = 148;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long need = (work + 255) / 256;
    const long cap = (long)sms * 8;
    return (int)(need < 1 ? 1 : (need < cap ? need : cap));
}

// device buffer from the stream-ordered pool, released on the stream it was allocated on
template <typename T>
struct DBuf {
    T *p = nullptr;
    cudaStream_t s = 0;
    DBuf() = default;
    DBuf(size_t n, cudaStream_t stream) : s(stream) { p = dev_alloc_n<T>(n, s); }
    void alloc(size_t n, cudaStream_t stream) {
        dev_free(p, s);
        s = stream;
        p = dev_alloc_n<T>(n, s);
    }
    ~DBuf() { dev_free(p, s); }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
};

void reset_red(Red *r, cudaStream_t s) {
    Red h{};
    h.mn = ~0ull;
    h.mx = 0ull;
    BINDER_CUDA(cudaMemcpyAsync(r, &h, sizeof(Red), cudaMemcpyHostToDevice, s));
}

Red read_red(const Red *r, cudaStream_t s) {
    Red h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, r, sizeof(Red), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    return h;
}

}  // namespace

void jacobian3d_device(const double *field_aos, int nx, int ny, int nz, const double vs[3],
                       double *J, cudaStream_t s) {
    const long V = (long)nx * ny * nz;
    count_launch(), jacobian_kernel<<<grid_for(V), 256, 0, s>>>(field_aos, 3, 1, nx, ny, nz,
                                                1.0 / (vs[0] * vs[1] * vs[2]), J, 0.0, 0.0, nullptr);
    BINDER_CUDA(cudaGetLastError());
}

void jacobian2d_device(const double *field_aos, int nx, int ny, const double vs[2], double *J,
                       cudaStream_t s) {
    const long V = (long)nx * ny;
    count_launch(), jacobian2d_kernel<<<grid_for(V), 256, 0, s>>>(
                        field_aos, 2, 1, nx, ny, 1.0 / (vs[0] * vs[1]), J, 0.0, 0.0, nullptr);
    BINDER_CUDA(cudaGetLastError());
}

void jacobian2d(const double *field_host, int nx, int ny, const double vs[2], double *J_host) {
    BINDER_CHECK(nx > 0 && ny > 0, "dimensions must be positive");
    const long V = (long)nx * ny;
    cudaStream_t s = nullptr;
    BINDER_CUDA(cudaStreamCreate(&s));
    try {
        DBuf<double> f(V * 2, s), J(V, s);
        BINDER_CUDA(cudaMemcpyAsync(f.p, field_host, sizeof(double) * V * 2, cudaMemcpyHostToDevice, s));
        jacobian2d_device(f.p, nx, ny, vs, J.p, s);
        BINDER_CUDA(cudaMemcpyAsync(J_host, J.p, sizeof(double) * V, cudaMemcpyDeviceToHost, s));
        BINDER_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamSynchronize(s);  // the buffers' stream-ordered frees
    cudaStreamDestroy(s);
}

// ---- Jacobian through a fixed device scratch array ------------------------------------------
// Some callers cannot afford cudaMalloc / cudaFree on every call: a framework whose caching
// allocator already holds most of the GPU's memory (a fresh cudaMalloc then fails even though the
// framework has room), or a loop that keeps other streams busy and cannot take the device-wide
// synchronisation cudaFree implies.  This variant stages the field, the determinants and the
// summary record in one array that is part of the library's device image, sized for grids of up
// to kJacobianNoAllocMaxVoxels voxels (16 MiB in all), so a call allocates nothing.
namespace {
constexpr size_t kNoAllocHeader = 256;  // the reduction record, padded
static_assert(sizeof(Red) <= kNoAllocHeader, "reduction record does not fit its slot");
// [Red | field: 3 * max doubles | J: max doubles]
static __device__ __align__(256) unsigned char
    g_jacobian_scratch[kNoAllocHeader + 4 * sizeof(double) * kJacobianNoAllocMaxVoxels];
constexpr int kNoAllocMaxDevices = 64;

// address of the scratch array on the current device, looked up once per device (with that
// device current) and kept for the life of the process; the lock guards only this table, not the
// scratch itself.  A cudaDeviceReset after the first call may place the module elsewhere in the
// next context, so the entry point does not support a device reset after its first call.
unsigned char *jacobian_scratch_address() {
    static std::mutex mu;
    static unsigned char *addr[kNoAllocMaxDevices] = {};
    int dev = -1;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CHECK(dev >= 0 && dev < kNoAllocMaxDevices, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        BINDER_CUDA(cudaGetSymbolAddress(&p, g_jacobian_scratch));
        addr[dev] = static_cast<unsigned char *>(p);
    }
    return addr[dev];
}

// the record's starting values: min/max as empty ordered keys, counts zero
__global__ void clear_red_kernel(Red *r) {
    r->mn = ~0ull;
    r->mx = 0ull;
    r->below = r->above = r->negative = 0ull;
    r->sum[0] = r->sum[1] = r->sum[2] = 0.0;
    r->count = 0;
    r->pad = 0;
}
}  // namespace

void jacobian3d_noalloc(const double *field_host, int nx, int ny, int nz, const double vs[3],
                        double *J_host, JacStats *stats) {
    BINDER_CHECK(nx > 0 && ny > 0 && nz > 0, "dimensions must be positive");
    const long V = (long)nx * ny * nz;
    if (V > kJacobianNoAllocMaxVoxels)
        throw Error(kInvalidArgument,
                    "grid of " + std::to_string(V) + " voxels exceeds the no-allocation limit of " +
                        std::to_string(kJacobianNoAllocMaxVoxels) + " voxels");
    unsigned char *base = jacobian_scratch_address();
    Red *red = reinterpret_cast<Red *>(base);
    double *df = reinterpret_cast<double *>(base + kNoAllocHeader);
    double *dj = df + 3 * kJacobianNoAllocMaxVoxels;
    // the calling thread's per-thread default stream: unlike the legacy stream 0 it does not
    // wait for (or hold up) work on the caller's other blocking streams
    const cudaStream_t s = cudaStreamPerThread;
    count_launch(), clear_red_kernel<<<1, 1, 0, s>>>(red);
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaMemcpyAsync(df, field_host, sizeof(double) * V * 3, cudaMemcpyHostToDevice, s));
    // e1 = e2 = 0: `below` and `above` count J < 0 and J > 0
    count_launch(), jacobian_kernel<<<grid_for(V), 256, 0, s>>>(
        df, 3, 1, nx, ny, nz, 1.0 / (vs[0] * vs[1] * vs[2]), dj, 0.0, 0.0, red);
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaMemcpyAsync(J_host, dj, sizeof(double) * V, cudaMemcpyDeviceToHost, s));
    Red h{};
    BINDER_CUDA(cudaMemcpyAsync(&h, red, sizeof(Red), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->jmin = unordered(h.mn);
        stats->jmax = unordered(h.mx);
        stats->below = (long long)h.below;
        stats->above = (long long)h.above;
        stats->negative = (long long)h.negative;
    }
}

namespace {
__global__ void float_soa_to_physical_kernel(const float *d, long V, int N, Scale sc, double *pos) {
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x)
        for (int n = 0; n < N; ++n) pos[n * V + p] = (double)d[n * V + p] * sc.v[n];
}
__global__ void physical_to_float_soa_kernel(const double *pos, long V, int N, Scale sc, float *d) {
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < V;
         p += (long)gridDim.x * blockDim.x)
        for (int n = 0; n < N; ++n) d[n * V + p] = (float)(pos[n * V + p] / sc.v[n]);
}
}  // namespace

struct TopologyWorkspace::Impl {
    int nx, ny, nz;
    int N;  // 3, or 2 for an image (nz == 1)
    long V, cells;
    cudaStream_t st;  // pool stream of every buffer
    // always present: what the Jacobian statistics need
    DBuf<double> pos;
    DBuf<Red> red;
    DBuf<unsigned> flags;
    // allocated when a correction first iterates (most calls find every Jacobian in range)
    bool ready = false;
    DBuf<double> grad, jc, div, t1, t2;
    DBuf<int> list, sorted;
    DBuf<int> slot;  // image node -> shared-memory slot of the 2D limiter, -1 between calls
    DBuf<double> H[3], cs[3];
    Impl(int x, int y, int z, cudaStream_t s)
        : nx(x), ny(y), nz(z), N(z == 1 ? 2 : 3), V((long)x * y * z),
          cells(z == 1 ? (long)(x - 1) * (y - 1) : (long)(x - 1) * (y - 1) * (z - 1)), st(s),
          pos(V * N, s), red(1, s), flags(1, s) {}
    void ensure() {
        if (ready) return;
        grad.alloc(V * N * N, st);
        jc.alloc(cells * (nz == 1 ? 4 : 8), st);
        div.alloc(V * N, st);
        t1.alloc(V * N, st);
        t2.alloc(V * N, st);
        list.alloc(cells, st);
        sorted.alloc(cells, st);
        if (nz == 1) {
            slot.alloc(V, st);
            BINDER_CUDA(cudaMemsetAsync(slot.p, 0xff, sizeof(int) * V, st));
        }
        const int dims[3] = {nx, ny, nz};
        const double pi = 3.14159265358979323846;
        for (int a = 0; a < 3; ++a) {
            const int n = dims[a];
            H[a].alloc((size_t)n * n, st);
            cs[a].alloc(n, st);
            std::vector<double> M((size_t)n * n), c(n);
            hartley_matrix(n, M.data());
            for (int k = 0; k < n; ++k) c[k] = std::cos(2.0 * pi * k / (n * 1.0));
            BINDER_CUDA(cudaMemcpyAsync(H[a].p, M.data(), sizeof(double) * n * n,
                                        cudaMemcpyHostToDevice, st));
            BINDER_CUDA(cudaMemcpyAsync(cs[a].p, c.data(), sizeof(double) * n,
                                        cudaMemcpyHostToDevice, st));
            BINDER_CUDA(cudaStreamSynchronize(st));  // the host tables go out of scope
        }
        ready = true;
    }
};

TopologyWorkspace::TopologyWorkspace(int nx, int ny, int nz, cudaStream_t s) {
    BINDER_CHECK(nx >= 2 && ny >= 2 && (nz >= 2 || nz == 1),
                 "topology correction needs at least 2 voxels per axis (nz == 1 for an image)");
    BINDER_CHECK(nx <= 256 && ny <= 256 && nz <= 256, "topology correction supports axes up to 256");
    impl_ = new Impl(nx, ny, nz, s);
}
TopologyWorkspace::~TopologyWorkspace() { delete impl_; }
double *TopologyWorkspace::positions() { return impl_->pos.p; }

// BINDER/src/cpu/topology_correction_3D.cpp:17-143 on the workspace's SoA physical positions
TopologyResult TopologyWorkspace::run(double e1, double e2, int max_outer, int max_inner,
                                      const double vs[3], cudaStream_t s) {
    if (impl_->N == 2) return run2d(e1, e2, max_outer, max_inner, vs, s);
    BINDER_CHECK(vs[0] > 0 && vs[1] > 0 && vs[2] > 0, "voxel sizes must be positive");
    Impl &w = *impl_;
    const int nx = w.nx, ny = w.ny, nz = w.nz;
    const long V = w.V, cells = w.cells;
    const double vol = 1.0 / (vs[0] * vs[1] * vs[2]);
    TopologyResult res{};
    BINDER_CUDA(cudaMemsetAsync(w.flags.p, 0, sizeof(unsigned), s));

    auto jac_stats = [&]() {
        reset_red(w.red.p, s);
        count_launch(), jacobian_kernel<<<grid_for(V), 256, 0, s>>>(w.pos.p, 1, V, nx, ny, nz, vol, nullptr, e1, e2,
                                                    w.red.p);
        BINDER_CUDA(cudaGetLastError());
        return read_red(w.red.p, s);
    };
    auto corners = [&]() {
        reset_red(w.red.p, s);
        count_launch(), corner_kernel<<<grid_for(cells), 256, 0, s>>>(w.pos.p, nx, ny, nz, vol, e1, e2, w.jc.p,
                                                      w.red.p);
        BINDER_CUDA(cudaGetLastError());
        return read_red(w.red.p, s);
    };

    Red r = jac_stats();
    double jmin = unordered(r.mn), jmax = unordered(r.mx);
    res.below_before = (long long)r.below;
    res.above_before = (long long)r.above;
    const int nlev = 4 * (nx - 2) + 2 * (ny - 2) + (nz - 2) + 1;
    const size_t lim_smem = sizeof(int) * (2 * (size_t)nlev + 1);
    BINDER_CUDA(cudaFuncSetAttribute(limiter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)lim_smem));
    int outer = 0;
    while ((jmin < e1 || jmax > e2) && outer < max_outer) {
        w.ensure();
        Red c = corners();
        int inner = 0;
        while ((c.below > 0 || c.above > 0) && inner < max_inner) {
            count_launch(), gradient_kernel<<<grid_for(V), 256, 0, s>>>(w.pos.p, nx, ny, nz, vs[0], vs[1], vs[2],
                                                        w.grad.p);
            reset_red(w.red.p, s);
            count_launch(), flag_cells_kernel<<<grid_for(cells), 256, 0, s>>>(w.jc.p, nx, ny, nz, e1, e2, w.list.p,
                                                              w.red.p);
            count_launch(), limiter_kernel<<<1, 256, lim_smem, s>>>(w.list.p, w.sorted.p, w.jc.p, w.grad.p, nx, ny,
                                                     nz, e1, e2, nlev, w.red.p, w.flags.p);
            BINDER_CUDA(cudaGetLastError());
            count_launch(), sum_kernel<<<grid_for(V), 256, 0, s>>>(w.pos.p, V, 3, w.red.p);
            count_launch(), divergence_kernel<<<grid_for(V), 256, 0, s>>>(w.grad.p, nx, ny, nz, w.div.p);
            BINDER_CUDA(cudaGetLastError());
            Red sr = read_red(w.red.p, s);
            double mean[3];
            for (int n = 0; n < 3; ++n) mean[n] = sr.sum[n] / (nx * ny * nz);

            // u = -(1/V) H (H div / lambda): separable Hartley passes z, y, [x fused], y, z
            AxisArgs<double> a{};
            a.comp_stride = V;
            a.ny = ny;
            a.nz = nz;
            a.cos_x = w.cs[0].p;
            a.cos_y = w.cs[1].p;
            a.cos_z = w.cs[2].p;
            a.in = w.div.p; a.out = w.t1.p; a.M = w.H[2].p; a.n = nz; a.outer = (long)nx * ny; a.s = 1;
            launch_axis_pass(a, kEpiNone, 3, s);
            a.in = w.t1.p; a.out = w.t2.p; a.M = w.H[1].p; a.n = ny; a.outer = nx; a.s = nz;
            launch_axis_pass(a, kEpiNone, 3, s);
            a.in = w.t2.p; a.out = w.t1.p; a.M = w.H[0].p; a.M2 = w.H[0].p; a.n = nx; a.outer = 1;
            a.s = (long)ny * nz;
            launch_axis_pass(a, kEpiPoisson, 3, s);
            a.in = w.t1.p; a.out = w.t2.p; a.M = w.H[1].p; a.M2 = nullptr; a.n = ny; a.outer = nx;
            a.s = nz;
            launch_axis_pass(a, kEpiNone, 3, s);
            // last pass: physical positions u * vs + mean
            a.in = w.t2.p; a.out = w.pos.p; a.M = w.H[2].p; a.n = nz; a.outer = (long)nx * ny; a.s = 1;
            for (int n = 0; n < 3; ++n) {
                a.out_scale[n] = vs[n];
                a.out_offset[n] = mean[n];
            }
            launch_axis_pass(a, kEpiTopoOut, 3, s);
            c = corners();
            inner++;
            res.inner_iterations++;
        }
        r = jac_stats();
        jmin = unordered(r.mn);
        jmax = unordered(r.mx);
        outer++;
    }
    res.outer_iterations = outer;
    r = jac_stats();
    res.below_after = (long long)r.below;
    res.above_after = (long long)r.above;
    BINDER_CUDA(cudaMemcpyAsync(&res.flags, w.flags.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    return res;
}

// BINDER/src/cpu/topology_correction_2D.cpp:17-163: the 3D loop structure with 4 corners per
// cell, 2x2 gradient matrices and a 2D Poisson solve (separable Hartley passes y, [x fused], y)
TopologyResult TopologyWorkspace::run2d(double e1, double e2, int max_outer, int max_inner,
                                        const double vs[3], cudaStream_t s) {
    BINDER_CHECK(vs[0] > 0 && vs[1] > 0, "voxel sizes must be positive");
    Impl &w = *impl_;
    const int nx = w.nx, ny = w.ny;
    const long V = w.V, cells = w.cells;
    const double vol = 1.0 / (vs[0] * vs[1]);
    TopologyResult res{};
    BINDER_CUDA(cudaMemsetAsync(w.flags.p, 0, sizeof(unsigned), s));

    auto jac_stats = [&]() {
        reset_red(w.red.p, s);
        count_launch(), jacobian2d_kernel<<<grid_for(V), 256, 0, s>>>(w.pos.p, 1, V, nx, ny, vol,
                                                                      nullptr, e1, e2, w.red.p);
        BINDER_CUDA(cudaGetLastError());
        return read_red(w.red.p, s);
    };
    auto corners = [&]() {
        reset_red(w.red.p, s);
        count_launch(), corner2d_kernel<<<grid_for(cells), 256, 0, s>>>(w.pos.p, nx, ny, vol, e1,
                                                                        e2, w.jc.p, w.red.p);
        BINDER_CUDA(cudaGetLastError());
        return read_red(w.red.p, s);
    };

    Red r = jac_stats();
    double jmin = unordered(r.mn), jmax = unordered(r.mx);
    res.below_before = (long long)r.below;
    res.above_before = (long long)r.above;
    const int nlev = 2 * (nx - 2) + (ny - 2) + 1;
    const size_t lim_smem =
        ((sizeof(int) * (2 * (size_t)nlev + 1) + 15) & ~(size_t)15) + kStageBytes;
    BINDER_CUDA(cudaFuncSetAttribute(limiter2d_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim_smem));
    int outer = 0;
    while ((jmin < e1 || jmax > e2) && outer < max_outer) {
        w.ensure();
        Red c = corners();
        int inner = 0;
        while ((c.below > 0 || c.above > 0) && inner < max_inner) {
            count_launch(), gradient2d_kernel<<<grid_for(V), 256, 0, s>>>(w.pos.p, nx, ny, vs[0],
                                                                          vs[1], w.grad.p);
            reset_red(w.red.p, s);
            count_launch(), flag_cells2d_kernel<<<grid_for(cells), 256, 0, s>>>(
                                w.jc.p, nx, ny, e1, e2, w.list.p, w.red.p);
            count_launch(), limiter2d_kernel<<<1, kLimiterThreads, lim_smem, s>>>(
                                w.list.p, w.sorted.p, w.jc.p, w.grad.p, nx, ny, e1, e2, nlev,
                                w.red.p, w.flags.p, w.slot.p);
            BINDER_CUDA(cudaGetLastError());
            count_launch(), sum_kernel<<<grid_for(V), 256, 0, s>>>(w.pos.p, V, 2, w.red.p);
            count_launch(), divergence2d_kernel<<<grid_for(V), 256, 0, s>>>(w.grad.p, nx, ny,
                                                                            w.div.p);
            BINDER_CUDA(cudaGetLastError());
            Red sr = read_red(w.red.p, s);
            double mean[2];
            for (int n = 0; n < 2; ++n) mean[n] = sr.sum[n] / (nx * ny);

            // u = -(1/V) H (H div / lambda) on the nx x ny grid (the volume nx x ny x 1, whose
            // unit z axis contributes cos 0 = 1 to lambda = 6 - 2cos_x - 2cos_y - 2cos_z)
            AxisArgs<double> a{};
            a.comp_stride = V;
            a.ny = ny;
            a.nz = 1;
            a.cos_x = w.cs[0].p;
            a.cos_y = w.cs[1].p;
            a.cos_z = w.cs[2].p;
            a.in = w.div.p; a.out = w.t1.p; a.M = w.H[1].p; a.n = ny; a.outer = nx; a.s = 1;
            launch_axis_pass(a, kEpiNone, 2, s);
            // the x passes as two launches (forward with -1/lambda, inverse), each split into row
            // blocks: fused into one, a 2D image's x pass fills only a few CTAs
            a.in = w.t1.p; a.out = w.t2.p; a.M = w.H[0].p; a.n = nx; a.outer = 1; a.s = ny;
            launch_axis_pass(a, kEpiPoissonFwd, 2, s);
            a.in = w.t2.p; a.out = w.t1.p;
            launch_axis_pass(a, kEpiNone, 2, s);
            // last pass: physical positions u * vs + mean
            a.in = w.t1.p; a.out = w.pos.p; a.M = w.H[1].p; a.M2 = nullptr; a.n = ny; a.outer = nx;
            a.s = 1;
            for (int n = 0; n < 2; ++n) {
                a.out_scale[n] = vs[n];
                a.out_offset[n] = mean[n];
            }
            launch_axis_pass(a, kEpiTopoOut, 2, s);
            c = corners();
            inner++;
            res.inner_iterations++;
        }
        r = jac_stats();
        jmin = unordered(r.mn);
        jmax = unordered(r.mx);
        outer++;
    }
    res.outer_iterations = outer;
    r = jac_stats();
    res.below_after = (long long)r.below;
    res.above_after = (long long)r.above;
    BINDER_CUDA(cudaMemcpyAsync(&res.flags, w.flags.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    return res;
}

void TopologyWorkspace::load_float_grid(const float *d_soa, const double vs[3], cudaStream_t s) {
    const Scale sc{{vs[0], vs[1], vs[2]}};
    count_launch(), float_soa_to_physical_kernel<<<grid_for(impl_->V), 256, 0, s>>>(
                        d_soa, impl_->V, impl_->N, sc, impl_->pos.p);
    BINDER_CUDA(cudaGetLastError());
}

void TopologyWorkspace::store_float_grid(float *d_soa, const double vs[3], cudaStream_t s) {
    const Scale sc{{vs[0], vs[1], vs[2]}};
    count_launch(), physical_to_float_soa_kernel<<<grid_for(impl_->V), 256, 0, s>>>(
                        impl_->pos.p, impl_->V, impl_->N, sc, d_soa);
    BINDER_CUDA(cudaGetLastError());
}

TopologyResult topology_correct_3d(double *host, double e1, double e2, int max_outer,
                                   int max_inner, const double vs[3], int nx, int ny, int nz,
                                   cudaStream_t s) {
    BINDER_CHECK(vs[0] > 0 && vs[1] > 0 && vs[2] > 0, "voxel sizes must be positive");
    BINDER_CHECK(nz >= 2, "a 3D field needs nz >= 2 (use the 2D entry point for images)");
    return topology_correct(host, e1, e2, max_outer, max_inner, vs, nx, ny, nz, s);
}

TopologyResult topology_correct_2d(double *host, double e1, double e2, int max_outer,
                                   int max_inner, const double vs[2], int nx, int ny,
                                   cudaStream_t s) {
    BINDER_CHECK(vs[0] > 0 && vs[1] > 0, "voxel sizes must be positive");
    const double vs3[3] = {vs[0], vs[1], 1.0};
    return topology_correct(host, e1, e2, max_outer, max_inner, vs3, nx, ny, 1, s);
}

// host AoS field (grid units) -> device SoA physical -> correction -> back, in place
TopologyResult topology_correct(double *host, double e1, double e2, int max_outer, int max_inner,
                                const double vs[3], int nx, int ny, int nz, cudaStream_t s) {
    TopologyWorkspace ws(nx, ny, nz, s);
    const long V = (long)nx * ny * nz;
    const int N = nz == 1 ? 2 : 3;
    const Scale sc{{vs[0], vs[1], vs[2]}};
    DBuf<double> aos(V * N, s);
    BINDER_CUDA(cudaMemcpyAsync(aos.p, host, sizeof(double) * V * N, cudaMemcpyHostToDevice, s));
    count_launch(), aos_to_soa_kernel<<<grid_for(V), 256, 0, s>>>(aos.p, V, N, sc, ws.positions());
    BINDER_CUDA(cudaGetLastError());
    TopologyResult res = ws.run(e1, e2, max_outer, max_inner, vs, s);
    count_launch(), soa_to_aos_kernel<<<grid_for(V), 256, 0, s>>>(ws.positions(), V, N, sc, aos.p);
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaMemcpyAsync(host, aos.p, sizeof(double) * V * N, cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    return res;
}

}  // namespace binder
