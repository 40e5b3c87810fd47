// The DCT-prior M-step of a small 2D image (nx, ny <= 128) in one launch, for the images where
// the separate passes are each a couple of CTAs' latency.  One thread-block cluster of kG CTAs
// per component:
//   1. CTA q owns the rows [q R, (q + 1) R) (R = ceil(nx / kG)): forward DCT along y;
//   2. cluster barrier; CTA q gathers the columns [q W, (q + 1) W) (W = ceil(ny / kG)) of every
//      row from the other CTAs' shared memory (distributed shared memory), forward DCT along x,
//      prior scaling 1 / (1 + gamma sigma^2 D) [+ noise] with the costs, inverse DCT along x;
//   3. cluster barrier; CTA q gathers its rows back, inverse DCT along y, adds the pixel
//      positions and stores.
// Each product is out[k] = sum_j MT[j][k] in[j] with the pass matrix staged transposed in
// shared memory (lanes take consecutive k: conflict-free rows), FP32 FMA; the epilogue is that
// of the CUDA-core passes (transform.cu): the same scaling, noise stream and FP64 costs.
#include <cooperative_groups.h>

#include "mstep2d.cuh"

namespace cg = cooperative_groups;

namespace binder {

namespace {

constexpr int kG = 8;          // CTAs per component (cluster size)
constexpr int kM2dThreads = 256;
constexpr int kSlab = (kM2dMaxN + kG - 1) / kG;  // rows / columns per CTA

struct M2dArgs {
    AxisArgs<float> a;
    const float *r;
    float *d;
    int nx, ny;
    const float *Fx, *Ix, *Fy, *Iy;
};

constexpr int kBatch = 8;  // independent loads in flight per thread in the copy loops

// dst[f] = src(f) for f < count, kBatch loads issued before their stores
template <typename F>
__device__ __forceinline__ void batched_copy(float *dst, int count, F &&src) {
    for (int f0 = threadIdx.x; f0 < count; f0 += blockDim.x * kBatch) {
        float v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int f = f0 + u * (int)blockDim.x;
            v[u] = f < count ? src(f) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int f = f0 + u * (int)blockDim.x;
            if (f < count) dst[f] = v[u];
        }
    }
}

// start copying the n x n matrix M into shared memory (cp.async: 16-byte pieces, 4-byte ones for
// a tail of n^2 % 4 floats; M and ms are 16-byte aligned); stage_wait() completes it
__device__ __forceinline__ void stage_async(float *ms, const float *M, int n) {
    const int nn = n * n, n4 = nn >> 2;
    for (int f = threadIdx.x; f < n4; f += blockDim.x)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(ms + 4 * f)),
                     "l"(M + 4 * f)
                     : "memory");
    for (int f = 4 * n4 + threadIdx.x; f < nn; f += blockDim.x)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(ms + f)),
                     "l"(M + f)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void stage_wait() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
}

// out(p, q) = sum_{j < len} X[j xs + p] Y[j ys + q yq] for p < P (<= 128) and q < Q (<= 16),
// register-tiled: lane l takes p = 4 l .. 4 l + 3, warp w takes q = 2 w, 2 w + 1, so every step
// is one (vector) load of X along p and two warp-uniform loads of Y for 8 FMAs
template <typename ST>
__device__ __forceinline__ void product(int P, int Q, int len, const float *X, int xs,
                                        const float *Y, int ys, int yq, ST &&store) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p0 = 4 * lane, q0 = 2 * warp;
    if (p0 >= P || q0 >= Q) return;  // no output here (no barrier follows inside)
    const bool vec = (xs & 3) == 0 && p0 + 3 < P;
    const bool q1 = q0 + 1 < Q;
    float acc[4][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
    for (int j = 0; j < len; ++j) {
        float xv[4];
        if (vec) {
            const float4 v = *reinterpret_cast<const float4 *>(X + j * xs + p0);
            xv[0] = v.x; xv[1] = v.y; xv[2] = v.z; xv[3] = v.w;
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) xv[e] = p0 + e < P ? X[j * xs + p0 + e] : 0.0f;
        }
        const float y0 = Y[j * ys + q0 * yq];
        const float y1 = q1 ? Y[j * ys + (q0 + 1) * yq] : 0.0f;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            acc[e][0] = fmaf(xv[e], y0, acc[e][0]);
            acc[e][1] = fmaf(xv[e], y1, acc[e][1]);
        }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (p0 + e >= P) break;
        store(p0 + e, q0, acc[e][0]);
        if (q1) store(p0 + e, q0 + 1, acc[e][1]);
    }
}

__global__ void __cluster_dims__(kG, 1, 1) __launch_bounds__(kM2dThreads)
    mstep2d_kernel(const M2dArgs p) {
    const AxisArgs<float> &a = p.a;
    if (a.skip && *a.skip) return;  // the same decision in every CTA of the cluster
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) float sm[];
    const int nx = p.nx, ny = p.ny;
    const int R = (nx + kG - 1) / kG, W = (ny + kG - 1) / kG;
    float *ms0 = sm;                         // [n][n] pass matrices (transposed: [j][k]),
    float *ms1 = ms0 + kM2dMaxN * kM2dMaxN;  // double-buffered
    float *rowA = ms1 + kM2dMaxN * kM2dMaxN; // [R][ny] this CTA's rows
    float *rowB = rowA + kSlab * kM2dMaxN;   // [R][ny]
    float *colA = rowB + kSlab * kM2dMaxN;   // [nx][nw] this CTA's columns (packed)
    float *colB = colA + kM2dMaxN * kSlab;   // [nx][nw]
    __shared__ double red[32];
    const int q = (int)cluster.block_rank();
    const int comp = (int)blockIdx.y;
    const long V = a.comp_stride;
    const int x0 = q * R, nr = max(0, min(R, nx - x0));  // my rows
    const int y0 = q * W, nw = max(0, min(W, ny - y0));  // my columns
    const int tid = threadIdx.x;

    // ---- 1. forward DCT along y of my rows: rowB[x][ky] = sum_y Fy[ky][y] rowA[x][y] ----------
    stage_async(ms0, p.Iy, ny);  // Iy[y][ky] = Fy[ky][y]
    {
        const float *src = p.r + comp * V + (long)x0 * ny;
        batched_copy(rowA, nr * ny, [&](int f) { return __ldg(src + f); });
    }
    stage_wait();
    stage_async(ms1, p.Ix, nx);  // Ix[x][kx] = Fx[kx][x], in flight during the y pass
    // p = ky (X = Iy rows y), q = xl (Y = rowA[xl][y])
    product(ny, nr, ny, ms0, ny, rowA, 1, ny,
            [&](int ky, int xl, float v) { rowB[xl * ny + ky] = v; });
    cluster.sync();  // every CTA's rowB is complete

    // ---- 2. my columns of every row, forward x, scaling, inverse x --------------------------
    if (nw > 0)
        batched_copy(colA, nx * nw, [&](int f) {
            const int x = f / nw, yl = f - x * nw;
            const int owner = x / R;
            const float *src = cluster.map_shared_rank(rowB, owner);
            return src[(x - owner * R) * ny + (y0 + yl)];
        });
    stage_wait();                // Ix; every thread is done with ms0 (the cluster barrier)
    stage_async(ms0, p.Fx, nx);  // inverse: x = sum_kx Fx[kx][x] c[kx]
    double part_cost = 0.0, part_raw = 0.0;
    {
        const double g = a.st->gamma[comp];
        const float gs2 = (float)(g * a.sigma2);
        const uint32_t sweep = (uint32_t)a.st->sweep;
        const bool want_raw = a.want_raw && (a.st->sweep % a.every == 0);
        if (nw > 0)
            // p = kx (X = Ix rows x), q = yl (Y = colA[x][yl])
            product(nx, nw, nx, ms1, nx, colA, nw, 1,
                [&](int kx, int yl, float acc) {
                    // coefficient (kx, ky) has flat index kx ny + ky (the x pass of transform.cu)
                    const long i = (long)kx * ny + (y0 + yl);
                    const float Dv = a.D[i];
                    const float f = 1.0f / (1.0f + gs2 * Dv);
                    float v = acc * f;
                    if (a.sample)
                        v += sqrtf((float)a.sigma2 * f) *
                             dct_prior_normal(a.seed, (uint32_t)i, sweep, a.chain, comp);
                    const double v2 = (double)v * (double)v;
                    part_cost += 0.5 * g * (double)Dv * v2;
                    if (want_raw) part_raw += a.eta2[comp] * a.rho_p * (double)Dv * v2;
                    colB[kx * nw + yl] = v;
                });
    }
    stage_wait();                // Fx, and colB complete
    stage_async(ms1, p.Fy, ny);  // inverse: y = sum_ky Fy[ky][y] c[ky]
    if (nw > 0)
        // p = x (X = Fx rows kx), q = yl (Y = colB[kx][yl])
        product(nx, nw, nx, ms0, nx, colB, nw, 1,
                [&](int x, int yl, float v) { colA[x * nw + yl] = v; });
    cluster.sync();  // every CTA's colA is complete (and nobody reads rowB any more)

    // ---- 3. my rows back, inverse y, positions -----------------------------------------------
    batched_copy(rowA, nr * ny, [&](int f) {
        const int xl = f / ny, y = f - xl * ny;
        const int owner = y / W;
        const int onw = min(W, ny - owner * W);  // the owner's packed column count
        const float *src = cluster.map_shared_rank(colA, owner);
        return src[(x0 + xl) * onw + (y - owner * W)];
    });
    stage_wait();  // Fy
    // p = y (X = Fy rows ky), q = xl (Y = rowA[xl][ky])
    product(ny, nr, ny, ms1, ny, rowA, 1, ny,
        [&](int y, int xl, float acc) {
            const long i = (long)(x0 + xl) * ny + y;
            const float xv =
                a.xpos ? a.xpos[comp * V + i] : (comp == 0 ? (float)(x0 + xl) : (float)y);
            p.d[comp * V + i] = acc + xv;
        });
    const double sc = block_sum(part_cost, red);
    if (tid == 0) atomicAdd(&a.st->lp_tr, sc);
    if (a.want_raw) {
        const double sr = block_sum(part_raw, red);
        if (tid == 0) atomicAdd(&a.st->raw_reg, sr);
    }
    cluster.sync();  // no CTA leaves while another may still read its shared memory
}

}  // namespace

void launch_mstep2d(const AxisArgs<float> &a, const float *r, float *d, int nx, int ny,
                    const float *Fx, const float *Ix, const float *Fy, const float *Iy,
                    cudaStream_t s) {
    BINDER_CHECK(nx >= 1 && ny >= 1 && nx <= kM2dMaxN && ny <= kM2dMaxN,
                 "the fused 2D M-step needs nx, ny <= 128");
    const size_t smem = (size_t)(2 * kM2dMaxN * kM2dMaxN + 4 * kSlab * kM2dMaxN) * sizeof(float);
    static bool configured = false;
    if (!configured) {
        BINDER_CUDA(cudaFuncSetAttribute(mstep2d_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = true;
    }
    M2dArgs p{a, r, d, nx, ny, Fx, Ix, Fy, Iy};
    count_launch(), mstep2d_kernel<<<dim3(kG, 2, 1), kM2dThreads, smem, s>>>(p);
    BINDER_CUDA(cudaGetLastError());
}

}  // namespace binder
