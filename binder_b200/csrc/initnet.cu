// Learned initialiser: hand-written BF16 tensor-core GEMM (tcgen05, FP32 accumulation in TMEM),
// implicit-GEMM 3D convolutions built on it (im2col gathers into BF16 operand matrices), the
// element-wise layers, the loss and Adam.  See initnet.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "initnet.cuh"
#include "layout.cuh"
#include "umma.cuh"

namespace binder {

namespace {

constexpr uint64_t kGemmWaitNs = 2000000000ull;  // bounded mbarrier waits (2 s)
constexpr int kGemmBM = 128;                     // UMMA M: one TMEM lane per output row
constexpr int kGemmBK = 64;                      // K elements per pipeline stage (4 MMAs of 16)
constexpr int kGemmStages = 3;

// ---- GEMM: C[M][N] (+)= A[M][K] . B[N][K]^T ----------------------------------------------------
// One CTA of 128 threads per 128 x BN output tile and K split.  Every thread copies its share of
// each K stage into shared memory with cp.async (rows past M / N zero-filled), in the canonical
// no-swizzle K-major layout: 16-byte K columns of 8 elements, 8-row groups 128 bytes apart.
// Thread 0 issues the stage's four kind::f16 MMAs (K = 16 each) and commits them to the stage's
// mbarrier; a stage is refilled only after that mbarrier has completed.  The accumulator lives
// in TMEM (lane = tile row, column = tile column) and is read back with tcgen05.ld.
template <int BN>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr uint32_t kAStage = kGemmBM * kGemmBK * 2;  // bytes
    constexpr uint32_t kBStage = BN * kGemmBK * 2;
    unsigned char *As = smem;
    unsigned char *Bs = smem + kGemmStages * kAStage;
    uint64_t *bar = reinterpret_cast<uint64_t *>(Bs + kGemmStages * kBStage);
    uint64_t *drain = bar + kGemmStages;  // used once, on the error path
    uint32_t *holder = reinterpret_cast<uint32_t *>(drain + 1);
    int *s_err = reinterpret_cast<int *>(holder + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr uint32_t ncols = BN < 32 ? 32u : (uint32_t)BN;

    if (warp == 0) umma::tmem_alloc(holder, ncols);
    if (tid == 32) {
        for (int s = 0; s < kGemmStages; ++s) umma::mbar_init(&bar[s], 1);
        umma::mbar_init(drain, 1);
        *s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *holder;

    const long m0 = (long)blockIdx.x * kGemmBM, n0 = (long)blockIdx.y * BN;
    const long k_begin = (long)blockIdx.z * g.k_split;
    long k_end = k_begin + g.k_split;
    if (k_end > g.K) k_end = g.K;
    const int nk = k_end > k_begin ? (int)((k_end - k_begin) / kGemmBK) : 0;

    auto load_stage = [&](int kc, int stage) {
        const long k0 = k_begin + (long)kc * kGemmBK;
        unsigned char *as = As + stage * kAStage;
        unsigned char *bs = Bs + stage * kBStage;
        // A: 128 rows x 8 K columns of 16 bytes
        for (int q = tid; q < kGemmBM * 8; q += 128) {
            const int row = q >> 3, kc8 = q & 7;
            const long m = m0 + row;
            const bool ok = m < g.M;
            const uint16_t *src = g.A + (ok ? m : 0) * g.lda + k0 + kc8 * 8;
            umma::cp_async16_zfill(as + kc8 * (kGemmBM * 16) + (row >> 3) * 128 + (row & 7) * 16,
                                   src, ok ? 16u : 0u);
        }
        // B: BN rows x 8 K columns
        for (int q = tid; q < BN * 8; q += 128) {
            const int row = q >> 3, kc8 = q & 7;
            const long n = n0 + row;
            const bool ok = n < g.N;
            const uint16_t *src = g.B + (ok ? n : 0) * g.ldb + k0 + kc8 * 8;
            umma::cp_async16_zfill(bs + kc8 * (BN * 16) + (row >> 3) * 128 + (row & 7) * 16, src,
                                   ok ? 16u : 0u);
        }
    };

    constexpr uint32_t idesc = umma::instr_desc(kGemmBM, BN, umma::kFmtBF16);
    for (int s = 0; s < kGemmStages - 1; ++s) {
        if (s < nk) load_stage(s, s);
        umma::cp_async_commit();
    }
    for (int kc = 0; kc < nk; ++kc) {
        const int stage = kc % kGemmStages;
        asm volatile("cp.async.wait_group %0;" ::"n"(kGemmStages - 2) : "memory");
        umma::fence_proxy_async_smem();
        __syncthreads();
        if (*(volatile int *)s_err) break;
        if (tid == 0) {
            umma::fence_after_sync();
            const uint32_t abase = umma::smem_u32(As + stage * kAStage);
            const uint32_t bbase = umma::smem_u32(Bs + stage * kBStage);
#pragma unroll
            for (int ks = 0; ks < kGemmBK / 16; ++ks) {
                const uint64_t ad = umma::smem_desc(abase + ks * 2 * (kGemmBM * 16), kGemmBM * 16, 128);
                const uint64_t bd = umma::smem_desc(bbase + ks * 2 * (BN * 16), BN * 16, 128);
                umma::mma_bf16(tmem, ad, bd, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
            }
            umma::commit(&bar[stage]);
        }
        // refill the stage chunk kc - 1 used, once its MMAs have completed
        const int next = kc + kGemmStages - 1;
        if (next < nk) {
            if (kc >= 1) {
                const int prev = kc - 1;
                if (!umma::mbar_wait(&bar[prev % kGemmStages], (uint32_t)(prev / kGemmStages) & 1u,
                                     kGemmWaitNs))
                    *(volatile int *)s_err = 1;
            }
            load_stage(next, next % kGemmStages);
        }
        umma::cp_async_commit();
    }
    umma::cp_async_wait_all();
    if (nk > 0 && !*(volatile int *)s_err) {
        const int last = nk - 1;
        if (!umma::mbar_wait(&bar[last % kGemmStages], (uint32_t)(last / kGemmStages) & 1u,
                             kGemmWaitNs))
            *(volatile int *)s_err = 1;
    }
    __syncthreads();
    umma::fence_after_sync();
    if (!*(volatile int *)s_err && nk > 0) {
        const long m = m0 + warp * 32 + lane;
        const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int cc = 0; cc < BN / 32 + (BN % 32 ? 1 : 0); ++cc) {
            float v[32];
            if (BN % 32 == 0 || cc * 32 + 32 <= BN) {
                umma::tmem_ld32(tl + (uint32_t)(cc * 32), v);
            } else {
                float h[16];
                umma::tmem_ld16(tl + (uint32_t)(cc * 32), h);
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = h[j], v[16 + j] = 0.0f;
            }
            if (m < g.M) {
                float *crow = g.C + m * g.ldc;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const long n = n0 + cc * 32 + j;
                    if (cc * 32 + j < BN && n < g.N) {
                        if (g.accumulate) atomicAdd(crow + n, v[j]);
                        else crow[n] = v[j];
                    }
                }
            }
        }
    }
    if (*(volatile int *)s_err) {
        // let every MMA this CTA issued complete before its TMEM goes back (bounded)
        if (tid == 0) {
            umma::commit(drain);  // arrives once every MMA thread 0 issued has completed
            umma::mbar_wait(drain, 0, kGemmWaitNs);
            atomicExch(g.err, 1);
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, ncols);
}

template <int BN>
void launch_gemm_bn(const GemmArgs &g, cudaStream_t s) {
    const size_t smem = (size_t)kGemmStages * (kGemmBM + BN) * kGemmBK * 2 + 128;
    BINDER_CUDA(cudaFuncSetAttribute(gemm_bf16_kernel<BN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long splits = (g.K + g.k_split - 1) / g.k_split;
    const dim3 grid((unsigned)((g.M + kGemmBM - 1) / kGemmBM), (unsigned)((g.N + BN - 1) / BN),
                    (unsigned)splits);
    count_launch(), gemm_bf16_kernel<BN><<<grid, 128, smem, s>>>(g);
    BINDER_CUDA(cudaGetLastError());
}

// ---- element-wise and gather kernels ------------------------------------------------------------
// Activations are channels-last [B][S][S][S][C]; voxel index v = ((b * S + x) * S + y) * S + z.

__device__ __forceinline__ uint16_t bf16_bits(float f) {
    const __nv_bfloat16 h = __float2bfloat16_rn(f);
    return *reinterpret_cast<const uint16_t *>(&h);
}
__device__ __forceinline__ float bf16_value(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// im2col of a 3 x 3 x 3 stride-1 convolution with zero padding: row v of `out` holds, at
// k = tap * C + c (tap = (dx * 3 + dy) * 3 + dz, offsets -1 .. 1), the input at v + offset, and
// zeros for k >= 27 C up to the padded row length Kp.  One thread per 8-element output chunk.
__global__ void im2col_kernel(const uint16_t *in, int B, int S, int C, int Kp, uint16_t *out) {
    const long V = (long)S * S * S;
    const long chunks = (long)B * V * (Kp / 8);
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < chunks;
         q += (long)gridDim.x * blockDim.x) {
        const long v = q / (Kp / 8);
        const int k0 = (int)(q - v * (Kp / 8)) * 8;
        const long b = v / V;
        const long r = v - b * V;
        const int x = (int)(r / ((long)S * S)), y = (int)((r / S) % S), z = (int)(r % S);
        uint16_t vals[8];
        if (C % 8 == 0 && k0 < 27 * C) {
            const int tap = k0 / C, c0 = k0 - tap * C;
            const int X = x + tap / 9 - 1, Y = y + (tap / 3) % 3 - 1, Z = z + tap % 3 - 1;
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (X >= 0 && X < S && Y >= 0 && Y < S && Z >= 0 && Z < S)
                w = *reinterpret_cast<const uint4 *>(
                    in + ((((b * S + X) * S + Y) * S + Z) * C + c0));
            *reinterpret_cast<uint4 *>(out + v * Kp + k0) = w;
            continue;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = k0 + j;
            uint16_t val = 0;
            if (k < 27 * C) {
                const int tap = k / C, c = k - tap * C;
                const int X = x + tap / 9 - 1, Y = y + (tap / 3) % 3 - 1, Z = z + tap % 3 - 1;
                if (X >= 0 && X < S && Y >= 0 && Y < S && Z >= 0 && Z < S)
                    val = in[(((b * S + X) * S + Y) * S + Z) * C + c];
            }
            vals[j] = val;
        }
        uint4 w;
        w.x = vals[0] | ((uint32_t)vals[1] << 16);
        w.y = vals[2] | ((uint32_t)vals[3] << 16);
        w.z = vals[4] | ((uint32_t)vals[5] << 16);
        w.w = vals[6] | ((uint32_t)vals[7] << 16);
        *reinterpret_cast<uint4 *>(out + v * Kp + k0) = w;
    }
}

// out[c][r] = in[r][c] for an R x Cc BF16 matrix (leading dimensions ldi, ldo), 32 x 32 tiles
// through shared memory; columns past Cc of `out`'s rows are not written
__global__ void transpose_bf16_kernel(const uint16_t *in, long R, long Cc, long ldi, uint16_t *out,
                                      long ldo) {
    __shared__ uint16_t t[32][33];
    const long r0 = (long)blockIdx.x * 32, c0 = (long)blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long r = r0 + j, c = c0 + threadIdx.x;
        t[j][threadIdx.x] = (r < R && c < Cc) ? in[r * ldi + c] : (uint16_t)0;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const long c = c0 + j, r = r0 + threadIdx.x;
        if (c < Cc && r < R) out[c * ldo + r] = t[threadIdx.x][j];
    }
}

// pre-activation z = gemm + bias (kept, FP32 [M][C]) and the layer output: leaky ReLU in BF16
// ([M][C]), or, for the linear head, z itself in FP32
__global__ void bias_act_kernel(float *z, long M, int C, long ldz, const float *bias, float slope,
                                int act, uint16_t *ybf, float *yf) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < M * C;
         q += (long)gridDim.x * blockDim.x) {
        const long m = q / C;
        const int c = (int)(q - m * C);
        const float v = z[m * ldz + c] + bias[c];
        z[m * ldz + c] = v;
        if (act) ybf[q] = bf16_bits(v > 0.0f ? v : slope * v);
        else yf[q] = v;
    }
}

// gradient through the leaky ReLU: dz = dy * (z > 0 ? 1 : slope), as FP32 and as the BF16 GEMM
// operand
__global__ void act_backward_kernel(const float *dy, const float *z, long M, int C, long ldz,
                                    float slope, int act, float *dz, uint16_t *dzb) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < M * C;
         q += (long)gridDim.x * blockDim.x) {
        const long m = q / C;
        const int c = (int)(q - m * C);
        const float g = act ? (z[m * ldz + c] > 0.0f ? dy[q] : slope * dy[q]) : dy[q];
        dz[q] = g;
        dzb[q] = bf16_bits(g);
    }
}

// db[c] += sum over rows of dz[m][c]: one CTA per column block, FP32 block reductions
__global__ void column_sum_kernel(const float *dz, long M, int C, float *db) {
    __shared__ float red[32];
    const int c = blockIdx.y;
    float s = 0.0f;
    for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < M;
         m += (long)gridDim.x * blockDim.x)
        s += dz[m * C + c];
    s = block_sum(s, red);
    if (threadIdx.x == 0) atomicAdd(&db[c], s);
}

// 2 x 2 x 2 average pooling of a BF16 activation [B][S^3][C] into [B][(S/2)^3][C]
__global__ void avgpool2_kernel(const uint16_t *in, int B, int S, int C, uint16_t *out) {
    const int H = S / 2;
    const long n = (long)B * H * H * H * C;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q % C);
        long v = q / C;
        const int z = (int)(v % H), y = (int)((v / H) % H), x = (int)((v / ((long)H * H)) % H);
        const long b = v / ((long)H * H * H);
        float s = 0.0f;
        for (int d = 0; d < 8; ++d) {
            const int X = 2 * x + (d >> 2), Y = 2 * y + ((d >> 1) & 1), Z = 2 * z + (d & 1);
            s += bf16_value(in[(((b * S + X) * S + Y) * S + Z) * C + c]);
        }
        out[q] = bf16_bits(0.125f * s);
    }
}

// its gradient: every fine voxel receives 1/8 of its coarse voxel's gradient (added to dx)
__global__ void avgpool2_backward_kernel(const float *dy, int B, int S, int C, float *dx) {
    const long n = (long)B * S * S * S * C;
    const int H = S / 2;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q % C);
        long v = q / C;
        const int z = (int)(v % S), y = (int)((v / S) % S), x = (int)((v / ((long)S * S)) % S);
        const long b = v / ((long)S * S * S);
        dx[q] += 0.125f * dy[(((b * H + x / 2) * H + y / 2) * H + z / 2) * C + c];
    }
}

// nearest-neighbour 2x up-sampling of a BF16 activation [B][S^3][C] into [B][(2S)^3][C]
__global__ void upsample2_kernel(const uint16_t *in, int B, int S, int C, uint16_t *out) {
    const int T = 2 * S;
    const long n = (long)B * T * T * T * C;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q % C);
        long v = q / C;
        const int z = (int)(v % T), y = (int)((v / T) % T), x = (int)((v / ((long)T * T)) % T);
        const long b = v / ((long)T * T * T);
        out[q] = in[(((b * S + x / 2) * S + y / 2) * S + z / 2) * C + c];
    }
}

// its gradient: the sum of the 8 fine gradients (added to dx)
__global__ void upsample2_backward_kernel(const float *dy, int B, int S, int C, float *dx) {
    const int T = 2 * S;
    const long n = (long)B * S * S * S * C;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q % C);
        long v = q / C;
        const int z = (int)(v % S), y = (int)((v / S) % S), x = (int)((v / ((long)S * S)) % S);
        const long b = v / ((long)S * S * S);
        float s = 0.0f;
        for (int d = 0; d < 8; ++d) {
            const int X = 2 * x + (d >> 2), Y = 2 * y + ((d >> 1) & 1), Z = 2 * z + (d & 1);
            s += dy[(((b * T + X) * T + Y) * T + Z) * C + c];
        }
        dx[q] += s;
    }
}

// out = a + b (BF16 activations, FP32 sum rounded once)
__global__ void add_bf16_kernel(const uint16_t *a, const uint16_t *b, long n, uint16_t *out) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x)
        out[q] = bf16_bits(bf16_value(a[q]) + bf16_value(b[q]));
}

// FP32 input [B][V][Cin] (moving, fixed) to the BF16 network input
__global__ void to_bf16_kernel(const float *in, long n, uint16_t *out) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x)
        out[q] = bf16_bits(in[q]);
}

// mean squared error: partial sums of (y - t)^2 into *loss (FP64) and dy = 2 (y - t) / n
__global__ void mse_kernel(const float *y, const float *t, long n, double *loss, float *dy) {
    __shared__ double red[32];
    double s = 0.0;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x) {
        const float d = y[q] - t[q];
        s += (double)d * d;
        dy[q] = 2.0f * d / (float)n;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) atomicAdd(loss, s / (double)n);
}

// Adam (Kingma & Ba 2015) on FP32 master parameters with bias-corrected moments
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, long n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.0f - b1) * gq;
        const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    }
}

// BF16 operand copies of a layer's FP32 weights W [Cout][27 Cin]: the forward operand
// wf [Cout][Kp] (zero-padded columns) and the flipped, transposed operand of the data gradient
// wb [Cin][Kq] with wb[ci][t' Cout + co] = W[co][(26 - t') Cin + ci]
__global__ void weight_formats_kernel(const float *W, int Cin, int Cout, int Kp, int Kq,
                                      uint16_t *wf, uint16_t *wb) {
    const long n1 = (long)Cout * Kp, n2 = (long)Cin * Kq;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n1 + n2;
         q += (long)gridDim.x * blockDim.x) {
        if (q < n1) {
            const int co = (int)(q / Kp), k = (int)(q - (long)co * Kp);
            wf[q] = k < 27 * Cin ? bf16_bits(W[(long)co * 27 * Cin + k]) : (uint16_t)0;
        } else {
            const long r = q - n1;
            const int ci = (int)(r / Kq), k = (int)(r - (long)ci * Kq);
            uint16_t val = 0;
            if (k < 27 * Cout) {
                const int tp = k / Cout, co = k - tp * Cout;
                val = bf16_bits(W[(long)co * 27 * Cin + (26 - tp) * Cin + ci]);
            }
            wb[r] = val;
        }
    }
}

}  // namespace

void launch_gemm_bf16(const GemmArgs &g, cudaStream_t s) {
    BINDER_CHECK(g.M > 0 && g.N > 0 && g.K > 0, "GEMM sizes must be positive");
    BINDER_CHECK(g.K % kGemmBK == 0 && g.k_split % kGemmBK == 0 && g.k_split > 0,
                 "GEMM K and its split must be multiples of 64");
    BINDER_CHECK(g.lda % 8 == 0 && g.ldb % 8 == 0 && g.lda >= g.K && g.ldb >= g.K,
                 "GEMM leading dimensions must be multiples of 8 and at least K");
    BINDER_CHECK((reinterpret_cast<uintptr_t>(g.A) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(g.B) & 15) == 0,
                 "GEMM operands must be 16-byte aligned");
    BINDER_CHECK(g.accumulate || g.k_split >= g.K, "a split K must accumulate");
    BINDER_CHECK(g.err != nullptr, "GEMM needs an error word");
    if (g.N <= 32) launch_gemm_bn<32>(g, s);
    else if (g.N <= 64) launch_gemm_bn<64>(g, s);
    else launch_gemm_bn<128>(g, s);
}


// ---- the network ------------------------------------------------------------------------------
namespace {

int grid_for_n(long n) {
    long b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148L * 16 ? 148L * 16 : b));
}
int round64(int k) { return (k + 63) / 64 * 64; }
constexpr float kSlope = 0.1f;  // leaky ReLU

// deterministic host normals for the weight initialisation (splitmix64 + Box-Muller)
struct HostRng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

}  // namespace

// one 3 x 3 x 3 convolution + bias (+ leaky ReLU) at spatial size S
struct InitNet::Layer {
    int cin, cout, S;
    bool act;
    int Kp, Kq;       // padded im2col row lengths of the input and of the output gradient
    long woff, boff;  // offsets of W [cout][27 cin] and b [cout] in the flat parameters
    uint16_t *wf = nullptr, *wb = nullptr;  // BF16 operands (forward, data gradient)
    float *z = nullptr;                     // pre-activation [M][cout]
    uint16_t *y = nullptr;                  // BF16 output [M][cout] (hidden layers)
    float *yf = nullptr;                    // FP32 output [M][cout] (the head)
    float *dy = nullptr;                    // gradient of the loss w.r.t. the output
};

struct InitNet::Impl {
    cudaStream_t s = nullptr;
    int *err = nullptr;
    std::vector<Layer> L;
    float *P = nullptr, *G = nullptr, *Am = nullptr, *Av = nullptr;
    double *loss = nullptr;
    uint16_t *x0 = nullptr;                     // BF16 input [B][S^3][2]
    uint16_t *p0 = nullptr, *p1 = nullptr, *p2 = nullptr, *u3 = nullptr, *s2 = nullptr;
    float *dp0 = nullptr, *dp1 = nullptr, *dp2 = nullptr, *du3 = nullptr, *ds2 = nullptr;
    float *in_f = nullptr, *tgt = nullptr;      // staging of the caller's FP32 input / target
    uint16_t *col = nullptr, *colT = nullptr, *dzT = nullptr, *dzb = nullptr;
    float *dz = nullptr;
    long adam_t = 0;
    std::vector<void *> owned;
    template <typename T>
    T *alloc(size_t n) {
        T *p = dev_alloc_n<T>(n < 1 ? 1 : n, s);
        owned.push_back(p);
        return p;
    }
};

namespace {
__global__ void add_f32_kernel(float *dst, const float *src, long n) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long)gridDim.x * blockDim.x)
        dst[q] += src[q];
}
}  // namespace

InitNet::InitNet(int batch, int size, uint64_t seed, int in_channels)
    : impl_(new Impl()), B_(batch), S_(size), Cin_(in_channels) {
    BINDER_CHECK(batch >= 1 && batch <= 64, "batch must be in [1, 64]");
    BINDER_CHECK(size >= 8 && size % 8 == 0 && size <= 256,
                 "the input size must be a multiple of 8 in [8, 256]");
    Impl &m = *impl_;
    BINDER_CUDA(cudaStreamCreate(&m.s));
    m.err = m.alloc<int>(1);
    BINDER_CUDA(cudaMemsetAsync(m.err, 0, sizeof(int), m.s));
    const int S0 = size, S1 = size / 2, S2 = size / 4, S3 = size / 8;
    // encoder (channels 16-32-64-128, two convolutions per level), decoder to the 4-voxel grid
    BINDER_CHECK(in_channels >= 1 && in_channels <= 16, "input channels must be in [1, 16]");
    const int spec[11][4] = {{in_channels, 16, S0, 1},   {16, 16, S0, 1},   {16, 32, S1, 1},
                             {32, 32, S1, 1},  {32, 64, S2, 1},   {64, 64, S2, 1},
                             {64, 128, S3, 1}, {128, 128, S3, 1}, {128, 64, S2, 1},
                             {64, 64, S2, 1},  {64, 3, S2, 0}};
    long off = 0;
    size_t col_max = 0, dzt_max = 0;
    for (const auto &q : spec) {
        Layer l;
        l.cin = q[0]; l.cout = q[1]; l.S = q[2]; l.act = q[3] != 0;
        l.Kp = round64(27 * l.cin);
        l.Kq = round64(27 * l.cout);
        l.woff = off;
        off += 27L * l.cin * l.cout;
        l.boff = off;
        off += l.cout;
        const long M = (long)batch * l.S * l.S * l.S;
        const long Mp = round64((int)M);  // the weight-gradient GEMM's K, padded with zeros
        col_max = std::max(col_max, (size_t)Mp * std::max(l.Kp, l.Kq));
        dzt_max = std::max(dzt_max, (size_t)Mp * l.cout);
        m.L.push_back(l);
    }
    nparam_ = off;
    m.P = m.alloc<float>(nparam_);
    m.G = m.alloc<float>(nparam_);
    m.Am = m.alloc<float>(nparam_);
    m.Av = m.alloc<float>(nparam_);
    BINDER_CUDA(cudaMemsetAsync(m.Am, 0, sizeof(float) * nparam_, m.s));
    BINDER_CUDA(cudaMemsetAsync(m.Av, 0, sizeof(float) * nparam_, m.s));
    m.loss = m.alloc<double>(1);
    for (auto &l : m.L) {
        const long M = (long)batch * l.S * l.S * l.S;
        l.wf = m.alloc<uint16_t>((size_t)l.cout * l.Kp);
        l.wb = m.alloc<uint16_t>((size_t)l.cin * l.Kq);
        l.z = m.alloc<float>((size_t)M * l.cout);
        if (l.act) l.y = m.alloc<uint16_t>((size_t)M * l.cout);
        else l.yf = m.alloc<float>((size_t)M * l.cout);
        l.dy = m.alloc<float>((size_t)M * l.cout);
    }
    auto vox = [&](int S) { return (size_t)batch * S * S * S; };
    m.x0 = m.alloc<uint16_t>(vox(S0) * in_channels);
    m.in_f = m.alloc<float>(vox(S0) * in_channels);
    m.tgt = m.alloc<float>(vox(S2) * 3);
    m.p0 = m.alloc<uint16_t>(vox(S1) * 16);
    m.p1 = m.alloc<uint16_t>(vox(S2) * 32);
    m.p2 = m.alloc<uint16_t>(vox(S3) * 64);
    m.u3 = m.alloc<uint16_t>(vox(S2) * 128);
    m.s2 = m.alloc<uint16_t>(vox(S2) * 64);
    m.dp0 = m.alloc<float>(vox(S1) * 16);
    m.dp1 = m.alloc<float>(vox(S2) * 32);
    m.dp2 = m.alloc<float>(vox(S3) * 64);
    m.du3 = m.alloc<float>(vox(S2) * 128);
    m.ds2 = m.alloc<float>(vox(S2) * 64);
    m.col = m.alloc<uint16_t>(col_max);
    m.colT = m.alloc<uint16_t>(col_max);
    m.dz = m.alloc<float>(vox(S0) * 16);
    m.dzb = m.alloc<uint16_t>(vox(S0) * 16);
    m.dzT = m.alloc<uint16_t>(dzt_max);
    // He-normal weights (the head 100 times smaller, so an untrained net predicts ~ 0), zero bias
    std::vector<float> h((size_t)nparam_, 0.0f);
    HostRng rng{seed * 0x2545F4914F6CDD1Dull + 1};
    for (size_t i = 0; i < m.L.size(); ++i) {
        const Layer &l = m.L[i];
        const double sd = std::sqrt(2.0 / (27.0 * l.cin)) * (l.act ? 1.0 : 0.01);
        for (long q = 0; q < 27L * l.cin * l.cout; ++q) h[l.woff + q] = (float)(sd * rng.normal());
    }
    set_parameters(h.data());
}

InitNet::~InitNet() {
    Impl &m = *impl_;
    cudaStreamSynchronize(m.s);
    for (void *p : m.owned) dev_free_p(p, m.s);
    cudaStreamSynchronize(m.s);
    cudaStreamDestroy(m.s);
    delete impl_;
}

void InitNet::set_parameters(const float *in) {
    Impl &m = *impl_;
    BINDER_CUDA(cudaMemcpyAsync(m.P, in, sizeof(float) * nparam_, cudaMemcpyDefault, m.s));
    for (auto &l : m.L) {
        const long n = (long)l.cout * l.Kp + (long)l.cin * l.Kq;
        count_launch(), weight_formats_kernel<<<grid_for_n(n), 256, 0, m.s>>>(
                            m.P + l.woff, l.cin, l.cout, l.Kp, l.Kq, l.wf, l.wb);
    }
    BINDER_CUDA(cudaGetLastError());
    BINDER_CUDA(cudaStreamSynchronize(m.s));
}

void InitNet::get_parameters(float *out) const {
    Impl &m = *impl_;
    BINDER_CUDA(cudaMemcpyAsync(out, m.P, sizeof(float) * nparam_, cudaMemcpyDefault, m.s));
    BINDER_CUDA(cudaStreamSynchronize(m.s));
}

double InitNet::forward_backward(const float *in, const float *target, bool backward) {
    Impl &m = *impl_;
    const cudaStream_t s = m.s;
    const int B = B_;
    auto M_of = [&](const Layer &l) { return (long)B * l.S * l.S * l.S; };
    auto im2col = [&](const uint16_t *x, int S, int C, int Kp) {
        const long chunks = (long)B * S * S * S * (Kp / 8);
        count_launch(), im2col_kernel<<<grid_for_n(chunks), 256, 0, s>>>(x, B, S, C, Kp, m.col);
    };
    auto transpose = [&](const uint16_t *src, long R, long Cc, long ldi, uint16_t *dst, long ldo) {
        const dim3 g((unsigned)((R + 31) / 32), (unsigned)((Cc + 31) / 32));
        count_launch(), transpose_bf16_kernel<<<g, dim3(32, 8), 0, s>>>(src, R, Cc, ldi, dst, ldo);
    };
    auto gemm_run = [&](const uint16_t *A, long lda, const uint16_t *Bm, long ldb, int M, int N,
                        int K, float *C, long ldc, int k_split, int acc) {
        GemmArgs g{A, Bm, C, M, N, K, lda, ldb, ldc, k_split, acc, m.err};
        launch_gemm_bf16(g, s);
    };
    auto forward = [&](Layer &l, const uint16_t *x) {
        const long M = M_of(l);
        im2col(x, l.S, l.cin, l.Kp);
        gemm_run(m.col, l.Kp, l.wf, l.Kp, (int)M, l.cout, l.Kp, l.z, l.cout, l.Kp, 0);
        count_launch(), bias_act_kernel<<<grid_for_n(M * l.cout), 256, 0, s>>>(
                            l.z, M, l.cout, l.cout, m.P + l.boff, kSlope, l.act ? 1 : 0, l.y, l.yf);
    };
    auto backward_layer = [&](Layer &l, const uint16_t *x, float *dx) {
        const long M = M_of(l);
        count_launch(), act_backward_kernel<<<grid_for_n(M * l.cout), 256, 0, s>>>(
                            l.dy, l.z, M, l.cout, l.cout, kSlope, l.act ? 1 : 0, m.dz, m.dzb);
        const int cb = (int)std::min<long>((M + 255) / 256, 64);
        count_launch(), column_sum_kernel<<<dim3((unsigned)cb, (unsigned)l.cout), 256, 0, s>>>(
                            m.dz, M, l.cout, m.G + l.boff);
        // weight gradient: dW [cout][27 cin] = dz^T . im2col(x), K = the voxels (zero-padded to a
        // multiple of 64), split over CTAs
        const long Mp = round64((int)M);
        if (Mp != M) {
            BINDER_CUDA(cudaMemsetAsync(m.dzT, 0, sizeof(uint16_t) * Mp * l.cout, s));
            BINDER_CUDA(cudaMemsetAsync(m.colT, 0, sizeof(uint16_t) * Mp * l.Kp, s));
        }
        transpose(m.dzb, M, l.cout, l.cout, m.dzT, Mp);
        im2col(x, l.S, l.cin, l.Kp);
        transpose(m.col, M, l.Kp, l.Kp, m.colT, Mp);
        long splits = Mp / 4096;
        splits = splits < 1 ? 1 : (splits > 256 ? 256 : splits);
        const int ks = round64((int)((Mp + splits - 1) / splits));
        gemm_run(m.dzT, Mp, m.colT, Mp, l.cout, 27 * l.cin, (int)Mp, m.G + l.woff, 27L * l.cin, ks,
                 1);
        // data gradient: dx [M][cin] += im2col(dz) . flipped W, accumulated onto what dx holds
        if (dx) {
            im2col(m.dzb, l.S, l.cout, l.Kq);
            gemm_run(m.col, l.Kq, l.wb, l.Kq, (int)M, l.cin, l.Kq, dx, l.cin, l.Kq, 1);
        }
    };
    auto vox = [&](int S) { return (long)B * S * S * S; };
    std::vector<Layer> &L = m.L;
    const int S0 = S_, S1 = S_ / 2, S2 = S_ / 4, S3 = S_ / 8;

    BINDER_CUDA(cudaMemcpyAsync(m.in_f, in, sizeof(float) * vox(S0) * Cin_, cudaMemcpyDefault, s));
    count_launch(), to_bf16_kernel<<<grid_for_n(vox(S0) * Cin_), 256, 0, s>>>(m.in_f, vox(S0) * Cin_,
                                                                              m.x0);
    forward(L[0], m.x0);
    forward(L[1], L[0].y);
    count_launch(), avgpool2_kernel<<<grid_for_n(vox(S1) * 16), 256, 0, s>>>(L[1].y, B, S0, 16, m.p0);
    forward(L[2], m.p0);
    forward(L[3], L[2].y);
    count_launch(), avgpool2_kernel<<<grid_for_n(vox(S2) * 32), 256, 0, s>>>(L[3].y, B, S1, 32, m.p1);
    forward(L[4], m.p1);
    forward(L[5], L[4].y);
    count_launch(), avgpool2_kernel<<<grid_for_n(vox(S3) * 64), 256, 0, s>>>(L[5].y, B, S2, 64, m.p2);
    forward(L[6], m.p2);
    forward(L[7], L[6].y);
    count_launch(), upsample2_kernel<<<grid_for_n(vox(S2) * 128), 256, 0, s>>>(L[7].y, B, S3, 128, m.u3);
    forward(L[8], m.u3);
    count_launch(), add_bf16_kernel<<<grid_for_n(vox(S2) * 64), 256, 0, s>>>(L[8].y, L[5].y,
                                                                              vox(S2) * 64, m.s2);
    forward(L[9], m.s2);
    forward(L[10], L[9].y);
    BINDER_CUDA(cudaGetLastError());
    if (!target) return 0.0;

    BINDER_CUDA(cudaMemcpyAsync(m.tgt, target, sizeof(float) * vox(S2) * 3, cudaMemcpyDefault, s));
    BINDER_CUDA(cudaMemsetAsync(m.loss, 0, sizeof(double), s));
    count_launch(), mse_kernel<<<grid_for_n(vox(S2) * 3), 256, 0, s>>>(L[10].yf, m.tgt, vox(S2) * 3,
                                                                       m.loss, L[10].dy);
    if (backward) {
        BINDER_CUDA(cudaMemsetAsync(m.G, 0, sizeof(float) * nparam_, s));
        for (size_t i = 0; i < L.size() - 1; ++i)
            BINDER_CUDA(cudaMemsetAsync(L[i].dy, 0, sizeof(float) * M_of(L[i]) * L[i].cout, s));
        BINDER_CUDA(cudaMemsetAsync(m.dp0, 0, sizeof(float) * vox(S1) * 16, s));
        BINDER_CUDA(cudaMemsetAsync(m.dp1, 0, sizeof(float) * vox(S2) * 32, s));
        BINDER_CUDA(cudaMemsetAsync(m.dp2, 0, sizeof(float) * vox(S3) * 64, s));
        BINDER_CUDA(cudaMemsetAsync(m.du3, 0, sizeof(float) * vox(S2) * 128, s));
        BINDER_CUDA(cudaMemsetAsync(m.ds2, 0, sizeof(float) * vox(S2) * 64, s));
        backward_layer(L[10], L[9].y, L[9].dy);
        backward_layer(L[9], m.s2, m.ds2);
        // the skip sum feeds the decoder convolution and the encoder's level-2 output
        BINDER_CUDA(cudaMemcpyAsync(L[8].dy, m.ds2, sizeof(float) * vox(S2) * 64,
                                    cudaMemcpyDeviceToDevice, s));
        count_launch(), add_f32_kernel<<<grid_for_n(vox(S2) * 64), 256, 0, s>>>(L[5].dy, m.ds2,
                                                                                 vox(S2) * 64);
        backward_layer(L[8], m.u3, m.du3);
        count_launch(), upsample2_backward_kernel<<<grid_for_n(vox(S3) * 128), 256, 0, s>>>(
                            m.du3, B, S3, 128, L[7].dy);
        backward_layer(L[7], L[6].y, L[6].dy);
        backward_layer(L[6], m.p2, m.dp2);
        count_launch(), avgpool2_backward_kernel<<<grid_for_n(vox(S2) * 64), 256, 0, s>>>(
                            m.dp2, B, S2, 64, L[5].dy);
        backward_layer(L[5], L[4].y, L[4].dy);
        backward_layer(L[4], m.p1, m.dp1);
        count_launch(), avgpool2_backward_kernel<<<grid_for_n(vox(S1) * 32), 256, 0, s>>>(
                            m.dp1, B, S1, 32, L[3].dy);
        backward_layer(L[3], L[2].y, L[2].dy);
        backward_layer(L[2], m.p0, m.dp0);
        count_launch(), avgpool2_backward_kernel<<<grid_for_n(vox(S0) * 16), 256, 0, s>>>(
                            m.dp0, B, S0, 16, L[1].dy);
        backward_layer(L[1], L[0].y, L[0].dy);
        backward_layer(L[0], m.x0, nullptr);
        BINDER_CUDA(cudaGetLastError());
    }
    double loss = 0.0;
    int err = 0;
    BINDER_CUDA(cudaMemcpyAsync(&loss, m.loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaMemcpyAsync(&err, m.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    BINDER_CUDA(cudaStreamSynchronize(s));
    if (err) throw Error(kDeviceFault, "a tensor-core GEMM wait timed out");
    return loss;
}

void InitNet::predict(const float *in, float *out) {
    Impl &m = *impl_;
    forward_backward(in, nullptr, false);
    const long n = (long)B_ * (S_ / 4) * (S_ / 4) * (S_ / 4) * 3;
    BINDER_CUDA(cudaMemcpyAsync(out, m.L.back().yf, sizeof(float) * n, cudaMemcpyDefault, m.s));
    int err = 0;
    BINDER_CUDA(cudaMemcpyAsync(&err, m.err, sizeof(int), cudaMemcpyDeviceToHost, m.s));
    BINDER_CUDA(cudaStreamSynchronize(m.s));
    if (err) throw Error(kDeviceFault, "a tensor-core GEMM wait timed out");
}

double InitNet::gradients(const float *in, const float *target, float *grads_out) {
    Impl &m = *impl_;
    const double loss = forward_backward(in, target, true);
    if (grads_out) {
        BINDER_CUDA(cudaMemcpyAsync(grads_out, m.G, sizeof(float) * nparam_, cudaMemcpyDefault,
                                    m.s));
        BINDER_CUDA(cudaStreamSynchronize(m.s));
    }
    return loss;
}

double InitNet::train_step(const float *in, const float *target, double lr, float *grads_out) {
    Impl &m = *impl_;
    const double loss = gradients(in, target, grads_out);
    ++m.adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)m.adam_t), c2 = 1.0f - std::pow(b2, (float)m.adam_t);
    count_launch(), adam_kernel<<<grid_for_n(nparam_), 256, 0, m.s>>>(m.P, m.G, m.Am, m.Av, nparam_,
                                                                       (float)lr, b1, b2, 1e-8f, c1, c2);
    for (auto &l : m.L) {
        const long n = (long)l.cout * l.Kp + (long)l.cin * l.Kq;
        count_launch(), weight_formats_kernel<<<grid_for_n(n), 256, 0, m.s>>>(
                            m.P + l.woff, l.cin, l.cout, l.Kp, l.Kq, l.wf, l.wb);
    }
    BINDER_CUDA(cudaGetLastError());
    return loss;
}

void gemm_bf16_host(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K) {
    BINDER_CHECK(M > 0 && N > 0 && K > 0 && K % 64 == 0, "M, N > 0 and K a positive multiple of 64");
    cudaStream_t s = nullptr;
    BINDER_CUDA(cudaStreamCreate(&s));
    uint16_t *a = nullptr, *b = nullptr;
    float *c = nullptr;
    int *err = nullptr;
    try {
        a = dev_alloc_n<uint16_t>((size_t)M * K, s);
        b = dev_alloc_n<uint16_t>((size_t)N * K, s);
        c = dev_alloc_n<float>((size_t)M * N, s);
        err = dev_alloc_n<int>(1, s);
        BINDER_CUDA(cudaMemcpyAsync(a, A, sizeof(uint16_t) * M * K, cudaMemcpyHostToDevice, s));
        BINDER_CUDA(cudaMemcpyAsync(b, B, sizeof(uint16_t) * N * K, cudaMemcpyHostToDevice, s));
        BINDER_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        // K split over CTAs when K is long (atomic accumulation), as the weight gradients run
        const int ks = K > 4096 ? 1024 : K;
        if (ks < K) BINDER_CUDA(cudaMemsetAsync(c, 0, sizeof(float) * M * N, s));
        GemmArgs g{a, b, c, M, N, K, K, K, N, ks, ks < K ? 1 : 0, err};
        launch_gemm_bf16(g, s);
        int h = 0;
        BINDER_CUDA(cudaMemcpyAsync(C, c, sizeof(float) * M * N, cudaMemcpyDeviceToHost, s));
        BINDER_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        BINDER_CUDA(cudaStreamSynchronize(s));
        if (h) throw Error(kDeviceFault, "a tensor-core GEMM wait timed out");
    } catch (...) {
        dev_free_p(a, s); dev_free_p(b, s); dev_free_p(c, s); dev_free_p(err, s);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    dev_free_p(a, s); dev_free_p(b, s); dev_free_p(c, s); dev_free_p(err, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
}

}  // namespace binder
