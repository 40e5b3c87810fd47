// Tensor-core (tcgen05 / TMEM) version of the separable transform passes of transform.cu.
//
// One CTA (4 warps) owns a tile of 128 lines of one component.  The pass is the GEMM
//   D[line][k] = sum_j X[line][j] * M[k][j]      (M = the n x n transform, rows = outputs)
// with A = the 128 x n data tile and B = M, both K-major in shared memory in the canonical
// no-swizzle layout (8-row x 16-byte core matrices), streamed in K chunks of 16 (A: registers
// prefetched one chunk ahead into a 2-stage ring; B: cp.async into a 3-slot ring one chunk ahead),
// accumulated in TMEM by tcgen05.mma (M = 128, N = n padded to 16).
// Precision: TF32 operands (one plane), or "3xTF32" -- hi/lo TF32 planes and the three products
// hi*hi + hi*lo + lo*hi, which keeps FP32-level accuracy -- always with FP32 accumulation.
// The x-axis pass of the DCT prior is fused: forward GEMM into TMEM columns [0, Npad), the prior
// scaling / noise / costs applied while TMEM chunks are re-staged as the A operand of the inverse
// GEMM, which accumulates into TMEM columns [Npad, 2 Npad).
#include <cmath>
#include <cstring>
#include <vector>

#include "layout.cuh"
#include "transform.cuh"
#include "umma.cuh"
#include <cuda_bf16.h>

#include "umma_transform.cuh"

namespace binder {
namespace {

constexpr int kLines = 128;            // UMMA M
constexpr int kKC = 16;                // K elements per pipeline chunk
constexpr int kAPlane = kLines * kKC;  // floats per A plane per stage (8 KB)
constexpr uint64_t kWaitLimit = 2000000000ull;  // 2 s of wall time per barrier wait

struct UArgs {
    const float *in;
    float *out;
    long V;
    int n, Npad, nkc;
    long outer, s;
    const float *B1, *B2;  // preformatted [nkc][2 planes][Npad * kKC]
    // spectral epilogue
    const float *D;
    DevState *st;
    double sigma2;
    int sample, want_raw, every;
    const float *noise;  // precomputed prior-sampling normals [components][V], or null
    uint64_t seed;
    uint32_t chain;
    double rho_p;
    double eta2[3];
    // positions epilogue
    const float *xpos;
    int ny, nz;
    int dims;  // 3, or 2 for an image (the contiguous axis is then component 1)
    int comp0;  // component of blockIdx.z == 0
    int ncomp;  // components of one persistent launch
    int chain_comps;  // components per chain of a batch of chains (0: one chain)
    const int *skip;
};

// out of line: the epilogue loops are unrolled, and an inlined Philox + Box-Muller per element
// would bloat them (instruction-cache misses) even in EM, where the branch is never taken
__device__ __noinline__ float prior_normal_tc(uint64_t seed, uint32_t i, uint32_t sweep,
                                              uint32_t chain, int comp) {
    const u32x4 r = philox_draw(seed, i, sweep, comp < 2 ? 2u : 3u, chain);
    const float u1 = u01_f24(r.x), u2 = u01_f24(r.y);
    const float rad = sqrtf(-2.0f * logf(u1));
    float sn, cs;
    sincospif(2.0f * u2, &sn, &cs);
    return comp == 1 ? rad * sn : rad * cs;
}

// 16-byte slot of the K-major A plane holding row `line`, K elements 4q .. 4q+3 of the chunk:
// 16-byte K columns 2 KB apart (LBO), 8-row groups 128 B apart (SBO), rows 16 B apart
__device__ __forceinline__ int a_slot(int line, int q) {
    return q * 512 + (line >> 3) * 32 + (line & 7) * 4;
}

template <int PLANES>
__device__ __forceinline__ void store_split(float *plane0, int off, float4 v) {
    const float4 hi = make_float4(umma::to_tf32(v.x), umma::to_tf32(v.y), umma::to_tf32(v.z),
                                  umma::to_tf32(v.w));
    *reinterpret_cast<float4 *>(plane0 + off) = hi;
    if (PLANES == 2) {
        const float4 lo = make_float4(umma::to_tf32(v.x - hi.x), umma::to_tf32(v.y - hi.y),
                                      umma::to_tf32(v.z - hi.z), umma::to_tf32(v.w - hi.w));
        *reinterpret_cast<float4 *>(plane0 + kAPlane + off) = lo;
    }
}

// byte offset in a BF16 A plane of row `line`, K elements 4q .. 4q+3 of the chunk: two 16-byte K
// columns of 8 elements 2 KB apart (LBO), 8-row groups 128 B apart (SBO), rows 16 B apart; four
// elements fill half of a 16-byte slot
__device__ __forceinline__ int a_slot_b16(int line, int q) {
    return (q >> 1) * 2048 + (line >> 3) * 128 + (line & 7) * 16 + (q & 1) * 8;
}

// FP32 -> BF16 hi (round to nearest even) and, with PLANES == 2, lo = BF16(x - hi): the split of
// the 3-product BF16 pass (hi.hi + hi.lo + lo.hi keeps ~16 mantissa bits of every product)
template <int PLANES>
__device__ __forceinline__ void store_split_b16(unsigned char *plane0, int off, float4 v) {
    const __nv_bfloat162 h01 = __floats2bfloat162_rn(v.x, v.y);
    const __nv_bfloat162 h23 = __floats2bfloat162_rn(v.z, v.w);
    uint2 hw;
    hw.x = *reinterpret_cast<const uint32_t *>(&h01);
    hw.y = *reinterpret_cast<const uint32_t *>(&h23);
    *reinterpret_cast<uint2 *>(plane0 + off) = hw;
    if (PLANES == 2) {
        // hi as FP32: the BF16 bits in the upper half of the word (exact)
        const float hx = __uint_as_float(hw.x << 16), hy = __uint_as_float(hw.x & 0xffff0000u);
        const float hz = __uint_as_float(hw.y << 16), hq = __uint_as_float(hw.y & 0xffff0000u);
        const __nv_bfloat162 l01 = __floats2bfloat162_rn(v.x - hx, v.y - hy);
        const __nv_bfloat162 l23 = __floats2bfloat162_rn(v.z - hz, v.w - hq);
        uint2 lw;
        lw.x = *reinterpret_cast<const uint32_t *>(&l01);
        lw.y = *reinterpret_cast<const uint32_t *>(&l23);
        *reinterpret_cast<uint2 *>(plane0 + kAPlane * 2 + off) = lw;
    }
}

// A chunk for this thread: contiguous axis -> 4 float4 of 4 lines; strided -> its own line
struct AChunk {
    float4 v[4];
};

template <int MODE, int PLANES>
__global__ void __launch_bounds__(128, 2) umma_axis_kernel(const UArgs a) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Npad = a.Npad, n = a.n;
    const uint32_t bplane = (uint32_t)Npad * kKC;  // floats per B plane
    float *As = reinterpret_cast<float *>(smem_raw);   // [2 stages][PLANES][kAPlane]
    float *Bs = As + 2 * PLANES * kAPlane;             // [3 slots][PLANES][bplane]
    uint64_t *mbar = reinterpret_cast<uint64_t *>(Bs + 3 * PLANES * bplane);  // [3]
    uint32_t *holder = reinterpret_cast<uint32_t *>(mbar + 3);
    int *s_err = reinterpret_cast<int *>(holder + 1);
    __shared__ double red[32];

    const bool fused = (MODE == kEpiSpectral);
    const uint32_t want = fused ? 2u * Npad : (uint32_t)Npad;
    uint32_t ncols = 32;
    while (ncols < want) ncols <<= 1;

    if (warp == 0) umma::tmem_alloc(holder, ncols);
    if (tid == 0) {
        umma::mbar_init(&mbar[0], 1);
        umma::mbar_init(&mbar[1], 1);
        umma::mbar_init(&mbar[2], 1);
        *s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *holder;
    const uint32_t tlane = (uint32_t)(warp * 32) << 16;

    const int comp = a.comp0 + (int)blockIdx.z;
    // components of a batch of chains are numbered chain * chain_comps + component: the chain
    // picks the state and the Philox chain index, the component within it everything else
    const int bch = a.chain_comps ? comp / a.chain_comps : 0;
    const int cn = comp - bch * a.chain_comps;
    DevState *const st = a.st ? a.st + bch : nullptr;
    const uint32_t chain = a.chain + (uint32_t)bch;
    const float *in = a.in + comp * a.V;
    float *out = a.out + comp * a.V;
    const long nlines = a.outer * a.s;
    const long l0 = (long)blockIdx.x * kLines;
    const bool contig = (a.s == 1);
    // this thread's line (TMEM lane == tile row == tid)
    const long lg = l0 + tid;
    const bool valid = lg < nlines;
    const long o = valid ? lg / a.s : 0, t = valid ? lg - o * a.s : 0;
    const long lbase = o * (long)n * a.s + t;  // element (line, j) at lbase + j * s
    const uint32_t idesc = umma::instr_desc(kLines, Npad, umma::kFmtTF32);
    // contiguous-axis load mapping: 8 lines x 4 float4 per warp instruction
    const int cr = lane & 7, cq = lane >> 3;

    uint32_t chunk = 0;  // running chunk counter over both GEMMs: stage = chunk & 1
    double part_cost = 0.0, part_raw = 0.0;
    const uint32_t sweep = ((MODE == kEpiSpectral || MODE == kEpiSpectralOut) && a.sample) ? (uint32_t)st->sweep : 0u;
    const bool want_raw = (MODE == kEpiSpectral || MODE == kEpiSpectralOut) && a.want_raw && (st->sweep % a.every == 0);
    const double gamma = (MODE == kEpiSpectral || MODE == kEpiSpectralOut) ? st->gamma[cn] : 0.0;
    const float gs2 = (float)(gamma * a.sigma2);

    auto load_global = [&](int kc, AChunk &r) {
        if (contig) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int line = (warp + 4 * i) * 8 + cr;
                const long g = l0 + line;
                const int j0 = kc * kKC + cq * 4;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (g < nlines) {
                    const float *p = in + g * n + j0;
                    if ((n & 3) == 0 && j0 + 3 < n) {
                        v = __ldg(reinterpret_cast<const float4 *>(p));
                    } else {
                        v.x = j0 < n ? __ldg(p) : 0.f;
                        v.y = j0 + 1 < n ? __ldg(p + 1) : 0.f;
                        v.z = j0 + 2 < n ? __ldg(p + 2) : 0.f;
                        v.w = j0 + 3 < n ? __ldg(p + 3) : 0.f;
                    }
                }
                r.v[i] = v;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j0 = kc * kKC + q * 4;
                float4 v;
                v.x = (valid && j0 < n) ? __ldg(in + lbase + (long)j0 * a.s) : 0.f;
                v.y = (valid && j0 + 1 < n) ? __ldg(in + lbase + (long)(j0 + 1) * a.s) : 0.f;
                v.z = (valid && j0 + 2 < n) ? __ldg(in + lbase + (long)(j0 + 2) * a.s) : 0.f;
                v.w = (valid && j0 + 3 < n) ? __ldg(in + lbase + (long)(j0 + 3) * a.s) : 0.f;
                r.v[q] = v;
            }
        }
    };
    auto store_global_chunk = [&](const AChunk &r, float *Ap) {
        if (contig) {
#pragma unroll
            for (int i = 0; i < 4; ++i) store_split<PLANES>(Ap, a_slot((warp + 4 * i) * 8 + cr, cq), r.v[i]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) store_split<PLANES>(Ap, a_slot(tid, q), r.v[q]);
        }
    };

    // ---- one GEMM into TMEM columns [col_off, col_off + Npad); src 0 = global, 1 = TMEM acc0 ----
    // A ring of 2 stages, B ring of 3: the B chunk for c+1 is requested (cp.async) as soon as the
    // MMAs of chunk c-2 are known complete, so its L2 latency overlaps chunk c.
    auto issue_b = [&](const float *Bg, int kc, uint32_t c) {
        if (kc < a.nkc) {
            const float *srcb = Bg + (size_t)kc * 2 * bplane;
            float *Bp = Bs + (c % 3) * PLANES * bplane;
            const int nv = PLANES * (int)bplane / 4;
            for (int qv = tid; qv < nv; qv += 128) umma::cp_async16(Bp + 4 * qv, srcb + 4 * qv);
        }
        umma::cp_async_commit();  // possibly empty: keeps one group per chunk
    };
    auto gemm = [&](const float *Bg, uint32_t col_off, int src) {
        AChunk pre;
        float dpre[16];
        if (src == 0) load_global(0, pre);
        auto load_d = [&](int kc) {
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int k = kc * kKC + m;
                dpre[m] = (valid && k < n) ? __ldg(a.D + (long)k * a.s + t) : 0.0f;
            }
        };
        if (src == 1) load_d(0);
        issue_b(Bg, 0, chunk);
        for (int kc = 0; kc < a.nkc; ++kc) {
            const uint32_t c = chunk++;
            const int stage = c & 1;
            // one thread waits for the MMAs that last read this stage; the rest wait at the barrier
            if (tid == 0 && c >= 2 && !umma::mbar_wait(&mbar[stage], ((c >> 1) - 1) & 1, kWaitLimit))
                *s_err = 1;
            __syncthreads();
            if (*s_err) {
                umma::cp_async_wait_all();
                return;
            }
            issue_b(Bg, kc + 1, c + 1);  // its ring slot was last read by chunk c - 2
            float *Ap = As + stage * PLANES * kAPlane;
            float *Bp = Bs + (c % 3) * PLANES * bplane;
            // A operand
            if (src == 0) {
                store_global_chunk(pre, Ap);
                if (kc + 1 < a.nkc) load_global(kc + 1, pre);  // in flight during this chunk's MMAs
            } else {
                // fused x pass: forward coefficients of this chunk from TMEM, prior scaling,
                // noise and costs, re-staged as the A operand of the inverse GEMM
                float v[16];
                umma::tmem_ld16(tmem + tlane + (uint32_t)(kc * kKC), v);
                float ccost = 0.0f;
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const int k = kc * kKC + m;
                    float cval = 0.0f;
                    if (valid && k < n) {
                        const float Dv = dpre[m];
                        const float f = __frcp_rn(fmaf(gs2, Dv, 1.0f));
                        cval = v[m] * f;
                        if (a.sample)
                            cval += sqrtf((float)a.sigma2 * f) *
                                    prior_normal_tc(a.seed, (uint32_t)((long)k * a.s + t), sweep,
                                                    chain, cn);
                        ccost += Dv * cval * cval;
                    }
                    v[m] = cval;
                }
                part_cost += 0.5 * gamma * (double)ccost;
                if (want_raw) part_raw += a.eta2[cn] * a.rho_p * (double)ccost;
                if (kc + 1 < a.nkc) load_d(kc + 1);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    store_split<PLANES>(Ap, a_slot(tid, q),
                                        make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]));
            }
            asm volatile("cp.async.wait_group 1;" ::: "memory");  // B chunk c has landed
            umma::fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) {
                umma::fence_after_sync();
                const uint32_t abase = umma::smem_u32(Ap), bbase = umma::smem_u32(Bp);
#pragma unroll
                for (int ks = 0; ks < kKC / 8; ++ks) {
                    const uint32_t ao = (uint32_t)ks * 2u * 2048u;
                    const uint32_t bo = (uint32_t)ks * 2u * (uint32_t)Npad * 16u;
                    const uint64_t ahi = umma::smem_desc(abase + ao, 2048u, 128u);
                    const uint64_t bhi = umma::smem_desc(bbase + bo, (uint32_t)Npad * 16u, 128u);
                    umma::mma_tf32(tmem + col_off, ahi, bhi, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
                    if (PLANES == 2) {
                        const uint64_t alo = umma::smem_desc(abase + kAPlane * 4u + ao, 2048u, 128u);
                        const uint64_t blo =
                            umma::smem_desc(bbase + bplane * 4u + bo, (uint32_t)Npad * 16u, 128u);
                        umma::mma_tf32(tmem + col_off, ahi, blo, idesc, 1u);
                        umma::mma_tf32(tmem + col_off, alo, bhi, idesc, 1u);
                    }
                }
                umma::commit(&mbar[stage]);
            }
        }
        umma::cp_async_wait_all();  // the trailing (empty) group
        // wait for the whole accumulation
        const uint32_t last = chunk - 1;
        if (tid == 0 && !umma::mbar_wait(&mbar[last & 1], (last >> 1) & 1, kWaitLimit)) *s_err = 1;
        __syncthreads();
        umma::fence_after_sync();
    };

    gemm(a.B1, 0u, 0);
    uint32_t acc_col = 0;
    if (fused && !*s_err) {
        gemm(a.B2, (uint32_t)Npad, 1);
        acc_col = (uint32_t)Npad;
    }

    if (!*s_err) {
        // ---- epilogue: 32 TMEM columns at a time -------------------------------------------
        const int nchunks = (n + 31) / 32;
        if (contig) {
            // each warp stages its 32 lines x 32 columns in shared memory (row pitch 33, no bank
            // conflicts) and writes them back as coalesced 128-byte rows; the pipeline buffers
            // are free once the accumulation has completed
            float *stg = reinterpret_cast<float *>(smem_raw) + warp * 32 * 33;
            // positions pass (z axis): row g = x * ny + y; each lane owns the coordinate of row
            // `lane` of this warp and the row loop broadcasts it
            float rowc = 0.0f;
            if (MODE == kEpiPositions && !a.xpos) {
                const int gi = (int)(l0 + warp * 32 + lane);  // 3D: x * ny + y; 2D: x
                rowc = a.dims == 2 ? (float)gi
                                   : (cn == 0 ? (float)(gi / a.ny) : (float)(gi % a.ny));
            }
            for (int cc = 0; cc < nchunks; ++cc) {
                float v[32];
                umma::tmem_ld32(tmem + tlane + acc_col + (uint32_t)(cc * 32), v);
#pragma unroll
                for (int m = 0; m < 32; ++m) stg[lane * 33 + m] = v[m];
                __syncwarp();
                const int k = cc * 32 + lane;
#pragma unroll 4
                for (int r = 0; r < 32; ++r) {
                    const long g = l0 + warp * 32 + r;
                    const float rc = __shfl_sync(0xffffffffu, rowc, r);
                    if (g < nlines && k < n) {
                        float val = stg[r * 33 + lane];
                        if (MODE == kEpiPositions)
                            val += a.xpos ? __ldg(a.xpos + cn * a.V + g * n + k)
                                          : (cn == a.dims - 1 ? (float)k : rc);
                        out[g * n + k] = val;
                    }
                }
                __syncwarp();
            }
        } else {
            // prior eigenvalues of coefficient (k, t) at flat index k * s + t, one 32-chunk ahead
            // in registers: loaded beside the stores to `out` they would be serialised behind them
            float dnext[32];
            auto load_dchunk = [&](int cc) {
#pragma unroll
                for (int m = 0; m < 32; ++m) {
                    const int k = cc * 32 + m;
                    dnext[m] = (valid && k < n) ? __ldg(a.D + (long)k * a.s + t) : 0.0f;
                }
            };
            if (MODE == kEpiSpectralOut) load_dchunk(0);
            for (int cc = 0; cc < nchunks; ++cc) {
                float v[32], dcur[32];
                umma::tmem_ld32(tmem + tlane + acc_col + (uint32_t)(cc * 32), v);
                if (MODE == kEpiSpectralOut) {
#pragma unroll
                    for (int m = 0; m < 32; ++m) dcur[m] = dnext[m];
                    if (cc + 1 < nchunks) load_dchunk(cc + 1);
                }
                if (!valid) continue;
                // prior costs of this chunk: FP32 partial sums over 32 coefficients, FP64 across
                float ccost = 0.0f, craw = 0.0f;
                float *op = out + lbase;
#pragma unroll
                for (int m = 0; m < 32; ++m) {
                    const int k = cc * 32 + m;
                    if (k < n) {
                        float val = v[m];
                        if (MODE == kEpiSpectralOut) {
                            // forward x pass: coefficient (k, t) has flat index k * s + t
                            const float Dv = dcur[m];
                            const float f = __frcp_rn(fmaf(gs2, Dv, 1.0f));
                            val *= f;
                            if (a.sample)
                                val += sqrtf((float)a.sigma2 * f) *
                                       prior_normal_tc(a.seed, (uint32_t)((long)k * a.s + t), sweep,
                                                       chain, cn);
                            const float dv2 = Dv * val * val;
                            ccost += dv2;
                            craw += dv2;
                        }
                        op[(long)k * a.s] = val;
                    }
                }
                if (MODE == kEpiSpectralOut) {
                    part_cost += 0.5 * gamma * (double)ccost;
                    if (want_raw) part_raw += a.eta2[cn] * a.rho_p * (double)craw;
                }
            }
        }
    }

    if (MODE == kEpiSpectral || MODE == kEpiSpectralOut) {
        const double sc = block_sum(part_cost, red);
        if (tid == 0) atomicAdd(&st->lp_tr, sc);
        if (a.want_raw) {
            const double sr = block_sum(part_raw, red);
            if (tid == 0) atomicAdd(&st->raw_reg, sr);
        }
    }

    // ---- teardown: after an error, drain every tcgen05 op still in flight (bounded) -------------
    if (*s_err) {
        umma::cp_async_wait_all();
        if (tid == 0) {
            umma::commit(&mbar[2]);
            umma::mbar_wait(&mbar[2], 0, kWaitLimit);
            if (st) atomicOr(&st->flags, (unsigned)kFlagTensorTimeout);
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, ncols);
}


// ---- warp-specialised pass: 4 producer / epilogue warps + 1 MMA warp -------------------------
// Warps 0-3 own the tile's 128 lines (thread tid <-> line tid <-> TMEM lane tid): they load the
// data chunks from global memory (prefetched kPre chunks ahead in registers), split them into
// TF32 planes in an A stage, copy their part of the matrix chunk into a B slot (cp.async), and
// arrive on full[stage].  Warp 4 (one lane) waits on full[], issues the chunk's MMAs and commits
// them to done[]; the producers only wait on done[] before reusing a stage, two chunks later, so
// the MMA issue -- which blocks while the tensor core's queue is full -- never stalls them.
constexpr int kWsThreads = 160;
constexpr int kPre = 2;  // A chunks in flight per producer thread

template <int MODE, int PLANES, bool BF>
__global__ void __launch_bounds__(kWsThreads, 2) umma_ws_kernel(const UArgs a) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp < 4;
    const int Npad = a.Npad, n = a.n, nkc = a.nkc;
    // operands are TF32 in 4-byte elements, or BF16 (BF) in 2-byte elements with the same
    // canonical layout of 16-byte K columns
    constexpr uint32_t EB = BF ? 2u : 4u;
    constexpr uint32_t kAPlaneB = kAPlane * EB;            // bytes per A plane
    const uint32_t bplaneB = (uint32_t)Npad * kKC * EB;    // bytes per B plane
    unsigned char *As = smem_raw;                          // [2 stages][PLANES][kAPlaneB]
    unsigned char *Bs = As + 2 * PLANES * kAPlaneB;        // [3 slots][PLANES][bplaneB]
    uint64_t *full = reinterpret_cast<uint64_t *>(Bs + 3 * PLANES * bplaneB);  // [2]
    uint64_t *done = full + 2;                                               // [3]
    uint64_t *drain = done + 3;                                              // [1]
    uint32_t *holder = reinterpret_cast<uint32_t *>(drain + 1);
    int *s_err = reinterpret_cast<int *>(holder + 1);
    __shared__ double red[32];

    uint32_t ncols = 32;
    while (ncols < (uint32_t)Npad) ncols <<= 1;
    if (warp == 0) umma::tmem_alloc(holder, ncols);
    if (tid == 32) {
        umma::mbar_init(&full[0], 128);
        umma::mbar_init(&full[1], 128);
        for (int i = 0; i < 3; ++i) umma::mbar_init(&done[i], 1);
        umma::mbar_init(drain, 1);
        *s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *holder;
    const uint32_t tlane = (uint32_t)((warp & 3) * 32) << 16;

    const int comp = a.comp0 + (int)blockIdx.z;
    // components of a batch of chains are numbered chain * chain_comps + component: the chain
    // picks the state (and, in the noise buffer, its block of components), the component within
    // it everything else
    const int bch = a.chain_comps ? comp / a.chain_comps : 0;
    const int cn = comp - bch * a.chain_comps;
    DevState *const st = a.st ? a.st + bch : nullptr;
    const float *in = a.in + comp * a.V;
    float *out = a.out + comp * a.V;
    const long nlines = a.outer * a.s;
    const long l0 = (long)blockIdx.x * kLines;
    const bool contig = (a.s == 1);
    const long lg = l0 + (producer ? tid : 0);
    const bool valid = producer && lg < nlines;
    const long o = valid ? lg / a.s : 0, t = valid ? lg - o * a.s : 0;
    const long lbase = o * (long)n * a.s + t;  // element (line, j) at lbase + j * s
    const int cr = lane & 7, cq = lane >> 3;   // contiguous-axis load mapping
    float dfirst[32];  // prior eigenvalues of the epilogue's first 32 coefficients

    if (!producer) {
        // ---- MMA warp ------------------------------------------------------------------------
        if (lane == 0) {
            const uint32_t idesc =
                umma::instr_desc(kLines, Npad, BF ? umma::kFmtBF16 : umma::kFmtTF32);
            for (int kc = 0; kc < nkc; ++kc) {
                if (!umma::mbar_wait(&full[kc & 1], (uint32_t)(kc >> 1) & 1u, kWaitLimit) ||
                    *(volatile int *)s_err) {
                    *(volatile int *)s_err = 1;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t abase = umma::smem_u32(As + (kc & 1) * PLANES * kAPlaneB);
                const uint32_t bbase = umma::smem_u32(Bs + (kc % 3) * PLANES * bplaneB);
                if (BF) {
                    // one kind::f16 MMA (K = 16) covers the chunk: its two 16-byte K columns
                    const uint64_t ahi = umma::smem_desc(abase, 2048u, 128u);
                    const uint64_t bhi = umma::smem_desc(bbase, (uint32_t)Npad * 16u, 128u);
                    umma::mma_bf16(tmem, ahi, bhi, idesc, kc > 0 ? 1u : 0u);
                    if (PLANES == 2) {
                        const uint64_t alo = umma::smem_desc(abase + kAPlaneB, 2048u, 128u);
                        const uint64_t blo =
                            umma::smem_desc(bbase + bplaneB, (uint32_t)Npad * 16u, 128u);
                        umma::mma_bf16(tmem, ahi, blo, idesc, 1u);
                        umma::mma_bf16(tmem, alo, bhi, idesc, 1u);
                    }
                } else {
#pragma unroll
                    for (int ks = 0; ks < kKC / 8; ++ks) {
                        const uint32_t ao = (uint32_t)ks * 2u * 2048u;
                        const uint32_t bo = (uint32_t)ks * 2u * (uint32_t)Npad * 16u;
                        const uint64_t ahi = umma::smem_desc(abase + ao, 2048u, 128u);
                        const uint64_t bhi =
                            umma::smem_desc(bbase + bo, (uint32_t)Npad * 16u, 128u);
                        umma::mma_tf32(tmem, ahi, bhi, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
                        if (PLANES == 2) {
                            const uint64_t alo =
                                umma::smem_desc(abase + kAPlaneB + ao, 2048u, 128u);
                            const uint64_t blo = umma::smem_desc(bbase + bplaneB + bo,
                                                                 (uint32_t)Npad * 16u, 128u);
                            umma::mma_tf32(tmem, ahi, blo, idesc, 1u);
                            umma::mma_tf32(tmem, alo, bhi, idesc, 1u);
                        }
                    }
                }
                umma::commit(&done[kc % 3]);
            }
        }
    } else {
        // ---- producers -----------------------------------------------------------------------
        auto load_global = [&](int kc, AChunk &r) {
            if (kc >= nkc) return;
            if (contig) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int line = (warp + 4 * i) * 8 + cr;
                    const long g = l0 + line;
                    const int j0 = kc * kKC + cq * 4;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (g < nlines) {
                        const float *p = in + g * n + j0;
                        if ((n & 3) == 0 && j0 + 3 < n) {
                            v = __ldg(reinterpret_cast<const float4 *>(p));
                        } else {
                            v.x = j0 < n ? __ldg(p) : 0.f;
                            v.y = j0 + 1 < n ? __ldg(p + 1) : 0.f;
                            v.z = j0 + 2 < n ? __ldg(p + 2) : 0.f;
                            v.w = j0 + 3 < n ? __ldg(p + 3) : 0.f;
                        }
                    }
                    r.v[i] = v;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int j0 = kc * kKC + q * 4;
                    float4 v;
                    v.x = (valid && j0 < n) ? __ldg(in + lbase + (long)j0 * a.s) : 0.f;
                    v.y = (valid && j0 + 1 < n) ? __ldg(in + lbase + (long)(j0 + 1) * a.s) : 0.f;
                    v.z = (valid && j0 + 2 < n) ? __ldg(in + lbase + (long)(j0 + 2) * a.s) : 0.f;
                    v.w = (valid && j0 + 3 < n) ? __ldg(in + lbase + (long)(j0 + 3) * a.s) : 0.f;
                    r.v[q] = v;
                }
            }
        };
        auto issue_b = [&](int kc) {
            if (kc < nkc) {
                const unsigned char *srcb =
                    reinterpret_cast<const unsigned char *>(a.B1) + (size_t)kc * 2 * bplaneB;
                unsigned char *Bp = Bs + (kc % 3) * PLANES * bplaneB;
                const int nv = PLANES * (int)bplaneB / 16;
                for (int qv = tid; qv < nv; qv += 128)
                    umma::cp_async16(Bp + 16 * qv, srcb + 16 * qv);
            }
            umma::cp_async_commit();  // possibly empty: one group per chunk
        };
        // one chunk: false once this warp has to stop (a wait gave up, or another warp did)
        auto step = [&](int kc, AChunk &cur) -> bool {
            // stage kc & 1 and slot (kc + 1) % 3 were last read by the MMAs of chunk kc - 2
            if (kc >= 2) {
                const bool ok = umma::mbar_wait(&done[(kc - 2) % 3],
                                                (uint32_t)((kc - 2) / 3) & 1u, kWaitLimit);
                if (__any_sync(0xffffffffu, !ok) || *(volatile int *)s_err) {
                    *(volatile int *)s_err = 1;
                    return false;
                }
            }
            issue_b(kc + 1);
            unsigned char *Ap = As + (kc & 1) * PLANES * kAPlaneB;
            if (contig) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int line = (warp + 4 * i) * 8 + cr;
                    if (BF) store_split_b16<PLANES>(Ap, a_slot_b16(line, cq), cur.v[i]);
                    else store_split<PLANES>(reinterpret_cast<float *>(Ap), a_slot(line, cq),
                                             cur.v[i]);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (BF) store_split_b16<PLANES>(Ap, a_slot_b16(tid, q), cur.v[q]);
                    else store_split<PLANES>(reinterpret_cast<float *>(Ap), a_slot(tid, q),
                                             cur.v[q]);
                }
            }
            load_global(kc + kPre, cur);                          // in flight for kPre chunks
            asm volatile("cp.async.wait_group 1;" ::: "memory");  // my part of B chunk kc landed
            umma::fence_proxy_async_smem();
            umma::mbar_arrive(&full[kc & 1]);
            return true;
        };
        AChunk pre[kPre];  // chunks kc .. kc + kPre - 1 in flight; static indices after unrolling
#pragma unroll
        for (int q = 0; q < kPre; ++q) load_global(q, pre[q]);
        issue_b(0);
        bool go = true;
        for (int kc = 0; kc < nkc && go; kc += kPre) {
#pragma unroll
            for (int q = 0; q < kPre; ++q)
                if (go && kc + q < nkc) go = step(kc + q, pre[q]);
        }
        umma::cp_async_wait_all();
        if (MODE == kEpiSpectralOut) {  // in flight while the last MMAs finish
#pragma unroll
            for (int m = 0; m < 32; ++m)
                dfirst[m] = (valid && m < n) ? __ldg(a.D + (long)m * a.s + t) : 0.0f;
        }
        // the whole accumulation
        if (!*(volatile int *)s_err) {
            const bool ok = umma::mbar_wait(&done[(nkc - 1) % 3],
                                            (uint32_t)((nkc - 1) / 3) & 1u, kWaitLimit);
            if (__any_sync(0xffffffffu, !ok)) *(volatile int *)s_err = 1;
        }
    }
    __syncthreads();
    umma::fence_after_sync();

    double part_cost = 0.0, part_raw = 0.0;
    const bool want_raw = MODE == kEpiSpectralOut && a.want_raw && (st->sweep % a.every == 0);
    const double gamma = MODE == kEpiSpectralOut ? st->gamma[cn] : 0.0;
    const float gs2 = (float)(gamma * a.sigma2);
    if (producer && !*s_err) {
        // ---- epilogue: 32 TMEM columns at a time -------------------------------------------
        const int nchunks = (n + 31) / 32;
        // the prior scaling runs per line (its unit-stride case, a one-row image, included)
        if (contig && MODE != kEpiSpectralOut) {
            float *stg = reinterpret_cast<float *>(smem_raw) + warp * 32 * 33;
            float rowc = 0.0f;
            if (MODE == kEpiPositions && !a.xpos) {
                const int gi = (int)(l0 + warp * 32 + lane);  // 3D: x * ny + y; 2D: x
                rowc = a.dims == 2 ? (float)gi
                                   : (cn == 0 ? (float)(gi / a.ny) : (float)(gi % a.ny));
            }
            for (int cc = 0; cc < nchunks; ++cc) {
                float v[32];
                umma::tmem_ld32(tmem + tlane + (uint32_t)(cc * 32), v);
#pragma unroll
                for (int m = 0; m < 32; ++m) stg[lane * 33 + m] = v[m];
                __syncwarp();
                const int k = cc * 32 + lane;
#pragma unroll 4
                for (int r = 0; r < 32; ++r) {
                    const long g = l0 + warp * 32 + r;
                    const float rc = __shfl_sync(0xffffffffu, rowc, r);
                    if (g < nlines && k < n) {
                        float val = stg[r * 33 + lane];
                        if (MODE == kEpiPositions)
                            val += a.xpos ? __ldg(a.xpos + cn * a.V + g * n + k)
                                          : (cn == a.dims - 1 ? (float)k : rc);
                        out[g * n + k] = val;
                    }
                }
                __syncwarp();
            }
        } else {
            float dnext[32];
            auto load_dchunk = [&](int cc) {
#pragma unroll
                for (int m = 0; m < 32; ++m) {
                    const int k = cc * 32 + m;
                    dnext[m] = (valid && k < n) ? __ldg(a.D + (long)k * a.s + t) : 0.0f;
                }
            };
            if (MODE == kEpiSpectralOut)
#pragma unroll
                for (int m = 0; m < 32; ++m) dnext[m] = dfirst[m];
            for (int cc = 0; cc < nchunks; ++cc) {
                float v[32], dcur[32], nz[32];
                // the chunk's prior noise, all 32 loads in flight before the first is used (read
                // one element at a time between the stores, each waited a full memory latency)
                if (MODE == kEpiSpectralOut && a.sample) {
#pragma unroll
                    for (int m = 0; m < 32; ++m) {
                        const int k = cc * 32 + m;
                        nz[m] = (valid && k < n)
                                    ? __ldg(a.noise + comp * a.V + (long)k * a.s + t)
                                    : 0.0f;
                    }
                }
                umma::tmem_ld32(tmem + tlane + (uint32_t)(cc * 32), v);
                if (MODE == kEpiSpectralOut) {
#pragma unroll
                    for (int m = 0; m < 32; ++m) dcur[m] = dnext[m];
                    if (cc + 1 < nchunks) load_dchunk(cc + 1);
                }
                if (!valid) continue;
                float ccost = 0.0f;
                float *op = out + lbase;
#pragma unroll
                for (int m = 0; m < 32; ++m) {
                    const int k = cc * 32 + m;
                    if (k < n) {
                        float val = v[m];
                        if (MODE == kEpiSpectralOut) {
                            const float Dv = dcur[m];
                            const float f = __fdividef(1.0f, fmaf(gs2, Dv, 1.0f));
                            val *= f;
                            if (a.sample) val += sqrtf((float)a.sigma2 * f) * nz[m];
                            ccost += Dv * val * val;
                        }
                        op[(long)k * a.s] = val;
                    }
                }
                if (MODE == kEpiSpectralOut) {
                    part_cost += 0.5 * gamma * (double)ccost;
                    if (want_raw) part_raw += a.eta2[cn] * a.rho_p * (double)ccost;
                }
            }
        }
    }
    if (MODE == kEpiSpectralOut) {
        const double sc = block_sum(part_cost, red);
        if (tid == 0) atomicAdd(&st->lp_tr, sc);
        if (a.want_raw) {
            const double sr = block_sum(part_raw, red);
            if (tid == 0) atomicAdd(&st->raw_reg, sr);
        }
    }

    // ---- teardown: after an error, let every tcgen05 op still in flight finish (bounded) ----
    if (*s_err && tid == 128) {
        umma::commit(drain);  // arrives once all MMAs this thread issued have completed
        umma::mbar_wait(drain, 0, kWaitLimit);
        if (st) atomicOr(&st->flags, (unsigned)kFlagTensorTimeout);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, ncols);
}

template <int MODE, int PLANES, bool BF>
void launch_ws(const UArgs &a, int ncomp, cudaStream_t s) {
    // A stages, B slots, then 6 mbarriers, the TMEM address and the error word
    size_t need = (size_t)(2 * PLANES * kAPlane + 3 * PLANES * a.Npad * kKC) * (BF ? 2 : 4) + 64;
    const size_t staging = (size_t)4 * 32 * 33 * sizeof(float) + 64;  // contiguous-axis epilogue
    if (need < staging) need = staging;
    uint32_t ncols = 32;
    while (ncols < (uint32_t)a.Npad) ncols <<= 1;
    // never more CTAs per SM than its 512 TMEM columns hold at once (a surplus CTA would only
    // wait inside tcgen05.alloc): pad the shared-memory request accordingly
    const size_t per_sm = 228 * 1024;
    const size_t max_ctas = 512 / ncols;
    const size_t floor_smem = per_sm / (max_ctas + 1) + 1024;
    const size_t smem = need > floor_smem ? need : floor_smem;
    BINDER_CHECK(smem <= 227 * 1024, "tensor-core transform tile does not fit in shared memory");
    BINDER_CUDA(cudaFuncSetAttribute(umma_ws_kernel<MODE, PLANES, BF>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BINDER_CUDA(cudaFuncSetAttribute(umma_ws_kernel<MODE, PLANES, BF>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    const long tiles = (a.outer * a.s + kLines - 1) / kLines;
    BINDER_CHECK(tiles < (1L << 31), "transform grid too large");
    dim3 grid((unsigned)tiles, 1, (unsigned)ncomp);
    count_launch(), umma_ws_kernel<MODE, PLANES, BF><<<grid, kWsThreads, smem, s>>>(a);
    BINDER_CUDA(cudaGetLastError());
}

// ---- persistent pass: 4 producer warps, 1 MMA warp, 4 epilogue warps -------------------------
// One CTA per SM walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... of every component of the
// pass, as one flat sequence of K chunks (chunk g = tile g / nkc, K chunk g % nkc), so the A
// stages and B slots of the warp-specialised pipeline above run on across tile boundaries.  The
// accumulator is double-buffered in TMEM (buffer it & 1 for the CTA's it-th tile): the MMA warp
// commits a finished tile to accf[b]; warps 5-8 drain it (TMEM -> registers -> global, the
// epilogues of umma_ws_kernel) and release it on acce[b] while the next tile accumulates in the
// other buffer.  Every wait is bounded; on expiry the CTA sets an error flag and winds down.
constexpr int kPtProd = 256;                  // producer threads (warps 0-7)
constexpr int kPtMma = kPtProd;               // the MMA thread (warp 8, lane 0)
constexpr int kPtThreads = kPtProd + 32 + 128;  // + MMA warp + 4 epilogue warps
// A stages (kPtStages, a template parameter: 3 where shared memory allows, else 2) bound how far
// the producers run ahead of the MMAs' completion; B is copied kPtDist chunks ahead into
// kPtStages + kPtDist slots
constexpr int kPtDist = 2;
constexpr int kPtRaw = 4;                 // raw FP32 A slots (A copied kPtRaw - 1 chunks ahead)
constexpr int kRawContig = 20;            // floats per line of a contiguous-axis raw slot (padded)
constexpr int kRawSlot = kLines * kRawContig;  // floats per raw slot (either layout fits)

// cp.async of `bytes` (4 or 16) with zero fill: src_bytes of them read from global memory
__device__ __forceinline__ void cp_async_zfill(float *dst, const float *src, int bytes,
                                               int src_bytes) {
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(umma::smem_u32(dst)),
                     "l"(src), "r"(src_bytes)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(umma::smem_u32(dst)),
                     "l"(src), "r"(src_bytes)
                     : "memory");
}

// barrier 1 over the kPtProd producer threads, OR of `pred` returned to all of them
__device__ __forceinline__ bool producers_sync_or(bool pred) {
    uint32_t r;
    __syncwarp();
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, 256, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void producers_sync() {
    __syncwarp();
    asm volatile("bar.sync 1, 256;" ::: "memory");
}

template <int MODE, int PLANES, int kPtStages>
__global__ void __launch_bounds__(kPtThreads, 1) umma_pt_kernel(const UArgs a) {
    constexpr int kPtSlots = kPtStages + kPtDist;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Npad = a.Npad, n = a.n, nkc = a.nkc;
    const uint32_t bplane = (uint32_t)Npad * kKC;
    float *As = reinterpret_cast<float *>(smem_raw);  // [kPtStages][PLANES][kAPlane]
    float *Bs = As + kPtStages * PLANES * kAPlane;    // [kPtSlots][PLANES][bplane]
    float *raw = Bs + kPtSlots * PLANES * bplane;     // [kPtRaw][kRawSlot] raw A chunks
    float *stg0 = raw + kPtRaw * kRawSlot;            // [4 warps][32][33] epilogue staging
    uint64_t *full = reinterpret_cast<uint64_t *>(stg0 + 4 * 32 * 33);  // [kPtStages]
    uint64_t *done = full + kPtStages;                                  // [kPtSlots]
    uint64_t *accf = done + kPtSlots;                                   // [2]
    uint64_t *acce = accf + 2;                                          // [2]
    uint64_t *drain = acce + 2;                                         // [1]
    uint32_t *holder = reinterpret_cast<uint32_t *>(drain + 1);
    int *s_err = reinterpret_cast<int *>(holder + 1);
    __shared__ double red[32];

    uint32_t acols = 32;  // columns of one accumulator
    while (acols < (uint32_t)Npad) acols <<= 1;
    const uint32_t ncols = 2 * acols;
    if (warp == 0) umma::tmem_alloc(holder, ncols);
    if (tid == 32) {
        for (int i = 0; i < kPtStages; ++i) umma::mbar_init(&full[i], kPtProd);
        for (int i = 0; i < kPtSlots; ++i) umma::mbar_init(&done[i], 1);
        umma::mbar_init(&accf[0], 1);
        umma::mbar_init(&accf[1], 1);
        umma::mbar_init(&acce[0], 128);
        umma::mbar_init(&acce[1], 128);
        umma::mbar_init(drain, 1);
        *s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *holder;

    const long nlines = a.outer * a.s;
    const long tiles = (nlines + kLines - 1) / kLines;  // per component
    const long total = tiles * a.ncomp;
    const long G = gridDim.x;
    const int my_tiles = blockIdx.x < total ? (int)((total - 1 - blockIdx.x) / G + 1) : 0;
    const long nchunk = (long)my_tiles * nkc;
    const bool contig = (a.s == 1);

    double part_cost = 0.0, part_raw = 0.0;

    if (warp == kPtProd / 32) {
        // ---- MMA warp ------------------------------------------------------------------------
        if (lane == 0) {
            const uint32_t idesc = umma::instr_desc(kLines, Npad, umma::kFmtTF32);
            long g = 0;
            for (int it = 0; it < my_tiles; ++it) {
                const int b = it & 1;
                if (it >= 2 && (!umma::mbar_wait(&acce[b], (uint32_t)((it - 2) >> 1) & 1u,
                                                 kWaitLimit) ||
                                *(volatile int *)s_err)) {
                    *(volatile int *)s_err = 1;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t tacc = tmem + (uint32_t)b * acols;
                bool ok = true;
                for (int kc = 0; kc < nkc; ++kc, ++g) {
                    if (!umma::mbar_wait_spin(&full[g % kPtStages],
                                              (uint32_t)(g / kPtStages) & 1u, kWaitLimit) ||
                        *(volatile int *)s_err) {
                        ok = false;
                        break;
                    }
                    umma::fence_after_sync();
                    const uint32_t abase =
                        umma::smem_u32(As + (g % kPtStages) * PLANES * kAPlane);
                    const uint32_t bbase = umma::smem_u32(Bs + (g % kPtSlots) * PLANES * bplane);
#pragma unroll
                    for (int ks = 0; ks < kKC / 8; ++ks) {
                        const uint32_t ao = (uint32_t)ks * 2u * 2048u;
                        const uint32_t bo = (uint32_t)ks * 2u * (uint32_t)Npad * 16u;
                        const uint64_t ahi = umma::smem_desc(abase + ao, 2048u, 128u);
                        const uint64_t bhi =
                            umma::smem_desc(bbase + bo, (uint32_t)Npad * 16u, 128u);
                        umma::mma_tf32(tacc, ahi, bhi, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
                        if (PLANES == 2) {
                            const uint64_t alo =
                                umma::smem_desc(abase + kAPlane * 4u + ao, 2048u, 128u);
                            const uint64_t blo = umma::smem_desc(bbase + bplane * 4u + bo,
                                                                 (uint32_t)Npad * 16u, 128u);
                            umma::mma_tf32(tacc, ahi, blo, idesc, 1u);
                            umma::mma_tf32(tacc, alo, bhi, idesc, 1u);
                        }
                    }
                    umma::commit(&done[g % kPtSlots]);
                }
                if (!ok) {
                    *(volatile int *)s_err = 1;
                    break;
                }
                umma::commit(&accf[b]);  // arrives when this tile's MMAs have completed
            }
        }
    } else if (warp < kPtProd / 32) {
        // ---- producers -----------------------------------------------------------------------
        // A chunks are copied raw (FP32) into a kPtRaw-slot ring by cp.async, kPtRaw - 1 chunks
        // ahead, then split into TF32 planes from shared memory (thread tid <-> row tid & 127,
        // K slots 2 (tid >> 7) and 2 (tid >> 7) + 1).  Layouts:
        //   strided axis:    raw[j][line] (16 x 128); 16-byte copies of 4 neighbouring lines when
        //                    s % 4 == 0 (the 4 lines then share o and start 16-byte aligned),
        //                    4-byte copies of the thread's row and K half otherwise;
        //   contiguous axis: raw[line][kRawContig]; 16-byte copies of 4 elements of a line when
        //                    n % 4 == 0 (every line then starts 16-byte aligned), else 4-byte.
        // Out-of-range lines and elements are zero-filled (source bytes 0).
        const bool wide = contig ? (n & 3) == 0 : (a.s & 3) == 0;
        const int row = tid & (kLines - 1), half = tid >> 7;
        // the A chunks are copied in order: a cursor over (tile, K chunk) instead of divisions
        long cg = 0;        // next chunk to copy
        int ckc = 0;        // its K chunk
        long ctau = blockIdx.x;
        const float *cin = nullptr;
        long cl0 = 0;
        const float *lbase[2];  // this thread's line (group) bases, per tile
        bool lval[2];
        auto set_tile = [&]() {
            const long cm = ctau / tiles;
            cin = a.in + (a.comp0 + cm) * a.V;
            cl0 = (ctau - cm * tiles) * kLines;
            if (contig) {
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const long gl = cl0 + (wide ? (tid >> 2) + 64 * i : row);
                    lval[i] = gl < nlines;
                    lbase[i] = lval[i] ? cin + gl * n : cin;
                }
            } else {
                const long lg = cl0 + (wide ? 4 * lane : row);
                const bool v = lg < nlines;
                const long o = v ? lg / a.s : 0, t = v ? lg - o * a.s : 0;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    lval[i] = v;
                    lbase[i] = cin + o * (long)n * a.s + t;
                }
            }
        };
        set_tile();
        // raw copy of chunk cg into its slot, cursor advanced (no copy past the last chunk)
        auto copy_next = [&]() {
            if (cg >= nchunk) return;
            float *rs = raw + (cg % kPtRaw) * kRawSlot;
            const int jb = ckc * kKC;
            if (contig) {
                if (wide) {
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const int line = (tid >> 2) + 64 * i, qd = tid & 3;
                        const int j0 = jb + 4 * qd;
                        const bool ok = lval[i] && j0 < n;
                        cp_async_zfill(rs + line * kRawContig + 4 * qd,
                                       ok ? lbase[i] + j0 : cin, 16, ok ? 16 : 0);
                    }
                } else {
#pragma unroll
                    for (int jh = 0; jh < kKC / 2; ++jh) {
                        const int jj = 8 * half + jh;
                        const bool ok = lval[0] && jb + jj < n;
                        cp_async_zfill(rs + row * kRawContig + jj, ok ? lbase[0] + jb + jj : cin,
                                       4, ok ? 4 : 0);
                    }
                }
            } else {
                if (wide) {
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const int jj = warp + 8 * i;
                        const bool ok = lval[0] && jb + jj < n;
                        cp_async_zfill(rs + jj * kLines + 4 * lane,
                                       ok ? lbase[0] + (long)(jb + jj) * a.s : cin, 16,
                                       ok ? 16 : 0);
                    }
                } else {
#pragma unroll
                    for (int jh = 0; jh < kKC / 2; ++jh) {
                        const int jj = 8 * half + jh;
                        const bool ok = lval[0] && jb + jj < n;
                        cp_async_zfill(rs + jj * kLines + row,
                                       ok ? lbase[0] + (long)(jb + jj) * a.s : cin, 4,
                                       ok ? 4 : 0);
                    }
                }
            }
            ++cg;
            if (++ckc == nkc) {
                ckc = 0;
                ctau += G;
                if (cg < nchunk) set_tile();
            }
        };
        int kb = 0;   // matrix chunk of the next B copy
        long gb = 0;  // chunk of the next B copy
        auto issue_b = [&]() {
            if (gb < nchunk) {
                const float *srcb = a.B1 + (size_t)kb * 2 * bplane;
                float *Bp = Bs + (gb % kPtSlots) * PLANES * bplane;
                const int nv = PLANES * (int)bplane / 4;
                for (int qv = tid; qv < nv; qv += kPtProd)
                    umma::cp_async16(Bp + 4 * qv, srcb + 4 * qv);
            }
            ++gb;
            if (++kb == nkc) kb = 0;
        };
        // prologue: groups 0 .. kPtRaw - 2 hold raw chunks 0 .. kPtRaw - 2 and B chunks
        // 0 .. kPtDist - 1; step g adds one group with raw chunk g + kPtRaw - 1 and B chunk
        // g + kPtDist, so raw(g) and B(g) are complete once at most 2 groups are pending
        static_assert(kPtRaw - 1 >= kPtDist && kPtRaw >= 3, "group accounting");
        for (int q = 0; q < kPtRaw - 1; ++q) {
            copy_next();
            if (q < kPtDist) issue_b();
            umma::cp_async_commit();
        }
        for (long g = 0; g < nchunk; ++g) {
            // A stage g % kPtStages and B slot (g + kPtDist) % kPtSlots were last read by the
            // MMAs of chunk g - kPtStages; the raw slot of chunk g + kPtRaw - 1 by the split of
            // chunk g - 1.  One stop decision for all producers.
            bool stop = *(volatile int *)s_err != 0;
            if (g >= kPtStages) {
                const long gp = g - kPtStages;
                stop |= !umma::mbar_wait_spin(&done[gp % kPtSlots],
                                              (uint32_t)(gp / kPtSlots) & 1u, kWaitLimit);
            }
            if (producers_sync_or(stop)) {
                *(volatile int *)s_err = 1;
                break;
            }
            copy_next();
            issue_b();
            umma::cp_async_commit();
            asm volatile("cp.async.wait_group 2;" ::: "memory");
            producers_sync();  // every producer's copies of raw chunk g have landed
            const float *rs = raw + (g % kPtRaw) * kRawSlot;
            float *Ap = As + (g % kPtStages) * PLANES * kAPlane;
#pragma unroll
            for (int qh = 0; qh < 2; ++qh) {
                const int q = 2 * half + qh;
                float4 v;
                if (contig) {
                    v = *reinterpret_cast<const float4 *>(rs + row * kRawContig + 4 * q);
                } else {
                    v.x = rs[(4 * q + 0) * kLines + row];
                    v.y = rs[(4 * q + 1) * kLines + row];
                    v.z = rs[(4 * q + 2) * kLines + row];
                    v.w = rs[(4 * q + 3) * kLines + row];
                }
                store_split<PLANES>(Ap, a_slot(row, q), v);
            }
            umma::fence_proxy_async_smem();  // this thread's part of B chunk g and A stage
            umma::mbar_arrive(&full[g % kPtStages]);
        }
        umma::cp_async_wait_all();
    } else {
        // ---- epilogue warps 5-8: TMEM lane quarter ew = warp % 4 -----------------------------
        const int ew = warp & 3;
        const uint32_t tlane = (uint32_t)(ew * 32) << 16;
        const int row = ew * 32 + lane;  // this thread's row of the tile
        float *stg = stg0 + ew * 32 * 33;
        const uint32_t sweep = (MODE == kEpiSpectralOut && a.sample) ? (uint32_t)a.st->sweep : 0u;
        const bool want_raw =
            MODE == kEpiSpectralOut && a.want_raw && (a.st->sweep % a.every == 0);
        const int nchunks = (n + 31) / 32;
        for (int it = 0; it < my_tiles; ++it) {
            const int b = it & 1;
            const bool ok = umma::mbar_wait(&accf[b], (uint32_t)(it >> 1) & 1u, kWaitLimit);
            if (__any_sync(0xffffffffu, !ok || *(volatile int *)s_err)) {
                *(volatile int *)s_err = 1;
                break;
            }
            umma::fence_after_sync();
            const uint32_t tacc = tmem + tlane + (uint32_t)b * acols;
            const long tau = blockIdx.x + (long)it * G;
            const long cm = tau / tiles;
            const int comp = a.comp0 + (int)cm;
            float *out = a.out + comp * a.V;
            const long l0 = (tau - cm * tiles) * kLines;
            if (contig && MODE != kEpiSpectralOut) {
                float rowc = 0.0f;
                if (MODE == kEpiPositions && !a.xpos) {
                    const int gi = (int)(l0 + ew * 32 + lane);  // 3D: x * ny + y; 2D: x
                    rowc = a.dims == 2 ? (float)gi
                                       : (comp == 0 ? (float)(gi / a.ny) : (float)(gi % a.ny));
                }
                for (int cc = 0; cc < nchunks; ++cc) {
                    float v[32];
                    umma::tmem_ld32(tacc + (uint32_t)(cc * 32), v);
#pragma unroll
                    for (int m = 0; m < 32; ++m) stg[lane * 33 + m] = v[m];
                    __syncwarp();
                    const int k = cc * 32 + lane;
#pragma unroll 4
                    for (int r = 0; r < 32; ++r) {
                        const long gl = l0 + ew * 32 + r;
                        const float rc = __shfl_sync(0xffffffffu, rowc, r);
                        if (gl < nlines && k < n) {
                            float val = stg[r * 33 + lane];
                            if (MODE == kEpiPositions)
                                val += a.xpos ? __ldg(a.xpos + comp * a.V + gl * n + k)
                                              : (comp == a.dims - 1 ? (float)k : rc);
                            out[gl * n + k] = val;
                        }
                    }
                    __syncwarp();
                }
            } else {
                const long lg = l0 + row;
                const bool valid = lg < nlines;
                const long o = valid ? lg / a.s : 0, t = valid ? lg - o * a.s : 0;
                float *op = out + o * (long)n * a.s + t;
                const double gamma = MODE == kEpiSpectralOut ? a.st->gamma[comp] : 0.0;
                const float gs2 = (float)(gamma * a.sigma2);
                float ccost = 0.0f;
                for (int cc = 0; cc < nchunks; ++cc) {
                    float v[32];
                    umma::tmem_ld32(tacc + (uint32_t)(cc * 32), v);
                    if (!valid) continue;
#pragma unroll
                    for (int m = 0; m < 32; ++m) {
                        const int k = cc * 32 + m;
                        if (k < n) {
                            float val = v[m];
                            if (MODE == kEpiSpectralOut) {
                                const float Dv = __ldg(a.D + (long)k * a.s + t);
                                const float f = __fdividef(1.0f, fmaf(gs2, Dv, 1.0f));
                                val *= f;
                                if (a.sample)
                                    val += sqrtf((float)a.sigma2 * f) *
                                           prior_normal_tc(a.seed, (uint32_t)((long)k * a.s + t),
                                                           sweep, a.chain, comp);
                                ccost += Dv * val * val;
                            }
                            op[(long)k * a.s] = val;
                        }
                    }
                }
                if (MODE == kEpiSpectralOut) {
                    part_cost += 0.5 * gamma * (double)ccost;
                    if (want_raw) part_raw += a.eta2[comp] * a.rho_p * (double)ccost;
                }
            }
            // this tile's TMEM reads are complete (tcgen05.wait::ld): release the buffer
            umma::fence_before_sync();
            umma::mbar_arrive(&acce[b]);
        }
    }

    if (MODE == kEpiSpectralOut) {
        const double sc = block_sum(part_cost, red);
        if (tid == 0) atomicAdd(&a.st->lp_tr, sc);
        if (a.want_raw) {
            const double sr = block_sum(part_raw, red);
            if (tid == 0) atomicAdd(&a.st->raw_reg, sr);
        }
    }
    // ---- teardown: after an error, let every tcgen05 op still in flight finish (bounded) ----
    __syncthreads();
    if (*s_err && tid == kPtMma) {
        umma::commit(drain);
        umma::mbar_wait(drain, 0, kWaitLimit);
        if (a.st) atomicOr(&a.st->flags, (unsigned)kFlagTensorTimeout);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, ncols);
}

template <int MODE, int PLANES, int S>
size_t pt_smem(int Npad) {
    return (size_t)(S * PLANES * kAPlane + (S + kPtDist) * PLANES * Npad * kKC +
                    kPtRaw * kRawSlot + 4 * 32 * 33) * sizeof(float) + 256;
}

template <int MODE, int PLANES, int S>
void launch_pt_s(const UArgs &a, size_t need, cudaStream_t s) {
    uint32_t acols = 32;
    while (acols < (uint32_t)a.Npad) acols <<= 1;
    // never more CTAs per SM than its 512 TMEM columns hold at once (a surplus CTA would only
    // wait inside tcgen05.alloc): pad the shared-memory request accordingly
    const size_t per_sm = 228 * 1024;
    const size_t max_ctas = 512 / (2 * acols);
    const size_t floor_smem = per_sm / (max_ctas + 1) + 1024;
    const size_t smem = need > floor_smem ? need : floor_smem;
    BINDER_CHECK(smem <= 227 * 1024, "tensor-core transform tile does not fit in shared memory");
    BINDER_CUDA(cudaFuncSetAttribute(umma_pt_kernel<MODE, PLANES, S>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BINDER_CUDA(cudaFuncSetAttribute(umma_pt_kernel<MODE, PLANES, S>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    int dev = 0, sms = 148;
    BINDER_CUDA(cudaGetDevice(&dev));
    BINDER_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long tiles = (a.outer * a.s + kLines - 1) / kLines * a.ncomp;
    const long grid = tiles < (long)sms * (long)max_ctas ? tiles : (long)sms * (long)max_ctas;
    count_launch(), umma_pt_kernel<MODE, PLANES, S><<<(unsigned)grid, kPtThreads, smem, s>>>(a);
    BINDER_CUDA(cudaGetLastError());
}

template <int MODE, int PLANES>
void launch_pt(const UArgs &a, cudaStream_t s) {
    const size_t n3 = pt_smem<MODE, PLANES, 3>(a.Npad);
    if (n3 <= 227 * 1024) launch_pt_s<MODE, PLANES, 3>(a, n3, s);
    else launch_pt_s<MODE, PLANES, 2>(a, pt_smem<MODE, PLANES, 2>(a.Npad), s);
}

float tf32_rna_host(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) {
        u += 0x1000u;
        u &= 0xFFFFE000u;
    }
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// FP32 -> BF16 bits, round to nearest even (NaN kept a quiet NaN); host side of the B planes
uint16_t bf16_rne_host(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

float bf16_to_float_host(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

template <int MODE, int PLANES>
void launch_umma(const UArgs &a, int ncomp, cudaStream_t s) {
    size_t need = (size_t)(2 * PLANES * kAPlane + 3 * PLANES * a.Npad * kKC) * sizeof(float) + 64;
    const size_t staging = (size_t)4 * 32 * 33 * sizeof(float) + 64;  // contiguous-axis epilogue
    if (need < staging) need = staging;
    const uint32_t want = MODE == kEpiSpectral ? 2u * a.Npad : (uint32_t)a.Npad;
    uint32_t ncols = 32;
    while (ncols < want) ncols <<= 1;
    // never let more CTAs share an SM than its 512 TMEM columns can hold at once (a surplus CTA
    // would only wait inside tcgen05.alloc): pad the shared-memory request accordingly
    const size_t per_sm = 228 * 1024;
    const size_t max_ctas = 512 / ncols;
    const size_t floor_smem = per_sm / (max_ctas + 1) + 1024;
    const size_t smem = need > floor_smem ? need : floor_smem;
    BINDER_CHECK(smem <= 227 * 1024, "tensor-core transform tile does not fit in shared memory");
    BINDER_CUDA(cudaFuncSetAttribute(umma_axis_kernel<MODE, PLANES>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // the whole unified L1 / shared array as shared memory: with the default carveout the
    // driver may configure too little for two of these CTAs, halving the SM's occupancy
    BINDER_CUDA(cudaFuncSetAttribute(umma_axis_kernel<MODE, PLANES>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    const long tiles = (a.outer * a.s + kLines - 1) / kLines;
    BINDER_CHECK(tiles < (1L << 31), "transform grid too large");
    dim3 grid((unsigned)tiles, 1, (unsigned)ncomp);
    count_launch(), umma_axis_kernel<MODE, PLANES><<<grid, 128, smem, s>>>(a);
    BINDER_CUDA(cudaGetLastError());
}

}  // namespace

// ------------------------------------------------------------------------------------------
void UmmaMatrix::init(const double *M, int n_, cudaStream_t s) {
    n = n_;
    Npad = ((n + 15) / 16) * 16;
    nkc = (n + kKC - 1) / kKC;
    const size_t plane = (size_t)Npad * kKC;
    std::vector<float> host((size_t)nkc * 2 * plane, 0.0f);
    for (int kc = 0; kc < nkc; ++kc)
        for (int k = 0; k < n; ++k)
            for (int jj = 0; jj < kKC; ++jj) {
                const int j = kc * kKC + jj;
                if (j >= n) continue;
                const float v = (float)M[(size_t)k * n + j];
                const float hi = tf32_rna_host(v);
                const float lo = tf32_rna_host(v - hi);
                const size_t off = (size_t)(jj / 4) * (Npad * 4) + (k / 8) * 32 + (k % 8) * 4 + (jj % 4);
                host[(size_t)kc * 2 * plane + off] = hi;
                host[(size_t)kc * 2 * plane + plane + off] = lo;
            }
    // the same chunks as BF16 hi / lo planes (2-byte elements, the same canonical layout: 16-byte
    // K columns of 8 elements Npad * 16 bytes apart, 8-row groups 128 bytes apart)
    std::vector<uint16_t> host16((size_t)nkc * 2 * plane, 0);
    for (int kc = 0; kc < nkc; ++kc)
        for (int k = 0; k < n; ++k)
            for (int jj = 0; jj < kKC; ++jj) {
                const int j = kc * kKC + jj;
                if (j >= n) continue;
                const float v = (float)M[(size_t)k * n + j];
                const uint16_t hi = bf16_rne_host(v);
                const uint16_t lo = bf16_rne_host(v - bf16_to_float_host(hi));
                const size_t off = (size_t)(jj / 8) * (Npad * 8) + (k / 8) * 64 + (k % 8) * 8 + (jj % 8);
                host16[(size_t)kc * 2 * plane + off] = hi;
                host16[(size_t)kc * 2 * plane + plane + off] = lo;
            }
    dev = dev_alloc_n<float>(host.size(), s);
    dev16 = dev_alloc_n<uint16_t>(host16.size(), s);
    BINDER_CUDA(cudaMemcpyAsync(dev, host.data(), host.size() * sizeof(float),
                                cudaMemcpyHostToDevice, s));
    BINDER_CUDA(cudaMemcpyAsync(dev16, host16.data(), host16.size() * sizeof(uint16_t),
                                cudaMemcpyHostToDevice, s));
    BINDER_CUDA(cudaStreamSynchronize(s));  // `host` goes out of scope
}

void UmmaMatrix::release(cudaStream_t s) {
    dev_free_p(dev, s);
    dev_free_p(dev16, s);
}

void launch_axis_pass_tc(const AxisArgs<float> &b, const UmmaMatrix &M1, const UmmaMatrix *M2,
                         int mode, int ncomp, int planes, cudaStream_t s, bool persistent,
                         bool bf16) {
    BINDER_CHECK(b.n == M1.n, "matrix / axis length mismatch");
    BINDER_CHECK(planes == 1 || planes == 2, "planes must be 1 (one product) or 2 (split)");
    BINDER_CHECK(!bf16 || !persistent, "BF16 operands run on the per-tile passes");
    UArgs a{};
    a.in = b.in; a.out = b.out; a.V = b.comp_stride; a.n = b.n; a.Npad = M1.Npad; a.nkc = M1.nkc;
    a.outer = b.outer; a.s = b.s;
    a.B1 = bf16 ? reinterpret_cast<const float *>(M1.dev16) : M1.dev;
    a.B2 = M2 ? M2->dev : nullptr;
    a.D = b.D; a.st = b.st; a.sigma2 = b.sigma2; a.sample = b.sample; a.want_raw = b.want_raw;
    a.noise = b.noise;
    a.every = b.every < 1 ? 1 : b.every; a.seed = b.seed; a.chain = b.chain; a.rho_p = b.rho_p;
    for (int i = 0; i < 3; ++i) a.eta2[i] = b.eta2[i];
    a.xpos = b.xpos; a.ny = b.ny; a.nz = b.nz; a.dims = b.dims; a.comp0 = b.comp0; a.skip = b.skip;
    a.ncomp = ncomp;
    a.chain_comps = b.chain_comps;
    // a persistent CTA's tiles span components, so its per-CTA cost sums could mix chains
    BINDER_CHECK(!persistent || b.chain_comps == 0,
                 "a batch of chains runs on the per-tile tensor-core passes");
    if (persistent && mode != kEpiSpectral) {
        BINDER_CHECK(mode != kEpiSpectralOut || b.outer == 1,
                     "prior scaling runs on the outermost axis");
        switch (mode) {
            case kEpiNone:
                if (planes == 2) launch_pt<kEpiNone, 2>(a, s);
                else launch_pt<kEpiNone, 1>(a, s);
                break;
            case kEpiPositions:
                if (planes == 2) launch_pt<kEpiPositions, 2>(a, s);
                else launch_pt<kEpiPositions, 1>(a, s);
                break;
            case kEpiSpectralOut:
                if (planes == 2) launch_pt<kEpiSpectralOut, 2>(a, s);
                else launch_pt<kEpiSpectralOut, 1>(a, s);
                break;
            default: BINDER_CHECK(false, "unsupported epilogue on the tensor-core path");
        }
        return;
    }
#define BINDER_UMMA_CASE(MODE)                                                    \
    case MODE:                                                                    \
        if (bf16) {                                                               \
            if (planes == 2) launch_ws<MODE, 2, true>(a, ncomp, s);               \
            else launch_ws<MODE, 1, true>(a, ncomp, s);                           \
        } else {                                                                  \
            if (planes == 2) launch_ws<MODE, 2, false>(a, ncomp, s);              \
            else launch_ws<MODE, 1, false>(a, ncomp, s);                          \
        }                                                                         \
        break;
    switch (mode) {
        BINDER_UMMA_CASE(kEpiNone)
        BINDER_UMMA_CASE(kEpiPositions)
        case kEpiSpectralOut:
            BINDER_CHECK(b.outer == 1, "prior scaling runs on the outermost axis");
            if (bf16) {
                if (planes == 2) launch_ws<kEpiSpectralOut, 2, true>(a, ncomp, s);
                else launch_ws<kEpiSpectralOut, 1, true>(a, ncomp, s);
            } else {
                if (planes == 2) launch_ws<kEpiSpectralOut, 2, false>(a, ncomp, s);
                else launch_ws<kEpiSpectralOut, 1, false>(a, ncomp, s);
            }
            break;
        case kEpiSpectral:
            BINDER_CHECK(!bf16, "the fused prior pass runs with TF32 operands");
            BINDER_CHECK(M2 && M2->n == b.n, "fused pass needs the inverse matrix");
            BINDER_CHECK(b.outer == 1, "fused prior pass runs on the outermost axis");
            if (planes == 2) launch_umma<kEpiSpectral, 2>(a, ncomp, s);
            else launch_umma<kEpiSpectral, 1>(a, ncomp, s);
            break;
        default: BINDER_CHECK(false, "unsupported epilogue on the tensor-core path");
    }
#undef BINDER_UMMA_CASE
}

}  // namespace binder
