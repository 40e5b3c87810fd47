// Shared device/host helpers for the binder_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace binder {

// ------------------------------------------------------------------------------------------
// errors: every CUDA call is checked; failures become std::runtime_error, which the C-ABI layer
// turns into a non-zero status plus binder_last_error() text.
// ------------------------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

enum Status : int {
    kOk = 0,
    kInvalidArgument = 1,
    kCudaError = 2,
    kUnsupported = 3,
    kNotReady = 4,
    kDeviceFault = 5,  // a bounded device-side loop gave up (see device status word)
};

#define BINDER_CUDA(call)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::binder::Error(::binder::kCudaError, std::string(#call) + ": " +            \
                                                           cudaGetErrorString(e_));            \
    } while (0)

#define BINDER_CHECK(cond, msg)                                                                \
    do {                                                                                       \
        if (!(cond)) throw ::binder::Error(::binder::kInvalidArgument, (msg));                  \
    } while (0)

// device status bits (written by kernels, read by the host between launches)
enum DeviceFlag : unsigned {
    kFlagGammaCapped = 1u << 0,    // a Marsaglia-Tsang sampler reached its attempt cap
    kFlagLimiterCapped = 1u << 1,  // a gradient-limiter blend loop reached its step cap
    kFlagNonFinite = 1u << 2,      // a reduction produced a non-finite value
    kFlagTensorTimeout = 1u << 3,  // a tensor-core pass gave up waiting on its MMA barrier
};

// ------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11).  Counter layout used across the library:
//   ctr = {index, sweep, tag | attempt << 8, chain}, key = {seed_lo, seed_hi}
// tags: 1 categorical draw (per voxel), 2/3 prior-sampling normals (per DCT coefficient),
//       4 Dirichlet gammas (per theta entry), 5 the gamma-prior precision nu.
// ------------------------------------------------------------------------------------------
struct u32x4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ u32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                        uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    return {c0, c1, c2, c3};
}

__host__ __device__ __forceinline__ u32x4 philox_draw(uint64_t seed, uint32_t index, uint32_t sweep,
                                                      uint32_t tag, uint32_t chain) {
    return philox4x32_10(index, sweep, tag, chain, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// uniform in (0,1) with 23 random bits; exactly representable in float
__host__ __device__ __forceinline__ float u01_f24(uint32_t x) {
    return ((float)(x >> 9) + 0.5f) * (1.0f / 8388608.0f);
}
// prior-sampling normal for DCT coefficient i of component comp (Box-Muller on Philox tag 2 for
// the x / y components, tag 3 for z; the oracle draws the same stream)
__device__ __forceinline__ float dct_prior_normal(uint64_t seed, uint32_t i, uint32_t sweep,
                                                  uint32_t chain, int comp) {
    const u32x4 r = philox_draw(seed, i, sweep, comp < 2 ? 2u : 3u, chain);
    const float u1 = u01_f24(r.x), u2 = u01_f24(r.y);
    const float rad = sqrtf(-2.0f * logf(u1));
    float sn, cs;
    sincospif(2.0f * u2, &sn, &cs);
    return comp == 1 ? rad * sn : rad * cs;
}

// uniform in (0,1) with 32 random bits in double
__host__ __device__ __forceinline__ double u01_d32(uint32_t x) {
    return ((double)x + 0.5) * (1.0 / 4294967296.0);
}

// ------------------------------------------------------------------------------------------
// reductions
// ------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum, result valid in thread 0; `scratch` holds >= 32 elements
template <typename T>
__device__ __forceinline__ T block_sum(T v, T *scratch) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    T r = T(0);
    if (wid == 0) {
        r = lane < nw ? scratch[lane] : T(0);
        r = warp_sum(r);
    }
    return r;
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// process-wide count of kernels this library has launched (graph replays count every node)
long long &launch_counter();
inline void count_launch(long long n = 1) { launch_counter() += n; }

}  // namespace binder
