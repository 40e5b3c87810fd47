// Tensor-core (tcgen05) separable transform passes -- see umma_transform.cu.
#pragma once

#include "transform.cuh"

namespace binder {

// An n x n transform matrix preformatted for the UMMA B operand: K chunks of 16, each a hi and a
// lo TF32 plane in the canonical no-swizzle K-major layout, rows padded to a multiple of 16 (and
// the same as BF16 hi / lo planes for the BF16 passes).
struct UmmaMatrix {
    int n = 0, Npad = 0, nkc = 0;
    float *dev = nullptr;
    uint16_t *dev16 = nullptr;  // the same chunks as BF16 hi / lo planes (2-byte elements)
    // device copy from the stream-ordered pool on stream s (synchronised before returning)
    void init(const double *M, int n, cudaStream_t s);
    void release(cudaStream_t s);
};

// precision of the DCT passes
enum TransformPrecision : int {
    kPrecFP32Simt = 0,   // FP32 FMA (CUDA cores)
    kPrecTF32x3 = 1,     // tensor cores, 3xTF32 split: FP32-level accuracy
    kPrecTF32 = 2,       // tensor cores, one TF32 product
    kPrecBF16x3 = 3,     // tensor cores, BF16 hi / lo split, three products (~16-bit operands)
    kPrecBF16 = 4,       // tensor cores, one BF16 product
};

// One pass on the tensor cores: modes kEpiNone, kEpiPositions, kEpiSpectral (M2 = inverse).
// persistent: one launch for all ncomp components, one CTA per SM walking the tiles with a
// double-buffered TMEM accumulator (modes kEpiNone, kEpiPositions, kEpiSpectralOut)
void launch_axis_pass_tc(const AxisArgs<float> &a, const UmmaMatrix &M1, const UmmaMatrix *M2,
                         int mode, int ncomp, int planes, cudaStream_t s, bool persistent = false,
                         bool bf16 = false);

}  // namespace binder
