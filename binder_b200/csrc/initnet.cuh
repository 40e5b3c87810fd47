// Learned initialiser of the registration: a 3D convolutional encoder-decoder that predicts a
// coarse displacement field from a moving / fixed image pair, trained and run on hand-written
// sm_100a kernels (BF16 operands on tcgen05 with FP32 accumulation in TMEM, FP32 master weights
// and Adam).  The registration itself has the last word: the prediction only seeds the positions
// the EM starts from (the final_locations argument of Registration).
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace binder {

// C[M][N] (=, or += with atomic adds across K splits) A[M][K] . B[N][K]^T: A and B BF16 row-major
// with K contiguous (leading dimensions multiples of 8 elements), C FP32 row-major.  K is a
// multiple of 64 (the caller pads both operands with zeros); rows past M or N read as zero.
struct GemmArgs {
    const uint16_t *A;
    const uint16_t *B;
    float *C;
    int M, N, K;
    long lda, ldb, ldc;
    int k_split;     // K elements per split (multiple of 64); gridDim.z = ceil(K / k_split)
    int accumulate;  // 1: atomically add into C (C zeroed by the caller); 0: store
    int *err;        // set to 1 when a bounded wait gives up
};
void launch_gemm_bf16(const GemmArgs &g, cudaStream_t s);
// the same on host arrays (row-major, leading dimensions K, K, N), through device copies
void gemm_bf16_host(const uint16_t *A, const uint16_t *B, float *C, int M, int N, int K);

class InitNet {
  public:
    // in_channels: input channels per voxel (2: moving and fixed intensities)
    InitNet(int batch, int size, uint64_t seed, int in_channels = 2);
    ~InitNet();
    // forward pass of `in` (device or host memory, FP32 [B][S^3][in_channels]) into out (FP32
    // [B][(S/4)^3][3], host or device)
    void predict(const float *in, float *out);
    // one Adam step on the mean squared error against `target` ([B][(S/4)^3][3]); returns the
    // loss before the step.  grads_out (optional, host, parameter_count() floats) receives the
    // gradient of that loss, in the parameter order of get_parameters.
    double train_step(const float *in, const float *target, double lr, float *grads_out);
    // the gradient of the loss without a step (for checks)
    double gradients(const float *in, const float *target, float *grads_out);
    long parameter_count() const { return nparam_; }
    void get_parameters(float *out) const;  // FP32 master copy, layer by layer: W [Cout][27 Cin], b [Cout]
    void set_parameters(const float *in);
    int batch() const { return B_; }
    int in_channels() const { return Cin_; }
    int size() const { return S_; }

  private:
    struct Layer;
    struct Impl;
    Impl *impl_;
    int B_, S_, Cin_;
    long nparam_;
    double forward_backward(const float *in, const float *target, bool backward);
};

}  // namespace binder
