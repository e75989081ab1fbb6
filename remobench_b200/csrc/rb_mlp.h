// The learned scorer's parameter layout and device state (see rb_mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace rb {

constexpr int kIn = 16, kHidden = 64, kOut = 2;

// FP32 master parameters: W1 [64][16], b1 [64], W2 [64][64], b2 [64], W3 [2][64], b3 [2].
constexpr int kPW1 = 0;
constexpr int kPB1 = kPW1 + kHidden * kIn;
constexpr int kPW2 = kPB1 + kHidden;
constexpr int kPB2 = kPW2 + kHidden * kHidden;
constexpr int kPW3 = kPB2 + kHidden;
constexpr int kPB3 = kPW3 + kOut * kHidden;
constexpr int kNumParams = kPB3 + kOut;  // 5378

// BF16 copies of the three weight matrices, packed W1 | W2 | W3.
constexpr int kQW1 = 0;
constexpr int kQW2 = kQW1 + kHidden * kIn;
constexpr int kQW3 = kQW2 + kHidden * kHidden;
constexpr int kNumQuant = kQW3 + kOut * kHidden;

// Index of master parameter i in the BF16 copy, or -1 for a bias.
__host__ __device__ inline int quantIndex(int i) {
    if (i >= kPW1 && i < kPB1) return kQW1 + (i - kPW1);
    if (i >= kPW2 && i < kPB2) return kQW2 + (i - kPW2);
    if (i >= kPW3 && i < kPB3) return kQW3 + (i - kPW3);
    return -1;
}

struct MlpState {
    float* params;       // [kNumParams] FP32 master
    float* grad;         // [kNumParams]
    float* m;            // Adam first moment
    float* v;            // Adam second moment
    __nv_bfloat16* wq;   // [kNumQuant]
    float* loss;         // [1] summed per-sample loss of the last gradient
};

struct AdamStep {
    float lr, beta1, beta2, eps;
    float bc1, bc2;      // 1 - beta^t bias corrections
};

void launchMlpPredict(const MlpState& st, const float* x, uint32_t n, float* y, int grid, cudaStream_t s);
void launchMlpGrad(const MlpState& st, const float* x, const float* t, uint32_t n, int grid, cudaStream_t s);
void launchMlpAdam(const MlpState& st, const AdamStep& a, cudaStream_t s);
void launchMlpQuantize(const MlpState& st, cudaStream_t s);
cudaError_t configureMlp();

}  // namespace rb
