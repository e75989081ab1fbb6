// The learned scorer: a 16 -> 64 -> 64 -> 2 MLP with GELU, BF16 weights and
// activations, FP32 accumulation; inference, the gradient of the training loss,
// and Adam. The reference has no learned component (plans/04_NeuralPass.md is
// empty); the network, its inputs and targets are this project's.
//
// Outputs: y0 = predicted (final - partial) surface variation x 300, y1 = closure logit.
// Loss per sample: (y0 - t0)^2 + BCE(sigmoid(y1), t1), averaged over the batch.
// GELU is the tanh form (Hendrycks & Gimpel, arXiv:1606.08415):
//   gelu(z) = 0.5 z (1 + tanh(c (z + 0.044715 z^3))), c = sqrt(2 / pi).
// Adam: Kingma & Ba, arXiv:1412.6980, with bias correction.
//
// Layout of one warp's work: the warp takes one sample at a time; lane l owns
// hidden neurons l and l + 32 of both hidden layers, so a layer's activations
// are spread over the warp and the next layer gathers them with shuffles. The
// weight gradient of the 64 x 64 layer accumulates in a per-warp shared-memory
// copy (rows padded to 65 floats so the lanes' rows fall in different banks);
// the small layers' gradients stay in registers. At the end the block sums its
// warps' copies and adds them to the global gradient.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "rb_mlp.h"

namespace rb {

constexpr int kWarps = 8;
constexpr int kRow = 65;  // padded row of the per-warp dW2 copy

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__device__ __forceinline__ float gelu(float z, float* dgelu) {
    const float c = 0.7978845608028654f;
    const float u = c * (z + 0.044715f * z * z * z);
    const float t = tanhf(u);
    if (dgelu) {
        const float du = c * (1.0f + 3.0f * 0.044715f * z * z);
        *dgelu = 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * du;
    }
    return 0.5f * z * (1.0f + t);
}

struct SmemWeights {
    __nv_bfloat16 w1[kHidden * kIn];
    __nv_bfloat16 w2[kHidden * kHidden];
    __nv_bfloat16 w3[kOut * kHidden];
    float b1[kHidden], b2[kHidden], b3[kOut];
};

__device__ void loadWeights(SmemWeights& s, const __nv_bfloat16* wq, const float* params) {
    for (int i = threadIdx.x; i < kHidden * kIn; i += blockDim.x) s.w1[i] = wq[kQW1 + i];
    for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) s.w2[i] = wq[kQW2 + i];
    for (int i = threadIdx.x; i < kOut * kHidden; i += blockDim.x) s.w3[i] = wq[kQW3 + i];
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
        s.b1[i] = params[kPB1 + i];
        s.b2[i] = params[kPB2 + i];
    }
    if (threadIdx.x < kOut) s.b3[threadIdx.x] = params[kPB3 + threadIdx.x];
}

struct Fwd {
    float xb[kIn];
    float z1[2], a1b[2], dg1[2];
    float z2[2], a2b[2], dg2[2];
    float y[2];
};

// One sample through the network; every lane of the warp calls it.
__device__ __forceinline__ void forward(const SmemWeights& s, const float* x, Fwd& f, uint32_t lane) {
#pragma unroll
    for (int k = 0; k < kIn; k++) f.xb[k] = bf16r(x[k]);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = lane + 32 * h;
        float acc = s.b1[j];
#pragma unroll
        for (int k = 0; k < kIn; k++) acc += __bfloat162float(s.w1[j * kIn + k]) * f.xb[k];
        f.z1[h] = acc;
        f.a1b[h] = bf16r(gelu(acc, &f.dg1[h]));
    }
    float acc2[2] = {s.b2[lane], s.b2[lane + 32]};
#pragma unroll 8
    for (int k = 0; k < 32; k++) {
        const float v0 = __shfl_sync(0xFFFFFFFFu, f.a1b[0], k);
        const float v1 = __shfl_sync(0xFFFFFFFFu, f.a1b[1], k);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int j = lane + 32 * h;
            acc2[h] += __bfloat162float(s.w2[j * kHidden + k]) * v0 + __bfloat162float(s.w2[j * kHidden + k + 32]) * v1;
        }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        f.z2[h] = acc2[h];
        f.a2b[h] = bf16r(gelu(acc2[h], &f.dg2[h]));
    }
#pragma unroll
    for (int o = 0; o < kOut; o++) {
        float p = __bfloat162float(s.w3[o * kHidden + lane]) * f.a2b[0] +
                  __bfloat162float(s.w3[o * kHidden + lane + 32]) * f.a2b[1];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) p += __shfl_xor_sync(0xFFFFFFFFu, p, off);
        f.y[o] = p + s.b3[o];
    }
}

__global__ void __launch_bounds__(kWarps * 32) k_mlp_predict(const __nv_bfloat16* wq, const float* params,
                                                             const float* x, uint32_t n, float* y) {
    __shared__ SmemWeights s;
    loadWeights(s, wq, params);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t stride = gridDim.x * kWarps;
    for (uint32_t i = blockIdx.x * kWarps + warp; i < n; i += stride) {
        Fwd f;
        forward(s, x + (size_t)i * kIn, f, lane);
        if (lane == 0) {
            y[2 * i] = f.y[0];
            y[2 * i + 1] = f.y[1];
        }
    }
}

// Gradient of the mean loss over n samples, added into grad (kNumParams
// floats, zeroed by the caller); loss sum added into lossSum.
__global__ void __launch_bounds__(kWarps * 32) k_mlp_grad(const __nv_bfloat16* wq, const float* params,
                                                          const float* x, const float* t, uint32_t n,
                                                          float* grad, float* lossSum) {
    __shared__ SmemWeights s;
    extern __shared__ float s_dw2[];  // [kWarps][kHidden * kRow]
    loadWeights(s, wq, params);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    float* myDw2 = s_dw2 + (size_t)warp * kHidden * kRow;
    for (int i = lane; i < kHidden * kRow; i += 32) myDw2[i] = 0.0f;
    __syncthreads();
    const float invN = 1.0f / (float)n;
    float dw1[2][kIn];
    float db1[2] = {0, 0}, db2[2] = {0, 0}, dw3[kOut][2] = {{0, 0}, {0, 0}}, db3[kOut] = {0, 0};
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int k = 0; k < kIn; k++) dw1[h][k] = 0.0f;
    float loss = 0.0f;
    const uint32_t stride = gridDim.x * kWarps;
    for (uint32_t i = blockIdx.x * kWarps + warp; i < n; i += stride) {
        Fwd f;
        forward(s, x + (size_t)i * kIn, f, lane);
        const float t0 = t[2 * i], t1 = t[2 * i + 1];
        const float e = f.y[0] - t0;
        const float sig = 1.0f / (1.0f + expf(-f.y[1]));
        // BCE with logits, stable form: max(y,0) - y t + log(1 + exp(-|y|))
        const float bce = fmaxf(f.y[1], 0.0f) - f.y[1] * t1 + log1pf(expf(-fabsf(f.y[1])));
        if (lane == 0) loss += e * e + bce;  // every lane holds the sample's outputs; count it once
        const float dy[2] = {2.0f * e * invN, (sig - t1) * invN};
        // layer 3
        float dz2[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = lane + 32 * h;
            float da2 = 0.0f;
#pragma unroll
            for (int o = 0; o < kOut; o++) {
                dw3[o][h] += dy[o] * f.a2b[h];
                da2 += __bfloat162float(s.w3[o * kHidden + k]) * dy[o];
            }
            dz2[h] = da2 * f.dg2[h];
            db2[h] += dz2[h];
        }
#pragma unroll
        for (int o = 0; o < kOut; o++) db3[o] += dy[o];
        // layer 2: dW2[j][k] += dz2[j] a1b[k] (lane owns rows j = lane, lane + 32);
        // da1[k] = sum_j W2[j][k] dz2[j] (lane owns k = lane, lane + 32)
        float da1[2] = {0.0f, 0.0f};
#pragma unroll 4
        for (int q = 0; q < 32; q++) {
            const float a0 = __shfl_sync(0xFFFFFFFFu, f.a1b[0], q);
            const float a1 = __shfl_sync(0xFFFFFFFFu, f.a1b[1], q);
            myDw2[lane * kRow + q] += dz2[0] * a0;
            myDw2[lane * kRow + q + 32] += dz2[0] * a1;
            myDw2[(lane + 32) * kRow + q] += dz2[1] * a0;
            myDw2[(lane + 32) * kRow + q + 32] += dz2[1] * a1;
            const float d0 = __shfl_sync(0xFFFFFFFFu, dz2[0], q);
            const float d1 = __shfl_sync(0xFFFFFFFFu, dz2[1], q);
            da1[0] += __bfloat162float(s.w2[q * kHidden + lane]) * d0 +
                      __bfloat162float(s.w2[(q + 32) * kHidden + lane]) * d1;
            da1[1] += __bfloat162float(s.w2[q * kHidden + lane + 32]) * d0 +
                      __bfloat162float(s.w2[(q + 32) * kHidden + lane + 32]) * d1;
        }
        // layer 1
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const float dz1 = da1[h] * f.dg1[h];
            db1[h] += dz1;
#pragma unroll
            for (int k = 0; k < kIn; k++) dw1[h][k] += dz1 * f.xb[k];
        }
    }
    __syncwarp();
    // fold the warp's register accumulators into the global gradient
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int j = lane + 32 * h;
        for (int k = 0; k < kIn; k++) atomicAdd(&grad[kPW1 + j * kIn + k], dw1[h][k]);
        atomicAdd(&grad[kPB1 + j], db1[h]);
        atomicAdd(&grad[kPB2 + j], db2[h]);
        for (int o = 0; o < kOut; o++) atomicAdd(&grad[kPW3 + o * kHidden + j], dw3[o][h]);
    }
    if (lane == 0)
        for (int o = 0; o < kOut; o++) atomicAdd(&grad[kPB3 + o], db3[o]);
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, off);
    if (lane == 0) atomicAdd(lossSum, loss);
    __syncthreads();
    // the block's warps' dW2 copies, summed, into the global gradient
    for (int e = threadIdx.x; e < kHidden * kHidden; e += blockDim.x) {
        const int j = e / kHidden, k = e % kHidden;
        float v = 0.0f;
        for (int w = 0; w < kWarps; w++) v += s_dw2[(size_t)w * kHidden * kRow + j * kRow + k];
        atomicAdd(&grad[kPW2 + e], v);
    }
}

__global__ void k_mlp_adam(float* params, const float* grad, float* m, float* v, __nv_bfloat16* wq, AdamStep a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNumParams; i += gridDim.x * blockDim.x) {
        const float g = grad[i];
        const float mi = a.beta1 * m[i] + (1.0f - a.beta1) * g;
        const float vi = a.beta2 * v[i] + (1.0f - a.beta2) * g * g;
        m[i] = mi;
        v[i] = vi;
        const float mh = mi / a.bc1, vh = vi / a.bc2;
        const float w = params[i] - a.lr * mh / (sqrtf(vh) + a.eps);
        params[i] = w;
        const int q = quantIndex(i);
        if (q >= 0) wq[q] = __float2bfloat16_rn(w);
    }
}

__global__ void k_mlp_quantize(const float* params, __nv_bfloat16* wq) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNumParams; i += gridDim.x * blockDim.x) {
        const int q = quantIndex(i);
        if (q >= 0) wq[q] = __float2bfloat16_rn(params[i]);
    }
}

void launchMlpPredict(const MlpState& st, const float* x, uint32_t n, float* y, int grid, cudaStream_t s) {
    if (n == 0) return;
    k_mlp_predict<<<grid, kWarps * 32, 0, s>>>(st.wq, st.params, x, n, y);
}

size_t mlpGradSmem() { return (size_t)kWarps * kHidden * kRow * sizeof(float); }

cudaError_t configureMlp() {
    return cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlpGradSmem());
}

void launchMlpGrad(const MlpState& st, const float* x, const float* t, uint32_t n, int grid, cudaStream_t s) {
    if (n == 0) return;
    k_mlp_grad<<<grid, kWarps * 32, mlpGradSmem(), s>>>(st.wq, st.params, x, t, n, st.grad, st.loss);
}

void launchMlpAdam(const MlpState& st, const AdamStep& a, cudaStream_t s) {
    k_mlp_adam<<<(kNumParams + 255) / 256, 256, 0, s>>>(st.params, st.grad, st.m, st.v, st.wq, a);
}

void launchMlpQuantize(const MlpState& st, cudaStream_t s) {
    k_mlp_quantize<<<(kNumParams + 255) / 256, 256, 0, s>>>(st.params, st.wq);
}

}  // namespace rb
