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
// Every contraction runs on the tensor cores as mma.sync.m16n8k16 (BF16 in,
// FP32 accumulate). A warp takes 16 samples: the layers are GEMMs of the
// warp's [16 x K] activations with the [K x N] weights, and a layer's FP32
// result tile, rounded to BF16, is already laid out as the next layer's A
// operand, so activations never leave registers. The backward pass computes
// dA1 = dZ2 W2 per warp the same way; the weight gradients dW2 = dZ2^T A1 and
// dW1 = dZ1^T X are contractions over samples, so each block stages its 64
// samples' dZ2, A1, dZ1 and X transposed in shared memory and each warp
// accumulates one 16-row slice of dW2 and dW1 across the block's samples.
// Bias gradients, the 64 x 2 output layer and its gradient are sums and dot
// products with 2 outputs: warp shuffles, not GEMMs.
//
// Fragment layouts (PTX ISA, mma.m16n8k16 with .bf16): lane = 4 g + t;
// A (16 x 16, row-major): {a0, a1, a2, a3} = rows {g, g + 8, g, g + 8}, columns
// {2t, 2t + 1} (+ 8 for a2, a3); B (16 x 8): {b0, b1} = rows {2t, 2t + 1}
// (+ 8 for b1), column g; C (16 x 8): {c0, c1, c2, c3} = (row g, columns 2t,
// 2t + 1), (row g + 8, the same columns).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "rb_mlp.h"

namespace rb {

constexpr int kWarps = 4;                  // warps per block
constexpr int kTile = 16;                  // samples per warp and tile
constexpr int kBlockSamples = kWarps * kTile;
// shared-memory row strides in BF16 elements, padded so that the 8 rows a
// fragment load touches fall in different banks
constexpr int kW1Row = 24;                 // W1 [64][16]
constexpr int kW2Row = 72;                 // W2 and W2^T [64][64]
constexpr int kW3Row = 72;                 // W3 padded to [8][64]
constexpr int kSRow = 72;                  // per-sample columns of the staged transposes [.][64]

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&p);
}

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

// D += A B on the tensor cores.
__device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

struct SmemWeights {
    __nv_bfloat16 w1[kHidden * kW1Row];   // W1[n][k]
    __nv_bfloat16 w2[kHidden * kW2Row];   // W2[n][k]
    __nv_bfloat16 w2t[kHidden * kW2Row];  // W2^T[k][n] (backward)
    __nv_bfloat16 w3[8 * kW3Row];         // W3[n][k], rows 2..7 zero
    float b1[kHidden], b2[kHidden], b3[8];
    float w3f[kOut][kHidden];             // W3 as FP32 values of its BF16 copy (backward dot products)
};

__device__ void loadWeights(SmemWeights& s, const __nv_bfloat16* wq, const float* params) {
    for (int i = threadIdx.x; i < kHidden * kIn; i += blockDim.x) s.w1[(i / kIn) * kW1Row + i % kIn] = wq[kQW1 + i];
    for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) {
        const int n = i / kHidden, k = i % kHidden;
        s.w2[n * kW2Row + k] = wq[kQW2 + i];
        s.w2t[k * kW2Row + n] = wq[kQW2 + i];
    }
    for (int i = threadIdx.x; i < 8 * kHidden; i += blockDim.x) {
        const int n = i / kHidden, k = i % kHidden;
        const __nv_bfloat16 w = n < kOut ? wq[kQW3 + n * kHidden + k] : __float2bfloat16_rn(0.0f);
        s.w3[n * kW3Row + k] = w;
        if (n < kOut) s.w3f[n][k] = __bfloat162float(w);
    }
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
        s.b1[i] = params[kPB1 + i];
        s.b2[i] = params[kPB2 + i];
    }
    if (threadIdx.x < 8) s.b3[threadIdx.x] = threadIdx.x < kOut ? params[kPB3 + threadIdx.x] : 0.0f;
}

// One warp's forward pass over samples [base, base + 16) (rows past n are
// zeros). Leaves the layers' values in fragment layout.
struct Fwd {
    uint32_t xa[4];        // X rounded to BF16: A operand of layer 1
    uint32_t a1[4][4];     // A1 rounded to BF16: A operand of layer 2, per k-step
    uint32_t a2[4][4];     // A2 rounded to BF16: A operand of layer 3
    float dg1[8][4];       // gelu'(Z1) per C element of layer 1
    float dg2[8][4];       // gelu'(Z2)
    float y[4];            // layer 3's C tile: (row g, outputs 2t, 2t + 1), (row g + 8, ...)
};

template <bool kGrad>
__device__ __forceinline__ void forwardTile(const SmemWeights& s, const float* __restrict__ x, uint32_t n,
                                            uint32_t base, Fwd& f) {
    const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
    // layer 1: X [16 x 16] x W1^T
    {
        const uint32_t r0 = base + g, r1 = base + g + 8;
        float2 v00 = make_float2(0.f, 0.f), v01 = v00, v10 = v00, v11 = v00;
        if (r0 < n) {
            v00 = *reinterpret_cast<const float2*>(x + (size_t)r0 * kIn + 2 * t);
            v01 = *reinterpret_cast<const float2*>(x + (size_t)r0 * kIn + 2 * t + 8);
        }
        if (r1 < n) {
            v10 = *reinterpret_cast<const float2*>(x + (size_t)r1 * kIn + 2 * t);
            v11 = *reinterpret_cast<const float2*>(x + (size_t)r1 * kIn + 2 * t + 8);
        }
        f.xa[0] = pack2(v00.x, v00.y);
        f.xa[1] = pack2(v10.x, v10.y);
        f.xa[2] = pack2(v01.x, v01.y);
        f.xa[3] = pack2(v11.x, v11.y);
    }
    float c[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int col = 8 * i + 2 * t;
        c[i][0] = s.b1[col];
        c[i][1] = s.b1[col + 1];
        c[i][2] = s.b1[col];
        c[i][3] = s.b1[col + 1];
        const __nv_bfloat16* w = s.w1 + (8 * i + g) * kW1Row + 2 * t;
        mma(c[i], f.xa, lds32(w), lds32(w + 8));
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int e = 0; e < 4; e++) c[i][e] = gelu(c[i][e], kGrad ? &f.dg1[i][e] : nullptr);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        f.a1[j][0] = pack2(c[2 * j][0], c[2 * j][1]);
        f.a1[j][1] = pack2(c[2 * j][2], c[2 * j][3]);
        f.a1[j][2] = pack2(c[2 * j + 1][0], c[2 * j + 1][1]);
        f.a1[j][3] = pack2(c[2 * j + 1][2], c[2 * j + 1][3]);
    }
    // layer 2: A1 [16 x 64] x W2^T
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int col = 8 * i + 2 * t;
        c[i][0] = s.b2[col];
        c[i][1] = s.b2[col + 1];
        c[i][2] = s.b2[col];
        c[i][3] = s.b2[col + 1];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const __nv_bfloat16* w = s.w2 + (8 * i + g) * kW2Row + 16 * j + 2 * t;
            mma(c[i], f.a1[j], lds32(w), lds32(w + 8));
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int e = 0; e < 4; e++) c[i][e] = gelu(c[i][e], kGrad ? &f.dg2[i][e] : nullptr);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        f.a2[j][0] = pack2(c[2 * j][0], c[2 * j][1]);
        f.a2[j][1] = pack2(c[2 * j][2], c[2 * j][3]);
        f.a2[j][2] = pack2(c[2 * j + 1][0], c[2 * j + 1][1]);
        f.a2[j][3] = pack2(c[2 * j + 1][2], c[2 * j + 1][3]);
    }
    // layer 3: A2 [16 x 64] x W3^T, the two outputs padded to an 8-wide tile
    f.y[0] = s.b3[2 * t];
    f.y[1] = s.b3[2 * t + 1];
    f.y[2] = s.b3[2 * t];
    f.y[3] = s.b3[2 * t + 1];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const __nv_bfloat16* w = s.w3 + g * kW3Row + 16 * j + 2 * t;
        mma(f.y, f.a2[j], lds32(w), lds32(w + 8));
    }
}

__global__ void __launch_bounds__(kWarps * 32) k_mlp_predict(const __nv_bfloat16* wq, const float* params,
                                                             const float* __restrict__ x, uint32_t n, float* y) {
    __shared__ SmemWeights s;
    loadWeights(s, wq, params);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3u;
    for (uint32_t base = (blockIdx.x * kWarps + warp) * kTile; base < n; base += gridDim.x * kBlockSamples) {
        Fwd f;
        forwardTile<false>(s, x, n, base, f);
        if (t == 0) {
            if (base + g < n) *reinterpret_cast<float2*>(y + 2 * (size_t)(base + g)) = make_float2(f.y[0], f.y[1]);
            if (base + g + 8 < n)
                *reinterpret_cast<float2*>(y + 2 * (size_t)(base + g + 8)) = make_float2(f.y[2], f.y[3]);
        }
    }
}

// The block's staged transposes for the weight-gradient GEMMs: per neuron (or
// input), its value for each of the block's 64 samples.
struct SmemStage {
    __nv_bfloat16 dz2t[kHidden * kSRow];  // dZ2^T [layer-2 neuron][sample]
    __nv_bfloat16 a1t[kHidden * kSRow];   // A1^T  [layer-1 neuron][sample]
    __nv_bfloat16 dz1t[kHidden * kSRow];  // dZ1^T [layer-1 neuron][sample]
    __nv_bfloat16 xt[kIn * kSRow];        // X^T   [input][sample]
    float red[kOut * kHidden + kHidden + kHidden + 8];  // dW3, db2, db1, db3 block sums
};

// Sum of v over the 8 row groups of a fragment (lanes with equal t).
__device__ __forceinline__ float sumRows(float v) {
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 4);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 8);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 16);
    return v;
}

// Gradient of the mean loss over n samples, added into grad (kNumParams
// floats, zeroed by the caller); loss sum added into lossSum.
__global__ void __launch_bounds__(kWarps * 32) k_mlp_grad(const __nv_bfloat16* wq, const float* params,
                                                          const float* __restrict__ x, const float* __restrict__ tgt,
                                                          uint32_t n, float* grad, float* lossSum) {
    // 55 KB: over the static limit, so dynamic
    extern __shared__ __align__(16) unsigned char s_raw[];
    SmemWeights& s = *reinterpret_cast<SmemWeights*>(s_raw);
    SmemStage& st = *reinterpret_cast<SmemStage*>(s_raw + ((sizeof(SmemWeights) + 15) & ~size_t(15)));
    loadWeights(s, wq, params);
    for (int i = threadIdx.x; i < (int)(sizeof(st.red) / sizeof(float)); i += blockDim.x) st.red[i] = 0.0f;
    __syncthreads();
    float* sdw3 = st.red;
    float* sdb2 = st.red + kOut * kHidden;
    float* sdb1 = sdb2 + kHidden;
    float* sdb3 = sdb1 + kHidden;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3u;
    const float invN = 1.0f / (float)n;
    // this warp's slices of the weight gradients: rows 16 warp .. +15 of dW2 (8 column tiles) and dW1 (2)
    float dw2[8][4], dw1[2][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int e = 0; e < 4; e++) dw2[i][e] = 0.0f;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int e = 0; e < 4; e++) dw1[i][e] = 0.0f;
    float loss = 0.0f;
    for (uint32_t block0 = blockIdx.x * kBlockSamples; block0 < n; block0 += gridDim.x * kBlockSamples) {
        const uint32_t base = block0 + warp * kTile;
        const uint32_t col0 = warp * kTile;  // this warp's sample columns in the staged transposes
        Fwd f;
        forwardTile<true>(s, x, n, base, f);
        // the loss and dY per sample (lanes t == 0 hold the outputs of rows g and g + 8)
        float dy[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
        if (t == 0) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t r = base + g + 8 * h;
                if (r >= n) continue;
                const float y0 = f.y[2 * h], y1 = f.y[2 * h + 1];
                const float2 tv = *reinterpret_cast<const float2*>(tgt + 2 * (size_t)r);
                const float e = y0 - tv.x;
                const float sig = 1.0f / (1.0f + expf(-y1));
                // BCE with logits, stable form: max(y,0) - y t + log(1 + exp(-|y|))
                loss += e * e + fmaxf(y1, 0.0f) - y1 * tv.y + log1pf(expf(-fabsf(y1)));
                dy[h][0] = 2.0f * e * invN;
                dy[h][1] = (sig - tv.y) * invN;
            }
        }
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
            for (int o = 0; o < 2; o++) dy[h][o] = __shfl_sync(0xFFFFFFFFu, dy[h][o], lane & ~3u);
        {
            // db3: every lane of a row group holds its rows' dY; count it once (t == 0)
            const float s0 = sumRows(t == 0 ? dy[0][0] + dy[1][0] : 0.0f);
            const float s1 = sumRows(t == 0 ? dy[0][1] + dy[1][1] : 0.0f);
            if (lane == 0) {
                atomicAdd(&sdb3[0], s0);
                atomicAdd(&sdb3[1], s1);
            }
        }
        // layer 3 backward: dW3 += dY^T A2, dA2 = dY W3, dZ2 = dA2 gelu'(Z2)
        float dz2[8][4];
#pragma unroll
        for (int i = 0; i < 8; i++) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int col = 8 * i + 2 * t + (e & 1);
                const int h = e >> 1;
                dz2[i][e] = (dy[h][0] * s.w3f[0][col] + dy[h][1] * s.w3f[1][col]) * f.dg2[i][e];
            }
            // A2 values of this tile (BF16 as stored in the fragments)
            const __nv_bfloat162 lo = *reinterpret_cast<const __nv_bfloat162*>(&f.a2[i >> 1][(i & 1) * 2]);
            const __nv_bfloat162 hi = *reinterpret_cast<const __nv_bfloat162*>(&f.a2[i >> 1][(i & 1) * 2 + 1]);
            const float a2v[4] = {__low2float(lo), __high2float(lo), __low2float(hi), __high2float(hi)};
#pragma unroll
            for (int o = 0; o < 2; o++) {
                float w0 = dy[0][o] * a2v[0] + dy[1][o] * a2v[2];
                float w1 = dy[0][o] * a2v[1] + dy[1][o] * a2v[3];
                w0 = sumRows(w0);
                w1 = sumRows(w1);
                if (g == 0) {
                    atomicAdd(&sdw3[o * kHidden + 8 * i + 2 * t], w0);
                    atomicAdd(&sdw3[o * kHidden + 8 * i + 2 * t + 1], w1);
                }
            }
            float b0 = sumRows(dz2[i][0] + dz2[i][2]), b1 = sumRows(dz2[i][1] + dz2[i][3]);
            if (g == 0) {
                atomicAdd(&sdb2[8 * i + 2 * t], b0);
                atomicAdd(&sdb2[8 * i + 2 * t + 1], b1);
            }
        }
        // dZ2 as the A operand of dA1 = dZ2 W2 (K = layer-2 neurons), and staged transposed
        uint32_t dza[4][4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            dza[j][0] = pack2(dz2[2 * j][0], dz2[2 * j][1]);
            dza[j][1] = pack2(dz2[2 * j][2], dz2[2 * j][3]);
            dza[j][2] = pack2(dz2[2 * j + 1][0], dz2[2 * j + 1][1]);
            dza[j][3] = pack2(dz2[2 * j + 1][2], dz2[2 * j + 1][3]);
        }
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int col = 8 * i + 2 * t + (e & 1);
                const int row = g + 8 * (e >> 1);
                st.dz2t[col * kSRow + col0 + row] = __float2bfloat16_rn(dz2[i][e]);
            }
        // A1 and X staged transposed (their BF16 values)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&f.a1[j][q]);
                const int col = 16 * j + 2 * t + 8 * (q >> 1);
                const int row = g + 8 * (q & 1);
                st.a1t[col * kSRow + col0 + row] = v.x;
                st.a1t[(col + 1) * kSRow + col0 + row] = v.y;
            }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&f.xa[q]);
            const int col = 2 * t + 8 * (q >> 1);
            const int row = g + 8 * (q & 1);
            st.xt[col * kSRow + col0 + row] = v.x;
            st.xt[(col + 1) * kSRow + col0 + row] = v.y;
        }
        // layer 2 backward: dA1 = dZ2 W2, dZ1 = dA1 gelu'(Z1)
#pragma unroll
        for (int i = 0; i < 8; i++) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                // B[k][n] = W2[k][n]: k = layer-2 neuron, n = layer-1 neuron
                const __nv_bfloat16* w = s.w2t + (8 * i + g) * kW2Row + 16 * j + 2 * t;
                mma(c, dza[j], lds32(w), lds32(w + 8));
            }
            float dz1[4];
#pragma unroll
            for (int e = 0; e < 4; e++) dz1[e] = c[e] * f.dg1[i][e];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int col = 8 * i + 2 * t + (e & 1);
                const int row = g + 8 * (e >> 1);
                st.dz1t[col * kSRow + col0 + row] = __float2bfloat16_rn(dz1[e]);
            }
            float b0 = sumRows(dz1[0] + dz1[2]), b1 = sumRows(dz1[1] + dz1[3]);
            if (g == 0) {
                atomicAdd(&sdb1[8 * i + 2 * t], b0);
                atomicAdd(&sdb1[8 * i + 2 * t + 1], b1);
            }
        }
        __syncthreads();
        // the weight gradients over the block's 64 samples: this warp's 16 rows
        const int m0 = 16 * warp;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            uint32_t a[4];
            const __nv_bfloat16* p = st.dz2t + (m0 + g) * kSRow + 16 * k + 2 * t;
            a[0] = lds32(p);
            a[1] = lds32(p + 8 * kSRow);
            a[2] = lds32(p + 8);
            a[3] = lds32(p + 8 * kSRow + 8);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const __nv_bfloat16* b = st.a1t + (8 * i + g) * kSRow + 16 * k + 2 * t;
                mma(dw2[i], a, lds32(b), lds32(b + 8));
            }
            const __nv_bfloat16* q = st.dz1t + (m0 + g) * kSRow + 16 * k + 2 * t;
            a[0] = lds32(q);
            a[1] = lds32(q + 8 * kSRow);
            a[2] = lds32(q + 8);
            a[3] = lds32(q + 8 * kSRow + 8);
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const __nv_bfloat16* b = st.xt + (8 * i + g) * kSRow + 16 * k + 2 * t;
                mma(dw1[i], a, lds32(b), lds32(b + 8));
            }
        }
        __syncthreads();
    }
    // this warp's slices of dW2 and dW1, and the block's shuffled sums, into the global gradient
    const int m0 = 16 * warp;
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int row = m0 + g + 8 * (e >> 1), col = 8 * i + 2 * t + (e & 1);
            atomicAdd(&grad[kPW2 + row * kHidden + col], dw2[i][e]);
        }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int row = m0 + g + 8 * (e >> 1), col = 8 * i + 2 * t + (e & 1);
            atomicAdd(&grad[kPW1 + row * kIn + col], dw1[i][e]);
        }
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, off);
    if (lane == 0) atomicAdd(lossSum, loss);
    __syncthreads();
    for (int i = threadIdx.x; i < kOut * kHidden; i += blockDim.x) atomicAdd(&grad[kPW3 + i], sdw3[i]);
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
        atomicAdd(&grad[kPB2 + i], sdb2[i]);
        atomicAdd(&grad[kPB1 + i], sdb1[i]);
    }
    if (threadIdx.x < kOut) atomicAdd(&grad[kPB3 + threadIdx.x], sdb3[threadIdx.x]);
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
    const uint32_t tiles = (n + kBlockSamples - 1) / kBlockSamples;
    k_mlp_predict<<<tiles < (uint32_t)grid ? (int)tiles : grid, kWarps * 32, 0, s>>>(st.wq, st.params, x, n, y);
}

constexpr size_t kGradSmem = ((sizeof(SmemWeights) + 15) & ~size_t(15)) + sizeof(SmemStage);

cudaError_t configureMlp() {
    return cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
}

void launchMlpGrad(const MlpState& st, const float* x, const float* t, uint32_t n, int grid, cudaStream_t s) {
    if (n == 0) return;
    const uint32_t tiles = (n + kBlockSamples - 1) / kBlockSamples;
    k_mlp_grad<<<tiles < (uint32_t)grid ? (int)tiles : grid, kWarps * 32, kGradSmem, s>>>(st.wq, st.params, x, t, n,
                                                                                           st.grad, st.loss);
}

void launchMlpAdam(const MlpState& st, const AdamStep& a, cudaStream_t s) {
    k_mlp_adam<<<(kNumParams + 255) / 256, 256, 0, s>>>(st.params, st.grad, st.m, st.v, st.wq, a);
}

void launchMlpQuantize(const MlpState& st, cudaStream_t s) {
    k_mlp_quantize<<<(kNumParams + 255) / 256, 256, 0, s>>>(st.params, st.wq);
}

}  // namespace rb
