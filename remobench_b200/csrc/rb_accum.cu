// Accumulate stage: per-leaf running sums behind a watermark, one block per
// dirty leaf (restates kernels/remolod/remolod_accum.cu:47-233).
//
// The reference sums node-local coordinates in [0, 1] as doubles, so its sums
// depend on the order the points are folded in. Here each point is quantised
// to its 28-bit octree coordinate P (the reference's MAX_DEPTH_GRIDSIZE grid,
// remolod_octree.cu:167-169) and taken relative to its leaf,
//   q = clamp(P - (N << (28 - L)), 0, 2^(28 - L))   per axis,
// and Σq (u64) and Σqqᵀ (128-bit) are exact integers: any fold order gives the
// same bits. Colour sums are exact integers of the 8-bit channels.
//
// Bound: reading 16 B per new point (plus its chunk-table entry). The watermark
// `count` makes the pass incremental: only [count, numPoints) is read.
#include <cuda_runtime.h>

#include "rb_kernels.h"
#include "rb_state.h"

namespace rb {

__device__ __forceinline__ uint32_t aq(float c, float mn, float size, float scale) {
    float d = __fsub_rn(c, mn);
    return __float2uint_rz(__fdiv_rn(__fmul_rn(scale, d), size));
}

// remoMortonSpread / remoMortonCode (remolod_accum.cu:24-36)
__device__ __forceinline__ unsigned long long mortonSpread(uint32_t v) {
    unsigned long long x = (unsigned long long)v & 0xFFFFFull;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__device__ __forceinline__ void add128(unsigned long long& lo, unsigned long long& hi,
                                       unsigned long long v) {
    const unsigned long long o = lo;
    lo = o + v;
    hi += (lo < o) ? 1ull : 0ull;
}

__device__ __forceinline__ bool leafRow(const Dev& d, uint32_t node) {
    const int4* row = reinterpret_cast<const int4*>(d.child + node * 8u);
    const int4 a = row[0], b = row[1];
    return (a.x & a.y & a.z & a.w & b.x & b.y & b.z & b.w) == -1;
}

constexpr int kAccumThreads = 256;
constexpr int kAccumWarps = kAccumThreads / 32;
constexpr int kNumSums = 3 + 12 + 3 + 3;  // s1, s2 (lo, hi), c1, c2

// Folds one leaf's [count, numPoints) or clears an inner node's sums.
// useList: iterate the dirty list; otherwise every node.
__global__ void __launch_bounds__(kAccumThreads) k_accumulate(Dev d, uint32_t batchIndex, int useList) {
    __shared__ unsigned long long s_red[kNumSums][kAccumWarps];
    __shared__ unsigned long long s_morton[kAccumWarps];
    const Counters* c = d.ctr;
    const uint32_t total = useList ? (c->numDirty < d.maxNodes ? c->numDirty : d.maxNodes) : c->numNodes;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t ppc = d.ppc;
    for (uint32_t w = blockIdx.x; w < total; w += gridDim.x) {
        const uint32_t node = useList ? d.dirtyList[w] : w;
        AccumI* a = &d.accum[node];
        if (!leafRow(d, node)) {
            if (threadIdx.x == 0 && a->count != 0) {
                AccumI z = {};
                *a = z;
            }
            continue;
        }
        const uint32_t from = a->count;
        const uint32_t to = d.numPoints[node];
        if (to <= from) continue;
        const uint32_t cap = d.numPointChunks[node] * ppc;
        const uint32_t end = to < cap ? to : cap;
        const uint32_t lv = d.level[node];
        const uint32_t sh = 28u - lv;
        const long long lim = 1ll << sh;
        const long long bx = (long long)d.nodeX[node] << sh;
        const long long by = (long long)d.nodeY[node] << sh;
        const long long bz = (long long)d.nodeZ[node] << sh;
        const uint32_t toff = d.ptTableOff[node];

        unsigned long long s1[3] = {0, 0, 0};
        unsigned long long lo[6] = {0, 0, 0, 0, 0, 0}, hi[6] = {0, 0, 0, 0, 0, 0};
        unsigned long long c1[3] = {0, 0, 0}, c2[3] = {0, 0, 0};
        unsigned long long wm = 0;
        for (uint32_t s = from + threadIdx.x; s < end; s += blockDim.x) {
            const uint32_t phys = d.tablePool[toff + s / ppc];
            if (phys == kNone) continue;
            const float4 v = __ldg(reinterpret_cast<const float4*>(chunkPoints(d, phys) + s % ppc));
            const uint32_t P[3] = {aq(v.x, d.boxMin[0], d.octreeSize, 268435456.0f),
                                   aq(v.y, d.boxMin[1], d.octreeSize, 268435456.0f),
                                   aq(v.z, d.boxMin[2], d.octreeSize, 268435456.0f)};
            long long q[3] = {(long long)P[0] - bx, (long long)P[1] - by, (long long)P[2] - bz};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                q[k] = q[k] < 0 ? 0 : (q[k] > lim ? lim : q[k]);
                s1[k] += (unsigned long long)q[k];
            }
            add128(lo[0], hi[0], (unsigned long long)(q[0] * q[0]));
            add128(lo[1], hi[1], (unsigned long long)(q[0] * q[1]));
            add128(lo[2], hi[2], (unsigned long long)(q[0] * q[2]));
            add128(lo[3], hi[3], (unsigned long long)(q[1] * q[1]));
            add128(lo[4], hi[4], (unsigned long long)(q[1] * q[2]));
            add128(lo[5], hi[5], (unsigned long long)(q[2] * q[2]));
            const uint32_t col = __float_as_uint(v.w);
            const uint32_t ch[3] = {col & 255u, (col >> 8) & 255u, (col >> 16) & 255u};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                c1[k] += ch[k];
                c2[k] += ch[k] * ch[k];
            }
            uint32_t X = aq(v.x, d.boxMin[0], d.octreeSize, 1048576.0f);
            uint32_t Y = aq(v.y, d.boxMin[1], d.octreeSize, 1048576.0f);
            uint32_t Z = aq(v.z, d.boxMin[2], d.octreeSize, 1048576.0f);
            X = X < 1048575u ? X : 1048575u;
            Y = Y < 1048575u ? Y : 1048575u;
            Z = Z < 1048575u ? Z : 1048575u;
            const unsigned long long m = (mortonSpread(X) << 2) | (mortonSpread(Y) << 1) | mortonSpread(Z);
            wm = m > wm ? m : wm;
        }
        // warp reduction
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                s1[k] += __shfl_down_sync(0xFFFFFFFFu, s1[k], off);
                c1[k] += __shfl_down_sync(0xFFFFFFFFu, c1[k], off);
                c2[k] += __shfl_down_sync(0xFFFFFFFFu, c2[k], off);
            }
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const unsigned long long ol = __shfl_down_sync(0xFFFFFFFFu, lo[k], off);
                const unsigned long long oh = __shfl_down_sync(0xFFFFFFFFu, hi[k], off);
                const unsigned long long nl = lo[k] + ol;
                hi[k] += oh + (nl < lo[k] ? 1ull : 0ull);
                lo[k] = nl;
            }
            const unsigned long long om = __shfl_down_sync(0xFFFFFFFFu, wm, off);
            wm = om > wm ? om : wm;
        }
        if (lane == 0) {
            for (int k = 0; k < 3; k++) {
                s_red[k][warp] = s1[k];
                s_red[15 + k][warp] = c1[k];
                s_red[18 + k][warp] = c2[k];
            }
            for (int k = 0; k < 6; k++) {
                s_red[3 + k][warp] = lo[k];
                s_red[9 + k][warp] = hi[k];
            }
            s_morton[warp] = wm;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            AccumI acc = *a;
            unsigned long long m = 0;
            for (int w2 = 0; w2 < kAccumWarps; w2++) {
                for (int k = 0; k < 3; k++) {
                    acc.s1[k] += s_red[k][w2];
                    acc.c1[k] += s_red[15 + k][w2];
                    acc.c2[k] += s_red[18 + k][w2];
                }
                for (int k = 0; k < 6; k++) {
                    acc.s2hi[k] += s_red[9 + k][w2];
                    add128(acc.s2lo[k], acc.s2hi[k], s_red[3 + k][w2]);
                }
                m = s_morton[w2] > m ? s_morton[w2] : m;
            }
            acc.count = to;
            acc.lastTouchedBatch = batchIndex;
            *a = acc;
            atomicMax(&d.accumGlobals->mortonWatermark, m);
            atomicAdd(&d.accumGlobals->numAccumulated, (unsigned long long)(to - from));
            atomicAdd(&d.accumGlobals->pointsFolded, to - from);
            atomicAdd(&d.accumGlobals->numLeavesFolded, 1u);
        }
        __syncthreads();
    }
}

// kernel_accum_verify (remolod_accum.cu:214-233)
__global__ void __launch_bounds__(256) k_accum_verify(Dev d) {
    const uint32_t nn = d.ctr->numNodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const uint32_t cnt = d.accum[i].count;
        if (leafRow(d, i)) {
            if (cnt) atomicAdd(&d.accumGlobals->sumLeafCounts, (unsigned long long)cnt);
        } else if (cnt != 0) {
            atomicAdd(&d.accumGlobals->innerWithSums, 1u);
        }
    }
}

void launchAccumulate(const Dev& d, uint32_t batchIndex, int useList, int grid, cudaStream_t s) {
    k_accumulate<<<grid, kAccumThreads, 0, s>>>(d, batchIndex, useList);
}
void launchAccumVerify(const Dev& d, int grid, cudaStream_t s) { k_accum_verify<<<grid, 256, 0, s>>>(d); }

}  // namespace rb
