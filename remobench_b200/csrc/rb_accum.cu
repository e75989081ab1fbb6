// Accumulate stage: per-leaf running sums behind a watermark, restating
// kernels/remolod/remolod_accum.cu:47-233. A plan splits every dirty leaf's
// new points into fixed-size work items spread over the whole grid.
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

// The watermark is the largest 60-bit Morton code of the folded points.
// Codes are compared without building them: the dimension whose coordinates
// differ in the highest bit decides (x before y before z at the same bit, the
// order of the interleave), found with the test "msb(p) < msb(q)" =
// p < q && p < (p ^ q) (Chan, "Closest-point problems simplified on the RAM",
// SODA 2002). Only the block's largest point is spread into a code.
__device__ __forceinline__ bool msbLess(uint32_t p, uint32_t q) { return p < q && p < (p ^ q); }

__device__ __forceinline__ bool mortonLess(uint32_t ax, uint32_t ay, uint32_t az, uint32_t bx, uint32_t by,
                                           uint32_t bz) {
    const uint32_t dx = ax ^ bx, dy = ay ^ by, dz = az ^ bz;
    uint32_t da = dx, a = ax, b = bx;
    if (msbLess(da, dy)) {
        da = dy;
        a = ay;
        b = by;
    }
    if (msbLess(da, dz)) {
        a = az;
        b = bz;
    }
    return a < b;
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
// Points per work item: a leaf's new range is split over several blocks, so
// a fold over a few hundred big leaves still fills the GPU.
constexpr uint32_t kAccumChunk = 4096;

// 128-bit atomic add on a (lo, hi) pair: the add that wraps lo carries into hi.
__device__ __forceinline__ void atomicAdd128(unsigned long long* lo, unsigned long long* hi,
                                             unsigned long long vlo, unsigned long long vhi) {
    const unsigned long long old = atomicAdd(lo, vlo);
    const unsigned long long carry = (old + vlo < old) ? 1ull : 0ull;
    if (vhi + carry) atomicAdd(hi, vhi + carry);
}

// The fold's plan (one block): the nodes to visit (the dirty list, or every
// node), each leaf's new range [count, min(numPoints, capacity)) read before
// any block updates count, and each node's first work item. An inner node
// with sums is one item (cleared); a leaf with new points one item per
// kAccumChunk points. Folded-leaf and point totals are counted here.
__global__ void __launch_bounds__(1024) k_accum_plan(Dev d, int useList) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_run, s_leaves;
    __shared__ unsigned long long s_points;
    Counters* c = d.ctr;
    const uint32_t total = useList ? (c->numDirty < d.maxNodes ? c->numDirty : d.maxNodes) : c->numNodes;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_run = 0;
        s_leaves = 0;
        s_points = 0;
    }
    __syncthreads();
    for (uint32_t w0 = 0; w0 < total; w0 += blockDim.x) {
        const uint32_t w = w0 + threadIdx.x;
        uint32_t items = 0, from = 0, to = 0;
        if (w < total) {
            const uint32_t node = useList ? d.dirtyList[w] : w;
            if (!leafRow(d, node)) {
                items = d.accum[node].count != 0u ? 1u : 0u;
            } else {
                from = d.accum[node].count;
                const uint32_t cap = d.numPointChunks[node] * d.ppc;
                const uint32_t np = d.numPoints[node];
                to = np < cap ? np : cap;
                if (to > from) {
                    items = (to - from + kAccumChunk - 1u) / kAccumChunk;
                    atomicAdd(&s_leaves, 1u);
                    atomicAdd(&s_points, (unsigned long long)(to - from));
                } else {
                    to = from;
                }
            }
            d.accumFrom[w] = from;
            d.accumTo[w] = to;
        }
        // block-wide exclusive scan of the item counts
        uint32_t x = items;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31u) s_warp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t v = lane < blockDim.x / 32u ? s_warp[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
                if (lane >= (uint32_t)o) v += y;
            }
            s_warp[lane] = v;
        }
        __syncthreads();
        const uint32_t pre = s_run + (warp > 0 ? s_warp[warp - 1] : 0u) + x - items;
        if (w < total) d.accumItem[w] = pre;
        __syncthreads();
        if (threadIdx.x == 0) s_run += s_warp[blockDim.x / 32u - 1u];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        d.accumItem[total] = s_run;
        c->accumItems = s_run;
        d.accumGlobals->numAccumulated += s_points;
        d.accumGlobals->pointsFolded += (uint32_t)s_points;
        d.accumGlobals->numLeavesFolded += s_leaves;
    }
}

// Folds the plan's work items: each a kAccumChunk-point slice of one leaf's
// new range (partial sums added atomically into the leaf's exact sums; any
// order gives the same bits), or an inner node's sums cleared.
__global__ void __launch_bounds__(kAccumThreads, 4) k_accumulate(Dev d, uint32_t batchIndex, int useList) {
    __shared__ unsigned long long s_red[kNumSums][kAccumWarps];
    __shared__ unsigned long long s_morton[kAccumWarps];
    const Counters* c = d.ctr;
    const uint32_t total = useList ? (c->numDirty < d.maxNodes ? c->numDirty : d.maxNodes) : c->numNodes;
    const uint32_t items = c->accumItems;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t ppc = d.ppc;
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x) {
        // the node whose items hold this one: last w with accumItem[w] <= it
        uint32_t lo = 0, hi = total;
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (d.accumItem[mid] <= it) lo = mid;
            else hi = mid;
        }
        const uint32_t w = lo;
        const uint32_t node = useList ? d.dirtyList[w] : w;
        AccumI* a = &d.accum[node];
        const uint32_t from0 = d.accumFrom[w], to = d.accumTo[w];
        if (to == from0) {  // an inner node holding sums
            if (threadIdx.x == 0) {
                AccumI z = {};
                *a = z;
            }
            continue;
        }
        const uint32_t k0 = it - d.accumItem[w];
        const uint32_t from = from0 + k0 * kAccumChunk;
        const uint32_t end = min(to, from + kAccumChunk);
        const uint32_t lv = d.level[node];
        const uint32_t sh = 28u - lv;
        const long long lim = 1ll << sh;
        const long long bx = (long long)d.nodeX[node] << sh;
        const long long by = (long long)d.nodeY[node] << sh;
        const long long bz = (long long)d.nodeZ[node] << sh;
        const uint32_t toff = d.ptTableOff[node];

        // Per thread at most kAccumChunk / kAccumThreads = 16 points per item:
        // Σq < 2^32 · 16 needs u64, Σq·q < 16 · 2^56 fits u64 without carries,
        // colour sums fit u32; the 128-bit carries start at the warp reduction.
        unsigned long long s1[3] = {0, 0, 0};
        unsigned long long p2[6] = {0, 0, 0, 0, 0, 0};
        uint32_t c1[3] = {0, 0, 0}, c2[3] = {0, 0, 0};
        uint32_t mx = 0, my = 0, mz = 0;  // the largest point in Morton order so far
        for (uint32_t s0 = from + threadIdx.x; s0 < end; s0 += 2u * blockDim.x) {
            // two points per step: independent chunk-table and point loads in flight
            float4 v2[2];
            bool ok[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t s = s0 + (uint32_t)h * blockDim.x;
                ok[h] = false;
                if (s < end) {
                    const uint32_t phys = d.tablePool[toff + s / ppc];
                    if (phys != kNone) {
                        v2[h] = __ldg(reinterpret_cast<const float4*>(chunkPoints(d, phys) + s % ppc));
                        ok[h] = true;
                    }
                }
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (!ok[h]) continue;
                const float4 v = v2[h];
                const uint32_t P[3] = {aq(v.x, d.boxMin[0], d.octreeSize, 268435456.0f),
                                       aq(v.y, d.boxMin[1], d.octreeSize, 268435456.0f),
                                       aq(v.z, d.boxMin[2], d.octreeSize, 268435456.0f)};
                // clamped to [0, 2^(28 - level)]: 32-bit values, 64-bit products
                uint32_t q[3];
                const long long r[3] = {(long long)P[0] - bx, (long long)P[1] - by, (long long)P[2] - bz};
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    q[k] = (uint32_t)(r[k] < 0 ? 0 : (r[k] > lim ? lim : r[k]));
                    s1[k] += q[k];
                }
                p2[0] += (unsigned long long)q[0] * q[0];
                p2[1] += (unsigned long long)q[0] * q[1];
                p2[2] += (unsigned long long)q[0] * q[2];
                p2[3] += (unsigned long long)q[1] * q[1];
                p2[4] += (unsigned long long)q[1] * q[2];
                p2[5] += (unsigned long long)q[2] * q[2];
                const uint32_t col = __float_as_uint(v.w);
                const uint32_t ch[3] = {col & 255u, (col >> 8) & 255u, (col >> 16) & 255u};
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    c1[k] += ch[k];
                    c2[k] += ch[k] * ch[k];
                }
                // the 20-bit coordinate is the 28-bit one shifted (power-of-two scaling
                // commutes with round-to-nearest); only a saturated conversion differs
                uint32_t X = P[0] < 0xFFFFFF00u ? P[0] >> 8 : aq(v.x, d.boxMin[0], d.octreeSize, 1048576.0f);
                uint32_t Y = P[1] < 0xFFFFFF00u ? P[1] >> 8 : aq(v.y, d.boxMin[1], d.octreeSize, 1048576.0f);
                uint32_t Z = P[2] < 0xFFFFFF00u ? P[2] >> 8 : aq(v.z, d.boxMin[2], d.octreeSize, 1048576.0f);
                X = X < 1048575u ? X : 1048575u;
                Y = Y < 1048575u ? Y : 1048575u;
                Z = Z < 1048575u ? Z : 1048575u;
                if (mortonLess(mx, my, mz, X, Y, Z)) {
                    mx = X;
                    my = Y;
                    mz = Z;
                }
            }
        }
        unsigned long long wm = (mortonSpread(mx) << 2) | (mortonSpread(my) << 1) | mortonSpread(mz);
        unsigned long long lo2[6], hi2[6] = {0, 0, 0, 0, 0, 0};
        unsigned long long c1w[3], c2w[3];
#pragma unroll
        for (int k = 0; k < 6; k++) lo2[k] = p2[k];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            c1w[k] = c1[k];
            c2w[k] = c2[k];
        }
        // warp reduction
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                s1[k] += __shfl_down_sync(0xFFFFFFFFu, s1[k], off);
                c1w[k] += __shfl_down_sync(0xFFFFFFFFu, c1w[k], off);
                c2w[k] += __shfl_down_sync(0xFFFFFFFFu, c2w[k], off);
            }
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const unsigned long long ol = __shfl_down_sync(0xFFFFFFFFu, lo2[k], off);
                const unsigned long long oh = __shfl_down_sync(0xFFFFFFFFu, hi2[k], off);
                const unsigned long long nl = lo2[k] + ol;
                hi2[k] += oh + (nl < lo2[k] ? 1ull : 0ull);
                lo2[k] = nl;
            }
            const unsigned long long om = __shfl_down_sync(0xFFFFFFFFu, wm, off);
            wm = om > wm ? om : wm;
        }
        if (lane == 0) {
            for (int k = 0; k < 3; k++) {
                s_red[k][warp] = s1[k];
                s_red[15 + k][warp] = c1w[k];
                s_red[18 + k][warp] = c2w[k];
            }
            for (int k = 0; k < 6; k++) {
                s_red[3 + k][warp] = lo2[k];
                s_red[9 + k][warp] = hi2[k];
            }
            s_morton[warp] = wm;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long t1[3] = {0, 0, 0}, tc1[3] = {0, 0, 0}, tc2[3] = {0, 0, 0};
            unsigned long long tlo[6] = {0, 0, 0, 0, 0, 0}, thi[6] = {0, 0, 0, 0, 0, 0};
            unsigned long long m = 0;
            for (int w2 = 0; w2 < kAccumWarps; w2++) {
                for (int k = 0; k < 3; k++) {
                    t1[k] += s_red[k][w2];
                    tc1[k] += s_red[15 + k][w2];
                    tc2[k] += s_red[18 + k][w2];
                }
                for (int k = 0; k < 6; k++) {
                    thi[k] += s_red[9 + k][w2];
                    add128(tlo[k], thi[k], s_red[3 + k][w2]);
                }
                m = s_morton[w2] > m ? s_morton[w2] : m;
            }
            for (int k = 0; k < 3; k++) {
                atomicAdd(&a->s1[k], t1[k]);
                atomicAdd(&a->c1[k], tc1[k]);
                atomicAdd(&a->c2[k], tc2[k]);
            }
            for (int k = 0; k < 6; k++) atomicAdd128(&a->s2lo[k], &a->s2hi[k], tlo[k], thi[k]);
            // every item of a leaf writes the same watermark and batch
            a->count = to;
            a->lastTouchedBatch = batchIndex;
            atomicMax(&d.accumGlobals->mortonWatermark, m);
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
    k_accum_plan<<<1, 1024, 0, s>>>(d, useList);
    k_accumulate<<<grid, kAccumThreads, 0, s>>>(d, batchIndex, useList);
}
void launchAccumVerify(const Dev& d, int grid, cudaStream_t s) { k_accum_verify<<<grid, 256, 0, s>>>(d); }

}  // namespace rb
