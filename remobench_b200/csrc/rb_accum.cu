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

// 128-bit atomic add on a (lo, hi) pair: the add that wraps lo carries into hi.
__device__ __forceinline__ void atomicAdd128(unsigned long long* lo, unsigned long long* hi,
                                             unsigned long long vlo, unsigned long long vhi) {
    const unsigned long long old = atomicAdd(lo, vlo);
    const unsigned long long carry = (old + vlo < old) ? 1ull : 0ull;
    if (vhi + carry) atomicAdd(hi, vhi + carry);
}

// The fold's plan: the nodes to visit (the dirty list, or every node), each
// leaf's new range [count, min(numPoints, capacity)) read before any fold
// updates count, and each node's work items. An inner node with sums is one
// item (cleared); a leaf with new points one item per point chunk its new
// range touches. Sums are exact, so the order of items is free: each block
// claims a contiguous run of item indices with one atomic (Counters::
// accumItems, zeroed before the launch) and writes every item's plan entry,
// so a warp of the fold finds its item with one load. Items can pass
// accumUnitCap (every live point chunk plus every node) only once the arena
// has run out (RB_OVF_ARENA): those are not folded. Folded-leaf and point
// totals are added per block.
__global__ void __launch_bounds__(256) k_accum_plan(Dev d, int useList) {
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_base, s_leaves;
    __shared__ unsigned long long s_points;
    Counters* c = d.ctr;
    const uint32_t total = useList ? (c->numDirty < d.maxNodes ? c->numDirty : d.maxNodes) : c->numNodes;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_leaves = 0;
        s_points = 0;
    }
    __syncthreads();
    // the same number of steps in every thread of the block
    for (uint32_t w0 = blockIdx.x * blockDim.x; w0 < total; w0 += gridDim.x * blockDim.x) {
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
                    items = (to - 1u) / d.ppc - from / d.ppc + 1u;
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
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (uint32_t k = 0; k < blockDim.x / 32u; k++) {
                const uint32_t t = s_warp[k];
                s_warp[k] = run;
                run += t;
            }
            s_base = run ? atomicAdd(&c->accumItems, run) : 0u;
        }
        __syncthreads();
        const uint32_t first = s_base + s_warp[warp] + x - items;
        if (w < total) {
            d.accumItem[w] = first;
            for (uint32_t u = first; u < first + items && u < d.accumUnitCap; u++) d.accumUnitW[u] = w;
        }
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_leaves) {
        atomicAdd(&d.accumGlobals->numAccumulated, s_points);
        atomicAdd(&d.accumGlobals->pointsFolded, (uint32_t)s_points);
        atomicAdd(&d.accumGlobals->numLeavesFolded, s_leaves);
    }
}

// 128-bit sum of two (lo, hi) pairs.
__device__ __forceinline__ void add128pair(unsigned long long& lo, unsigned long long& hi, unsigned long long olo,
                                           unsigned long long ohi) {
    const unsigned long long nl = lo + olo;
    hi += ohi + (nl < lo ? 1ull : 0ull);
    lo = nl;
}

// Folds the plan's work items, one warp per item: an item is the part of one
// leaf's new range inside one point chunk (at most ppc points, one chunk-table
// read), its partial sums added atomically into the leaf's exact sums -- any
// order gives the same bits -- or an inner node's sums cleared. Lane k of the
// warp issues the atomic of sum k, so an item's 21 updates go out together.
// The watermark is merged per block in shared memory, one global atomic per
// block. Three blocks per SM (80 registers, a few bytes spilled) fold 9% faster
// than the two that 93 registers allow.
__global__ void __launch_bounds__(kAccumThreads, 3) k_accumulate(Dev d, uint32_t batchIndex, int useList) {
    __shared__ unsigned long long s_morton;
    const Counters* c = d.ctr;
    const uint32_t items = c->accumItems;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ppc = d.ppc;
    if (threadIdx.x == 0) s_morton = 0ull;
    __syncthreads();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long blockMax = 0ull;  // lane 0's running watermark
    for (uint32_t it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < items; it += warps) {
        if (it >= d.accumUnitCap) break;  // only past an arena overflow (see k_accum_plan)
        const uint32_t w = d.accumUnitW[it];
        const uint32_t node = useList ? d.dirtyList[w] : w;
        AccumI* a = &d.accum[node];
        const uint32_t from0 = d.accumFrom[w], to = d.accumTo[w];
        if (to == from0) {  // an inner node holding sums
            if (lane == 0) {
                AccumI z = {};
                *a = z;
            }
            continue;
        }
        const uint32_t ci = from0 / ppc + (it - d.accumItem[w]);
        const uint32_t from = from0 > ci * ppc ? from0 : ci * ppc;
        const uint32_t end = to < (ci + 1u) * ppc ? to : (ci + 1u) * ppc;
        const uint32_t lv = d.level[node];
        const uint32_t sh = 28u - lv;
        const long long lim = 1ll << sh;
        const long long bx = (long long)d.nodeX[node] << sh;
        const long long by = (long long)d.nodeY[node] << sh;
        const long long bz = (long long)d.nodeZ[node] << sh;
        const uint32_t phys = d.tablePool[d.ptTableOff[node] + ci];

        // Per lane at most ppc / 32 + 1 points: Σq < 2^28 · 32 needs u64, Σq·q <
        // 32 · 2^56 fits u64 without carries, colour sums fit u32; the 128-bit
        // carries start at the warp reduction.
        unsigned long long s1[3] = {0, 0, 0};
        unsigned long long p2[6] = {0, 0, 0, 0, 0, 0};
        uint32_t c1[3] = {0, 0, 0}, c2[3] = {0, 0, 0};
        uint32_t mx = 0, my = 0, mz = 0;  // the largest point in Morton order so far
        if (phys != kNone) {
            const float4* cp = reinterpret_cast<const float4*>(chunkPoints(d, phys));
            const uint32_t base = ci * ppc;
            for (uint32_t s0 = from + lane; s0 < end; s0 += 4u * 32u) {
                // four points per step: their loads in flight together
                float4 v4[4];
                bool ok[4];
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const uint32_t sidx = s0 + (uint32_t)h * 32u;
                    ok[h] = sidx < end;
                    if (ok[h]) v4[h] = __ldg(cp + (sidx - base));
                }
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    if (!ok[h]) continue;
                    const float4 v = v4[h];
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
        }
        // the warp's sums: 21 values (s1 x3, s2 lo/hi x6, c1 x3, c2 x3) and the watermark
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
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                s1[k] += __shfl_xor_sync(0xFFFFFFFFu, s1[k], off);
                c1w[k] += __shfl_xor_sync(0xFFFFFFFFu, c1w[k], off);
                c2w[k] += __shfl_xor_sync(0xFFFFFFFFu, c2w[k], off);
            }
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const unsigned long long ol = __shfl_xor_sync(0xFFFFFFFFu, lo2[k], off);
                const unsigned long long oh = __shfl_xor_sync(0xFFFFFFFFu, hi2[k], off);
                add128pair(lo2[k], hi2[k], ol, oh);
            }
            const unsigned long long om = __shfl_xor_sync(0xFFFFFFFFu, wm, off);
            wm = om > wm ? om : wm;
        }
        // every lane holds the totals: lane k issues sum k's atomic (values
        // picked by unrolled selects, so the arrays stay in registers)
        if (lane < 3u) {
            unsigned long long v1 = 0, vc1 = 0, vc2 = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                if (lane == (uint32_t)k) {
                    v1 = s1[k];
                    vc1 = c1w[k];
                    vc2 = c2w[k];
                }
            }
            atomicAdd(&a->s1[lane], v1);
            atomicAdd(&a->c1[lane], vc1);
            atomicAdd(&a->c2[lane], vc2);
        } else if (lane < 9u) {
            unsigned long long vlo = 0, vhi = 0;
#pragma unroll
            for (int k = 0; k < 6; k++) {
                if (lane == 3u + (uint32_t)k) {
                    vlo = lo2[k];
                    vhi = hi2[k];
                }
            }
            atomicAdd128(&a->s2lo[lane - 3u], &a->s2hi[lane - 3u], vlo, vhi);
        } else if (lane == 9u) {
            // every item of a leaf writes the same watermark and batch
            a->count = to;
            a->lastTouchedBatch = batchIndex;
        }
        if (wm > blockMax) blockMax = wm;
    }
    if (lane == 0 && blockMax != 0ull) atomicMax(&s_morton, blockMax);
    __syncthreads();
    if (threadIdx.x == 0 && s_morton != 0ull) atomicMax(&d.accumGlobals->mortonWatermark, s_morton);
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
    cudaMemsetAsync(&d.ctr->accumItems, 0, sizeof(uint32_t), s);
    k_accum_plan<<<grid, 256, 0, s>>>(d, useList);
    k_accumulate<<<grid, kAccumThreads, 0, s>>>(d, batchIndex, useList);
}
void launchAccumVerify(const Dev& d, int grid, cudaStream_t s) { k_accum_verify<<<grid, 256, 0, s>>>(d); }

}  // namespace rb
