// Refinement's colour filtering (wiki/02_KernelPipeline.md:228-243: "average
// colour across a node's samples", listed by the reference and not built
// there): a voxel's colour becomes the mean colour of the points below its
// node that fall in its cell, instead of one representative point's.
//
// The reference's notes rule out a dense per-node colour grid (128^3 RGBA
// sums would be ~16 MB per node) and ask for a sparse accumulator keyed off
// the voxels. Here the accumulator has one entry per voxel being filtered,
// found through a table keyed by (filtered node, cell):
//   k_cf_plan   the queue prefix whose voxels fit the capacity, each node's
//               first entry (one block);
//   k_cf_index  every entry's cell from its voxel's centre into the table;
//   k_cf_gather one block per leaf below a filtered node: each point adds its
//               colour to the entry of its cell in every filtered ancestor;
//   k_cf_apply  means (rounded half up, alpha kept) written into the voxels,
//               the table and the node marks cleared for the next call.
// Integer sums: the result does not depend on the order points arrive in.
#include <cuda_runtime.h>

#include "rb_kernels.h"
#include "rb_refine.h"
#include "rb_state.h"

namespace rb {

namespace {

__device__ __forceinline__ uint32_t quant28r(float c, float mn, float size) {
    const float d = __fsub_rn(c, mn);
    return __float2uint_rz(__fdiv_rn(__fmul_rn(268435456.0f, d), size));
}

__device__ __forceinline__ uint32_t cellOf(uint32_t x28, uint32_t y28, uint32_t z28, uint32_t level) {
    const uint32_t sh = (uint32_t)kMaxDepth + 1u - level;
    return ((x28 >> sh) & 127u) + ((y28 >> sh) & 127u) * 128u + ((z28 >> sh) & 127u) * 16384u;
}

__device__ __forceinline__ uint32_t slotOf(unsigned long long key, uint32_t mask) {
    unsigned long long h = key * 0x9E3779B97F4A7C15ull;
    h ^= h >> 31;
    return (uint32_t)h & mask;
}

// The cell a voxel of node `node` stands for, from its centre
// nodeMin + size (c + 0.5) / 128 (half a cell from either boundary).
__device__ __forceinline__ uint32_t voxelCell(const Dev& d, uint32_t node, const Point& v) {
    const float size = __fdiv_rn(d.octreeSize, __int_as_float((int)((127u + d.level[node]) << 23)));
    const float scale = __fdiv_rn(128.0f, size);
    const float mn[3] = {__fmaf_rn((float)d.nodeX[node], size, d.boxMin[0]),
                         __fmaf_rn((float)d.nodeY[node], size, d.boxMin[1]),
                         __fmaf_rn((float)d.nodeZ[node], size, d.boxMin[2])};
    const float pv[3] = {v.x, v.y, v.z};
    uint32_t c[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int q = __float2int_rd(__fmul_rn(__fsub_rn(pv[a], mn[a]), scale));
        c[a] = (uint32_t)min(max(q, 0), 127);
    }
    return c[0] + 128u * c[1] + 16384u * c[2];
}

__global__ void __launch_bounds__(1024) k_cf_plan(Dev d, RefineScratch r, const uint32_t* queue, uint32_t queueLen,
                                                  uint32_t budget) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_run, s_stop;
    const uint32_t n = queueLen < budget ? queueLen : budget;
    if (threadIdx.x == 0) {
        s_run = 0;
        s_stop = n;
    }
    __syncthreads();
    for (uint32_t k0 = 0; k0 < n; k0 += blockDim.x) {
        const uint32_t k = k0 + threadIdx.x;
        uint32_t nv = 0, node = 0;
        if (k < n) {
            node = queue[k];
            nv = d.numVoxels[node];
            const uint32_t stored = d.numVoxelsStored[node], cap = d.numVoxelChunks[node] * d.ppc;
            nv = nv < stored ? nv : stored;
            nv = nv < cap ? nv : cap;
        }
        uint32_t tot;
        const uint32_t pre = blockExclusiveScanRefine(nv, &tot, s_warp);
        const uint32_t base = s_run + pre;
        // the prefix that fits: every node whose voxels end within the capacity
        if (k < n && base + nv > r.capacity) atomicMin(&s_stop, k);
        __syncthreads();
        if (k < n && k < s_stop) {
            r.voxNode[k] = node;
            r.voxBase[k] = base;
            r.refSlot[node] = k;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_run += tot;
        __syncthreads();
        if (s_stop < n) break;
    }
    if (threadIdx.x == 0) {
        const uint32_t m = s_stop;
        uint32_t total = 0;
        if (m > 0) {
            const uint32_t last = r.voxNode[m - 1];
            uint32_t nv = d.numVoxels[last];
            const uint32_t stored = d.numVoxelsStored[last], cap = d.numVoxelChunks[last] * d.ppc;
            nv = nv < stored ? nv : stored;
            nv = nv < cap ? nv : cap;
            total = r.voxBase[m - 1] + nv;
        }
        r.voxBase[m] = total;
        r.ctr->nodes = m;
        r.ctr->voxels = total;
        r.ctr->points = 0;
    }
}

__global__ void __launch_bounds__(256) k_cf_index(Dev d, RefineScratch r) {
    const uint32_t nodes = r.ctr->nodes, total = r.ctr->voxels;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nodes;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (r.voxBase[mid] <= e) lo = mid;
            else hi = mid;
        }
        const uint32_t node = r.voxNode[lo], s = e - r.voxBase[lo];
        const uint32_t phys = d.tablePool[d.vxTableOff[node] + s / d.ppc];
        Point v = {0.f, 0.f, 0.f, 0u};
        if (phys != kNone) v = reinterpret_cast<const Point*>(d.arena + (uint64_t)phys * 16u)[s % d.ppc];
        const unsigned long long key = ((unsigned long long)lo << 21) | voxelCell(d, node, v);
        r.acc[e] = make_ulonglong4(0ull, 0ull, 0ull, 0ull);
        r.entrySlot[e] = kNone;
        if (phys == kNone) continue;
        uint32_t slot = slotOf(key, r.hashMask);
        for (uint32_t probe = 0; probe <= r.hashMask; probe++) {
            const unsigned long long prev = atomicCAS(&r.hashKeys[slot], ~0ull, key);
            if (prev == ~0ull) {
                r.hashVals[slot] = e;
                r.entrySlot[e] = slot;
                break;
            }
            if (prev == key) break;  // one voxel per cell: not reached
            slot = (slot + 1u) & r.hashMask;
        }
    }
}

__device__ __forceinline__ uint32_t findEntry(const RefineScratch& r, unsigned long long key) {
    uint32_t slot = slotOf(key, r.hashMask);
    for (uint32_t probe = 0; probe <= r.hashMask; probe++) {
        const unsigned long long k = r.hashKeys[slot];
        if (k == key) return r.hashVals[slot];
        if (k == ~0ull) return kNone;
        slot = (slot + 1u) & r.hashMask;
    }
    return kNone;
}

// One block per leaf (grid-stride over the node pool); leaves with no
// filtered ancestor return at once.
__global__ void __launch_bounds__(256) k_cf_gather(Dev d, RefineScratch r) {
    __shared__ uint32_t s_slot[kMaxDepth + 1], s_lv[kMaxDepth + 1];
    __shared__ uint32_t s_n;
    const uint32_t nn = d.ctr->numNodes;
    const uint32_t ppc = d.ppc;
    unsigned long long visited = 0;
    for (uint32_t leaf = blockIdx.x; leaf < nn; leaf += gridDim.x) {
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t m = 0;
            const uint32_t lv = d.level[leaf];
            const int4* row = reinterpret_cast<const int4*>(d.child + leaf * 8u);
            const int4 a = row[0], b = row[1];
            const bool isLeaf = (a.x & a.y & a.z & a.w & b.x & b.y & b.z & b.w) == -1;
            if (isLeaf && d.numPoints[leaf] > 0) {
                for (uint32_t l = 0; l < lv && l < (uint32_t)kMaxDepth; l++) {
                    const uint32_t anc = d.anc[(size_t)leaf * kMaxDepth + l].x;
                    const uint32_t k = r.refSlot[anc];
                    if (k != kNone) {
                        s_slot[m] = k;
                        s_lv[m] = l;
                        m++;
                    }
                }
                // a filtered leaf's own points (a root that never split keeps voxels)
                const uint32_t k = r.refSlot[leaf];
                if (k != kNone) {
                    s_slot[m] = k;
                    s_lv[m] = lv;
                    m++;
                }
            }
            s_n = m;
        }
        __syncthreads();
        const uint32_t m = s_n;
        if (m == 0) continue;
        uint32_t np = d.numPoints[leaf];
        const uint32_t cap = d.numPointChunks[leaf] * ppc;
        np = np < cap ? np : cap;
        const uint32_t off = d.ptTableOff[leaf];
        for (uint32_t s = threadIdx.x; s < np; s += blockDim.x) {
            const uint32_t phys = d.tablePool[off + s / ppc];
            if (phys == kNone) continue;
            const Point p = reinterpret_cast<const Point*>(d.arena + (uint64_t)phys * 16u)[s % ppc];
            const uint32_t x = quant28r(p.x, d.boxMin[0], d.octreeSize), y = quant28r(p.y, d.boxMin[1], d.octreeSize),
                           z = quant28r(p.z, d.boxMin[2], d.octreeSize);
            for (uint32_t j = 0; j < m; j++) {
                const unsigned long long key = ((unsigned long long)s_slot[j] << 21) | cellOf(x, y, z, s_lv[j]);
                const uint32_t e = findEntry(r, key);
                visited++;
                if (e == kNone) continue;
                atomicAdd(&r.acc[e].x, (unsigned long long)(p.color & 255u));
                atomicAdd(&r.acc[e].y, (unsigned long long)((p.color >> 8) & 255u));
                atomicAdd(&r.acc[e].z, (unsigned long long)((p.color >> 16) & 255u));
                atomicAdd(&r.acc[e].w, 1ull);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) visited += __shfl_xor_sync(0xFFFFFFFFu, visited, o);
    if ((threadIdx.x & 31u) == 0 && visited) atomicAdd(&r.ctr->points, visited);
}

__global__ void __launch_bounds__(256) k_cf_apply(Dev d, RefineScratch r) {
    const uint32_t nodes = r.ctr->nodes, total = r.ctr->voxels;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nodes;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (r.voxBase[mid] <= e) lo = mid;
            else hi = mid;
        }
        const uint32_t node = r.voxNode[lo], s = e - r.voxBase[lo];
        const ulonglong4 a = r.acc[e];
        const uint32_t phys = d.tablePool[d.vxTableOff[node] + s / d.ppc];
        if (a.w > 0 && phys != kNone) {
            Point* v = reinterpret_cast<Point*>(d.arena + (uint64_t)phys * 16u) + s % d.ppc;
            const unsigned long long half = a.w / 2u;
            const uint32_t cr = (uint32_t)((a.x + half) / a.w), cg = (uint32_t)((a.y + half) / a.w),
                           cb = (uint32_t)((a.z + half) / a.w);
            v->color = (v->color & 0xFF000000u) | cr | (cg << 8) | (cb << 16);
        }
        if (r.entrySlot[e] != kNone) r.hashKeys[r.entrySlot[e]] = ~0ull;
    }
    // every planned node's mark, voxels or not, for the next call
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nodes; k += gridDim.x * blockDim.x)
        r.refSlot[r.voxNode[k]] = kNone;
}

}  // namespace

__device__ uint32_t blockExclusiveScanRefine(uint32_t v, uint32_t* total, uint32_t* s_warp) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t prefix = (warp > 0 ? s_warp[warp - 1] : 0u) + x - v;
    *total = s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return prefix;
}

void launchRefineColors(const Dev& d, const RefineScratch& r, const uint32_t* queue, uint32_t queueLen,
                        uint32_t budget, int grid, cudaStream_t s) {
    k_cf_plan<<<1, 1024, 0, s>>>(d, r, queue, queueLen, budget);
    k_cf_index<<<grid, 256, 0, s>>>(d, r);
    k_cf_gather<<<grid, 256, 0, s>>>(d, r);
    k_cf_apply<<<grid, 256, 0, s>>>(d, r);
}

}  // namespace rb
