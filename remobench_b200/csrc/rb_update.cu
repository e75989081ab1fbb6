// Update stage: count -> split -> make room -> 128^3 voxel sampling -> chunk
// acquisition -> point and voxel insertion, one batch at a time.
//
// Restates kernels/remolod/remolod_octree.cu:95-1060 (addBatch and its phases)
// as phase kernels on one stream. Every kernel here is plain SIMT integer work
// bound by latency and L2 atomics, not by tensor cores; see the per-kernel
// notes for what each reads and writes.
//
// Parity-critical float arithmetic (quantisation, voxel centres) uses the
// explicitly rounded intrinsics (__fsub_rn, __fmul_rn, __fdiv_rn, __fmaf_rn),
// so nvcc cannot contract or approximate it; the CPU oracle performs the same
// operations in the same order.
#include <cuda_runtime.h>

#include <cstring>

#include "rb_kernels.h"
#include "rb_state.h"

namespace rb {

__device__ __forceinline__ uint32_t quant20(float c, float mn, float size) {
    float d = __fsub_rn(c, mn);
    return __float2uint_rz(__fdiv_rn(__fmul_rn(1048576.0f, d), size));
}

__device__ __forceinline__ uint32_t quant28(float c, float mn, float size) {
    float d = __fsub_rn(c, mn);
    return __float2uint_rz(__fdiv_rn(__fmul_rn(268435456.0f, d), size));
}

__device__ __forceinline__ Point loadPoint(const Point* p) {
    float4 v = __ldg(reinterpret_cast<const float4*>(p));
    Point q;
    q.x = v.x;
    q.y = v.y;
    q.z = v.z;
    q.color = __float_as_uint(v.w);
    return q;
}

__device__ __forceinline__ uint32_t childIndex(uint32_t x, uint32_t y, uint32_t z, uint32_t level) {
    const uint32_t s = kMaxDepth - level - 1;
    return (((x >> s) & 1u) << 2) | (((y >> s) & 1u) << 1) | ((z >> s) & 1u);
}

// remolod_octree.cu:182-201: at most kMaxDepth steps from the root.
__device__ __forceinline__ uint32_t descendFromRoot(const Dev& d, uint32_t x, uint32_t y, uint32_t z) {
    uint32_t cur = 0;
    for (uint32_t level = 0; level < (uint32_t)kMaxDepth; level++) {
        int32_t c = __ldg(&d.child[cur * 8u + childIndex(x, y, z, level)]);
        if (c < 0) break;
        cur = (uint32_t)c;
    }
    return cur;
}

__device__ __forceinline__ uint32_t laneId() { return threadIdx.x & 31u; }

// Warp-aggregated count at a leaf (remolod_octree.cu:203-220). Every lane of
// the warp must call it; lanes with nothing to count pass kNone.
__device__ __forceinline__ void countAt(const Dev& d, uint32_t leaf) {
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, leaf);
    if (leaf == kNone) return;
    if ((int)laneId() != __ffs(peers) - 1) return;
    const uint32_t g = __popc(peers);
    const uint32_t old = atomicAdd(&d.counter[leaf], g);
    if (old <= d.maxPointsPerNode && old + g > d.maxPointsPerNode) {
        const uint32_t k = atomicAdd(&d.ctr->numSpill, 1u);
        if (k < d.spillingCap) d.spillNodes[k] = leaf;
        else atomicOr(&d.ctr->overflowFlags, (uint32_t)kOvfSpilling);
    }
}

__device__ __forceinline__ unsigned long long globalTimerNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Batch start (kernel_construct's loop head, remolod_octree.cu:1190-1240): the
// memory check, and for device-driven builds the batch cursor -- which slot
// holds batch batchletIndex and how many points it has -- and the call's time
// budget. A stopped batch leaves every later phase kernel a no-op.
// Adds g points to a leaf's counter and lists the leaf when its count first
// passes the split limit (the same test as countAt).
__device__ __forceinline__ void addCount(const Dev& d, uint32_t leaf, uint32_t g) {
    const uint32_t old = atomicAdd(&d.counter[leaf], g);
    if (old <= d.maxPointsPerNode && old + g > d.maxPointsPerNode) {
        const uint32_t k = atomicAdd(&d.ctr->numSpill, 1u);
        if (k < d.spillingCap) d.spillNodes[k] = leaf;
        else atomicOr(&d.ctr->overflowFlags, (uint32_t)kOvfSpilling);
    }
}

// Block-level counting: the points of one block's contiguous range fall into
// a handful of leaves, so counts are merged per block in shared memory and
// each leaf's counter takes one atomic per block instead of one per warp (a
// few hot counters otherwise serialise thousands of atomics). The final sums
// and the set of leaves crossing the limit are the same.
constexpr uint32_t kBlockLeaves = 64;

struct BlockCounts {
    uint32_t leaf[kBlockLeaves];
    uint32_t cnt[kBlockLeaves];
};

__device__ __forceinline__ void blockCountsInit(BlockCounts& b) {
    for (uint32_t t = threadIdx.x; t < kBlockLeaves; t += blockDim.x) {
        b.leaf[t] = kNone;
        b.cnt[t] = 0;
    }
}

// Every lane of the warp calls it; lanes with nothing to count pass kNone.
// hist: key is a child-octant bin (node * 8 + octant) of hist8, which takes
// plain additions; otherwise key is a leaf whose counter is bumped.
template <bool hist>
__device__ __forceinline__ void blockCountAt(const Dev& d, BlockCounts& b, uint32_t leaf) {
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, leaf);
    if (leaf == kNone || (int)laneId() != __ffs(peers) - 1) return;
    const uint32_t g = __popc(peers);
    uint32_t slot = (leaf * 0x9E3779B1u) >> 26;
    for (uint32_t probe = 0; probe < 8u; probe++) {
        const uint32_t cur = atomicCAS(&b.leaf[slot], kNone, leaf);
        if (cur == kNone || cur == leaf) {
            atomicAdd(&b.cnt[slot], g);
            return;
        }
        slot = (slot + 1u) & (kBlockLeaves - 1u);
    }
    // crowded table: count globally
    if (hist) atomicAdd(&d.hist8[leaf], g);
    else addCount(d, leaf, g);
}

// After a barrier: the block's sums into the leaves' counters (or hist8).
template <bool hist>
__device__ __forceinline__ void blockCountsFlush(const Dev& d, BlockCounts& b) {
    for (uint32_t t = threadIdx.x; t < kBlockLeaves; t += blockDim.x) {
        if (b.leaf[t] == kNone || b.cnt[t] == 0u) continue;
        if (hist) atomicAdd(&d.hist8[b.leaf[t]], b.cnt[t]);
        else addCount(d, b.leaf[t], b.cnt[t]);
    }
}

// Block-level slot reservation: each item takes the next slot of its key's
// counter (a leaf's point count, a node's voxel count). Items of one block
// merge per key in shared memory, so each key's counter takes one atomic per
// block and pass instead of one per warp. Every thread of the block calls it
// with its key (kNone: no item); it returns the item's slot.
struct BlockSlots {
    uint32_t key[kBlockLeaves];
    uint32_t cnt[kBlockLeaves];
    uint32_t base[kBlockLeaves];
};

__device__ __forceinline__ void blockSlotsInit(BlockSlots& b) {
    for (uint32_t t = threadIdx.x; t < kBlockLeaves; t += blockDim.x) {
        b.key[t] = kNone;
        b.cnt[t] = 0;
    }
}

__device__ __forceinline__ uint32_t blockReserve(BlockSlots& b, uint32_t* counters, uint32_t key) {
    const uint32_t lane = laneId();
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
    const int leader = __ffs(peers) - 1;
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    uint32_t s = kNone, off = 0;
    if (key != kNone && (int)lane == leader) {
        const uint32_t g = __popc(peers);
        uint32_t h = (key * 0x9E3779B1u) >> 26;
        for (uint32_t probe = 0; probe < 8u; probe++) {
            const uint32_t cur = atomicCAS(&b.key[h], kNone, key);
            if (cur == kNone || cur == key) {
                s = h;
                off = atomicAdd(&b.cnt[h], g);
                break;
            }
            h = (h + 1u) & (kBlockLeaves - 1u);
        }
        if (s == kNone) off = atomicAdd(&counters[key], g);  // crowded table: reserve globally
    }
    s = __shfl_sync(0xFFFFFFFFu, s, leader);
    off = __shfl_sync(0xFFFFFFFFu, off, leader);
    __syncthreads();
    // one global reservation per key; the table empties for the next pass
    // (the next pass writes base only after its own first barrier)
    for (uint32_t t = threadIdx.x; t < kBlockLeaves; t += blockDim.x) {
        if (b.key[t] != kNone) b.base[t] = atomicAdd(&counters[b.key[t]], b.cnt[t]);
        b.key[t] = kNone;
        b.cnt[t] = 0;
    }
    __syncthreads();
    return key == kNone ? kNone : (s != kNone ? b.base[s] : 0u) + off + rank;
}

__device__ __forceinline__ void resetBatchCounters(Counters* c);

__global__ void k_batch_begin(Dev d, uint32_t fromRing) {
    Counters* c = d.ctr;
    uint32_t reason = 0;
    if (fromRing) {
        const RingDesc* r = d.ring;
        const uint32_t b = c->batchletIndex;
        if (b >= r->numUploaded) {
            reason = kStopNoBatch;
        } else {
            uint32_t slot, n;
            if (r->streamMode) {
                const uint32_t rel = b - r->first;
                const unsigned long long off = (unsigned long long)rel * r->batchSize;
                slot = rel % r->numSlots;
                n = off < r->total ? (uint32_t)min((unsigned long long)r->batchSize, r->total - off) : 0u;
            } else {
                slot = b % r->numSlots;
                n = r->sizes[slot < kMaxRingSlots ? slot : 0u];
            }
            if (n > r->slotCap) n = r->slotCap;
            c->curPts = r->base + (unsigned long long)slot * r->slotCap * sizeof(Point);
            c->curN = n;
        }
    }
    if (reason == 0 && c->refOffset + d.safetyMargin >= d.persistentCapacity) reason = kStopMemory;
    // the budget is checked between batches: a call always builds its first batch
    if (reason == 0 && fromRing && d.ring->budgetNs != 0ull && c->callBatches > 0u &&
        globalTimerNs() - c->buildStartNs > d.ring->budgetNs)
        reason = kStopTime;
    if (reason == kStopMemory) c->memCapacityReached = 1u;
    else if (reason == 0) c->memCapacityReached = 0u;
    c->batchStop = reason ? 1u : 0u;
    c->stopReason = reason;
    resetBatchCounters(c);
}

// The per-batch state every batch (and a deepening pass) starts from.
__device__ __forceinline__ void resetBatchCounters(Counters* c) {
    c->numSpill = 0;
    c->numSpilled = 0;
    c->numNew = 0;
    c->numLift = 0;
    c->levelMode = c->gridsPartial;
    c->numSplit = 0;
    c->spillChunkTotal = 0;
    c->iter = 1;
    c->expandGuard = 0;
    c->numZero = 0;
    c->histValid = 0;
    c->countLo = 0;
    c->countHi = 0;
    c->hashNeedsClear = 0;  // the last batch's k_vox_store emptied the table
    c->deepActive = 0;
    c->deepRoots = 0;
    c->barArrive = 0;
    c->barRelease = 0;
}

// Iteration 1 of expand (doCounting over the batch, remolod_octree.cu:225-229):
// descend every batch point, remember its leaf, count it there.
// pts == nullptr: the batch at the device cursor (Counters::curPts / curN).
#define RB_BATCH_AT_CURSOR(d, pts, n)                                   \
    do {                                                                \
        if ((pts) == nullptr) {                                         \
            (pts) = reinterpret_cast<const Point*>((d).ctr->curPts);    \
            (n) = (d).ctr->curN;                                        \
        }                                                               \
    } while (0)

// Each block takes one contiguous, warp-aligned range of the batch.
__global__ void __launch_bounds__(256) k_count_first(Dev d, const Point* __restrict__ pts, uint32_t n) {
    __shared__ BlockCounts s_counts;
    if (d.ctr->batchStop) return;
    RB_BATCH_AT_CURSOR(d, pts, n);
    blockCountsInit(s_counts);
    __syncthreads();
    const uint32_t per = (((n + gridDim.x - 1u) / gridDim.x) + 31u) & ~31u;
    const uint32_t begin = min(n, blockIdx.x * per), end = min(n, begin + per);
    for (uint32_t base = begin; base < end; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t leaf = kNone;
        if (i < end) {
            const Point p = loadPoint(pts + i);
            leaf = descendFromRoot(d, quant20(p.x, d.boxMin[0], d.octreeSize),
                                   quant20(p.y, d.boxMin[1], d.octreeSize),
                                   quant20(p.z, d.boxMin[2], d.octreeSize));
            d.leafOf[i] = leaf;
        }
        blockCountAt<false>(d, s_counts, leaf);
    }
    __syncthreads();
    blockCountsFlush<false>(d, s_counts);
}

// Iterations 2.. of expand. The reference re-descends every batch and spilled
// point from the root and counts only at leaves created by the last split
// (countIteration, remolod_octree.cu:203). A point can only reach such a leaf
// if its own leaf was split, so only those points move, from the leaf they
// were in, through the nodes the last split made (one or two levels, see
// k_split); the counts that result are the same.
//
// Points reaching a node in [countLo, countHi) (the deepest nodes the split
// made) are counted per child octant into hist8: k_expand_cond sums a node's
// eight bins into its counter and lists the nodes over the limit, and the next
// split reads the bins to split the spilling nodes' spilling children in the
// same launch.
//
// prevStamp == 0: device-driven; the stamp of the last split's first round,
// and no counting (only moving) once the pass limit is reached.
__device__ __forceinline__ void recountBody(const Dev& d, const Point* __restrict__ pts, uint32_t n,
                                            uint32_t prevStamp, uint32_t gated) {
    Counters* c = d.ctr;
    if (c->batchStop || (gated && c->loopMore == 0u)) return;
    // Past the pass limit the loop counts no more (the nodes the last split
    // made keep counter 0), but points still move to their leaves: insertion
    // stores a point in the leaf the finished tree gives it.
    bool counting = true;
    if (prevStamp == 0u) {
        counting = c->iter <= d.maxExpandIters;
        prevStamp = c->lastStamp;
    }
    RB_BATCH_AT_CURSOR(d, pts, n);
    __shared__ BlockCounts s_counts;
    blockCountsInit(s_counts);
    __syncthreads();
    const uint32_t lo = c->countLo, hi = c->countHi;
    const uint32_t ns = c->numSpilled < d.spillCap ? c->numSpilled : d.spillCap;
    const uint32_t total = n + ns;
    const uint32_t per = (((total + gridDim.x - 1u) / gridDim.x) + 31u) & ~31u;
    const uint32_t begin = min(total, blockIdx.x * per), end = min(total, begin + per);
    for (uint32_t base = begin; base < end; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t bin = kNone;
        if (i < end) {
            const bool batchPt = i < n;
            uint32_t cur = batchPt ? d.leafOf[i] : d.spillLeaf[i - n];
            if (d.splitIter[cur] == prevStamp) {
                const Point p = batchPt ? loadPoint(pts + i) : d.spillPts[i - n];
                const uint32_t x = quant20(p.x, d.boxMin[0], d.octreeSize),
                               y = quant20(p.y, d.boxMin[1], d.octreeSize),
                               z = quant20(p.z, d.boxMin[2], d.octreeSize);
                uint32_t lv = d.level[cur];
                while (lv < (uint32_t)kMaxDepth) {
                    const int32_t nx = d.child[cur * 8u + childIndex(x, y, z, lv)];
                    if (nx < 0) break;
                    cur = (uint32_t)nx;
                    lv += 1u;
                }
                if (batchPt) d.leafOf[i] = cur;
                else d.spillLeaf[i - n] = cur;
                if (counting && cur >= lo && cur < hi)
                    bin = cur * 8u + (lv < (uint32_t)kMaxDepth ? childIndex(x, y, z, lv) : 0u);
            }
        }
        if (__any_sync(0xFFFFFFFFu, bin != kNone)) blockCountAt<true>(d, s_counts, bin);
    }
    __syncthreads();
    blockCountsFlush<true>(d, s_counts);
}

__global__ void __launch_bounds__(256) k_recount(Dev d, const Point* __restrict__ pts, uint32_t n,
                                                 uint32_t prevStamp, uint32_t gated) {
    recountBody(d, pts, n, prevStamp, gated);
}

// Block-wide exclusive scan of one value per thread (blockDim.x == 1024).
__device__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* total, uint32_t* s_warp) {
    const uint32_t lane = laneId(), warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
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

// The expand loop's test, after each count. After a recount it turns the
// child-octant bins of the nodes in [countLo, countHi) into their counters and
// lists those over the limit, in increasing id (doCounting's spilling nodes,
// remolod_octree.cu:213-218); after the first count the crossing list stands.
// Device-driven builds (h != 0) set the loop's condition: another pass while
// nodes spill, at most 40 passes (max_expand_iters <= 31 are needed).
// One block of 1024 threads.
__device__ __forceinline__ void expandCondBody(const Dev& d, cudaGraphConditionalHandle h, uint32_t gated) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_run;
    Counters* c = d.ctr;
    // a pass after the loop ended: keep it ended (every thread reads the flag
    // before the barrier after which thread 0 rewrites it)
    if (gated && c->loopMore == 0u) {
        if (threadIdx.x == 0) {
            c->condSkips++;
            if (h != 0ull) cudaGraphSetConditional(h, 0u);
        }
        return;
    }
    const uint32_t lo = c->countLo, hi = c->countHi;
    const bool stop = c->batchStop != 0u;
    if (threadIdx.x == 0) s_run = 0;
    __syncthreads();
    if (!stop && hi > lo) {
        for (uint32_t f0 = lo; f0 < hi; f0 += blockDim.x) {
            const uint32_t f = f0 + threadIdx.x;
            uint32_t spill = 0;
            if (f < hi) {
                const uint4* hb = reinterpret_cast<const uint4*>(d.hist8 + (size_t)f * 8u);
                const uint4 a = hb[0], b = hb[1];
                const uint32_t cnt = a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
                d.counter[f] = cnt;
                spill = cnt > d.maxPointsPerNode ? 1u : 0u;
            }
            uint32_t tot;
            const uint32_t pre = blockExclusiveScan(spill, &tot, s_warp);
            if (spill && s_run + pre < d.spillingCap) d.spillNodes[s_run + pre] = f;
            __syncthreads();
            if (threadIdx.x == 0) s_run += tot;
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        if (!stop && hi > lo) {
            uint32_t ns = s_run;
            if (ns > d.spillingCap) {
                atomicOr(&c->overflowFlags, (uint32_t)kOvfSpilling);
                ns = d.spillingCap;
            }
            c->numSpill = ns;
            c->histValid = 1u;  // the listed nodes' bins are their children's counts
            c->countLo = 0;
            c->countHi = 0;
        }
        c->condRuns++;
        const uint32_t g = ++c->expandGuard;
        const bool more = !stop && c->numSpill > 0u && g <= 40u;
        c->loopMore = more ? 1u : 0u;
        if (h != 0ull) cudaGraphSetConditional(h, more ? 1u : 0u);
    }
}

__global__ void __launch_bounds__(1024) k_expand_cond(Dev d, cudaGraphConditionalHandle h, uint32_t gated) {
    expandCondBody(d, h, gated);
}

// Ascending bitonic sort of n ids in place (single block); pads with kNone.
__device__ void bitonicSort(uint32_t* a, uint32_t n) {
    uint32_t m = 1;
    while (m < n) m <<= 1;
    for (uint32_t i = n + threadIdx.x; i < m; i += blockDim.x) a[i] = kNone;
    __syncthreads();
    for (uint32_t k = 2; k <= m; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint32_t ai = a[i], al = a[l];
                    const bool up = (i & k) == 0;
                    if ((ai > al) == up) {
                        a[i] = al;
                        a[l] = ai;
                    }
                }
            }
            __syncthreads();
        }
    }
}

constexpr uint32_t kSortSmem = 8192;

// per split node, for its children (the first kSplitInfo nodes of a pass)
struct SplitInfo {
    uint32_t node, lv, X, Y, Z, grid;
};
constexpr uint32_t kSplitInfo = 512;

// Ascending bitonic sort of one value per lane.
__device__ __forceinline__ uint32_t warpSortAscending(uint32_t v) {
    const uint32_t lane = laneId();
#pragma unroll
    for (uint32_t k = 2; k <= 32u; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = __shfl_xor_sync(0xFFFFFFFFu, v, j);
            const bool keepMin = ((lane & j) == 0u) == ((lane & k) == 0u);
            v = keepMin ? min(v, o) : max(v, o);
        }
    }
    return v;
}

// A grid for a node that splits: one a collapsed node returned (already
// charged to the store), else a new one from the arena, charged as the
// reference's allocator charges it. Pool grids are zeroed with the others.
__device__ __forceinline__ uint32_t takeGrid(const Dev& d, Counters* c) {
    atomicAdd(&c->numGrids, 1u);
    // the pool's size changes only between batches
    const uint32_t pool = c->gridPoolSize;
    if (pool != 0u) {
        const uint32_t k = atomicAdd(&c->gridPoolTaken, 1u);
        if (k < pool) return d.gridPool[pool - 1u - k];
    }
    atomicAdd(reinterpret_cast<unsigned long long*>(&c->refOffset), (unsigned long long)refAllocSize(kGridBytes));
    return arenaAlloc(d, kGridUnits);
}

// The pool after a batch: the grids its splits took are gone from it.
__device__ __forceinline__ void settleGridPool(Counters* c) {
    const uint32_t t = c->gridPoolTaken < c->gridPoolSize ? c->gridPoolTaken : c->gridPoolSize;
    c->gridPoolSize -= t;
    c->gridPoolTaken = 0;
}

// The bookkeeping of the k-th split node of a pass (remolod_octree.cu:303-400):
// its grid, its split stamp, its record for the spill copy (spill slots and
// copy items from the given prefixes), its chunks' queue positions, the grid
// to zero, the dirty list; its fields for the children phase.
__device__ __forceinline__ void splitBook(const Dev& d, Counters* c, uint32_t k, uint32_t node, uint32_t np,
                                          uint32_t owned, uint32_t spillBase, uint32_t chunkBase, uint32_t stamp,
                                          SplitInfo* s_info) {
    uint32_t g = d.grid[node];
    if (g == kNone) {
        g = takeGrid(d, c);
        d.grid[node] = g;
    }
    d.splitIter[node] = stamp;
    SplitRec r;
    r.node = node;
    r.numPoints = np;
    r.tableOff = d.ptTableOff[node];
    r.spillBase = spillBase;
    r.chunkBase = chunkBase;
    r.numChunks = owned;
    // the node's chunks go back to the queue (remolod_octree.cu:349-360);
    // k_spill_copy writes them at these positions, one per work item
    r.queueBase = owned ? atomicSub(&c->numAllocatedChunks, owned) - owned : kNone;
    d.numPoints[node] = 0;
    d.numPointChunks[node] = 0;
    d.ptTableOff[node] = kNone;
    d.ptTableCap[node] = 0;
    r.grid = g;
    d.splitRecs[k] = r;
    // its grid is zeroed after the expand loop (nothing reads it before voxel
    // sampling), so passes without stored points copy nothing
    if (g != kNone) {
        const uint32_t z = atomicAdd(&c->numZero, 1u);
        if (z < d.zeroCap) d.zeroList[z] = g;
    }
    if (k < kSplitInfo) {
        SplitInfo info;
        info.node = node;
        info.lv = d.level[node];
        info.X = d.nodeX[node];
        info.Y = d.nodeY[node];
        info.Z = d.nodeZ[node];
        info.grid = g;
        s_info[k] = info;
    }
    if (d.dirtyStamp[node] != c->buildStamp) {
        d.dirtyStamp[node] = c->buildStamp;
        const uint32_t di = atomicAdd(&c->numDirty, 1u);
        if (di < d.maxNodes) d.dirtyList[di] = node;
    }
}

// doSplitting (remolod_octree.cu:303-400) for the nodes the last count found,
// in increasing node id, each taking the next block of 8 ids. One block of
// 1024 threads. Up to 32 spilling nodes (the usual case: 14 nodes per batch on
// the reference's 36M cloud, wiki/03_ExpandStageFindings.md:63) are sorted,
// scanned and booked by one warp with no block barrier; more go through a
// block-wide sort and scans.
__device__ __forceinline__ void splitBody(const Dev& d, uint32_t stamp, uint32_t gated) {
    __shared__ uint32_t s_sort[kSortSmem];
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_runPts, s_runChunks, s_acc, s_nn, s_run2;
    __shared__ SplitInfo s_info[kSplitInfo];
    Counters* c = d.ctr;
    if (c->batchStop || (gated && c->loopMore == 0u)) return;
    // stamp 0: device-driven, (batch << 5) | pass as the host loop would pass it;
    // read before any thread reaches the barriers below, after which c->iter moves
    const uint32_t it0 = c->iter;
    if (stamp == 0u) stamp = (c->batchletIndex << 5) | it0;
    const bool histValid = c->histValid != 0u;
    uint32_t ns = c->numSpill;
    if (ns > d.spillingCap) ns = d.spillingCap;
    if (ns == 0) {
        if (threadIdx.x == 0) c->numSplit = 0;
        return;
    }
    const uint32_t spilledBefore = c->numSpilled;
    uint32_t nn, acc;
    if (ns <= 32u) {
        if (threadIdx.x < 32u) {
            const uint32_t lane = threadIdx.x;
            const uint32_t node = warpSortAscending(lane < ns ? d.spillNodes[lane] : kNone);
            const uint32_t n0 = c->numNodes;
            const uint32_t room = d.maxNodes > n0 ? (d.maxNodes - n0) / 8u : 0u;
            const uint32_t a = ns < room ? ns : room;
            uint32_t np = 0, owned = 0;
            if (lane < a) {
                owned = d.numPointChunks[node];
                const uint32_t cap = owned * d.ppc;
                np = d.numPoints[node] < cap ? d.numPoints[node] : cap;
            }
            uint32_t xp = np, xc = owned;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t yp = __shfl_up_sync(0xFFFFFFFFu, xp, o);
                const uint32_t yc = __shfl_up_sync(0xFFFFFFFFu, xc, o);
                if (lane >= (uint32_t)o) {
                    xp += yp;
                    xc += yc;
                }
            }
            if (lane < a) splitBook(d, c, lane, node, np, owned, spilledBefore + xp - np, xc - owned, stamp, s_info);
            const uint32_t totPts = __shfl_sync(0xFFFFFFFFu, xp, 31);
            const uint32_t totCh = __shfl_sync(0xFFFFFFFFu, xc, 31);
            if (lane == 0) {
                if (a < ns) c->nodePoolOverflow = 1;
                s_runPts = totPts;
                s_runChunks = totCh;
                s_acc = a;
                s_nn = n0;
            }
        }
        __syncthreads();
        acc = s_acc;
        nn = s_nn;
    } else {
        uint32_t* list;
        if (ns <= kSortSmem) {
            for (uint32_t i = threadIdx.x; i < ns; i += blockDim.x) s_sort[i] = d.spillNodes[i];
            __syncthreads();
            bitonicSort(s_sort, ns);
            list = s_sort;
        } else {
            // rare: sorts in the spilling-node buffer itself (sized to a power of two)
            bitonicSort(d.spillNodes, ns);
            list = d.spillNodes;
        }
        nn = c->numNodes;
        const uint32_t room = d.maxNodes > nn ? (d.maxNodes - nn) / 8u : 0u;
        acc = ns < room ? ns : room;
        if (threadIdx.x == 0) {
            if (acc < ns) c->nodePoolOverflow = 1;
            s_runPts = 0;
            s_runChunks = 0;
        }
        __syncthreads();
        for (uint32_t k0 = 0; k0 < acc; k0 += blockDim.x) {
            const uint32_t k = k0 + threadIdx.x;
            uint32_t node = 0, np = 0, owned = 0;
            if (k < acc) {
                node = list[k];
                owned = d.numPointChunks[node];
                const uint32_t cap = owned * d.ppc;
                np = d.numPoints[node] < cap ? d.numPoints[node] : cap;
            }
            uint32_t totPts, totCh;
            const uint32_t prePts = blockExclusiveScan(np, &totPts, s_warp);
            const uint32_t preCh = blockExclusiveScan(owned, &totCh, s_warp);
            if (k < acc)
                splitBook(d, c, k, node, np, owned, spilledBefore + s_runPts + prePts, s_runChunks + preCh, stamp,
                          s_info);
            __syncthreads();
            if (threadIdx.x == 0) {
                s_runPts += totPts;
                s_runChunks += totCh;
            }
            __syncthreads();
        }
    }
    // the children: one thread each, the next 8 ids after the pool's end per node
    for (uint32_t t = threadIdx.x; t < 8u * acc; t += blockDim.x) {
        const uint32_t k = t >> 3, i = t & 7u;
        SplitInfo info;
        if (k < kSplitInfo) {
            info = s_info[k];
        } else {
            info.node = d.splitRecs[k].node;
            info.grid = d.splitRecs[k].grid;
            info.lv = d.level[info.node];
            info.X = d.nodeX[info.node];
            info.Y = d.nodeY[info.node];
            info.Z = d.nodeZ[info.node];
        }
        const uint32_t node = info.node;
        const uint32_t ch = nn + t;
        const uint32_t lv = info.lv + 1u;
#pragma unroll
        for (int q = 0; q < 8; q++) d.child[ch * 8u + q] = -1;
        // the last recount binned the node's points by child octant: the
        // child's count is known already
        d.counter[ch] = histValid ? d.hist8[node * 8u + i] : 0u;
        reinterpret_cast<uint4*>(d.hist8 + (size_t)ch * 8u)[0] = make_uint4(0, 0, 0, 0);
        reinterpret_cast<uint4*>(d.hist8 + (size_t)ch * 8u)[1] = make_uint4(0, 0, 0, 0);
        d.numPoints[ch] = 0;
        d.level[ch] = lv;
        d.nodeX[ch] = 2u * info.X + ((i >> 2) & 1u);
        d.nodeY[ch] = 2u * info.Y + ((i >> 1) & 1u);
        d.nodeZ[ch] = 2u * info.Z + (i & 1u);
        d.grid[ch] = kNone;
        d.numVoxels[ch] = 0;
        d.numVoxelsStored[ch] = 0;
        d.numPointChunks[ch] = 0;
        d.numVoxelChunks[ch] = 0;
        d.ptTableOff[ch] = kNone;
        d.ptTableCap[ch] = 0;
        d.vxTableOff[ch] = kNone;
        d.vxTableCap[ch] = 0;
        d.splitIter[ch] = 0;
        d.dirtyStamp[ch] = 0;
        AccumI z = {};
        d.accum[ch] = z;
        const uint2* prow = d.anc + (size_t)node * kMaxDepth;
        uint2* crow = d.anc + (size_t)ch * kMaxDepth;
#pragma unroll
        for (uint32_t l = 0; l < (uint32_t)kMaxDepth; l++)
            if (l + 1u < lv) crow[l] = prow[l];
        crow[lv - 1u] = make_uint2(node, info.grid);
        d.parent[ch] = make_uint2(node, info.grid);
        d.child[node * 8u + i] = (int32_t)ch;
    }
    // Round two: with the octant counts known, the children over the limit are
    // split now, as the next pass would (in increasing id, the next 8 ids each),
    // if that pass would run (a recount follows this split: it0 < pass limit).
    // Their children's counts are unknown: the next recount counts them.
    __syncthreads();
    const uint32_t nn2 = nn + 8u * acc;
    uint32_t acc2 = 0;
    bool round2 = false;
    if (histValid && acc > 0u && it0 < d.maxExpandIters) {
        round2 = true;
        const uint32_t room2 = d.maxNodes > nn2 ? (d.maxNodes - nn2) / 8u : 0u;
        const uint32_t stamp2 = (c->batchletIndex << 5) | (it0 + 1u);
        if (threadIdx.x == 0) s_run2 = 0;
        __syncthreads();
        for (uint32_t t0 = 0; t0 < 8u * acc; t0 += blockDim.x) {
            const uint32_t t = t0 + threadIdx.x;
            const uint32_t f = (t < 8u * acc && d.counter[nn + t] > d.maxPointsPerNode) ? 1u : 0u;
            uint32_t tot;
            const uint32_t pre = blockExclusiveScan(f, &tot, s_warp);
            const uint32_t j = s_run2 + pre;
            if (f && j < room2) {
                const uint32_t node = nn + t;
                uint32_t g = takeGrid(d, c);
                d.grid[node] = g;
                d.splitIter[node] = stamp2;
                if (g != kNone) {
                    const uint32_t zi = atomicAdd(&c->numZero, 1u);
                    if (zi < d.zeroCap) d.zeroList[zi] = g;
                }
                d.dirtyStamp[node] = c->buildStamp;
                const uint32_t di = atomicAdd(&c->numDirty, 1u);
                if (di < d.maxNodes) d.dirtyList[di] = node;
                if (j < d.spillingCap) d.spillNodes[j] = node;
                if (j < kSplitInfo) {
                    SplitInfo info;
                    info.node = node;
                    info.lv = d.level[node];
                    info.X = d.nodeX[node];
                    info.Y = d.nodeY[node];
                    info.Z = d.nodeZ[node];
                    info.grid = g;
                    s_info[j] = info;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) s_run2 += tot;
            __syncthreads();
        }
        const uint32_t want = s_run2;
        acc2 = want < room2 ? want : room2;
        if (acc2 > d.spillingCap) acc2 = d.spillingCap;
        if (threadIdx.x == 0 && acc2 < want) c->nodePoolOverflow = 1;
        for (uint32_t t = threadIdx.x; t < 8u * acc2; t += blockDim.x) {
            const uint32_t k = t >> 3, i = t & 7u;
            SplitInfo info;
            if (k < kSplitInfo) {
                info = s_info[k];
            } else {
                info.node = d.spillNodes[k];
                info.grid = d.grid[info.node];
                info.lv = d.level[info.node];
                info.X = d.nodeX[info.node];
                info.Y = d.nodeY[info.node];
                info.Z = d.nodeZ[info.node];
            }
            const uint32_t node = info.node;
            const uint32_t ch = nn2 + t;
            const uint32_t lv = info.lv + 1u;
#pragma unroll
            for (int q = 0; q < 8; q++) d.child[ch * 8u + q] = -1;
            d.counter[ch] = 0;
            reinterpret_cast<uint4*>(d.hist8 + (size_t)ch * 8u)[0] = make_uint4(0, 0, 0, 0);
            reinterpret_cast<uint4*>(d.hist8 + (size_t)ch * 8u)[1] = make_uint4(0, 0, 0, 0);
            d.numPoints[ch] = 0;
            d.level[ch] = lv;
            d.nodeX[ch] = 2u * info.X + ((i >> 2) & 1u);
            d.nodeY[ch] = 2u * info.Y + ((i >> 1) & 1u);
            d.nodeZ[ch] = 2u * info.Z + (i & 1u);
            d.grid[ch] = kNone;
            d.numVoxels[ch] = 0;
            d.numVoxelsStored[ch] = 0;
            d.numPointChunks[ch] = 0;
            d.numVoxelChunks[ch] = 0;
            d.ptTableOff[ch] = kNone;
            d.ptTableCap[ch] = 0;
            d.vxTableOff[ch] = kNone;
            d.vxTableCap[ch] = 0;
            d.splitIter[ch] = 0;
            d.dirtyStamp[ch] = 0;
            AccumI z = {};
            d.accum[ch] = z;
            const uint2* prow = d.anc + (size_t)node * kMaxDepth;
            uint2* crow = d.anc + (size_t)ch * kMaxDepth;
#pragma unroll
            for (uint32_t l = 0; l < (uint32_t)kMaxDepth; l++)
                if (l + 1u < lv) crow[l] = prow[l];
            crow[lv - 1u] = make_uint2(node, info.grid);
            d.parent[ch] = make_uint2(node, info.grid);
            d.child[node * 8u + i] = (int32_t)ch;
        }
    }
    if (threadIdx.x == 0) {
        c->numNodes = nn2 + 8u * acc2;
        c->numSplit = acc;
        c->spillChunkTotal = s_runChunks;
        uint32_t total = spilledBefore + s_runPts;
        if (total > d.spillCap) {
            atomicOr(&c->overflowFlags, (uint32_t)kOvfSpilled);
            total = d.spillCap;
        }
        c->numSpilled = total;
        c->nodesSplit += acc + acc2;
        c->numSpill = 0;
        c->lastStamp = stamp;
        c->iter = it0 + (round2 ? 2u : 1u);
        // the nodes whose points the next recount counts
        if (!histValid) {
            c->countLo = nn;
            c->countHi = nn2;
        } else if (acc2 > 0u) {
            c->countLo = nn2;
            c->countHi = nn2 + 8u * acc2;
        } else {
            c->countLo = 0;
            c->countHi = 0;
        }
        c->histValid = 0;
    }
}

__global__ void __launch_bounds__(1024) k_split(Dev d, uint32_t stamp, uint32_t gated) { splitBody(d, stamp, gated); }

// The split nodes' stored points move to the spill list (remolod_octree.cu:250-285)
// and their chunks return to the queue (:349-360): one work item per owned
// chunk, strided over blocks.
__device__ __forceinline__ void spillCopyBody(const Dev& d, uint32_t gated) {
    const Counters* c = d.ctr;
    if (c->batchStop || (gated && c->loopMore == 0u)) return;
    const uint32_t nsplit = c->numSplit;
    const uint32_t nchunk = c->spillChunkTotal;
    for (uint32_t w = blockIdx.x; w < nchunk; w += gridDim.x) {
        {
            // binary search for the record holding work item w
            uint32_t lo = 0, hi = nsplit;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (d.splitRecs[mid].chunkBase <= w) lo = mid;
                else hi = mid;
            }
            const SplitRec r = d.splitRecs[lo];
            const uint32_t j = w - r.chunkBase;
            const uint32_t phys = d.tablePool[r.tableOff + j];
            if (threadIdx.x == 0 && r.queueBase + j < d.maxPtChunks) d.chunkQueue[r.queueBase + j] = phys;
            if (phys == kNone) continue;
            const uint32_t first = j * d.ppc;
            uint32_t last = first + d.ppc;
            if (last > r.numPoints) last = r.numPoints;
            for (uint32_t s = first + threadIdx.x; s < last; s += blockDim.x) {
                const uint32_t slot = r.spillBase + s;
                if (slot >= d.spillCap) break;
                d.spillPts[slot] = chunkPoints(d, phys)[s - first];
                d.spillIdx[slot] = chunkIndices(d, phys)[s - first];
                d.spillLeaf[slot] = r.node;
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_spill_copy(Dev d, uint32_t gated) { spillCopyBody(d, gated); }

// ------------------------------------------------------------ expand round
//
// The reference's expand loop (remolod_octree.cu:402-462) counts, splits the
// nodes over the limit, moves their points one level down and counts again,
// up to 20 times per batch. The nodes a batch splits are decided by its first
// count alone: iteration 1 lists the spilling leaves (the roots), and every
// later iteration counts only nodes made by the previous split, i.e. the cubes
// below the roots. So one pass that bins every point below a root by its cube
// at depths 1..kDeepLevels gives every count those iterations would take, and
// the splits, the ids they hand out and every counter follow from the counts
// in the reference's order: iteration by iteration, the spilling nodes in
// increasing id, each taking the next 8 ids. A round is four kernels --
// k_deep_book (book the roots' splits), k_deep_bin (spill their stored points
// and bin every point below a root), k_deep_split (all splits of iterations
// 1 .. 1 + kDeepLevels - 1) and k_deep_move (every moved point to its final
// leaf) -- instead of a count, split and recount per iteration. Cubes still
// over the limit at depth kDeepLevels (rare: 50,000 points in 1/4096 of a
// spilling node) go on through the per-iteration passes, as do batches whose
// first count lists more than kDeepRoots nodes or a node at the deepest level.

// A new node: child `i` of `parent` at id `ch` (doSplitting's child set-up,
// remolod_octree.cu:323-347), with its ancestor row.
__device__ __forceinline__ void makeChild(const Dev& d, uint32_t ch, uint32_t parent, uint32_t i) {
    // the parent's fields and its whole ancestor row in one round of loads
    // (row entries at and past its level are read and ignored)
    const uint32_t plv = d.level[parent], pg = d.grid[parent];
    const uint32_t px = d.nodeX[parent], py = d.nodeY[parent], pz = d.nodeZ[parent];
    const uint2* prow = d.anc + (size_t)parent * kMaxDepth;
    uint2 arow[kMaxDepth];
#pragma unroll
    for (uint32_t l = 0; l < (uint32_t)kMaxDepth; l++) arow[l] = prow[l];
    const uint32_t lv = plv + 1u;
#pragma unroll
    for (int q = 0; q < 8; q++) d.child[ch * 8u + q] = -1;
    d.counter[ch] = 0;
    reinterpret_cast<uint4*>(d.hist8 + (size_t)ch * 8u)[0] = make_uint4(0, 0, 0, 0);
    reinterpret_cast<uint4*>(d.hist8 + (size_t)ch * 8u)[1] = make_uint4(0, 0, 0, 0);
    d.numPoints[ch] = 0;
    d.level[ch] = lv;
    d.nodeX[ch] = 2u * px + ((i >> 2) & 1u);
    d.nodeY[ch] = 2u * py + ((i >> 1) & 1u);
    d.nodeZ[ch] = 2u * pz + (i & 1u);
    d.grid[ch] = kNone;
    d.numVoxels[ch] = 0;
    d.numVoxelsStored[ch] = 0;
    d.numPointChunks[ch] = 0;
    d.numVoxelChunks[ch] = 0;
    d.ptTableOff[ch] = kNone;
    d.ptTableCap[ch] = 0;
    d.vxTableOff[ch] = kNone;
    d.vxTableCap[ch] = 0;
    d.splitIter[ch] = 0;
    d.dirtyStamp[ch] = 0;
    AccumI z = {};
    d.accum[ch] = z;
    uint2* crow = d.anc + (size_t)ch * kMaxDepth;
#pragma unroll
    for (uint32_t l = 0; l < (uint32_t)kMaxDepth; l++)
        if (l + 1u < lv) crow[l] = arow[l];
    crow[lv - 1u] = make_uint2(parent, pg);
    d.parent[ch] = make_uint2(parent, pg);
    d.child[parent * 8u + i] = (int32_t)ch;
}

// The bookkeeping every split shares: a grid if the node has none (allocated
// once, zeroed at every split, :365-387), its split stamp, the grid on the
// zero list and the node on the dirty list.
__device__ __forceinline__ uint32_t bookSplit(const Dev& d, Counters* c, uint32_t node, uint32_t stamp) {
    // The node's fields in one round of loads, then the counter atomics back
    // to back: the single-block kernels that call this are bound by their
    // chain of dependent round trips. Every split takes a zero-list slot; one
    // left without a grid (arena exhausted) holds kNone and is skipped.
    uint32_t g = d.grid[node];
    const uint32_t bs = c->buildStamp;
    const bool dirty = d.dirtyStamp[node] == bs;
    const uint32_t z = atomicAdd(&c->numZero, 1u);
    const uint32_t di = dirty ? kNone : atomicAdd(&c->numDirty, 1u);
    if (g == kNone) {
        g = takeGrid(d, c);
        d.grid[node] = g;
    }
    d.splitIter[node] = stamp;
    if (z < d.zeroCap) d.zeroList[z] = g;
    if (!dirty) {
        d.dirtyStamp[node] = bs;
        if (di < d.maxNodes) d.dirtyList[di] = node;
    }
    return g;
}

// Root k of the round: its split bookkeeping and its record for k_deep_bin
// (spill slots from prePts, copy items from preCh).
__device__ __forceinline__ void deepBookRoot(const Dev& d, Counters* c, uint32_t k, uint32_t node, uint32_t np,
                                             uint32_t owned, uint32_t spillBase, uint32_t chunkBase, uint32_t stamp) {
    // issued ahead of the split's own atomics, used after them
    const uint32_t tableOff = d.ptTableOff[node];
    // the node's chunks go back to the queue (remolod_octree.cu:349-360)
    const uint32_t queueBase = owned ? atomicSub(&c->numAllocatedChunks, owned) - owned : kNone;
    const uint32_t g = bookSplit(d, c, node, stamp);
    SplitRec r;
    r.node = node;
    r.numPoints = np;
    r.tableOff = tableOff;
    r.spillBase = spillBase;
    r.chunkBase = chunkBase;
    r.numChunks = owned;
    r.grid = g;
    r.queueBase = queueBase;
    d.splitRecs[k] = r;
    d.numPoints[node] = 0;
    d.numPointChunks[node] = 0;
    d.ptTableOff[node] = kNone;
    d.ptTableCap[node] = 0;
    d.deepSlot[node] = k;
}

// The round's counters, by one thread.
__device__ __forceinline__ void deepBookCounters(const Dev& d, Counters* c, uint32_t ns, uint32_t acc,
                                                 uint32_t spilledBefore, uint32_t totPts, uint32_t totCh,
                                                 uint32_t stamp, uint32_t levels, uint32_t n0) {
    if (acc < ns) c->nodePoolOverflow = 1;
    uint32_t total = spilledBefore + totPts;
    if (total > d.spillCap) {
        atomicOr(&c->overflowFlags, (uint32_t)kOvfSpilled);
        total = d.spillCap;
    }
    c->numSpilled = total;
    c->numSplit = acc;
    c->spillChunkTotal = totCh;
    c->nodesSplit += acc;
    c->numSpill = 0;
    c->lastStamp = stamp;
    c->histValid = 0;
    c->countLo = 0;
    c->countHi = 0;
    c->deepRoots = acc;
    c->deepLevels = levels;
    c->deepBase = n0;
    c->deepStamp = stamp;
    c->deepActive = 1;
}

// Iteration 1's splits (doSplitting for the first count's spilling nodes, in
// increasing id): their bookkeeping, where their stored points go in the
// spill list, their chunks' queue positions. The children are made by
// k_deep_split with the later generations. One block of 1024 threads; up to
// 32 roots (most batches) are sorted, scanned and booked by one warp with no
// block barrier. Leaves the round off (the per-iteration passes take the
// batch) when no node can be split, more than kDeepRoots spill, or a root
// lies too deep to bin below.
__global__ void __launch_bounds__(1024) k_deep_book(Dev d) {
    __shared__ uint32_t s_sort[kDeepRoots];
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_maxLevel;
    Counters* c = d.ctr;
    if (c->batchStop) return;
    uint32_t ns = c->numSpill;
    if (ns > d.spillingCap) ns = d.spillingCap;
    if (ns == 0u || ns > kDeepRoots) return;
    const uint32_t n0 = c->numNodes;
    const uint32_t room = d.maxNodes > n0 ? (d.maxNodes - n0) / 8u : 0u;
    const uint32_t acc = ns < room ? ns : room;
    if (acc == 0u) return;
    const uint32_t stamp = (c->batchletIndex << 5) | c->iter;
    const uint32_t spilledBefore = c->numSpilled;
    if (ns <= 32u) {
        if (threadIdx.x >= 32u) return;
        const uint32_t lane = threadIdx.x;
        const uint32_t node = warpSortAscending(lane < ns ? d.spillNodes[lane] : kNone);
        // the root's level, chunks and points in one round of loads
        uint32_t lvl = 0, np = 0, owned = 0;
        if (lane < acc) {
            lvl = d.level[node];
            owned = d.numPointChunks[node];
            const uint32_t stored = d.numPoints[node];
            const uint32_t cap = owned * d.ppc;
            np = stored < cap ? stored : cap;
        }
        const uint32_t maxLevel = __reduce_max_sync(0xFFFFFFFFu, lvl);
        if (maxLevel >= (uint32_t)kMaxDepth) return;
        const uint32_t depthRoom = (uint32_t)kMaxDepth - maxLevel;
        const uint32_t levels = depthRoom < kDeepLevels ? depthRoom : kDeepLevels;
        uint32_t xp = np, xc = owned;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t yp = __shfl_up_sync(0xFFFFFFFFu, xp, o);
            const uint32_t yc = __shfl_up_sync(0xFFFFFFFFu, xc, o);
            if (lane >= (uint32_t)o) {
                xp += yp;
                xc += yc;
            }
        }
        const uint32_t totPts = __shfl_sync(0xFFFFFFFFu, xp, 31), totCh = __shfl_sync(0xFFFFFFFFu, xc, 31);
        if (lane < acc) deepBookRoot(d, c, lane, node, np, owned, spilledBefore + xp - np, xc - owned, stamp);
        if (lane == 0u) deepBookCounters(d, c, ns, acc, spilledBefore, totPts, totCh, stamp, levels, n0);
        return;
    }
    for (uint32_t i = threadIdx.x; i < ns; i += blockDim.x) s_sort[i] = d.spillNodes[i];
    if (threadIdx.x == 0) s_maxLevel = 0;
    __syncthreads();
    bitonicSort(s_sort, ns);
    for (uint32_t k = threadIdx.x; k < acc; k += blockDim.x) atomicMax(&s_maxLevel, d.level[s_sort[k]]);
    __syncthreads();
    const uint32_t maxLevel = s_maxLevel;
    if (maxLevel >= (uint32_t)kMaxDepth) return;
    const uint32_t depthRoom = (uint32_t)kMaxDepth - maxLevel;
    const uint32_t levels = depthRoom < kDeepLevels ? depthRoom : kDeepLevels;
    // acc <= kDeepRoots < blockDim.x: one scan covers every root
    const uint32_t k = threadIdx.x;
    uint32_t node = 0, np = 0, owned = 0;
    if (k < acc) {
        node = s_sort[k];
        owned = d.numPointChunks[node];
        const uint32_t cap = owned * d.ppc;
        np = d.numPoints[node] < cap ? d.numPoints[node] : cap;
    }
    uint32_t totPts, totCh;
    const uint32_t prePts = blockExclusiveScan(np, &totPts, s_warp);
    const uint32_t preCh = blockExclusiveScan(owned, &totCh, s_warp);
    if (k < acc) deepBookRoot(d, c, k, node, np, owned, spilledBefore + prePts, preCh, stamp);
    if (threadIdx.x == 0) deepBookCounters(d, c, ns, acc, spilledBefore, totPts, totCh, stamp, levels, n0);
}

// The depths of the expand round's pyramid that are counted point by point:
// the odd ones and the deepest. Every other depth is one below a counted one,
// so its count is the sum of eight counted cubes (deepCount): three rounds of
// binning per point instead of five.
__device__ __forceinline__ bool deepBinned(uint32_t depth, uint32_t levels) {
    return (depth & 1u) != 0u || depth == levels;
}

// The points in cube `code` at `depth` below root slot `slot`.
__device__ __forceinline__ uint32_t deepCount(const Dev& d, uint32_t slot, uint32_t depth, uint32_t code,
                                              uint32_t levels) {
    const uint32_t* row = d.deepCnt + (size_t)slot * kDeepCells;
    if (deepBinned(depth, levels)) return row[deepOffset(depth) + code];
    // the eight cubes one depth down are contiguous (code << 3 | octant)
    const uint4* k = reinterpret_cast<const uint4*>(row + deepOffset(depth + 1u) + (code << 3));
    const uint4 a = k[0], b = k[1];
    return a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
}

// A block's bin counts, merged in shared memory before they reach the global
// bins: the coarse cubes (8 per root at depth 1) are shared by most of a
// batch's points, and one global atomic per warp on them serialises in one L2
// slice. Keys are bin indices (slot * kDeepCells + cube), below 2^25.
constexpr uint32_t kDeepBlockBins = 1024;
struct DeepBlockBins {
    uint32_t key[kDeepBlockBins];
    uint32_t cnt[kDeepBlockBins];
};

__device__ __forceinline__ void deepBinsInit(DeepBlockBins& b) {
    for (uint32_t t = threadIdx.x; t < kDeepBlockBins; t += blockDim.x) {
        b.key[t] = kNone;
        b.cnt[t] = 0;
    }
}

// After a barrier: the block's counts into the global bins.
__device__ __forceinline__ void deepBinsFlush(const Dev& d, DeepBlockBins& b) {
    for (uint32_t t = threadIdx.x; t < kDeepBlockBins; t += blockDim.x)
        if (b.key[t] != kNone && b.cnt[t] != 0u) atomicAdd(&d.deepCnt[b.key[t]], b.cnt[t]);
}

// One point below root slot `slot` (at level lv) into its cubes at depths
// 1..levels. Every lane of the warp calls it; lanes with no point pass
// active = false. Equal cubes in a warp add once, into the block's table
// (or straight into the global bin when its probe run is full). Only the
// depths deepBinned names are counted; a cube at another depth holds the
// points of its eight cubes one depth down (deepCount).
__device__ __forceinline__ void deepBin(const Dev& d, DeepBlockBins& bins, bool active, uint32_t slot, uint32_t lv,
                                        const Point& p, uint32_t levels, uint32_t* codeOut) {
    uint32_t x = 0, y = 0, z = 0;
    if (active) {
        x = quant20(p.x, d.boxMin[0], d.octreeSize);
        y = quant20(p.y, d.boxMin[1], d.octreeSize);
        z = quant20(p.z, d.boxMin[2], d.octreeSize);
    }
    uint32_t code = 0;
#pragma unroll
    for (uint32_t j = 1; j <= kDeepLevels; j++) {
        if (j > levels) break;  // the same for every lane
        code = (code << 3) | (active ? childIndex(x, y, z, lv + j - 1u) : 0u);
        if (!deepBinned(j, levels)) continue;  // the same for every lane
        const uint32_t key = active ? slot * kDeepCells + deepOffset(j) + code : kNone;
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
        if (active && (int)laneId() == __ffs(peers) - 1) {
            const uint32_t g = (uint32_t)__popc(peers);
            uint32_t h = (key * 0x9E3779B1u) >> 22;
            bool done = false;
            for (uint32_t probe = 0; probe < 8u; probe++) {
                const uint32_t cur = atomicCAS(&bins.key[h], kNone, key);
                if (cur == kNone || cur == key) {
                    atomicAdd(&bins.cnt[h], g);
                    done = true;
                    break;
                }
                h = (h + 1u) & (kDeepBlockBins - 1u);
            }
            if (!done) atomicAdd(&d.deepCnt[key], g);
        }
    }
    // the cube at the deepest depth, for k_deep_move
    if (active) *codeOut = code;
}

// The roots' stored points move to the spill list (remolod_octree.cu:250-285)
// and their chunks return to the queue (:349-360), one work item per owned
// chunk; then every batch point whose leaf is a root, each block a contiguous
// run of the batch (neighbouring points share cubes). Each is binned below
// its root.
__global__ void __launch_bounds__(256) k_deep_bin(Dev d, const Point* __restrict__ pts, uint32_t n) {
    __shared__ DeepBlockBins s_bins;
    const Counters* c = d.ctr;
    if (c->batchStop || !c->deepActive) return;
    RB_BATCH_AT_CURSOR(d, pts, n);
    deepBinsInit(s_bins);
    __syncthreads();
    const uint32_t levels = c->deepLevels, stamp = c->deepStamp;
    const uint32_t nsplit = c->numSplit, nchunk = c->spillChunkTotal;
    for (uint32_t w = blockIdx.x; w < nchunk; w += gridDim.x) {
        uint32_t lo = 0, hi = nsplit;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (d.splitRecs[mid].chunkBase <= w) lo = mid;
            else hi = mid;
        }
        const SplitRec r = d.splitRecs[lo];
        const uint32_t j = w - r.chunkBase;
        const uint32_t phys = d.tablePool[r.tableOff + j];
        if (threadIdx.x == 0 && r.queueBase + j < d.maxPtChunks) d.chunkQueue[r.queueBase + j] = phys;
        if (phys == kNone) continue;
        const uint32_t lv = d.level[r.node];
        const uint32_t first = j * d.ppc;
        const uint32_t last = first + d.ppc < r.numPoints ? first + d.ppc : r.numPoints;
        for (uint32_t b = first; b < last; b += blockDim.x) {
            const uint32_t s = b + threadIdx.x;
            const uint32_t slot = r.spillBase + s;
            const bool active = s < last && slot < d.spillCap;
            Point q = {0.f, 0.f, 0.f, 0u};
            if (active) {
                q = chunkPoints(d, phys)[s - first];
                d.spillPts[slot] = q;
                d.spillIdx[slot] = chunkIndices(d, phys)[s - first];
                d.spillLeaf[slot] = r.node;
            }
            deepBin(d, s_bins, active, lo, lv, q, levels, d.spillCode + (active ? slot : 0u));
        }
    }
    const uint32_t per = (((n + gridDim.x - 1u) / gridDim.x) + 31u) & ~31u;
    const uint32_t begin = min(n, blockIdx.x * per), end = min(n, begin + per);
    for (uint32_t base = begin; base < end; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t leaf = 0;
        bool active = false;
        Point p = {0.f, 0.f, 0.f, 0u};
        if (i < end) {
            // the point with its leaf: one round trip instead of two
            p = loadPoint(pts + i);
            leaf = d.leafOf[i];
            active = d.splitIter[leaf] == stamp;
        }
        if (!__any_sync(0xFFFFFFFFu, active)) continue;
        uint32_t slot = 0, lv = 0;
        if (active) {
            slot = d.deepSlot[leaf];
            lv = d.level[leaf];
        }
        deepBin(d, s_bins, active, slot, lv, p, levels, d.moveCode + i);
    }
    __syncthreads();
    deepBinsFlush(d, s_bins);
}

// Iterations 2 .. 1 + kDeepLevels from the binned counts: generation g (the
// nodes made by iteration g's splits, g >= 1) is counted in iteration g + 1;
// its nodes over the limit split in that iteration, in increasing id, each
// taking the next 8 ids (the pool guard refuses them once fewer than 8 ids
// remain, :318-321), and the loop ends at the first iteration that splits
// nothing or at the pass limit. Nodes of the last generation counted and
// still over the limit are handed to the per-iteration passes. One block of
// 1024 threads.
__global__ void __launch_bounds__(1024) k_deep_split(Dev d) {
    __shared__ uint32_t s_warp[32];
    Counters* c = d.ctr;
    if (c->batchStop || !c->deepActive) return;
    const uint32_t roots = c->deepRoots, levels = c->deepLevels, base = c->deepBase, it0 = c->iter;
    const uint32_t batchTag = c->batchletIndex << 5;
    // generation 1: the roots' children, 8 consecutive ids per root in slot order
    for (uint32_t t = threadIdx.x; t < 8u * roots; t += blockDim.x) {
        makeChild(d, base + t, d.splitRecs[t >> 3].node, t & 7u);
        d.deepMeta[t] = ((t >> 3) << 16) | (t & 7u);
        d.deepNode[(size_t)(t >> 3) * kDeepCells + deepOffset(1u) + (t & 7u)] = base + t;
    }
    __syncthreads();
    uint32_t lo = base, hi = base + 8u * roots;
    uint32_t splits = 0, itEnd = 0, cont = 0;
    for (uint32_t g = 1;; g++) {
        const uint32_t it = it0 + g;  // the iteration that counts generation g
        if (it > d.maxExpandIters) {
            itEnd = it;  // the loop ended after the split that made generation g
            break;
        }
        const uint32_t room = d.maxNodes > hi ? (d.maxNodes - hi) / 8u : 0u;
        // running totals, the same in every thread (the scan returns them to all)
        uint32_t want = 0, contRun = 0;
        for (uint32_t t0 = lo; t0 < hi; t0 += blockDim.x) {
            const uint32_t node = t0 + threadIdx.x;
            uint32_t cnt = 0;
            if (node < hi) {
                const uint32_t meta = d.deepMeta[node - base];
                cnt = deepCount(d, meta >> 16, g, meta & 0xFFFFu, levels);
                d.counter[node] = cnt;
            }
            const bool over = node < hi && cnt > d.maxPointsPerNode;
            const uint32_t wantSplit = (over && g < levels) ? 1u : 0u;
            const uint32_t wantCont = (over && g == levels) ? 1u : 0u;
            // one scan for both lists: splits in the low half, continuations
            // in the high half (at most blockDim.x of each per step)
            uint32_t tot;
            const uint32_t pre = blockExclusiveScan(wantSplit | (wantCont << 16), &tot, s_warp);
            const uint32_t j = want + (pre & 0xFFFFu);
            if (wantSplit && j < room) {
                bookSplit(d, c, node, batchTag | it);
                d.deepPar[j] = node;
            }
            const uint32_t jc = contRun + (pre >> 16);
            if (wantCont && jc < d.spillingCap) d.spillNodes[jc] = node;
            want += tot & 0xFFFFu;
            contRun += tot >> 16;
        }
        const uint32_t nacc = want < room ? want : room;
        if (threadIdx.x == 0 && nacc < want) c->nodePoolOverflow = 1;
        if (nacc == 0u) {
            cont = contRun;
            // continuation: the per-iteration passes split them in this
            // iteration; every spiller refused: one more, empty, count
            itEnd = cont > 0u ? it : (want > 0u ? it + 1u : it);
            break;
        }
        splits += nacc;
        __syncthreads();  // the split list (deepPar) and the parents' grids are written
        // the children of this iteration's splits, ids [hi, hi + 8 nacc)
        for (uint32_t t = threadIdx.x; t < 8u * nacc; t += blockDim.x) {
            const uint32_t parent = d.deepPar[t >> 3];
            const uint32_t pm = d.deepMeta[parent - base];
            makeChild(d, hi + t, parent, t & 7u);
            const uint32_t meta = (pm & 0xFFFF0000u) | (((pm & 0xFFFFu) << 3) | (t & 7u));
            d.deepMeta[hi + t - base] = meta;
            d.deepNode[(size_t)(meta >> 16) * kDeepCells + deepOffset(g + 1u) + (meta & 0xFFFFu)] = hi + t;
        }
        __syncthreads();
        lo = hi;
        hi += 8u * nacc;
    }
    if (threadIdx.x == 0) {
        c->numNodes = hi;
        c->nodesSplit += splits;
        c->iter = itEnd;
        if (cont > d.spillingCap) {
            atomicOr(&c->overflowFlags, (uint32_t)kOvfSpilling);
            cont = d.spillingCap;
        }
        c->numSpill = cont;
    }
}

// Every point the round moved -- batch points and spilled points whose leaf
// is a root -- to its leaf in the finished subtree: the deepest node the round
// made along the point's cube path (k_deep_bin's code), read from the round's
// node table at every depth at once instead of walking down from the root.
__global__ void __launch_bounds__(256) k_deep_move(Dev d, const Point* __restrict__ pts, uint32_t n) {
    const Counters* c = d.ctr;
    if (c->batchStop || !c->deepActive) return;
    RB_BATCH_AT_CURSOR(d, pts, n);
    const uint32_t stamp = c->deepStamp, levels = c->deepLevels;
    const uint32_t ns = c->numSpilled < d.spillCap ? c->numSpilled : d.spillCap;
    const uint32_t total = n + ns;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const bool batchPt = i < n;
        uint32_t cur = batchPt ? d.leafOf[i] : d.spillLeaf[i - n];
        // issued beside the leaf id: most points of a batch sit in the roots
        const uint32_t code = batchPt ? d.moveCode[i] : d.spillCode[i - n];
        if (d.splitIter[cur] != stamp) continue;
        const uint32_t* row = d.deepNode + (size_t)d.deepSlot[cur] * kDeepCells;
        uint32_t ids[kDeepLevels];
#pragma unroll
        for (uint32_t j = 1; j <= kDeepLevels; j++)
            ids[j - 1u] = j <= levels ? row[deepOffset(j) + (code >> (3u * (levels - j)))] : kNone;
#pragma unroll
        for (uint32_t j = kDeepLevels; j >= 1u; j--) {
            if (ids[j - 1u] != kNone) {
                cur = ids[j - 1u];
                break;
            }
        }
        if (batchPt) d.leafOf[i] = cur;
        else d.spillLeaf[i - n] = cur;
    }
}

// The grids of the nodes split in this batch (zeroed at every split,
// :372-387) and the expand round's bins, cleared once after the expand loop
// (nothing reads a split grid before voxel sampling). Work items of 16 KB
// spread over every block of the caller's grid.
__device__ void zeroGridsBody(const Dev& d) {
    const Counters* c = d.ctr;
    if (c->batchStop) return;
    const uint32_t nz = c->numZero < d.zeroCap ? c->numZero : d.zeroCap;
    constexpr uint32_t kPiece = 1024;  // uint4 per work item
    constexpr uint32_t kPieces = kGridWords / 4u / kPiece;
    const uint32_t deepUnits = (c->deepRoots * kDeepCells + 3u) / 4u;  // rows are contiguous from slot 0
    const uint32_t deepItems = (deepUnits + kPiece - 1u) / kPiece;
    const uint4 z = make_uint4(0, 0, 0, 0), none = make_uint4(kNone, kNone, kNone, kNone);
    for (uint32_t w = blockIdx.x; w < nz * kPieces + 2u * deepItems; w += gridDim.x) {
        if (w < nz * kPieces) {
            const uint32_t zg = d.zeroList[w / kPieces];
            if (zg == kNone) continue;
            uint4* g = reinterpret_cast<uint4*>(gridWordsAt(d, zg)) + (w % kPieces) * kPiece;
            for (uint32_t q = threadIdx.x; q < kPiece; q += blockDim.x) g[q] = z;
        } else {
            // the round's bins back to zero, its node table back to kNone
            const uint32_t k = w - nz * kPieces;
            const bool nodes = k >= deepItems;
            const uint32_t u0 = (nodes ? k - deepItems : k) * kPiece;
            uint4* g = reinterpret_cast<uint4*>(nodes ? d.deepNode : d.deepCnt);
            for (uint32_t q = u0 + threadIdx.x; q < u0 + kPiece && q < deepUnits; q += blockDim.x) g[q] = nodes ? none : z;
        }
    }
}

__global__ void __launch_bounds__(256) k_zero_grids(Dev d) { zeroGridsBody(d); }

// After the expand loop, before voxel sampling and insertion. Once the loop
// stopped at its pass limit, a point's recorded leaf may have been split
// after its last count: its descent is finished here, so both sampling and
// insertion read the leaf the finished tree gives it. In arrival mode
// (Counters::arrivalMode, or this batch stopped at the limit) the points
// reaching each leaf are counted for the point-chunk allocation. Otherwise
// nothing to do: every recorded leaf is final and counters are whole.
__device__ void finishLeavesBody(const Dev& d, const Point* __restrict__ pts, uint32_t n) {
    const Counters* c = d.ctr;
    if (c->batchStop) return;
    const bool stale = c->iter > d.maxExpandIters;
    if (!stale && c->arrivalMode == 0u) return;
    RB_BATCH_AT_CURSOR(d, pts, n);
    const uint32_t ns = c->numSpilled < d.spillCap ? c->numSpilled : d.spillCap;
    const uint32_t total = n + ns;
    const uint32_t lane = laneId();
    // the same number of steps in every lane of a warp
    for (uint32_t b = blockIdx.x * blockDim.x; b < total; b += gridDim.x * blockDim.x) {
        const uint32_t i = b + threadIdx.x;
        const bool active = i < total;
        uint32_t leaf = kNone;
        if (active) {
            const bool batchPt = i < n;
            leaf = batchPt ? d.leafOf[i] : d.spillLeaf[i - n];
            if (stale) {
                const Point p = batchPt ? loadPoint(pts + i) : d.spillPts[i - n];
                const uint32_t x = quant20(p.x, d.boxMin[0], d.octreeSize),
                               y = quant20(p.y, d.boxMin[1], d.octreeSize),
                               z = quant20(p.z, d.boxMin[2], d.octreeSize);
                const uint32_t from = leaf;
                uint32_t lv = d.level[leaf];
                while (lv < (uint32_t)kMaxDepth) {
                    const int32_t nx = d.child[leaf * 8u + childIndex(x, y, z, lv)];
                    if (nx < 0) break;
                    leaf = (uint32_t)nx;
                    lv += 1u;
                }
                if (leaf != from) {
                    if (batchPt) d.leafOf[i] = leaf;
                    else d.spillLeaf[i - n] = leaf;
                }
            }
        }
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, leaf);
        if (active && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&d.arrive[leaf], (uint32_t)__popc(peers));
    }
}

__global__ void __launch_bounds__(256) k_finish_leaves(Dev d, const Point* __restrict__ pts, uint32_t n) {
    finishLeavesBody(d, pts, n);
}

// Grid-wide barrier of a cooperative launch. Every block is resident, so the
// wait ends once each block arrives; the polls are still bounded (about a
// second), after which the block records kOvfSync, the others stop waiting
// when they see it, and the caller returns. Thread 0 of each block keeps the
// barrier's epoch count.
__device__ bool gridBarrier(Counters* c, uint32_t& epoch) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        epoch += 1u;
        uint32_t ok = 1;
        __threadfence();
        const uint32_t arrived = atomicAdd(&c->barArrive, 1u) + 1u;
        if (arrived == epoch * gridDim.x) {
            __threadfence();
            atomicExch(&c->barRelease, epoch);
        } else {
            const volatile uint32_t* rel = &c->barRelease;
            const volatile uint32_t* flags = &c->overflowFlags;
            for (uint32_t spins = 0; *rel < epoch; spins++) {
                if (spins > (1u << 24) || (*flags & kOvfSync)) {
                    atomicOr(&c->overflowFlags, (uint32_t)kOvfSync);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0u;
}

// The per-iteration passes (split, spill copy, recount, loop test) for a
// batch the expand round left unfinished -- nodes still over the limit at its
// deepest binned level, or a first count it did not take -- as one
// cooperative kernel with grid barriers between the phases, so the batch
// graph needs no conditional node; then the batch's split grids are zeroed
// (zeroGridsBody), which saves the graph a node. Most batches only zero: the
// round left nothing to split. Launched with one 1024-thread block per SM.
__global__ void __launch_bounds__(1024, 1) k_expand_rest(Dev d) {
    Counters* c = d.ctr;
    if (c->batchStop) return;
    // no block writes numSpill before the first barrier: every block decides alike
    if (c->numSpill != 0u) {
        uint32_t epoch = 0;
        for (uint32_t pass = 0; pass < 64u; pass++) {
            if (!gridBarrier(c, epoch)) return;
            if (blockIdx.x == 0) splitBody(d, 0u, 0u);
            if (!gridBarrier(c, epoch)) return;
            spillCopyBody(d, 0u);
            if (!gridBarrier(c, epoch)) return;
            recountBody(d, nullptr, 0u, 0u, 0u);
            if (!gridBarrier(c, epoch)) return;
            if (blockIdx.x == 0) expandCondBody(d, 0ull, 0u);
            if (!gridBarrier(c, epoch)) return;
            // the next pass's split comes after its first barrier: all read alike
            if (c->loopMore == 0u) break;
        }
    }
    zeroGridsBody(d);
    finishLeavesBody(d, nullptr, 0u);
}

__device__ __forceinline__ uint32_t hashSlot(unsigned long long key, uint32_t mask) {
    unsigned long long h = key * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    return (uint32_t)h & mask;
}

// Records a claimed table slot in the batch's list of new cells.
__device__ __forceinline__ void listNewCell(const Dev& d, uint32_t e, uint32_t slot) {
    if (e < d.newCap) {
        d.hashNew[e] = slot;
    } else {
        atomicOr(&d.ctr->overflowFlags, (uint32_t)kOvfBacklog);
        d.ctr->hashNeedsClear = 1u;
        d.ctr->gridsPartial = 1u;
    }
}

// Inserts (key -> min val) into the per-batch cell table, probing from slot.
__device__ void hashInsertFrom(const Dev& d, unsigned long long key, unsigned long long val, uint32_t slot) {
    for (uint32_t probe = 0; probe < 256u; probe++) {
        unsigned long long* ks = &d.hashSlots[slot].x;
        unsigned long long* vs = &d.hashSlots[slot].y;
        // key and value in one 16-byte read: a present key whose value is
        // already lower needs no atomic (values only decrease)
        const ulonglong2 kv = __ldcg(&d.hashSlots[slot]);
        unsigned long long cur = kv.x;
        if (cur == key && kv.y <= val && d.voxelMode == 0u) return;
        if (cur == kHashEmpty) {
            cur = atomicCAS(ks, kHashEmpty, key);
            if (cur == kHashEmpty) {
                listNewCell(d, atomicAdd(&d.ctr->numNew, 1u), slot);
                cur = key;
            }
        }
        if (cur == key) {
            if (d.voxelMode == 0u) atomicMin(vs, val);
            else atomicCAS(vs, kHashEmpty, val);
            return;
        }
        slot = (slot + 1u) & d.hashMask;
    }
    atomicOr(&d.ctr->overflowFlags, (uint32_t)kOvfBacklog);
    d.ctr->hashNeedsClear = 1u;
    d.ctr->gridsPartial = 1u;
}

__device__ __forceinline__ uint32_t cellAt(uint32_t x28, uint32_t y28, uint32_t z28, uint32_t level) {
    const uint32_t sh = (uint32_t)kMaxDepth + 1u - level;
    return ((x28 >> sh) & 127u) + ((y28 >> sh) & 127u) * 128u + ((z28 >> sh) & 127u) * 16384u;
}

// Per-block cache of cells this block's points lead, direct-mapped: entry
// (tag << 32) | global point index, tag = key >> kCellCacheBits (under 2^31,
// since node ids stay below 2^21), position = the key's low bits plus a hash of
// the tag, so tag and position give back the key.
constexpr uint32_t kCellCacheBits = 11;
constexpr uint32_t kCellCache = 1u << kCellCacheBits;
// Per-warp buffer of claimed table slots: under 32 waiting plus one claim per lane.
constexpr uint32_t kWarpCells = 64u;

// The warp's buffered slots into the batch's list of new cells, with one
// counter atomic (a single counter bumped by every claim serialises the
// claims of the whole grid). Every lane of the warp calls it.
__device__ __forceinline__ void flushWarpCells(const Dev& d, const uint32_t* wbuf, uint32_t count) {
    if (count == 0u) return;
    const uint32_t lane = laneId();
    uint32_t e0 = 0;
    if (lane == 0u) e0 = atomicAdd(&d.ctr->numNew, count);
    e0 = __shfl_sync(0xFFFFFFFFu, e0, 0);
    for (uint32_t t = lane; t < count; t += 32u) listNewCell(d, e0 + t, wbuf[t]);
    __syncwarp();
}

// voxelSampling (remolod_octree.cu:677-740) + sampleVoxel's test (:95-119),
// first half. A point tests the cell of every node on its path whose grid
// exists: the ancestors of its leaf, and the leaf itself while it has a grid
// (a root that has never split). Its cell in node N at level l is the top
// 7 + l bits of its 28-bit coordinates, so its cells on the path are prefixes
// of its cell at the deepest tested level D; and a bit is only ever set
// together with the same point's bits at every level above (a grid is zeroed
// when its node splits, before any node below it exists). So the levels whose
// cell was empty before this batch are a run ending at D, and the point's
// whole contribution follows from one test: its cell at D. When that bit is
// clear, the cell goes into the batch's table, which keeps per cell the lowest
// global point index reaching it (or the first to arrive); k_vox_lift then
// carries every new cell's representative up to the levels above. The set of
// new cells and their representatives are exactly the per-level sampling's.
//
// Bits are not written here, so every point sees the pre-batch grids. One
// leader per run of equal cells in the warp (batch points ascend in index with
// the lane, so a run's first lane holds its lowest index; spilled points use a
// full match), then a per-block direct-mapped cache drops a leader whose cell
// an earlier point of the block already leads (a lower index, or any point in
// first-come mode). Claimed slots are buffered per warp and listed 32 at a
// time with one counter atomic.
__global__ void __launch_bounds__(256) k_vox_sample(Dev d, const Point* __restrict__ pts, uint32_t n) {
    __shared__ uint32_t s_wbuf[256 / 32][kWarpCells];
    __shared__ unsigned long long s_cells[kCellCache];
    const Counters* c = d.ctr;
    if (c->batchStop || c->levelMode) return;
    for (uint32_t t = threadIdx.x; t < kCellCache; t += blockDim.x) s_cells[t] = ~0ull;
    __syncthreads();
    // single 64-bit accesses: an entry is read and written whole
    volatile unsigned long long* cells = s_cells;
    RB_BATCH_AT_CURSOR(d, pts, n);
    uint32_t* wbuf = s_wbuf[threadIdx.x >> 5];
    uint32_t wbufN = 0;  // the same in every lane of the warp
    const uint32_t ns = c->numSpilled < d.spillCap ? c->numSpilled : d.spillCap;
    const uint32_t total = n + ns;
    const uint32_t firstIndex = (uint32_t)c->numPointsProcessed;
    const bool lowest = d.voxelMode == 0u;
    const uint32_t lane = laneId();
    const uint32_t per = (((total + gridDim.x - 1u) / gridDim.x) + 31u) & ~31u;
    const uint32_t begin = min(total, blockIdx.x * per), end = min(total, begin + per);
    for (uint32_t base = begin; base < end; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const bool active = i < end;
        Point p = {0.f, 0.f, 0.f, 0u};
        uint32_t gidx = 0, leaf = 0;
        if (active && i < n) {
            p = loadPoint(pts + i);
            gidx = firstIndex + i;
            leaf = d.leafOf[i];
        } else if (active) {
            p = d.spillPts[i - n];
            gidx = d.spillIdx[i - n];
            leaf = d.spillLeaf[i - n];
        }
        // the deepest tested node: the leaf while it has a grid, else its parent
        unsigned long long key = kHashEmpty;
        if (active) {
            // level, grid and parent in one round of loads
            const uint32_t lv = d.level[leaf];
            uint32_t node = leaf, g = d.grid[leaf], tl = lv;
            const uint2 a = lv > 0u ? d.parent[leaf] : make_uint2(kNone, kNone);
            if (g == kNone && lv > 0u) {
                node = a.x;
                g = a.y;
                tl = lv - 1u;
            }
            if (g != kNone) {
                const uint32_t x28 = quant28(p.x, d.boxMin[0], d.octreeSize);
                const uint32_t y28 = quant28(p.y, d.boxMin[1], d.octreeSize);
                const uint32_t z28 = quant28(p.z, d.boxMin[2], d.octreeSize);
                const uint32_t vi = cellAt(x28, y28, z28, tl);
                if (((__ldg(gridWordsAt(d, g) + (vi >> 5)) >> (vi & 31u)) & 1u) == 0u)
                    key = ((unsigned long long)node << 21) | (unsigned long long)vi;
            }
        }
        // one leader per cell in the warp
        bool first;
        if (__all_sync(0xFFFFFFFFu, !active || i < n)) {
            const unsigned long long prev = __shfl_up_sync(0xFFFFFFFFu, key, 1);
            first = key != kHashEmpty && (lane == 0u || prev != key);
        } else {
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
            if (lowest) first = key != kHashEmpty && gidx == __reduce_min_sync(peers, gidx);
            else first = key != kHashEmpty && lane == (uint32_t)(__ffs(peers) - 1);
        }
        if (first) {
            const uint32_t tag = (uint32_t)(key >> kCellCacheBits);
            const uint32_t e = ((uint32_t)key + ((tag * 0x9E3779B1u) >> (32u - kCellCacheBits))) & (kCellCache - 1u);
            const unsigned long long held = cells[e];
            if ((uint32_t)(held >> 32) == tag && (!lowest || (uint32_t)held < gidx)) first = false;
            else cells[e] = ((unsigned long long)tag << 32) | gidx;
        }
        // the leader's table update: read, claim an empty slot, lower the index
        bool claimed = false;
        uint32_t slot = 0;
        if (first) {
            const unsigned long long val = ((unsigned long long)gidx << 32) | p.color;
            slot = hashSlot(key, d.hashMask);
            const ulonglong2 kv = __ldcg(&d.hashSlots[slot]);
            unsigned long long cur = kv.x;
            bool update = false;
            if (cur == key) {
                update = lowest ? kv.y > val : kv.y == kHashEmpty;
            } else if (cur == kHashEmpty) {
                cur = atomicCAS(&d.hashSlots[slot].x, kHashEmpty, key);
                claimed = cur == kHashEmpty;
                update = claimed || cur == key;
                if (!update) hashInsertFrom(d, key, val, (slot + 1u) & d.hashMask);
            } else {
                hashInsertFrom(d, key, val, (slot + 1u) & d.hashMask);
            }
            if (update) {
                if (lowest) atomicMin(&d.hashSlots[slot].y, val);
                else atomicCAS(&d.hashSlots[slot].y, kHashEmpty, val);
            }
        }
        // claimed slots wait in the warp's buffer; 32 or more go to the list of
        // new cells with one counter atomic
        const unsigned cm = __ballot_sync(0xFFFFFFFFu, claimed);
        if (claimed) wbuf[wbufN + (uint32_t)__popc(cm & ((1u << lane) - 1u))] = slot;
        __syncwarp();
        wbufN += (uint32_t)__popc(cm);
        if (wbufN >= 32u) {
            flushWarpCells(d, wbuf, wbufN);
            wbufN = 0;
        }
    }
    flushWarpCells(d, wbuf, wbufN);
}

// Inserts (key -> val) for k_vox_lift. Returns whether the walk goes on: it
// stops where the cell already holds a lower index (lowest mode) or any point
// (first-come mode), since that point's own walk carries it further up. Cells
// it claims go to the block's list (s_list, s_n).
__device__ __forceinline__ bool liftInsert(const Dev& d, unsigned long long key, unsigned long long val,
                                           uint32_t* s_list, uint32_t* s_n) {
    const bool lowest = d.voxelMode == 0u;
    uint32_t slot = hashSlot(key, d.hashMask);
    for (uint32_t probe = 0; probe < 256u; probe++) {
        const ulonglong2 kv = __ldcg(&d.hashSlots[slot]);
        unsigned long long cur = kv.x;
        if (cur == key) {
            if (lowest) return kv.y > val && atomicMin(&d.hashSlots[slot].y, val) > val;
            return kv.y == kHashEmpty && atomicCAS(&d.hashSlots[slot].y, kHashEmpty, val) == kHashEmpty;
        }
        if (cur == kHashEmpty) {
            cur = atomicCAS(&d.hashSlots[slot].x, kHashEmpty, key);
            if (cur == kHashEmpty) {
                s_list[atomicAdd(s_n, 1u)] = slot;
                if (lowest) return atomicMin(&d.hashSlots[slot].y, val) > val;
                return atomicCAS(&d.hashSlots[slot].y, kHashEmpty, val) == kHashEmpty;
            }
            if (cur == key) {
                if (lowest) return atomicMin(&d.hashSlots[slot].y, val) > val;
                return atomicCAS(&d.hashSlots[slot].y, kHashEmpty, val) == kHashEmpty;
            }
        }
        slot = (slot + 1u) & d.hashMask;
    }
    atomicOr(&d.ctr->overflowFlags, (uint32_t)kOvfBacklog);
    d.ctr->hashNeedsClear = 1u;
    d.ctr->gridsPartial = 1u;
    return false;
}

constexpr uint32_t kLiftThreads = 256;
constexpr uint32_t kLiftChunk = 4;  // ancestor levels a walk loads at once

// voxelSampling's second half: every cell k_vox_sample listed carries its
// representative up its node's ancestors. At each level above, its prefix
// cell is a new cell of this batch exactly when that cell's bit was clear
// before the batch (the bits are still the pre-batch ones here), and its
// representative is the lowest index over the cells below it; a walk stops at
// the first set bit, or where a lower index is already in place. Cells the
// walks claim are listed after k_vox_sample's, through a second counter
// (numLift), one block reservation per pass; a walk claims at most one cell
// per level, so a pass's claims fit kLiftThreads x kMaxDepth entries.
__global__ void __launch_bounds__(kLiftThreads) k_vox_lift(Dev d) {
    __shared__ uint32_t s_list[kLiftThreads * kMaxDepth];
    __shared__ uint32_t s_n, s_base;
    const Counters* c = d.ctr;
    if (c->batchStop || c->levelMode) return;
    const uint32_t walkers = c->numNew < d.newCap ? c->numNew : d.newCap;
    const uint32_t listed = c->numNew;
    for (uint32_t b = blockIdx.x * kLiftThreads; b < walkers; b += gridDim.x * kLiftThreads) {
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        const uint32_t e = b + threadIdx.x;
        if (e < walkers) {
            const uint32_t slot = d.hashNew[e];
            const ulonglong2 kv = __ldcg(&d.hashSlots[slot]);
            const uint32_t node = (uint32_t)(kv.x >> 21), vi = (uint32_t)(kv.x & 0x1FFFFFull);
            const uint32_t lv = d.level[node];
            // the cell's coordinates at 7 + lv bits per axis
            const uint32_t px = (d.nodeX[node] << 7) | (vi & 127u);
            const uint32_t py = (d.nodeY[node] << 7) | ((vi >> 7) & 127u);
            const uint32_t pz = (d.nodeZ[node] << 7) | (vi >> 14);
            const uint2* row = d.anc + (size_t)node * kMaxDepth;
            // the ancestors and their grid words four levels at a time, then
            // the table updates one level after another
            bool go = true;
            for (uint32_t top = lv; go && top > 0u;) {
                const uint32_t cnt = top < kLiftChunk ? top : kLiftChunk;
                uint2 an[kLiftChunk];
                uint32_t cl[kLiftChunk], word[kLiftChunk];
#pragma unroll
                for (uint32_t k = 0; k < kLiftChunk; k++)
                    an[k] = k < cnt ? row[top - 1u - k] : make_uint2(kNone, kNone);
#pragma unroll
                for (uint32_t k = 0; k < kLiftChunk; k++) {
                    const uint32_t sh = k + 1u + (lv - top);
                    cl[k] = ((px >> sh) & 127u) + ((py >> sh) & 127u) * 128u + ((pz >> sh) & 127u) * 16384u;
                    word[k] = an[k].y != kNone ? __ldg(gridWordsAt(d, an[k].y) + (cl[k] >> 5)) : ~0u;
                }
#pragma unroll
                for (uint32_t k = 0; k < kLiftChunk; k++) {
                    if (!go || k >= cnt) break;
                    if ((word[k] >> (cl[k] & 31u)) & 1u) {
                        go = false;
                        break;
                    }
                    go = liftInsert(d, ((unsigned long long)an[k].x << 21) | cl[k], kv.y, s_list, &s_n);
                }
                top -= cnt;
            }
        }
        __syncthreads();
        const uint32_t cnt = s_n;
        if (threadIdx.x == 0 && cnt) s_base = atomicAdd(&d.ctr->numLift, cnt);
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < cnt; t += kLiftThreads) {
            // listed after k_vox_sample's cells: positions listed + numLift
            const unsigned long long pos = (unsigned long long)listed + s_base + t;
            listNewCell(d, pos < 0xFFFFFFFFull ? (uint32_t)pos : 0xFFFFFFFFu, s_list[t]);
        }
    }
}

// The level-by-level form of voxel sampling, for the batches after one whose
// new cells outran the list (Counters::gridsPartial, until the next reset).
// Cells a full list dropped keep their bits clear while cells below them may
// have been set, so a clear bit no longer follows from the deepest tested
// level and k_vox_sample's single test would miss them; this form tests every
// level on its own and finds every lost cell again.
constexpr uint32_t kInsertGroup = 4;  // table updates a lane keeps in flight
constexpr uint32_t kWarpCellsLevels = 32u + 32u * kInsertGroup;

// Every (point, level) pair whose cell bit was clear before this batch is a
// candidate; the table keeps, per cell, the lowest global point index reaching
// it (or the first to arrive). Bits are not written here, so every pair sees
// the pre-batch grid, and the set of new cells is exactly the reference's.
//
// Latency, not bandwidth, bounds this kernel, so it runs as three phases of
// independent memory operations instead of a chain per level: (1) the grid
// words of every level at once (the ancestor row replaces the root-to-leaf
// pointer chase); (2) per level, one leader per run of equal cells in the warp
// (batch points ascend in index with the lane, so a run's first lane holds its
// lowest index; spilled points use a full match); (3) each lane's table
// updates in groups: all slot reads, then all claims, then all minimum
// updates, with one new-cell counter bump per warp and group. A slot already
// holding a lower index is left alone. Between (2) and (3) a leader whose cell
// an earlier point of the same block already leads (a lower index, or any
// point in first-come mode) drops out: that point's update keeps the table's
// result, and most of a block's leaders repeat cells its other warps lead.
__global__ void __launch_bounds__(256) k_vox_sample_levels(Dev d, const Point* __restrict__ pts, uint32_t n) {
    __shared__ uint32_t s_wbuf[256 / 32][kWarpCellsLevels];
    __shared__ unsigned long long s_cells[kCellCache];
    const Counters* c = d.ctr;
    if (c->batchStop || !c->levelMode) return;
    for (uint32_t t = threadIdx.x; t < kCellCache; t += blockDim.x) s_cells[t] = ~0ull;
    __syncthreads();
    // single 64-bit accesses: an entry is read and written whole
    volatile unsigned long long* cells = s_cells;
    RB_BATCH_AT_CURSOR(d, pts, n);
    uint32_t* wbuf = s_wbuf[threadIdx.x >> 5];
    uint32_t wbufN = 0;  // the same in every lane of the warp
    const uint32_t ns = c->numSpilled < d.spillCap ? c->numSpilled : d.spillCap;
    const uint32_t total = n + ns;
    const uint32_t firstIndex = (uint32_t)c->numPointsProcessed;
    const bool lowest = d.voxelMode == 0u;
    const uint32_t lane = laneId();
    const uint32_t per = (((total + gridDim.x - 1u) / gridDim.x) + 31u) & ~31u;
    const uint32_t begin = min(total, blockIdx.x * per), end = min(total, begin + per);
    for (uint32_t base = begin; base < end; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const bool active = i < end;
        Point p = {0.f, 0.f, 0.f, 0u};
        uint32_t gidx = 0, leaf = 0;
        if (active && i < n) {
            p = loadPoint(pts + i);
            gidx = firstIndex + i;
            leaf = d.leafOf[i];
        } else if (active) {
            p = d.spillPts[i - n];
            gidx = d.spillIdx[i - n];
            leaf = d.spillLeaf[i - n];
        }
        uint32_t x28 = 0, y28 = 0, z28 = 0, lv = 0;
        if (active) {
            x28 = quant28(p.x, d.boxMin[0], d.octreeSize);
            y28 = quant28(p.y, d.boxMin[1], d.octreeSize);
            z28 = quant28(p.z, d.boxMin[2], d.octreeSize);
            lv = d.level[leaf];
        }
        // (1) which levels' cells were empty before this batch
        const uint2* row = d.anc + (size_t)leaf * kMaxDepth;
        uint32_t mask = 0;
        for (uint32_t l0 = 0; l0 < (uint32_t)kMaxDepth; l0 += 8u) {
            if (!__any_sync(0xFFFFFFFFu, active && lv > l0)) break;
            uint2 a[8];
#pragma unroll
            for (uint32_t k = 0; k < 8u; k++)
                a[k] = (active && l0 + k < lv) ? row[l0 + k] : make_uint2(kNone, kNone);
            uint32_t w[8];
#pragma unroll
            for (uint32_t k = 0; k < 8u; k++) {
                w[k] = ~0u;
                if (a[k].y != kNone)
                    w[k] = __ldg(gridWordsAt(d, a[k].y) + (cellAt(x28, y28, z28, l0 + k) >> 5));
            }
#pragma unroll
            for (uint32_t k = 0; k < 8u; k++)
                if (((w[k] >> (cellAt(x28, y28, z28, l0 + k) & 31u)) & 1u) == 0u) mask |= 1u << (l0 + k);
        }
        // the point's own node samples too while it has a grid (a root that has never split)
        if (active) {
            const uint32_t g = d.grid[leaf];
            if (g != kNone) {
                const uint32_t vi = cellAt(x28, y28, z28, lv);
                if (((__ldg(gridWordsAt(d, g) + (vi >> 5)) >> (vi & 31u)) & 1u) == 0u) mask |= 1u << lv;
            }
        }
        // (2) the levels this lane updates the table for
        const bool ordered = __all_sync(0xFFFFFFFFu, !active || i < n);
        uint32_t lead = 0;
        uint32_t todo = __reduce_or_sync(0xFFFFFFFFu, mask);
        while (todo) {
            const uint32_t l = (uint32_t)(__ffs(todo) - 1);
            todo &= todo - 1u;
            unsigned long long key = kHashEmpty;
            if ((mask >> l) & 1u) {
                const uint32_t node = l < lv ? row[l].x : leaf;
                key = ((unsigned long long)node << 21) | (unsigned long long)cellAt(x28, y28, z28, l);
            }
            bool first;
            if (ordered) {
                const unsigned long long prev = __shfl_up_sync(0xFFFFFFFFu, key, 1);
                first = key != kHashEmpty && (lane == 0u || prev != key);
            } else {
                const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
                if (lowest) first = key != kHashEmpty && gidx == __reduce_min_sync(peers, gidx);
                else first = key != kHashEmpty && lane == (uint32_t)(__ffs(peers) - 1);
            }
            if (first) {
                const uint32_t tag = (uint32_t)(key >> kCellCacheBits);
                const uint32_t e = ((uint32_t)key + ((tag * 0x9E3779B1u) >> (32u - kCellCacheBits))) & (kCellCache - 1u);
                const unsigned long long held = cells[e];
                if ((uint32_t)(held >> 32) == tag && (!lowest || (uint32_t)held < gidx)) first = false;
                else cells[e] = ((unsigned long long)tag << 32) | gidx;
            }
            if (first) lead |= 1u << l;
        }
        // (3) table updates, kInsertGroup levels at a time
        const unsigned long long val = ((unsigned long long)gidx << 32) | p.color;
        while (__any_sync(0xFFFFFFFFu, lead != 0u)) {
            unsigned long long key[kInsertGroup];
            uint32_t slot[kInsertGroup];
            uint32_t nk = 0;
#pragma unroll
            for (uint32_t j = 0; j < kInsertGroup; j++) {
                key[j] = kHashEmpty;
                slot[j] = 0;
                if (lead) {
                    const uint32_t l = (uint32_t)(__ffs(lead) - 1);
                    lead &= lead - 1u;
                    const uint32_t node = l < lv ? row[l].x : leaf;
                    key[j] = ((unsigned long long)node << 21) | (unsigned long long)cellAt(x28, y28, z28, l);
                    slot[j] = hashSlot(key[j], d.hashMask);
                    nk = j + 1u;
                }
            }
            ulonglong2 kv[kInsertGroup];
#pragma unroll
            for (uint32_t j = 0; j < kInsertGroup; j++)
                kv[j] = j < nk ? __ldcg(&d.hashSlots[slot[j]]) : make_ulonglong2(kHashEmpty, 0ull);
            // 0: settled, 1: update the value, 2: claim the slot, 3: probe further
            uint32_t state[kInsertGroup];
            unsigned long long got[kInsertGroup];
#pragma unroll
            for (uint32_t j = 0; j < kInsertGroup; j++) {
                state[j] = 0u;
                got[j] = kHashEmpty;
                if (j < nk) {
                    if (kv[j].x == key[j]) state[j] = (lowest ? kv[j].y > val : kv[j].y == kHashEmpty) ? 1u : 0u;
                    else if (kv[j].x == kHashEmpty) state[j] = 2u;
                    else state[j] = 3u;
                }
                if (state[j] == 2u) got[j] = atomicCAS(&d.hashSlots[slot[j]].x, kHashEmpty, key[j]);
            }
            uint32_t claimed = 0;
#pragma unroll
            for (uint32_t j = 0; j < kInsertGroup; j++) {
                if (state[j] == 2u) {
                    if (got[j] == kHashEmpty) claimed |= 1u << j;
                    state[j] = (got[j] == kHashEmpty || got[j] == key[j]) ? 1u : 3u;
                }
                if (state[j] == 1u) {
                    if (lowest) atomicMin(&d.hashSlots[slot[j]].y, val);
                    else atomicCAS(&d.hashSlots[slot[j]].y, kHashEmpty, val);
                } else if (state[j] == 3u) {
                    hashInsertFrom(d, key[j], val, (slot[j] + 1u) & d.hashMask);
                }
            }
            // the claimed slots wait in the warp's buffer; 32 or more go to the
            // list of new cells with one counter atomic
            const uint32_t nc = (uint32_t)__popc(claimed);
            uint32_t pre = nc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, pre, o);
                if (lane >= (uint32_t)o) pre += y;
            }
            const uint32_t added = __shfl_sync(0xFFFFFFFFu, pre, 31);
            uint32_t pos = wbufN + pre - nc;
#pragma unroll
            for (uint32_t j = 0; j < kInsertGroup; j++)
                if ((claimed >> j) & 1u) wbuf[pos++] = slot[j];
            __syncwarp();
            wbufN += added;
            if (wbufN >= 32u) {
                flushWarpCells(d, wbuf, wbufN);
                wbufN = 0;
            }
        }
    }
    flushWarpCells(d, wbuf, wbufN);
}

// The new cells both halves of voxel sampling listed, at most the list's capacity.
__device__ __forceinline__ uint32_t newCellCount(const Dev& d) {
    const unsigned long long t = (unsigned long long)d.ctr->numNew + d.ctr->numLift;
    return t < d.newCap ? (uint32_t)t : d.newCap;
}

// blockReserve for kEntriesPerThread keys per thread at once: every key's
// count merges into the block table first, then one barrier pair hands out
// the global reservations. Every thread of the block calls it. Kernels that
// use it take kEntriesPerThread items per thread (a block's items in steps of
// blockDim.x) and issue each step's loads for all of them before using any.
constexpr uint32_t kEntriesPerThread = 4;

__device__ __forceinline__ void blockReserveMany(BlockSlots& b, uint32_t* counters,
                                                 const uint32_t (&key)[kEntriesPerThread],
                                                 uint32_t (&out)[kEntriesPerThread]) {
    const uint32_t lane = laneId();
    uint32_t at[kEntriesPerThread], off[kEntriesPerThread], rank[kEntriesPerThread];
#pragma unroll
    for (uint32_t j = 0; j < kEntriesPerThread; j++) {
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, key[j]);
        const int leader = __ffs(peers) - 1;
        rank[j] = __popc(peers & ((1u << lane) - 1u));
        uint32_t s = kNone, o = 0;
        if (key[j] != kNone && (int)lane == leader) {
            const uint32_t g = __popc(peers);
            uint32_t h = (key[j] * 0x9E3779B1u) >> 26;
            for (uint32_t probe = 0; probe < 8u; probe++) {
                const uint32_t cur = atomicCAS(&b.key[h], kNone, key[j]);
                if (cur == kNone || cur == key[j]) {
                    s = h;
                    o = atomicAdd(&b.cnt[h], g);
                    break;
                }
                h = (h + 1u) & (kBlockLeaves - 1u);
            }
            if (s == kNone) o = atomicAdd(&counters[key[j]], g);  // crowded table: reserve globally
        }
        at[j] = __shfl_sync(0xFFFFFFFFu, s, leader);
        off[j] = __shfl_sync(0xFFFFFFFFu, o, leader);
    }
    __syncthreads();
    // one global reservation per key; the table empties for the next call
    // (which writes base only after its own first barrier)
    for (uint32_t t = threadIdx.x; t < kBlockLeaves; t += blockDim.x) {
        if (b.key[t] != kNone) b.base[t] = atomicAdd(&counters[b.key[t]], b.cnt[t]);
        b.key[t] = kNone;
        b.cnt[t] = 0;
    }
    __syncthreads();
#pragma unroll
    for (uint32_t j = 0; j < kEntriesPerThread; j++)
        out[j] = key[j] == kNone ? kNone : (at[j] != kNone ? b.base[at[j]] : 0u) + off[j] + rank[j];
}

// Sets the new cells' bits and gives each new voxel its slot in its node
// (sampleVoxel :119-138). Keys are unique, so every bit is set exactly once.
// A thread takes kEntriesPerThread list entries (a block's entries in steps of
// blockDim.x) and issues each step's loads for all of them before using any,
// so one iteration waits on three rounds of memory instead of three per entry.
__global__ void __launch_bounds__(256) k_vox_commit(Dev d) {
    __shared__ BlockSlots s_slots;
    const Counters* c = d.ctr;
    if (c->batchStop) return;
    blockSlotsInit(s_slots);
    __syncthreads();
    const uint32_t nnew = newCellCount(d);
    const uint32_t per = (((nnew + gridDim.x - 1u) / gridDim.x) + 31u) & ~31u;
    const uint32_t begin = min(nnew, blockIdx.x * per), end = min(nnew, begin + per);
    for (uint32_t base = begin; base < end; base += blockDim.x * kEntriesPerThread) {
        uint32_t e[kEntriesPerThread], slot[kEntriesPerThread], node[kEntriesPerThread];
        ulonglong2 kv[kEntriesPerThread];
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++) {
            e[j] = base + j * blockDim.x + threadIdx.x;
            slot[j] = e[j] < end ? d.hashNew[e[j]] : kNone;
        }
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++)
            kv[j] = slot[j] != kNone ? d.hashSlots[slot[j]] : make_ulonglong2(kHashEmpty, 0ull);
        uint32_t g[kEntriesPerThread];
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++) {
            node[j] = kNone;
            g[j] = 0;
            if (slot[j] != kNone) {
                // the table is final here: move the cell out of it and free the slot
                d.hashSlots[slot[j]] = make_ulonglong2(kHashEmpty, kHashEmpty);
                node[j] = (uint32_t)(kv[j].x >> 21);
                g[j] = d.grid[node[j]];
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++) {
            if (node[j] == kNone) continue;
            const uint32_t vi = (uint32_t)(kv[j].x & 0x1FFFFFull);
            atomicOr(gridWordsAt(d, g[j]) + (vi >> 5), 1u << (vi & 31u));
            d.hashNewNode[e[j]] = node[j];
            d.hashNewCell[e[j]] = vi;
            d.hashNewColor[e[j]] = (uint32_t)(kv[j].y & 0xFFFFFFFFull);
        }
        uint32_t s[kEntriesPerThread];
        blockReserveMany(s_slots, d.numVoxels, node, s);
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++)
            if (node[j] != kNone) d.hashNewSlot[e[j]] = s[j];
    }
}

// Grows a node's chunk table to hold `need` entries, keeping the first `keep`.
__device__ bool ensureTable(const Dev& d, uint32_t* offArr, uint32_t* capArr, uint32_t node,
                            uint32_t need, uint32_t keep) {
    const uint32_t cap = capArr[node];
    if (need <= cap) return true;
    uint32_t ncap = 64u;
    while (ncap < need) ncap <<= 1;
    const uint32_t off = atomicAdd(&d.ctr->tableBump, ncap);
    if ((uint64_t)off + ncap > d.tablePoolCap) {
        atomicOr(&d.ctr->overflowFlags, (uint32_t)kOvfTables);
        return false;
    }
    const uint32_t old = offArr[node];
    for (uint32_t j = 0; j < keep && old != kNone; j++) d.tablePool[off + j] = d.tablePool[old + j];
    offArr[node] = off;
    capArr[node] = ncap;
    return true;
}

__device__ __forceinline__ bool isLeaf(const Dev& d, uint32_t node) {
    const int4* row = reinterpret_cast<const int4*>(d.child + node * 8u);
    const int4 a = row[0], b = row[1];
    return (a.x & a.y & a.z & a.w & b.x & b.y & b.z & b.w) == -1;
}

__device__ __forceinline__ void markDirty(const Dev& d, uint32_t node) {
    Counters* c = d.ctr;
    if (d.dirtyStamp[node] == c->buildStamp) return;
    d.dirtyStamp[node] = c->buildStamp;
    const uint32_t di = atomicAdd(&c->numDirty, 1u);
    if (di < d.maxNodes) d.dirtyList[di] = node;
    else atomicOr(&c->overflowFlags, (uint32_t)kOvfDirty);
}

// allocatePointChunks (remolod_octree.cu:742-792), one thread per node. Chunk
// ids come from the recycled queue first, then from the pool; the reference
// store's offset advances by one chunk for every pool chunk, so
// memCapacityReached falls where it would. It runs beside the voxel path
// (k_vox_sample .. k_vox_store): the two share only the arena and table-pool
// bump counters and the store offset, all advanced by atomics.
__global__ void __launch_bounds__(256) k_alloc_points(Dev d) {
    Counters* c = d.ctr;
    if (c->batchStop) return;
    const uint32_t nn = c->numNodes;
    const uint32_t poolBefore = c->chunkPoolSize;
    const uint32_t ppc = d.ppc;
    // A leaf's counter is its stored points plus this batch's arrivals while
    // every leaf is counted in the batch it is made in (the reference's rule
    // sizes by the counter). Once an expand loop stopped at its pass limit,
    // the need is the larger of the counter and the points that reach it.
    const bool arrivals = c->arrivalMode != 0u || c->iter > d.maxExpandIters;
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < nn;
         node += gridDim.x * blockDim.x) {
        const uint32_t npts = d.numPoints[node];
        uint32_t cnt = d.counter[node];
        if (arrivals) {
            const uint32_t reach = npts + d.arrive[node];
            d.arrive[node] = 0;
            if (reach > cnt) cnt = reach;
        }
        if (npts < cnt && isLeaf(d, node)) {
            const uint32_t req = (cnt + ppc - 1u) / ppc;
            const uint32_t ex = (npts + ppc - 1u) / ppc;
            if (req > ex && ensureTable(d, d.ptTableOff, d.ptTableCap, node, req, ex)) {
                const uint32_t off = d.ptTableOff[node];
                const uint32_t extra = req - ex;
                // logical queue positions [idx0, idx0 + extra): recycled below
                // poolBefore, fresh from the arena at and above it
                const uint32_t idx0 = atomicAdd(&c->numAllocatedChunks, extra);
                const uint32_t firstFresh = idx0 > poolBefore ? idx0 : poolBefore;
                const uint32_t fresh = idx0 + extra > firstFresh ? idx0 + extra - firstFresh : 0u;
                uint32_t freshBase = kNone;
                if (fresh) {
                    freshBase = arenaAlloc(d, fresh * d.ptChunkUnits);
                    atomicAdd(&c->numPtChunks, fresh);
                    atomicAdd(reinterpret_cast<unsigned long long*>(&c->refOffset),
                              (unsigned long long)fresh * refAllocSize(kRefChunkBytes));
                }
                for (uint32_t e = 0; e < extra; e++) {
                    const uint32_t idx = idx0 + e;
                    uint32_t phys;
                    if (idx < poolBefore) {
                        phys = idx < d.maxPtChunks ? d.chunkQueue[idx] : kNone;
                    } else {
                        phys = freshBase == kNone ? kNone : freshBase + (idx - firstFresh) * d.ptChunkUnits;
                    }
                    d.tablePool[off + ex + e] = phys;
                }
                d.numPointChunks[node] = req;
            }
            markDirty(d, node);
        }
    }
}

// allocateVoxelChunks (:885-916), one thread per node, after k_vox_commit
// has counted the batch's new voxels.
__global__ void __launch_bounds__(256) k_alloc_voxels(Dev d) {
    Counters* c = d.ctr;
    if (c->batchStop) return;
    const uint32_t nn = c->numNodes;
    const uint32_t ppc = d.ppc;
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < nn;
         node += gridDim.x * blockDim.x) {
        const uint32_t nv = d.numVoxels[node];
        const uint32_t reqv = (nv + ppc - 1u) / ppc;
        const uint32_t havev = d.numVoxelChunks[node];
        if (reqv > havev && ensureTable(d, d.vxTableOff, d.vxTableCap, node, reqv, havev)) {
            const uint32_t off = d.vxTableOff[node];
            const uint32_t extra = reqv - havev;
            const uint32_t base = arenaAlloc(d, extra * d.vxChunkUnits);
            atomicAdd(&c->numVxChunks, extra);
            atomicAdd(reinterpret_cast<unsigned long long*>(&c->refOffset),
                      (unsigned long long)extra * refAllocSize(kRefChunkBytes));
            for (uint32_t e = 0; e < extra; e++)
                d.tablePool[off + havev + e] = base == kNone ? kNone : base + e * d.vxChunkUnits;
            d.numVoxelChunks[node] = reqv;
        }
        // every new voxel of this batch is stored by k_vox_store (insertVoxels, :918-938)
        d.numVoxelsStored[node] = nv;
    }
}

// insertPoints (remolod_octree.cu:794-883): batch points, then spilled points,
// each into the leaf expand left it in. Slots are handed out per warp and leaf.
__global__ void __launch_bounds__(256) k_insert(Dev d, const Point* __restrict__ pts, uint32_t n) {
    __shared__ BlockSlots s_slots;
    Counters* c = d.ctr;
    if (c->batchStop) return;
    RB_BATCH_AT_CURSOR(d, pts, n);
    blockSlotsInit(s_slots);
    __syncthreads();
    const uint32_t ns = c->numSpilled < d.spillCap ? c->numSpilled : d.spillCap;
    const uint32_t total = n + ns;
    const uint32_t firstIndex = (uint32_t)c->numPointsProcessed;
    const uint32_t ppc = d.ppc;
    const uint32_t per = (((total + gridDim.x - 1u) / gridDim.x) + 31u) & ~31u;
    const uint32_t begin = min(total, blockIdx.x * per), end = min(total, begin + per);
    for (uint32_t base = begin; base < end; base += blockDim.x * kEntriesPerThread) {
        uint32_t leaf[kEntriesPerThread], gidx[kEntriesPerThread];
        Point p[kEntriesPerThread];
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++) {
            const uint32_t i = base + j * blockDim.x + threadIdx.x;
            leaf[j] = kNone;
            gidx[j] = 0;
            p[j] = Point{0.f, 0.f, 0.f, 0u};
            if (i >= end) {
            } else if (i < n) {
                leaf[j] = d.leafOf[i];
                p[j] = loadPoint(pts + i);
                gidx[j] = firstIndex + i;
            } else {
                leaf[j] = d.spillLeaf[i - n];
                p[j] = d.spillPts[i - n];
                gidx[j] = d.spillIdx[i - n];
            }
        }
        uint32_t slot[kEntriesPerThread];
        blockReserveMany(s_slots, d.numPoints, leaf, slot);
        uint32_t cap[kEntriesPerThread], off[kEntriesPerThread];
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++) {
            cap[j] = 0;
            off[j] = 0;
            if (leaf[j] != kNone) {
                cap[j] = d.numPointChunks[leaf[j]] * ppc;
                off[j] = d.ptTableOff[leaf[j]];
            }
        }
        uint32_t phys[kEntriesPerThread];
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++)
            phys[j] = (leaf[j] != kNone && slot[j] < cap[j]) ? d.tablePool[off[j] + slot[j] / ppc] : kNone;
#pragma unroll
        for (uint32_t j = 0; j < kEntriesPerThread; j++) {
            if (leaf[j] == kNone) continue;
            if (phys[j] == kNone) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&c->droppedPoints), 1ull);
                continue;
            }
            chunkPoints(d, phys[j])[slot[j] % ppc] = p[j];
            chunkIndices(d, phys[j])[slot[j] % ppc] = gidx[j];
        }
    }
}

// insertVoxels (remolod_octree.cu:918-938): every new cell's voxel at its cell
// centre (:124-134) with its representative's colour, from the compact lists
// k_vox_commit made.
__global__ void __launch_bounds__(256) k_vox_store(Dev d) {
    const Counters* c = d.ctr;
    if (c->batchStop) return;
    const uint32_t nnew = newCellCount(d);
    const uint32_t ppc = d.ppc;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < nnew; e += gridDim.x * blockDim.x) {
        const uint32_t node = d.hashNewNode[e];
        const uint32_t s = d.hashNewSlot[e];
        const uint32_t vi = d.hashNewCell[e];
        const uint32_t px = vi & 127u, py = (vi >> 7) & 127u, pz = vi >> 14;
        const uint32_t lv = d.level[node];
        const float nodeSize = __fdiv_rn(d.octreeSize, __int_as_float((int)((127u + lv) << 23)));
        const float mnx = __fmaf_rn((float)d.nodeX[node], nodeSize, d.boxMin[0]);
        const float mny = __fmaf_rn((float)d.nodeY[node], nodeSize, d.boxMin[1]);
        const float mnz = __fmaf_rn((float)d.nodeZ[node], nodeSize, d.boxMin[2]);
        Point v;
        v.x = __fadd_rn(mnx, __fdiv_rn(__fmul_rn(nodeSize, __fadd_rn((float)px, 0.5f)), 128.0f));
        v.y = __fadd_rn(mny, __fdiv_rn(__fmul_rn(nodeSize, __fadd_rn((float)py, 0.5f)), 128.0f));
        v.z = __fadd_rn(mnz, __fdiv_rn(__fmul_rn(nodeSize, __fadd_rn((float)pz, 0.5f)), 128.0f));
        v.color = d.hashNewColor[e];
        if (s < d.numVoxelChunks[node] * ppc) {
            const uint32_t phys = d.tablePool[d.vxTableOff[node] + s / ppc];
            if (phys != kNone) chunkPoints(d, phys)[s % ppc] = v;
        }
    }
    // new cells beyond the list's capacity left entries that k_vox_commit
    // could not name: empty the whole table for the next batch
    if (c->hashNeedsClear) {
        const uint32_t size = d.hashMask + 1u;
        const ulonglong2 empty = make_ulonglong2(kHashEmpty, kHashEmpty);
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x)
            d.hashSlots[i] = empty;
    }
}

// Refinement's deepening (wiki/02_KernelPipeline.md:228-243: "local split and
// redistribute", listed by the reference and not built there), begun like a
// batch with no points: the memory check of a batch (remolod_octree.cu:1181-1210),
// the per-batch state, then the leaves among the first `budget` queue entries
// above the deepest level with at least minPoints stored points become this
// pass's spilling nodes, in queue order. The batch kernels that follow (the expand round from
// k_deep_book, or the per-iteration passes) split them as doSplitting would:
// 8 consecutive ids each in increasing id, the pool guard refusing once fewer
// than 8 remain (:318-321), their stored points to the spill list and their
// chunks to the queue; voxel sampling gives each its voxels; insertion puts the
// points into the children. One block.
__global__ void __launch_bounds__(1024) k_deepen_begin(Dev d, const uint32_t* queue, uint32_t queueLen,
                                                         uint32_t budget, uint32_t minPoints) {
    __shared__ uint32_t s_warp[32];
    Counters* c = d.ctr;
    if (threadIdx.x == 0) {
        const bool full = c->refOffset + d.safetyMargin >= d.persistentCapacity;
        c->memCapacityReached = full ? 1u : 0u;
        c->batchStop = full ? 1u : 0u;
        c->stopReason = full ? kStopMemory : 0u;
        resetBatchCounters(c);
        c->curN = 0;
        c->deepenSelected = 0;
    }
    __syncthreads();
    if (c->batchStop) return;
    const uint32_t k = budget < queueLen ? budget : queueLen;
    const uint32_t minPts = minPoints > 0u ? minPoints : 1u;
    uint32_t count = 0;
    for (uint32_t b = 0; b < k; b += blockDim.x) {
        const uint32_t i = b + threadIdx.x;
        uint32_t node = kNone, take = 0;
        if (i < k) {
            node = queue[i];
            take = node < c->numNodes && isLeaf(d, node) && d.level[node] < (uint32_t)kMaxDepth &&
                           d.numPoints[node] >= minPts
                       ? 1u
                       : 0u;
        }
        uint32_t tot;
        const uint32_t pre = blockExclusiveScan(take, &tot, s_warp);
        if (take && count + pre < d.spillingCap) d.spillNodes[count + pre] = node;
        count += tot;
    }
    if (threadIdx.x == 0) {
        const uint32_t sel = count < d.spillingCap ? count : d.spillingCap;
        if (count > d.spillingCap) atomicOr(&c->overflowFlags, (uint32_t)kOvfSpilling);
        c->numSpill = sel;
        c->deepenSelected = sel;
    }
}

// The end of a deepening pass: a batch's bookkeeping without a batch (the
// batch index and the points processed stay).
__global__ void k_deepen_end(Dev d) {
    Counters* c = d.ctr;
    if (c->batchStop) return;
    if (c->numAllocatedChunks > c->chunkPoolSize) c->chunkPoolSize = c->numAllocatedChunks;
    c->spilledPointsTotal += c->numSpilled;
    if (c->iter > d.maxExpandIters) c->arrivalMode = 1u;
    settleGridPool(c);
}

// Refinement's collapsing (wiki/02_KernelPipeline.md:228-243, "merge a node
// back up", listed by the reference and not built there: it needs somewhere
// to return the 256 KB grid, CLAUDE.md:185-187). A node whose eight children
// are all leaves, holding at most maxPoints points between them, becomes a
// leaf again with all their points: its chunks are allocated first (recycled
// queue chunks, then fresh ones, charged as a batch's are), the children's
// points are copied in, then the children's chunks return to the queue, the
// children become empty unreachable leaves (the pool only grows, as the
// reference's does), the node drops its voxels (their chunks are not reused)
// and its grid goes to the grid pool, where the next split takes it. The
// node's exact sums restart from zero and it is marked dirty, so Accumulate
// folds all its points. Candidates come from the caller (d.spillNodes).
constexpr uint32_t kCollapseMax = 4096;

// Sorts the candidates, drops duplicates and ineligible nodes, books each
// merged leaf's chunks. One block. Records in splitRecs: node, numPoints (its
// points), chunkBase (its first copy item), numChunks (its children's chunks),
// grid, queueBase (its first allocation index), spillBase (chunks it needs).
__global__ void __launch_bounds__(1024) k_collapse_plan(Dev d, uint32_t count, uint32_t maxPoints) {
    __shared__ uint32_t s_ids[kCollapseMax];
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_fresh;
    Counters* c = d.ctr;
    const uint32_t n = count < kCollapseMax ? count : kCollapseMax;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) s_ids[i] = d.spillNodes[i];
    __syncthreads();
    bitonicSort(s_ids, n);
    const uint32_t nn = c->numNodes, ppc = d.ppc;
    const uint32_t maxPts = maxPoints ? maxPoints : d.maxPointsPerNode;
    uint32_t sel = 0, reqRun = 0, ownRun = 0;
    for (uint32_t b = 0; b < n; b += blockDim.x) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t node = i < n ? s_ids[i] : kNone;
        uint32_t take = 0, total = 0, owned = 0;
        if (node < nn && (i == 0 || s_ids[i - 1] != node) && d.level[node] > 0u && !isLeaf(d, node)) {
            take = 1;
            for (uint32_t q = 0; q < 8u; q++) {
                const int32_t ch = d.child[node * 8u + q];
                if (ch < 0 || (uint32_t)ch >= nn || !isLeaf(d, (uint32_t)ch)) {
                    take = 0;
                    break;
                }
                const uint32_t oc = d.numPointChunks[ch], np = d.numPoints[ch];
                total += np < oc * ppc ? np : oc * ppc;
                owned += oc;
            }
            if (total > maxPts) take = 0;
        }
        const uint32_t req = take ? (total + ppc - 1u) / ppc : 0u;
        uint32_t tSel, tReq, tOwn;
        const uint32_t pSel = blockExclusiveScan(take, &tSel, s_warp);
        const uint32_t pReq = blockExclusiveScan(req, &tReq, s_warp);
        const uint32_t pOwn = blockExclusiveScan(take ? owned : 0u, &tOwn, s_warp);
        if (take) {
            SplitRec r;
            r.node = node;
            r.numPoints = total;
            r.tableOff = kNone;
            r.spillBase = req;
            r.chunkBase = ownRun + pOwn;
            r.numChunks = owned;
            r.grid = d.grid[node];
            r.queueBase = reqRun + pReq;
            d.splitRecs[sel + pSel] = r;
            atomicAdd(&c->collapsePoints, (unsigned long long)total);
        }
        sel += tSel;
        reqRun += tReq;
        ownRun += tOwn;
    }
    // the merged leaves' chunks: logical queue positions [A, A + reqRun),
    // recycled below the pool's size, fresh from the arena at and above it
    const uint32_t A = c->numAllocatedChunks, pool = c->chunkPoolSize;
    const uint32_t firstFresh = A > pool ? A : pool;
    const uint32_t fresh = A + reqRun > firstFresh ? A + reqRun - firstFresh : 0u;
    if (threadIdx.x == 0) {
        s_fresh = kNone;
        if (fresh) {
            s_fresh = arenaAlloc(d, fresh * d.ptChunkUnits);
            atomicAdd(&c->numPtChunks, fresh);
            c->refOffset += (unsigned long long)fresh * refAllocSize(kRefChunkBytes);
        }
        c->collapseSelected = sel;
        c->collapseItems = ownRun;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < sel; k += blockDim.x) {
        const SplitRec r = d.splitRecs[k];
        const uint32_t req = r.spillBase;
        if (req && ensureTable(d, d.ptTableOff, d.ptTableCap, r.node, req, 0u)) {
            const uint32_t off = d.ptTableOff[r.node];
            for (uint32_t e = 0; e < req; e++) {
                const uint32_t idx = A + r.queueBase + e;
                uint32_t phys;
                if (idx < pool) phys = idx < d.maxPtChunks ? d.chunkQueue[idx] : kNone;
                else phys = s_fresh == kNone ? kNone : s_fresh + (idx - firstFresh) * d.ptChunkUnits;
                d.tablePool[off + e] = phys;
            }
            d.numPointChunks[r.node] = req;
        }
        d.numPoints[r.node] = r.numPoints;
        d.counter[r.node] = r.numPoints;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        c->numAllocatedChunks = A + reqRun;
        if (c->numAllocatedChunks > c->chunkPoolSize) c->chunkPoolSize = c->numAllocatedChunks;
    }
}

// The children's points into the merged leaves: one work item per child
// chunk, the destination slot the child's offset among its siblings plus the
// slot in the child. The children's tables are intact until k_collapse_finish.
__global__ void __launch_bounds__(256) k_collapse_copy(Dev d) {
    const Counters* c = d.ctr;
    const uint32_t sel = c->collapseSelected, items = c->collapseItems, ppc = d.ppc;
    for (uint32_t w = blockIdx.x; w < items; w += gridDim.x) {
        uint32_t lo = 0, hi = sel;
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (d.splitRecs[mid].chunkBase <= w) lo = mid;
            else hi = mid;
        }
        const SplitRec r = d.splitRecs[lo];
        uint32_t j = w - r.chunkBase, base = 0, ch = kNone;
        for (uint32_t q = 0; q < 8u; q++) {
            const uint32_t cq = (uint32_t)d.child[r.node * 8u + q];
            const uint32_t oc = d.numPointChunks[cq];
            if (j < oc) {
                ch = cq;
                break;
            }
            j -= oc;
            const uint32_t np = d.numPoints[cq];
            base += np < oc * ppc ? np : oc * ppc;
        }
        if (ch == kNone) continue;
        const uint32_t oc = d.numPointChunks[ch];
        const uint32_t np = d.numPoints[ch] < oc * ppc ? d.numPoints[ch] : oc * ppc;
        const uint32_t first = j * ppc, last = first + ppc < np ? first + ppc : np;
        const uint32_t src = d.tablePool[d.ptTableOff[ch] + j];
        const uint32_t dcap = d.numPointChunks[r.node] * ppc;
        if (src == kNone) continue;
        for (uint32_t s = first + threadIdx.x; s < last; s += blockDim.x) {
            const uint32_t slot = base + s;
            if (slot >= dcap) continue;
            const uint32_t dst = d.tablePool[d.ptTableOff[r.node] + slot / ppc];
            if (dst == kNone) continue;
            chunkPoints(d, dst)[slot % ppc] = chunkPoints(d, src)[s - first];
            chunkIndices(d, dst)[slot % ppc] = chunkIndices(d, src)[s - first];
        }
    }
}

// The children's chunks back to the queue (after the merged leaves took
// theirs), the children emptied, the merged nodes' voxels dropped and their
// grids into the pool; dirty marks for Accumulate. One block.
__global__ void __launch_bounds__(1024) k_collapse_finish(Dev d) {
    Counters* c = d.ctr;
    const uint32_t sel = c->collapseSelected, own = c->collapseItems;
    const uint32_t A = c->numAllocatedChunks, qbase = A - own;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < sel; k += blockDim.x) {
        const SplitRec r = d.splitRecs[k];
        uint32_t pos = qbase + r.chunkBase;
        AccumI z = {};
        for (uint32_t q = 0; q < 8u; q++) {
            const uint32_t ch = (uint32_t)d.child[r.node * 8u + q];
            const uint32_t oc = d.numPointChunks[ch];
            for (uint32_t j = 0; j < oc; j++, pos++)
                if (pos < d.maxPtChunks) d.chunkQueue[pos] = d.tablePool[d.ptTableOff[ch] + j];
            d.numPoints[ch] = 0;
            d.counter[ch] = 0;
            d.numPointChunks[ch] = 0;
            d.ptTableOff[ch] = kNone;
            d.ptTableCap[ch] = 0;
            d.accum[ch] = z;
            d.child[r.node * 8u + q] = -1;
        }
        atomicAdd(&c->collapseVoxels, (unsigned long long)d.numVoxels[r.node]);
        d.numVoxels[r.node] = 0;
        d.numVoxelsStored[r.node] = 0;
        d.numVoxelChunks[r.node] = 0;
        d.vxTableOff[r.node] = kNone;
        d.vxTableCap[r.node] = 0;
        d.splitIter[r.node] = 0;
        d.accum[r.node] = z;
        if (r.grid != kNone) {
            d.gridPool[atomicAdd(&c->gridPoolSize, 1u)] = r.grid;
            d.grid[r.node] = kNone;
            atomicSub(&c->numGrids, 1u);
        }
        markDirty(d, r.node);
    }
    __syncthreads();
    if (threadIdx.x == 0) c->numAllocatedChunks = qbase;
}

// n == kNone: the batch at the device cursor.
__global__ void k_batch_end(Dev d, uint32_t n) {
    Counters* c = d.ctr;
    if (c->batchStop) return;
    if (n == kNone) n = c->curN;
    c->callBatches += 1;
    if (c->numAllocatedChunks > c->chunkPoolSize) c->chunkPoolSize = c->numAllocatedChunks;
    c->batchletIndex += 1;
    c->numPointsProcessed += n;
    c->spilledPointsTotal += c->numSpilled;
    c->expandIters += c->iter < d.maxExpandIters ? c->iter : d.maxExpandIters;
    if (c->iter > d.maxExpandIters) c->arrivalMode = 1u;
    settleGridPool(c);
}

// Stats sweep (remolod_octree.cu:1271-1310).
__global__ void __launch_bounds__(256) k_sweep(Dev d) {
    const uint32_t nn = d.ctr->numNodes;
    const uint32_t ppc = d.ppc;
    SweepStats* s = d.sweep;
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < nn;
         node += gridDim.x * blockDim.x) {
        const uint32_t np = d.numPoints[node];
        const uint32_t lv = d.level[node];
        atomicMax(&s->maxLevel, lv);
        if (isLeaf(d, node)) {
            atomicAdd(&s->numLeaves, 1u);
            atomicAdd(&s->numPoints, (unsigned long long)np);
            atomicAdd(&s->numChunksPoints, (np + ppc - 1u) / ppc);
            atomicMax(&s->maxPointsPerNode, np);
            if (d.counter[node] < np) atomicAdd(&s->counterUnderflows, 1u);
            if (np > 0) atomicAdd(&s->numNonemptyLeaves, 1u);
        } else {
            const uint32_t nv = d.numVoxels[node];
            atomicAdd(&s->numInner, 1u);
            atomicAdd(&s->numVoxels, (unsigned long long)nv);
            atomicAdd(&s->numChunksVoxels, (nv + ppc - 1u) / ppc);
        }
    }
}

// reset (remolod_reset.cu:41-85): the root, its grid, and the counters.
__global__ void k_reset_root(Dev d) {
    Counters* c = d.ctr;
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        Counters z = {};
        z.buildStamp = c->buildStamp;
        *c = z;
        c->refOffset = 16;
        c->numNodes = 1;
        for (int q = 0; q < 8; q++) d.child[q] = -1;
        d.counter[0] = 0;
        d.numPoints[0] = 0;
        d.level[0] = 0;
        d.nodeX[0] = d.nodeY[0] = d.nodeZ[0] = 0;
        d.grid[0] = 0;  // the root grid is the arena's first allocation
        d.numVoxels[0] = 0;
        d.numVoxelsStored[0] = 0;
        d.numPointChunks[0] = 0;
        d.numVoxelChunks[0] = 0;
        d.ptTableOff[0] = kNone;
        d.ptTableCap[0] = 0;
        d.vxTableOff[0] = kNone;
        d.vxTableCap[0] = 0;
        d.splitIter[0] = 0;
        d.dirtyStamp[0] = 0;
        AccumI za = {};
        d.accum[0] = za;
        c->arenaBump = kGridUnits;
        c->numGrids = 1;
        c->refOffset += refAllocSize(kGridBytes);
    }
    uint4* g = reinterpret_cast<uint4*>(gridWordsAt(d, 0));
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < kGridWords / 4u;
         q += gridDim.x * blockDim.x)
        g[q] = z;
}

// ------------------------------------------------------------------ launches

void launchBatchBegin(const Dev& d, cudaStream_t s) { k_batch_begin<<<1, 1, 0, s>>>(d, 0u); }
void launchDeepenBegin(const Dev& d, const uint32_t* queue, uint32_t queueLen, uint32_t budget, uint32_t minPoints,
                       cudaStream_t s) {
    k_deepen_begin<<<1, 1024, 0, s>>>(d, queue, queueLen, budget, minPoints);
}
void launchDeepenEnd(const Dev& d, cudaStream_t s) { k_deepen_end<<<1, 1, 0, s>>>(d); }
void launchCollapse(const Dev& d, uint32_t count, uint32_t maxPoints, int grid, cudaStream_t s) {
    k_collapse_plan<<<1, 1024, 0, s>>>(d, count, maxPoints);
    k_collapse_copy<<<grid, 256, 0, s>>>(d);
    k_collapse_finish<<<1, 1024, 0, s>>>(d);
}
void launchCountFirst(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s) {
    k_count_first<<<grid, 256, 0, s>>>(d, pts, n);
}
void launchRecount(const Dev& d, const Point* pts, uint32_t n, uint32_t prevStamp, int grid,
                   cudaStream_t s) {
    k_recount<<<grid, 256, 0, s>>>(d, pts, n, prevStamp, 0u);
}
void launchSplit(const Dev& d, uint32_t stamp, cudaStream_t s) { k_split<<<1, 1024, 0, s>>>(d, stamp, 0u); }
void launchExpandCond(const Dev& d, cudaStream_t s) { k_expand_cond<<<1, 1024, 0, s>>>(d, 0ull, 0u); }
void launchSpillCopy(const Dev& d, int grid, cudaStream_t s) { k_spill_copy<<<grid, 256, 0, s>>>(d, 0u); }
void launchZeroGrids(const Dev& d, int grid, cudaStream_t s) { k_zero_grids<<<grid, 256, 0, s>>>(d); }
void launchDeepBook(const Dev& d, cudaStream_t s) { k_deep_book<<<1, 1024, 0, s>>>(d); }
void launchDeepBin(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s) {
    k_deep_bin<<<grid, 256, 0, s>>>(d, pts, n);
}
void launchDeepSplit(const Dev& d, cudaStream_t s) { k_deep_split<<<1, 1024, 0, s>>>(d); }
void launchDeepMove(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s) {
    k_deep_move<<<grid, 256, 0, s>>>(d, pts, n);
}

// k_expand_rest's cooperative grid: every block resident at once.
cudaError_t expandRestGrid(int numSMs, int* grid) {
    int perSM = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_expand_rest, 1024, 0);
    if (e != cudaSuccess) return e;
    if (perSM < 1) return cudaErrorCooperativeLaunchTooLarge;
    *grid = numSMs;  // one block per SM is all the passes need
    return cudaSuccess;
}

cudaError_t launchExpandRest(const Dev& d, int grid, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(1024);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_expand_rest, d);
}
void launchVoxSample(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s) {
    k_vox_sample<<<grid, 256, 0, s>>>(d, pts, n);
}
void launchVoxLift(const Dev& d, int grid, cudaStream_t s) { k_vox_lift<<<grid, kLiftThreads, 0, s>>>(d); }
void launchVoxSampleLevels(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s) {
    k_vox_sample_levels<<<grid, 256, 0, s>>>(d, pts, n);
}
void launchVoxCommit(const Dev& d, int grid, cudaStream_t s) { k_vox_commit<<<grid, 256, 0, s>>>(d); }
void launchFinishLeaves(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s) {
    k_finish_leaves<<<grid, 256, 0, s>>>(d, pts, n);
}
void launchAllocPoints(const Dev& d, int grid, cudaStream_t s) { k_alloc_points<<<grid, 256, 0, s>>>(d); }
void launchAllocVoxels(const Dev& d, int grid, cudaStream_t s) { k_alloc_voxels<<<grid, 256, 0, s>>>(d); }
void launchInsert(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s) {
    k_insert<<<grid, 256, 0, s>>>(d, pts, n);
}
void launchVoxStore(const Dev& d, int grid, cudaStream_t s) { k_vox_store<<<grid, 256, 0, s>>>(d); }
void launchBatchEnd(const Dev& d, uint32_t n, cudaStream_t s) { k_batch_end<<<1, 1, 0, s>>>(d, n); }
void launchSweep(const Dev& d, int grid, cudaStream_t s) { k_sweep<<<grid, 256, 0, s>>>(d); }
void launchResetRoot(const Dev& d, int grid, cudaStream_t s) { k_reset_root<<<grid, 256, 0, s>>>(d); }

// One batch as a CUDA graph: the phase kernels of runBatch, every kernel
// reading its batch from the device cursor, the expand round's leftovers in
// the cooperative k_expand_rest. After it the graph forks: the voxel path
// (k_vox_sample, or after a lost cell k_vox_sample_levels on a branch of its
// own; k_vox_lift, k_vox_commit, k_alloc_voxels, k_vox_store) and the point path
// (k_alloc_points, k_insert) read the finished tree and write disjoint node
// fields and chunks, so the point path runs in the voxel path's shadow; they
// join before k_batch_end. One graph launch builds the batch at batchletIndex
// with no host round trip and no conditional node; a stopped batch (memory,
// no batch uploaded, time budget) runs through as no-ops.
cudaError_t captureBatchGraph(const Dev& d, int pointGrid, int fixedGrid, int restGrid, cudaGraphExec_t* out) {
    *out = nullptr;
    cudaStream_t cs = nullptr, cs2 = nullptr, cs3 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, joinLevels = nullptr;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs3, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&joinLevels, cudaEventDisableTiming);
    bool capturing = false;
    while (e == cudaSuccess) {
        if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) break;
        capturing = true;
        k_batch_begin<<<1, 1, 0, cs>>>(d, 1u);
        k_count_first<<<pointGrid, 256, 0, cs>>>(d, nullptr, 0u);
        k_deep_book<<<1, 1024, 0, cs>>>(d);
        k_deep_bin<<<pointGrid, 256, 0, cs>>>(d, nullptr, 0u);
        k_deep_split<<<1, 1024, 0, cs>>>(d);
        k_deep_move<<<pointGrid, 256, 0, cs>>>(d, nullptr, 0u);
        if ((e = launchExpandRest(d, restGrid, cs)) != cudaSuccess) break;
        if ((e = cudaEventRecord(fork, cs)) != cudaSuccess) break;
        if ((e = cudaStreamWaitEvent(cs2, fork, 0)) != cudaSuccess) break;
        k_alloc_points<<<fixedGrid, 256, 0, cs2>>>(d);
        k_insert<<<pointGrid, 256, 0, cs2>>>(d, nullptr, 0u);
        if ((e = cudaEventRecord(join, cs2)) != cudaSuccess) break;
        // the two forms of voxel sampling exclude each other (Counters::levelMode):
        // the one that returns at once runs beside the other, off the path
        if ((e = cudaStreamWaitEvent(cs3, fork, 0)) != cudaSuccess) break;
        k_vox_sample_levels<<<pointGrid, 256, 0, cs3>>>(d, nullptr, 0u);
        if ((e = cudaEventRecord(joinLevels, cs3)) != cudaSuccess) break;
        k_vox_sample<<<pointGrid, 256, 0, cs>>>(d, nullptr, 0u);
        if ((e = cudaStreamWaitEvent(cs, joinLevels, 0)) != cudaSuccess) break;
        k_vox_lift<<<pointGrid, kLiftThreads, 0, cs>>>(d);
        k_vox_commit<<<fixedGrid, 256, 0, cs>>>(d);
        k_alloc_voxels<<<fixedGrid, 256, 0, cs>>>(d);
        k_vox_store<<<fixedGrid, 256, 0, cs>>>(d);
        if ((e = cudaStreamWaitEvent(cs, join, 0)) != cudaSuccess) break;
        k_batch_end<<<1, 1, 0, cs>>>(d, kNone);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        capturing = false;
        if ((e = cudaStreamEndCapture(cs, &graph)) != cudaSuccess) break;
        e = cudaGraphInstantiate(out, graph, 0ull);
        break;
    }
    if (capturing) {
        cudaGraph_t dropped = nullptr;
        cudaStreamEndCapture(cs, &dropped);
        if (dropped) cudaGraphDestroy(dropped);
    }
    if (graph) cudaGraphDestroy(graph);
    if (join) cudaEventDestroy(join);
    if (joinLevels) cudaEventDestroy(joinLevels);
    if (fork) cudaEventDestroy(fork);
    if (cs2) cudaStreamDestroy(cs2);
    if (cs3) cudaStreamDestroy(cs3);
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
    }
    return e;
}

}  // namespace rb
