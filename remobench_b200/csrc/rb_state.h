// Device-side state of one LOD context: the node pool as structure-of-arrays,
// the chunk and grid pools, per-batch scratch and the counter block. Shared by
// every kernel translation unit and by the host orchestration in rb_capi.cu.
//
// Data model (restates kernels/remolod/remolod_structures.cuh:12-135 for the
// B200): nodes are integer ids into flat arrays, not pointers; a node's 8
// children are one 32-byte row of `child`, so a descent step is one sector
// load; a leaf's points live in 1000-point chunks reached through a per-node
// chunk table instead of a linked list, so slot s is table[s / 1000] with no
// walk (the reference walks the list from its head for every point,
// remolod_octree.cu:853-857).
#pragma once

#include <stdint.h>

#include <vector_types.h>

namespace rb {

constexpr int kMaxDepth = 20;                 // remolod_structures.cuh:18
constexpr uint32_t kGridSize = 128;           // :16
constexpr uint32_t kGridWords = 65536;        // 128^3 bits as 32-bit words (:66-68)
constexpr uint64_t kGridBytes = 262144ull;
constexpr uint64_t kRefChunkBytes = 16016ull; // sizeof(Chunk) in the reference (:59-64)
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint64_t kHashEmpty = ~0ull;

// AllocatorGlobal::alloc's rounding (kernels/simlod/utils.h.cu:195)
__host__ __device__ inline uint64_t refAllocSize(uint64_t size) {
    return 16ull * ((size + 16ull) / 16ull);
}

struct Point {
    float x, y, z;
    uint32_t color;
};

// Counter block, one per context, in device memory.
struct Counters {
    uint32_t numNodes;
    uint32_t arenaBump;         // arena units (16 B) handed out
    uint32_t numGrids;          // grids handed out
    uint32_t numPtChunks;       // point chunks ever taken from the arena
    uint32_t numVxChunks;       // voxel chunks ever taken from the arena
    uint32_t tableBump;         // chunk-table entries handed out
    uint32_t numAllocatedChunks;  // Stats::numAllocatedChunks (logical queue length)
    uint32_t chunkPoolSize;       // Stats::chunkPoolSize
    uint32_t batchletIndex;       // Stats::batchletIndex
    uint64_t numPointsProcessed;  // Stats::numPointsProcessed
    uint64_t refOffset;           // the reference store's AllocatorGlobal::offset
    // per batch
    uint32_t batchStop;           // memCapacityReached for this batch
    uint32_t iter;                // expand iteration being counted (1-based)
    uint32_t numSpill;            // spilling nodes found by the last count
    uint32_t numSplit;            // nodes split by the last split
    uint32_t numSpilled;          // spilled points this batch
    uint32_t numNew;              // new voxel cells this batch
    uint32_t numLift;             // new voxel cells k_vox_lift listed after numNew
    uint32_t levelMode;           // this batch samples voxels level by level (gridsPartial at its start)
    uint32_t deepenSelected;      // leaves a deepening pass took from the queue
    uint32_t collapseSelected;    // nodes a collapsing pass merges
    uint32_t collapseItems;       // their children's point chunks (copy and release work items)
    unsigned long long collapsePoints;  // points the pass moved into the merged leaves
    unsigned long long collapseVoxels;  // voxels the merged nodes dropped
    uint32_t gridPoolSize;        // grids collapsed nodes returned (Dev::gridPool), taken again by splits
    uint32_t gridPoolTaken;       // pool grids taken in this batch (settled at its end)
    uint32_t spillChunkTotal;     // copy work items of the last split
    uint32_t loopMore;            // the last loop test's answer: another expand pass
    // flags and diagnostics (sticky until reset)
    uint32_t memCapacityReached;
    uint32_t nodePoolOverflow;
    uint32_t gridsPartial;        // a batch lost new cells to a full list: later batches sample level by level
    uint32_t overflowFlags;       // RB_OVF_* bits
    uint32_t condSkips;           // unrolled expand passes skipped after the loop ended (wraps)
    uint64_t droppedPoints;
    uint64_t expandIters;
    uint64_t nodesSplit;
    uint64_t spilledPointsTotal;
    // dirty list for Accumulate
    uint32_t numDirty;
    uint32_t buildStamp;
    // device-driven batches: the batch being built, read by every phase kernel
    // launched without explicit points (pts == nullptr)
    uint32_t curN;
    unsigned long long curPts;    // device address of the batch's first point
    unsigned long long buildStartNs;  // %globaltimer at the start of the build call
    uint32_t lastStamp;           // splitIter stamp of the last split
    uint32_t stopReason;          // 0 none, kStopMemory, kStopNoBatch, kStopTime
    uint32_t expandGuard;         // expand passes of this batch (loop bound)
    uint32_t hashNeedsClear;      // the cell table holds entries its list cannot name
    uint32_t callBatches;         // batches built since the build call began
    uint32_t accumItems;          // work items of the current Accumulate launch
    uint32_t numZero;             // grids of nodes split this batch, to zero after expand
    uint32_t histValid;           // hist8 holds the child-octant counts of the nodes to split next
    uint32_t countLo, countHi;    // nodes [countLo, countHi) whose points the next recount counts
    uint32_t condRuns;            // runs of the expand loop's test since allocation (wraps)
    // the batch's multi-level expand round (rb_update.cu, k_deep_*): active
    // when its roots (the first count's spilling nodes) were booked
    uint32_t deepActive;
    uint32_t deepRoots;           // roots booked, in increasing id (slot order)
    uint32_t deepLevels;          // levels below the roots whose counts are binned
    uint32_t deepBase;            // id of the roots' first child
    uint32_t deepStamp;           // split stamp of the roots
    // grid barrier of the cooperative expand kernel (k_expand_rest), per batch
    uint32_t barArrive;
    uint32_t barRelease;
    // set by the first batch whose expand loop stopped at its pass limit
    // (until the next reset): its last split's nodes were not counted, so
    // leaves' counters may lag their points, and point chunks are sized from
    // the points that reach each leaf (Dev::arrive)
    uint32_t arrivalMode;
};

enum StopReason : uint32_t { kStopMemory = 1u, kStopNoBatch = 2u, kStopTime = 3u };

// Where batch b lives, for device-driven builds (PointSource's BatchView,
// include/remo/PointSource.h:43-67). Ring mode: slot b % numSlots holds
// sizes[slot] points. Stream mode (host ingest): batch b is the (b - first)-th
// of a run of total points cut into batchSize-point batches.
constexpr uint32_t kMaxRingSlots = 256;
struct RingDesc {
    unsigned long long base;      // device address of slot 0
    uint32_t slotCap;             // points per slot
    uint32_t numSlots;
    uint32_t numUploaded;         // batches [0, numUploaded) are readable
    uint32_t streamMode;          // 0 ring, 1 stream
    uint32_t first;               // stream mode: batch index of the run's first batch
    uint32_t batchSize;           // stream mode
    unsigned long long total;     // stream mode: points in the run
    unsigned long long budgetNs;  // device time budget of the call, 0 = none
    uint32_t sizes[kMaxRingSlots];
};

enum OverflowBits : uint32_t {
    kOvfSpilled = 1u,     // spill list full
    kOvfBacklog = 2u,     // voxel hash full or probe limit
    kOvfSpilling = 4u,    // spilling-node list full
    kOvfArena = 8u,       // arena full (grids and chunks)
    kOvfTables = 64u,     // chunk-table pool full
    kOvfDirty = 128u,     // dirty list full
    kOvfDrawList = 256u,  // render draw list full
    kOvfSync = 512u,      // a grid barrier gave up waiting (an error, not a capacity)
};

// One node split by the last split pass: where its stored points go.
struct SplitRec {
    uint32_t node;
    uint32_t numPoints;     // points stored before the split
    uint32_t tableOff;      // its point chunk table (kept readable for the copy)
    uint32_t spillBase;     // first spill slot of its points
    uint32_t chunkBase;     // first copy work item
    uint32_t numChunks;     // chunks it owned (copy and recycle work items)
    uint32_t grid;
    uint32_t queueBase;     // chunk-queue position of its first recycled chunk, kNone: none
};

// Exact integer sums of one node (see rb_accum.cu).
struct AccumI {
    unsigned long long s1[3];
    unsigned long long s2lo[6];
    unsigned long long s2hi[6];
    unsigned long long c1[3];
    unsigned long long c2[3];
    uint32_t count;
    uint32_t lastTouchedBatch;
    uint32_t state;
    uint32_t pad;
};

struct AccumGlobals {
    unsigned long long mortonWatermark;
    unsigned long long numAccumulated;
    unsigned long long sumLeafCounts;
    uint32_t pointsFolded;
    uint32_t numLeavesFolded;
    uint32_t innerWithSums;
    uint32_t pad;
};

// Stats sweep output (remolod_octree.cu:1271-1310).
struct SweepStats {
    uint32_t numInner, numLeaves, numNonemptyLeaves, maxPointsPerNode;
    unsigned long long numPoints, numVoxels;
    uint32_t numChunksPoints, numChunksVoxels, counterUnderflows, maxLevel;
};

// Everything a kernel needs, passed by value.
struct Dev {
    // node pool
    int32_t* child;          // [maxNodes * 8], -1: none
    uint32_t* counter;
    uint32_t* numPoints;
    uint32_t* level;
    uint32_t* nodeX;
    uint32_t* nodeY;
    uint32_t* nodeZ;
    uint32_t* grid;          // arena unit offset of the node's occupancy grid, kNone: none
    uint32_t* numVoxels;
    uint32_t* numVoxelsStored;
    uint32_t* numPointChunks;
    uint32_t* numVoxelChunks;
    uint32_t* ptTableOff;
    uint32_t* ptTableCap;
    uint32_t* vxTableOff;
    uint32_t* vxTableCap;
    uint32_t* splitIter;     // 1-based expand iteration of the split in this batch, 0: none
    // ancestors of every node, root first: row n holds (id, grid) of the nodes
    // at levels 0 .. level(n)-1 above n. Written once when n is created (its
    // ancestors are inner then and keep their grids), so one row gives every
    // grid a point of n must test, with no pointer chase.
    uint2* anc;              // [maxNodes * kMaxDepth]
    uint2* parent;           // [maxNodes] (id, grid) of the parent: row n of anc at level(n) - 1
    uint32_t* gridPool;      // [maxNodes] grids returned by collapsed nodes
    uint32_t* dirtyStamp;
    AccumI* accum;
    // storage: one arena in 16-byte units holding grids (256 KB), point chunks
    // (ppc points, then ppc global point indices) and voxel chunks (ppc voxels);
    // chunk tables and grid ids hold arena unit offsets
    uint8_t* arena;
    uint32_t* tablePool;
    uint32_t* chunkQueue;    // [maxPtChunks] recycled chunk ids (remolod_octree.cu:349-360)
    // per-batch scratch
    uint32_t* leafOf;        // [slotCapacity]
    Point* spillPts;         // [spillCap]
    uint32_t* spillIdx;
    uint32_t* spillLeaf;
    uint32_t* spillNodes;    // [spillingCap] nodes whose counter crossed the limit
    SplitRec* splitRecs;     // [spillingCap]
    // the batch's new-cell table: one 16-byte slot per cell, key (node << 21 |
    // cell) and value (global point index << 32 | colour) in the same sector
    ulonglong2* hashSlots;   // [hashMask + 1], kHashEmpty in both halves: free
    uint32_t* hashNew;       // [newCap] slots inserted this batch
    uint32_t* hashNewNode;   // node of each new cell
    uint32_t* hashNewSlot;   // slot of the new voxel within its node
    uint32_t* hashNewCell;   // cell index (x + 128 y + 16384 z) of each new cell
    uint32_t* hashNewColor;  // colour of its representative point
    uint32_t* dirtyList;     // [maxNodes]
    Counters* ctr;
    RingDesc* ring;
    SweepStats* sweep;
    AccumGlobals* accumGlobals;
    // Accumulate's plan: per visited node, its point range and first work item
    uint32_t* accumFrom;     // [maxNodes]
    uint32_t* accumTo;       // [maxNodes]
    uint32_t* accumItem;     // [maxNodes + 1] exclusive prefix of work items
    uint32_t* accumUnitW;    // [accumUnitCap] plan entry of each work item
    uint32_t accumUnitCap;   // point chunks + nodes: every fold's items fit
    uint32_t* zeroList;      // [zeroCap] grids to zero after the expand loop
    // per node, its points per child octant, counted by the recount for the
    // nodes made by the last split: one level of lookahead for the next split
    uint32_t* hist8;         // [maxNodes * 8]
    // per node, the batch's points whose leaf it is; counted after the expand
    // loop (finishLeavesBody) and cleared by k_alloc_points, in arrival mode
    // only (Counters::arrivalMode)
    uint32_t* arrive;        // [maxNodes]
    // multi-level expand round: per root slot, the points below it counted at
    // every depth 1..kDeepLevels ([kDeepRoots][kDeepCells]); per root node its
    // slot; per node made by the round, (slot << 16) | its code below the root;
    // per generation, the nodes split in id order
    uint32_t* deepCnt;
    uint32_t* deepNode;      // [kDeepRoots * kDeepCells] the node the round made for each cube, kNone elsewhere
    uint32_t* moveCode;      // [slot capacity] each binned batch point's cube code at the round's deepest depth
    uint32_t* spillCode;     // [spillCap] the same for the roots' stored points, by spill slot
    uint32_t* deepSlot;      // [maxNodes]
    uint32_t* deepMeta;      // [maxNodes]
    uint32_t* deepPar;       // [maxNodes / 8 + 1]
    uint32_t zeroCap;
    // capacities and constants
    uint32_t maxNodes;
    uint32_t maxPointsPerNode;
    uint32_t ppc;            // points per chunk
    uint32_t maxPtChunks;    // chunk queue capacity
    uint32_t arenaUnits;
    uint32_t ptChunkUnits;
    uint32_t vxChunkUnits;
    uint32_t tablePoolCap;
    uint32_t spillCap;
    uint32_t spillingCap;
    uint32_t hashMask;
    uint32_t newCap;
    uint32_t maxExpandIters;
    uint32_t voxelMode;      // 0: lowest index wins, 1: first to arrive
    uint64_t persistentCapacity;  // the reference store's capacity (bytes)
    uint64_t safetyMargin;
    float boxMin[3];
    float octreeSize;
};

constexpr uint32_t kGridUnits = (uint32_t)(kGridBytes / 16u);

// The multi-level expand round bins the points below each of up to kDeepRoots
// spilling nodes at depths 1..kDeepLevels below it: depth j has 8^j cells,
// stored from deepOffset(j), kDeepCells per root in all (37,448 at five
// depths: 76.7 MB for 512 roots). Five depths cover the expand loops of 1M-
// point batches of a lidar sweep: they take 5 or 6 iterations (4 and 5 split
// generations) in 88 of 100 batches, at most 9.
constexpr uint32_t kDeepLevels = 5;
constexpr uint32_t kDeepRoots = 512;
__host__ __device__ constexpr uint32_t deepOffset(uint32_t depth) { return ((1u << (3u * depth)) - 8u) / 7u; }
constexpr uint32_t kDeepCells = deepOffset(kDeepLevels + 1u);

#ifdef __CUDACC__
__device__ __forceinline__ Point* chunkPoints(const Dev& d, uint32_t phys) {
    return reinterpret_cast<Point*>(d.arena + (uint64_t)phys * 16u);
}
__device__ __forceinline__ uint32_t* chunkIndices(const Dev& d, uint32_t phys) {
    return reinterpret_cast<uint32_t*>(d.arena + (uint64_t)phys * 16u + (uint64_t)d.ppc * 16u);
}
__device__ __forceinline__ uint32_t* gridWordsAt(const Dev& d, uint32_t g) {
    return reinterpret_cast<uint32_t*>(d.arena + (uint64_t)g * 16u);
}
// Bump allocation of `units` 16-byte units; kNone when the arena is full.
__device__ __forceinline__ uint32_t arenaAlloc(const Dev& d, uint32_t units) {
    const uint32_t off = atomicAdd(&d.ctr->arenaBump, units);
    if ((uint64_t)off + units > d.arenaUnits) {
        atomicOr(&d.ctr->overflowFlags, (uint32_t)kOvfArena);
        return kNone;
    }
    return off;
}
#endif

}  // namespace rb
