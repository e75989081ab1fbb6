// Refinement passes beyond the LOD-cut mask (rb_refine.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb_state.h"

namespace rb {

struct RefineCounters {
    uint32_t nodes;               // queue prefix filtered
    uint32_t voxels;              // accumulator entries in use
    unsigned long long points;    // (point, filtered ancestor) pairs summed
};

// Colour filtering's scratch, sized at allocation: one accumulator entry per
// voxel being filtered (capacity), a (node slot, cell) -> entry table of twice
// that, and per node its slot in the call (kNone outside a call).
struct RefineScratch {
    uint32_t* refSlot;            // [maxNodes]
    uint32_t* voxNode;            // [maxNodes + 1] filtered node per slot
    uint32_t* voxBase;            // [maxNodes + 1] first entry per slot, then the total
    ulonglong4* acc;              // [capacity] r, g, b sums and the count
    uint32_t* entrySlot;          // [capacity] the entry's table slot
    unsigned long long* hashKeys; // [hashMask + 1], ~0: free
    uint32_t* hashVals;           // [hashMask + 1]
    RefineCounters* ctr;
    uint32_t capacity;
    uint32_t hashMask;
};

__device__ uint32_t blockExclusiveScanRefine(uint32_t v, uint32_t* total, uint32_t* s_warp);

void launchRefineColors(const Dev& d, const RefineScratch& r, const uint32_t* queue, uint32_t queueLen,
                        uint32_t budget, int grid, cudaStream_t s);

}  // namespace rb
