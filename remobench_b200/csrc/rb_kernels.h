// Kernel launch wrappers shared by the stage translation units and the host
// orchestration (rb_capi.cu). Host code never sees a kernel symbol directly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb_state.h"

namespace rb {

// Per-frame render parameters (the subset of SharedUniforms,
// include/remo/HostDeviceCommon.h:28-60, that the LOD cut and splat read).
struct Frame {
    float width, height;
    float transform[16];        // row-major, clip = M (x, y, z, 1)
    float transformFrozen[16];  // LOD-selection and frustum transform
    float boxMin[3], boxMax[3];
    float lodPixelBudget;
    int32_t pointSize;
    int32_t colorMode;          // 0 rgb, 1 by node, 2 by level, 3 white
    uint32_t showBoundingBox;
};

struct RenderScratch {
    uint32_t numItems;
    uint32_t overflow;
    unsigned long long samples;
};

// Update
void launchBatchBegin(const Dev& d, cudaStream_t s);
// One batch at the device cursor as an instantiated graph (see rb_update.cu).
cudaError_t captureBatchGraph(const Dev& d, int pointGrid, int fixedGrid, int restGrid, cudaGraphExec_t* out);
// The cooperative expand-pass kernel: its grid, and one launch.
cudaError_t expandRestGrid(int numSMs, int* grid);
cudaError_t launchExpandRest(const Dev& d, int grid, cudaStream_t s);
void launchCountFirst(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s);
void launchRecount(const Dev& d, const Point* pts, uint32_t n, uint32_t prevStamp, int grid, cudaStream_t s);
void launchSplit(const Dev& d, uint32_t stamp, cudaStream_t s);
void launchZeroGrids(const Dev& d, int grid, cudaStream_t s);
// the expand round (rb_update.cu): book the first count's splits, bin the
// points below them, make every split the counts decide, move the points
void launchDeepBook(const Dev& d, cudaStream_t s);
void launchDeepBin(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s);
void launchDeepSplit(const Dev& d, cudaStream_t s);
void launchDeepMove(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s);
void launchExpandCond(const Dev& d, cudaStream_t s);
void launchSpillCopy(const Dev& d, int grid, cudaStream_t s);
void launchVoxSample(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s);
void launchVoxLift(const Dev& d, int grid, cudaStream_t s);
void launchVoxSampleLevels(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s);
void launchDeepenBegin(const Dev& d, const uint32_t* queue, uint32_t queueLen, uint32_t budget, uint32_t minPoints,
                       cudaStream_t s);
void launchDeepenEnd(const Dev& d, cudaStream_t s);
void launchCollapse(const Dev& d, uint32_t count, uint32_t maxPoints, int grid, cudaStream_t s);
void launchVoxCommit(const Dev& d, int grid, cudaStream_t s);
void launchFinishLeaves(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s);
void launchAllocPoints(const Dev& d, int grid, cudaStream_t s);
void launchAllocVoxels(const Dev& d, int grid, cudaStream_t s);
void launchInsert(const Dev& d, const Point* pts, uint32_t n, int grid, cudaStream_t s);
void launchVoxStore(const Dev& d, int grid, cudaStream_t s);
void launchBatchEnd(const Dev& d, uint32_t n, cudaStream_t s);
void launchSweep(const Dev& d, int grid, cudaStream_t s);
void launchResetRoot(const Dev& d, int grid, cudaStream_t s);

// Accumulate
void launchAccumulate(const Dev& d, uint32_t batchIndex, int useList, int grid, cudaStream_t s);
void launchAccumVerify(const Dev& d, int grid, cudaStream_t s);

// Rasterize
void launchFbClear(unsigned long long* fb, uint64_t npx, int grid, cudaStream_t s);
void launchNodeFlags(const Dev& d, const Frame& f, uint8_t* vis, uint8_t* large, const uint8_t* force,
                     RenderScratch* rs, int grid, cudaStream_t s);
void launchFrontier(const Dev& d, const uint8_t* vis, const uint8_t* large, RenderScratch* rs,
                    uint32_t* items, uint32_t cap, int grid, cudaStream_t s);
void launchRaster(const Dev& d, const Frame& f, unsigned long long* fb, const RenderScratch* rs,
                  const uint32_t* items, uint32_t cap, int grid, cudaStream_t s);
void launchRasterFlat(const Frame& f, unsigned long long* fb, const Point* pts, uint64_t n, int grid,
                      cudaStream_t s);
void launchEdl(const unsigned long long* src, unsigned long long* dst, uint32_t w, uint32_t h,
               float strength, int grid, cudaStream_t s);
void launchResolve(const unsigned long long* fb, uint32_t* rgba, uint64_t npx, int grid, cudaStream_t s);
// The draw items' bounding boxes as lines (remo_lines.cuh:120-137), after EDL.
void launchWireframe(const Dev& d, const Frame& f, unsigned long long* fb, const RenderScratch* rs,
                     const uint32_t* items, uint32_t cap, int grid, cudaStream_t s);

}  // namespace rb
