// Headless driver-API launcher for the reference's own kernels -- TEST
// INFRASTRUCTURE ONLY. It loads the cubins built by oracle/ref/build_ref.py from
// the reference's kernels/remolod/*.cu and launches them with the buffers,
// argument lists and launch shapes of src/pipelines/RemolodPipeline.cpp
// (allocate :105-195, reset launch :340-389, construct launch :393-420,
// accumulate :242-294, render :543-601), without the GL shell. The reference's
// host-side structs (Uniforms, Stats, SharedUniforms, RenderArgs, AccumArgs)
// come from its headers at compile time.
#include <cuda.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "HostDeviceInterface.h"  // kernels/simlod: Uniforms, Stats
#include "remo/HostDeviceCommon.h"
#include "remo/RemoAccum.h"

namespace {

constexpr uint64_t kSlot = 1000000;      // PointSource kSlotCapacity
constexpr uint32_t kRingSlots = 50;      // BATCH_STREAM_SIZE
constexpr uint32_t kMaxNodes = 200000;   // MAX_NODES_CAPACITY
constexpr uint32_t kNodeBytes = 152;
constexpr uint64_t kMomentary = 512ull << 20;

struct Handle {
    CUcontext ctx = nullptr;
    CUdevice dev = 0;
    int numSMs = 0;
    CUmodule mReset = nullptr, mOctree = nullptr, mAccum = nullptr, mRender = nullptr;
    CUfunction fReset = nullptr, fConstruct = nullptr, fAccum = nullptr, fVerify = nullptr, fRender = nullptr;
    CUdeviceptr ring = 0, sizes = 0, uploaded = 0, momentary = 0, persistent = 0, nodes = 0, accums = 0,
                accumGlobals = 0, stats = 0, frameStart = 0, cudaPrint = 0, diag = 0, timeline = 0,
                resetSizes = 0, resetUploaded = 0, scratch = 0;
    uint64_t persistentBytes = 0, scratchBytes = 0;
    float boxMin[3] = {0, 0, 0}, boxMax[3] = {0, 0, 0};
    uint32_t hostSizes[kRingSlots] = {};
    uint32_t numUploaded = 0;
    uint32_t batchesConsumed = 0;
    std::string err;
};

bool ck(Handle* h, CUresult r, const char* what) {
    if (r == CUDA_SUCCESS) return true;
    const char* s = nullptr;
    cuGetErrorString(r, &s);
    h->err = std::string(what) + ": " + (s ? s : "?");
    return false;
}

#define CK(h, call) \
    if (!ck((h), (call), #call)) return -1

Uniforms makeUniforms(const Handle* h) {
    // RemolodPipeline::fillUniforms (:227-240)
    Uniforms u;
    std::memset(&u, 0, sizeof(u));
    u.boxMin.x = h->boxMin[0];
    u.boxMin.y = h->boxMin[1];
    u.boxMin.z = h->boxMin[2];
    u.boxMax.x = h->boxMax[0];
    u.boxMax.y = h->boxMax[1];
    u.boxMax.z = h->boxMax[2];
    u.persistentBufferCapacity = h->persistentBytes;
    u.momentaryBufferCapacity = kMomentary;
    return u;
}

int gridFor(Handle* h, CUfunction f, int block, int smFactor) {
    // CudaContext::gridForKernel (src/cuda/CudaContext.cpp:53-68)
    int perSM = 0;
    if (cuOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, f, block, 0) != CUDA_SUCCESS || perSM < 1) perSM = 1;
    const int resident = perSM * h->numSMs;
    if (smFactor <= 0) return resident;
    return std::min(smFactor * h->numSMs, resident);
}

}  // namespace

extern "C" {

int ref_accumulate(void* hp, void* globalsOut);

const char* ref_last_error(void* hp) { return hp ? static_cast<Handle*>(hp)->err.c_str() : "null"; }

int ref_open(const char* cubinDir, const char* variant, void** out) {
    Handle* h = new Handle();
    *out = h;
    CK(h, cuInit(0));
    CK(h, cuDeviceGet(&h->dev, 0));
    CK(h, cuDevicePrimaryCtxRetain(&h->ctx, h->dev));
    CK(h, cuCtxSetCurrent(h->ctx));
    CK(h, cuDeviceGetAttribute(&h->numSMs, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, h->dev));
    const std::string d = std::string(cubinDir) + "/";
    const std::string v = std::string(".") + variant + ".cubin";
    CK(h, cuModuleLoad(&h->mReset, (d + "remolod_reset" + v).c_str()));
    CK(h, cuModuleLoad(&h->mOctree, (d + "remolod_octree" + v).c_str()));
    CK(h, cuModuleLoad(&h->mAccum, (d + "remolod_accum" + v).c_str()));
    CK(h, cuModuleLoad(&h->mRender, (d + "remolod_render" + v).c_str()));
    CK(h, cuModuleGetFunction(&h->fReset, h->mReset, "kernel"));
    CK(h, cuModuleGetFunction(&h->fConstruct, h->mOctree, "kernel_construct"));
    CK(h, cuModuleGetFunction(&h->fAccum, h->mAccum, "kernel_accumulate"));
    CK(h, cuModuleGetFunction(&h->fVerify, h->mAccum, "kernel_accum_verify"));
    CK(h, cuModuleGetFunction(&h->fRender, h->mRender, "kernel_render"));
    return 0;
}

// RemolodPipeline::allocate (:105-195) with a caller-chosen persistent store,
// plus the 50-slot ring PointSource owns (src/io/PointSource.cpp:146-163).
int ref_alloc(void* hp, uint64_t persistentBytes, const float boxMin[3], const float boxMax[3]) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    h->persistentBytes = persistentBytes;
    for (int a = 0; a < 3; a++) {
        h->boxMin[a] = boxMin[a];
        h->boxMax[a] = boxMax[a];
    }
    auto alloc = [&](CUdeviceptr* p, uint64_t bytes) -> bool {
        if (!ck(h, cuMemAlloc(p, bytes), "cuMemAlloc")) return false;
        return ck(h, cuMemsetD8(*p, 0, bytes), "cuMemsetD8");
    };
    if (!alloc(&h->ring, kRingSlots * kSlot * 16) || !alloc(&h->sizes, kRingSlots * 4) ||
        !alloc(&h->uploaded, 4) || !alloc(&h->momentary, kMomentary) || !alloc(&h->persistent, persistentBytes) ||
        !alloc(&h->nodes, (uint64_t)kMaxNodes * kNodeBytes) ||
        !alloc(&h->accums, (uint64_t)kMaxNodes * sizeof(remo::NodeAccum)) ||
        !alloc(&h->accumGlobals, sizeof(remo::AccumGlobals)) || !alloc(&h->stats, sizeof(Stats)) ||
        !alloc(&h->frameStart, 8) || !alloc(&h->cudaPrint, 1024) || !alloc(&h->diag, sizeof(remo::DeviceDiagnostics)) ||
        !alloc(&h->timeline, sizeof(remo::DeviceTimeline)) || !alloc(&h->resetSizes, kRingSlots * 4) ||
        !alloc(&h->resetUploaded, 4))
        return -1;
    return 0;
}

// The reset launch (RemolodPipeline.cpp:340-389): cooperative 1x1x1, then the
// accumulator side array and globals zeroed.
int ref_reset(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    Uniforms u = makeUniforms(h);
    void* args[] = {&u, &h->persistent, &h->nodes, &h->stats, &h->cudaPrint, &h->resetUploaded, &h->resetSizes};
    CK(h, cuLaunchCooperativeKernel(h->fReset, 1, 1, 1, 1, 1, 1, 0, 0, args));
    CK(h, cuCtxSynchronize());
    CK(h, cuMemsetD8(h->accums, 0, (uint64_t)kMaxNodes * sizeof(remo::NodeAccum)));
    CK(h, cuMemsetD8(h->accumGlobals, 0, sizeof(remo::AccumGlobals)));
    h->numUploaded = 0;
    h->batchesConsumed = 0;
    std::memset(h->hostSizes, 0, sizeof(h->hostSizes));
    CK(h, cuMemsetD8(h->sizes, 0, kRingSlots * 4));
    CK(h, cuMemsetD8(h->uploaded, 0, 4));
    return 0;
}

// The producer side of PointSource::pump (src/io/PointSource.cpp:275-339):
// batch b into slot b % 50, then batchSizes and numBatchesUploaded.
int ref_upload(void* hp, uint32_t batch, const void* pts, uint32_t n) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    if (n > kSlot) {
        h->err = "batch larger than a slot";
        return -1;
    }
    const uint32_t slot = batch % kRingSlots;
    CK(h, cuMemcpyHtoD(h->ring + (CUdeviceptr)slot * kSlot * 16, pts, (size_t)n * 16));
    h->hostSizes[slot] = n;
    CK(h, cuMemcpyHtoD(h->sizes, h->hostSizes, sizeof(h->hostSizes)));
    h->numUploaded = batch + 1;
    CK(h, cuMemcpyHtoD(h->uploaded, &h->numUploaded, 4));
    return 0;
}

// One kernel_construct launch (RemolodPipeline.cpp:393-420); returns the
// batchlet index after it.
int ref_construct(void* hp, uint32_t* batchletIndex) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    Uniforms u = makeUniforms(h);
    void* args[] = {&u,          &h->ring,       &h->momentary, &h->persistent, &h->nodes, &h->stats,
                    &h->frameStart, &h->cudaPrint, &h->uploaded,   &h->sizes,      &h->timeline};
    const int grid = gridFor(h, h->fConstruct, 256, 1);
    CK(h, cuLaunchCooperativeKernel(h->fConstruct, (unsigned)grid, 1, 1, 256, 1, 1, 0, 0, args));
    CK(h, cuCtxSynchronize());
    Stats s;
    CK(h, cuMemcpyDtoH(&s, h->stats, sizeof(Stats)));
    h->batchesConsumed = s.batchletIndex;
    *batchletIndex = s.batchletIndex;
    return 0;
}

// ref_construct with the launch bracketed by CUDA events (GpuScope,
// include/remo/GpuProfiler.h:143-158); *ms receives the kernel's device time.
int ref_construct_timed(void* hp, uint32_t* batchletIndex, float* ms) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    CUevent a, b;
    CK(h, cuEventCreate(&a, CU_EVENT_DEFAULT));
    CK(h, cuEventCreate(&b, CU_EVENT_DEFAULT));
    Uniforms u = makeUniforms(h);
    void* args[] = {&u,          &h->ring,       &h->momentary, &h->persistent, &h->nodes, &h->stats,
                    &h->frameStart, &h->cudaPrint, &h->uploaded,   &h->sizes,      &h->timeline};
    const int grid = gridFor(h, h->fConstruct, 256, 1);
    CK(h, cuEventRecord(a, 0));
    CK(h, cuLaunchCooperativeKernel(h->fConstruct, (unsigned)grid, 1, 1, 256, 1, 1, 0, 0, args));
    CK(h, cuEventRecord(b, 0));
    CK(h, cuEventSynchronize(b));
    CK(h, cuEventElapsedTime(ms, a, b));
    cuEventDestroy(a);
    cuEventDestroy(b);
    Stats s;
    CK(h, cuMemcpyDtoH(&s, h->stats, sizeof(Stats)));
    h->batchesConsumed = s.batchletIndex;
    *batchletIndex = s.batchletIndex;
    return 0;
}

// ref_accumulate's two launches timed the same way.
int ref_accumulate_timed(void* hp, void* globalsOut, float* ms) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    CUevent a, b;
    CK(h, cuEventCreate(&a, CU_EVENT_DEFAULT));
    CK(h, cuEventCreate(&b, CU_EVENT_DEFAULT));
    CK(h, cuEventRecord(a, 0));
    const int rc = ref_accumulate(hp, globalsOut);
    CK(h, cuEventRecord(b, 0));
    CK(h, cuEventSynchronize(b));
    CK(h, cuEventElapsedTime(ms, a, b));
    cuEventDestroy(a);
    cuEventDestroy(b);
    return rc;
}

// runAccumulator (RemolodPipeline.cpp:242-294).
int ref_accumulate(void* hp, void* globalsOut) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    remo::AccumGlobals g;
    CK(h, cuMemcpyDtoH(&g, h->accumGlobals, sizeof(g)));
    g.sumLeafCounts = 0;
    g.innerWithSums = 0;
    g.pointsFolded = 0;
    g.numLeavesFolded = 0;
    CK(h, cuMemcpyHtoD(h->accumGlobals, &g, sizeof(g)));
    Stats s;
    CK(h, cuMemcpyDtoH(&s, h->stats, sizeof(Stats)));
    const float sx = h->boxMax[0] - h->boxMin[0], sy = h->boxMax[1] - h->boxMin[1],
                sz = h->boxMax[2] - h->boxMin[2];
    remo::AccumArgs a = {};
    a.nodes = reinterpret_cast<void*>(h->nodes);
    a.accums = reinterpret_cast<void*>(h->accums);
    a.globals = reinterpret_cast<void*>(h->accumGlobals);
    a.numNodes = s.numNodes;
    a.batchIndex = h->batchesConsumed;
    a.octreeMinX = h->boxMin[0];
    a.octreeMinY = h->boxMin[1];
    a.octreeMinZ = h->boxMin[2];
    a.octreeSize = std::max(std::max(sx, sy), sz);
    void* args[] = {&a};
    const int grid = gridFor(h, h->fAccum, 256, 0);
    CK(h, cuLaunchKernel(h->fAccum, (unsigned)grid, 1, 1, 256, 1, 1, 0, 0, args, nullptr));
    CK(h, cuLaunchKernel(h->fVerify, (unsigned)grid, 1, 1, 256, 1, 1, 0, 0, args, nullptr));
    CK(h, cuCtxSynchronize());
    CK(h, cuMemcpyDtoH(globalsOut, h->accumGlobals, sizeof(remo::AccumGlobals)));
    return 0;
}

// kernel_render (RemolodPipeline.cpp:559-601) into a CUDA-array surface; the
// packed framebuffer is the first allocation of the scratch buffer
// (remolod_render.cu:78-81), read back before the next launch.
int ref_render(void* hp, const float* transform, const float* frozen, float width, float height,
               float budget, int pointSize, uint64_t* fbOut, void* diagOut) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    const uint64_t px = (uint64_t)width * (uint64_t)height;
    uint64_t need = std::max<uint64_t>(px * 64, 64ull << 20) + (16ull << 20);
    if (need > h->scratchBytes) {
        if (h->scratch) cuMemFree(h->scratch);
        h->scratch = 0;
        CK(h, cuMemAlloc(&h->scratch, need));
        h->scratchBytes = need;
    }
    CUDA_ARRAY3D_DESCRIPTOR ad = {};
    ad.Width = (size_t)width;
    ad.Height = (size_t)height;
    ad.Depth = 0;
    ad.Format = CU_AD_FORMAT_UNSIGNED_INT8;
    ad.NumChannels = 4;
    ad.Flags = CUDA_ARRAY3D_SURFACE_LDST;
    CUarray arr = nullptr;
    CK(h, cuArray3DCreate(&arr, &ad));
    CUDA_RESOURCE_DESC rd = {};
    rd.resType = CU_RESOURCE_TYPE_ARRAY;
    rd.res.array.hArray = arr;
    CUsurfObject surf = 0;
    CK(h, cuSurfObjectCreate(&surf, &rd));
    remo::RenderArgs ra;
    std::memset(&ra, 0, sizeof(ra));
    remo::SharedUniforms& u = ra.uniforms;
    u.width = width;
    u.height = height;
    std::memcpy(&u.transform, transform, 64);
    std::memcpy(&u.transformFrozen, frozen, 64);
    u.boxMin = {h->boxMin[0], h->boxMin[1], h->boxMin[2]};
    u.boxMax = {h->boxMax[0], h->boxMax[1], h->boxMax[2]};
    u.lodPixelBudget = budget;
    u.pointSize = pointSize;
    u.showPoints = 1;
    u.enableEDL = 0;
    u.showBoundingBox = 0;
    u.colorMode = remo::COLOR_RGB;
    ra.scratch = reinterpret_cast<uint32_t*>(h->scratch);
    ra.scratchCapacity = h->scratchBytes;
    ra.surface = (uint64_t)surf;
    void* args[] = {&ra, &h->nodes, &h->stats, &h->diag};
    const int grid = gridFor(h, h->fRender, 256, 0);
    CK(h, cuLaunchCooperativeKernel(h->fRender, (unsigned)grid, 1, 1, 256, 1, 1, 0, 0, args));
    CK(h, cuCtxSynchronize());
    CK(h, cuMemcpyDtoH(fbOut, h->scratch, px * 8));
    CK(h, cuMemcpyDtoH(diagOut, h->diag, sizeof(remo::DeviceDiagnostics)));
    cuSurfObjectDestroy(surf);
    cuArrayDestroy(arr);
    return 0;
}

uint64_t ref_sizeof(int what) {
    switch (what) {
        case 0: return sizeof(Stats);
        case 1: return sizeof(remo::NodeAccum);
        case 2: return sizeof(remo::AccumGlobals);
        case 3: return sizeof(remo::DeviceDiagnostics);
        case 4: return sizeof(Uniforms);
        default: return 0;
    }
}

// Raw reads for the structural comparison.
int ref_read(void* hp, int what, void* out, uint64_t bytes, uint64_t* base) {
    Handle* h = static_cast<Handle*>(hp);
    CK(h, cuCtxSetCurrent(h->ctx));
    CUdeviceptr src = 0;
    switch (what) {
        case 0: src = h->stats; break;
        case 1: src = h->nodes; break;
        case 2: src = h->persistent; break;
        case 3: src = h->accums; break;
        default: h->err = "unknown buffer"; return -1;
    }
    if (base) *base = (uint64_t)src;
    CK(h, cuMemcpyDtoH(out, src, bytes));
    return 0;
}

void ref_close(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    if (!h) return;
    cuCtxSetCurrent(h->ctx);
    for (CUdeviceptr p : {h->ring, h->sizes, h->uploaded, h->momentary, h->persistent, h->nodes, h->accums,
                          h->accumGlobals, h->stats, h->frameStart, h->cudaPrint, h->diag, h->timeline,
                          h->resetSizes, h->resetUploaded, h->scratch})
        if (p) cuMemFree(p);
    for (CUmodule m : {h->mReset, h->mOctree, h->mAccum, h->mRender})
        if (m) cuModuleUnload(m);
    if (h->ctx) cuDevicePrimaryCtxRelease(h->dev);
    delete h;
}

}  // extern "C"
