// The reference's plugin interface, headless (include/remo/ILodPipeline.h:17-170):
// the same virtuals, ids and data crossing it. GL surfaces become device buffers,
// CUDA driver-API handles become plain device addresses. Implementations forward
// to the C ABI (rb_capi.h); nothing here computes on the CPU.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "gpu_profiler.h"
#include "rb_capi.h"

namespace rbhost {

class PointSource;
struct CloudMeta;

// PipelineInfo (ILodPipeline.h:20-63). bytesPerPointEstimate is the appetite
// allocate() sizes with; minBytesPerPointEstimate the floor fits() refuses on;
// minStoreBytes the smallest store a truncating pipeline runs with (0: cannot
// truncate); fixedBytesEstimate the part that does not scale with the cloud.
struct PipelineInfo {
    std::string id;
    std::string displayName;
    bool progressive = false;
    bool needsWholeCloudResident = false;
    uint32_t ringSlots = 0;
    double bytesPerPointEstimate = 0.0;
    double minBytesPerPointEstimate = 0.0;
    uint64_t minStoreBytes = 0;
    uint64_t fixedBytesEstimate = 0;
};

// DeviceBudget (:65-69)
struct DeviceBudget {
    uint64_t vramTotal = 0;
    uint64_t vramFreeAtStartup = 0;
    uint64_t bytes = 0;
};

// RenderTargets (:71-75): surface is a device buffer of width*height RGBA8
// words (r in the low byte) in place of the GL surface.
struct RenderTargets {
    uint64_t surface = 0;
    int width = 0;
    int height = 0;
};

// FrameContext (:77-86). uniforms is the headless SharedUniforms subset.
struct FrameContext {
    rb_frame uniforms{};
    RenderTargets targets;
    void* stream = nullptr;  // cudaStream_t; null = the context's own stream
    int numSMs = 0;
    bool strictTiming = false;
    GpuProfiler* profiler = nullptr;
};

// PipelineStats (:88-111)
struct PipelineStats {
    uint64_t numPoints = 0;
    uint64_t numVoxels = 0;
    uint64_t numPointsIngested = 0;
    uint32_t numNodes = 0;
    uint32_t numInner = 0;
    uint32_t numLeaves = 0;
    uint32_t maxDepth = 0;
    uint32_t maxPointsPerNode = 0;
    uint32_t numVisibleNodes = 0;
    uint64_t numVisiblePoints = 0;
    uint64_t numVisibleVoxels = 0;
    uint64_t bytesAllocated = 0;
    uint64_t bytesCapacity = 0;
    uint64_t samplesPerLevel[24] = {};
    bool memCapacityReached = false;
    bool nodeCapacityReached = false;
    bool allocOverflow = false;
};

// TimingScopes (:113-116): the profiler scopes a pipeline's build and render
// time is recorded under.
struct TimingScopes {
    std::vector<std::string> build;
    std::string render;
};

// ILodPipeline (:118-146)
class ILodPipeline {
public:
    virtual ~ILodPipeline() = default;
    virtual PipelineInfo info() const = 0;
    // Creates the device context; allocates no device memory.
    virtual bool initPrograms(std::string* err) = 0;
    virtual bool allocate(const CloudMeta& meta, const DeviceBudget& budget, std::string* err) = 0;
    virtual void release() = 0;
    virtual void reset() = 0;
    // One frame's worth of ingest; true while there is more to do.
    virtual bool build(PointSource& source, const FrameContext& frame) = 0;
    virtual void render(const FrameContext& frame) = 0;
    virtual const PipelineStats& stats() const = 0;
    virtual TimingScopes timingScopes() const = 0;
    virtual void guiControls() {}
    virtual void guiStats(const GpuProfiler& profiler) { (void)profiler; }
    virtual std::vector<std::string> diagnostics() const { return {}; }
    // The C-ABI context behind the pipeline (null before initPrograms): the
    // entry for Analysis, Refinement and the learned scorer, which the
    // reference's interface has no virtuals for.
    virtual struct rb_ctx* context() const { return nullptr; }
};

// BuildTotals / buildTotals (:148-166)
struct BuildTotals {
    double ms = 0.0;
    uint64_t launches = 0;
    bool measured = false;
};

BuildTotals buildTotals(const GpuProfiler& profiler, const TimingScopes& scopes);

using PipelineFactory = std::function<std::unique_ptr<ILodPipeline>()>;

// The three registered pipelines (src/shell/App.cpp:85-95). device is the
// CUDA ordinal the pipeline's context runs on.
std::unique_ptr<ILodPipeline> makeRemolodPipeline(int device = 0);
std::unique_ptr<ILodPipeline> makeSimlodPipeline(int device = 0);
std::unique_ptr<ILodPipeline> makeFlatPipeline(int device = 0);

}  // namespace rbhost
