// The three pipelines of the reference (src/pipelines/RemolodPipeline.cpp,
// SimlodPipeline.cpp, FlatPipeline.cpp) as thin forwards to the C ABI. The
// PipelineInfo figures are the reference's, so the registry gates a cloud
// exactly as it does; the per-frame build/render sequence, the reset→rewind
// handshake and the consumption signal follow RemolodPipeline.cpp:298-441.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "lod_pipeline.h"
#include "point_source.h"

namespace rbhost {

BuildTotals buildTotals(const GpuProfiler& profiler, const TimingScopes& scopes) {
    BuildTotals totals;
    for (const std::string& name : scopes.build) {
        const ScopeStats* s = profiler.find(name);
        if (!s) continue;
        totals.ms += s->total();
        totals.launches += s->count();
        totals.measured = true;
    }
    return totals;
}

namespace {

// Store coefficients (RemolodPipeline.cpp:23-37): 48 B/pt appetite, 26 B/pt
// measured floor, 512 MB smallest store, 512 MB momentary buffer, 200k nodes.
constexpr double kBytesPerPointPersistent = 48.0;
constexpr double kMinBytesPerPointPersistent = 26.0;
constexpr uint64_t kMinPersistentBytes = 512ull << 20;
constexpr uint64_t kMomentaryBytes = 512ull << 20;
constexpr uint32_t kMaxNodes = 200000;
constexpr uint64_t kNodeBytes = 152;       // the reference's Node record
constexpr uint64_t kNodeAccumBytes = 112;  // its NodeAccum side record

struct Event {
    cudaEvent_t e = nullptr;
    Event() { cudaEventCreate(&e); }
    ~Event() {
        if (e) cudaEventDestroy(e);
    }
};

// Shared base: one rb_ctx, a device framebuffer sized to the target, a
// stream handed to the context so frame.stream orders our work.
class CtxPipeline : public ILodPipeline {
public:
    CtxPipeline(uint32_t kind, int device, const char* id, const char* name)
        : m_kind(kind), m_device(device), m_id(id), m_name(name) {}
    ~CtxPipeline() override {
        release();
        if (m_ctx) rb_destroy(m_ctx);
        if (m_stream) cudaStreamDestroy(m_stream);
    }

    bool initPrograms(std::string* err) override {
        if (m_ctx) return true;
        rb_config cfg;
        rb_config_defaults(&cfg);
        cfg.pipeline = m_kind;
        cfg.device = m_device;
        cfg.max_nodes = kMaxNodes;
        // Accumulate is timed under its own scope (remolod.accumulate), so the
        // pipeline calls it after each build instead of folding it into rb_build.
        cfg.accumulate = 0;
        configure(cfg);
        if (cudaSetDevice(m_device) != cudaSuccess ||
            cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            if (err) *err = "no CUDA device " + std::to_string(m_device);
            return false;
        }
        const rb_status st = rb_create(&cfg, &m_ctx);
        if (st != RB_OK) {
            if (err) *err = std::string("rb_create: ") + rb_status_string(st);
            m_ctx = nullptr;
            return false;
        }
        return true;
    }

    void release() override {
        if (m_fb) {
            cudaSetDevice(m_device);
            cudaFree(m_fb);
        }
        m_fb = nullptr;
        m_fbPixels = 0;
        if (m_ctx) rb_release(m_ctx);
        m_complete = false;
        m_needsReset = true;
    }

    const PipelineStats& stats() const override { return m_stats; }
    struct rb_ctx* context() const override { return m_ctx; }

    std::vector<std::string> diagnostics() const override {
        std::vector<std::string> out;
        if (!m_ctx) return out;
        rb_stats s;
        if (rb_read_stats(m_ctx, &s) != RB_OK) return out;
        char buf[256];
        std::snprintf(buf, sizeof(buf), "expand iterations %llu, nodes split %llu, spilled points %llu",
                      (unsigned long long)s.expand_iters, (unsigned long long)s.nodes_split,
                      (unsigned long long)s.spilled_points);
        out.push_back(buf);
        if (s.overflow_flags) {
            std::snprintf(buf, sizeof(buf), "overflow flags 0x%x (dropped points %llu)", s.overflow_flags,
                          (unsigned long long)s.dropped_points);
            out.push_back(buf);
        }
        if (s.counter_underflows) {
            std::snprintf(buf, sizeof(buf), "counter underflows %u", s.counter_underflows);
            out.push_back(buf);
        }
        return out;
    }

protected:
    virtual void configure(rb_config&) {}

    bool allocateCtx(const CloudMeta& meta, const DeviceBudget& budget, std::string* err) {
        release();
        m_stats = PipelineStats{};
        m_stats.bytesCapacity = budget.bytes;
        if (!m_ctx) {
            if (err) *err = "initPrograms was not called";
            return false;
        }
        if (meta.numPoints == 0) {
            if (err) *err = "cloud is empty";
            return false;
        }
        rb_cloud_meta m{};
        m.num_points = meta.numPoints;
        for (int a = 0; a < 3; a++) {
            m.box_min[a] = 0.0f;
            m.box_max[a] = meta.boxSize[a];
        }
        const rb_status st = rb_allocate(m_ctx, &m, budget.bytes);
        if (st != RB_OK) {
            if (err) *err = rb_last_error(m_ctx);
            return false;
        }
        m_numPoints = meta.numPoints;
        rb_stats s;
        if (rb_read_stats(m_ctx, &s) == RB_OK) m_stats.bytesAllocated = s.bytes_allocated;
        return true;
    }

    // frame.stream when the caller gives one, else the pipeline's own stream.
    void bindStream(const FrameContext& frame) {
        void* s = frame.stream ? frame.stream : static_cast<void*>(m_stream);
        if (s != m_boundStream) {
            rb_set_stream(m_ctx, s);
            m_boundStream = s;
        }
    }

    bool ensureFramebuffer(const FrameContext& frame) {
        const uint64_t pixels = uint64_t(frame.targets.width) * uint64_t(frame.targets.height);
        if (pixels == 0) return false;
        if (pixels <= m_fbPixels) return true;
        cudaSetDevice(m_device);
        if (m_fb) cudaFree(m_fb);
        m_fb = nullptr;
        m_fbPixels = 0;
        if (cudaMalloc(&m_fb, pixels * sizeof(uint64_t)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        m_fbPixels = pixels;
        return true;
    }

    static rb_frame uniformsFor(const FrameContext& frame) {
        rb_frame f = frame.uniforms;
        f.width = static_cast<float>(frame.targets.width);
        f.height = static_cast<float>(frame.targets.height);
        return f;
    }

    uint32_t m_kind;
    int m_device;
    std::string m_id, m_name;
    rb_ctx* m_ctx = nullptr;
    cudaStream_t m_stream = nullptr;
    void* m_boundStream = nullptr;
    void* m_fb = nullptr;
    uint64_t m_fbPixels = 0;
    uint64_t m_numPoints = 0;
    bool m_complete = false;
    bool m_needsReset = true;
    PipelineStats m_stats;
};

class ProgressivePipeline final : public CtxPipeline {
public:
    ProgressivePipeline(uint32_t kind, int device, const char* id, const char* name, bool accumulate)
        : CtxPipeline(kind, device, id, name), m_accumulate(accumulate) {}

    PipelineInfo info() const override {
        PipelineInfo info;
        info.id = m_id;
        info.displayName = m_name;
        info.progressive = true;
        info.needsWholeCloudResident = false;
        info.ringSlots = 50;
        info.bytesPerPointEstimate = kBytesPerPointPersistent;
        info.minBytesPerPointEstimate = kMinBytesPerPointPersistent;
        info.minStoreBytes = kMinPersistentBytes;
        info.fixedBytesEstimate = kMomentaryBytes + uint64_t(kMaxNodes) * (kNodeBytes + (m_accumulate ? kNodeAccumBytes : 0));
        return info;
    }

    bool allocate(const CloudMeta& meta, const DeviceBudget& budget, std::string* err) override {
        if (!allocateCtx(meta, budget, err)) return false;
        m_needsReset = true;
        m_complete = false;
        return true;
    }

    void reset() override {
        m_needsReset = true;
        m_complete = false;
        m_batchesConsumed = 0;
    }

    TimingScopes timingScopes() const override {
        TimingScopes scopes;
        scopes.build = {m_id + ".reset", m_id + ".construct"};
        if (m_accumulate) scopes.build.push_back(m_id + ".accumulate");
        scopes.render = m_id + ".render";
        return scopes;
    }

    bool build(PointSource& source, const FrameContext& frame) override {
        if (!m_ctx || !m_numPoints) return false;
        bindStream(frame);
        if (m_needsReset) {
            if (frame.profiler) frame.profiler->clearPrefix(m_id + ".");
            const double ms = timed(frame, [&] { return rb_reset(m_ctx); });
            if (ms < 0) return false;
            if (frame.profiler) frame.profiler->addSample(m_id + ".reset", ms);
            m_needsReset = false;
            m_complete = false;
            m_batchesConsumed = 0;
            // The builder's batch counter is back at zero: so is the producer.
            source.rewind();
            return true;
        }
        if (m_complete) return false;
        const BatchView view = source.view();
        if (view.slots == 0 || view.batchSizes == nullptr || view.numBatchesUploaded == 0) return true;
        rb_batch_view v{};
        v.slots = view.slots;
        v.batch_sizes = view.batchSizes;
        v.num_batches_uploaded = view.numBatchesUploaded;
        v.slot_capacity = view.slotCapacity;
        v.num_slots = view.numSlots;
        v.num_batches_total = view.numBatchesTotal;
        rb_build_result r{};
        const rb_status st = rb_build(m_ctx, &v, &r);
        if (st != RB_OK) {
            if (!m_buildErrorReported) {
                m_buildErrorReported = true;
                std::fprintf(stderr, "rbhost: %s refused to build: %s\n", m_name.c_str(), rb_last_error(m_ctx));
            }
            return false;
        }
        if (frame.profiler) frame.profiler->addSample(m_id + ".construct", r.device_ms);
        const bool advanced = r.batches_consumed > m_batchesConsumed;
        m_batchesConsumed = r.batches_consumed;
        source.setBatchesConsumed(m_batchesConsumed);
        if (m_accumulate && advanced) {
            rb_accum_globals g;
            const double ms = timed(frame, [&] { return rb_accumulate(m_ctx, m_batchesConsumed, &g); });
            if (ms >= 0 && frame.profiler) frame.profiler->addSample(m_id + ".accumulate", ms);
        }
        readStats();
        if (view.numBatchesTotal > 0 && m_batchesConsumed >= view.numBatchesTotal) {
            m_complete = true;
            return false;
        }
        return true;
    }

    void render(const FrameContext& frame) override {
        if (!m_ctx || !m_numPoints || frame.targets.surface == 0) return;
        if (!ensureFramebuffer(frame)) return;
        bindStream(frame);
        const rb_frame f = uniformsFor(frame);
        rb_render_result rr{};
        if (rb_render(m_ctx, &f, reinterpret_cast<uint64_t>(m_fb), frame.targets.surface, 0, &rr) != RB_OK) return;
        if (frame.profiler) frame.profiler->addSample(m_id + ".render", rr.device_ms);
        m_stats.numVisibleNodes = rr.draw_items;
        // The draw list does not separate points from voxels: all visible samples.
        m_stats.numVisiblePoints = rr.draw_samples;
        m_stats.numVisibleVoxels = 0;
        m_stats.allocOverflow = rr.drawlist_overflow != 0;
    }

private:
    template <class F>
    double timed(const FrameContext& frame, F&& call) {
        (void)frame;
        cudaStream_t s = static_cast<cudaStream_t>(m_boundStream);
        Event a, b;
        cudaEventRecord(a.e, s);
        if (call() != RB_OK) return -1.0;
        cudaEventRecord(b.e, s);
        cudaEventSynchronize(b.e);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a.e, b.e);
        return ms;
    }

    void readStats() {
        rb_stats s;
        if (rb_read_stats(m_ctx, &s) != RB_OK) return;
        m_stats.numPoints = s.num_points;
        m_stats.numVoxels = s.num_voxels;
        m_stats.numPointsIngested = s.num_points_ingested;
        m_stats.numNodes = s.num_nodes;
        m_stats.numInner = s.num_inner;
        m_stats.numLeaves = s.num_leaves;
        m_stats.maxDepth = s.max_depth;
        m_stats.maxPointsPerNode = s.max_points_per_node;
        m_stats.bytesAllocated = s.bytes_allocated;
        m_stats.memCapacityReached = s.mem_capacity_reached != 0;
        m_stats.nodeCapacityReached = s.node_capacity_reached != 0 || s.num_nodes >= kMaxNodes;
    }

    bool m_accumulate;
    uint32_t m_batchesConsumed = 0;
    bool m_buildErrorReported = false;
};

class FlatPipeline final : public CtxPipeline {
public:
    explicit FlatPipeline(int device) : CtxPipeline(RB_PIPELINE_FLAT, device, "flat", "Flat") {}

    PipelineInfo info() const override {
        PipelineInfo info;
        info.id = "flat";
        info.displayName = "Flat";
        info.progressive = false;
        info.needsWholeCloudResident = true;
        return info;  // no per-point store: the resident cloud is its whole cost
    }

    bool allocate(const CloudMeta& meta, const DeviceBudget& budget, std::string* err) override {
        if (!allocateCtx(meta, budget, err)) return false;
        m_stats.numPoints = meta.numPoints;
        m_points = 0;
        return true;
    }

    void release() override {
        CtxPipeline::release();
        m_points = 0;
    }

    void reset() override { m_stats.allocOverflow = false; }

    TimingScopes timingScopes() const override {
        TimingScopes scopes;
        scopes.render = "flat.render";
        return scopes;
    }

    bool build(PointSource& source, const FrameContext&) override {
        if (!source.isFullyResident()) return true;
        if (m_points != 0) return false;
        m_points = source.residentPoints();
        m_stats.numPoints = source.meta().numPoints;
        m_stats.numPointsIngested = m_stats.numPoints;
        m_stats.numVisiblePoints = m_stats.numPoints;
        return false;
    }

    void render(const FrameContext& frame) override {
        if (!m_ctx || m_points == 0 || frame.targets.surface == 0) return;
        if (!ensureFramebuffer(frame)) return;
        bindStream(frame);
        const rb_frame f = uniformsFor(frame);
        rb_render_result rr{};
        if (rb_render_flat(m_ctx, &f, m_points, m_stats.numPoints, reinterpret_cast<uint64_t>(m_fb),
                           frame.targets.surface, &rr) != RB_OK)
            return;
        if (frame.profiler) frame.profiler->addSample("flat.render", rr.device_ms);
        m_stats.numVisiblePoints = rr.draw_samples;
    }

private:
    uint64_t m_points = 0;
};

}  // namespace

std::unique_ptr<ILodPipeline> makeRemolodPipeline(int device) {
    return std::make_unique<ProgressivePipeline>(RB_PIPELINE_REMOLOD, device, "remolod", "RemoLOD", true);
}
std::unique_ptr<ILodPipeline> makeSimlodPipeline(int device) {
    return std::make_unique<ProgressivePipeline>(RB_PIPELINE_SIMLOD, device, "simlod", "SimLOD", false);
}
std::unique_ptr<ILodPipeline> makeFlatPipeline(int device) { return std::make_unique<FlatPipeline>(device); }

}  // namespace rbhost
