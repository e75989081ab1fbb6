// PipelineRegistry (include/remo/PipelineRegistry.h:11-67): the registered
// pipelines, the memory gate that refuses or warns before a run starts, and
// the switch that re-shapes the point source for the incoming pipeline.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "lod_pipeline.h"
#include "point_source.h"

namespace rbhost {

// kernel_construct stops ingesting this close to its store's capacity
// (progressive_octree_voxels.cu `safetyMargin`; rb_config.safety_margin).
constexpr uint64_t kPersistentSafetyMargin = 200000000ull;

// A progressive pipeline reads batch B from ring slot B % 50, so a resident
// (non-wrapping) feed can describe at most 50 slots (kernels/simlod/simlod_layout.h:70-83).
constexpr uint32_t kBatchStreamSize = 50;
constexpr uint64_t kMaxAddressablePoints = uint64_t(kSlotCapacity) * kBatchStreamSize;

class PipelineRegistry {
public:
    void add(PipelineFactory factory);
    const std::vector<PipelineInfo>& list() const { return m_infos; }
    ILodPipeline* active() const { return m_active.get(); }
    const std::string& activeId() const { return m_activeId; }
    const PipelineInfo* find(const std::string& id) const;

    // Per-point floor + input term (whole cloud or ring) + fixed overhead.
    uint64_t minBytesRequired(const PipelineInfo& info, const CloudMeta& meta) const;
    // The budget below which the pipeline cannot run at all.
    uint64_t refusalFloor(const PipelineInfo& info, const CloudMeta& meta) const;
    bool fits(const PipelineInfo& info, const CloudMeta& meta, const DeviceBudget& budget) const;
    std::string unsupportedReason(const PipelineInfo& info, const CloudMeta& meta, const DeviceBudget& budget) const;
    // Predicted fraction of the cloud the budget holds, in [0, 1].
    double predictedCompletion(const PipelineInfo& info, const CloudMeta& meta, const DeviceBudget& budget) const;
    // Empty when the whole cloud is predicted to fit, else one line.
    std::string completionWarning(const PipelineInfo& info, const CloudMeta& meta, const DeviceBudget& budget) const;

    bool switchTo(const std::string& id, PointSource* source, const CloudMeta& meta, const DeviceBudget& budget,
                  std::string* err);
    bool reloadForCloud(PointSource* source, const CloudMeta& meta, const DeviceBudget& budget, std::string* err);

    // Releases the active pipeline (before the device context goes away).
    void shutdown();

private:
    struct Entry {
        PipelineInfo info;
        PipelineFactory factory;
    };
    std::vector<Entry> m_entries;
    std::vector<PipelineInfo> m_infos;
    std::unique_ptr<ILodPipeline> m_active;
    std::string m_activeId;
};

// Input bytes the pipeline's feed takes: 16 B per point of a resident cloud,
// or a ring no deeper than the cloud (src/shell/PipelineRegistry.cpp:54-66).
uint64_t inputBytesFor(const PipelineInfo& info, const CloudMeta& meta);

}  // namespace rbhost
