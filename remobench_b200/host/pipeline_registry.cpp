// The registry's gate arithmetic and switch sequence follow
// src/shell/PipelineRegistry.cpp:20-274 step for step, so a cloud/budget pair
// is refused, warned about or accepted exactly as the reference decides.
#include "pipeline_registry.h"

#include <algorithm>
#include <cstdio>

namespace rbhost {

void PipelineRegistry::add(PipelineFactory factory) {
    if (!factory) return;
    std::unique_ptr<ILodPipeline> probe = factory();
    if (!probe) {
        std::fprintf(stderr, "rbhost: pipeline factory returned null at registration\n");
        return;
    }
    PipelineInfo info = probe->info();
    probe.reset();
    if (info.id.empty()) {
        std::fprintf(stderr, "rbhost: pipeline has an empty id; not registered\n");
        return;
    }
    if (find(info.id)) {
        std::fprintf(stderr, "rbhost: duplicate pipeline id '%s'; not registered\n", info.id.c_str());
        return;
    }
    m_infos.push_back(info);
    m_entries.push_back({std::move(info), std::move(factory)});
}

const PipelineInfo* PipelineRegistry::find(const std::string& id) const {
    for (const Entry& e : m_entries)
        if (e.info.id == id) return &e.info;
    return nullptr;
}

uint64_t inputBytesFor(const PipelineInfo& info, const CloudMeta& meta) {
    if (!info.needsWholeCloudResident && info.ringSlots > 0) {
        const uint64_t total = (meta.numPoints + kSlotCapacity - 1) / kSlotCapacity;
        const uint64_t slots = std::min<uint64_t>(info.ringSlots, total);
        return slots * kSlotCapacity * sizeof(rb_point);
    }
    return meta.numPoints * sizeof(rb_point);
}

uint64_t PipelineRegistry::minBytesRequired(const PipelineInfo& info, const CloudMeta& meta) const {
    const double perPoint = info.minBytesPerPointEstimate * static_cast<double>(meta.numPoints);
    return static_cast<uint64_t>(perPoint) + inputBytesFor(info, meta) + info.fixedBytesEstimate;
}

uint64_t PipelineRegistry::refusalFloor(const PipelineInfo& info, const CloudMeta& meta) const {
    // A pipeline that truncates cleanly is refused only when it cannot run at all.
    if (info.minStoreBytes == 0) return minBytesRequired(info, meta);
    return info.minStoreBytes + inputBytesFor(info, meta) + info.fixedBytesEstimate;
}

bool PipelineRegistry::fits(const PipelineInfo& info, const CloudMeta& meta, const DeviceBudget& budget) const {
    return refusalFloor(info, meta) <= budget.bytes;
}

double PipelineRegistry::predictedCompletion(const PipelineInfo& info, const CloudMeta& meta,
                                             const DeviceBudget& budget) const {
    if (meta.numPoints == 0) return 1.0;
    if (info.minBytesPerPointEstimate <= 0.0) return fits(info, meta, budget) ? 1.0 : 0.0;
    const uint64_t overhead = inputBytesFor(info, meta) + info.fixedBytesEstimate;
    if (budget.bytes <= overhead) return 0.0;
    const uint64_t room = budget.bytes - overhead;
    const uint64_t want = static_cast<uint64_t>(info.bytesPerPointEstimate * static_cast<double>(meta.numPoints));
    const uint64_t persistent = std::min(want, room);
    const uint64_t usable = persistent > kPersistentSafetyMargin ? persistent - kPersistentSafetyMargin : 0;
    const double points = static_cast<double>(usable) / info.minBytesPerPointEstimate;
    return std::clamp(points / static_cast<double>(meta.numPoints), 0.0, 1.0);
}

std::string PipelineRegistry::completionWarning(const PipelineInfo& info, const CloudMeta& meta,
                                                const DeviceBudget& budget) const {
    const double fraction = predictedCompletion(info, meta, budget);
    if (fraction >= 0.999) return {};
    char buf[256];
    std::snprintf(buf, sizeof(buf),
                  "the budget holds about %.0f%% of this cloud; ingest will stop cleanly on a truncated tree "
                  "(memCapacityReached). %.1f GB of budget would hold all of it.",
                  fraction * 100.0, static_cast<double>(minBytesRequired(info, meta)) / 1e9);
    return buf;
}

std::string PipelineRegistry::unsupportedReason(const PipelineInfo& info, const CloudMeta& meta,
                                                const DeviceBudget& budget) const {
    if (!fits(info, meta, budget)) {
        const double inputGB = static_cast<double>(inputBytesFor(info, meta)) / 1e9;
        const char* input = info.needsWholeCloudResident ? "resident cloud" : "ring";
        char buf[384];
        if (info.minStoreBytes == 0) {
            std::snprintf(buf, sizeof(buf),
                          "needs %.1f GB for %llu points and cannot build a partial tree (%.0f B/pt structure + "
                          "%.1f GB %s + %.2f GB fixed); the budget is %.1f GB",
                          static_cast<double>(minBytesRequired(info, meta)) / 1e9,
                          static_cast<unsigned long long>(meta.numPoints), info.minBytesPerPointEstimate, inputGB,
                          input, static_cast<double>(info.fixedBytesEstimate) / 1e9,
                          static_cast<double>(budget.bytes) / 1e9);
        } else {
            std::snprintf(buf, sizeof(buf),
                          "cannot run at all below %.1f GB (%.1f GB %s + %.2f GB fixed + %.2f GB smallest store); "
                          "the budget is %.1f GB. The whole cloud would need %.1f GB.",
                          static_cast<double>(refusalFloor(info, meta)) / 1e9, inputGB, input,
                          static_cast<double>(info.fixedBytesEstimate) / 1e9,
                          static_cast<double>(info.minStoreBytes) / 1e9, static_cast<double>(budget.bytes) / 1e9,
                          static_cast<double>(minBytesRequired(info, meta)) / 1e9);
        }
        return buf;
    }
    // A resident feed to a progressive pipeline only addresses 50 slots.
    if (info.needsWholeCloudResident && info.ringSlots == 0 && info.progressive &&
        meta.numPoints > kMaxAddressablePoints) {
        char buf[384];
        std::snprintf(buf, sizeof(buf),
                      "%s is configured for a resident cloud, and the builder addresses batch N at slot N %% %u, so "
                      "a resident feed can only describe %.0fM points; this cloud has %.0fM. A streaming ring has "
                      "no such limit.",
                      info.displayName.c_str(), kBatchStreamSize, static_cast<double>(kMaxAddressablePoints) / 1e6,
                      static_cast<double>(meta.numPoints) / 1e6);
        return buf;
    }
    return {};
}

bool PipelineRegistry::switchTo(const std::string& id, PointSource* source, const CloudMeta& meta,
                                const DeviceBudget& budget, std::string* err) {
    const Entry* entry = nullptr;
    for (const Entry& e : m_entries)
        if (e.info.id == id) entry = &e;
    if (!entry) {
        if (err) *err = "unknown pipeline: " + id;
        return false;
    }
    const std::string reason = unsupportedReason(entry->info, meta, budget);
    if (!reason.empty()) {
        if (err) *err = entry->info.displayName + ": " + reason;
        return false;
    }
    if (m_active) {
        m_active->release();
        m_active.reset();
        m_activeId.clear();
    }
    // The feed's shape is the incoming pipeline's, decided before it allocates
    // because the two share one budget.
    if (source) {
        const PointSource::Mode mode =
            entry->info.needsWholeCloudResident ? PointSource::Mode::Whole : PointSource::Mode::Stream;
        if (!source->start(mode, entry->info.ringSlots, budget.bytes, err)) return false;
        source->rewind();
    }
    std::unique_ptr<ILodPipeline> pipeline = entry->factory();
    if (!pipeline) {
        if (err) *err = "factory returned null for " + id;
        return false;
    }
    if (!pipeline->initPrograms(err)) return false;
    if (!pipeline->allocate(meta, budget, err)) return false;
    pipeline->reset();
    m_active = std::move(pipeline);
    m_activeId = id;
    return true;
}

bool PipelineRegistry::reloadForCloud(PointSource* source, const CloudMeta& meta, const DeviceBudget& budget,
                                      std::string* err) {
    if (!m_active) {
        if (err) *err = "no active pipeline";
        return false;
    }
    m_active->release();
    if (source) {
        const PipelineInfo* info = find(m_activeId);
        const bool resident = !info || info->needsWholeCloudResident;
        const PointSource::Mode mode = resident ? PointSource::Mode::Whole : PointSource::Mode::Stream;
        if (!source->start(mode, info ? info->ringSlots : 0, budget.bytes, err)) return false;
        source->rewind();
    }
    if (!m_active->allocate(meta, budget, err)) return false;
    m_active->reset();
    return true;
}

void PipelineRegistry::shutdown() {
    if (m_active) m_active->release();
    m_active.reset();
    m_activeId.clear();
}

}  // namespace rbhost
