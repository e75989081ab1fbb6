// The pipeline registry: registration, the memory gate and pipeline switches.
//
// The gate decides, before any device memory is touched, whether a pipeline
// may run a cloud in a byte budget, and how much of the cloud it will hold.
// Its decisions are the reference registry's (src/shell/PipelineRegistry.cpp:
// 20-274), restated here from these rules:
//
//   feed     bytes of point input the pipeline keeps on the device: the whole
//            cloud at 16 B a point for a resident feed, else a ring of
//            min(ringSlots, batches in the cloud) slots of kSlotCapacity points;
//   need     what the whole cloud takes: minBytesPerPoint x points + feed +
//            the pipeline's fixed buffers;
//   floor    the smallest budget it runs in at all: `need` for a pipeline that
//            cannot stop on a partial tree (minStoreBytes == 0), else its
//            smallest store + feed + fixed buffers;
//   fraction of the cloud predicted to fit: the store is the pipeline's
//            appetite (bytesPerPoint x points) capped by what the budget
//            leaves after feed and fixed buffers; ingest stops kSafetyMargin
//            short of the store's end, and each stored point costs
//            minBytesPerPoint (so a small cloud is predicted at 0% although
//            allocate() would raise its store to the 512 MB floor -- kept, as
//            the reference predicts it);
//   ceiling  a resident feed to a progressive builder can only describe
//            kRingDepth batches, because the builder finds batch b at slot
//            b mod kRingDepth.
//
// A switch gates first, then releases the running pipeline, re-shapes the
// point source for the incoming one (both share the budget), and brings the
// incoming pipeline up: create, initPrograms, allocate, reset.
#include "pipeline_registry.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>

namespace rbhost {

namespace {

double gigabytes(uint64_t bytes) { return static_cast<double>(bytes) / 1e9; }

std::string format(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return buf;
}

// Every figure the gate derives for one (pipeline, cloud, budget).
struct GateFigures {
    uint64_t feed = 0;       // device bytes of point input
    uint64_t need = 0;       // budget that holds the whole cloud
    uint64_t floor = 0;      // budget below which the pipeline is refused
    bool fits = false;
    double fraction = 0.0;   // predicted share of the cloud ingested
};

bool streams(const PipelineInfo& info) { return !info.needsWholeCloudResident && info.ringSlots > 0; }

PointSource::Mode feedMode(const PipelineInfo* info) {
    return (info == nullptr || info->needsWholeCloudResident) ? PointSource::Mode::Whole : PointSource::Mode::Stream;
}

GateFigures gate(const PipelineInfo& info, const CloudMeta& meta, uint64_t budget) {
    GateFigures g;
    g.feed = inputBytesFor(info, meta);
    const uint64_t overhead = g.feed + info.fixedBytesEstimate;
    g.need = static_cast<uint64_t>(info.minBytesPerPointEstimate * static_cast<double>(meta.numPoints)) + overhead;
    const bool truncates = info.minStoreBytes != 0;
    g.floor = truncates ? info.minStoreBytes + overhead : g.need;
    g.fits = g.floor <= budget;
    if (meta.numPoints == 0) {
        g.fraction = 1.0;
    } else if (info.minBytesPerPointEstimate <= 0.0) {
        g.fraction = g.fits ? 1.0 : 0.0;  // no per-point store: all or nothing
    } else if (budget > overhead) {
        const uint64_t appetite =
            static_cast<uint64_t>(info.bytesPerPointEstimate * static_cast<double>(meta.numPoints));
        const uint64_t store = std::min(appetite, budget - overhead);
        const uint64_t usable = store > kPersistentSafetyMargin ? store - kPersistentSafetyMargin : 0;
        const double storedPoints = static_cast<double>(usable) / info.minBytesPerPointEstimate;
        g.fraction = std::clamp(storedPoints / static_cast<double>(meta.numPoints), 0.0, 1.0);
    }
    return g;
}

}  // namespace

uint64_t inputBytesFor(const PipelineInfo& info, const CloudMeta& meta) {
    constexpr uint64_t kPointBytes = sizeof(rb_point);
    if (!streams(info)) return meta.numPoints * kPointBytes;
    const uint64_t batches = (meta.numPoints + kSlotCapacity - 1) / kSlotCapacity;
    return std::min<uint64_t>(info.ringSlots, batches) * kSlotCapacity * kPointBytes;
}

void PipelineRegistry::add(PipelineFactory factory) {
    // a throwaway instance tells the registry what the factory makes
    std::unique_ptr<ILodPipeline> sample = factory ? factory() : nullptr;
    if (!sample) {
        std::fprintf(stderr, "rbhost: registration skipped: the factory is empty or made no pipeline\n");
        return;
    }
    PipelineInfo info = sample->info();
    sample.reset();
    const char* why = info.id.empty() ? "it has no id" : (find(info.id) ? "its id is taken" : nullptr);
    if (why) {
        std::fprintf(stderr, "rbhost: pipeline '%s' not registered: %s\n", info.id.c_str(), why);
        return;
    }
    m_infos.push_back(info);
    m_entries.push_back(Entry{std::move(info), std::move(factory)});
}

const PipelineInfo* PipelineRegistry::find(const std::string& id) const {
    const auto it = std::find_if(m_entries.begin(), m_entries.end(), [&](const Entry& e) { return e.info.id == id; });
    return it == m_entries.end() ? nullptr : &it->info;
}

uint64_t PipelineRegistry::minBytesRequired(const PipelineInfo& info, const CloudMeta& meta) const {
    return gate(info, meta, 0).need;
}

uint64_t PipelineRegistry::refusalFloor(const PipelineInfo& info, const CloudMeta& meta) const {
    return gate(info, meta, 0).floor;
}

bool PipelineRegistry::fits(const PipelineInfo& info, const CloudMeta& meta, const DeviceBudget& budget) const {
    return gate(info, meta, budget.bytes).fits;
}

double PipelineRegistry::predictedCompletion(const PipelineInfo& info, const CloudMeta& meta,
                                             const DeviceBudget& budget) const {
    return gate(info, meta, budget.bytes).fraction;
}

std::string PipelineRegistry::completionWarning(const PipelineInfo& info, const CloudMeta& meta,
                                                const DeviceBudget& budget) const {
    const GateFigures g = gate(info, meta, budget.bytes);
    if (g.fraction >= 0.999) return {};
    return format("predicted to take in about %.0f%% of the cloud before its store fills; the build then ends on "
                  "a partial tree (memCapacityReached). The whole cloud needs a %.1f GB budget.",
                  g.fraction * 100.0, gigabytes(g.need));
}

std::string PipelineRegistry::unsupportedReason(const PipelineInfo& info, const CloudMeta& meta,
                                                const DeviceBudget& budget) const {
    const GateFigures g = gate(info, meta, budget.bytes);
    const char* feedName = info.needsWholeCloudResident ? "resident cloud" : "ring";
    if (!g.fits && info.minStoreBytes == 0) {
        return format("refused: the whole cloud (%llu points) needs %.1f GB -- %.0f B per point, a %.1f GB %s and "
                      "%.2f GB of fixed buffers -- and this pipeline cannot stop on a partial tree; the budget is "
                      "%.1f GB",
                      static_cast<unsigned long long>(meta.numPoints), gigabytes(g.need),
                      info.minBytesPerPointEstimate, gigabytes(g.feed), feedName,
                      gigabytes(info.fixedBytesEstimate), gigabytes(budget.bytes));
    }
    if (!g.fits) {
        return format("refused: the budget is %.1f GB, below this pipeline's floor of %.1f GB (a %.1f GB %s, "
                      "%.2f GB of fixed buffers and a %.2f GB smallest store); the whole cloud needs %.1f GB",
                      gigabytes(budget.bytes), gigabytes(g.floor), gigabytes(g.feed), feedName,
                      gigabytes(info.fixedBytesEstimate), gigabytes(info.minStoreBytes), gigabytes(g.need));
    }
    if (info.progressive && info.needsWholeCloudResident && info.ringSlots == 0 &&
        meta.numPoints > kMaxAddressablePoints) {
        return format("refused: %s keeps the cloud resident, but its builder finds batch b in slot b mod %u, so a "
                      "resident feed reaches only the first %.0fM points of this %.0fM-point cloud; a streaming ring "
                      "has no such ceiling",
                      info.displayName.c_str(), kBatchStreamSize, kMaxAddressablePoints / 1e6,
                      static_cast<double>(meta.numPoints) / 1e6);
    }
    return {};
}

bool PipelineRegistry::switchTo(const std::string& id, PointSource* source, const CloudMeta& meta,
                                const DeviceBudget& budget, std::string* err) {
    auto fail = [&](const std::string& msg) {
        if (err) *err = msg;
        return false;
    };
    const auto entry = std::find_if(m_entries.begin(), m_entries.end(), [&](const Entry& e) { return e.info.id == id; });
    if (entry == m_entries.end()) return fail("unknown pipeline: " + id);
    const std::string refusal = unsupportedReason(entry->info, meta, budget);
    if (!refusal.empty()) return fail(entry->info.displayName + ": " + refusal);

    // one pipeline holds device memory at a time: the old one goes first
    shutdown();
    if (source) {
        if (!source->start(feedMode(&entry->info), entry->info.ringSlots, budget.bytes, err)) return false;
        source->rewind();
    }
    std::unique_ptr<ILodPipeline> incoming = entry->factory();
    if (!incoming) return fail("the factory of " + id + " made no pipeline");
    if (!incoming->initPrograms(err) || !incoming->allocate(meta, budget, err)) return false;
    incoming->reset();
    m_active = std::move(incoming);
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
        if (!source->start(feedMode(info), info ? info->ringSlots : 0, budget.bytes, err)) return false;
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
