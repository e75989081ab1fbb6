// Prints the registry's gate decisions for a fixed table of clouds and
// budgets as "key value" lines; tests/test_host.py checks them. Touches no
// GPU: registration, gating and the unknown-id path make no CUDA call.
#include <cstdio>
#include <string>

#include "lod_pipeline.h"
#include "pipeline_registry.h"
#include "point_source.h"

using namespace rbhost;

namespace {

// A resident progressive pipeline: the only kind the 50-slot ceiling applies to.
class ResidentProgressive final : public ILodPipeline {
public:
    PipelineInfo info() const override {
        PipelineInfo i;
        i.id = "resident";
        i.displayName = "Resident";
        i.progressive = true;
        i.needsWholeCloudResident = true;
        i.ringSlots = 0;
        i.bytesPerPointEstimate = 48.0;
        i.minBytesPerPointEstimate = 26.0;
        i.minStoreBytes = 512ull << 20;
        return i;
    }
    bool initPrograms(std::string*) override { return true; }
    bool allocate(const CloudMeta&, const DeviceBudget&, std::string*) override { return true; }
    void release() override {}
    void reset() override {}
    bool build(PointSource&, const FrameContext&) override { return false; }
    void render(const FrameContext&) override {}
    const PipelineStats& stats() const override { return m_stats; }
    TimingScopes timingScopes() const override { return {}; }

private:
    PipelineStats m_stats;
};

void report(const PipelineRegistry& reg, const char* tag, const char* id, uint64_t points, double budgetBytes) {
    const PipelineInfo* info = reg.find(id);
    if (!info) {
        std::printf("%s.missing 1\n", tag);
        return;
    }
    CloudMeta meta;
    meta.numPoints = points;
    DeviceBudget b;
    b.bytes = static_cast<uint64_t>(budgetBytes);
    std::printf("%s.input %llu\n", tag, (unsigned long long)inputBytesFor(*info, meta));
    std::printf("%s.min_required %llu\n", tag, (unsigned long long)reg.minBytesRequired(*info, meta));
    std::printf("%s.floor %llu\n", tag, (unsigned long long)reg.refusalFloor(*info, meta));
    std::printf("%s.fits %d\n", tag, reg.fits(*info, meta, b) ? 1 : 0);
    std::printf("%s.predicted %.9f\n", tag, reg.predictedCompletion(*info, meta, b));
    std::printf("%s.warning %s\n", tag, reg.completionWarning(*info, meta, b).c_str());
    std::printf("%s.reason %s\n", tag, reg.unsupportedReason(*info, meta, b).c_str());
}

}  // namespace

int main() {
    PipelineRegistry reg;
    reg.add([] { return makeRemolodPipeline(0); });
    reg.add([] { return makeSimlodPipeline(0); });
    reg.add([] { return makeFlatPipeline(0); });
    reg.add([] { return makeRemolodPipeline(0); });  // duplicate id: not registered
    reg.add([] { return std::unique_ptr<ILodPipeline>(new ResidentProgressive()); });
    reg.add(nullptr);
    std::printf("registered %zu\n", reg.list().size());
    for (const PipelineInfo& i : reg.list())
        std::printf("info.%s %s %d %d %u %.1f %.1f %llu %llu\n", i.id.c_str(), i.displayName.c_str(),
                    i.progressive ? 1 : 0, i.needsWholeCloudResident ? 1 : 0, i.ringSlots, i.bytesPerPointEstimate,
                    i.minBytesPerPointEstimate, (unsigned long long)i.minStoreBytes,
                    (unsigned long long)i.fixedBytesEstimate);

    report(reg, "remolod_100M_3GB", "remolod", 100000000ull, 3e9);
    report(reg, "remolod_100M_1.9GB", "remolod", 100000000ull, 1.9e9);
    report(reg, "simlod_1B_180GB", "simlod", 1000000000ull, 180e9);
    report(reg, "remolod_2M_8GB", "remolod", 2000000ull, 8e9);
    report(reg, "flat_100M_1.5GB", "flat", 100000000ull, 1.5e9);
    report(reg, "flat_100M_2GB", "flat", 100000000ull, 2e9);
    report(reg, "resident_60M_100GB", "resident", 60000000ull, 100e9);
    report(reg, "resident_40M_100GB", "resident", 40000000ull, 100e9);

    CloudMeta meta;
    meta.numPoints = 1000;
    DeviceBudget b;
    b.bytes = 1ull << 40;
    std::string err;
    const bool ok = reg.switchTo("nonesuch", nullptr, meta, b, &err);
    std::printf("switch_unknown %d %s\n", ok ? 1 : 0, err.c_str());
    err.clear();
    const bool ok2 = reg.reloadForCloud(nullptr, meta, b, &err);
    std::printf("reload_inactive %d %s\n", ok2 ? 1 : 0, err.c_str());
    b.bytes = 1000;
    err.clear();
    const bool ok3 = reg.switchTo("remolod", nullptr, meta, b, &err);
    std::printf("switch_refused %d %s\n", ok3 ? 1 : 0, err.c_str());
    return 0;
}
