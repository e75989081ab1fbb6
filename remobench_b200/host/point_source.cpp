// Host-memory and synthetic point sources over a device ring
// (src/io/PointSource.cpp:94-345, headless): same window, rewind and overrun
// rules; uploads are cudaMemcpyAsync on the source's own stream, finished
// before pump() returns so the consumer's next build sees them.
#include "point_source.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>

#include "simlod_file.h"
#include "synth.h"

namespace rbhost {

double CloudMeta::worstQuantisationError() const {
    double worst = 0.0;
    for (int a = 0; a < 3; a++) {
        const double extent = boxMaxOrig[a] - boxMinOrig[a];
        if (extent <= 0.0) continue;
        int e = 0;
        std::frexp(extent, &e);
        worst = std::max(worst, std::ldexp(0.5, e - 24));  // half an ulp of float at the far corner
    }
    return worst;
}

namespace {

static uint32_t batchCount(uint64_t numPoints, uint32_t batch) {
    return static_cast<uint32_t>((numPoints + batch - 1) / batch);
}

// Reads points [first, first + count) of the cloud into dst (host memory).
using RangeReader = std::function<bool(uint64_t first, uint64_t count, rb_point* dst, std::string* err)>;

// A cloud fed to the device ring either from host memory (uploaded straight
// from its registered pages) or from a reader that fills a pinned staging
// batch per upload (a .simlod file streamed from disk, as the reference's
// SimlodFileProducer does).
class MemorySource final : public PointSource {
public:
    MemorySource(std::vector<rb_point> points, const CloudMeta& meta, uint32_t batchSize, int device)
        : m_points(std::move(points)), m_meta(meta), m_batch(std::max<uint32_t>(1, std::min(batchSize, kSlotCapacity))),
          m_device(device) {
        m_meta.numPoints = m_points.size();
    }
    MemorySource(RangeReader reader, const CloudMeta& meta, uint32_t batchSize, int device)
        : m_reader(std::move(reader)), m_meta(meta),
          m_batch(std::max<uint32_t>(1, std::min(batchSize, kSlotCapacity))), m_device(device) {}
    ~MemorySource() override {
        stop();
        if (m_registered) cudaHostUnregister(m_points.data());
        if (m_staging) cudaFreeHost(m_staging);
        if (m_stream) cudaStreamDestroy(m_stream);
    }

    const CloudMeta& meta() const override { return m_meta; }

    bool start(Mode mode, uint32_t ringSlots, uint64_t maxDeviceBytes, std::string* err) override {
        if (m_meta.numPoints == 0) {
            if (err) *err = "the source holds no points";
            return false;
        }
        // Whole mode puts batch B at base + B * kSlotCapacity with no gaps, so the
        // resident cloud is one contiguous array: its batches are slot-sized.
        const uint32_t batch = mode == Mode::Whole ? kSlotCapacity : m_batch;
        const uint32_t total = batchCount(m_meta.numPoints, batch);
        if (mode == Mode::Stream && ringSlots == 0) {
            if (err) *err = "Stream mode was asked for with a ring depth of 0 slots";
            return false;
        }
        const uint32_t slots = mode == Mode::Whole ? total : std::min(ringSlots, total);
        if (m_slots && m_mode == mode && m_numSlots == slots && m_curBatch == batch) {
            rewind();
            return true;
        }
        stop();
        if (cudaSetDevice(m_device) != cudaSuccess) {
            if (err) *err = "cudaSetDevice failed";
            return false;
        }
        const uint64_t bytes = mode == Mode::Whole ? m_meta.numPoints * sizeof(rb_point)
                                                   : uint64_t(slots) * kSlotCapacity * sizeof(rb_point);
        if (maxDeviceBytes && bytes > maxDeviceBytes) {
            if (err)
                *err = "the " + std::string(mode == Mode::Whole ? "resident cloud" : "ring") + " needs " +
                       std::to_string(bytes >> 20) + " MB, over the " + std::to_string(maxDeviceBytes >> 20) +
                       " MB budget";
            return false;
        }
        if (!m_stream && cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking) != cudaSuccess) {
            if (err) *err = "cudaStreamCreate failed";
            return false;
        }
        if (!m_reader && !m_registered) {
            // Pinned pages make the uploads run at full PCIe / C2C rate; pageable
            // copies still work if registration is refused.
            m_registered = cudaHostRegister(m_points.data(), m_points.size() * sizeof(rb_point),
                                            cudaHostRegisterDefault) == cudaSuccess;
            if (!m_registered) cudaGetLastError();
        }
        if (m_reader && !m_staging &&
            cudaMallocHost(reinterpret_cast<void**>(&m_staging), uint64_t(kSlotCapacity) * sizeof(rb_point)) !=
                cudaSuccess) {
            cudaGetLastError();
            m_staging = nullptr;
            if (err) *err = "cudaMallocHost failed for the file staging batch";
            return false;
        }
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            if (err) *err = "cudaMalloc failed for the point ring (" + std::to_string(bytes >> 20) + " MB)";
            return false;
        }
        m_slots = reinterpret_cast<uint64_t>(p);
        m_mode = mode;
        m_curBatch = batch;
        m_numSlots = slots;
        m_numBatchesTotal = total;
        m_sizes.assign(slots, 0);
        rewind();
        return true;
    }

    void rewind() override {
        m_produced = 0;
        m_consumed = 0;
        m_uploaded = 0;
        m_overran = false;
        std::fill(m_sizes.begin(), m_sizes.end(), 0u);
        if (m_mode == Mode::Whole) pump();
    }

    void stop() override {
        if (m_slots) {
            cudaSetDevice(m_device);
            cudaFree(reinterpret_cast<void*>(m_slots));
        }
        m_slots = 0;
        m_numSlots = m_numBatchesTotal = 0;
        m_produced = m_consumed = 0;
        m_uploaded = 0;
        m_sizes.clear();
    }

    void pump() override {
        if (!m_slots) return;
        // Slot B % numSlots still holds batch B - numSlots until the consumer is past it.
        const uint64_t limit = std::min<uint64_t>(m_numBatchesTotal, uint64_t(m_consumed) + m_numSlots);
        bool issued = false;
        while (m_produced < limit) {
            if (!uploadBatch(m_produced)) break;
            ++m_produced;
            issued = true;
        }
        if (issued) cudaStreamSynchronize(m_stream);
    }

    BatchView view() const override {
        BatchView v;
        v.slots = m_slots;
        v.batchSizes = m_sizes.empty() ? nullptr : m_sizes.data();
        v.numBatchesUploaded = static_cast<uint32_t>(m_produced);
        v.slotCapacity = m_mode == Mode::Whole ? m_curBatch : kSlotCapacity;
        v.numSlots = m_numSlots;
        v.numBatchesTotal = m_numBatchesTotal;
        v.wrapping = m_numBatchesTotal > m_numSlots;
        return v;
    }

    uint64_t numPointsUploaded() const override { return m_uploaded; }
    bool isFullyResident() const override {
        return m_mode == Mode::Whole && m_slots != 0 && m_uploaded == m_meta.numPoints;
    }
    uint64_t residentPoints() const override { return m_mode == Mode::Whole ? m_slots : 0; }

    void setBatchesConsumed(uint32_t numBatches) override {
        numBatches = std::min(numBatches, m_numBatchesTotal);
        if (numBatches > m_consumed) m_consumed = numBatches;
    }
    bool overranConsumer() const override { return m_overran; }

private:
    bool uploadBatch(uint64_t b) {
        if (b >= uint64_t(m_consumed) + m_numSlots) {
            if (!m_overran) {
                m_overran = true;
                std::fprintf(stderr,
                             "rbhost: ring overrun -- batch %llu would overwrite a slot the consumer has not "
                             "read (consumed %u, depth %u); refused\n",
                             static_cast<unsigned long long>(b), m_consumed, m_numSlots);
            }
            return false;
        }
        const uint64_t first = b * m_curBatch;
        const uint64_t count = std::min<uint64_t>(m_curBatch, m_meta.numPoints - first);
        const uint32_t slot = static_cast<uint32_t>(b % m_numSlots);
        const uint64_t stride = m_mode == Mode::Whole ? m_curBatch : kSlotCapacity;
        rb_point* dst = reinterpret_cast<rb_point*>(m_slots) + uint64_t(slot) * stride;
        const rb_point* src = m_points.data() + first;
        if (m_reader) {
            // the staging batch is reused: the previous upload must be done
            if (cudaStreamSynchronize(m_stream) != cudaSuccess) return false;
            std::string err;
            if (!m_reader(first, count, m_staging, &err)) {
                std::fprintf(stderr, "rbhost: %s\n", err.c_str());
                return false;
            }
            src = m_staging;
        }
        if (cudaMemcpyAsync(dst, src, count * sizeof(rb_point), cudaMemcpyHostToDevice, m_stream) != cudaSuccess)
            return false;
        m_sizes[slot] = static_cast<uint32_t>(count);
        m_uploaded += count;
        return true;
    }

    std::vector<rb_point> m_points;
    RangeReader m_reader;
    rb_point* m_staging = nullptr;  // pinned, one slot of points (reader sources)
    CloudMeta m_meta;
    uint32_t m_batch;
    int m_device;
    bool m_registered = false;
    cudaStream_t m_stream = nullptr;
    Mode m_mode = Mode::Whole;
    uint32_t m_curBatch = kSlotCapacity;
    uint64_t m_slots = 0;
    uint32_t m_numSlots = 0;
    uint32_t m_numBatchesTotal = 0;
    std::vector<uint32_t> m_sizes;
    uint64_t m_produced = 0;
    uint32_t m_consumed = 0;
    uint64_t m_uploaded = 0;
    bool m_overran = false;
};

}  // namespace

std::unique_ptr<PointSource> makeMemorySource(std::vector<rb_point> points, const CloudMeta& meta,
                                              uint32_t batchSize, int device) {
    return std::make_unique<MemorySource>(std::move(points), meta, batchSize, device);
}

std::unique_ptr<PointSource> makeSyntheticSource(int config, uint64_t numPoints, uint64_t seed,
                                                 uint32_t batchSize, int device, std::string* err) {
    rb_synth_config cfg;
    if (rb_synth_default_config(config, &cfg) != 0) {
        if (err) *err = "unknown synthetic configuration " + std::to_string(config);
        return nullptr;
    }
    cfg.seed = seed;
    if (numPoints) cfg.num_points = numPoints;
    if (batchSize) cfg.batch_size = batchSize;
    if (cfg.batch_size > kSlotCapacity) {
        if (err) *err = "batch size exceeds the slot capacity";
        return nullptr;
    }
    rb_synth_scene_info info;
    if (rb_synth_scene_info_get(&cfg, &info) != 0) {
        if (err) *err = "scene construction failed";
        return nullptr;
    }
    CloudMeta meta;
    meta.numPoints = cfg.num_points;
    for (int a = 0; a < 3; a++) {
        meta.boxMinOrig[a] = info.box_min[a];
        meta.boxMaxOrig[a] = info.box_max[a];
        meta.translation[a] = -info.box_min[a];
        meta.boxSize[a] = static_cast<float>(info.box_max[a] - info.box_min[a]);
    }
    meta.isSyntheticFixture = true;
    std::vector<rb_point> pts(cfg.num_points);
    static_assert(sizeof(rb_point) == sizeof(rb_synth_point), "point layouts differ");
    if (rb_synth_generate(&cfg, 0, cfg.num_points, 1, reinterpret_cast<rb_synth_point*>(pts.data())) != 0) {
        if (err) *err = "point generation failed";
        return nullptr;
    }
    return makeMemorySource(std::move(pts), meta, cfg.batch_size, device);
}

std::unique_ptr<PointSource> makeSimlodSource(const std::string& path, uint32_t batchSize, int device,
                                              std::string* err) {
    SimlodInfo info;
    if (!readSimlodHeader(path, info, err)) return nullptr;
    // the observed box, not the header's (src/io/PointSource.cpp:515-531)
    double bounds[6];
    if (!readSimlodBounds(path, info, bounds, err)) return nullptr;
    CloudMeta meta;
    meta.numPoints = info.numPoints;
    for (int a = 0; a < 3; a++) {
        meta.boxMinOrig[a] = bounds[a];
        meta.boxMaxOrig[a] = bounds[3 + a];
        // deriveTranslation (PointSource.cpp:360-366)
        meta.translation[a] = -bounds[a];
        meta.boxSize[a] = static_cast<float>(bounds[3 + a] + meta.translation[a]);
    }
    const double t[3] = {meta.translation[0], meta.translation[1], meta.translation[2]};
    RangeReader reader = [path, info, t](uint64_t first, uint64_t count, rb_point* dst, std::string* e) {
        return readSimlodRange(path, info, t, first, count, dst, e);
    };
    return std::make_unique<MemorySource>(std::move(reader), meta, batchSize ? batchSize : kSlotCapacity, device);
}

}  // namespace rbhost
