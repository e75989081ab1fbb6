// PointSource (include/remo/PointSource.h:16-125), headless: a cloud held in
// host memory (or produced batch by batch by the seeded generator) fed to a
// device ring of kSlotCapacity-point slots (Stream) or made resident whole
// (Whole), with the reference's producer window and consumption handshake.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "rb_capi.h"

namespace rbhost {

// Points per slot (PointSource.h:34-41): the ring's stride whatever the batch sizes.
constexpr uint32_t kSlotCapacity = 1000000;

// CloudMeta (PointSource.h:16-32). Points are stored relative to boxMinOrig,
// so the octree box is [0, boxSize].
struct CloudMeta {
    uint64_t numPoints = 0;
    double boxMinOrig[3] = {0, 0, 0};
    double boxMaxOrig[3] = {0, 0, 0};
    double translation[3] = {0, 0, 0};
    float boxSize[3] = {0, 0, 0};
    bool isSyntheticFixture = false;
    // Largest error of storing a coordinate as float relative to boxMinOrig
    // (half a float ulp at the far corner of the box).
    double worstQuantisationError() const;
};

// BatchView (PointSource.h:43-67). slots is a device address; batchSizes is
// host memory (numSlots entries) and numBatchesUploaded a host count, since
// the C ABI reads both at the call.
struct BatchView {
    uint64_t slots = 0;
    const uint32_t* batchSizes = nullptr;
    uint32_t numBatchesUploaded = 0;
    uint32_t slotCapacity = kSlotCapacity;
    uint32_t numSlots = 0;
    uint32_t numBatchesTotal = 0;
    bool wrapping = false;
};

class PointSource {
public:
    enum class Mode { Stream, Whole };
    virtual ~PointSource() = default;
    virtual const CloudMeta& meta() const = 0;
    // Re-entrant: a different mode restarts ingest in that mode. ringSlots is
    // ignored in Whole mode. Fails if the ring or cloud exceeds maxDeviceBytes.
    virtual bool start(Mode mode, uint32_t ringSlots, uint64_t maxDeviceBytes, std::string* err) = 0;
    // Back to batch 0 in the current mode (any consumer reset calls this).
    virtual void rewind() = 0;
    virtual void stop() = 0;
    // Uploads every batch the consumer window allows: batch B may be written
    // only once the consumer has read batch B - numSlots.
    virtual void pump() = 0;
    virtual BatchView view() const = 0;
    virtual uint64_t numPointsUploaded() const = 0;
    virtual bool isFullyResident() const = 0;
    virtual uint64_t residentPoints() const = 0;  // device address in Whole mode, else 0
    // The consumption signal in batches (Stats::batchletIndex); only moves forward.
    virtual void setBatchesConsumed(uint32_t numBatches) = 0;
    // Set once if the producer was ever asked to write past the window.
    virtual bool overranConsumer() const = 0;
};

// A cloud already in host memory (coordinates relative to meta.boxMinOrig).
// batchSize <= kSlotCapacity points go into each slot.
std::unique_ptr<PointSource> makeMemorySource(std::vector<rb_point> points, const CloudMeta& meta,
                                              uint32_t batchSize = kSlotCapacity, int device = 0);

// A .simlod file (simlod_file.h) streamed from disk batch by batch: the
// observed box, points translated to its minimum.
std::unique_ptr<PointSource> makeSimlodSource(const std::string& path, uint32_t batchSize, int device,
                                              std::string* err);

// The seeded synthetic lidar generator (synth.h), configuration 1, 2, 3 or 5,
// generating each batch when the window opens for it. numPoints 0 keeps the
// configuration's size.
std::unique_ptr<PointSource> makeSyntheticSource(int config, uint64_t numPoints, uint64_t seed,
                                                 uint32_t batchSize, int device, std::string* err);

}  // namespace rbhost
