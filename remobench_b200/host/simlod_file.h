// The .simlod point-cloud file (src/io/RawReader.h:10-16): a 24-byte header
// of six floats (a bounding box the loader never trusts) followed by 16-byte
// points {float x, y, z; uint32 rgba}, so point i sits at byte 24 + 16 i and
// any range can be read without parsing. The cloud's box is the observed one,
// scanned before the first upload, and points are stored relative to its
// minimum (src/io/PointSource.cpp:360-379).
#pragma once

#include <cstdint>
#include <string>

#include "rb_capi.h"

namespace rbhost {

struct SimlodInfo {
    uint64_t numPoints = 0;
    float headerBox[6] = {};  // min xyz, max xyz as written; informational only
};

// Size checks and the header: the payload must be a whole number of points, and
// at least one.
bool readSimlodHeader(const std::string& path, SimlodInfo& info, std::string* err);

// The observed bounds (min xyz, max xyz) of every point, in double.
bool readSimlodBounds(const std::string& path, const SimlodInfo& info, double bounds[6], std::string* err);

// Points [first, first + count) into out, each coordinate plus float(translation).
bool readSimlodRange(const std::string& path, const SimlodInfo& info, const double translation[3], uint64_t first,
                     uint64_t count, rb_point* out, std::string* err);

// Writes a .simlod file: the header box, then the points as given.
bool writeSimlod(const std::string& path, const rb_point* pts, uint64_t count, const float box[6], std::string* err);

}  // namespace rbhost
