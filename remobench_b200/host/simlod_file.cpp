// .simlod reading and writing with plain stdio: the reads are large and
// sequential (the bounds scan walks the file in 1 MB blocks; a batch is one
// seek and one read), so no buffering layer is needed.
#include "simlod_file.h"

#include <algorithm>
#include <cstdio>
#include <memory>
#include <vector>

namespace rbhost {

namespace {

constexpr uint64_t kHeaderBytes = 24;
constexpr uint64_t kPointBytes = 16;
constexpr uint64_t kScanBlock = 65536;  // points per read of the bounds scan (1 MB)

struct FileCloser {
    void operator()(std::FILE* f) const {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<std::FILE, FileCloser>;

File openAt(const std::string& path, uint64_t byteOffset, std::string* err) {
    File f(std::fopen(path.c_str(), "rb"));
    if (!f) {
        if (err) *err = "cannot open " + path;
        return nullptr;
    }
    if (fseeko(f.get(), static_cast<off_t>(byteOffset), SEEK_SET) != 0) {
        if (err) *err = "cannot seek to byte " + std::to_string(byteOffset) + " of " + path;
        return nullptr;
    }
    return f;
}

}  // namespace

bool readSimlodHeader(const std::string& path, SimlodInfo& info, std::string* err) {
    File f = openAt(path, 0, err);
    if (!f) return false;
    if (fseeko(f.get(), 0, SEEK_END) != 0) {
        if (err) *err = "cannot size " + path;
        return false;
    }
    const off_t size = ftello(f.get());
    if (size < 0 || static_cast<uint64_t>(size) < kHeaderBytes) {
        if (err) *err = path + " is shorter than the 24-byte .simlod header";
        return false;
    }
    const uint64_t payload = static_cast<uint64_t>(size) - kHeaderBytes;
    if (payload % kPointBytes != 0) {
        if (err) *err = path + ": " + std::to_string(payload) + " bytes after the header is not a whole number of " +
                        "16-byte points (a truncated file?)";
        return false;
    }
    if (payload == 0) {
        if (err) *err = path + " has a header and no points";
        return false;
    }
    std::rewind(f.get());
    if (std::fread(info.headerBox, sizeof(float), 6, f.get()) != 6) {
        if (err) *err = "cannot read the header of " + path;
        return false;
    }
    info.numPoints = payload / kPointBytes;
    return true;
}

bool readSimlodBounds(const std::string& path, const SimlodInfo& info, double bounds[6], std::string* err) {
    File f = openAt(path, kHeaderBytes, err);
    if (!f) return false;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    std::vector<rb_point> block(static_cast<size_t>(std::min<uint64_t>(kScanBlock, info.numPoints)));
    for (uint64_t done = 0; done < info.numPoints;) {
        const uint64_t n = std::min<uint64_t>(kScanBlock, info.numPoints - done);
        if (std::fread(block.data(), kPointBytes, n, f.get()) != n) {
            if (err) *err = "short read at point " + std::to_string(done) + " of " + path;
            return false;
        }
        for (uint64_t i = 0; i < n; i++) {
            const double v[3] = {block[i].x, block[i].y, block[i].z};
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], v[a]);
                hi[a] = std::max(hi[a], v[a]);
            }
        }
        done += n;
    }
    for (int a = 0; a < 3; a++) {
        bounds[a] = lo[a];
        bounds[3 + a] = hi[a];
    }
    return true;
}

bool readSimlodRange(const std::string& path, const SimlodInfo& info, const double translation[3], uint64_t first,
                     uint64_t count, rb_point* out, std::string* err) {
    if (first > info.numPoints || count > info.numPoints - first) {
        if (err) *err = "points [" + std::to_string(first) + ", " + std::to_string(first + count) + ") lie past the " +
                        std::to_string(info.numPoints) + " points of " + path;
        return false;
    }
    File f = openAt(path, kHeaderBytes + first * kPointBytes, err);
    if (!f) return false;
    if (std::fread(out, kPointBytes, count, f.get()) != count) {
        if (err) *err = "short read of " + std::to_string(count) + " points from " + path;
        return false;
    }
    const float t[3] = {static_cast<float>(translation[0]), static_cast<float>(translation[1]),
                        static_cast<float>(translation[2])};
    if (t[0] == 0.0f && t[1] == 0.0f && t[2] == 0.0f) return true;
    for (uint64_t i = 0; i < count; i++) {
        out[i].x += t[0];
        out[i].y += t[1];
        out[i].z += t[2];
    }
    return true;
}

bool writeSimlod(const std::string& path, const rb_point* pts, uint64_t count, const float box[6], std::string* err) {
    File f(std::fopen(path.c_str(), "wb"));
    if (!f) {
        if (err) *err = "cannot create " + path;
        return false;
    }
    if (std::fwrite(box, sizeof(float), 6, f.get()) != 6 || std::fwrite(pts, kPointBytes, count, f.get()) != count) {
        if (err) *err = "short write to " + path;
        return false;
    }
    if (std::fflush(f.get()) != 0) {
        if (err) *err = "cannot flush " + path;
        return false;
    }
    return true;
}

}  // namespace rbhost
