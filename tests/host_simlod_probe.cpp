// Reads a .simlod file through the C++ host's reader and prints what it found
// as "key value" lines for tests/test_simlod.py: the header, the observed
// bounds, the derived translation and an order-dependent digest of every
// translated point, read in two ranges. Touches no GPU.
#include <cstdio>
#include <string>
#include <vector>

#include "simlod_file.h"

using namespace rbhost;

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string path = argv[1];
    std::string err;
    SimlodInfo info;
    if (!readSimlodHeader(path, info, &err)) {
        std::printf("error %s\n", err.c_str());
        return 1;
    }
    std::printf("points %llu\n", static_cast<unsigned long long>(info.numPoints));
    std::printf("header %.9g %.9g %.9g %.9g %.9g %.9g\n", info.headerBox[0], info.headerBox[1], info.headerBox[2],
                info.headerBox[3], info.headerBox[4], info.headerBox[5]);
    double b[6];
    if (!readSimlodBounds(path, info, b, &err)) {
        std::printf("error %s\n", err.c_str());
        return 1;
    }
    std::printf("bounds %.17g %.17g %.17g %.17g %.17g %.17g\n", b[0], b[1], b[2], b[3], b[4], b[5]);
    const double t[3] = {-b[0], -b[1], -b[2]};
    const uint64_t half = info.numPoints / 2;
    std::vector<rb_point> pts(info.numPoints);
    if (!readSimlodRange(path, info, t, 0, half, pts.data(), &err) ||
        !readSimlodRange(path, info, t, half, info.numPoints - half, pts.data() + half, &err)) {
        std::printf("error %s\n", err.c_str());
        return 1;
    }
    uint64_t h = 1469598103934665603ull;
    for (const rb_point& p : pts) {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(&p);
        for (int k = 0; k < 4; k++) h = (h ^ w[k]) * 1099511628211ull;
    }
    std::printf("digest %llu\n", static_cast<unsigned long long>(h));
    rb_point tmp;
    std::printf("past_end %d\n", readSimlodRange(path, info, t, info.numPoints, 1, &tmp, &err) ? 1 : 0);
    return 0;
}
