// Headless frame loop of the reference's viewer (src/shell/App.cpp:395-470)
// over the C++ host layer: each frame renders, refills the ring within the
// consumer's window, then builds (render -> pump -> build), with the
// registry's gate, a pipeline switch after N frames and the frame dump
// (App.cpp:472-620: a PPM plus the stats report). Options follow
// src/main.cpp:251-320 where the reference has them.
//
//   rb_harness [--pipeline remolod|simlod|flat] [--synthetic N] [--config C] [--seed S]
//              [--batch B] [--size W H] [--device-budget GB] [--device D]
//              [--dump-frame out.ppm] [--dump-after F] [--switch-to ID] [--switch-after F]
//              [--max-frames F] [--frame-file uniforms.bin] [--surface-out rgba.bin]
//              [--strict-timing] [--trace] [--bounding-boxes] [--color-mode M] [--file cloud.simlod]
//
// Without --dump-after the loop runs until the build is complete (or stops on
// memCapacityReached), renders one more frame and stops. The last stdout line
// is a JSON summary.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lod_pipeline.h"
#include "pipeline_registry.h"
#include "point_source.h"

using namespace rbhost;

namespace {

struct Options {
    std::string pipeline = "remolod";
    std::string switchTo;
    long switchAfter = -1;
    uint64_t synthetic = 0;
    int config = 1;
    uint64_t seed = 1;
    uint32_t batch = 0;
    int width = 1920, height = 1080;
    double budgetGB = 0.0;
    int device = 0;
    std::string dumpFrame;
    long dumpAfter = -1;
    long maxFrames = 100000;
    std::string frameFile;
    std::string surfaceOut;
    bool strictTiming = false;
    bool trace = false;
    std::string file;       // a .simlod cloud streamed from disk instead of the generator
    bool boxes = false;     // the viewer's bounding-box toggle (SharedUniforms::showBoundingBox)
    int colorMode = 0;      // SharedUniforms::colorMode: rgb, node, lod, white
};

void usage() {
    std::fprintf(stderr,
                 "usage: rb_harness [--pipeline ID] [--synthetic N] [--config C] [--seed S] [--batch B]\n"
                 "                  [--size W H] [--device-budget GB] [--device D] [--dump-frame PATH]\n"
                 "                  [--dump-after F] [--switch-to ID] [--switch-after F] [--max-frames F]\n"
                 "                  [--frame-file PATH] [--surface-out PATH] [--strict-timing] [--trace]\n"
                 "                  [--bounding-boxes] [--color-mode rgb|node|lod|white] [--file PATH.simlod]\n");
}

bool parse(int argc, char** argv, Options* o) {
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&](const char* name) -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "rb_harness: %s needs a value\n", name);
                return nullptr;
            }
            return argv[++i];
        };
        const char* v = nullptr;
        if (a == "-h" || a == "--help") {
            usage();
            std::exit(0);
        } else if (a == "--pipeline") {
            if (!(v = next("--pipeline"))) return false;
            o->pipeline = v;
        } else if (a == "--switch-to") {
            if (!(v = next("--switch-to"))) return false;
            o->switchTo = v;
        } else if (a == "--switch-after") {
            if (!(v = next("--switch-after"))) return false;
            o->switchAfter = std::atol(v);
        } else if (a == "--synthetic") {
            if (!(v = next("--synthetic"))) return false;
            o->synthetic = std::strtoull(v, nullptr, 10);
        } else if (a == "--config") {
            if (!(v = next("--config"))) return false;
            o->config = std::atoi(v);
        } else if (a == "--seed") {
            if (!(v = next("--seed"))) return false;
            o->seed = std::strtoull(v, nullptr, 10);
        } else if (a == "--batch") {
            if (!(v = next("--batch"))) return false;
            o->batch = static_cast<uint32_t>(std::strtoul(v, nullptr, 10));
        } else if (a == "--size") {
            if (!(v = next("--size"))) return false;
            o->width = std::atoi(v);
            if (!(v = next("--size"))) return false;
            o->height = std::atoi(v);
        } else if (a == "--device-budget") {
            if (!(v = next("--device-budget"))) return false;
            o->budgetGB = std::atof(v);
        } else if (a == "--device") {
            if (!(v = next("--device"))) return false;
            o->device = std::atoi(v);
        } else if (a == "--dump-frame") {
            if (!(v = next("--dump-frame"))) return false;
            o->dumpFrame = v;
        } else if (a == "--dump-after") {
            if (!(v = next("--dump-after"))) return false;
            o->dumpAfter = std::atol(v);
        } else if (a == "--max-frames") {
            if (!(v = next("--max-frames"))) return false;
            o->maxFrames = std::atol(v);
        } else if (a == "--frame-file") {
            if (!(v = next("--frame-file"))) return false;
            o->frameFile = v;
        } else if (a == "--surface-out") {
            if (!(v = next("--surface-out"))) return false;
            o->surfaceOut = v;
        } else if (a == "--strict-timing") {
            o->strictTiming = true;
        } else if (a == "--trace") {
            o->trace = true;
        } else if (a == "--file") {
            if (!(v = next("--file"))) return false;
            o->file = v;
        } else if (a == "--bounding-boxes") {
            o->boxes = true;
        } else if (a == "--color-mode") {
            if (!(v = next("--color-mode"))) return false;
            const std::string m = v;
            const char* modes[] = {"rgb", "node", "lod", "white"};
            o->colorMode = -1;
            for (int k = 0; k < 4; k++)
                if (m == modes[k]) o->colorMode = k;
            if (o->colorMode < 0) {
                std::fprintf(stderr, "rb_harness: --color-mode takes rgb, node, lod or white\n");
                return false;
            }
        } else {
            std::fprintf(stderr, "rb_harness: unknown option %s\n", a.c_str());
            usage();
            return false;
        }
    }
    if (o->width <= 0 || o->height <= 0) {
        std::fprintf(stderr, "rb_harness: --size needs positive dimensions\n");
        return false;
    }
    return true;
}

// Orbit camera (src/shell/OrbitControls.h:68-93, glm::perspective at 60
// degrees, near/far = extent * 1e-4 / * 100): world = T(target) Rz(yaw)
// Rx(pitch) flip T(0, 0, radius); clip = P * world^-1, row-major.
struct Mat4 {
    double m[16];
    static Mat4 identity() {
        Mat4 r{};
        for (int i = 0; i < 4; i++) r.m[i * 5] = 1.0;
        return r;
    }
    Mat4 operator*(const Mat4& b) const {
        Mat4 r{};
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
                double s = 0.0;
                for (int k = 0; k < 4; k++) s += m[i * 4 + k] * b.m[k * 4 + j];
                r.m[i * 4 + j] = s;
            }
        return r;
    }
};

Mat4 translate(double x, double y, double z) {
    Mat4 r = Mat4::identity();
    r.m[3] = x;
    r.m[7] = y;
    r.m[11] = z;
    return r;
}

Mat4 rotateZ(double a) {
    Mat4 r = Mat4::identity();
    r.m[0] = std::cos(a);
    r.m[1] = -std::sin(a);
    r.m[4] = std::sin(a);
    r.m[5] = std::cos(a);
    return r;
}

Mat4 rotateX(double a) {
    Mat4 r = Mat4::identity();
    r.m[5] = std::cos(a);
    r.m[6] = -std::sin(a);
    r.m[9] = std::sin(a);
    r.m[10] = std::cos(a);
    return r;
}

rb_frame orbitFrame(const CloudMeta& meta, int width, int height, double yaw, double pitch, uint64_t counter) {
    const double sx = meta.boxSize[0], sy = meta.boxSize[1], sz = meta.boxSize[2];
    const double fovy = 60.0 * M_PI / 180.0;
    const double extent = std::sqrt(sx * sx + sy * sy + sz * sz);
    const double radius = (extent * 0.5) / std::tan(fovy * 0.5) * 1.1;
    const double ext = std::max(std::max(sx, sy), std::max(sz, 1.0));
    const double nearZ = ext * 1e-4, farZ = ext * 100.0;
    // view = world^-1 = T(0,0,-r) flip^T Rx(-pitch) Rz(-yaw) T(-target)
    Mat4 flipT = Mat4::identity();
    flipT.m[5] = 0.0;
    flipT.m[6] = 1.0;
    flipT.m[9] = -1.0;
    flipT.m[10] = 0.0;
    const Mat4 view = translate(0, 0, -radius) * flipT * rotateX(-pitch) * rotateZ(-yaw) *
                      translate(-sx * 0.5, -sy * 0.5, -sz * 0.5);
    Mat4 proj{};
    const double f = 1.0 / std::tan(fovy * 0.5);
    proj.m[0] = f / (double(width) / double(height));
    proj.m[5] = f;
    proj.m[10] = -(farZ + nearZ) / (farZ - nearZ);
    proj.m[11] = -2.0 * farZ * nearZ / (farZ - nearZ);
    proj.m[14] = -1.0;
    const Mat4 vp = proj * view;
    rb_frame fr;
    std::memset(&fr, 0, sizeof(fr));
    fr.width = float(width);
    fr.height = float(height);
    for (int i = 0; i < 16; i++) {
        fr.transform[i] = float(vp.m[i]);
        fr.transform_frozen[i] = float(vp.m[i]);
    }
    for (int a = 0; a < 3; a++) {
        fr.box_min[a] = 0.0f;
        fr.box_max[a] = meta.boxSize[a];
    }
    fr.lod_pixel_budget = 128.0f;
    fr.point_size = 1;
    fr.enable_edl = 0;
    fr.edl_strength = 0.4f;
    fr.frame_counter = counter;
    return fr;
}

uint64_t fnv1a(const std::vector<uint32_t>& words) {
    uint64_t h = 1469598103934665603ull;
    for (uint32_t w : words)
        for (int b = 0; b < 4; b++) {
            h ^= (w >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    return h;
}

bool writePpm(const std::string& path, const std::vector<uint32_t>& rgba, int w, int h) {
    FILE* out = std::fopen(path.c_str(), "wb");
    if (!out) return false;
    std::fprintf(out, "P6\n%d %d\n255\n", w, h);
    std::vector<unsigned char> row(size_t(w) * 3);
    for (int y = h - 1; y >= 0; --y) {  // bottom-up rows, as the GL readback
        for (int x = 0; x < w; ++x) {
            const uint32_t c = rgba[size_t(y) * w + x];
            row[x * 3 + 0] = c & 0xff;
            row[x * 3 + 1] = (c >> 8) & 0xff;
            row[x * 3 + 2] = (c >> 16) & 0xff;
        }
        std::fwrite(row.data(), 1, row.size(), out);
    }
    std::fclose(out);
    return true;
}

void printReport(const PipelineRegistry& reg, const GpuProfiler& prof, const CloudMeta& meta,
                 const DeviceBudget& budget) {
    std::printf("  device budget       %.3f GB (%.3f GB free of %.3f GB at startup)\n", budget.bytes / 1e9,
                budget.vramFreeAtStartup / 1e9, budget.vramTotal / 1e9);
    const ILodPipeline* p = reg.active();
    if (!p) {
        std::printf("rb_harness: no active pipeline\n");
        return;
    }
    const PipelineStats& s = p->stats();
    std::printf("rb_harness: pipeline=%s\n", reg.activeId().c_str());
    std::printf("  points              %llu\n", (unsigned long long)s.numPoints);
    std::printf("  voxels              %llu\n", (unsigned long long)s.numVoxels);
    std::printf("  nodes               %u (inner %u, leaves %u)\n", s.numNodes, s.numInner, s.numLeaves);
    std::printf("  octree depth        %u (root = 0)\n", s.maxDepth);
    std::printf("  visible samples     %llu\n", (unsigned long long)(s.numVisiblePoints + s.numVisibleVoxels));
    std::printf("  visible nodes       %u (drawn this frame)\n", s.numVisibleNodes);
    std::printf("  max points/node     %u\n", s.maxPointsPerNode);
    for (const std::string& line : p->diagnostics()) std::printf("  %s\n", line.c_str());
    const TimingScopes scopes = p->timingScopes();
    const BuildTotals bt = buildTotals(prof, scopes);
    if (bt.measured)
        std::printf("  build device ms     %.2f (%llu launches)\n", bt.ms, (unsigned long long)bt.launches);
    else
        std::printf("  build device ms     not measured\n");
    if (const ScopeStats* r = scopes.render.empty() ? nullptr : prof.find(scopes.render))
        std::printf("  render device ms    %.2f  (median %.2f, p95 %.2f, n=%llu)\n", r->last(), r->median(),
                    r->percentile(0.95), (unsigned long long)r->count());
    if (const PipelineInfo* info = reg.find(reg.activeId())) {
        if (meta.numPoints > 0 && info->minBytesPerPointEstimate > 0.0) {
            const double predicted = reg.predictedCompletion(*info, meta, budget);
            const double observed = double(s.numPointsIngested) / double(meta.numPoints);
            std::printf("  ingested            %.1f%% of the cloud (predicted %.1f%% at %.0f B/pt)\n",
                        observed * 100.0, predicted * 100.0, info->minBytesPerPointEstimate);
        }
    }
    std::printf("  scopes\n");
    for (const std::string& name : prof.scopeNames()) {
        const ScopeStats* st = prof.find(name);
        if (!st) continue;
        std::printf("    %-20s n=%-6llu last %7.3f  med %7.3f  p95 %7.3f  min %7.3f  max %7.3f  total %9.2f\n",
                    name.c_str(), (unsigned long long)st->count(), st->last(), st->median(), st->percentile(0.95),
                    st->min(), st->max(), st->total());
    }
    if (s.allocOverflow) std::printf("  WARNING allocator overflow\n");
    if (s.nodeCapacityReached) std::printf("  WARNING node pool exhausted\n");
    if (s.memCapacityReached) std::printf("  WARNING memory budget reached\n");
}

}  // namespace

int main(int argc, char** argv) {
    Options opt;
    if (!parse(argc, argv, &opt)) return 2;

    int nDev = 0;
    if (cudaGetDeviceCount(&nDev) != cudaSuccess || nDev <= opt.device) {
        std::fprintf(stderr, "rb_harness: no CUDA device %d\n", opt.device);
        return 1;
    }
    cudaSetDevice(opt.device);
    size_t freeB = 0, totalB = 0;
    cudaMemGetInfo(&freeB, &totalB);
    DeviceBudget budget;
    budget.vramTotal = totalB;
    budget.vramFreeAtStartup = freeB;
    budget.bytes = opt.budgetGB > 0.0 ? uint64_t(opt.budgetGB * 1e9) : uint64_t(freeB * 0.85);

    std::string err;
    const auto tGen = std::chrono::steady_clock::now();
    std::unique_ptr<PointSource> source =
        opt.file.empty() ? makeSyntheticSource(opt.config, opt.synthetic, opt.seed, opt.batch, opt.device, &err)
                         : makeSimlodSource(opt.file, opt.batch, opt.device, &err);
    if (!source) {
        std::fprintf(stderr, "rb_harness: %s\n", err.c_str());
        return 1;
    }
    const double genS = std::chrono::duration<double>(std::chrono::steady_clock::now() - tGen).count();
    const CloudMeta meta = source->meta();

    PipelineRegistry reg;
    const int dev = opt.device;
    reg.add([dev] { return makeRemolodPipeline(dev); });
    reg.add([dev] { return makeSimlodPipeline(dev); });
    reg.add([dev] { return makeFlatPipeline(dev); });

    bool failed = false;
    std::string refused;
    if (const PipelineInfo* info = reg.find(opt.pipeline)) {
        const std::string warn = reg.completionWarning(*info, meta, budget);
        if (!warn.empty()) std::printf("rb_harness: %s: %s\n", info->displayName.c_str(), warn.c_str());
    }
    if (!reg.switchTo(opt.pipeline, source.get(), meta, budget, &err)) {
        refused = err;
        std::fprintf(stderr, "rb_harness: %s\n", err.c_str());
        failed = true;
    }

    void* surface = nullptr;
    const size_t pixels = size_t(opt.width) * size_t(opt.height);
    if (cudaMalloc(&surface, pixels * 4) != cudaSuccess) {
        std::fprintf(stderr, "rb_harness: cannot allocate the %dx%d surface\n", opt.width, opt.height);
        return 1;
    }
    cudaMemset(surface, 0, pixels * 4);

    rb_frame fixedUniforms{};
    bool haveFixed = false;
    if (!opt.frameFile.empty()) {
        FILE* f = std::fopen(opt.frameFile.c_str(), "rb");
        if (!f || std::fread(&fixedUniforms, sizeof(fixedUniforms), 1, f) != 1) {
            std::fprintf(stderr, "rb_harness: cannot read %zu bytes of uniforms from %s\n", sizeof(rb_frame),
                         opt.frameFile.c_str());
            if (f) std::fclose(f);
            return 2;
        }
        std::fclose(f);
        haveFixed = true;
    }

    GpuProfiler prof;
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, opt.device);
    long frame = 0;
    long completeAt = -1;
    bool more = true;
    const auto t0 = std::chrono::steady_clock::now();
    while (!failed && frame < opt.maxFrames) {
        if (!opt.switchTo.empty() && frame == opt.switchAfter) {
            if (!reg.switchTo(opt.switchTo, source.get(), meta, budget, &err)) {
                std::fprintf(stderr, "rb_harness: switch refused: %s\n", err.c_str());
                refused = err;
                failed = true;
                break;
            }
            more = true;
            completeAt = -1;
        }
        ILodPipeline* p = reg.active();
        FrameContext fc;
        fc.uniforms = haveFixed ? fixedUniforms
                                : orbitFrame(meta, opt.width, opt.height, 0.35 + 0.02 * frame, -0.6, uint64_t(frame));
        fc.uniforms.frame_counter = uint64_t(frame);
        if (opt.boxes) fc.uniforms.show_bounding_box = 1;
        if (opt.colorMode) fc.uniforms.color_mode = opt.colorMode;
        fc.targets.surface = reinterpret_cast<uint64_t>(surface);
        fc.targets.width = opt.width;
        fc.targets.height = opt.height;
        fc.numSMs = prop.multiProcessorCount;
        fc.strictTiming = opt.strictTiming;
        fc.profiler = &prof;

        p->render(fc);
        source->pump();
        const bool stillMore = p->build(*source, fc);
        if (opt.trace) {
            const PipelineStats& s = p->stats();
            std::printf("{\"frame\": %ld, \"pipeline\": \"%s\", \"pointsIngested\": %llu, \"nodes\": %u, "
                        "\"visibleSamples\": %llu, \"more\": %s}\n",
                        frame, reg.activeId().c_str(), (unsigned long long)s.numPointsIngested, s.numNodes,
                        (unsigned long long)(s.numVisiblePoints + s.numVisibleVoxels), stillMore ? "true" : "false");
        }
        ++frame;
        if (opt.dumpAfter >= 0) {
            if (frame > opt.dumpAfter) break;
            continue;
        }
        // No dump frame given: stop one frame after the build is done (or can do no more).
        if (more && (!stillMore || p->stats().memCapacityReached)) {
            more = false;
            completeAt = frame;
        } else if (!more && frame > completeAt) {
            break;
        }
    }
    cudaDeviceSynchronize();
    const double wallS = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    std::vector<uint32_t> rgba(pixels);
    cudaMemcpy(rgba.data(), surface, pixels * 4, cudaMemcpyDeviceToHost);
    if (!opt.dumpFrame.empty()) {
        if (!writePpm(opt.dumpFrame, rgba, opt.width, opt.height)) {
            std::fprintf(stderr, "rb_harness: cannot write %s\n", opt.dumpFrame.c_str());
            failed = true;
        } else {
            std::printf("rb_harness: wrote %s (%dx%d)\n", opt.dumpFrame.c_str(), opt.width, opt.height);
        }
        printReport(reg, prof, meta, budget);
    }
    if (!opt.surfaceOut.empty()) {
        FILE* f = std::fopen(opt.surfaceOut.c_str(), "wb");
        if (!f || std::fwrite(rgba.data(), 4, pixels, f) != pixels) failed = true;
        if (f) std::fclose(f);
    }

    PipelineStats s;
    TimingScopes scopes;
    if (reg.active()) {
        s = reg.active()->stats();
        scopes = reg.active()->timingScopes();
    }
    const BuildTotals bt = buildTotals(prof, scopes);
    const ScopeStats* rs = scopes.render.empty() ? nullptr : prof.find(scopes.render);
    double predicted = 0.0;
    if (const PipelineInfo* info = reg.find(reg.activeId().empty() ? opt.pipeline : reg.activeId()))
        predicted = reg.predictedCompletion(*info, meta, budget);
    std::string refusedJson;
    for (char c : refused) {
        if (c == '"' || c == '\\') refusedJson += '\\';
        refusedJson += c;
    }
    std::printf(
        "{\"pipeline\": \"%s\", \"ok\": %s, \"frames\": %ld, \"cloud_points\": %llu, \"points\": %llu, "
        "\"voxels\": %llu, \"points_ingested\": %llu, \"nodes\": %u, \"inner\": %u, \"leaves\": %u, "
        "\"max_depth\": %u, \"max_points_per_node\": %u, \"visible_nodes\": %u, \"visible_samples\": %llu, "
        "\"mem_capacity_reached\": %s, \"node_capacity_reached\": %s, \"overran_consumer\": %s, "
        "\"predicted_completion\": %.4f, \"build_ms\": %.3f, \"build_launches\": %llu, \"render_ms_median\": %.4f, "
        "\"surface_fnv1a\": \"%016llx\", \"generate_s\": %.2f, \"wall_s\": %.3f, \"budget_bytes\": %llu, "
        "\"refused\": \"%s\"}\n",
        reg.activeId().c_str(), failed ? "false" : "true", frame, (unsigned long long)meta.numPoints,
        (unsigned long long)s.numPoints, (unsigned long long)s.numVoxels, (unsigned long long)s.numPointsIngested,
        s.numNodes, s.numInner, s.numLeaves, s.maxDepth, s.maxPointsPerNode, s.numVisibleNodes,
        (unsigned long long)(s.numVisiblePoints + s.numVisibleVoxels), s.memCapacityReached ? "true" : "false",
        s.nodeCapacityReached ? "true" : "false", source->overranConsumer() ? "true" : "false", predicted, bt.ms,
        (unsigned long long)bt.launches, rs ? rs->median() : 0.0, (unsigned long long)fnv1a(rgba), genS, wallS,
        (unsigned long long)budget.bytes, refusedJson.c_str());
    std::fflush(stdout);

    reg.shutdown();
    source.reset();
    cudaFree(surface);
    return failed ? 1 : 0;
}
