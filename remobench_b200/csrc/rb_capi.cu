// The C ABI (include/rb_capi.h): context lifetime, buffer sizing, and the host
// side of each stage -- the launch sequencing RemolodPipeline performs in the
// reference (src/pipelines/RemolodPipeline.cpp:105-601), on one CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rb_capi.h"
#include "rb_analysis.h"
#include "rb_ctx_access.h"
#include "rb_kernels.h"
#include "rb_mlp.h"
#include "rb_refine.h"
#include "rb_state.h"

using rb::Counters;
using rb::Dev;
using rb::kNone;

// Per-kernel launch counts (always) and CUDA-event durations (when profiling).
enum KernelId : int {
    K_BUILD_BEGIN, K_BATCH_BEGIN, K_COUNT_FIRST, K_SPLIT, K_SPILL_COPY, K_RECOUNT, K_VOX_SAMPLE,
    K_VOX_COMMIT, K_ALLOC_POINTS, K_INSERT, K_VOX_STORE, K_BATCH_END, K_ACCUMULATE, K_ACCUM_VERIFY,
    K_SWEEP, K_RESET_ROOT, K_FB_CLEAR, K_NODE_FLAGS, K_FRONTIER, K_RASTER, K_RASTER_FLAT, K_EDL,
    K_RESOLVE, K_ROLL, K_ANALYZE, K_QUEUE, K_REFINE, K_SCORE, K_MLP_PREDICT, K_MLP_GRAD, K_MLP_ADAM,
    K_EXPAND_COND, K_ZERO_GRIDS, K_EXPAND_PASS, K_DEEP_BOOK, K_DEEP_BIN, K_DEEP_SPLIT, K_DEEP_MOVE,
    K_EXPAND_REST, K_WIREFRAME, K_REFINE_COLORS, K_ALLOC_VOXELS, K_FINISH_LEAVES, K_VOX_LIFT, K_VOX_SAMPLE_LEVELS, K_DEEPEN, K_COLLAPSE, K_NUM
};
static const char* const kKernelNames[K_NUM] = {
    "k_build_begin", "k_batch_begin", "k_count_first", "k_split", "k_spill_copy", "k_recount",
    "k_vox_sample", "k_vox_commit", "k_alloc_points", "k_insert", "k_vox_store", "k_batch_end",
    "k_accumulate", "k_accum_verify", "k_sweep", "k_reset_root", "k_fb_clear", "k_node_flags",
    "k_frontier", "k_raster", "k_raster_flat", "k_edl", "k_resolve", "k_roll_level", "k_analyze",
    "k_queue", "k_refine", "k_score", "k_mlp_predict", "k_mlp_grad", "k_mlp_adam",
    "k_expand_cond", "k_zero_grids",
    // not a kernel: per-iteration expand passes run inside k_expand_rest
    "expand_pass", "k_deep_book", "k_deep_bin", "k_deep_split", "k_deep_move", "k_expand_rest",
    "k_wireframe", "k_refine_colors", "k_alloc_voxels", "k_finish_leaves", "k_vox_lift", "k_vox_sample_levels", "k_deepen", "k_collapse"};

struct Profiler {
    bool on = false;
    uint64_t launches[K_NUM] = {};
    double ms[K_NUM] = {};
    uint64_t timed[K_NUM] = {};
    uint64_t units[K_NUM] = {};  // points (or pixels, nodes) handed to the kernel
    std::vector<cudaEvent_t> pool;
    struct Pending {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    cudaEvent_t take() {
        if (pool.empty()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    void resolve() {
        for (auto& p : pending) {
            float t = 0.0f;
            if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
                ms[p.id] += t;
                timed[p.id] += 1;
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    ~Profiler() {
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

struct rb_ctx {
    Profiler prof;
    rb_config cfg{};
    std::string err;
    int device = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evStart = nullptr, evStop = nullptr;
    bool allocated = false;
    Dev d{};
    std::vector<void*> allocs;
    uint64_t bytes = 0;
    Counters* hostCtr = nullptr;  // pinned mirror
    rb::SweepStats* hostSweep = nullptr;
    rb::AccumGlobals* hostAccum = nullptr;
    rb::RenderScratch* hostRs = nullptr;
    // render scratch
    uint8_t* vis = nullptr;
    uint8_t* large = nullptr;
    uint32_t* items = nullptr;
    rb::RenderScratch* rs = nullptr;
    // analysis
    rb::RollSum* roll = nullptr;
    rb::NodeAnalysis* analysis = nullptr;
    unsigned long long* akeys = nullptr;
    uint32_t* ahist = nullptr;
    unsigned long long* acand = nullptr;
    uint32_t* aqueue = nullptr;
    rb::AnalysisCounters* actr = nullptr;
    rb::AnalysisCounters* hostActr = nullptr;
    bool analyzed = false;
    float* features = nullptr;
    float* predictions = nullptr;
    rb::MlpState mlp{};
    rb::RefineScratch refine{};
    rb::RefineCounters* hostRefine = nullptr;  // pinned
    bool mlpReady = false;
    uint32_t adamT = 0;
    // device-driven batches: one graph per batch, the ring descriptor it reads
    cudaGraphExec_t batchGraph = nullptr;
    bool graphTried = false;
    rb::RingDesc* hostRing = nullptr;  // pinned staging for d.ring
    // host-ingest ring
    rb::Point* ingestRing = nullptr;
    uint32_t ingestSlots = 0;
    cudaEvent_t slotFree[4] = {};
    cudaEvent_t slotFull[4] = {};
    // cloud
    uint64_t numPoints = 0;
    uint32_t batchesConsumed = 0;
    bool accumAll = true;         // next accumulate must visit every node
    uint32_t lastVisibleNodes = 0;
    uint64_t lastVisibleSamples = 0;
};

namespace {

rb_status fail(rb_ctx* c, rb_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

#define RB_CUDA(c, call)                                                                      \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail((c), RB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
rb_status devAlloc(rb_ctx* c, T** p, uint64_t count, const char* what) {
    void* q = nullptr;
    const uint64_t bytes = std::max<uint64_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, RB_ERR_OUT_OF_MEMORY,
                    std::string("cudaMalloc failed for ") + what + " (" + std::to_string(bytes >> 20) + " MB)");
    }
    c->allocs.push_back(q);
    c->bytes += bytes;
    *p = static_cast<T*>(q);
    return RB_OK;
}

constexpr uint32_t kQueueSortCap = 16384;

uint32_t nextPow2(uint64_t v) {
    uint64_t m = 1;
    while (m < v) m <<= 1;
    return (uint32_t)std::min<uint64_t>(m, 1ull << 31);
}

int pointGrid(const rb_ctx* c, uint64_t n) {
    const uint64_t blocks = (n + 255) / 256;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)c->numSMs * 8));
}

// Launches `stmt` as kernel `id`, bracketed by events when profiling.
#define LAUNCH(c, id, nunits, stmt)                                       \
    do {                                                                  \
        (c)->prof.launches[id] += 1;                                      \
        (c)->prof.units[id] += (uint64_t)(nunits);                        \
        if ((c)->prof.on) {                                               \
            cudaEvent_t a_ = (c)->prof.take(), b_ = (c)->prof.take();     \
            cudaEventRecord(a_, (c)->stream);                             \
            stmt;                                                         \
            cudaEventRecord(b_, (c)->stream);                             \
            (c)->prof.pending.push_back({(id), a_, b_});                  \
        } else {                                                          \
            stmt;                                                         \
        }                                                                 \
    } while (0)

rb_status readCounters(rb_ctx* c) {
    RB_CUDA(c, cudaMemcpyAsync(c->hostCtr, c->d.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, c->stream));
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    return RB_OK;
}

__global__ void k_build_begin(Counters* c) {
    c->buildStamp += 1;
    c->numDirty = 0;
    c->callBatches = 0;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    c->buildStartNs = t;
}

// One batch through addBatch's phases (remolod_octree.cu:940-1060). Returns
// RB_OK with *stopped set when the memory check refused the batch.
rb_status runBatchAfterCount(rb_ctx* c, const rb::Point* pts, uint32_t n, uint64_t work, bool* stopped, bool deepen);

rb_status runBatch(rb_ctx* c, const rb::Point* pts, uint32_t n, uint32_t batchIndex, bool* stopped) {
    const Dev& d = c->d;
    cudaStream_t s = c->stream;
    *stopped = false;
    LAUNCH(c, K_BATCH_BEGIN, 1, rb::launchBatchBegin(d, s));
    LAUNCH(c, K_COUNT_FIRST, n, rb::launchCountFirst(d, pts, n, pointGrid(c, n), s));
    return runBatchAfterCount(c, pts, n, n, stopped, false);
}

// The phases after the first count: the expand round, the per-iteration
// passes, voxel sampling and insertion; a deepening pass (no batch points, its
// spilling nodes taken from the Analysis queue) ends without counting a batch.
// `work` sizes the grids of the point kernels.
rb_status runBatchAfterCount(rb_ctx* c, const rb::Point* pts, uint32_t n, uint64_t work, bool* stopped,
                             bool deepen) {
    const Dev& d = c->d;
    cudaStream_t s = c->stream;
    *stopped = false;
    const int fixedGrid = c->numSMs * 4;
    // the same kernels as the batch graph, with k_expand_rest's loop on the
    // host; split and recount take their stamps from the device counters
    LAUNCH(c, K_DEEP_BOOK, 1, rb::launchDeepBook(d, s));
    LAUNCH(c, K_DEEP_BIN, n, rb::launchDeepBin(d, pts, n, pointGrid(c, work), s));
    LAUNCH(c, K_DEEP_SPLIT, 1, rb::launchDeepSplit(d, s));
    LAUNCH(c, K_DEEP_MOVE, n, rb::launchDeepMove(d, pts, n, pointGrid(c, work), s));
    for (uint32_t pass = 0; pass < 64u; pass++) {
        rb_status st = readCounters(c);
        if (st != RB_OK) return st;
        if (c->hostCtr->batchStop) {
            *stopped = true;
            return RB_OK;
        }
        // k_expand_rest's loop: a first pass if the round left spilling
        // nodes, then more while the loop test says so
        if (pass == 0 ? c->hostCtr->numSpill == 0 : c->hostCtr->loopMore == 0) break;
        // the per-iteration passes k_expand_rest runs on the device
        c->prof.launches[K_EXPAND_PASS] += 1;
        LAUNCH(c, K_SPLIT, c->hostCtr->numSpill, rb::launchSplit(d, 0u, s));
        LAUNCH(c, K_SPILL_COPY, 0, rb::launchSpillCopy(d, fixedGrid, s));
        LAUNCH(c, K_RECOUNT, n, rb::launchRecount(d, pts, n, 0u, pointGrid(c, work), s));
        LAUNCH(c, K_EXPAND_COND, 1, rb::launchExpandCond(d, s));
    }
    LAUNCH(c, K_ZERO_GRIDS, 0, rb::launchZeroGrids(d, fixedGrid, s));
    LAUNCH(c, K_FINISH_LEAVES, n, rb::launchFinishLeaves(d, pts, n, pointGrid(c, work), s));
    LAUNCH(c, K_VOX_SAMPLE, n, rb::launchVoxSample(d, pts, n, pointGrid(c, work), s));
    LAUNCH(c, K_VOX_SAMPLE_LEVELS, n, rb::launchVoxSampleLevels(d, pts, n, pointGrid(c, work), s));
    LAUNCH(c, K_VOX_LIFT, 0, rb::launchVoxLift(d, pointGrid(c, work), s));
    // four blocks per SM: fewer blocks, fewer reservations on a node's voxel counter
    LAUNCH(c, K_VOX_COMMIT, 0, rb::launchVoxCommit(d, fixedGrid, s));
    LAUNCH(c, K_ALLOC_VOXELS, 0, rb::launchAllocVoxels(d, fixedGrid, s));
    LAUNCH(c, K_VOX_STORE, 0, rb::launchVoxStore(d, fixedGrid, s));
    LAUNCH(c, K_ALLOC_POINTS, 0, rb::launchAllocPoints(d, fixedGrid, s));
    LAUNCH(c, K_INSERT, n, rb::launchInsert(d, pts, n, pointGrid(c, work), s));
    if (deepen) LAUNCH(c, K_DEEPEN, 1, rb::launchDeepenEnd(d, s));
    else LAUNCH(c, K_BATCH_END, 1, rb::launchBatchEnd(d, n, s));
    RB_CUDA(c, cudaGetLastError());
    return RB_OK;
}

// The device-driven path: on unless profiling (per-kernel events need
// separate launches) or use_graphs is 0; captured at the first build.
bool graphPath(rb_ctx* c) {
    if (!c->cfg.use_graphs || c->prof.on) return false;
    if (!c->graphTried) {
        c->graphTried = true;
        const int pointGrid = c->numSMs * 8, fixedGrid = c->numSMs * 4;
        int restGrid = 0;
        if (rb::expandRestGrid(c->numSMs, &restGrid) != cudaSuccess ||
            rb::captureBatchGraph(c->d, pointGrid, fixedGrid, restGrid, &c->batchGraph) != cudaSuccess) {
            cudaGetLastError();
            c->batchGraph = nullptr;
        }
    }
    return c->batchGraph != nullptr;
}

// Launches of graph batches, for the per-kernel counts: sixteen kernels per
// batch (k_expand_rest zeroes the split grids and finishes the leaves); the
// per-iteration passes k_expand_rest ran (one loop test each) are counted as
// expand_pass, not as launches.
void countGraphLaunches(rb_ctx* c, uint64_t batches, uint32_t condBefore, uint64_t points) {
    const uint32_t passes = c->hostCtr->condRuns - condBefore;
    for (int k : {K_BATCH_BEGIN, K_COUNT_FIRST, K_DEEP_BOOK, K_DEEP_BIN, K_DEEP_SPLIT, K_DEEP_MOVE, K_EXPAND_REST,
                  K_VOX_SAMPLE, K_VOX_SAMPLE_LEVELS, K_VOX_LIFT, K_VOX_COMMIT, K_ALLOC_VOXELS, K_VOX_STORE, K_ALLOC_POINTS, K_INSERT,
                  K_BATCH_END})
        c->prof.launches[k] += batches;
    c->prof.launches[K_EXPAND_PASS] += passes;
    for (int k : {K_COUNT_FIRST, K_DEEP_BIN, K_DEEP_MOVE, K_VOX_SAMPLE, K_INSERT}) c->prof.units[k] += points;
}

// A grid barrier of k_expand_rest gave up: the batch is not trustworthy.
rb_status checkSync(rb_ctx* c) {
    if (c->hostCtr->overflowFlags & rb::kOvfSync)
        return fail(c, RB_ERR_CUDA, "a device grid barrier timed out in the expand passes (RB_OVF_SYNC)");
    return RB_OK;
}

rb_status uploadRing(rb_ctx* c) {
    RB_CUDA(c, cudaMemcpyAsync(c->d.ring, c->hostRing, sizeof(rb::RingDesc), cudaMemcpyHostToDevice, c->stream));
    return RB_OK;
}

rb_status accumulate(rb_ctx* c, uint32_t batchIndex) {
    const Dev& d = c->d;
    // sumLeafCounts .. innerWithSums restart per launch (RemolodPipeline.cpp:251-256)
    RB_CUDA(c, cudaMemsetAsync(reinterpret_cast<uint8_t*>(d.accumGlobals) + 16, 0, 20, c->stream));
    LAUNCH(c, K_ACCUMULATE, 0, rb::launchAccumulate(d, batchIndex, c->accumAll ? 0 : 1, c->numSMs * 8, c->stream));
    LAUNCH(c, K_ACCUM_VERIFY, 0, rb::launchAccumVerify(d, c->numSMs * 2, c->stream));
    // the dirty list restarts: it names the nodes touched since this fold
    LAUNCH(c, K_BUILD_BEGIN, 1, (k_build_begin<<<1, 1, 0, c->stream>>>(c->d.ctr)));
    RB_CUDA(c, cudaGetLastError());
    c->accumAll = false;
    return RB_OK;
}

}  // namespace

extern "C" {

uint32_t rb_abi_version(void) { return RB_ABI_VERSION; }

const char* rb_status_string(rb_status s) {
    switch (s) {
        case RB_OK: return "ok";
        case RB_ERR_INVALID_ARG: return "invalid argument";
        case RB_ERR_CUDA: return "CUDA error";
        case RB_ERR_OUT_OF_MEMORY: return "out of device memory";
        case RB_ERR_STATE: return "call out of order";
        case RB_ERR_RING: return "ring depth mismatch";
        case RB_ERR_CAPACITY: return "beyond a configured capacity";
        case RB_ERR_NO_DEVICE: return "no CUDA device";
        case RB_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

void rb_config_defaults(rb_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->struct_size = sizeof(rb_config);
    cfg->pipeline = RB_PIPELINE_REMOLOD;
    cfg->device = 0;
    cfg->max_nodes = 200000;
    cfg->max_points_per_node = 50000;
    cfg->points_per_chunk = 1000;
    cfg->max_expand_iters = 20;
    cfg->ring_slots = 50;
    cfg->slot_capacity = 1000000;
    cfg->max_batches_per_build = 20;
    cfg->time_budget_ms = 10.0f;
    cfg->voxel_mode = RB_VOXEL_LOWEST_INDEX;
    cfg->accumulate = 1;
    cfg->spilled_capacity = 10000000;
    cfg->spilling_nodes_capacity = 100000;
    cfg->drawlist_capacity = 131072;
    cfg->safety_margin = 200000000ull;
    cfg->use_graphs = 1;
}

rb_status rb_create(const rb_config* cfg, rb_ctx** out) {
    if (!cfg || !out || cfg->struct_size != sizeof(rb_config)) return RB_ERR_INVALID_ARG;
    if (cfg->pipeline > RB_PIPELINE_FLAT || cfg->max_nodes < 9 || cfg->points_per_chunk == 0 ||
        cfg->slot_capacity == 0 || cfg->ring_slots == 0 || cfg->max_expand_iters == 0 ||
        cfg->max_expand_iters > 31 || cfg->voxel_mode > RB_VOXEL_FIRST_COME ||
        cfg->max_nodes > (1u << 21) || cfg->backlog_capacity > (1u << 28))
        return RB_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return RB_ERR_NO_DEVICE;
    }
    if (cfg->device < 0 || cfg->device >= ndev) return RB_ERR_INVALID_ARG;
    rb_ctx* c = new rb_ctx();
    c->cfg = *cfg;
    c->device = cfg->device;
    *out = c;
    return RB_OK;
}

void rb_release(rb_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void* p : c->allocs) cudaFree(p);
    c->allocs.clear();
    c->bytes = 0;
    if (c->hostCtr) cudaFreeHost(c->hostCtr);
    if (c->hostSweep) cudaFreeHost(c->hostSweep);
    if (c->hostAccum) cudaFreeHost(c->hostAccum);
    if (c->hostRs) cudaFreeHost(c->hostRs);
    if (c->hostActr) cudaFreeHost(c->hostActr);
    c->hostActr = nullptr;
    if (c->hostRefine) cudaFreeHost(c->hostRefine);
    c->hostRefine = nullptr;
    c->refine = rb::RefineScratch{};
    if (c->batchGraph) cudaGraphExecDestroy(c->batchGraph);
    c->batchGraph = nullptr;
    c->graphTried = false;
    if (c->hostRing) cudaFreeHost(c->hostRing);
    c->hostRing = nullptr;
    c->analyzed = false;
    c->mlp = rb::MlpState{};
    c->mlpReady = false;
    c->adamT = 0;
    c->hostCtr = nullptr;
    c->hostSweep = nullptr;
    c->hostAccum = nullptr;
    c->hostRs = nullptr;
    for (int i = 0; i < 4; i++) {
        if (c->slotFree[i]) cudaEventDestroy(c->slotFree[i]);
        if (c->slotFull[i]) cudaEventDestroy(c->slotFull[i]);
        c->slotFree[i] = c->slotFull[i] = nullptr;
    }
    c->d = Dev{};
    c->vis = c->large = nullptr;
    c->items = nullptr;
    c->rs = nullptr;
    c->ingestRing = nullptr;
    c->allocated = false;
}

void rb_destroy(rb_ctx* c) {
    if (!c) return;
    rb_release(c);
    if (c->evStart) cudaEventDestroy(c->evStart);
    if (c->evStop) cudaEventDestroy(c->evStop);
    if (c->copyStream) cudaStreamDestroy(c->copyStream);
    if (c->ownStream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* rb_last_error(const rb_ctx* c) { return c ? c->err.c_str() : "null context"; }

rb_status rb_set_stream(rb_ctx* c, void* stream) {
    if (!c) return RB_ERR_INVALID_ARG;
    if (c->ownStream && c->stream) cudaStreamDestroy(c->stream);
    c->stream = static_cast<cudaStream_t>(stream);
    c->ownStream = false;
    return RB_OK;
}

rb_status rb_allocate(rb_ctx* c, const rb_cloud_meta* meta, uint64_t budget) {
    if (!c || !meta) return RB_ERR_INVALID_ARG;
    if (meta->num_points == 0) return fail(c, RB_ERR_INVALID_ARG, "cloud is empty");
    rb_release(c);
    RB_CUDA(c, cudaSetDevice(c->device));
    cudaDeviceProp prop{};
    RB_CUDA(c, cudaGetDeviceProperties(&prop, c->device));
    c->numSMs = prop.multiProcessorCount;
    if (!c->stream) {
        RB_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->ownStream = true;
    }
    if (!c->copyStream) RB_CUDA(c, cudaStreamCreateWithFlags(&c->copyStream, cudaStreamNonBlocking));
    if (!c->evStart) RB_CUDA(c, cudaEventCreate(&c->evStart));
    if (!c->evStop) RB_CUDA(c, cudaEventCreate(&c->evStop));

    const rb_config& cfg = c->cfg;
    c->numPoints = meta->num_points;
    Dev& d = c->d;
    d.maxNodes = cfg.max_nodes;
    d.maxPointsPerNode = cfg.max_points_per_node;
    d.ppc = cfg.points_per_chunk;
    d.maxExpandIters = cfg.max_expand_iters;
    d.voxelMode = cfg.voxel_mode;
    d.safetyMargin = cfg.safety_margin;
    for (int a = 0; a < 3; a++) d.boxMin[a] = meta->box_min[a];
    // remolod_octree.cu:1148-1149
    const float sx = meta->box_max[0] - meta->box_min[0], sy = meta->box_max[1] - meta->box_min[1],
                sz = meta->box_max[2] - meta->box_min[2];
    d.octreeSize = std::max(std::max(sx, sy), sz);
    if (!(d.octreeSize > 0.0f)) return fail(c, RB_ERR_INVALID_ARG, "empty bounding box");

    if (cfg.pipeline == RB_PIPELINE_FLAT) {
        // flat keeps no tree: render scratch only
        if (devAlloc(c, &c->rs, 1, "render scratch") != RB_OK) return RB_ERR_OUT_OF_MEMORY;
        RB_CUDA(c, cudaMallocHost(&c->hostRs, sizeof(rb::RenderScratch)));
        RB_CUDA(c, cudaMallocHost(&c->hostCtr, sizeof(Counters)));
        c->allocated = true;
        return RB_OK;
    }

    // Store sizing (RemolodPipeline.cpp:118-157): 48 B/pt appetite, 512 MB
    // floor, clamped to what the budget leaves after the ring and fixed parts.
    size_t freeB = 0, totalB = 0;
    RB_CUDA(c, cudaMemGetInfo(&freeB, &totalB));
    if (budget == 0) budget = (uint64_t)(freeB * 0.85);
    const uint64_t batches = (meta->num_points + cfg.slot_capacity - 1) / cfg.slot_capacity;
    const uint64_t ringBytes = std::min<uint64_t>(cfg.ring_slots, batches) * cfg.slot_capacity * 16ull;
    const uint64_t available = budget > ringBytes ? budget - ringBytes : 0;
    const uint64_t fixedBytes = (uint64_t)cfg.max_nodes * (152 + 112) + (512ull << 20);
    const uint64_t minPersistent = 512ull << 20;
    if (available < fixedBytes + minPersistent)
        return fail(c, RB_ERR_OUT_OF_MEMORY,
                    "not enough device memory: needs at least " +
                        std::to_string((fixedBytes + minPersistent) >> 20) + " MB, " +
                        std::to_string(available >> 20) + " MB available");
    uint64_t want = std::max<uint64_t>((uint64_t)(48.0 * (double)meta->num_points), minPersistent);
    d.persistentCapacity = std::min<uint64_t>(want, available - fixedBytes);
    if (cfg.store_capacity) {
        // a caller-sized store (the reference launcher's persistent size)
        if (cfg.store_capacity > available - fixedBytes)
            return fail(c, RB_ERR_OUT_OF_MEMORY,
                        "store_capacity " + std::to_string(cfg.store_capacity >> 20) + " MB exceeds the " +
                            std::to_string((available - fixedBytes) >> 20) + " MB the budget leaves");
        d.persistentCapacity = cfg.store_capacity;
    }

    // The arena: the reference store's worst case plus the wider point chunks
    // (indices kept beside the points): at most 1.25 x its capacity.
    const uint64_t ptChunkBytes = ((uint64_t)d.ppc * 20ull + 15ull) & ~15ull;
    d.ptChunkUnits = (uint32_t)(ptChunkBytes / 16ull);
    d.vxChunkUnits = d.ppc;
    uint64_t arenaBytes = d.persistentCapacity + d.persistentCapacity / 4 + (64ull << 20);
    arenaBytes = std::min<uint64_t>(arenaBytes, (uint64_t)UINT32_MAX * 16ull);
    d.arenaUnits = (uint32_t)(arenaBytes / 16ull);
    const uint64_t maxChunks = arenaBytes / (uint64_t)(d.vxChunkUnits * 16ull) + 1;
    d.maxPtChunks = (uint32_t)std::min<uint64_t>(maxChunks, UINT32_MAX);
    d.tablePoolCap = (uint32_t)std::min<uint64_t>(128ull * cfg.max_nodes + 4ull * maxChunks, 1ull << 31);
    d.spillCap = cfg.spilled_capacity;
    d.spillingCap = cfg.spilling_nodes_capacity;
    // the cell table keeps its load at or under one half
    const uint32_t hashSize = cfg.backlog_capacity ? nextPow2(2ull * cfg.backlog_capacity)
                                                   : nextPow2(4ull * cfg.slot_capacity);
    d.hashMask = hashSize - 1;
    d.newCap = cfg.backlog_capacity ? cfg.backlog_capacity : hashSize / 2;

    const uint32_t N = cfg.max_nodes;
    rb_status st = RB_OK;
#define ALLOC(ptr, n, what) \
    if ((st = devAlloc(c, &(ptr), (n), (what))) != RB_OK) { rb_release(c); return st; }
    ALLOC(d.child, (uint64_t)N * 8, "node children");
    ALLOC(d.counter, N, "node counters");
    ALLOC(d.numPoints, N, "node point counts");
    ALLOC(d.level, N, "node levels");
    ALLOC(d.nodeX, N, "node X");
    ALLOC(d.nodeY, N, "node Y");
    ALLOC(d.nodeZ, N, "node Z");
    ALLOC(d.grid, N, "node grids");
    ALLOC(d.numVoxels, N, "node voxel counts");
    ALLOC(d.numVoxelsStored, N, "node stored voxel counts");
    ALLOC(d.numPointChunks, N, "node point chunk counts");
    ALLOC(d.numVoxelChunks, N, "node voxel chunk counts");
    ALLOC(d.ptTableOff, N, "point table offsets");
    ALLOC(d.ptTableCap, N, "point table capacities");
    ALLOC(d.vxTableOff, N, "voxel table offsets");
    ALLOC(d.vxTableCap, N, "voxel table capacities");
    ALLOC(d.splitIter, N, "split stamps");
    ALLOC(d.anc, (uint64_t)N * rb::kMaxDepth, "ancestor table");
    ALLOC(d.parent, N, "parent table");
    ALLOC(d.gridPool, N, "grid pool");
    ALLOC(d.dirtyStamp, N, "dirty stamps");
    ALLOC(d.accum, N, "accumulators");
    ALLOC(d.dirtyList, N, "dirty list");
    ALLOC(d.arena, arenaBytes, "the arena (grids and chunks)");
    ALLOC(d.tablePool, d.tablePoolCap, "chunk tables");
    ALLOC(d.chunkQueue, d.maxPtChunks, "chunk queue");
    ALLOC(d.leafOf, cfg.slot_capacity, "per-point leaves");
    ALLOC(d.spillPts, d.spillCap, "spilled points");
    ALLOC(d.spillIdx, d.spillCap, "spilled point indices");
    ALLOC(d.spillLeaf, d.spillCap, "spilled point leaves");
    ALLOC(d.spillNodes, nextPow2(d.spillingCap), "spilling nodes");
    ALLOC(d.splitRecs, d.spillingCap, "split records");
    ALLOC(d.hashSlots, hashSize, "voxel cell table");
    ALLOC(d.hashNew, d.newCap, "new voxel cells");
    ALLOC(d.hashNewNode, d.newCap, "new voxel nodes");
    ALLOC(d.hashNewSlot, d.newCap, "new voxel slots");
    ALLOC(d.hashNewCell, d.newCap, "new voxel cell indices");
    ALLOC(d.hashNewColor, d.newCap, "new voxel colours");
    ALLOC(d.ctr, 1, "counters");
    ALLOC(d.ring, 1, "ring descriptor");
    ALLOC(d.sweep, 1, "sweep stats");
    ALLOC(d.accumGlobals, 1, "accumulator globals");
    ALLOC(d.accumFrom, N, "accumulate plan ranges");
    ALLOC(d.accumTo, N, "accumulate plan ranges");
    ALLOC(d.accumItem, (uint64_t)N + 1, "accumulate plan items");
    d.accumUnitCap = (uint32_t)std::min<uint64_t>((uint64_t)d.maxPtChunks + N, UINT32_MAX);
    ALLOC(d.accumUnitW, d.accumUnitCap, "accumulate work items");
    ALLOC(d.hist8, (uint64_t)N * 8, "child-octant counts");
    ALLOC(d.arrive, N, "points reaching each leaf");
    ALLOC(d.deepCnt, (uint64_t)rb::kDeepRoots * rb::kDeepCells, "expand round bins");
    ALLOC(d.deepNode, (uint64_t)rb::kDeepRoots * rb::kDeepCells, "expand round node table");
    ALLOC(d.moveCode, cfg.slot_capacity, "expand round point codes");
    ALLOC(d.spillCode, d.spillCap, "expand round spilled point codes");
    ALLOC(d.deepSlot, N, "expand round root slots");
    ALLOC(d.deepMeta, N, "expand round node codes");
    ALLOC(d.deepPar, N / 8u + 1u, "expand round split lists");
    d.zeroCap = N / 8u + 1u;
    ALLOC(d.zeroList, d.zeroCap, "grids to zero");
    ALLOC(c->vis, N, "visible flags");
    ALLOC(c->large, N, "large flags");
    ALLOC(c->items, std::max<uint32_t>(cfg.drawlist_capacity, 1), "draw list");
    ALLOC(c->rs, 1, "render scratch");
    ALLOC(c->roll, N, "rolled sums");
    ALLOC(c->analysis, N, "node analysis");
    ALLOC(c->akeys, N, "queue keys");
    ALLOC(c->ahist, 65536, "queue histogram");
    ALLOC(c->acand, kQueueSortCap, "queue candidates");
    ALLOC(c->aqueue, kQueueSortCap, "queue");
    ALLOC(c->actr, 1, "analysis counters");
    ALLOC(c->features, (uint64_t)N * rb::kIn, "scorer features");
    ALLOC(c->predictions, (uint64_t)N * rb::kOut, "scorer predictions");
    ALLOC(c->mlp.params, rb::kNumParams, "scorer parameters");
    ALLOC(c->mlp.grad, rb::kNumParams, "scorer gradient");
    ALLOC(c->mlp.m, rb::kNumParams, "Adam first moment");
    ALLOC(c->mlp.v, rb::kNumParams, "Adam second moment");
    ALLOC(c->mlp.wq, rb::kNumQuant, "scorer BF16 weights");
    ALLOC(c->mlp.loss, 1, "scorer loss");
    c->ingestSlots = 3;
    ALLOC(c->ingestRing, (uint64_t)c->ingestSlots * cfg.slot_capacity, "ingest ring");
    {
        rb::RefineScratch& r = c->refine;
        r.capacity = cfg.refine_voxel_capacity ? cfg.refine_voxel_capacity : 2097152u;
        r.hashMask = nextPow2(2ull * r.capacity) - 1u;
        ALLOC(r.refSlot, N, "refinement node marks");
        ALLOC(r.voxNode, (uint64_t)N + 1, "refinement nodes");
        ALLOC(r.voxBase, (uint64_t)N + 1, "refinement voxel offsets");
        ALLOC(r.acc, r.capacity, "refinement colour sums");
        ALLOC(r.entrySlot, r.capacity, "refinement entry slots");
        ALLOC(r.hashKeys, (uint64_t)r.hashMask + 1, "refinement cell table keys");
        ALLOC(r.hashVals, (uint64_t)r.hashMask + 1, "refinement cell table values");
        ALLOC(r.ctr, 1, "refinement counters");
    }
#undef ALLOC
    RB_CUDA(c, cudaMemsetAsync(d.hashSlots, 0xFF, (size_t)hashSize * 16, c->stream));
    RB_CUDA(c, cudaMemsetAsync(d.ctr, 0, sizeof(Counters), c->stream));
    RB_CUDA(c, cudaMemsetAsync(d.deepCnt, 0, (size_t)rb::kDeepRoots * rb::kDeepCells * 4, c->stream));
    RB_CUDA(c, cudaMemsetAsync(d.deepNode, 0xFF, (size_t)rb::kDeepRoots * rb::kDeepCells * 4, c->stream));
    RB_CUDA(c, cudaMemsetAsync(d.arrive, 0, (size_t)N * 4, c->stream));
    RB_CUDA(c, cudaMemsetAsync(c->refine.refSlot, 0xFF, (size_t)N * 4, c->stream));
    RB_CUDA(c, cudaMemsetAsync(c->refine.hashKeys, 0xFF, ((size_t)c->refine.hashMask + 1) * 8, c->stream));
    RB_CUDA(c, cudaMallocHost(&c->hostRefine, sizeof(rb::RefineCounters)));
    RB_CUDA(c, cudaMemsetAsync(d.accumGlobals, 0, sizeof(rb::AccumGlobals), c->stream));
    RB_CUDA(c, cudaMallocHost(&c->hostCtr, sizeof(Counters)));
    std::memset(c->hostCtr, 0, sizeof(Counters));
    RB_CUDA(c, cudaMallocHost(&c->hostSweep, sizeof(rb::SweepStats)));
    RB_CUDA(c, cudaMallocHost(&c->hostAccum, sizeof(rb::AccumGlobals)));
    RB_CUDA(c, cudaMallocHost(&c->hostRs, sizeof(rb::RenderScratch)));
    RB_CUDA(c, cudaMallocHost(&c->hostActr, sizeof(rb::AnalysisCounters)));
    RB_CUDA(c, cudaMallocHost(&c->hostRing, sizeof(rb::RingDesc)));
    std::memset(c->hostRing, 0, sizeof(rb::RingDesc));
    RB_CUDA(c, cudaMemsetAsync(d.ring, 0, sizeof(rb::RingDesc), c->stream));
    RB_CUDA(c, rb::configureQueueSort(kQueueSortCap));
    RB_CUDA(c, rb::configureMlp());
    for (uint32_t i = 0; i < c->ingestSlots; i++) {
        RB_CUDA(c, cudaEventCreateWithFlags(&c->slotFree[i], cudaEventDisableTiming));
        RB_CUDA(c, cudaEventCreateWithFlags(&c->slotFull[i], cudaEventDisableTiming));
    }
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    // the allocation-free render's static scratch is reserved here, where
    // allocating is expected, not at its first call
    RB_CUDA(c, rb::noallocPrepare(c->device));
    c->allocated = true;
    return rb_reset(c);
}

rb_status rb_reset(rb_ctx* c) {
    if (!c) return RB_ERR_INVALID_ARG;
    if (!c->allocated) return fail(c, RB_ERR_STATE, "reset before allocate");
    if (c->cfg.pipeline == RB_PIPELINE_FLAT) return RB_OK;
    RB_CUDA(c, cudaSetDevice(c->device));
    LAUNCH(c, K_RESET_ROOT, 1, rb::launchResetRoot(c->d, c->numSMs * 2, c->stream));
    RB_CUDA(c, cudaMemsetAsync(c->d.accumGlobals, 0, sizeof(rb::AccumGlobals), c->stream));
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->batchesConsumed = 0;
    c->accumAll = true;
    return readCounters(c);  // the host mirror starts from the reset counters
}

static rb_status buildFrom(rb_ctx* c, const rb::Point* ring, const uint32_t* sizes, uint32_t slots,
                           uint32_t slotCap, uint32_t numUploaded, uint32_t maxBatches, rb_build_result* out) {
    const auto t0 = std::chrono::steady_clock::now();
    const uint32_t first = c->batchesConsumed;
    const uint32_t avail = numUploaded > first ? numUploaded - first : 0u;
    uint32_t nb = std::min(avail, maxBatches);
    for (uint32_t i = 0; i < std::min(slots, numUploaded); i++)
        if (sizes[i] > slotCap) return fail(c, RB_ERR_CAPACITY, "batch larger than its ring slot");
    const bool graphs = graphPath(c);
    if (graphs) {
        if (slots > rb::kMaxRingSlots) return fail(c, RB_ERR_CAPACITY, "more ring slots than a device build handles");
        rb::RingDesc& r = *c->hostRing;
        r.base = reinterpret_cast<unsigned long long>(ring);
        r.slotCap = slotCap;
        r.numSlots = slots;
        r.numUploaded = numUploaded;
        r.streamMode = 0;
        r.first = 0;
        r.batchSize = 0;
        r.total = 0;
        r.budgetNs = c->cfg.time_budget_ms > 0.0f ? (unsigned long long)(c->cfg.time_budget_ms * 1e6) : 0ull;
        for (uint32_t i = 0; i < slots; i++) r.sizes[i] = sizes[i];
        rb_status st = uploadRing(c);
        if (st != RB_OK) return st;
    }
    RB_CUDA(c, cudaEventRecord(c->evStart, c->stream));
    LAUNCH(c, K_BUILD_BEGIN, 1, (k_build_begin<<<1, 1, 0, c->stream>>>(c->d.ctr)));
    uint32_t done = 0;
    bool stopped = false;
    if (graphs) {
        const uint32_t condBefore = c->hostCtr->condRuns;
        const uint64_t pointsBefore = c->hostCtr->numPointsProcessed;
        for (uint32_t k = 0; k < nb; k++) RB_CUDA(c, cudaGraphLaunch(c->batchGraph, c->stream));
        rb_status st = readCounters(c);
        if (st != RB_OK) return st;
        if ((st = checkSync(c)) != RB_OK) return st;
        done = c->hostCtr->batchletIndex - first;
        stopped = c->hostCtr->batchStop && c->hostCtr->stopReason == rb::kStopMemory;
        countGraphLaunches(c, nb, condBefore, c->hostCtr->numPointsProcessed - pointsBefore);
        nb = 0;  // the batches ran on the device
    }
    for (uint32_t b = first; b < first + nb; b++) {
        const uint32_t slot = b % slots;
        const uint32_t n = sizes[slot];
        rb_status st = runBatch(c, ring + (uint64_t)slot * slotCap, n, b, &stopped);
        if (st != RB_OK) return st;
        if (stopped) break;
        done++;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (c->cfg.time_budget_ms > 0.0f && ms > c->cfg.time_budget_ms) break;
    }
    c->batchesConsumed = first + done;
    if (c->cfg.accumulate && c->cfg.pipeline == RB_PIPELINE_REMOLOD) {
        rb_status st = accumulate(c, c->batchesConsumed);
        if (st != RB_OK) return st;
    } else if (done > 0) {
        c->accumAll = true;
    }
    RB_CUDA(c, cudaEventRecord(c->evStop, c->stream));
    RB_CUDA(c, cudaEventSynchronize(c->evStop));
    if (out) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->evStart, c->evStop);
        out->batches_consumed = c->batchesConsumed;
        out->batches_this_call = done;
        out->mem_capacity_reached = stopped ? 1u : 0u;
        out->device_ms = ms;
        out->more = 0;
    }
    return RB_OK;
}

rb_status rb_build(rb_ctx* c, const rb_batch_view* v, rb_build_result* out) {
    if (!c || !v) return RB_ERR_INVALID_ARG;
    if (!c->allocated) return fail(c, RB_ERR_STATE, "build before allocate");
    if (c->cfg.pipeline == RB_PIPELINE_FLAT) return RB_OK;
    if (out) std::memset(out, 0, sizeof(*out));
    if (v->slots == 0 || v->batch_sizes == nullptr || v->num_batches_uploaded == 0) return RB_OK;
    // RemolodPipeline.cpp:315-328: the kernel reads batch B from slot B % ring_slots
    const uint32_t K = c->cfg.ring_slots;
    const bool ok = v->num_slots == K || (v->num_batches_total <= K && v->num_slots >= v->num_batches_total);
    if (!ok)
        return fail(c, RB_ERR_RING,
                    "handed a " + std::to_string(v->num_slots) + "-slot ring but batches wrap at " +
                        std::to_string(K));
    if (v->slot_capacity != c->cfg.slot_capacity)
        return fail(c, RB_ERR_RING, "ring slot capacity differs from the configured slot capacity");
    RB_CUDA(c, cudaSetDevice(c->device));
    std::vector<uint32_t> sizes(K, 0);
    for (uint32_t i = 0; i < std::min(K, v->num_slots); i++) sizes[i] = v->batch_sizes[i];
    rb_status st = buildFrom(c, reinterpret_cast<const rb::Point*>(v->slots), sizes.data(), K,
                             v->slot_capacity, v->num_batches_uploaded, c->cfg.max_batches_per_build, out);
    if (st == RB_OK && out) out->more = (v->num_batches_total > 0 && c->batchesConsumed < v->num_batches_total);
    return st;
}

rb_status rb_ingest_host(rb_ctx* c, const rb_point* points, uint64_t n, uint32_t batchSize,
                         rb_build_result* out) {
    if (!c || (!points && n)) return RB_ERR_INVALID_ARG;
    if (!c->allocated) return fail(c, RB_ERR_STATE, "ingest before allocate");
    if (c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_UNSUPPORTED, "flat keeps no tree");
    if (batchSize == 0 || batchSize > c->cfg.slot_capacity)
        return fail(c, RB_ERR_CAPACITY, "batch size must be in [1, slot_capacity]");
    if (out) std::memset(out, 0, sizeof(*out));
    RB_CUDA(c, cudaSetDevice(c->device));
    const uint64_t nb = (n + batchSize - 1) / batchSize;
    const uint32_t S = c->ingestSlots;
    const uint32_t firstBatch = c->batchesConsumed;
    if ((uint64_t)firstBatch + nb > 0xFFFFFFFFull) return fail(c, RB_ERR_CAPACITY, "too many batches");
    const bool graphs = graphPath(c);
    uint64_t pointsBefore = 0;
    uint32_t condBefore = 0;
    if (graphs) {
        rb::RingDesc& r = *c->hostRing;
        r.base = reinterpret_cast<unsigned long long>(c->ingestRing);
        r.slotCap = c->cfg.slot_capacity;
        r.numSlots = S;
        r.numUploaded = firstBatch + (uint32_t)nb;
        r.streamMode = 1;
        r.first = firstBatch;
        r.batchSize = batchSize;
        r.total = n;
        r.budgetNs = 0;
        rb_status st = uploadRing(c);
        if (st != RB_OK) return st;
        condBefore = c->hostCtr->condRuns;
        pointsBefore = c->hostCtr->numPointsProcessed;
    }
    RB_CUDA(c, cudaEventRecord(c->evStart, c->stream));
    LAUNCH(c, K_BUILD_BEGIN, 1, (k_build_begin<<<1, 1, 0, c->stream>>>(c->d.ctr)));
    // the copy stream fills slot (b % S) once the compute stream released it
    auto issueCopy = [&](uint64_t b) -> rb_status {
        const uint32_t slot = (uint32_t)(b % S);
        const uint64_t first = b * batchSize;
        const uint64_t cnt = std::min<uint64_t>(batchSize, n - first);
        if (b >= S) RB_CUDA(c, cudaStreamWaitEvent(c->copyStream, c->slotFree[slot], 0));
        RB_CUDA(c, cudaMemcpyAsync(c->ingestRing + (uint64_t)slot * c->cfg.slot_capacity, points + first,
                                   cnt * sizeof(rb_point), cudaMemcpyHostToDevice, c->copyStream));
        RB_CUDA(c, cudaEventRecord(c->slotFull[slot], c->copyStream));
        return RB_OK;
    };
    for (uint64_t b = 0; b < std::min<uint64_t>(nb, S); b++) {
        rb_status st = issueCopy(b);
        if (st != RB_OK) return st;
    }
    uint32_t done = 0;
    bool stopped = false;
    const bool accumOn = c->cfg.accumulate && c->cfg.pipeline == RB_PIPELINE_REMOLOD;
    bool pendingFold = false;
    for (uint64_t b = 0; b < nb; b++) {
        const uint32_t slot = (uint32_t)(b % S);
        const uint64_t first = b * batchSize;
        const uint32_t cnt = (uint32_t)std::min<uint64_t>(batchSize, n - first);
        RB_CUDA(c, cudaStreamWaitEvent(c->stream, c->slotFull[slot], 0));
        rb_status st = RB_OK;
        if (graphs) {
            // the graph finds batch first + b at slot b % S itself; a batch the
            // memory check stops leaves the rest of the run as no-ops
            RB_CUDA(c, cudaGraphLaunch(c->batchGraph, c->stream));
        } else {
            st = runBatch(c, c->ingestRing + (uint64_t)slot * c->cfg.slot_capacity, cnt, c->batchesConsumed,
                          &stopped);
            if (st != RB_OK) return st;
        }
        RB_CUDA(c, cudaEventRecord(c->slotFree[slot], c->stream));
        if (stopped) break;
        c->batchesConsumed++;
        done++;
        if (b + S < nb) {
            st = issueCopy(b + S);
            if (st != RB_OK) return st;
        }
        // Accumulate at the frame cadence: after every max_batches_per_build batches
        if (accumOn && (done % std::max<uint32_t>(c->cfg.max_batches_per_build, 1)) == 0) {
            st = accumulate(c, c->batchesConsumed);
            if (st != RB_OK) return st;
            pendingFold = false;
        } else {
            pendingFold = true;
        }
    }
    if (accumOn && pendingFold) {
        rb_status st = accumulate(c, c->batchesConsumed);
        if (st != RB_OK) return st;
    } else if (!accumOn && done > 0) {
        c->accumAll = true;
    }
    RB_CUDA(c, cudaEventRecord(c->evStop, c->stream));
    RB_CUDA(c, cudaEventSynchronize(c->evStop));
    RB_CUDA(c, cudaStreamSynchronize(c->copyStream));
    if (graphs) {
        rb_status st = readCounters(c);
        if (st != RB_OK) return st;
        if ((st = checkSync(c)) != RB_OK) return st;
        c->batchesConsumed = c->hostCtr->batchletIndex;
        done = c->batchesConsumed - firstBatch;
        stopped = c->hostCtr->batchStop && c->hostCtr->stopReason == rb::kStopMemory;
        countGraphLaunches(c, nb, condBefore, c->hostCtr->numPointsProcessed - pointsBefore);
    }
    if (out) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->evStart, c->evStop);
        out->batches_consumed = c->batchesConsumed;
        out->batches_this_call = done;
        out->mem_capacity_reached = stopped ? 1u : 0u;
        out->device_ms = ms;
    }
    return RB_OK;
}

rb_status rb_accumulate(rb_ctx* c, uint32_t batchIndex, rb_accum_globals* out) {
    if (!c) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = accumulate(c, batchIndex);
    if (st != RB_OK) return st;
    if (out) {
        RB_CUDA(c, cudaMemcpyAsync(c->hostAccum, c->d.accumGlobals, sizeof(rb::AccumGlobals),
                                   cudaMemcpyDeviceToHost, c->stream));
        RB_CUDA(c, cudaStreamSynchronize(c->stream));
        static_assert(sizeof(rb_accum_globals) == sizeof(rb::AccumGlobals), "AccumGlobals layout");
        std::memcpy(out, c->hostAccum, sizeof(*out));
    }
    return RB_OK;
}

static rb::Frame toFrame(const rb_frame* f) {
    rb::Frame r;
    r.width = f->width;
    r.height = f->height;
    std::memcpy(r.transform, f->transform, sizeof(r.transform));
    std::memcpy(r.transformFrozen, f->transform_frozen, sizeof(r.transformFrozen));
    for (int a = 0; a < 3; a++) {
        r.boxMin[a] = f->box_min[a];
        r.boxMax[a] = f->box_max[a];
    }
    r.lodPixelBudget = f->lod_pixel_budget;
    r.pointSize = f->point_size;
    r.colorMode = f->color_mode;
    r.showBoundingBox = f->show_bounding_box;
    return r;
}

static rb_status finishFrame(rb_ctx* c, const rb_frame* f, unsigned long long* fb, uint32_t* rgba,
                             uint64_t npx) {
    // EDL in place: it reads only its neighbours' depths, which it never
    // writes (a pixel's shading changes its colour half only)
    if (f->enable_edl)
        LAUNCH(c, K_EDL, npx, rb::launchEdl(fb, fb, (uint32_t)f->width, (uint32_t)f->height, f->edl_strength,
                                            c->numSMs * 8, c->stream));
    if (rgba) LAUNCH(c, K_RESOLVE, npx, rb::launchResolve(fb, rgba, npx, c->numSMs * 8, c->stream));
    return RB_OK;
}

rb_status rb_render(rb_ctx* c, const rb_frame* f, uint64_t fbDev, uint64_t rgbaDev, uint64_t forceDev,
                    rb_render_result* out) {
    if (!c || !f || !fbDev) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree to render");
    if (!(f->width >= 1.0f && f->height >= 1.0f)) return fail(c, RB_ERR_INVALID_ARG, "empty frame");
    RB_CUDA(c, cudaSetDevice(c->device));
    const uint64_t npx = (uint64_t)f->width * (uint64_t)f->height;
    auto* fb = reinterpret_cast<unsigned long long*>(fbDev);
    const rb::Frame fr = toFrame(f);
    const uint32_t cap = std::max<uint32_t>(c->cfg.drawlist_capacity, 1);
    RB_CUDA(c, cudaEventRecord(c->evStart, c->stream));
    LAUNCH(c, K_FB_CLEAR, npx, rb::launchFbClear(fb, npx, c->numSMs * 8, c->stream));
    LAUNCH(c, K_NODE_FLAGS, 0, rb::launchNodeFlags(c->d, fr, c->vis, c->large,
                                                   reinterpret_cast<const uint8_t*>(forceDev), c->rs,
                                                   c->numSMs * 4, c->stream));
    LAUNCH(c, K_FRONTIER, 0, rb::launchFrontier(c->d, c->vis, c->large, c->rs, c->items, cap, c->numSMs * 4,
                                                c->stream));
    LAUNCH(c, K_RASTER, 0, rb::launchRaster(c->d, fr, fb, c->rs, c->items, cap, c->numSMs * 8, c->stream));
    // EDL, then the boxes (remolod_render.cu:183-189), then the resolve
    rb_status st = finishFrame(c, f, fb, nullptr, npx);
    if (st != RB_OK) return st;
    if (f->show_bounding_box)
        LAUNCH(c, K_WIREFRAME, 0, rb::launchWireframe(c->d, fr, fb, c->rs, c->items, cap, c->numSMs * 8, c->stream));
    if (rgbaDev)
        LAUNCH(c, K_RESOLVE, npx, rb::launchResolve(fb, reinterpret_cast<uint32_t*>(rgbaDev), npx, c->numSMs * 8,
                                                    c->stream));
    if (st != RB_OK) return st;
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaEventRecord(c->evStop, c->stream));
    RB_CUDA(c, cudaMemcpyAsync(c->hostRs, c->rs, sizeof(rb::RenderScratch), cudaMemcpyDeviceToHost, c->stream));
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->lastVisibleNodes = c->hostRs->numItems;
    c->lastVisibleSamples = c->hostRs->samples;
    if (out) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->evStart, c->evStop);
        out->draw_items = c->hostRs->numItems;
        out->drawlist_overflow = c->hostRs->overflow;
        out->draw_samples = c->hostRs->samples;
        out->device_ms = ms;
    }
    return RB_OK;
}

rb_status rb_render_flat(rb_ctx* c, const rb_frame* f, uint64_t pointsDev, uint64_t n, uint64_t fbDev,
                         uint64_t rgbaDev, rb_render_result* out) {
    if (!c || !f || !fbDev || (!pointsDev && n)) return RB_ERR_INVALID_ARG;
    if (!c->allocated) return fail(c, RB_ERR_STATE, "render before allocate");
    if (!(f->width >= 1.0f && f->height >= 1.0f)) return fail(c, RB_ERR_INVALID_ARG, "empty frame");
    RB_CUDA(c, cudaSetDevice(c->device));
    const uint64_t npx = (uint64_t)f->width * (uint64_t)f->height;
    auto* fb = reinterpret_cast<unsigned long long*>(fbDev);
    const rb::Frame fr = toFrame(f);
    RB_CUDA(c, cudaEventRecord(c->evStart, c->stream));
    LAUNCH(c, K_FB_CLEAR, npx, rb::launchFbClear(fb, npx, c->numSMs * 8, c->stream));
    if (n)
        LAUNCH(c, K_RASTER_FLAT, n,
               rb::launchRasterFlat(fr, fb, reinterpret_cast<const rb::Point*>(pointsDev), n, c->numSMs * 16,
                                    c->stream));
    rb_status st = finishFrame(c, f, fb, reinterpret_cast<uint32_t*>(rgbaDev), npx);
    if (st != RB_OK) return st;
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaEventRecord(c->evStop, c->stream));
    RB_CUDA(c, cudaEventSynchronize(c->evStop));
    if (out) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->evStart, c->evStop);
        out->draw_items = (uint32_t)((n + 65535) / 65536);  // the reference's 64K slices
        out->drawlist_overflow = 0;
        out->draw_samples = n;
        out->device_ms = ms;
    }
    return RB_OK;
}

rb_status rb_read_stats(rb_ctx* c, rb_stats* o) {
    if (!c || !o) return RB_ERR_INVALID_ARG;
    std::memset(o, 0, sizeof(*o));
    if (!c->allocated) return fail(c, RB_ERR_STATE, "stats before allocate");
    o->bytes_allocated = c->bytes;
    if (c->cfg.pipeline == RB_PIPELINE_FLAT) return RB_OK;
    RB_CUDA(c, cudaSetDevice(c->device));
    RB_CUDA(c, cudaMemsetAsync(c->d.sweep, 0, sizeof(rb::SweepStats), c->stream));
    LAUNCH(c, K_SWEEP, 0, rb::launchSweep(c->d, c->numSMs * 4, c->stream));
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaMemcpyAsync(c->hostSweep, c->d.sweep, sizeof(rb::SweepStats), cudaMemcpyDeviceToHost, c->stream));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    const Counters& k = *c->hostCtr;
    const rb::SweepStats& s = *c->hostSweep;
    o->num_points = s.numPoints;
    o->num_voxels = s.numVoxels;
    o->num_points_ingested = k.numPointsProcessed;
    o->num_nodes = k.numNodes;
    o->num_inner = s.numInner;
    o->num_leaves = s.numLeaves;
    o->num_nonempty_leaves = s.numNonemptyLeaves;
    o->max_depth = s.maxLevel;
    o->max_points_per_node = s.maxPointsPerNode;
    o->num_chunks_points = s.numChunksPoints;
    o->num_chunks_voxels = s.numChunksVoxels;
    o->batchlet_index = k.batchletIndex;
    o->counter_underflows = s.counterUnderflows;
    o->num_allocated_chunks = k.numAllocatedChunks;
    o->chunk_pool_size = k.chunkPoolSize;
    o->persistent_offset = k.refOffset;
    o->persistent_capacity = c->d.persistentCapacity;
    o->dropped_points = k.droppedPoints;
    o->expand_iters = k.expandIters;
    o->nodes_split = k.nodesSplit;
    o->spilled_points = k.spilledPointsTotal;
    o->num_grids = k.numGrids;
    o->overflow_flags = k.overflowFlags;
    o->mem_capacity_reached = k.memCapacityReached;
    o->node_capacity_reached = k.nodePoolOverflow || k.numNodes >= c->cfg.max_nodes;
    o->num_visible_nodes = c->lastVisibleNodes;
    o->num_visible_samples = c->lastVisibleSamples;
    return RB_OK;
}

rb_status rb_read_nodes(rb_ctx* c, rb_node_info* out, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    const uint32_t nn = c->hostCtr->numNodes;
    *count = nn;
    if (!out) return RB_OK;
    if (capacity < nn) return fail(c, RB_ERR_CAPACITY, "node buffer too small");
    std::vector<int32_t> child((size_t)nn * 8);
    std::vector<uint32_t> a[10];
    uint32_t* src[10] = {c->d.counter, c->d.numPoints, c->d.level, c->d.nodeX, c->d.nodeY, c->d.nodeZ,
                         c->d.grid, c->d.numVoxels, c->d.numPointChunks, c->d.numVoxelChunks};
    RB_CUDA(c, cudaMemcpy(child.data(), c->d.child, (size_t)nn * 32, cudaMemcpyDeviceToHost));
    for (int k = 0; k < 10; k++) {
        a[k].resize(nn);
        RB_CUDA(c, cudaMemcpy(a[k].data(), src[k], (size_t)nn * 4, cudaMemcpyDeviceToHost));
    }
    for (uint32_t i = 0; i < nn; i++) {
        rb_node_info& o = out[i];
        bool leaf = true;
        for (int q = 0; q < 8; q++) {
            o.child[q] = child[(size_t)i * 8 + q];
            if (o.child[q] >= 0) leaf = false;
        }
        o.counter = a[0][i];
        o.num_points = a[1][i];
        o.level = a[2][i];
        o.X = a[3][i];
        o.Y = a[4][i];
        o.Z = a[5][i];
        o.has_grid = a[6][i] != kNone;
        o.num_voxels = a[7][i];
        o.num_point_chunks = a[8][i];
        o.num_voxel_chunks = a[9][i];
        o.is_leaf = leaf;
    }
    return RB_OK;
}

static rb_status readChunked(rb_ctx* c, uint32_t node, bool voxels, rb_point* pts, uint32_t* idx,
                             uint32_t capacity, uint32_t* count) {
    RB_CUDA(c, cudaSetDevice(c->device));
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    if (node >= c->hostCtr->numNodes) return fail(c, RB_ERR_INVALID_ARG, "node out of range");
    uint32_t n = 0, nch = 0, off = 0, stored = 0;
    RB_CUDA(c, cudaMemcpy(&n, (voxels ? c->d.numVoxels : c->d.numPoints) + node, 4, cudaMemcpyDeviceToHost));
    RB_CUDA(c, cudaMemcpy(&nch, (voxels ? c->d.numVoxelChunks : c->d.numPointChunks) + node, 4,
                          cudaMemcpyDeviceToHost));
    RB_CUDA(c, cudaMemcpy(&off, (voxels ? c->d.vxTableOff : c->d.ptTableOff) + node, 4, cudaMemcpyDeviceToHost));
    if (voxels) {
        RB_CUDA(c, cudaMemcpy(&stored, c->d.numVoxelsStored + node, 4, cudaMemcpyDeviceToHost));
        n = std::min(n, stored);
    }
    const uint32_t ppc = c->d.ppc;
    n = std::min<uint32_t>(n, nch * ppc);
    *count = n;
    if (!pts) return RB_OK;
    if (capacity < n) return fail(c, RB_ERR_CAPACITY, "point buffer too small");
    if (n == 0) return RB_OK;
    std::vector<uint32_t> table(nch);
    RB_CUDA(c, cudaMemcpy(table.data(), c->d.tablePool + off, (size_t)nch * 4, cudaMemcpyDeviceToHost));
    for (uint32_t j = 0; j * ppc < n; j++) {
        const uint32_t cnt = std::min(ppc, n - j * ppc);
        if (table[j] == kNone) return fail(c, RB_ERR_STATE, "chunk missing");
        const uint8_t* base = c->d.arena + (uint64_t)table[j] * 16ull;
        RB_CUDA(c, cudaMemcpy(pts + (size_t)j * ppc, base, (size_t)cnt * 16, cudaMemcpyDeviceToHost));
        if (idx && !voxels)
            RB_CUDA(c, cudaMemcpy(idx + (size_t)j * ppc, base + (uint64_t)ppc * 16, (size_t)cnt * 4,
                                  cudaMemcpyDeviceToHost));
    }
    return RB_OK;
}

rb_status rb_read_node_points(rb_ctx* c, uint32_t node, rb_point* pts, uint32_t* idx, uint32_t capacity,
                              uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    return readChunked(c, node, false, pts, idx, capacity, count);
}

rb_status rb_read_node_voxels(rb_ctx* c, uint32_t node, rb_point* vox, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    return readChunked(c, node, true, vox, nullptr, capacity, count);
}

rb_status rb_read_node_grid(rb_ctx* c, uint32_t node, uint32_t* words) {
    if (!c || !words) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    if (node >= c->hostCtr->numNodes) return fail(c, RB_ERR_INVALID_ARG, "node out of range");
    uint32_t g = kNone;
    RB_CUDA(c, cudaMemcpy(&g, c->d.grid + node, 4, cudaMemcpyDeviceToHost));
    if (g == kNone) return fail(c, RB_ERR_INVALID_ARG, "node has no grid");
    RB_CUDA(c, cudaMemcpy(words, c->d.arena + (uint64_t)g * 16ull, rb::kGridBytes, cudaMemcpyDeviceToHost));
    return RB_OK;
}

rb_status rb_analyze(rb_ctx* c, const rb_frame* f, const rb_analysis_params* p, rb_analysis_result* out) {
    if (!c || !f || !p) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree to analyse");
    if (p->queue_capacity == 0 || p->queue_capacity > kQueueSortCap)
        return fail(c, RB_ERR_CAPACITY, "queue_capacity must be in [1, 16384]");
    if (!(f->width >= 1.0f && f->height >= 1.0f)) return fail(c, RB_ERR_INVALID_ARG, "empty frame");
    RB_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const int grid = c->numSMs * 4;
    rb::AnalysisParams ap;
    ap.minPoints = p->min_points;
    ap.closureMargin = p->closure_margin;
    ap.currentBatch = c->batchesConsumed;
    ap.frontierOnly = p->frontier_only;
    ap.pixelBudget = p->pixel_budget;
    ap.scoreMode = p->score_mode;
    if (p->score_mode > RB_SCORE_LEARNED) return fail(c, RB_ERR_INVALID_ARG, "unknown score_mode");
    if (p->score_mode == RB_SCORE_LEARNED && !c->mlpReady)
        return fail(c, RB_ERR_STATE, "learned scoring needs rb_mlp_init or rb_mlp_set_params first");
    rb_status rst = readCounters(c);
    if (rst != RB_OK) return rst;
    const uint32_t numNodes = c->hostCtr->numNodes;
    const rb::Frame fr = toFrame(f);
    RB_CUDA(c, cudaEventRecord(c->evStart, s));
    RB_CUDA(c, cudaMemsetAsync(c->ahist, 0, 65536 * 4, s));
    RB_CUDA(c, cudaMemsetAsync(c->actr, 0, sizeof(rb::AnalysisCounters), s));
    for (int L = rb::kMaxDepth; L >= 0; L--)
        LAUNCH(c, K_ROLL, 0, rb::launchRollLevel(c->d, c->roll, (uint32_t)L, grid, s));
    LAUNCH(c, K_ANALYZE, 0, rb::launchAnalyze(c->d, c->roll, c->analysis, c->features, ap, fr, c->actr, grid, s));
    if (p->score_mode == RB_SCORE_LEARNED)
        LAUNCH(c, K_MLP_PREDICT, numNodes,
               rb::launchMlpPredict(c->mlp, c->features, numNodes, c->predictions, c->numSMs * 4, s));
    LAUNCH(c, K_SCORE, 0, rb::launchScore(c->d, c->analysis, c->predictions, c->akeys, ap, c->actr, grid, s));
    LAUNCH(c, K_QUEUE, 0, rb::launchQueue(c->d, c->akeys, c->ahist, c->acand, kQueueSortCap, p->queue_capacity,
                                          c->aqueue, c->actr, grid, s));
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaEventRecord(c->evStop, s));
    RB_CUDA(c, cudaMemcpyAsync(c->hostActr, c->actr, sizeof(rb::AnalysisCounters), cudaMemcpyDeviceToHost, s));
    RB_CUDA(c, cudaStreamSynchronize(s));
    c->analyzed = true;
    if (out) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->evStart, c->evStop);
        out->queue_length = c->hostActr->queueLength;
        out->eligible = c->hostActr->eligible;
        out->fp64_branch = c->hostActr->fp64Branch;
        out->overflow = c->hostActr->overflow;
        out->device_ms = ms;
        out->pad = 0;
    }
    return RB_OK;
}

static rb_status copyOut(rb_ctx* c, void* out, const void* src, size_t elem, uint32_t capacity, uint32_t* count,
                         uint32_t n) {
    *count = n;
    if (!out) return RB_OK;
    if (capacity < n) return fail(c, RB_ERR_CAPACITY, "output buffer too small");
    RB_CUDA(c, cudaMemcpy(out, src, (size_t)n * elem, cudaMemcpyDeviceToHost));
    return RB_OK;
}

rb_status rb_read_analysis(rb_ctx* c, rb_node_analysis* out, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->analyzed) return fail(c, RB_ERR_STATE, "read before rb_analyze");
    static_assert(sizeof(rb_node_analysis) == sizeof(rb::NodeAnalysis), "analysis layout");
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    return copyOut(c, out, c->analysis, sizeof(rb_node_analysis), capacity, count, c->hostCtr->numNodes);
}

rb_status rb_read_features(rb_ctx* c, float* out, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->analyzed) return fail(c, RB_ERR_STATE, "read before rb_analyze");
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    return copyOut(c, out, c->features, sizeof(float) * rb::kIn, capacity, count, c->hostCtr->numNodes);
}

static rb_status mlpUpload(rb_ctx* c, const float* params) {
    RB_CUDA(c, cudaMemcpy(c->mlp.params, params, sizeof(float) * rb::kNumParams, cudaMemcpyHostToDevice));
    RB_CUDA(c, cudaMemset(c->mlp.m, 0, sizeof(float) * rb::kNumParams));
    RB_CUDA(c, cudaMemset(c->mlp.v, 0, sizeof(float) * rb::kNumParams));
    rb::launchMlpQuantize(c->mlp, c->stream);
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->adamT = 0;
    c->mlpReady = true;
    return RB_OK;
}

static rb_status mlpCheck(rb_ctx* c) {
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT || !c->mlp.params)
        return fail(c, RB_ERR_STATE, "the scorer lives in an allocated remolod/simlod context");
    return RB_OK;
}

rb_status rb_mlp_init(rb_ctx* c, uint64_t seed) {
    if (!c) return RB_ERR_INVALID_ARG;
    rb_status st = mlpCheck(c);
    if (st != RB_OK) return st;
    RB_CUDA(c, cudaSetDevice(c->device));
    // Glorot-uniform weights (Glorot & Bengio 2010), zero biases; splitmix64 stream
    std::vector<float> p(rb::kNumParams, 0.0f);
    uint64_t x = seed;
    auto next = [&]() {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int rows, int cols) {
        const double a = std::sqrt(6.0 / (double)(rows + cols));
        for (int i = 0; i < rows * cols; i++) p[off + i] = (float)((2.0 * next() - 1.0) * a);
    };
    fill(rb::kPW1, rb::kHidden, rb::kIn);
    fill(rb::kPW2, rb::kHidden, rb::kHidden);
    fill(rb::kPW3, rb::kOut, rb::kHidden);
    return mlpUpload(c, p.data());
}

rb_status rb_mlp_set_params(rb_ctx* c, const float* params) {
    if (!c || !params) return RB_ERR_INVALID_ARG;
    rb_status st = mlpCheck(c);
    if (st != RB_OK) return st;
    RB_CUDA(c, cudaSetDevice(c->device));
    return mlpUpload(c, params);
}

rb_status rb_mlp_get_params(rb_ctx* c, float* params) {
    if (!c || !params) return RB_ERR_INVALID_ARG;
    rb_status st = mlpCheck(c);
    if (st != RB_OK) return st;
    if (!c->mlpReady) return fail(c, RB_ERR_STATE, "scorer not initialised");
    RB_CUDA(c, cudaSetDevice(c->device));
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    RB_CUDA(c, cudaMemcpy(params, c->mlp.params, sizeof(float) * rb::kNumParams, cudaMemcpyDeviceToHost));
    return RB_OK;
}

rb_status rb_mlp_predict(rb_ctx* c, uint64_t x, uint32_t n, uint64_t y) {
    if (!c || (n && (!x || !y))) return RB_ERR_INVALID_ARG;
    rb_status st = mlpCheck(c);
    if (st != RB_OK) return st;
    if (!c->mlpReady) return fail(c, RB_ERR_STATE, "scorer not initialised");
    RB_CUDA(c, cudaSetDevice(c->device));
    LAUNCH(c, K_MLP_PREDICT, n, rb::launchMlpPredict(c->mlp, reinterpret_cast<const float*>(x), n,
                                                      reinterpret_cast<float*>(y), c->numSMs * 8, c->stream));
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    return RB_OK;
}

static rb_status mlpGrad(rb_ctx* c, uint64_t x, uint64_t t, uint32_t n) {
    RB_CUDA(c, cudaMemsetAsync(c->mlp.grad, 0, sizeof(float) * rb::kNumParams, c->stream));
    RB_CUDA(c, cudaMemsetAsync(c->mlp.loss, 0, sizeof(float), c->stream));
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 63) / 64, (uint64_t)c->numSMs));
    LAUNCH(c, K_MLP_GRAD, n, rb::launchMlpGrad(c->mlp, reinterpret_cast<const float*>(x),
                                               reinterpret_cast<const float*>(t), n, grid, c->stream));
    RB_CUDA(c, cudaGetLastError());
    return RB_OK;
}

rb_status rb_mlp_gradients(rb_ctx* c, uint64_t x, uint64_t t, uint32_t n, float* grad, float* loss) {
    if (!c || !x || !t || n == 0) return RB_ERR_INVALID_ARG;
    rb_status st = mlpCheck(c);
    if (st != RB_OK) return st;
    if (!c->mlpReady) return fail(c, RB_ERR_STATE, "scorer not initialised");
    RB_CUDA(c, cudaSetDevice(c->device));
    st = mlpGrad(c, x, t, n);
    if (st != RB_OK) return st;
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (grad) RB_CUDA(c, cudaMemcpy(grad, c->mlp.grad, sizeof(float) * rb::kNumParams, cudaMemcpyDeviceToHost));
    if (loss) {
        RB_CUDA(c, cudaMemcpy(loss, c->mlp.loss, sizeof(float), cudaMemcpyDeviceToHost));
        *loss /= (float)n;
    }
    return RB_OK;
}

rb_status rb_mlp_train_step(rb_ctx* c, uint64_t x, uint64_t t, uint32_t n, float lr, float* loss) {
    if (!c || !x || !t || n == 0 || !(lr > 0.0f)) return RB_ERR_INVALID_ARG;
    rb_status st = mlpCheck(c);
    if (st != RB_OK) return st;
    if (!c->mlpReady) return fail(c, RB_ERR_STATE, "scorer not initialised");
    RB_CUDA(c, cudaSetDevice(c->device));
    st = mlpGrad(c, x, t, n);
    if (st != RB_OK) return st;
    c->adamT += 1;
    rb::AdamStep a;
    a.lr = lr;
    a.beta1 = 0.9f;
    a.beta2 = 0.999f;
    a.eps = 1e-8f;
    a.bc1 = (float)(1.0 - std::pow(0.9, (double)c->adamT));
    a.bc2 = (float)(1.0 - std::pow(0.999, (double)c->adamT));
    LAUNCH(c, K_MLP_ADAM, 0, rb::launchMlpAdam(c->mlp, a, c->stream));
    RB_CUDA(c, cudaGetLastError());
    if (loss) {
        RB_CUDA(c, cudaMemcpyAsync(loss, c->mlp.loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
        RB_CUDA(c, cudaStreamSynchronize(c->stream));
        *loss /= (float)n;
    }
    return RB_OK;
}

rb_status rb_read_queue(rb_ctx* c, uint32_t* ids, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->analyzed) return fail(c, RB_ERR_STATE, "read before rb_analyze");
    RB_CUDA(c, cudaSetDevice(c->device));
    return copyOut(c, ids, c->aqueue, 4, capacity, count, c->hostActr->queueLength);
}

rb_status rb_read_rollup(rb_ctx* c, uint64_t* out16, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->analyzed) return fail(c, RB_ERR_STATE, "read before rb_analyze");
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    const uint32_t nn = c->hostCtr->numNodes;
    *count = nn;
    if (!out16) return RB_OK;
    if (capacity < nn) return fail(c, RB_ERR_CAPACITY, "output buffer too small");
    std::vector<rb::RollSum> tmp(nn);
    RB_CUDA(c, cudaMemcpy(tmp.data(), c->roll, (size_t)nn * sizeof(rb::RollSum), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < nn; i++) {
        uint64_t* o = out16 + (size_t)i * 16;
        o[0] = tmp[i].n;
        for (int k = 0; k < 3; k++) o[1 + k] = tmp[i].s1[k];
        for (int k = 0; k < 12; k++) o[4 + k] = tmp[i].s2[k];
    }
    return RB_OK;
}

rb_status rb_refine(rb_ctx* c, uint32_t budget, uint64_t maskDev) {
    if (!c || !maskDev) return RB_ERR_INVALID_ARG;
    if (!c->analyzed) return fail(c, RB_ERR_STATE, "refine before rb_analyze");
    RB_CUDA(c, cudaSetDevice(c->device));
    LAUNCH(c, K_REFINE, budget, rb::launchRefineMask(c->d, c->aqueue, c->actr, budget,
                                                     reinterpret_cast<uint8_t*>(maskDev), c->numSMs * 2, c->stream));
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    return RB_OK;
}

rb_status rb_refine_colors(rb_ctx* c, uint32_t budget, rb_refine_result* out) {
    if (!c) return RB_ERR_INVALID_ARG;
    if (!c->analyzed) return fail(c, RB_ERR_STATE, "refine before rb_analyze");
    if (out) std::memset(out, 0, sizeof(*out));
    RB_CUDA(c, cudaSetDevice(c->device));
    const uint32_t qlen = c->hostActr->queueLength;
    LAUNCH(c, K_REFINE_COLORS, budget,
           rb::launchRefineColors(c->d, c->refine, c->aqueue, qlen, budget, c->numSMs * 4, c->stream));
    RB_CUDA(c, cudaGetLastError());
    RB_CUDA(c, cudaMemcpyAsync(c->hostRefine, c->refine.ctr, sizeof(rb::RefineCounters), cudaMemcpyDeviceToHost,
                               c->stream));
    RB_CUDA(c, cudaStreamSynchronize(c->stream));
    if (out) {
        out->nodes_filtered = c->hostRefine->nodes;
        out->voxels_filtered = c->hostRefine->voxels;
        out->points_visited = c->hostRefine->points;
    }
    return RB_OK;
}

rb_status rb_refine_deepen(rb_ctx* c, uint32_t budget, uint32_t min_points, rb_deepen_result* out) {
    if (!c) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    if (!c->analyzed) return fail(c, RB_ERR_STATE, "refine before rb_analyze");
    if (out) std::memset(out, 0, sizeof(*out));
    const uint32_t qlen = c->hostActr->queueLength;
    if (budget == 0 || qlen == 0) return RB_OK;  // nothing to take: no pass
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    const uint64_t splitBefore = c->hostCtr->nodesSplit;
    const uint32_t nodesBefore = c->hostCtr->numNodes;
    LAUNCH(c, K_DEEPEN, 1, rb::launchDeepenBegin(c->d, c->aqueue, qlen, budget, min_points, c->stream));
    bool stopped = false;
    // no batch points: every phase reads the spill list only
    st = runBatchAfterCount(c, c->d.spillPts, 0u, (uint64_t)c->numSMs * 8u * 256u, &stopped, true);
    if (st != RB_OK) return st;
    if ((st = readCounters(c)) != RB_OK) return st;
    const rb::Counters& k = *c->hostCtr;
    // the queue names nodes by their role before the pass
    c->analyzed = false;
    if (out) {
        out->stopped = k.batchStop ? 1u : 0u;
        out->nodes_selected = k.batchStop ? 0u : k.deepenSelected;
        out->nodes_split = (uint32_t)(k.nodesSplit - splitBefore);
        const uint32_t room = c->cfg.max_nodes > nodesBefore ? (c->cfg.max_nodes - nodesBefore) / 8u : 0u;
        out->nodes_refused = out->nodes_selected > room ? out->nodes_selected - room : 0u;
        out->points_moved = k.batchStop ? 0u : k.numSpilled;
        const uint64_t made = (uint64_t)k.numNew + k.numLift;
        out->voxels_made = k.batchStop ? 0u : (made < c->d.newCap ? made : c->d.newCap);
    }
    if (!k.batchStop && c->cfg.accumulate && c->cfg.pipeline == RB_PIPELINE_REMOLOD) {
        if ((st = accumulate(c, k.batchletIndex)) != RB_OK) return st;
        RB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return RB_OK;
}

rb_status rb_refine_collapse(rb_ctx* c, const uint32_t* nodes, uint32_t count, uint32_t max_points,
                             rb_collapse_result* out) {
    if (!c || (count && !nodes)) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    if (count > 4096u || count > c->d.spillingCap)
        return fail(c, RB_ERR_CAPACITY, "collapse takes at most 4096 candidate nodes per call");
    if (out) std::memset(out, 0, sizeof(*out));
    if (count == 0) return RB_OK;
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    const uint32_t poolBefore = c->hostCtr->gridPoolSize;
    RB_CUDA(c, cudaMemsetAsync(&c->d.ctr->collapsePoints, 0, 2 * sizeof(unsigned long long), c->stream));
    RB_CUDA(c, cudaMemcpyAsync(c->d.spillNodes, nodes, (size_t)count * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               c->stream));
    LAUNCH(c, K_COLLAPSE, count, rb::launchCollapse(c->d, count, max_points, c->numSMs * 4, c->stream));
    RB_CUDA(c, cudaGetLastError());
    if ((st = readCounters(c)) != RB_OK) return st;
    const rb::Counters& k = *c->hostCtr;
    c->analyzed = false;
    if (out) {
        out->nodes_collapsed = k.collapseSelected;
        out->grids_returned = k.gridPoolSize - poolBefore;
        out->points_moved = k.collapsePoints;
        out->voxels_dropped = k.collapseVoxels;
    }
    if (k.collapseSelected && c->cfg.accumulate && c->cfg.pipeline == RB_PIPELINE_REMOLOD) {
        if ((st = accumulate(c, k.batchletIndex)) != RB_OK) return st;
        RB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return RB_OK;
}

rb_status rb_set_profiling(rb_ctx* c, int on) {
    if (!c) return RB_ERR_INVALID_ARG;
    c->prof.resolve();
    c->prof.on = on != 0;
    return RB_OK;
}

rb_status rb_read_profile(rb_ctx* c, rb_kernel_profile* out, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (c->stream) RB_CUDA(c, cudaStreamSynchronize(c->stream));
    c->prof.resolve();
    *count = K_NUM;
    if (!out) return RB_OK;
    if (capacity < (uint32_t)K_NUM) return fail(c, RB_ERR_CAPACITY, "profile buffer too small");
    for (int k = 0; k < K_NUM; k++) {
        std::memset(&out[k], 0, sizeof(out[k]));
        std::snprintf(out[k].name, sizeof(out[k].name), "%s", kKernelNames[k]);
        out[k].launches = c->prof.launches[k];
        out[k].timed_launches = c->prof.timed[k];
        out[k].total_ms = c->prof.ms[k];
        out[k].units = c->prof.units[k];
    }
    return RB_OK;
}

rb_status rb_reset_profile(rb_ctx* c) {
    if (!c) return RB_ERR_INVALID_ARG;
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->prof.resolve();
    for (int k = 0; k < K_NUM; k++) {
        c->prof.launches[k] = c->prof.timed[k] = c->prof.units[k] = 0;
        c->prof.ms[k] = 0.0;
    }
    return RB_OK;
}

rb_status rb_read_accums(rb_ctx* c, rb_accum* out, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return RB_ERR_INVALID_ARG;
    if (!c->allocated || c->cfg.pipeline == RB_PIPELINE_FLAT) return fail(c, RB_ERR_STATE, "no tree");
    static_assert(sizeof(rb_accum) == sizeof(rb::AccumI), "accumulator layout");
    RB_CUDA(c, cudaSetDevice(c->device));
    rb_status st = readCounters(c);
    if (st != RB_OK) return st;
    const uint32_t nn = c->hostCtr->numNodes;
    *count = nn;
    if (!out) return RB_OK;
    if (capacity < nn) return fail(c, RB_ERR_CAPACITY, "accumulator buffer too small");
    RB_CUDA(c, cudaMemcpy(out, c->d.accum, (size_t)nn * sizeof(rb_accum), cudaMemcpyDeviceToHost));
    return RB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ access
#include "rb_ctx_access.h"

namespace rb {

bool ctxRenderAccess(rb_ctx* c, CtxRenderAccess* out) {
    if (!c || !out) return false;
    out->d = c->d;
    out->stream = c->stream;
    out->device = c->device;
    out->numSMs = c->numSMs;
    out->pipeline = c->cfg.pipeline;
    out->maxNodes = c->cfg.max_nodes;
    out->drawlistCapacity = c->cfg.drawlist_capacity;
    out->allocated = c->allocated;
    out->hostRs = c->hostRs;
    out->evStart = c->evStart;
    out->evStop = c->evStop;
    return true;
}

void ctxSetError(rb_ctx* c, const char* msg) {
    if (c) c->err = msg ? msg : "";
}

void ctxNoteVisible(rb_ctx* c, uint32_t nodes, uint64_t samples) {
    if (!c) return;
    c->lastVisibleNodes = nodes;
    c->lastVisibleSamples = samples;
}

}  // namespace rb
