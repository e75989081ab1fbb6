// rb_render_noalloc: the LOD render of rb_render without any device or host
// allocation.
//
// Who needs it: a caller that builds the tree up front and then renders from a
// place where it must not allocate -- a frame callback with a hard real-time
// budget that cannot take the allocator's lock or risk an allocation failure
// mid-frame, or an embedder that hands all device memory to its own pool after
// start-up, so that a later cudaMalloc would fail. rb_render keeps its scratch
// in the context and, when EDL is on, allocates a full-frame copy on first use;
// this entry point does neither.
//
// Its scratch -- per-node visible/large flags, the draw list and the three
// counters -- is one file-scope __device__ array of kScratchBytes (about 1 MB),
// which every GPU that loads this library holds until the process exits. Host
// code cannot use the array's name as a device address (on the host it names
// a host-side stand-in), so the first call on each device, with that device
// current, asks the runtime for the array's device address with
// cudaGetSymbolAddress and keeps it. Make that first call before any stream
// capture. All calls share the array and it keeps the last call's contents:
// the counters are cleared by the first kernel of every call, and the flags and
// the draw list are written before they are read. Calls that overlap on the
// GPU (two streams, two contexts on one device) race on the array.
//
// EDL is applied in place: it changes only the colour half of each pixel and
// reads only the depth half of its neighbours, so the result equals
// rb_render's, which shades from a copy.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/rb_capi.h"
#include "rb_ctx_access.h"
#include "rb_kernels.h"
#include "rb_state.h"

namespace {

constexpr uint32_t kNoAllocMaxNodes = 262144;  // two flag bytes per node
constexpr uint32_t kNoAllocMaxItems = 131072;  // draw list entries (the reference's capacity)
constexpr size_t kOffVis = 0;
constexpr size_t kOffLarge = kOffVis + kNoAllocMaxNodes;
constexpr size_t kOffItems = kOffLarge + kNoAllocMaxNodes;
constexpr size_t kOffCounters = kOffItems + (size_t)kNoAllocMaxItems * sizeof(uint32_t);
constexpr size_t kScratchBytes = kOffCounters + 256;
static_assert(kOffItems % 16 == 0 && kOffCounters % 256 == 0, "scratch layout alignment");
static_assert(sizeof(rb::RenderScratch) <= 256, "counter block must fit its slot");

static __device__ __align__(256) unsigned char g_renderScratch[kScratchBytes];

constexpr int kMaxDevices = 128;
std::mutex g_scratchMutex;
unsigned char* g_scratchAddr[kMaxDevices] = {};

// The array's device address on `device`, which must be current.
rb_status scratchAddress(rb_ctx* ctx, int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) {
        rb::ctxSetError(ctx, "rb_render_noalloc: device ordinal out of range");
        return RB_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    if (!g_scratchAddr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_renderScratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            rb::ctxSetError(ctx, (std::string("rb_render_noalloc: cudaGetSymbolAddress failed: ") +
                                  cudaGetErrorString(e)).c_str());
            return RB_ERR_CUDA;
        }
        g_scratchAddr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratchAddr[device];
    return RB_OK;
}

rb_status cudaFail(rb_ctx* ctx, const char* what, cudaError_t e) {
    rb::ctxSetError(ctx, (std::string("rb_render_noalloc: ") + what + ": " + cudaGetErrorString(e)).c_str());
    return RB_ERR_CUDA;
}

}  // namespace

extern "C" rb_status rb_render_noalloc(rb_ctx* ctx, const rb_frame* f, uint64_t fbDev, uint64_t rgbaDev,
                                       uint64_t forceDev, rb_render_result* out) {
    if (!ctx || !f || !fbDev) return RB_ERR_INVALID_ARG;
    rb::CtxRenderAccess a;
    if (!rb::ctxRenderAccess(ctx, &a)) return RB_ERR_INVALID_ARG;
    if (!a.allocated || a.pipeline == RB_PIPELINE_FLAT) {
        rb::ctxSetError(ctx, "rb_render_noalloc: no tree to render");
        return RB_ERR_STATE;
    }
    if (!(f->width >= 1.0f && f->height >= 1.0f)) {
        rb::ctxSetError(ctx, "rb_render_noalloc: empty frame");
        return RB_ERR_INVALID_ARG;
    }
    if (a.maxNodes > kNoAllocMaxNodes) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "rb_render_noalloc: the context's max_nodes (%u) exceeds this entry point's limit of %u",
                      a.maxNodes, kNoAllocMaxNodes);
        rb::ctxSetError(ctx, msg);
        return RB_ERR_CAPACITY;
    }
    const uint32_t cap = a.drawlistCapacity ? a.drawlistCapacity : 1u;
    if (cap > kNoAllocMaxItems) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "rb_render_noalloc: the context's drawlist_capacity (%u) exceeds this entry point's limit of %u",
                      cap, kNoAllocMaxItems);
        rb::ctxSetError(ctx, msg);
        return RB_ERR_CAPACITY;
    }
    cudaError_t e = cudaSetDevice(a.device);
    if (e != cudaSuccess) return cudaFail(ctx, "cudaSetDevice", e);
    unsigned char* base = nullptr;
    rb_status st = scratchAddress(ctx, a.device, &base);
    if (st != RB_OK) return st;
    uint8_t* vis = base + kOffVis;
    uint8_t* large = base + kOffLarge;
    uint32_t* items = reinterpret_cast<uint32_t*>(base + kOffItems);
    rb::RenderScratch* rs = reinterpret_cast<rb::RenderScratch*>(base + kOffCounters);

    const uint64_t npx = (uint64_t)f->width * (uint64_t)f->height;
    auto* fb = reinterpret_cast<unsigned long long*>(fbDev);
    rb::Frame fr;
    fr.width = f->width;
    fr.height = f->height;
    std::memcpy(fr.transform, f->transform, sizeof(fr.transform));
    std::memcpy(fr.transformFrozen, f->transform_frozen, sizeof(fr.transformFrozen));
    for (int k = 0; k < 3; k++) {
        fr.boxMin[k] = f->box_min[k];
        fr.boxMax[k] = f->box_max[k];
    }
    fr.lodPixelBudget = f->lod_pixel_budget;
    fr.pointSize = f->point_size;

    cudaStream_t s = a.stream;
    if ((e = cudaEventRecord(a.evStart, s)) != cudaSuccess) return cudaFail(ctx, "cudaEventRecord", e);
    rb::launchFbClear(fb, npx, a.numSMs * 8, s);
    // the first kernel zeroes the counter block (draw items, overflow, samples)
    rb::launchNodeFlags(a.d, fr, vis, large, reinterpret_cast<const uint8_t*>(forceDev), rs, a.numSMs * 4, s);
    rb::launchFrontier(a.d, vis, large, rs, items, cap, a.numSMs * 4, s);
    rb::launchRaster(a.d, fr, fb, rs, items, cap, a.numSMs * 8, s);
    if (f->enable_edl) rb::launchEdl(fb, fb, (uint32_t)f->width, (uint32_t)f->height, f->edl_strength,
                                     a.numSMs * 8, s);
    if (rgbaDev) rb::launchResolve(fb, reinterpret_cast<uint32_t*>(rgbaDev), npx, a.numSMs * 8, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return cudaFail(ctx, "kernel launch", e);
    if ((e = cudaEventRecord(a.evStop, s)) != cudaSuccess) return cudaFail(ctx, "cudaEventRecord", e);
    if ((e = cudaMemcpyAsync(a.hostRs, rs, sizeof(rb::RenderScratch), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cudaFail(ctx, "cudaMemcpyAsync", e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cudaFail(ctx, "cudaStreamSynchronize", e);
    rb::ctxNoteVisible(ctx, a.hostRs->numItems, a.hostRs->samples);
    if (out) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a.evStart, a.evStop);
        out->draw_items = a.hostRs->numItems;
        out->drawlist_overflow = a.hostRs->overflow;
        out->draw_samples = a.hostRs->samples;
        out->device_ms = ms;
        out->pad = 0;
    }
    return RB_OK;
}
