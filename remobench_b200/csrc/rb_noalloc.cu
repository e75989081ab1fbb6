// rb_render_noalloc: the LOD render of rb_render without any device or host
// allocation.
//
// Who needs it: a caller that builds the tree up front and then renders from a
// place where it must not allocate -- a frame callback with a hard real-time
// budget that cannot take the allocator's lock or risk an allocation failure
// mid-frame, or an embedder that hands all device memory to its own pool after
// start-up, so that a later cudaMalloc would fail. rb_render renders through
// per-context scratch that rb_allocate allocates with the tree; this entry
// point needs none of it.
//
// Its scratch -- per-node visible/large flags, the draw list and the three
// counters -- is one file-scope __device__ array of kScratchBytes (about 1 MB).
// Host code cannot use the array's name as a device address (on the host it
// names a host-side stand-in), so rb_allocate, with the context's device
// current, asks the runtime for the array's device address with
// cudaGetSymbolAddress and keeps it per device (noallocPrepare below). Under
// lazy module loading that lookup is also what loads this file's module and
// reserves the array on the device, so the reservation happens inside
// rb_allocate -- where allocation is expected -- and every rb_render_noalloc
// call afterwards is allocation-free. The array then stays reserved on that
// device until the process exits. Every rb_allocate looks the address up again,
// so a context allocated after a cudaDeviceReset gets the reloaded module's
// address; a context allocated before a reset must not be used after it.
//
// All calls share the array and it keeps the last call's contents: the
// counters are cleared by the first kernel of every call, and the flags and
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

// Looks the array's device address up on `device`, which must be current,
// and keeps it. Called by rb_allocate (see noallocPrepare).
cudaError_t resolveScratch(int device) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_renderScratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        return e != cudaSuccess ? e : cudaErrorInvalidSymbol;
    }
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    g_scratchAddr[device] = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

// The address rb_allocate resolved for `device`, or null.
unsigned char* scratchAddress(int device) {
    if (device < 0 || device >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    return g_scratchAddr[device];
}

rb_status cudaFail(rb_ctx* ctx, const char* what, cudaError_t e) {
    rb::ctxSetError(ctx, (std::string("rb_render_noalloc: ") + what + ": " + cudaGetErrorString(e)).c_str());
    return RB_ERR_CUDA;
}

}  // namespace

namespace rb {

cudaError_t noallocPrepare(int device) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    return resolveScratch(device);
}

}  // namespace rb

namespace {

// The render itself, with the context's device current.
rb_status renderNoalloc(rb_ctx* ctx, const rb::CtxRenderAccess& a, unsigned char* base, const rb_frame* f,
                        uint64_t fbDev, uint64_t rgbaDev, uint64_t forceDev, uint32_t cap, rb_render_result* out) {
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
    fr.colorMode = f->color_mode;
    fr.showBoundingBox = f->show_bounding_box;

    cudaError_t e;
    cudaStream_t s = a.stream;
    if ((e = cudaEventRecord(a.evStart, s)) != cudaSuccess) return cudaFail(ctx, "cudaEventRecord", e);
    rb::launchFbClear(fb, npx, a.numSMs * 8, s);
    // the first kernel zeroes the counter block (draw items, overflow, samples)
    rb::launchNodeFlags(a.d, fr, vis, large, reinterpret_cast<const uint8_t*>(forceDev), rs, a.numSMs * 4, s);
    rb::launchFrontier(a.d, vis, large, rs, items, cap, a.numSMs * 4, s);
    rb::launchRaster(a.d, fr, fb, rs, items, cap, a.numSMs * 8, s);
    if (f->enable_edl) rb::launchEdl(fb, fb, (uint32_t)f->width, (uint32_t)f->height, f->edl_strength,
                                     a.numSMs * 8, s);
    if (f->show_bounding_box) rb::launchWireframe(a.d, fr, fb, rs, items, cap, a.numSMs * 8, s);
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
    unsigned char* base = scratchAddress(a.device);
    if (!base) {
        rb::ctxSetError(ctx, "rb_render_noalloc: the scratch array's address was not resolved; rb_allocate does it");
        return RB_ERR_STATE;
    }
    // the caller's current device is put back on every return
    int callerDevice = -1;
    cudaError_t e = cudaGetDevice(&callerDevice);
    if (e != cudaSuccess) return cudaFail(ctx, "cudaGetDevice", e);
    if (callerDevice != a.device && (e = cudaSetDevice(a.device)) != cudaSuccess)
        return cudaFail(ctx, "cudaSetDevice", e);
    const rb_status st = renderNoalloc(ctx, a, base, f, fbDev, rgbaDev, forceDev, cap, out);
    if (callerDevice != a.device) cudaSetDevice(callerDevice);
    return st;
}
