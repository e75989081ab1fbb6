// Internal read access to a context for entry points that live outside
// rb_capi.cu (the allocation-free render in rb_noalloc.cu). Not part of the ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb_state.h"

struct rb_ctx;

namespace rb {

struct RenderScratch;

struct CtxRenderAccess {
    Dev d;                     // the tree (device pointers, capacities)
    cudaStream_t stream;
    int device;
    int numSMs;
    uint32_t pipeline;
    uint32_t maxNodes;
    uint32_t drawlistCapacity;
    bool allocated;
    RenderScratch* hostRs;     // pinned, allocated by rb_allocate
    cudaEvent_t evStart, evStop;
};

// Fills `out` from the context; false when ctx is null.
bool ctxRenderAccess(rb_ctx* ctx, CtxRenderAccess* out);
// Records an error message for rb_last_error.
void ctxSetError(rb_ctx* ctx, const char* msg);
// Records the last render's visible node and sample counts for rb_read_stats.
void ctxNoteVisible(rb_ctx* ctx, uint32_t nodes, uint64_t samples);
// Resolves the allocation-free render's static scratch on `device` (which must
// be current); rb_allocate calls it so that rb_render_noalloc never loads a
// module or reserves memory itself (rb_noalloc.cu).
cudaError_t noallocPrepare(int device);

}  // namespace rb
