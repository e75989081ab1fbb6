/*
 * rb_capi.h -- the C ABI of the B200 progressive-LOD path.
 *
 * The reference drives its LOD pipelines through the C++ plugin interface
 * ILodPipeline (include/remo/ILodPipeline.h:118-146); each implementation
 * launches NVRTC-compiled kernels with positional void* argument arrays
 * (src/pipelines/RemolodPipeline.cpp:346-347, :403-405). This header is the
 * boundary that replaces those launches: plain C, POD structs, device pointers
 * as uint64_t, no C++ or torch types. The C++ host (remobench_b200/host/) keeps
 * the ILodPipeline interface and forwards to these entry points; Python binds
 * them with ctypes.
 *
 * Threading: a context is not thread-safe; calls are ordered on its stream.
 * Errors: every entry point returns rb_status; rb_last_error() has the text.
 * Device-side capacity limits never fault: they set flags in rb_stats.
 */
#ifndef RB_CAPI_H
#define RB_CAPI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RB_ABI_VERSION 2u

typedef int32_t rb_status;
enum {
    RB_OK = 0,
    RB_ERR_INVALID_ARG = 1,
    RB_ERR_CUDA = 2,          /* a CUDA call failed; the text names it */
    RB_ERR_OUT_OF_MEMORY = 3,
    RB_ERR_STATE = 4,         /* call out of order (e.g. build before allocate) */
    RB_ERR_RING = 5,          /* ring depth does not match (RemolodPipeline.cpp:315-328) */
    RB_ERR_CAPACITY = 6,      /* a request beyond a configured maximum */
    RB_ERR_NO_DEVICE = 7,
    RB_ERR_UNSUPPORTED = 8
};

/* Pipeline ids registered by the reference (src/shell/App.cpp:85-95). */
enum { RB_PIPELINE_REMOLOD = 0, RB_PIPELINE_SIMLOD = 1, RB_PIPELINE_FLAT = 2 };

/* Voxel representative rule. LOWEST_INDEX: the cell's colour comes from the
 * lowest global point index that reaches it in the batch (deterministic).
 * FIRST_COME: from whichever point arrives first, as the reference does
 * (kernels/remolod/remolod_octree.cu:116-138). */
enum { RB_VOXEL_LOWEST_INDEX = 0, RB_VOXEL_FIRST_COME = 1 };

/* Overflow flag bits reported in rb_stats.overflow_flags. */
enum {
    RB_OVF_SPILLED = 1u,   /* spill list full (remolod_octree.cu:76) */
    RB_OVF_BACKLOG = 2u,   /* new-voxel table full (:26) */
    RB_OVF_SPILLING = 4u,  /* spilling-node list full (:40) */
    RB_OVF_ARENA = 8u,     /* grid/chunk arena full */
    RB_OVF_TABLES = 64u,   /* chunk-table pool full */
    RB_OVF_DIRTY = 128u,   /* accumulate dirty list full */
    RB_OVF_DRAWLIST = 256u, /* render draw list full (remolod_render.cu:22) */
    RB_OVF_SYNC = 512u      /* a device-side grid barrier gave up waiting: an error, the build
                               call fails with RB_ERR_CUDA */
};

/* 16-byte point (include/remo/HostDeviceCommon.h:15-18): rgba with r in the low byte. */
typedef struct rb_point {
    float x, y, z;
    uint32_t color;
} rb_point;

/* Constants of kernels/remolod/remolod_structures.cuh:12-25 and
 * remolod_octree.cu:26-76 as run-time parameters. */
typedef struct rb_config {
    uint32_t struct_size;            /* sizeof(rb_config) */
    uint32_t pipeline;               /* RB_PIPELINE_* */
    int32_t device;                  /* CUDA device ordinal */
    uint32_t max_nodes;              /* 200000 */
    uint32_t max_points_per_node;    /* 50000 */
    uint32_t points_per_chunk;       /* 1000 */
    uint32_t max_expand_iters;       /* 20 */
    uint32_t ring_slots;             /* 50 */
    uint32_t slot_capacity;          /* 1000000 points per ring slot */
    uint32_t max_batches_per_build;  /* 20 */
    float time_budget_ms;            /* 10; 0 = none. Device time since the rb_build call began, checked before each batch */
    uint32_t voxel_mode;             /* RB_VOXEL_* */
    uint32_t accumulate;             /* fold Accumulate into every build (remolod) */
    uint32_t spilled_capacity;       /* 10,000,000 */
    uint32_t spilling_nodes_capacity;/* 100,000 */
    uint32_t drawlist_capacity;      /* 131072 */
    uint64_t safety_margin;          /* 200,000,000 bytes */
    uint32_t use_graphs;             /* 1: each batch is one CUDA graph launch, expand loop on the device; 0: host-driven loop */
    uint32_t backlog_capacity;       /* new voxel cells one batch can list (remolod_octree.cu:26 holds 10,000,000);
                                        0 = 2 x slot_capacity rounded up to a power of two. The cell table has
                                        twice as many 16-byte slots, so 10,000,000 takes 512 MB and misses L2
                                        more often than the default's 64 MB at 1M-point slots. A batch with more
                                        new cells keeps the first ones and sets RB_OVF_BACKLOG, as the reference
                                        does at its limit. */
    uint64_t store_capacity;         /* 0: the reference store's capacity is sized from the cloud and the
                                        budget as RemolodPipeline::allocate does (48 B/pt, 512 MB floor,
                                        RemolodPipeline.cpp:118-157); else exactly this many bytes, for a
                                        caller with its own sizing (ref_alloc's persistent size). The
                                        memory check (remolod_octree.cu:1181-1210) stops at offset +
                                        safety_margin >= store_capacity. */
    uint32_t refine_voxel_capacity;  /* voxels one rb_refine_colors call can filter; 0 = 2,097,152 */
    uint32_t reserved[3];
} rb_config;

/* CloudMeta (include/remo/PointSource.h:16-32), headless subset. */
typedef struct rb_cloud_meta {
    uint64_t num_points;
    float box_min[3];
    float box_max[3];
} rb_cloud_meta;

/* BatchView (include/remo/PointSource.h:43-67). slots is a device pointer to
 * num_slots * slot_capacity points; batch_sizes is host memory (num_slots
 * entries), read at the call. */
typedef struct rb_batch_view {
    uint64_t slots;
    const uint32_t* batch_sizes;
    uint32_t num_batches_uploaded;
    uint32_t slot_capacity;
    uint32_t num_slots;
    uint32_t num_batches_total;
} rb_batch_view;

/* SharedUniforms subset (include/remo/HostDeviceCommon.h:28-60). Matrices are
 * row-major: clip = M * (x, y, z, 1). */
typedef struct rb_frame {
    float width, height;
    float transform[16];
    float transform_frozen[16];
    float box_min[3], box_max[3];
    float lod_pixel_budget;          /* 128 (src/shell/App.h:50-62) */
    int32_t point_size;              /* 1 */
    uint32_t enable_edl;
    float edl_strength;              /* 0.4 */
    uint64_t frame_counter;
    int32_t color_mode;              /* RB_COLOR_* (SharedUniforms::colorMode) */
    uint32_t show_bounding_box;      /* draw the draw items' boxes after EDL (remo_lines.cuh:120-137) */
} rb_frame;

/* Sample colour modes (include/remo/HostDeviceCommon.h:63-66). */
enum { RB_COLOR_RGB = 0, RB_COLOR_BY_NODE = 1, RB_COLOR_BY_LOD = 2, RB_COLOR_WHITE = 3 };

typedef struct rb_build_result {
    uint32_t batches_consumed;       /* Stats::batchletIndex after the call */
    uint32_t batches_this_call;
    uint32_t more;                   /* batches remain in the cloud */
    uint32_t mem_capacity_reached;
    float device_ms;                 /* CUDA-event time of the call's GPU work */
    uint32_t pad;
} rb_build_result;

/* PipelineStats (include/remo/ILodPipeline.h:88-111) plus the reference's
 * Stats (kernels/simlod/HostDeviceInterface.h:51-76) and diagnostics. */
typedef struct rb_stats {
    uint64_t num_points;
    uint64_t num_voxels;
    uint64_t num_points_ingested;
    uint32_t num_nodes;
    uint32_t num_inner;
    uint32_t num_leaves;
    uint32_t num_nonempty_leaves;
    uint32_t max_depth;
    uint32_t max_points_per_node;
    uint32_t num_chunks_points;
    uint32_t num_chunks_voxels;
    uint32_t batchlet_index;
    uint32_t counter_underflows;
    uint64_t num_allocated_chunks;
    uint64_t chunk_pool_size;
    uint64_t persistent_offset;      /* the reference store's allocator offset */
    uint64_t persistent_capacity;
    uint64_t bytes_allocated;        /* device bytes this context holds */
    uint64_t dropped_points;
    uint64_t expand_iters;
    uint64_t nodes_split;
    uint64_t spilled_points;
    uint32_t num_grids;
    uint32_t overflow_flags;         /* RB_OVF_* */
    uint32_t mem_capacity_reached;
    uint32_t node_capacity_reached;
    uint32_t num_visible_nodes;      /* last render */
    uint32_t pad;
    uint64_t num_visible_samples;
} rb_stats;

typedef struct rb_render_result {
    uint32_t draw_items;
    uint32_t drawlist_overflow;
    uint64_t draw_samples;
    float device_ms;
    uint32_t pad;
} rb_render_result;

/* AccumGlobals (include/remo/RemoAccum.h:33-41). */
typedef struct rb_accum_globals {
    uint64_t morton_watermark;
    uint64_t num_accumulated;
    uint64_t sum_leaf_counts;
    uint32_t points_folded;
    uint32_t num_leaves_folded;
    uint32_t inner_with_sums;
    uint32_t pad;
} rb_accum_globals;

/* Exact per-node sums (NodeAccum, include/remo/RemoAccum.h:24-31, in integers):
 * s1 = Σq, s2 = Σqqᵀ as 128-bit (xx xy xz yy yz zz), c1/c2 = Σ and Σ² of the
 * 8-bit r, g, b channels; q is the point's 28-bit octree coordinate relative to
 * the node, clamped to [0, 2^(28-level)]. */
typedef struct rb_accum {
    uint64_t s1[3];
    uint64_t s2_lo[6];
    uint64_t s2_hi[6];
    uint64_t c1[3];
    uint64_t c2[3];
    uint32_t count;                  /* watermark: slots folded so far */
    uint32_t last_touched_batch;
    uint32_t state;
    uint32_t pad;
} rb_accum;

/* One node of the pool, for parity dumps. */
typedef struct rb_node_info {
    int32_t child[8];
    uint32_t counter;
    uint32_t num_points;
    uint32_t level;
    uint32_t X, Y, Z;
    uint32_t has_grid;
    uint32_t num_voxels;
    uint32_t num_point_chunks;
    uint32_t num_voxel_chunks;
    uint32_t is_leaf;
} rb_node_info;

/* Per-kernel launch counts (always kept) and CUDA-event durations (kept
 * while profiling is on; each launch is bracketed by events on the context's
 * stream, so leave it off for timing whole calls). No reference counterpart:
 * the reference times phases with %globaltimer marks inside its cooperative
 * kernel (kernels/shared/remo_prelude.cuh:58-85). */
typedef struct rb_kernel_profile {
    char name[32];
    uint64_t launches;
    uint64_t timed_launches;
    double total_ms;
    uint64_t units;                  /* points (or pixels) handed to the kernel */
} rb_kernel_profile;

uint32_t rb_abi_version(void);
const char* rb_status_string(rb_status s);
void rb_config_defaults(rb_config* cfg);

/* Construction (no device allocation: ILodPipeline::initPrograms "must NOT
 * allocate", wiki/01_Overview.md:142-160) and teardown. */
rb_status rb_create(const rb_config* cfg, struct rb_ctx** out);
void rb_destroy(struct rb_ctx* ctx);
const char* rb_last_error(const struct rb_ctx* ctx);
rb_status rb_set_stream(struct rb_ctx* ctx, void* cuda_stream);

/* ILodPipeline::allocate / release (RemolodPipeline.cpp:105-212): sizes the
 * node pool, arena and scratch from the cloud and the byte budget. */
rb_status rb_allocate(struct rb_ctx* ctx, const rb_cloud_meta* meta, uint64_t budget_bytes);
void rb_release(struct rb_ctx* ctx);

/* ILodPipeline::reset + the reset kernel (kernels/remolod/remolod_reset.cu:23-87). */
rb_status rb_reset(struct rb_ctx* ctx);

/* ILodPipeline::build for the progressive pipelines (RemolodPipeline.cpp:296-438):
 * consumes up to max_batches_per_build uploaded batches from the ring within
 * the time budget, then (remolod) runs Accumulate. */
rb_status rb_build(struct rb_ctx* ctx, const rb_batch_view* view, rb_build_result* out);

/* End-to-end ingest of host points: streams them through a device ring with
 * copies overlapped on a second stream, n points in batches of batch_size
 * (<= slot_capacity), Accumulate after the last batch. */
rb_status rb_ingest_host(struct rb_ctx* ctx, const rb_point* points, uint64_t n, uint32_t batch_size,
                         rb_build_result* out);

/* kernel_accumulate + kernel_accum_verify (remolod_accum.cu:47-233). */
rb_status rb_accumulate(struct rb_ctx* ctx, uint32_t batch_index, rb_accum_globals* out);

/* ILodPipeline::render (RemolodPipeline.cpp:559-601) into a headless device
 * framebuffer: fb_dev holds width*height uint64 (depth<<32 | rgba); rgba_dev
 * (optional, 0 = none) receives the resolved colours. force_large_dev
 * (optional) marks nodes the LOD cut must open (Refinement). */
rb_status rb_render(struct rb_ctx* ctx, const rb_frame* frame, uint64_t fb_dev, uint64_t rgba_dev,
                    uint64_t force_large_dev, rb_render_result* out);

/* rb_render without any allocation; it has no counterpart in the reference.
 * It is for callers that build the tree ahead of time but must render where
 * they cannot allocate: a frame callback with a hard real-time budget that may
 * not take the allocator's lock or risk an allocation failure mid-frame, or an
 * embedder whose own pool owns all device memory after start-up. It calls no
 * cudaMalloc/cudaFree; its scratch (per-node flags, the draw list, three
 * counters) is a static device array of about 1 MB. rb_allocate resolves the
 * array's device address (cudaGetSymbolAddress, with the context's device
 * current), which under lazy module loading is also when the array is
 * reserved on that device; it stays reserved until the process exits, so
 * every rb_render_noalloc call is allocation-free. Limits: max_nodes <= 262144
 * and drawlist_capacity <= 131072, else RB_ERR_CAPACITY. Calls share the
 * array: calls that overlap on the GPU race. The caller's current device is
 * restored before return. A context allocated before a cudaDeviceReset must
 * not be used after it. Output equals rb_render's. */
rb_status rb_render_noalloc(struct rb_ctx* ctx, const rb_frame* frame, uint64_t fb_dev, uint64_t rgba_dev,
                            uint64_t force_large_dev, rb_render_result* out);

/* The flat pipeline (kernels/flat/flat_render.cu:9-76): every point of a
 * resident cloud. */
rb_status rb_render_flat(struct rb_ctx* ctx, const rb_frame* frame, uint64_t points_dev, uint64_t n,
                         uint64_t fb_dev, uint64_t rgba_dev, rb_render_result* out);

/* ILodPipeline::stats (+ the stats sweep, remolod_octree.cu:1271-1310). */
rb_status rb_read_stats(struct rb_ctx* ctx, rb_stats* out);

/* Parity dumps. */
rb_status rb_read_nodes(struct rb_ctx* ctx, rb_node_info* out, uint32_t capacity, uint32_t* count);
rb_status rb_read_node_points(struct rb_ctx* ctx, uint32_t node, rb_point* pts, uint32_t* idx,
                              uint32_t capacity, uint32_t* count);
rb_status rb_read_node_voxels(struct rb_ctx* ctx, uint32_t node, rb_point* vox, uint32_t capacity,
                              uint32_t* count);
rb_status rb_read_node_grid(struct rb_ctx* ctx, uint32_t node, uint32_t* words65536);
rb_status rb_read_accums(struct rb_ctx* ctx, rb_accum* out, uint32_t capacity, uint32_t* count);

/* Analysis (no reference kernel; wiki/02_KernelPipeline.md:204-224 describes
 * it): exact roll-up of the leaf sums, centred covariance, 3x3 eigen-solve,
 * surface variation and planarity x screen coverage, per-frame priority queue. */
typedef struct rb_analysis_params {
    uint32_t min_points;       /* nodes with fewer points score 0 (16) */
    uint32_t closure_margin;   /* batches without new points before a node is closed (8) */
    uint32_t frontier_only;    /* queue only nodes Refinement can open (1) */
    uint32_t queue_capacity;   /* top-K kept (<= 16384) */
    float pixel_budget;        /* the LOD cut's budget, to find the frontier (128) */
    uint32_t score_mode;       /* RB_SCORE_* */
} rb_analysis_params;

/* How Refinement ranks the frontier. PARTIAL: the current (partial) surface
 * variation; CLOSED: closure-lagged -- only closed nodes score, the plain
 * method; LEARNED: closed nodes by their surface variation, open nodes by
 * their partial one plus the learned scorer's predicted correction. */
enum { RB_SCORE_PARTIAL = 0, RB_SCORE_CLOSED = 1, RB_SCORE_LEARNED = 2 };

typedef struct rb_analysis_result {
    uint32_t queue_length;
    uint32_t eligible;         /* nodes with a positive score that may enter the queue */
    uint32_t fp64_branch;      /* eigen-solves that took the FP64 near-degenerate branch */
    uint32_t overflow;         /* more tied candidates than the queue sort holds */
    float device_ms;
    uint32_t pad;
} rb_analysis_result;

typedef struct rb_node_analysis {
    float eig[3];              /* descending, units of (node size)^2 */
    float normal[3];           /* eigenvector of eig[2] */
    float surface_variation;   /* eig[2] / sum */
    float planarity;           /* (eig[1] - eig[2]) / eig[0] */
    float coverage;            /* fraction of the frame under the node's projected box */
    float score;               /* surface variation x coverage */
    uint64_t count;            /* points in the subtree */
    uint32_t last_touched;     /* newest batch index that added points to the subtree */
    uint32_t closed;
    uint32_t flags;            /* 1: FP64 branch, 2: large, 4: frontier */
    uint32_t pad;
} rb_node_analysis;

rb_status rb_analyze(struct rb_ctx* ctx, const rb_frame* frame, const rb_analysis_params* params,
                     rb_analysis_result* out);
rb_status rb_read_analysis(struct rb_ctx* ctx, rb_node_analysis* out, uint32_t capacity, uint32_t* count);
rb_status rb_read_queue(struct rb_ctx* ctx, uint32_t* node_ids, uint32_t capacity, uint32_t* count);
/* Exact rolled sums per node: n, s1[3], s2 as (lo, hi) x 6 -- 16 uint64 per node. */
rb_status rb_read_rollup(struct rb_ctx* ctx, uint64_t* out16, uint32_t capacity, uint32_t* count);

/* Refinement, minimal budgeted form (wiki/02_KernelPipeline.md:228-243 lists
 * the passes; this is the budget consumer): the first `budget` nodes of the
 * last Analysis queue are written as 1 into the node mask at mask_dev (one
 * byte per node), which rb_render takes as force_large_dev. */
rb_status rb_refine(struct rb_ctx* ctx, uint32_t budget, uint64_t mask_dev);

/* Refinement's colour filtering (wiki/02_KernelPipeline.md:232, "average
 * colour across a node's samples"; the reference lists it, unbuilt): for the
 * first `budget` nodes of the last Analysis queue, in queue order while their
 * voxels fit refine_voxel_capacity, each voxel's colour becomes the mean
 * colour of the subtree's points that fall in its cell (per 8-bit channel,
 * rounded half up; alpha kept). The sums are kept only for the voxels being
 * filtered, keyed by (node, cell) -- the sparse accumulator the reference's
 * notes ask for instead of a dense per-node colour grid. */
typedef struct rb_refine_result {
    uint32_t nodes_filtered;   /* queue prefix taken */
    uint32_t voxels_filtered;
    uint64_t points_visited;   /* (point, filtered ancestor) pairs summed */
} rb_refine_result;
rb_status rb_refine_colors(struct rb_ctx* ctx, uint32_t budget, rb_refine_result* out);

/* Refinement's deepening (wiki/02_KernelPipeline.md:228-243, "local split and
 * redistribute"; the reference lists it, unbuilt): among the first `budget`
 * nodes of the last Analysis queue, every leaf above the deepest level
 * (level < 20) holding at least min_points points (0 counts as 1) is split as doSplitting splits a spilling node
 * (remolod_octree.cu:303-400): in increasing id, 8 consecutive ids each, a
 * grid (allocated once, zeroed), its points to the new children and its
 * chunks back to the queue. Voxel sampling then gives the deepened node its
 * voxels (the lowest global point index per cell) and insertion places the
 * points. The node pool guard refuses a split once fewer than 8 ids remain
 * and raises the node-pool flag, as a batch does; the memory check of a
 * batch refuses the whole pass (stopped, memCapacityReached). No batch is
 * consumed. Accumulate runs after it when the pipeline has Accumulate. The
 * Analysis queue is stale afterwards: call rb_analyze before the next
 * refinement call. */
typedef struct rb_deepen_result {
    uint32_t nodes_selected;   /* queue leaves with at least min_points points */
    uint32_t nodes_split;      /* splits made, the selected leaves the pool had room for first */
    uint32_t nodes_refused;    /* selected leaves the node pool had no room for */
    uint32_t stopped;          /* 1: the memory check refused the pass */
    uint64_t points_moved;     /* stored points redistributed to the new children */
    uint64_t voxels_made;      /* new voxels sampled for the deepened nodes */
} rb_deepen_result;
rb_status rb_refine_deepen(struct rb_ctx* ctx, uint32_t budget, uint32_t min_points, rb_deepen_result* out);

/* Refinement's collapsing (wiki/02_KernelPipeline.md:228-243, "merge a node
 * back up"; the reference lists it, unbuilt, since it needs a grid pool,
 * CLAUDE.md:185-187). Among the `count` node ids at nodes (host memory, at
 * most 4096; duplicates ignored), every node below the root whose eight
 * children are all leaves holding at most max_points points together (0: the
 * split limit) becomes a leaf again with all their points. Its chunks are
 * allocated first, then the children's chunks return to the queue; the
 * children stay as empty leaves nothing points to (node ids are not reused);
 * the node drops its voxels and returns its grid to a pool that later splits
 * take grids from before the arena. No batch is consumed; Accumulate runs
 * after it (remolod); an Analysis queue is stale afterwards. */
typedef struct rb_collapse_result {
    uint32_t nodes_collapsed;
    uint32_t grids_returned;
    uint64_t points_moved;     /* points now held by the merged leaves */
    uint64_t voxels_dropped;   /* voxels the merged nodes held */
} rb_collapse_result;
rb_status rb_refine_collapse(struct rb_ctx* ctx, const uint32_t* nodes, uint32_t count, uint32_t max_points,
                             rb_collapse_result* out);

/* The learned scorer (no reference counterpart: plans/04_NeuralPass.md is
 * empty): a 16 -> 64 -> 64 -> 2 MLP, GELU, BF16 weights and activations, FP32
 * accumulation, trained on the GPU with these entry points. Inputs are the 16
 * per-node features rb_analyze logs (rb_read_features); outputs are the
 * predicted change from the partial to the final surface variation (x 300)
 * and a closure logit. Parameters are
 * RB_MLP_NUM_PARAMS floats: W1[64][16], b1[64], W2[64][64], b2[64], W3[2][64], b3[2]. */
#define RB_MLP_NUM_PARAMS 5378
#define RB_NUM_FEATURES 16
rb_status rb_read_features(struct rb_ctx* ctx, float* out16, uint32_t capacity, uint32_t* count);
rb_status rb_mlp_init(struct rb_ctx* ctx, uint64_t seed);
rb_status rb_mlp_set_params(struct rb_ctx* ctx, const float* params);   /* also restarts Adam */
rb_status rb_mlp_get_params(struct rb_ctx* ctx, float* params);
/* y_dev[2 n] = network(x_dev[16 n]); device pointers. */
rb_status rb_mlp_predict(struct rb_ctx* ctx, uint64_t x_dev, uint32_t n, uint64_t y_dev);
/* Gradient of the mean loss over n samples (targets t_dev[2 n]) into grad
 * (host, RB_MLP_NUM_PARAMS floats), mean loss into *loss; no update. */
rb_status rb_mlp_gradients(struct rb_ctx* ctx, uint64_t x_dev, uint64_t t_dev, uint32_t n, float* grad,
                           float* loss);
/* One Adam step on n samples; *loss (optional) receives the batch's mean loss. */
rb_status rb_mlp_train_step(struct rb_ctx* ctx, uint64_t x_dev, uint64_t t_dev, uint32_t n, float lr,
                            float* loss);

/* Kernel timing (see rb_kernel_profile). */
rb_status rb_set_profiling(struct rb_ctx* ctx, int on);
rb_status rb_read_profile(struct rb_ctx* ctx, rb_kernel_profile* out, uint32_t capacity, uint32_t* count);
rb_status rb_reset_profile(struct rb_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif
