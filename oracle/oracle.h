/*
 * CPU oracle for the progressive LOD hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A single-threaded, deterministic C restatement of the reference pipeline's
 * Update (kernels/remolod/remolod_octree.cu:95-1320 with the allocator rules of
 * kernels/simlod/utils.h.cu:185-312), the reference's FP64 Accumulate
 * (kernels/remolod/remolod_accum.cu:47-233), the exact-integer Accumulate this
 * project specifies in its place, Analysis, and Rasterize
 * (kernels/remolod/remolod_render.cu:30-198, kernels/shared/remo_*.cuh).
 *
 * It is the checker the CUDA path is compared against. Only tests, the smoke
 * entry point and the benchmark's CPU-baseline arm may load it; the product
 * never links it. See each function for the reference lines it follows.
 *
 * Parity pinning: the reference ships no tests, fixtures or golden vectors for
 * this path (its only structural pins are on lidar files that are not
 * distributed), so this restatement is pinned against the reference's own
 * invariants, against hand-computed cases, and against outputs of the
 * reference's own kernels run on a B200 (tests/golden/ref_config1_*.npz, made
 * by tests/golden/make_ref_fixtures.py; checked in tests/test_ref_pin.py).
 */
#ifndef RB_ORACLE_H
#define RB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_point {
    float x, y, z;
    uint32_t color;
} or_point;

typedef struct or_config {
    uint32_t max_nodes;              /* 200000 (remolod_structures.cuh:14) */
    uint32_t max_points_per_node;    /* 50000 (:12) */
    uint32_t points_per_chunk;       /* 1000 (:15) */
    uint32_t max_expand_iters;       /* 20 (remolod_octree.cu:411) */
    uint64_t persistent_capacity;    /* bytes of the reference-equivalent store */
    uint64_t safety_margin;          /* 200,000,000 (remolod_octree.cu:1195) */
    uint32_t ring_slots;             /* 50 (remolod_structures.cuh:25) */
    uint32_t slot_capacity;          /* 1,000,000 (remolod_octree.cu:1167) */
    uint32_t max_batches_per_build;  /* 20 (remolod_octree.cu:1169) */
    uint32_t num_threads;            /* >1: multithreaded CPU builder (same result) */
} or_config;

typedef struct or_node_info {
    int32_t child[8];        /* -1: none */
    uint32_t counter;
    uint32_t num_points;
    uint32_t level;
    uint32_t X, Y, Z;
    int32_t grid;            /* -1: none */
    uint32_t num_voxels;
    uint32_t num_point_chunks;
    uint32_t num_voxel_chunks;
    uint32_t is_leaf;
} or_node_info;

typedef struct or_stats {
    uint32_t num_nodes, num_inner, num_leaves, num_nonempty_leaves;
    uint64_t num_points, num_voxels;
    uint32_t num_chunks_points, num_chunks_voxels;
    uint32_t batchlet_index;
    uint64_t num_points_processed;
    uint64_t num_allocated_chunks, chunk_pool_size;
    uint64_t persistent_offset;      /* reference-equivalent AllocatorGlobal offset */
    uint32_t mem_capacity_reached;
    uint32_t node_pool_overflow;
    uint32_t max_points_per_node;
    uint32_t counter_underflows;
    uint64_t dropped_points;         /* inserted into a leaf that holds no chunk */
    uint64_t expand_iters, nodes_split, spilled_points;
    uint32_t num_grids;
    uint32_t overflow_flags;         /* OR_OVERFLOW_* */
} or_stats;

#define OR_OVERFLOW_SPILLED 1u   /* more than 10M spilled points in a batch */
#define OR_OVERFLOW_BACKLOG 2u   /* more than 10M new voxels in a batch */
#define OR_OVERFLOW_SPILLING 4u  /* more than 100k spilling nodes in an iteration */

typedef struct or_tree or_tree;
typedef struct or_frame or_frame;

or_tree* or_create(const or_config* cfg);
void or_destroy(or_tree* t);

/* remolod_reset.cu:23-87: root node, root grid, allocator offset 16. */
void or_reset(or_tree* t, const float box_min[3], const float box_max[3]);

/* One batch through addBatch (remolod_octree.cu:940-1060). Returns 1 when the
 * memory check (remolod_octree.cu:1181-1210) refused the batch, else 0. */
int or_add_batch(or_tree* t, const or_point* pts, uint32_t n);
/* Refinement's deepening: the leaves among nodes[0..n) with at least
 * min_points points split and their points redistributed, as a batch with no
 * points whose spilling nodes they are. Returns 1 when the memory check
 * refuses it; *selected: the leaves taken. */
int or_deepen(or_tree* t, const uint32_t* nodes, uint32_t n, uint32_t min_points, uint32_t* selected);
/* Refinement's collapsing: each listed node whose children are all leaves
 * holding at most max_points points (0: the split limit) becomes a leaf with
 * their points; its grid goes to a pool later splits take from. */
int or_collapse(or_tree* t, const uint32_t* nodes, uint32_t n, uint32_t max_points, uint32_t* collapsed,
                uint64_t* points, uint64_t* voxels);

/* kernel_construct's batch loop over a ring (remolod_octree.cu:1169-1241),
 * without the wall-clock budget, then the stats sweep (:1271-1310). */
uint32_t or_build(or_tree* t, const or_point* ring, const uint32_t* batch_sizes,
                  uint32_t num_uploaded);

/* The stats sweep alone. */
void or_sweep(or_tree* t);

void or_get_stats(const or_tree* t, or_stats* s);
uint32_t or_num_nodes(const or_tree* t);
int or_get_node(const or_tree* t, uint32_t i, or_node_info* out);
/* points stored in leaf i (storage order) and their global point indices */
uint32_t or_leaf_points(const or_tree* t, uint32_t i, const or_point** pts, const uint32_t** idx);
/* voxels stored in node i */
uint32_t or_node_voxels(const or_tree* t, uint32_t i, const or_point** vox);
/* the node's 128^3 occupancy bits (65536 words) or NULL */
const uint32_t* or_node_grid(const or_tree* t, uint32_t i);

/* ---------------------------------------------------------- Accumulate */

/* Exact integer sums on node-local coordinates: q = clamp(P - (N << (28-L)), 0,
 * 2^(28-L)) per axis, P the point's 28-bit coordinate and N the node's
 * coordinate at its level L. s1 = sum q (u64), s2 = sum q q^T as 128-bit
 * (xx, xy, xz, yy, yz, zz; lo/hi words), colour sums of 8-bit channels. */
typedef struct or_accum_i {
    uint64_t s1[3];
    uint64_t s2_lo[6];
    uint64_t s2_hi[6];
    uint64_t c1[3];
    uint64_t c2[3];
    uint32_t count;
    uint32_t last_touched_batch;
    uint32_t state;
    uint32_t pad;
} or_accum_i;

/* The reference's double/float sums (remolod_accum.cu:103-208, RemoAccum.h:24-31). */
typedef struct or_accum_f {
    double g[9];
    float c[6];
    uint32_t count;
    uint32_t last_touched_batch;
} or_accum_f;

typedef struct or_accum_globals {
    uint64_t morton_watermark;
    uint64_t num_accumulated;
    uint64_t sum_leaf_counts;
    uint32_t points_folded;
    uint32_t num_leaves_folded;
    uint32_t inner_with_sums;
    uint32_t pad;
} or_accum_globals;

void or_accumulate(or_tree* t, uint32_t batch_index, or_accum_globals* g);
int or_get_accum_i(const or_tree* t, uint32_t i, or_accum_i* out);
int or_get_accum_f(const or_tree* t, uint32_t i, or_accum_f* out);

/* ------------------------------------------------------------ Analysis */

typedef struct or_analysis_node {
    double eig[3];          /* descending, in units of (node size)^2 */
    double normal[3];       /* eigenvector of the smallest eigenvalue */
    double surface_variation;
    double planarity;
    uint64_t count;
} or_analysis_node;

/* Roll the exact sums up the tree and solve every node's covariance with
 * cyclic Jacobi in FP64. out has or_num_nodes entries. */
void or_analyze_fp64(const or_tree* t, or_analysis_node* out);
/* Eigenvalues of a symmetric 3x3 (a00 a01 a02 a11 a12 a22) by cyclic Jacobi. */
void or_sym3_eig_jacobi(const double a[6], double eig[3], double vmin[3]);

/* The exact rolled sums behind or_analyze_fp64: per node 16 uint64 (n, s1[3],
 * s2 as lo/hi pairs xx xy xz yy yz zz) and the newest batch that added points
 * to the subtree (accumulators' last_touched_batch, rolled up by max). */
void or_rolled_sums(const or_tree* t, uint64_t* out16, uint32_t* last_touched);

typedef struct or_analysis_params {
    uint32_t min_points;
    uint32_t closure_margin;
    uint32_t current_batch;
    uint32_t frontier_only;
    float pixel_budget;
    uint32_t pad;
} or_analysis_params;

/* Screen coverage, flags (2: large, 4: frontier), closure and score
 * (surface variation x coverage, 0 below min_points) per node, from
 * or_analyze_fp64's eigenvalues; the projected extents use the LOD cut's float
 * arithmetic (remolod_render.cu:40-70). */
/* The learned scorer's 16 inputs per node as rb_analyze logs them (out16:
 * num_nodes x 16 floats); surface variation and planarity from the FP64
 * eigen-solve. */
void or_features(const or_tree* t, uint32_t current_batch, uint32_t closure_margin, float* out16);
void or_analysis_scores(const or_tree* t, const or_frame* f, const or_analysis_params* p,
                        const or_analysis_node* eig, float* coverage, uint32_t* flags, uint32_t* closed,
                        double* score);

/* ------------------------------------------------------------ Rasterize */

struct or_frame {
    float width, height;
    float transform[16];         /* row-major clip = M * (x, y, z, 1) */
    float transform_frozen[16];  /* LOD-selection transform */
    float box_min[3], box_max[3];
    float lod_pixel_budget;      /* 128 (src/shell/App.h:50-62) */
    int32_t point_size;
    uint32_t drawlist_capacity;  /* 131072 (remolod_render.cu:22) */
    /* optional: nodes forced large (Refinement); NULL or num_nodes bytes */
    const uint8_t* force_large;
    /* SharedUniforms::colorMode (HostDeviceCommon.h:63-66): 0 rgb, 1 by node,
     * 2 by level, 3 white */
    int32_t color_mode;
};

typedef struct or_render_result {
    uint32_t draw_items;
    uint32_t drawlist_overflow;
    uint64_t draw_samples;
} or_render_result;

#define OR_FB_CLEAR 0x7f80000000332211ull

/* kernel_render (remolod_render.cu:72-198) up to the resolve, pre-EDL. fb has
 * width*height entries. item_nodes (optional) receives the emitted node ids. */
void or_render(const or_tree* t, const or_frame* f, uint64_t* fb, or_render_result* r,
               uint32_t* item_nodes);
/* flat_render.cu:9-76: every point. */
void or_render_flat(const or_point* pts, uint64_t n, const or_frame* f, uint64_t* fb);
/* remo_framebuffer.cuh:78-122 with libm log2f/expf in place of the intrinsics. */
void or_edl(uint64_t* fb, uint32_t width, uint32_t height, float strength);
/* Refinement's colour filtering (wiki/02_KernelPipeline.md:228-243): for the
 * longest prefix of nodes[0..n) whose voxels fit capacity, each voxel's
 * colour becomes the mean colour (per 8-bit channel, rounded half up, alpha
 * kept) of the subtree's points in its cell. */
void or_refine_colors(or_tree* t, const uint32_t* nodes, uint32_t n, uint32_t capacity, uint32_t* nodes_filtered,
                      uint64_t* voxels_filtered);
/* remoDrawListWireframe (remo_lines.cuh:120-137): the 12 box edges of each of
 * the n draw items' nodes, drawn into fb (after EDL in the reference). */
void or_wireframe(const or_tree* t, const or_frame* f, uint64_t* fb, const uint32_t* item_nodes, uint32_t n);

#ifdef __cplusplus
}
#endif

#endif
