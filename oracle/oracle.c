/*
 * CPU oracle for the progressive LOD hot path -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h. Compiled with -ffp-contract=off so that every float operation
 * rounds once, as in the CUDA path built with -fmad=false.
 *
 * Deterministic rules this restatement fixes where the reference leaves a race
 * (each is also what the CUDA path implements):
 *  - spilling nodes are split in increasing node-id order, each taking the next
 *    block of 8 ids (remolod_octree.cu:309 takes them in atomic order);
 *  - a split the node pool cannot hold is refused before the node's points are
 *    moved to the spill list (the reference copies them first, :250-285, and
 *    re-inserts them as duplicates after refusing at :318-321);
 *  - a new voxel takes the colour of the lowest global point index that reaches
 *    its cell in the batch (the reference takes whichever thread sets the bit
 *    first, :116-138). Spilled points keep their original index.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAX_DEPTH 20
#define OR_GRID_WORDS 65536u          /* 128^3 bits as 32-bit words (remolod_structures.cuh:66-68) */
#define OR_GRID_BYTES 262144ull
#define OR_CHUNK_BYTES 16016ull       /* sizeof(Chunk): 1000 points + size + pad + next */
#define OR_SPILLED_CAPACITY 10000000u  /* (:76) */
#define OR_BACKLOG_CAPACITY 10000000u  /* (:26) */
#define OR_SPILLING_CAPACITY 100000u   /* (:40) */

typedef struct onode {
    int32_t child[8];
    uint32_t counter, num_points, level, X, Y, Z;
    int32_t grid;
    uint32_t num_voxels, num_voxels_stored;
    uint32_t num_point_chunks, num_voxel_chunks;
    or_point* pts;
    uint32_t* idx;
    uint32_t pts_cap;
    or_point* vox;
    uint32_t vox_cap;
    or_accum_i ai;
    or_accum_f af;
} onode;

typedef struct spill_pt {
    or_point p;
    uint32_t index;
} spill_pt;

struct or_tree {
    or_config cfg;
    onode* nodes;
    uint32_t num_nodes;
    uint32_t** grids;
    uint32_t num_grids, grids_cap;
    /* grids collapsed nodes returned; splits take them before new ones */
    int32_t* grid_pool;
    uint32_t grid_pool_n, grid_pool_cap;
    float box_min[3], box_max[3];
    float octree_size;
    or_stats st;
    /* per-batch scratch */
    spill_pt* spill;
    uint64_t spill_n, spill_cap;
};

/* ------------------------------------------------------------ helpers */

/* Threads for the batch loops: cfg.num_threads (0 or 1: one). Every threaded
 * loop either reads the tree only, or updates order-independent counters
 * atomically; everything order-dependent stays sequential, so the result is
 * the same for any thread count. */
static int or_threads(const or_tree* t) {
#ifdef _OPENMP
    return t->cfg.num_threads > 1u ? (int)t->cfg.num_threads : 1;
#else
    (void)t;
    return 1;
#endif
}

/* cvt.rzi.sat.u32.f32: NaN and negatives to 0, saturating at 2^32-1. */
static uint32_t cvt_u32(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

/* cvt.rzi.sat.s32.f32 */
static int32_t cvt_s32(float v) {
    if (v != v) return 0;
    if (v >= 2147483648.0f) return 2147483647;
    if (v <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)v;
}

/* remolod_octree.cu:163-169: X = u32(2^20 (x - min) / size), pX = u32(2^28 (x - min) / size) */
static void quantize(const or_tree* t, const or_point* p, uint32_t q20[3], uint32_t q28[3]) {
    const float c[3] = {p->x, p->y, p->z};
    for (int a = 0; a < 3; a++) {
        float d = c[a] - t->box_min[a];
        q20[a] = cvt_u32((1048576.0f * d) / t->octree_size);
        q28[a] = cvt_u32((268435456.0f * d) / t->octree_size);
    }
}

static uint32_t child_index(const uint32_t q20[3], int level) {
    const int s = OR_MAX_DEPTH - level - 1;
    return (((q20[0] >> s) & 1u) << 2) | (((q20[1] >> s) & 1u) << 1) | ((q20[2] >> s) & 1u);
}

/* remolod_octree.cu:182-201 (descend at most MAX_DEPTH levels) */
static uint32_t descend(const or_tree* t, const uint32_t q20[3]) {
    uint32_t cur = 0;
    for (int level = 0; level < OR_MAX_DEPTH; level++) {
        int32_t c = t->nodes[cur].child[child_index(q20, level)];
        if (c < 0) break;
        cur = (uint32_t)c;
    }
    return cur;
}

static int is_leaf(const onode* n) {
    for (int i = 0; i < 8; i++)
        if (n->child[i] >= 0) return 0;
    return 1;
}

/* AllocatorGlobal::alloc rounding (kernels/simlod/utils.h.cu:195) */
static uint64_t ref_alloc_size(uint64_t size) { return 16ull * ((size + 16ull) / 16ull); }

static uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1u) / b; }

static int32_t new_grid(or_tree* t) {
    if (t->grid_pool_n > 0) {
        const int32_t g = t->grid_pool[--t->grid_pool_n];
        memset(t->grids[g], 0, OR_GRID_WORDS * sizeof(uint32_t));
        return g;
    }
    if (t->num_grids == t->grids_cap) {
        uint32_t cap = t->grids_cap ? 2u * t->grids_cap : 64u;
        uint32_t** g = (uint32_t**)realloc(t->grids, cap * sizeof(uint32_t*));
        if (!g) abort();
        t->grids = g;
        t->grids_cap = cap;
    }
    uint32_t* words = (uint32_t*)calloc(OR_GRID_WORDS, sizeof(uint32_t));
    if (!words) abort();
    t->grids[t->num_grids] = words;
    t->st.persistent_offset += ref_alloc_size(OR_GRID_BYTES);
    return (int32_t)t->num_grids++;
}

static void node_init(onode* n) {
    memset(n, 0, sizeof(*n));
    for (int i = 0; i < 8; i++) n->child[i] = -1;
    n->grid = -1;
}

static void node_free_storage(onode* n) {
    free(n->pts);
    free(n->idx);
    free(n->vox);
    n->pts = NULL;
    n->idx = NULL;
    n->vox = NULL;
    n->pts_cap = n->vox_cap = 0;
}

/* --------------------------------------------------------- lifecycle */

or_tree* or_create(const or_config* cfg) {
    or_tree* t = (or_tree*)calloc(1, sizeof(or_tree));
    if (!t) return NULL;
    t->cfg = *cfg;
    if (!t->cfg.max_nodes) t->cfg.max_nodes = 200000u;
    if (!t->cfg.max_points_per_node) t->cfg.max_points_per_node = 50000u;
    if (!t->cfg.points_per_chunk) t->cfg.points_per_chunk = 1000u;
    if (!t->cfg.max_expand_iters) t->cfg.max_expand_iters = 20u;
    if (!t->cfg.safety_margin) t->cfg.safety_margin = 200000000ull;
    if (!t->cfg.ring_slots) t->cfg.ring_slots = 50u;
    if (!t->cfg.slot_capacity) t->cfg.slot_capacity = 1000000u;
    if (!t->cfg.max_batches_per_build) t->cfg.max_batches_per_build = 20u;
    if (!t->cfg.persistent_capacity) t->cfg.persistent_capacity = 1ull << 40;
    t->nodes = (onode*)calloc(t->cfg.max_nodes, sizeof(onode));
    if (!t->nodes) {
        free(t);
        return NULL;
    }
    return t;
}

static void release_all(or_tree* t) {
    for (uint32_t i = 0; i < t->num_nodes; i++) node_free_storage(&t->nodes[i]);
    for (uint32_t g = 0; g < t->num_grids; g++) free(t->grids[g]);
    t->num_grids = 0;
    t->grid_pool_n = 0;
    t->num_nodes = 0;
}

void or_destroy(or_tree* t) {
    if (!t) return;
    release_all(t);
    free(t->grids);
    free(t->grid_pool);
    free(t->nodes);
    free(t->spill);
    free(t);
}

/* remolod_reset.cu:41-85 */
void or_reset(or_tree* t, const float box_min[3], const float box_max[3]) {
    release_all(t);
    memset(&t->st, 0, sizeof(t->st));
    for (int a = 0; a < 3; a++) {
        t->box_min[a] = box_min[a];
        t->box_max[a] = box_max[a];
    }
    /* remolod_octree.cu:1148-1149 */
    float sx = box_max[0] - box_min[0], sy = box_max[1] - box_min[1], sz = box_max[2] - box_min[2];
    float m = sx > sy ? sx : sy;
    t->octree_size = m > sz ? m : sz;
    t->st.persistent_offset = 16;
    t->num_nodes = 1;
    node_init(&t->nodes[0]);
    t->nodes[0].grid = new_grid(t);
    t->st.num_nodes = 1;
}

/* ------------------------------------------------------------ Update */

static void spill_push(or_tree* t, const or_point* p, uint32_t index) {
    if (t->spill_n >= OR_SPILLED_CAPACITY) {
        t->st.overflow_flags |= OR_OVERFLOW_SPILLED;
        return;
    }
    if (t->spill_n == t->spill_cap) {
        uint64_t cap = t->spill_cap ? 2 * t->spill_cap : 65536;
        spill_pt* s = (spill_pt*)realloc(t->spill, cap * sizeof(spill_pt));
        if (!s) abort();
        t->spill = s;
        t->spill_cap = cap;
    }
    t->spill[t->spill_n].p = *p;
    t->spill[t->spill_n].index = index;
    t->spill_n++;
}

static int cmp_spill(const void* a, const void* b) {
    uint32_t x = ((const spill_pt*)a)->index, y = ((const spill_pt*)b)->index;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* doSplitting (remolod_octree.cu:303-400) for one accepted node. */
static void split_node(or_tree* t, uint32_t ni, uint32_t child_base) {
    onode* n = &t->nodes[ni];
    for (uint32_t i = 0; i < 8; i++) {
        onode* c = &t->nodes[child_base + i];
        node_init(c);
        c->level = n->level + 1;
        c->X = 2 * n->X + ((i >> 2) & 1u);
        c->Y = 2 * n->Y + ((i >> 1) & 1u);
        c->Z = 2 * n->Z + (i & 1u);
        n->child[i] = (int32_t)(child_base + i);
    }
    /* the node's stored points go to the spill list (doCounting :250-285) */
    uint32_t cap = n->num_point_chunks * t->cfg.points_per_chunk;
    uint32_t stored = n->num_points < cap ? n->num_points : cap;
    for (uint32_t s = 0; s < stored; s++) spill_push(t, &n->pts[s], n->idx[s]);
    /* chunks return to the queue (:349-360) */
    t->st.num_allocated_chunks -= n->num_point_chunks;
    n->num_point_chunks = 0;
    n->num_points = 0;
    free(n->pts);
    free(n->idx);
    n->pts = NULL;
    n->idx = NULL;
    n->pts_cap = 0;
    /* grid allocated once, zeroed at every split (:365-387) */
    if (n->grid < 0) n->grid = new_grid(t);
    else memset(t->grids[n->grid], 0, OR_GRID_WORDS * sizeof(uint32_t));
}

/* One counting pass over a point list: returns nothing, bumps counters of the
 * leaves that are still "fresh" for this iteration. */
typedef struct count_ctx {
    or_tree* t;
    uint32_t iter_tag;
    uint32_t* before;  /* counter snapshot at the start of the iteration */
    uint8_t* eligible; /* leaf counted in this iteration */
} count_ctx;

static void count_point(count_ctx* cc, const or_point* p, uint32_t* fresh_tag) {
    uint32_t q20[3], q28[3];
    quantize(cc->t, p, q20, q28);
    uint32_t leaf = descend(cc->t, q20);
    if (fresh_tag[leaf] < cc->iter_tag) __atomic_fetch_add(&cc->t->nodes[leaf].counter, 1u, __ATOMIC_RELAXED);
}

/* expand (remolod_octree.cu:402-462) */
static void expand(or_tree* t, const or_point* pts, uint32_t n, uint32_t batch_index,
                   uint32_t* fresh_tag) {
    const uint32_t iter_tag = batch_index + 1; /* countIteration (:429) */
    const uint32_t maxp = t->cfg.max_points_per_node;
    for (uint32_t it = 0; it < t->cfg.max_expand_iters; it++) {
        uint32_t nn = t->num_nodes;
        /* snapshot counters of nodes that count in this iteration */
        uint32_t* before = (uint32_t*)malloc((size_t)nn * sizeof(uint32_t));
        if (!before) abort();
        for (uint32_t i = 0; i < nn; i++) before[i] = t->nodes[i].counter;
        count_ctx cc = {t, iter_tag, before, NULL};
        const int nth = or_threads(t);
        const int64_t nb = (int64_t)n, nsp = (int64_t)t->spill_n;
#pragma omp parallel for num_threads(nth) schedule(static) if (nth > 1)
        for (int64_t i = 0; i < nb; i++) count_point(&cc, &pts[i], fresh_tag);
#pragma omp parallel for num_threads(nth) schedule(static) if (nth > 1)
        for (int64_t i = 0; i < nsp; i++) count_point(&cc, &t->spill[i].p, fresh_tag);
        /* spilling nodes: the counter crossed the limit in this iteration (:213-218) */
        uint32_t* spilling = NULL;
        uint32_t ns = 0;
        for (uint32_t i = 0; i < nn; i++) {
            if (fresh_tag[i] >= iter_tag) continue;
            if (before[i] <= maxp && t->nodes[i].counter > maxp) {
                if (ns % 1024 == 0) {
                    uint32_t* s = (uint32_t*)realloc(spilling, (ns + 1024) * sizeof(uint32_t));
                    if (!s) abort();
                    spilling = s;
                }
                spilling[ns++] = i;
            }
        }
        free(before);
        /* every node has now been counted in this iteration (:293-295) */
        for (uint32_t i = 0; i < nn; i++) fresh_tag[i] = iter_tag;
        t->st.expand_iters++;
        if (ns == 0) {
            free(spilling);
            break;
        }
        if (ns > OR_SPILLING_CAPACITY) {
            t->st.overflow_flags |= OR_OVERFLOW_SPILLING;
            ns = OR_SPILLING_CAPACITY;
        }
        for (uint32_t k = 0; k < ns; k++) {
            uint32_t ni = spilling[k];
            if (t->num_nodes + 8u > t->cfg.max_nodes) {
                t->st.node_pool_overflow = 1;
                continue;
            }
            uint32_t base = t->num_nodes;
            t->num_nodes += 8u;
            for (uint32_t c = 0; c < 8; c++) fresh_tag[base + c] = 0;
            split_node(t, ni, base);
            t->st.nodes_split++;
        }
        free(spilling);
        t->st.num_nodes = t->num_nodes;
    }
}

/* sampleVoxel (remolod_octree.cu:95-140) with the lowest-index rule: callers
 * visit points in increasing global index, so the first setter is the lowest. */
typedef struct voxel_new {
    uint32_t node;
    or_point v;
} voxel_new;

typedef struct vbacklog {
    voxel_new* v;
    uint64_t n, cap;
} vbacklog;

/* A (point, level) pair whose cell bit was clear before the batch. */
typedef struct vcand {
    uint32_t node, vi, color;
} vcand;

typedef struct vcands {
    vcand* v;
    uint64_t n, cap;
} vcands;

/* The candidate cells of one point's path, root first (reads the tree only). */
static void sample_candidates(const or_tree* t, const or_point* p, vcands* out) {
    uint32_t q20[3], q28[3];
    quantize(t, p, q20, q28);
    uint32_t cur = 0;
    for (int level = 0; level < OR_MAX_DEPTH; level++) {
        const onode* n = &t->nodes[cur];
        if (n->grid >= 0) {
            const uint32_t sh = (uint32_t)(OR_MAX_DEPTH + 1 - (int)n->level);
            uint32_t px = (q28[0] >> sh) % 128u;
            uint32_t py = (q28[1] >> sh) % 128u;
            uint32_t pz = (q28[2] >> sh) % 128u;
            uint32_t vi = px + py * 128u + pz * 16384u;
            if ((t->grids[n->grid][vi / 32u] & (1u << (vi % 32u))) == 0u) {
                if (out->n == out->cap) {
                    uint64_t cap = out->cap ? 2 * out->cap : 4096;
                    vcand* nv = (vcand*)realloc(out->v, cap * sizeof(vcand));
                    if (!nv) abort();
                    out->v = nv;
                    out->cap = cap;
                }
                out->v[out->n].node = cur;
                out->v[out->n].vi = vi;
                out->v[out->n].color = p->color;
                out->n++;
            }
        }
        int32_t c = n->child[child_index(q20, level)];
        if (c < 0) break;
        cur = (uint32_t)c;
    }
}

/* sampleVoxel's commit in visiting order: the first candidate of a cell sets
 * its bit and makes the voxel, at the cell centre with its colour. */
static void sample_commit(or_tree* t, const vcand* cd, vbacklog* bl) {
    onode* n = &t->nodes[cd->node];
    uint32_t* w = &t->grids[n->grid][cd->vi / 32u];
    uint32_t bit = 1u << (cd->vi % 32u);
    if (*w & bit) return;
    *w |= bit;
    n->num_voxels++;
    const uint32_t px = cd->vi % 128u, py = (cd->vi / 128u) % 128u, pz = cd->vi / 16384u;
    float node_size = t->octree_size / ldexpf(1.0f, (int)n->level);
    float mnx = fmaf((float)n->X, node_size, t->box_min[0]);
    float mny = fmaf((float)n->Y, node_size, t->box_min[1]);
    float mnz = fmaf((float)n->Z, node_size, t->box_min[2]);
    or_point v;
    v.x = mnx + node_size * ((float)px + 0.5f) / 128.0f;
    v.y = mny + node_size * ((float)py + 0.5f) / 128.0f;
    v.z = mnz + node_size * ((float)pz + 0.5f) / 128.0f;
    v.color = cd->color;
    if (bl->n >= OR_BACKLOG_CAPACITY) {
        t->st.overflow_flags |= OR_OVERFLOW_BACKLOG;
        return;
    }
    if (bl->n == bl->cap) {
        uint64_t cap = bl->cap ? 2 * bl->cap : 65536;
        voxel_new* nv = (voxel_new*)realloc(bl->v, cap * sizeof(voxel_new));
        if (!nv) abort();
        bl->v = nv;
        bl->cap = cap;
    }
    bl->v[bl->n].node = cd->node;
    bl->v[bl->n].v = v;
    bl->n++;
}

/* voxelSampling over the visiting order (spilled points by original index,
 * then the batch): candidates per contiguous range in parallel, committed in
 * order, which is the sequential result. */
static void sample_all(or_tree* t, const or_point* pts, uint32_t n, vbacklog* bl) {
    const int nth = or_threads(t);
    const uint64_t total = t->spill_n + n;
    vcands* parts = (vcands*)calloc((size_t)nth, sizeof(vcands));
    if (!parts) abort();
#pragma omp parallel num_threads(nth) if (nth > 1)
    {
        int tid = 0, tn = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        tn = omp_get_num_threads();
#endif
        const uint64_t lo = total * (uint64_t)tid / (uint64_t)tn, hi = total * (uint64_t)(tid + 1) / (uint64_t)tn;
        for (uint64_t i = lo; i < hi; i++)
            sample_candidates(t, i < t->spill_n ? &t->spill[i].p : &pts[i - t->spill_n], &parts[tid]);
    }
    for (int k = 0; k < nth; k++) {
        for (uint64_t i = 0; i < parts[k].n; i++) sample_commit(t, &parts[k].v[i], bl);
        free(parts[k].v);
    }
    free(parts);
}

static void ensure_pts_cap(onode* n, uint32_t cap) {
    if (cap <= n->pts_cap) return;
    or_point* p = (or_point*)realloc(n->pts, (size_t)cap * sizeof(or_point));
    uint32_t* i = (uint32_t*)realloc(n->idx, (size_t)cap * sizeof(uint32_t));
    if (!p || !i) abort();
    n->pts = p;
    n->idx = i;
    n->pts_cap = cap;
}

static void ensure_vox_cap(onode* n, uint32_t cap) {
    if (cap <= n->vox_cap) return;
    or_point* v = (or_point*)realloc(n->vox, (size_t)cap * sizeof(or_point));
    if (!v) abort();
    n->vox = v;
    n->vox_cap = cap;
}

/* allocatePointChunks (remolod_octree.cu:742-792). The reference sizes a
 * leaf's chunks by its counter, which equals its stored points plus the
 * batch's arrivals whenever every leaf was counted in the batch it was made.
 * A build whose expand loop stops at its pass limit leaves the last split's
 * nodes uncounted (counter 0, later lagging their stored points), where the
 * reference's rule would drop points (and its chunk walk has no defined
 * result); here the need is the larger of the two, so every arriving point
 * has a slot and the rule is the reference's wherever counters are whole.
 * arrivals[i]: the points of this batch whose leaf is node i. */
static void alloc_point_chunks(or_tree* t, const uint32_t* arrivals) {
    const uint32_t ppc = t->cfg.points_per_chunk;
    const uint64_t pool_before = t->st.chunk_pool_size;
    for (uint32_t i = 0; i < t->num_nodes; i++) {
        onode* n = &t->nodes[i];
        const uint32_t reach = n->num_points + arrivals[i];
        const uint32_t need = n->counter > reach ? n->counter : reach;
        if (!is_leaf(n) || !(n->num_points < need)) continue;
        uint32_t required = ceil_div(need, ppc);
        uint32_t existing = ceil_div(n->num_points, ppc);
        if (required <= existing) continue;
        uint32_t extra = required - existing;
        for (uint32_t k = 0; k < extra; k++) {
            uint64_t ci = t->st.num_allocated_chunks++;
            if (ci >= pool_before) t->st.persistent_offset += ref_alloc_size(OR_CHUNK_BYTES);
        }
        n->num_point_chunks = existing + extra;
        ensure_pts_cap(n, n->num_point_chunks * ppc);
    }
    if (t->st.num_allocated_chunks > t->st.chunk_pool_size)
        t->st.chunk_pool_size = t->st.num_allocated_chunks;
}

/* allocateVoxelChunks (remolod_octree.cu:885-916) */
static void alloc_voxel_chunks(or_tree* t) {
    const uint32_t ppc = t->cfg.points_per_chunk;
    for (uint32_t i = 0; i < t->num_nodes; i++) {
        onode* n = &t->nodes[i];
        uint32_t required = ceil_div(n->num_voxels, ppc);
        if (required == 0) continue;
        if (n->num_voxel_chunks == 0) {
            n->num_voxel_chunks = 1;
            t->st.persistent_offset += ref_alloc_size(OR_CHUNK_BYTES);
        }
        while (n->num_voxel_chunks < required) {
            n->num_voxel_chunks++;
            t->st.persistent_offset += ref_alloc_size(OR_CHUNK_BYTES);
        }
        ensure_vox_cap(n, n->num_voxel_chunks * ppc);
    }
}

/* insertPoints' per-point body (remolod_octree.cu:804-860) */
static uint32_t leaf_of(const or_tree* t, const or_point* p) {
    uint32_t q20[3], q28[3];
    quantize(t, p, q20, q28);
    return descend(t, q20);
}

static void insert_at(or_tree* t, uint32_t leaf, const or_point* p, uint32_t index) {
    onode* n = &t->nodes[leaf];
    uint32_t slot = n->num_points++;
    uint32_t cap = n->num_point_chunks * t->cfg.points_per_chunk;
    if (slot >= cap) {
        t->st.dropped_points++;
        return;
    }
    n->pts[slot] = *p;
    n->idx[slot] = index;
}

/* After expand: voxel sampling (spilled points by original index, then the
 * batch), chunk allocation, insertPoints and insertVoxels (addBatch's later
 * phases, remolod_octree.cu:940-1060). */
static void place_batch(or_tree* t, const or_point* pts, uint32_t n, uint32_t first_index) {
    qsort(t->spill, t->spill_n, sizeof(spill_pt), cmp_spill);
    vbacklog bl = {NULL, 0, 0};
    sample_all(t, pts, n, &bl);

    /* insertPoints' leaves: in parallel (the tree is fixed now) */
    const uint64_t total = (uint64_t)n + t->spill_n;
    uint32_t* leaves = (uint32_t*)malloc((size_t)(total ? total : 1) * sizeof(uint32_t));
    uint32_t* arrivals = (uint32_t*)calloc(t->num_nodes ? t->num_nodes : 1, sizeof(uint32_t));
    if (!leaves || !arrivals) abort();
    const int nth = or_threads(t);
    const int64_t tot = (int64_t)total;
#pragma omp parallel for num_threads(nth) schedule(static) if (nth > 1)
    for (int64_t i = 0; i < tot; i++)
        leaves[i] = leaf_of(t, i < (int64_t)n ? &pts[i] : &t->spill[i - (int64_t)n].p);
    for (uint64_t i = 0; i < total; i++) arrivals[leaves[i]]++;

    alloc_point_chunks(t, arrivals);
    alloc_voxel_chunks(t);
    free(arrivals);

    /* insertPoints: slots in order */
    for (uint32_t i = 0; i < n; i++) insert_at(t, leaves[i], &pts[i], first_index + i);
    for (uint64_t i = 0; i < t->spill_n; i++) insert_at(t, leaves[n + i], &t->spill[i].p, t->spill[i].index);
    free(leaves);

    /* insertVoxels (remolod_octree.cu:918-938) */
    for (uint64_t i = 0; i < bl.n; i++) {
        onode* nd = &t->nodes[bl.v[i].node];
        uint32_t slot = nd->num_voxels_stored++;
        if (slot < nd->num_voxel_chunks * t->cfg.points_per_chunk) nd->vox[slot] = bl.v[i].v;
    }
    free(bl.v);
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

int or_add_batch(or_tree* t, const or_point* pts, uint32_t n) {
    /* remolod_octree.cu:1181-1210 */
    if (t->st.persistent_offset + t->cfg.safety_margin >= t->cfg.persistent_capacity) {
        t->st.mem_capacity_reached = 1;
        return 1;
    }
    t->st.mem_capacity_reached = 0;
    const uint32_t batch_index = t->st.batchlet_index;
    const uint32_t first_index = (uint32_t)t->st.num_points_processed;
    t->spill_n = 0;

    uint32_t* fresh_tag = (uint32_t*)calloc(t->cfg.max_nodes, sizeof(uint32_t));
    if (!fresh_tag) abort();
    /* nodes that exist count with countIteration = batchIndex (set in the previous batch) */
    for (uint32_t i = 0; i < t->num_nodes; i++) fresh_tag[i] = batch_index;
    expand(t, pts, n, batch_index, fresh_tag);
    free(fresh_tag);
    t->st.spilled_points += t->spill_n;

    place_batch(t, pts, n, first_index);
    t->st.batchlet_index++;
    t->st.num_points_processed += n;
    return 0;
}

/* Refinement's deepening (wiki/02_KernelPipeline.md:228-243, "local split
 * and redistribute"). The leaves among nodes[0..n) holding at least
 * min_points points (0 counts as 1) split as a batch's spilling nodes do
 * (doSplitting, remolod_octree.cu:303-400): in increasing id, 8 consecutive
 * ids each, refused by the pool guard once fewer than 8 remain (:318-321).
 * That split is iteration 1 of an expand loop with no batch points: the
 * later iterations count the spilled points into the new children and split
 * any child over the limit (:402-462). The spilled points are then sampled
 * into voxels and inserted as a batch's are. The memory check of a batch
 * (:1181-1210) refuses the whole pass (returns 1). No batch is consumed:
 * batchlet_index, num_points_processed and expand_iters stay. */
int or_deepen(or_tree* t, const uint32_t* nodes, uint32_t n, uint32_t min_points, uint32_t* selected) {
    if (selected) *selected = 0;
    if (t->st.persistent_offset + t->cfg.safety_margin >= t->cfg.persistent_capacity) {
        t->st.mem_capacity_reached = 1;
        return 1;
    }
    t->st.mem_capacity_reached = 0;
    const uint32_t minp = min_points ? min_points : 1u;
    uint32_t* sel = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    if (!sel) abort();
    uint32_t ns = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t ni = nodes[i];
        if (ni < t->num_nodes && is_leaf(&t->nodes[ni]) && t->nodes[ni].level < OR_MAX_DEPTH &&
            t->nodes[ni].num_points >= minp)
            sel[ns++] = ni;
    }
    if (ns > OR_SPILLING_CAPACITY) {
        t->st.overflow_flags |= OR_OVERFLOW_SPILLING;
        ns = OR_SPILLING_CAPACITY;
    }
    if (selected) *selected = ns;
    qsort(sel, ns, sizeof(uint32_t), cmp_u32);
    const uint32_t batch_index = t->st.batchlet_index;
    t->spill_n = 0;
    uint32_t* fresh_tag = (uint32_t*)calloc(t->cfg.max_nodes, sizeof(uint32_t));
    if (!fresh_tag) abort();
    /* nodes that exist are not counted again in this pass */
    for (uint32_t i = 0; i < t->num_nodes; i++) fresh_tag[i] = batch_index + 1u;
    for (uint32_t k = 0; k < ns; k++) {
        if (t->num_nodes + 8u > t->cfg.max_nodes) {
            t->st.node_pool_overflow = 1;
            continue;
        }
        const uint32_t base = t->num_nodes;
        t->num_nodes += 8u;
        split_node(t, sel[k], base);
        t->st.nodes_split++;
    }
    t->st.num_nodes = t->num_nodes;
    free(sel);
    /* iterations 2.. of the loop: the seeded split was iteration 1 */
    const uint32_t iters = t->cfg.max_expand_iters, done = t->st.expand_iters;
    t->cfg.max_expand_iters = iters > 0u ? iters - 1u : 0u;
    expand(t, NULL, 0, batch_index, fresh_tag);
    t->cfg.max_expand_iters = iters;
    t->st.expand_iters = done;
    free(fresh_tag);
    t->st.spilled_points += t->spill_n;
    place_batch(t, NULL, 0, 0);
    return 0;
}

/* Refinement's collapsing ("merge a node back up",
 * wiki/02_KernelPipeline.md:228-243; it needs a grid pool, CLAUDE.md:185-187).
 * Each node among nodes[0..n) (duplicates ignored) below the root whose
 * eight children are all leaves holding at most max_points points together
 * (0: the split limit) becomes a leaf with their points, in child order. Its
 * chunks are taken first, as allocatePointChunks takes them (:742-792):
 * recycled, then new ones charged to the store; then the children's chunks
 * return to the queue and the children are left empty with nothing pointing
 * to them. The node drops its voxels and returns its grid to the pool; its
 * exact sums restart, so the next Accumulate folds all its points. */
int or_collapse(or_tree* t, const uint32_t* nodes, uint32_t n, uint32_t max_points, uint32_t* collapsed,
                uint64_t* points, uint64_t* voxels) {
    const uint32_t ppc = t->cfg.points_per_chunk;
    const uint32_t maxp = max_points ? max_points : t->cfg.max_points_per_node;
    uint32_t* ids = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t* rec = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    if (!ids || !rec) abort();
    memcpy(ids, nodes, (size_t)n * sizeof(uint32_t));
    qsort(ids, n, sizeof(uint32_t), cmp_u32);
    uint32_t nr = 0;
    uint64_t moved = 0, dropped = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t ni = ids[i];
        if ((i > 0 && ids[i - 1] == ni) || ni >= t->num_nodes) continue;
        const onode* nd = &t->nodes[ni];
        if (nd->level == 0 || is_leaf(nd)) continue;
        uint64_t total = 0;
        int ok = 1;
        for (int q = 0; q < 8 && ok; q++) {
            const int32_t ch = nd->child[q];
            if (ch < 0 || !is_leaf(&t->nodes[ch])) ok = 0;
            else {
                const onode* c = &t->nodes[ch];
                const uint32_t cap = c->num_point_chunks * ppc;
                total += c->num_points < cap ? c->num_points : cap;
            }
        }
        if (ok && total <= maxp) rec[nr++] = ni;
    }
    /* the merged leaves' chunks first */
    const uint64_t pool_before = t->st.chunk_pool_size;
    for (uint32_t k = 0; k < nr; k++) {
        onode* nd = &t->nodes[rec[k]];
        uint32_t total = 0;
        for (int q = 0; q < 8; q++) {
            const onode* c = &t->nodes[nd->child[q]];
            const uint32_t cap = c->num_point_chunks * ppc;
            total += c->num_points < cap ? c->num_points : cap;
        }
        const uint32_t req = ceil_div(total, ppc);
        for (uint32_t e = 0; e < req; e++) {
            const uint64_t ci = t->st.num_allocated_chunks++;
            if (ci >= pool_before) t->st.persistent_offset += ref_alloc_size(OR_CHUNK_BYTES);
        }
        ensure_pts_cap(nd, req * ppc > 0 ? req * ppc : 1);
        uint32_t at = 0;
        for (int q = 0; q < 8; q++) {
            const onode* c = &t->nodes[nd->child[q]];
            const uint32_t cap = c->num_point_chunks * ppc;
            const uint32_t np = c->num_points < cap ? c->num_points : cap;
            if (np) {
                memcpy(nd->pts + at, c->pts, (size_t)np * sizeof(or_point));
                memcpy(nd->idx + at, c->idx, (size_t)np * sizeof(uint32_t));
            }
            at += np;
        }
        nd->num_point_chunks = req;
        nd->num_points = total;
        nd->counter = total;
        moved += total;
    }
    if (t->st.num_allocated_chunks > t->st.chunk_pool_size) t->st.chunk_pool_size = t->st.num_allocated_chunks;
    /* then the children's chunks back to the queue, the voxels and the grid */
    for (uint32_t k = 0; k < nr; k++) {
        onode* nd = &t->nodes[rec[k]];
        for (int q = 0; q < 8; q++) {
            onode* c = &t->nodes[nd->child[q]];
            t->st.num_allocated_chunks -= c->num_point_chunks;
            free(c->pts);
            free(c->idx);
            c->pts = NULL;
            c->idx = NULL;
            c->pts_cap = 0;
            c->num_points = 0;
            c->counter = 0;
            c->num_point_chunks = 0;
            memset(&c->ai, 0, sizeof(c->ai));
            memset(&c->af, 0, sizeof(c->af));
            nd->child[q] = -1;
        }
        dropped += nd->num_voxels;
        free(nd->vox);
        nd->vox = NULL;
        nd->vox_cap = 0;
        nd->num_voxels = 0;
        nd->num_voxels_stored = 0;
        nd->num_voxel_chunks = 0;
        if (nd->grid >= 0) {
            if (t->grid_pool_n == t->grid_pool_cap) {
                uint32_t cap = t->grid_pool_cap ? 2u * t->grid_pool_cap : 64u;
                int32_t* g = (int32_t*)realloc(t->grid_pool, cap * sizeof(int32_t));
                if (!g) abort();
                t->grid_pool = g;
                t->grid_pool_cap = cap;
            }
            t->grid_pool[t->grid_pool_n++] = nd->grid;
            nd->grid = -1;
        }
        memset(&nd->ai, 0, sizeof(nd->ai));
        memset(&nd->af, 0, sizeof(nd->af));
    }
    free(ids);
    free(rec);
    if (collapsed) *collapsed = nr;
    if (points) *points = moved;
    if (voxels) *voxels = dropped;
    return 0;
}

/* stats sweep (remolod_octree.cu:1271-1310) */
void or_sweep(or_tree* t) {
    or_stats* s = &t->st;
    const uint32_t ppc = t->cfg.points_per_chunk;
    s->num_inner = s->num_leaves = s->num_nonempty_leaves = 0;
    s->num_points = s->num_voxels = 0;
    s->num_chunks_points = s->num_chunks_voxels = 0;
    s->max_points_per_node = 0;
    s->counter_underflows = 0;
    for (uint32_t i = 0; i < t->num_nodes; i++) {
        const onode* n = &t->nodes[i];
        if (is_leaf(n)) {
            s->num_leaves++;
            s->num_points += n->num_points;
            s->num_chunks_points += ceil_div(n->num_points, ppc);
            if (n->num_points > s->max_points_per_node) s->max_points_per_node = n->num_points;
            if (n->counter < n->num_points) s->counter_underflows++;
            if (n->num_points > 0) s->num_nonempty_leaves++;
        } else {
            s->num_inner++;
            s->num_voxels += n->num_voxels;
            s->num_chunks_voxels += ceil_div(n->num_voxels, ppc);
        }
    }
    s->num_nodes = t->num_nodes;
    s->num_grids = t->num_grids - t->grid_pool_n;
}

uint32_t or_build(or_tree* t, const or_point* ring, const uint32_t* batch_sizes,
                  uint32_t num_uploaded) {
    uint32_t first = t->st.batchlet_index;
    uint32_t avail = num_uploaded > first ? num_uploaded - first : 0u;
    uint32_t nb = avail < t->cfg.max_batches_per_build ? avail : t->cfg.max_batches_per_build;
    uint32_t done = 0;
    for (uint32_t b = first; b < first + nb; b++) {
        uint32_t slot = b % t->cfg.ring_slots;
        const or_point* p = ring + (uint64_t)slot * t->cfg.slot_capacity;
        if (or_add_batch(t, p, batch_sizes[slot]) != 0) break;
        done++;
    }
    or_sweep(t);
    return done;
}

void or_get_stats(const or_tree* t, or_stats* s) { *s = t->st; }
uint32_t or_num_nodes(const or_tree* t) { return t->num_nodes; }

int or_get_node(const or_tree* t, uint32_t i, or_node_info* o) {
    if (i >= t->num_nodes) return -1;
    const onode* n = &t->nodes[i];
    for (int k = 0; k < 8; k++) o->child[k] = n->child[k];
    o->counter = n->counter;
    o->num_points = n->num_points;
    o->level = n->level;
    o->X = n->X;
    o->Y = n->Y;
    o->Z = n->Z;
    o->grid = n->grid;
    o->num_voxels = n->num_voxels;
    o->num_point_chunks = n->num_point_chunks;
    o->num_voxel_chunks = n->num_voxel_chunks;
    o->is_leaf = (uint32_t)is_leaf(n);
    return 0;
}

uint32_t or_leaf_points(const or_tree* t, uint32_t i, const or_point** pts, const uint32_t** idx) {
    if (i >= t->num_nodes) return 0;
    const onode* n = &t->nodes[i];
    uint32_t cap = n->num_point_chunks * t->cfg.points_per_chunk;
    *pts = n->pts;
    *idx = n->idx;
    return n->num_points < cap ? n->num_points : cap;
}

uint32_t or_node_voxels(const or_tree* t, uint32_t i, const or_point** vox) {
    if (i >= t->num_nodes) return 0;
    const onode* n = &t->nodes[i];
    *vox = n->vox;
    uint32_t cap = n->num_voxel_chunks * t->cfg.points_per_chunk;
    return n->num_voxels_stored < cap ? n->num_voxels_stored : cap;
}

const uint32_t* or_node_grid(const or_tree* t, uint32_t i) {
    if (i >= t->num_nodes || t->nodes[i].grid < 0) return NULL;
    return t->grids[t->nodes[i].grid];
}

/* ------------------------------------------------------------ Accumulate */

/* remoMortonSpread / remoMortonCode (remolod_accum.cu:24-36) */
static uint64_t morton_spread(uint32_t v) {
    uint64_t x = (uint64_t)v & 0xFFFFFull;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

static uint64_t morton3(uint32_t X, uint32_t Y, uint32_t Z) {
    return (morton_spread(X) << 2) | (morton_spread(Y) << 1) | morton_spread(Z);
}

static void add128(uint64_t* lo, uint64_t* hi, uint64_t v) {
    uint64_t o = *lo;
    *lo = o + v;
    *hi += (*lo < o) ? 1u : 0u;
}

/* Folds [count, numPoints) of every leaf, clears inner nodes (remolod_accum.cu:69-211),
 * then the verify pass (:214-233). Both the exact integer sums and the
 * reference's FP64/FP32 sums are kept. */
void or_accumulate(or_tree* t, uint32_t batch_index, or_accum_globals* g) {
    g->sum_leaf_counts = 0;
    g->inner_with_sums = 0;
    g->points_folded = 0;
    g->num_leaves_folded = 0;
    const uint32_t ppc = t->cfg.points_per_chunk;
    const double inv_size = 1.0 / (double)t->octree_size;
    for (uint32_t i = 0; i < t->num_nodes; i++) {
        onode* n = &t->nodes[i];
        if (!is_leaf(n)) {
            if (n->ai.count != 0) memset(&n->ai, 0, sizeof(n->ai));
            if (n->af.count != 0) memset(&n->af, 0, sizeof(n->af));
            continue;
        }
        uint32_t from = n->ai.count, to = n->num_points;
        if (to <= from) continue;
        uint32_t cap = n->num_point_chunks * ppc;
        const uint32_t sh = 28u - n->level;
        const int64_t lim = (int64_t)1 << sh;
        const int64_t base[3] = {(int64_t)n->X << sh, (int64_t)n->Y << sh, (int64_t)n->Z << sh};
        const double level_scale = (double)(1ull << n->level);
        uint64_t wm = 0;
        for (uint32_t s = from; s < to; s++) {
            if (s >= cap) break;
            const or_point* p = &n->pts[s];
            uint32_t q20[3], q28[3];
            quantize(t, p, q20, q28);
            int64_t q[3];
            for (int a = 0; a < 3; a++) {
                int64_t v = (int64_t)q28[a] - base[a];
                if (v < 0) v = 0;
                if (v > lim) v = lim;
                q[a] = v;
                n->ai.s1[a] += (uint64_t)v;
            }
            const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
            for (int k = 0; k < 6; k++)
                add128(&n->ai.s2_lo[k], &n->ai.s2_hi[k], (uint64_t)(q[pa[k]] * q[pb[k]]));
            uint32_t c = p->color;
            uint32_t ch[3] = {c & 255u, (c >> 8) & 255u, (c >> 16) & 255u};
            for (int a = 0; a < 3; a++) {
                n->ai.c1[a] += ch[a];
                n->ai.c2[a] += (uint64_t)ch[a] * ch[a];
            }
            uint32_t mx = q20[0] < 1048575u ? q20[0] : 1048575u;
            uint32_t my = q20[1] < 1048575u ? q20[1] : 1048575u;
            uint32_t mz = q20[2] < 1048575u ? q20[2] : 1048575u;
            uint64_t m = morton3(mx, my, mz);
            if (m > wm) wm = m;
            /* the reference's double-precision variant (remolod_accum.cu:115-153) */
            double lx = ((double)p->x - (double)t->box_min[0]) * inv_size;
            double ly = ((double)p->y - (double)t->box_min[1]) * inv_size;
            double lz = ((double)p->z - (double)t->box_min[2]) * inv_size;
            lx = lx * level_scale - (double)n->X;
            ly = ly * level_scale - (double)n->Y;
            lz = lz * level_scale - (double)n->Z;
            lx = fmin(fmax(lx, 0.0), 1.0);
            ly = fmin(fmax(ly, 0.0), 1.0);
            lz = fmin(fmax(lz, 0.0), 1.0);
            n->af.g[0] += lx;
            n->af.g[1] += ly;
            n->af.g[2] += lz;
            n->af.g[3] += lx * lx;
            n->af.g[4] += lx * ly;
            n->af.g[5] += lx * lz;
            n->af.g[6] += ly * ly;
            n->af.g[7] += ly * lz;
            n->af.g[8] += lz * lz;
            float cr = (float)ch[0] * (1.0f / 255.0f);
            float cg = (float)ch[1] * (1.0f / 255.0f);
            float cb = (float)ch[2] * (1.0f / 255.0f);
            n->af.c[0] += cr;
            n->af.c[1] += cg;
            n->af.c[2] += cb;
            n->af.c[3] += cr * cr;
            n->af.c[4] += cg * cg;
            n->af.c[5] += cb * cb;
        }
        n->ai.count = to;
        n->ai.last_touched_batch = batch_index;
        n->af.count = to;
        n->af.last_touched_batch = batch_index;
        if (wm > g->morton_watermark) g->morton_watermark = wm;
        g->num_accumulated += (uint64_t)(to - from);
        g->points_folded += to - from;
        g->num_leaves_folded++;
    }
    for (uint32_t i = 0; i < t->num_nodes; i++) {
        const onode* n = &t->nodes[i];
        if (is_leaf(n)) g->sum_leaf_counts += n->ai.count;
        else if (n->ai.count != 0) g->inner_with_sums++;
    }
}

int or_get_accum_i(const or_tree* t, uint32_t i, or_accum_i* out) {
    if (i >= t->num_nodes) return -1;
    *out = t->nodes[i].ai;
    return 0;
}

int or_get_accum_f(const or_tree* t, uint32_t i, or_accum_f* out) {
    if (i >= t->num_nodes) return -1;
    *out = t->nodes[i].af;
    return 0;
}

/* ------------------------------------------------------------ Analysis */

typedef unsigned __int128 u128;
typedef __int128 i128;

typedef struct roll {
    u128 n;
    u128 s1[3];
    u128 s2[6];
} roll;

static void roll_node(const or_tree* t, uint32_t i, roll* out, roll* all) {
    const onode* n = &t->nodes[i];
    memset(out, 0, sizeof(*out));
    if (is_leaf(n)) {
        out->n = n->ai.count;
        for (int a = 0; a < 3; a++) out->s1[a] = n->ai.s1[a];
        for (int k = 0; k < 6; k++) out->s2[k] = ((u128)n->ai.s2_hi[k] << 64) | n->ai.s2_lo[k];
        return;
    }
    const uint32_t sh_child = 28u - (n->level + 1u);
    for (int c = 0; c < 8; c++) {
        if (n->child[c] < 0) continue;
        const roll* r = &all[n->child[c]];
        const onode* cn = &t->nodes[n->child[c]];
        u128 o[3] = {(u128)(cn->X - 2u * n->X) << sh_child, (u128)(cn->Y - 2u * n->Y) << sh_child,
                     (u128)(cn->Z - 2u * n->Z) << sh_child};
        out->n += r->n;
        for (int a = 0; a < 3; a++) out->s1[a] += r->s1[a] + r->n * o[a];
        const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
        for (int k = 0; k < 6; k++) {
            int a = pa[k], b = pb[k];
            out->s2[k] += r->s2[k] + o[a] * r->s1[b] + o[b] * r->s1[a] + r->n * o[a] * o[b];
        }
    }
}

void or_sym3_eig_jacobi(const double a_in[6], double eig[3], double vmin[3]) {
    double a[3][3] = {{a_in[0], a_in[1], a_in[2]}, {a_in[1], a_in[3], a_in[4]},
                      {a_in[2], a_in[4], a_in[5]}};
    double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 64; sweep++) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-36 * diag || off == 0.0) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0.0) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(tt * tt + 1.0), s = tt * c;
                for (int k = 0; k < 3; k++) {
                    double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {
                    double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = c * vkp - s * vkq;
                    v[k][q] = s * vkp + c * vkq;
                }
            }
    }
    int ord[3] = {0, 1, 2};
    double d[3] = {a[0][0], a[1][1], a[2][2]};
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (d[ord[j]] > d[ord[i]]) {
                int tmp = ord[i];
                ord[i] = ord[j];
                ord[j] = tmp;
            }
    for (int i = 0; i < 3; i++) eig[i] = d[ord[i]];
    for (int k = 0; k < 3; k++) vmin[k] = v[k][ord[2]];
}

void or_rolled_sums(const or_tree* t, uint64_t* out16, uint32_t* last_touched) {
    const uint32_t nn = t->num_nodes;
    roll* all = (roll*)calloc(nn ? nn : 1, sizeof(roll));
    uint32_t* lt = (uint32_t*)calloc(nn ? nn : 1, sizeof(uint32_t));
    if (!all || !lt) abort();
    for (uint32_t k = nn; k-- > 0;) {
        roll_node(t, k, &all[k], all);
        const onode* n = &t->nodes[k];
        if (is_leaf(n)) {
            lt[k] = n->ai.count ? n->ai.last_touched_batch : 0u;
        } else {
            uint32_t m = 0;
            for (int c = 0; c < 8; c++)
                if (n->child[c] >= 0 && all[n->child[c]].n > 0 && lt[n->child[c]] > m) m = lt[n->child[c]];
            lt[k] = m;
        }
    }
    for (uint32_t i = 0; i < nn; i++) {
        uint64_t* o = out16 + (size_t)i * 16;
        o[0] = (uint64_t)all[i].n;
        for (int a = 0; a < 3; a++) o[1 + a] = (uint64_t)all[i].s1[a];
        for (int k = 0; k < 6; k++) {
            o[4 + 2 * k] = (uint64_t)all[i].s2[k];
            o[4 + 2 * k + 1] = (uint64_t)(all[i].s2[k] >> 64);
        }
        if (last_touched) last_touched[i] = lt[i];
    }
    free(all);
    free(lt);
}

void or_analyze_fp64(const or_tree* t, or_analysis_node* out) {
    const uint32_t nn = t->num_nodes;
    roll* all = (roll*)calloc(nn ? nn : 1, sizeof(roll));
    if (!all) abort();
    /* children always have larger ids than their parent: roll up in reverse id order */
    for (uint32_t k = nn; k-- > 0;) roll_node(t, k, &all[k], all);
    for (uint32_t i = 0; i < nn; i++) {
        const roll* r = &all[i];
        or_analysis_node* o = &out[i];
        memset(o, 0, sizeof(*o));
        o->count = (uint64_t)r->n;
        if (r->n < 3) continue;
        const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
        const double unit = ldexp(1.0, (int)(28u - t->nodes[i].level));
        double nd = (double)r->n;
        double cov[6];
        for (int k = 0; k < 6; k++) {
            i128 c = (i128)(r->n * r->s2[k]) - (i128)(r->s1[pa[k]] * r->s1[pb[k]]);
            cov[k] = (double)c / (nd * nd) / (unit * unit);
        }
        or_sym3_eig_jacobi(cov, o->eig, o->normal);
        double tr = o->eig[0] + o->eig[1] + o->eig[2];
        o->surface_variation = tr > 0.0 ? o->eig[2] / tr : 0.0;
        o->planarity = o->eig[0] > 0.0 ? (o->eig[1] - o->eig[2]) / o->eig[0] : 0.0;
    }
    free(all);
}

/* The learned scorer's 16 inputs per node, as rb_analyze logs them: log
 * count, level, mean, normalised centred second moments, surface variation and
 * planarity (from the FP64 eigen-solve here), fill, colour variance, age. */
void or_features(const or_tree* t, uint32_t current_batch, uint32_t closure_margin, float* out16) {
    const uint32_t nn = t->num_nodes;
    uint64_t* sums = (uint64_t*)calloc((size_t)(nn ? nn : 1) * 16, sizeof(uint64_t));
    uint32_t* lt = (uint32_t*)calloc(nn ? nn : 1, sizeof(uint32_t));
    uint64_t* col = (uint64_t*)calloc((size_t)(nn ? nn : 1) * 6, sizeof(uint64_t));
    or_analysis_node* eig = (or_analysis_node*)calloc(nn ? nn : 1, sizeof(or_analysis_node));
    if (!sums || !lt || !col || !eig) abort();
    or_rolled_sums(t, sums, lt);
    or_analyze_fp64(t, eig);
    /* colour sums roll up unchanged: children have larger ids than their parent */
    for (uint32_t k = nn; k-- > 0;) {
        const onode* n = &t->nodes[k];
        uint64_t* c = col + (size_t)k * 6;
        if (is_leaf(n)) {
            for (int a = 0; a < 3; a++) {
                c[a] = n->ai.c1[a];
                c[3 + a] = n->ai.c2[a];
            }
        } else {
            for (int q = 0; q < 8; q++) {
                if (n->child[q] < 0) continue;
                const uint64_t* cc = col + (size_t)n->child[q] * 6;
                for (int a = 0; a < 6; a++) c[a] += cc[a];
            }
        }
    }
    const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
    for (uint32_t i = 0; i < nn; i++) {
        const onode* n = &t->nodes[i];
        const uint64_t* r = sums + (size_t)i * 16;
        const uint64_t cnt = r[0];
        float* ft = out16 + (size_t)i * 16;
        const double nd = cnt ? (double)cnt : 1.0;
        const double unit = ldexp(1.0, (int)(28u - n->level));
        ft[0] = log2f(1.0f + (float)cnt) * (1.0f / 24.0f);
        ft[1] = (float)n->level * (1.0f / 20.0f);
        for (int k = 0; k < 3; k++) ft[2 + k] = cnt ? (float)((double)r[1 + k] / (nd * unit)) : 0.0f;
        for (int k = 0; k < 6; k++) {
            float v = 0.0f;
            if (cnt >= 2) {
                const u128 s2 = ((u128)r[4 + 2 * k + 1] << 64) | r[4 + 2 * k];
                const i128 c = (i128)((u128)cnt * s2) - (i128)r[1 + pa[k]] * (i128)r[1 + pb[k]];
                v = (float)((double)c / (nd * nd * unit * unit) * 12.0);
            }
            ft[5 + k] = v;
        }
        ft[11] = (float)eig[i].surface_variation * 3.0f;
        ft[12] = (float)eig[i].planarity;
        const float fill = is_leaf(n) ? (float)n->num_points * (1.0f / 50000.0f) : (float)n->num_voxels * (1.0f / 16384.0f);
        ft[13] = fminf(fill, 4.0f);
        float cvar = 0.0f;
        if (cnt >= 2) {
            const uint64_t* c = col + (size_t)i * 6;
            for (int k = 0; k < 3; k++) {
                const double m = (double)c[k] / nd;
                cvar += (float)(((double)c[3 + k] / nd - m * m) / (255.0 * 255.0));
            }
        }
        ft[14] = cvar * (4.0f / 3.0f);
        const float age = current_batch > lt[i] ? (float)(current_batch - lt[i]) : 0.0f;
        ft[15] = fminf(age / (float)(closure_margin ? closure_margin : 1u), 2.0f);
    }
    free(sums);
    free(lt);
    free(col);
    free(eig);
}

static void box_extent(const or_frame* f, float cube, uint32_t level, uint32_t X, uint32_t Y, uint32_t Z,
                       float ext[4], int* any);

void or_analysis_scores(const or_tree* t, const or_frame* f, const or_analysis_params* p,
                        const or_analysis_node* eig, float* coverage, uint32_t* flags, uint32_t* closed,
                        double* score) {
    const uint32_t nn = t->num_nodes;
    uint32_t* lt = (uint32_t*)calloc(nn ? nn : 1, sizeof(uint32_t));
    uint64_t* sums = (uint64_t*)calloc((size_t)(nn ? nn : 1) * 16, sizeof(uint64_t));
    if (!lt || !sums) abort();
    or_rolled_sums(t, sums, lt);
    float sx = f->box_max[0] - f->box_min[0], sy = f->box_max[1] - f->box_min[1], sz = f->box_max[2] - f->box_min[2];
    float cube = fmaxf(fmaxf(sx, sy), sz);
    for (uint32_t i = 0; i < nn; i++) {
        const onode* n = &t->nodes[i];
        float e0[4], e1[4];
        int a0 = 0, a1 = 0;
        box_extent(f, cube, n->level, n->X, n->Y, n->Z, e0, &a0);
        if (n->level > 0) box_extent(f, cube, n->level - 1, n->X >> 1, n->Y >> 1, n->Z >> 1, e1, &a1);
        float cov = 0.0f;
        int large = 0, parent_large = n->level == 0;
        if (a0) {
            float x0 = fmaxf(e0[0], 0.0f), x1 = fminf(e0[1], f->width);
            float y0 = fmaxf(e0[2], 0.0f), y1 = fminf(e0[3], f->height);
            if (x1 > x0 && y1 > y0) cov = (x1 - x0) * (y1 - y0) / (f->width * f->height);
            large = (e0[1] - e0[0]) > p->pixel_budget || (e0[3] - e0[2]) > p->pixel_budget;
        }
        if (n->level > 0 && a1) parent_large = (e1[1] - e1[0]) > p->pixel_budget || (e1[3] - e1[2]) > p->pixel_budget;
        uint32_t fl = 0;
        if (large) fl |= 2u;
        if (!is_leaf(n) && !large && parent_large) fl |= 4u;
        coverage[i] = cov;
        flags[i] = fl;
        uint64_t cnt = sums[(size_t)i * 16];
        closed[i] = (p->current_batch >= lt[i] + p->closure_margin && cnt > 0) ? 1u : 0u;
        double sc = eig[i].surface_variation * (double)cov;
        if (cnt < p->min_points) sc = 0.0;
        score[i] = sc;
    }
    free(lt);
    free(sums);
}

/* ------------------------------------------------------------ Rasterize */

typedef struct f4 {
    float x, y, z, w;
} f4;

/* remoMatMul (remo_math.cuh:25-32), left-to-right sums */
static f4 matmul(const float* m, float x, float y, float z, float w) {
    f4 r;
    r.x = m[0] * x + m[1] * y + m[2] * z + m[3] * w;
    r.y = m[4] * x + m[5] * y + m[6] * z + m[7] * w;
    r.z = m[8] * x + m[9] * y + m[10] * z + m[11] * w;
    r.w = m[12] * x + m[13] * y + m[14] * z + m[15] * w;
    return r;
}

typedef struct plane {
    float nx, ny, nz, d;
} plane;

/* Frustum::fromViewProj (remo_math.cuh:52-67) */
static void frustum_planes(const float* m, plane pl[6]) {
    const float* r0 = m;
    const float* r1 = m + 4;
    const float* r2 = m + 8;
    const float* r3 = m + 12;
    float v[6][4];
    for (int k = 0; k < 4; k++) {
        v[0][k] = r3[k] - r0[k];
        v[1][k] = r3[k] + r0[k];
        v[2][k] = r3[k] + r1[k];
        v[3][k] = r3[k] - r1[k];
        v[4][k] = r3[k] - r2[k];
        v[5][k] = r3[k] + r2[k];
    }
    for (int i = 0; i < 6; i++) {
        float a = v[i][0], b = v[i][1], c = v[i][2], d = v[i][3];
        float len = sqrtf(a * a + b * b + c * c);
        float inv = len > 0.0f ? 1.0f / len : 0.0f;
        pl[i].nx = a * inv;
        pl[i].ny = b * inv;
        pl[i].nz = c * inv;
        pl[i].d = d * inv;
    }
}

/* Frustum::intersectsBox (remo_math.cuh:69-79) */
static int frustum_box(const plane pl[6], const float mn[3], const float mx[3]) {
    for (int i = 0; i < 6; i++) {
        float px = pl[i].nx > 0.0f ? mx[0] : mn[0];
        float py = pl[i].ny > 0.0f ? mx[1] : mn[1];
        float pz = pl[i].nz > 0.0f ? mx[2] : mn[2];
        if (pl[i].nx * px + pl[i].ny * py + pl[i].nz * pz + pl[i].d < 0.0f) return 0;
    }
    return 1;
}

/* the node's projected box (projectedExtent, remolod_render.cu:40-70) in the
 * frozen transform: [minX, maxX, minY, maxY] */
static void box_extent(const or_frame* f, float cube, uint32_t level, uint32_t X, uint32_t Y, uint32_t Z,
                       float ext[4], int* any) {
    float s = cube / ldexpf(1.0f, (int)level);
    float mn[3] = {f->box_min[0] + (float)X * s, f->box_min[1] + (float)Y * s, f->box_min[2] + (float)Z * s};
    float minX = 1e30f, minY = 1e30f, maxX = -1e30f, maxY = -1e30f;
    *any = 0;
    for (int c = 0; c < 8; c++) {
        float x = (c & 1) ? mn[0] + s : mn[0];
        float y = (c & 2) ? mn[1] + s : mn[1];
        float z = (c & 4) ? mn[2] + s : mn[2];
        const float* m = f->transform_frozen;
        float cx = m[0] * x + m[1] * y + m[2] * z + m[3];
        float cy = m[4] * x + m[5] * y + m[6] * z + m[7];
        float cw = m[12] * x + m[13] * y + m[14] * z + m[15];
        if (cw <= 0.0f) continue;
        float iw = 1.0f / cw;
        float px = (cx * iw * 0.5f + 0.5f) * f->width, py = (cy * iw * 0.5f + 0.5f) * f->height;
        minX = fminf(minX, px);
        maxX = fmaxf(maxX, px);
        minY = fminf(minY, py);
        maxY = fmaxf(maxY, py);
        *any = 1;
    }
    ext[0] = minX;
    ext[1] = maxX;
    ext[2] = minY;
    ext[3] = maxY;
}

/* nodeBounds (remolod_render.cu:30-38) */
static void node_bounds(const or_frame* f, const onode* n, float cube_size, float mn[3], float mx[3],
                        float* size) {
    float s = cube_size / ldexpf(1.0f, (int)n->level);
    mn[0] = f->box_min[0] + (float)n->X * s;
    mn[1] = f->box_min[1] + (float)n->Y * s;
    mn[2] = f->box_min[2] + (float)n->Z * s;
    mx[0] = mn[0] + s;
    mx[1] = mn[1] + s;
    mx[2] = mn[2] + s;
    *size = s;
}

/* projectedExtent (remolod_render.cu:40-70) */
static void projected_extent(const float mn[3], const float mx[3], const float* m, float w, float h,
                             float* dx, float* dy) {
    *dx = 0.0f;
    *dy = 0.0f;
    float minX = 1e30f, minY = 1e30f, maxX = -1e30f, maxY = -1e30f;
    int any = 0;
    for (int c = 0; c < 8; c++) {
        float x = (c & 1) ? mx[0] : mn[0];
        float y = (c & 2) ? mx[1] : mn[1];
        float z = (c & 4) ? mx[2] : mn[2];
        f4 clip = matmul(m, x, y, z, 1.0f);
        if (clip.w <= 0.0f) continue;
        float invW = 1.0f / clip.w;
        float sx = (clip.x * invW * 0.5f + 0.5f) * w;
        float sy = (clip.y * invW * 0.5f + 0.5f) * h;
        minX = fminf(minX, sx);
        maxX = fmaxf(maxX, sx);
        minY = fminf(minY, sy);
        maxY = fmaxf(maxY, sy);
        any = 1;
    }
    if (!any) return;
    *dx = maxX - minX;
    *dy = maxY - minY;
}

/* remoDrawPoint (remo_framebuffer.cuh:33-61) */
static void draw_point(uint64_t* fb, const or_frame* f, float x, float y, float z, uint32_t color) {
    f4 clip = matmul(f->transform, x, y, z, 1.0f);
    if (clip.w <= 0.0f) return;
    float invW = 1.0f / clip.w;
    float ndcX = clip.x * invW;
    float ndcY = clip.y * invW;
    float px = (ndcX * 0.5f + 0.5f) * f->width;
    float py = (ndcY * 0.5f + 0.5f) * f->height;
    float depth = clip.w;
    int32_t half = f->point_size / 2;
    int32_t ix = cvt_s32(px), iy = cvt_s32(py);
    int32_t W = cvt_s32(f->width), H = cvt_s32(f->height);
    if ((int64_t)ix + half < 0 || (int64_t)iy + half < 0 || (int64_t)ix - half >= W ||
        (int64_t)iy - half >= H)
        return;
    uint32_t bits;
    memcpy(&bits, &depth, 4);
    uint64_t packed = ((uint64_t)bits << 32) | color;
    for (int32_t oy = -half; oy <= half; oy++) {
        int64_t sy = (int64_t)iy + oy;
        if (sy < 0 || sy >= H) continue;
        for (int32_t ox = -half; ox <= half; ox++) {
            int64_t sx = (int64_t)ix + ox;
            if (sx < 0 || sx >= W) continue;
            uint64_t* px_ = &fb[(uint64_t)sy * (uint64_t)W + (uint64_t)sx];
            if (packed < *px_) *px_ = packed;
        }
    }
}

/* remoHashColor (kernels/shared/remo_prelude.cuh:87-97) */
static uint32_t hash_color(uint64_t key) {
    uint64_t h = (key + 0x9E3779B97F4A7C15ull) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    uint32_t r = 96u + (((uint32_t)h & 0xFFu) * 159u) / 255u;
    uint32_t g = 96u + (((uint32_t)(h >> 8) & 0xFFu) * 159u) / 255u;
    uint32_t b = 96u + (((uint32_t)(h >> 16) & 0xFFu) * 159u) / 255u;
    return r | (g << 8) | (b << 16) | (255u << 24);
}

/* remoSampleColor (remo_draw.cuh:104-116); the item key is the node's index */
static uint32_t sample_color(int32_t mode, uint32_t node, uint32_t level, uint32_t rgba) {
    switch (mode) {
        case 1: return hash_color(node);
        case 2: return hash_color((uint64_t)level * 2654435761ull);
        case 3: return 0xFFFFFFFFu;
        default: return rgba;
    }
}

void or_render(const or_tree* t, const or_frame* f, uint64_t* fb, or_render_result* r,
               uint32_t* item_nodes) {
    const uint64_t npx = (uint64_t)f->width * (uint64_t)f->height;
    for (uint64_t i = 0; i < npx; i++) fb[i] = OR_FB_CLEAR;
    memset(r, 0, sizeof(*r));
    uint32_t nn = t->num_nodes;
    if (nn > t->cfg.max_nodes) nn = t->cfg.max_nodes;
    if (nn == 0) return;
    float sx = f->box_max[0] - f->box_min[0], sy = f->box_max[1] - f->box_min[1],
          sz = f->box_max[2] - f->box_min[2];
    float cube = fmaxf(fmaxf(sx, sy), sz);
    plane pl[6];
    frustum_planes(f->transform_frozen, pl);
    uint8_t* vis = (uint8_t*)calloc(nn, 1);
    uint8_t* large = (uint8_t*)calloc(nn, 1);
    if (!vis || !large) abort();
    for (uint32_t i = 0; i < nn; i++) {
        const onode* n = &t->nodes[i];
        float mn[3], mx[3], s;
        node_bounds(f, n, cube, mn, mx, &s);
        int has = n->num_points > 0 || n->num_voxels > 0;
        vis[i] = (has && frustum_box(pl, mn, mx)) ? 1 : 0;
        float dx, dy;
        projected_extent(mn, mx, f->transform_frozen, f->width, f->height, &dx, &dy);
        large[i] = (dx > f->lod_pixel_budget || dy > f->lod_pixel_budget) ? 1 : 0;
        if (f->force_large && f->force_large[i]) large[i] = 1;
    }
    const uint32_t ppc = t->cfg.points_per_chunk;
    uint32_t cap = f->drawlist_capacity ? f->drawlist_capacity : 131072u;
    for (uint32_t i = 0; i < nn; i++) {
        if (!large[i]) continue;
        const onode* n = &t->nodes[i];
        uint32_t targets[8];
        uint32_t nt = 0;
        if (!is_leaf(n)) {
            for (int c = 0; c < 8; c++) {
                int32_t ci = n->child[c];
                if (ci < 0 || (uint32_t)ci >= nn) continue;
                if (large[ci] || !vis[ci]) continue;
                targets[nt++] = (uint32_t)ci;
            }
        } else if (vis[i]) {
            targets[nt++] = i;
        }
        for (uint32_t k = 0; k < nt; k++) {
            const onode* tn = &t->nodes[targets[k]];
            if (tn->num_points == 0 && tn->num_voxels == 0) continue;
            if (r->draw_items >= cap) {
                r->drawlist_overflow = 1;
                r->draw_items++;
                continue;
            }
            if (item_nodes) item_nodes[r->draw_items] = targets[k];
            r->draw_items++;
            r->draw_samples += (uint64_t)tn->num_points + tn->num_voxels;
            /* the walker stops at the end of the chunk list (remo_draw.cuh:78-102) */
            uint32_t np = tn->num_points, pc = tn->num_point_chunks * ppc;
            if (np > pc) np = pc;
            const uint32_t tid = targets[k];
            for (uint32_t s = 0; s < np; s++)
                draw_point(fb, f, tn->pts[s].x, tn->pts[s].y, tn->pts[s].z,
                           sample_color(f->color_mode, tid, tn->level, tn->pts[s].color));
            uint32_t nv = tn->num_voxels, vc = tn->num_voxel_chunks * ppc;
            if (nv > vc) nv = vc;
            if (nv > tn->num_voxels_stored) nv = tn->num_voxels_stored;
            for (uint32_t s = 0; s < nv; s++)
                draw_point(fb, f, tn->vox[s].x, tn->vox[s].y, tn->vox[s].z,
                           sample_color(f->color_mode, tid, tn->level, tn->vox[s].color));
        }
    }
    free(vis);
    free(large);
}

/* ------------------------------------------------------------ Refinement */

typedef struct cf_cell {
    uint32_t cell, slot;
} cf_cell;

static int cmp_cf_cell(const void* a, const void* b) {
    uint32_t x = ((const cf_cell*)a)->cell, y = ((const cf_cell*)b)->cell;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* The cell a voxel of n stands for, from its centre (half a cell from either
 * boundary), with the CUDA path's float operations. */
static uint32_t voxel_cell(const or_tree* t, const onode* n, const or_point* v) {
    float size = t->octree_size / ldexpf(1.0f, (int)n->level);
    float scale = 128.0f / size;
    const uint32_t xyz[3] = {n->X, n->Y, n->Z};
    const float pv[3] = {v->x, v->y, v->z};
    uint32_t c[3];
    for (int a = 0; a < 3; a++) {
        float mn = fmaf((float)xyz[a], size, t->box_min[a]);
        float q = floorf((pv[a] - mn) * scale);
        int qi = (int)q;
        c[a] = (uint32_t)(qi < 0 ? 0 : (qi > 127 ? 127 : qi));
    }
    return c[0] + 128u * c[1] + 16384u * c[2];
}

typedef struct cf_sums {
    uint64_t r, g, b, n;
} cf_sums;

static void cf_add_points(const or_tree* t, const onode* leaf, uint32_t level, const cf_cell* cells, uint32_t nv,
                          cf_sums* sums) {
    uint32_t np = leaf->num_points, cap = leaf->num_point_chunks * t->cfg.points_per_chunk;
    if (np > cap) np = cap;
    const uint32_t sh = (uint32_t)OR_MAX_DEPTH + 1u - level;
    for (uint32_t s = 0; s < np; s++) {
        uint32_t q20[3], q28[3];
        quantize(t, &leaf->pts[s], q20, q28);
        uint32_t cell = ((q28[0] >> sh) & 127u) + ((q28[1] >> sh) & 127u) * 128u + ((q28[2] >> sh) & 127u) * 16384u;
        uint32_t lo = 0, hi = nv;
        while (lo < hi) {
            uint32_t mid = (lo + hi) / 2;
            if (cells[mid].cell < cell) lo = mid + 1;
            else hi = mid;
        }
        if (lo >= nv || cells[lo].cell != cell) continue;
        cf_sums* e = &sums[cells[lo].slot];
        uint32_t col = leaf->pts[s].color;
        e->r += col & 255u;
        e->g += (col >> 8) & 255u;
        e->b += (col >> 16) & 255u;
        e->n += 1;
    }
}

void or_refine_colors(or_tree* t, const uint32_t* nodes, uint32_t n, uint32_t capacity, uint32_t* nodes_filtered,
                      uint64_t* voxels_filtered) {
    const uint32_t ppc = t->cfg.points_per_chunk;
    uint64_t total = 0;
    uint32_t m = 0;
    for (; m < n; m++) {
        const onode* nd = &t->nodes[nodes[m]];
        uint32_t nv = nd->num_voxels, cap = nd->num_voxel_chunks * ppc;
        if (nv > nd->num_voxels_stored) nv = nd->num_voxels_stored;
        if (nv > cap) nv = cap;
        if (total + nv > capacity) break;
        total += nv;
    }
    uint32_t* stack = (uint32_t*)malloc((size_t)(t->num_nodes + 1) * sizeof(uint32_t));
    if (!stack) abort();
    for (uint32_t k = 0; k < m; k++) {
        onode* nd = &t->nodes[nodes[k]];
        uint32_t nv = nd->num_voxels, cap = nd->num_voxel_chunks * ppc;
        if (nv > nd->num_voxels_stored) nv = nd->num_voxels_stored;
        if (nv > cap) nv = cap;
        if (nv == 0) continue;
        cf_cell* cells = (cf_cell*)malloc((size_t)nv * sizeof(cf_cell));
        cf_sums* sums = (cf_sums*)calloc(nv, sizeof(cf_sums));
        if (!cells || !sums) abort();
        for (uint32_t s = 0; s < nv; s++) {
            cells[s].cell = voxel_cell(t, nd, &nd->vox[s]);
            cells[s].slot = s;
        }
        qsort(cells, nv, sizeof(cf_cell), cmp_cf_cell);
        /* every leaf of the subtree, the node itself if it is one */
        uint32_t top = 0;
        stack[top++] = nodes[k];
        while (top) {
            const onode* c = &t->nodes[stack[--top]];
            if (is_leaf(c)) {
                cf_add_points(t, c, nd->level, cells, nv, sums);
                continue;
            }
            for (int q = 0; q < 8; q++)
                if (c->child[q] >= 0) stack[top++] = (uint32_t)c->child[q];
        }
        for (uint32_t s = 0; s < nv; s++) {
            if (sums[s].n == 0) continue;
            uint64_t h = sums[s].n / 2;
            uint32_t r = (uint32_t)((sums[s].r + h) / sums[s].n), g = (uint32_t)((sums[s].g + h) / sums[s].n),
                     b = (uint32_t)((sums[s].b + h) / sums[s].n);
            nd->vox[s].color = (nd->vox[s].color & 0xFF000000u) | r | (g << 8) | (b << 16);
        }
        free(cells);
        free(sums);
    }
    free(stack);
    *nodes_filtered = m;
    *voxels_filtered = total;
}

/* remoClipSegment2D (remo_lines.cuh:30-55), one boundary */
static int clip_test(float p, float q, float* t0, float* t1) {
    if (p == 0.0f) return q >= 0.0f;
    float r = q / p;
    if (p < 0.0f) {
        if (r > *t1) return 0;
        if (r > *t0) *t0 = r;
    } else {
        if (r < *t0) return 0;
        if (r < *t1) *t1 = r;
    }
    return 1;
}

/* remoDrawSegment (remo_lines.cuh:57-117) */
static void draw_segment(uint64_t* fb, const or_frame* f, const float a[3], const float b[3], uint32_t color) {
    f4 c0 = matmul(f->transform, a[0], a[1], a[2], 1.0f);
    f4 c1 = matmul(f->transform, b[0], b[1], b[2], 1.0f);
    const float min_w = 1.0e-6f;
    if (c0.w < min_w && c1.w < min_w) return;
    if (c0.w < min_w) {
        float t = (min_w - c0.w) / (c1.w - c0.w);
        f4 c = {c0.x + t * (c1.x - c0.x), c0.y + t * (c1.y - c0.y), c0.z + t * (c1.z - c0.z), min_w};
        c0 = c;
    } else if (c1.w < min_w) {
        float t = (min_w - c1.w) / (c0.w - c1.w);
        f4 c = {c1.x + t * (c0.x - c1.x), c1.y + t * (c0.y - c1.y), c1.z + t * (c0.z - c1.z), min_w};
        c1 = c;
    }
    float iw0 = 1.0f / c0.w, iw1 = 1.0f / c1.w;
    float sx0 = (c0.x * iw0 * 0.5f + 0.5f) * f->width, sy0 = (c0.y * iw0 * 0.5f + 0.5f) * f->height;
    float sx1 = (c1.x * iw1 * 0.5f + 0.5f) * f->width, sy1 = (c1.y * iw1 * 0.5f + 0.5f) * f->height;
    int32_t W = cvt_s32(f->width), H = cvt_s32(f->height);
    if (W <= 0 || H <= 0) return;
    float dx = sx1 - sx0, dy = sy1 - sy0, t0 = 0.0f, t1 = 1.0f;
    if (!clip_test(-dx, sx0, &t0, &t1) || !clip_test(dx, (float)(W - 1) - sx0, &t0, &t1) ||
        !clip_test(-dy, sy0, &t0, &t1) || !clip_test(dy, (float)(H - 1) - sy0, &t0, &t1))
        return;
    float ax = sx0 + t0 * (sx1 - sx0), ay = sy0 + t0 * (sy1 - sy0);
    float bx = sx0 + t1 * (sx1 - sx0), by = sy0 + t1 * (sy1 - sy0);
    int32_t steps = cvt_s32(fmaxf(fabsf(bx - ax), fabsf(by - ay))) + 1;
    float inv_steps = 1.0f / (float)steps;
    for (int32_t st = 0; st <= steps; st++) {
        float q = (float)st * inv_steps;
        int32_t ix = cvt_s32(ax + q * (bx - ax)), iy = cvt_s32(ay + q * (by - ay));
        if (ix < 0 || iy < 0 || ix >= W || iy >= H) continue;
        float s_t = t0 + q * (t1 - t0);
        float iw = iw0 + s_t * (iw1 - iw0);
        if (!(iw > 0.0f)) continue;
        float depth = 1.0f / iw;
        uint32_t bits;
        memcpy(&bits, &depth, 4);
        uint64_t packed = ((uint64_t)bits << 32) | color;
        uint64_t* px = &fb[(uint64_t)iy * (uint64_t)W + (uint64_t)ix];
        if (packed < *px) *px = packed;
    }
}

void or_wireframe(const or_tree* t, const or_frame* f, uint64_t* fb, const uint32_t* item_nodes, uint32_t n) {
    float cube = fmaxf(fmaxf(f->box_max[0] - f->box_min[0], f->box_max[1] - f->box_min[1]),
                       f->box_max[2] - f->box_min[2]);
    for (uint32_t k = 0; k < n; k++) {
        const onode* nd = &t->nodes[item_nodes[k]];
        float mn[3], mx[3], size;
        node_bounds(f, nd, cube, mn, mx, &size);
        if (!(size > 0.0f)) continue;
        uint32_t color = hash_color((uint64_t)nd->level * 2654435761ull);
        /* remoBoxEdge (remo_lines.cuh:11-27) */
        for (uint32_t e = 0; e < 12; e++) {
            uint32_t axis = e / 4u, rest = e % 4u;
            float off[3] = {0.0f, 0.0f, 0.0f};
            off[(axis + 1u) % 3u] = (rest & 1u) ? size : 0.0f;
            off[(axis + 2u) % 3u] = (rest & 2u) ? size : 0.0f;
            float a[3] = {mn[0] + off[0], mn[1] + off[1], mn[2] + off[2]};
            off[axis] = size;
            float b[3] = {mn[0] + off[0], mn[1] + off[1], mn[2] + off[2]};
            draw_segment(fb, f, a, b, color);
        }
    }
}

void or_render_flat(const or_point* pts, uint64_t n, const or_frame* f, uint64_t* fb) {
    const uint64_t npx = (uint64_t)f->width * (uint64_t)f->height;
    for (uint64_t i = 0; i < npx; i++) fb[i] = OR_FB_CLEAR;
    for (uint64_t i = 0; i < n; i++) draw_point(fb, f, pts[i].x, pts[i].y, pts[i].z, pts[i].color);
}

static float fb_depth(uint64_t px) {
    uint32_t bits = (uint32_t)(px >> 32);
    float d;
    memcpy(&d, &bits, 4);
    return d;
}

void or_edl(uint64_t* fb, uint32_t width, uint32_t height, float strength) {
    uint64_t npx = (uint64_t)width * height;
    uint64_t* src = (uint64_t*)malloc(npx * sizeof(uint64_t));
    if (!src) abort();
    memcpy(src, fb, npx * sizeof(uint64_t));
    const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    for (uint64_t i = 0; i < npx; i++) {
        int32_t x = (int32_t)(i % width), y = (int32_t)(i / width);
        float depth = fb_depth(src[i]);
        if (!(depth < 3.0e38f)) continue;
        float ld = log2f(depth);
        float resp = 0.0f;
        int taps = 0;
        for (int k = 0; k < 4; k++) {
            int32_t nx = x + off[k][0], ny = y + off[k][1];
            if (nx < 0 || ny < 0 || nx >= (int32_t)width || ny >= (int32_t)height) continue;
            float nd = fb_depth(src[(uint64_t)ny * width + nx]);
            if (!(nd < 3.0e38f)) continue;
            resp += fmaxf(0.0f, ld - log2f(nd));
            taps++;
        }
        if (taps == 0) continue;
        resp /= (float)taps;
        float shade = expf(-resp * 24.0f * strength);
        uint32_t c = (uint32_t)src[i];
        uint32_t r = (uint32_t)((float)(c & 255u) * shade);
        uint32_t g = (uint32_t)((float)((c >> 8) & 255u) * shade);
        uint32_t b = (uint32_t)((float)((c >> 16) & 255u) * shade);
        uint32_t packed = r | (g << 8) | (b << 16) | (255u << 24);
        fb[i] = (src[i] & 0xFFFFFFFF00000000ull) | packed;
    }
    free(src);
}
