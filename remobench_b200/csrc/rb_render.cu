// Rasterize stage: frustum test, pixel-budget LOD cut, one block per visible
// node, 64-bit depth|colour atomicMin splatting into a headless framebuffer.
//
// Restates kernels/remolod/remolod_render.cu:30-198 and
// kernels/shared/remo_{math,framebuffer,draw}.cuh. The framebuffer packs
// (float_bits(depth) << 32) | rgba, so atomicMin keeps the nearest sample and,
// on a depth tie, the smaller colour: the result does not depend on the order
// samples arrive in, which is what makes it bit-comparable with the CPU oracle.
//
// This file is compiled with -fmad=false: every float operation below rounds
// once, as in the oracle (compiled with -ffp-contract=off).
#include <cuda_runtime.h>

#include "rb_kernels.h"
#include "rb_state.h"

namespace rb {

constexpr unsigned long long kFbClear = 0x7f80000000332211ull;  // REMO_FB_CLEAR

struct F4 {
    float x, y, z, w;
};

// remoMatMul (remo_math.cuh:25-32)
__device__ __forceinline__ F4 matmul(const float* m, float x, float y, float z, float w) {
    F4 r;
    r.x = m[0] * x + m[1] * y + m[2] * z + m[3] * w;
    r.y = m[4] * x + m[5] * y + m[6] * z + m[7] * w;
    r.z = m[8] * x + m[9] * y + m[10] * z + m[11] * w;
    r.w = m[12] * x + m[13] * y + m[14] * z + m[15] * w;
    return r;
}

struct Plane {
    float nx, ny, nz, d;
};

// Frustum::fromViewProj (remo_math.cuh:52-67)
__device__ void frustumPlanes(const float* m, Plane pl[6]) {
    float v[6][4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[0][k] = m[12 + k] - m[k];
        v[1][k] = m[12 + k] + m[k];
        v[2][k] = m[12 + k] + m[4 + k];
        v[3][k] = m[12 + k] - m[4 + k];
        v[4][k] = m[12 + k] - m[8 + k];
        v[5][k] = m[12 + k] + m[8 + k];
    }
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const float a = v[i][0], b = v[i][1], c = v[i][2], dd = v[i][3];
        const float len = sqrtf(a * a + b * b + c * c);
        const float inv = len > 0.0f ? 1.0f / len : 0.0f;
        pl[i].nx = a * inv;
        pl[i].ny = b * inv;
        pl[i].nz = c * inv;
        pl[i].d = dd * inv;
    }
}

__device__ __forceinline__ bool frustumBox(const Plane* pl, const float mn[3], const float mx[3]) {
#pragma unroll
    for (int i = 0; i < 6; i++) {
        const float px = pl[i].nx > 0.0f ? mx[0] : mn[0];
        const float py = pl[i].ny > 0.0f ? mx[1] : mn[1];
        const float pz = pl[i].nz > 0.0f ? mx[2] : mn[2];
        if (pl[i].nx * px + pl[i].ny * py + pl[i].nz * pz + pl[i].d < 0.0f) return false;
    }
    return true;
}

__device__ __forceinline__ bool leafRowR(const Dev& d, uint32_t node) {
    const int4* row = reinterpret_cast<const int4*>(d.child + node * 8u);
    const int4 a = row[0], b = row[1];
    return (a.x & a.y & a.z & a.w & b.x & b.y & b.z & b.w) == -1;
}

// remoDrawPoint (remo_framebuffer.cuh:33-61)
__device__ __forceinline__ void drawPoint(unsigned long long* fb, const Frame& f, float x, float y,
                                          float z, uint32_t color) {
    const F4 clip = matmul(f.transform, x, y, z, 1.0f);
    if (clip.w <= 0.0f) return;
    const float invW = 1.0f / clip.w;
    const float ndcX = clip.x * invW;
    const float ndcY = clip.y * invW;
    const float px = (ndcX * 0.5f + 0.5f) * f.width;
    const float py = (ndcY * 0.5f + 0.5f) * f.height;
    const int32_t half = f.pointSize / 2;
    const int32_t ix = __float2int_rz(px), iy = __float2int_rz(py);
    const int32_t W = __float2int_rz(f.width), H = __float2int_rz(f.height);
    if ((long long)ix + half < 0 || (long long)iy + half < 0 || (long long)ix - half >= W ||
        (long long)iy - half >= H)
        return;
    const unsigned long long packed =
        ((unsigned long long)__float_as_uint(clip.w) << 32) | (unsigned long long)color;
    for (int32_t oy = -half; oy <= half; ++oy) {
        const long long sy = (long long)iy + oy;
        if (sy < 0 || sy >= H) continue;
        for (int32_t ox = -half; ox <= half; ++ox) {
            const long long sx = (long long)ix + ox;
            if (sx < 0 || sx >= W) continue;
            atomicMin(&fb[(unsigned long long)sy * (unsigned long long)W + (unsigned long long)sx], packed);
        }
    }
}

__global__ void __launch_bounds__(256) k_fb_clear(unsigned long long* fb, uint64_t npx) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npx;
         i += (uint64_t)gridDim.x * blockDim.x)
        fb[i] = kFbClear;
}

// Pass 1 (remolod_render.cu:113-131): visible and large per node.
__global__ void __launch_bounds__(256) k_node_flags(Dev d, Frame f, uint8_t* vis, uint8_t* large,
                                                    const uint8_t* forceLarge, RenderScratch* rs) {
    __shared__ Plane s_pl[6];
    if (threadIdx.x == 0) {
        Plane pl[6];
        frustumPlanes(f.transformFrozen, pl);
        for (int i = 0; i < 6; i++) s_pl[i] = pl[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        rs->numItems = 0;
        rs->overflow = 0;
        rs->samples = 0;
    }
    __syncthreads();
    uint32_t nn = d.ctr->numNodes;
    if (nn > d.maxNodes) nn = d.maxNodes;
    const float cube = fmaxf(fmaxf(f.boxMax[0] - f.boxMin[0], f.boxMax[1] - f.boxMin[1]),
                             f.boxMax[2] - f.boxMin[2]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const float s = cube / __int_as_float((int)((127u + d.level[i]) << 23));
        float mn[3], mx[3];
        mn[0] = f.boxMin[0] + (float)d.nodeX[i] * s;
        mn[1] = f.boxMin[1] + (float)d.nodeY[i] * s;
        mn[2] = f.boxMin[2] + (float)d.nodeZ[i] * s;
        mx[0] = mn[0] + s;
        mx[1] = mn[1] + s;
        mx[2] = mn[2] + s;
        const bool has = d.numPoints[i] > 0 || d.numVoxels[i] > 0;
        vis[i] = (has && frustumBox(s_pl, mn, mx)) ? 1 : 0;
        // projectedExtent (remolod_render.cu:40-70)
        float minX = 1e30f, minY = 1e30f, maxX = -1e30f, maxY = -1e30f;
        bool any = false;
        for (int corner = 0; corner < 8; corner++) {
            const float x = (corner & 1) ? mx[0] : mn[0];
            const float y = (corner & 2) ? mx[1] : mn[1];
            const float z = (corner & 4) ? mx[2] : mn[2];
            const F4 clip = matmul(f.transformFrozen, x, y, z, 1.0f);
            if (clip.w <= 0.0f) continue;
            const float invW = 1.0f / clip.w;
            const float sx = (clip.x * invW * 0.5f + 0.5f) * f.width;
            const float sy = (clip.y * invW * 0.5f + 0.5f) * f.height;
            minX = fminf(minX, sx);
            maxX = fmaxf(maxX, sx);
            minY = fminf(minY, sy);
            maxY = fmaxf(maxY, sy);
            any = true;
        }
        float dx = 0.0f, dy = 0.0f;
        if (any) {
            dx = maxX - minX;
            dy = maxY - minY;
        }
        bool lg = dx > f.lodPixelBudget || dy > f.lodPixelBudget;
        if (forceLarge && forceLarge[i]) lg = true;
        large[i] = lg ? 1 : 0;
    }
}

// Pass 2 (remolod_render.cu:134-178): the disjoint frontier. A large inner node
// emits its visible children that are not large; a large visible leaf emits
// itself.
__global__ void __launch_bounds__(256) k_frontier(Dev d, const uint8_t* vis, const uint8_t* large,
                                                  RenderScratch* rs, uint32_t* items, uint32_t cap) {
    uint32_t nn = d.ctr->numNodes;
    if (nn > d.maxNodes) nn = d.maxNodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        if (!large[i]) continue;
        uint32_t targets[8];
        uint32_t nt = 0;
        if (!leafRowR(d, i)) {
            for (int c = 0; c < 8; c++) {
                const int32_t ci = d.child[i * 8u + c];
                if (ci < 0 || (uint32_t)ci >= nn) continue;
                if (large[ci] || !vis[ci]) continue;
                targets[nt++] = (uint32_t)ci;
            }
        } else if (vis[i]) {
            targets[nt++] = i;
        }
        for (uint32_t k = 0; k < nt; k++) {
            const uint32_t t = targets[k];
            const uint32_t np = d.numPoints[t], nv = d.numVoxels[t];
            if (np == 0 && nv == 0) continue;
            const uint32_t idx = atomicAdd(&rs->numItems, 1u);
            if (idx >= cap) {
                rs->overflow = 1;
                continue;
            }
            items[idx] = t;
            atomicAdd(&rs->samples, (unsigned long long)np + nv);
        }
    }
}

// remoHashColor (kernels/shared/remo_prelude.cuh:87-97): a splitmix-style
// hash of the key, each channel mapped to [96, 255], alpha 255.
__device__ __forceinline__ uint32_t hashColor(unsigned long long key) {
    unsigned long long h = (key + 0x9E3779B97F4A7C15ull) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    const uint32_t r = 96u + (((uint32_t)h & 0xFFu) * 159u) / 255u;
    const uint32_t g = 96u + (((uint32_t)(h >> 8) & 0xFFu) * 159u) / 255u;
    const uint32_t b = 96u + (((uint32_t)(h >> 16) & 0xFFu) * 159u) / 255u;
    return r | (g << 8) | (b << 16) | (255u << 24);
}

// remoSampleColor (remo_draw.cuh:104-116): the colour every sample of a draw
// item takes in the non-RGB modes; the item key is the node's pool index.
__device__ __forceinline__ uint32_t itemColor(int32_t mode, uint32_t node, uint32_t level) {
    if (mode == 3) return 0xFFFFFFFFu;
    if (mode == 1) return hashColor(node);
    return hashColor((unsigned long long)level * 2654435761ull);
}

// remoRasterizeDrawList (remo_draw.cuh:118-167): one block per draw item; the
// block walks the node's chunks in order, so the loads of a chunk coalesce.
__global__ void __launch_bounds__(256) k_raster(Dev d, Frame f, unsigned long long* fb,
                                                const RenderScratch* rs, const uint32_t* items,
                                                uint32_t cap) {
    uint32_t ni = rs->numItems;
    if (ni > cap) ni = cap;
    const uint32_t ppc = d.ppc;
    for (uint32_t w = blockIdx.x; w < ni; w += gridDim.x) {
        const uint32_t node = items[w];
        const bool rgb = f.colorMode < 1 || f.colorMode > 3;
        const uint32_t fixed = rgb ? 0u : itemColor(f.colorMode, node, d.level[node]);
        uint32_t np = d.numPoints[node];
        const uint32_t pcap = d.numPointChunks[node] * ppc;
        if (np > pcap) np = pcap;
        const uint32_t poff = d.ptTableOff[node];
        // four samples per thread, each step's loads issued for all four first
        for (uint32_t s0 = threadIdx.x; s0 < np; s0 += 4u * blockDim.x) {
            float4 v[4];
            bool ok[4];
#pragma unroll
            for (uint32_t j = 0; j < 4u; j++) {
                const uint32_t s = s0 + j * blockDim.x;
                const uint32_t phys = s < np ? d.tablePool[poff + s / ppc] : kNone;
                ok[j] = phys != kNone;
                v[j] = ok[j] ? __ldg(reinterpret_cast<const float4*>(chunkPoints(d, phys) + s % ppc))
                             : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (uint32_t j = 0; j < 4u; j++)
                if (ok[j]) drawPoint(fb, f, v[j].x, v[j].y, v[j].z, rgb ? __float_as_uint(v[j].w) : fixed);
        }
        uint32_t nv = d.numVoxels[node];
        const uint32_t vcap = d.numVoxelChunks[node] * ppc;
        if (nv > vcap) nv = vcap;
        if (nv > d.numVoxelsStored[node]) nv = d.numVoxelsStored[node];
        const uint32_t voff = d.vxTableOff[node];
        for (uint32_t s0 = threadIdx.x; s0 < nv; s0 += 4u * blockDim.x) {
            float4 v[4];
            bool ok[4];
#pragma unroll
            for (uint32_t j = 0; j < 4u; j++) {
                const uint32_t s = s0 + j * blockDim.x;
                const uint32_t phys = s < nv ? d.tablePool[voff + s / ppc] : kNone;
                ok[j] = phys != kNone;
                v[j] = ok[j] ? __ldg(reinterpret_cast<const float4*>(chunkPoints(d, phys) + s % ppc))
                             : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (uint32_t j = 0; j < 4u; j++)
                if (ok[j]) drawPoint(fb, f, v[j].x, v[j].y, v[j].z, rgb ? __float_as_uint(v[j].w) : fixed);
        }
    }
}

// remoClipSegment2D (remo_lines.cuh:30-55): Liang-Barsky against
// [0, xmax] x [0, ymax]; false when the segment misses.
__device__ __forceinline__ bool clipTest(float p, float q, float& t0, float& t1) {
    if (p == 0.0f) return q >= 0.0f;
    const float r = q / p;
    if (p < 0.0f) {
        if (r > t1) return false;
        if (r > t0) t0 = r;
    } else {
        if (r < t0) return false;
        if (r < t1) t1 = r;
    }
    return true;
}

// remoDrawSegment (remo_lines.cuh:57-117): near-plane clip in clip space at
// w = 1e-6, screen clip, then one sample per step along the longer axis with
// depth from the interpolated 1/w.
__device__ void drawSegment(unsigned long long* fb, const Frame& f, float ax0, float ay0, float az0, float bx0,
                            float by0, float bz0, uint32_t color) {
    F4 c0 = matmul(f.transform, ax0, ay0, az0, 1.0f);
    F4 c1 = matmul(f.transform, bx0, by0, bz0, 1.0f);
    const float kMinW = 1.0e-6f;
    if (c0.w < kMinW && c1.w < kMinW) return;
    if (c0.w < kMinW) {
        const float t = (kMinW - c0.w) / (c1.w - c0.w);
        c0 = F4{c0.x + t * (c1.x - c0.x), c0.y + t * (c1.y - c0.y), c0.z + t * (c1.z - c0.z), kMinW};
    } else if (c1.w < kMinW) {
        const float t = (kMinW - c1.w) / (c0.w - c1.w);
        c1 = F4{c1.x + t * (c0.x - c1.x), c1.y + t * (c0.y - c1.y), c1.z + t * (c0.z - c1.z), kMinW};
    }
    const float invW0 = 1.0f / c0.w, invW1 = 1.0f / c1.w;
    const float sx0 = (c0.x * invW0 * 0.5f + 0.5f) * f.width;
    const float sy0 = (c0.y * invW0 * 0.5f + 0.5f) * f.height;
    const float sx1 = (c1.x * invW1 * 0.5f + 0.5f) * f.width;
    const float sy1 = (c1.y * invW1 * 0.5f + 0.5f) * f.height;
    const int32_t W = __float2int_rz(f.width), H = __float2int_rz(f.height);
    if (W <= 0 || H <= 0) return;
    const float dx = sx1 - sx0, dy = sy1 - sy0;
    float t0 = 0.0f, t1 = 1.0f;
    if (!clipTest(-dx, sx0, t0, t1) || !clipTest(dx, (float)(W - 1) - sx0, t0, t1) || !clipTest(-dy, sy0, t0, t1) ||
        !clipTest(dy, (float)(H - 1) - sy0, t0, t1))
        return;
    const float ax = sx0 + t0 * (sx1 - sx0), ay = sy0 + t0 * (sy1 - sy0);
    const float bx = sx0 + t1 * (sx1 - sx0), by = sy0 + t1 * (sy1 - sy0);
    const int32_t steps = __float2int_rz(fmaxf(fabsf(bx - ax), fabsf(by - ay))) + 1;
    const float invSteps = 1.0f / (float)steps;
    for (int32_t st = 0; st <= steps; ++st) {
        const float q = (float)st * invSteps;
        const int32_t ix = __float2int_rz(ax + q * (bx - ax));
        const int32_t iy = __float2int_rz(ay + q * (by - ay));
        if (ix < 0 || iy < 0 || ix >= W || iy >= H) continue;
        const float sT = t0 + q * (t1 - t0);
        const float invW = invW0 + sT * (invW1 - invW0);
        if (!(invW > 0.0f)) continue;
        const float depth = 1.0f / invW;
        atomicMin(&fb[(unsigned long long)iy * (unsigned long long)W + (unsigned long long)ix],
                  ((unsigned long long)__float_as_uint(depth) << 32) | (unsigned long long)color);
    }
}

// remoDrawListWireframe (remo_lines.cuh:120-137): the 12 edges of every draw
// item's node box (remoBoxEdge, :11-27: edge / 4 is the axis the edge runs
// along, edge % 4 picks the offsets on the other two), coloured by level.
__global__ void __launch_bounds__(256) k_wireframe(Dev d, Frame f, unsigned long long* fb,
                                                   const RenderScratch* rs, const uint32_t* items, uint32_t cap) {
    uint32_t ni = rs->numItems;
    if (ni > cap) ni = cap;
    const float cube = fmaxf(fmaxf(f.boxMax[0] - f.boxMin[0], f.boxMax[1] - f.boxMin[1]), f.boxMax[2] - f.boxMin[2]);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (uint64_t)ni * 12u;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t node = items[i / 12u];
        const uint32_t edge = (uint32_t)(i % 12u);
        const uint32_t lv = d.level[node];
        const float size = cube / __int_as_float((int)((127u + lv) << 23));
        if (!(size > 0.0f)) continue;
        const float mn[3] = {f.boxMin[0] + (float)d.nodeX[node] * size, f.boxMin[1] + (float)d.nodeY[node] * size,
                             f.boxMin[2] + (float)d.nodeZ[node] * size};
        const uint32_t axis = edge / 4u, rest = edge % 4u;
        float off[3] = {0.0f, 0.0f, 0.0f};
        off[(axis + 1u) % 3u] = (rest & 1u) ? size : 0.0f;
        off[(axis + 2u) % 3u] = (rest & 2u) ? size : 0.0f;
        const float a[3] = {mn[0] + off[0], mn[1] + off[1], mn[2] + off[2]};
        off[axis] = size;
        drawSegment(fb, f, a[0], a[1], a[2], mn[0] + off[0], mn[1] + off[1], mn[2] + off[2],
                    hashColor((unsigned long long)lv * 2654435761ull));
    }
}

// flat_render.cu:9-76: every point of a resident cloud.
__global__ void __launch_bounds__(256) k_raster_flat(Frame f, unsigned long long* fb,
                                                     const Point* __restrict__ pts, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(pts + i));
        drawPoint(fb, f, v.x, v.y, v.z, __float_as_uint(v.w));
    }
}

__device__ __forceinline__ float fbDepth(unsigned long long px) {
    return __uint_as_float((uint32_t)(px >> 32));
}

// remoApplyEDL (remo_framebuffer.cuh:78-122); libm log2f/expf in place of
// the reference's __log2f/__expf. It may run in place (src == dst): a pixel
// reads its neighbours' depths only, and shading rewrites a pixel's colour
// half only, so the result does not depend on which neighbours were already
// shaded.
__global__ void __launch_bounds__(256) k_edl(const unsigned long long* src, unsigned long long* dst,
                                             uint32_t width, uint32_t height, float strength) {
    const uint64_t npx = (uint64_t)width * height;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npx;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long pixel = src[i];
        if (dst != src) dst[i] = pixel;
        const int32_t x = (int32_t)(i % width), y = (int32_t)(i / width);
        const float depth = fbDepth(pixel);
        if (!(depth < 3.0e38f)) continue;
        const float ld = log2f(depth);
        float resp = 0.0f;
        int taps = 0;
        const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
        for (int k = 0; k < 4; k++) {
            const int32_t nx = x + off[k][0], ny = y + off[k][1];
            if (nx < 0 || ny < 0 || nx >= (int32_t)width || ny >= (int32_t)height) continue;
            const float nd = fbDepth(src[(uint64_t)ny * width + nx]);
            if (!(nd < 3.0e38f)) continue;
            resp += fmaxf(0.0f, ld - log2f(nd));
            taps++;
        }
        if (taps == 0) continue;
        resp /= (float)taps;
        const float shade = expf(-resp * 24.0f * strength);
        const uint32_t c = (uint32_t)pixel;
        const uint32_t r = (uint32_t)((float)(c & 255u) * shade);
        const uint32_t g = (uint32_t)((float)((c >> 8) & 255u) * shade);
        const uint32_t b = (uint32_t)((float)((c >> 16) & 255u) * shade);
        dst[i] = (pixel & 0xFFFFFFFF00000000ull) | (unsigned long long)(r | (g << 8) | (b << 16) | (255u << 24));
    }
}

// remoResolve (remo_framebuffer.cuh:63-76) into a plain RGBA buffer.
__global__ void __launch_bounds__(256) k_resolve(const unsigned long long* fb, uint32_t* rgba, uint64_t npx) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npx;
         i += (uint64_t)gridDim.x * blockDim.x)
        rgba[i] = (uint32_t)fb[i];
}

void launchFbClear(unsigned long long* fb, uint64_t npx, int grid, cudaStream_t s) {
    k_fb_clear<<<grid, 256, 0, s>>>(fb, npx);
}
void launchNodeFlags(const Dev& d, const Frame& f, uint8_t* vis, uint8_t* large, const uint8_t* force,
                     RenderScratch* rs, int grid, cudaStream_t s) {
    k_node_flags<<<grid, 256, 0, s>>>(d, f, vis, large, force, rs);
}
void launchFrontier(const Dev& d, const uint8_t* vis, const uint8_t* large, RenderScratch* rs,
                    uint32_t* items, uint32_t cap, int grid, cudaStream_t s) {
    k_frontier<<<grid, 256, 0, s>>>(d, vis, large, rs, items, cap);
}
void launchRaster(const Dev& d, const Frame& f, unsigned long long* fb, const RenderScratch* rs,
                  const uint32_t* items, uint32_t cap, int grid, cudaStream_t s) {
    k_raster<<<grid, 256, 0, s>>>(d, f, fb, rs, items, cap);
}
void launchRasterFlat(const Frame& f, unsigned long long* fb, const Point* pts, uint64_t n, int grid,
                      cudaStream_t s) {
    k_raster_flat<<<grid, 256, 0, s>>>(f, fb, pts, n);
}
void launchEdl(const unsigned long long* src, unsigned long long* dst, uint32_t w, uint32_t h, float strength,
               int grid, cudaStream_t s) {
    k_edl<<<grid, 256, 0, s>>>(src, dst, w, h, strength);
}
void launchResolve(const unsigned long long* fb, uint32_t* rgba, uint64_t npx, int grid, cudaStream_t s) {
    k_resolve<<<grid, 256, 0, s>>>(fb, rgba, npx);
}
void launchWireframe(const Dev& d, const Frame& f, unsigned long long* fb, const RenderScratch* rs,
                     const uint32_t* items, uint32_t cap, int grid, cudaStream_t s) {
    k_wireframe<<<grid, 256, 0, s>>>(d, f, fb, rs, items, cap);
}

}  // namespace rb
