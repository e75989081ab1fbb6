// Analysis stage: roll the leaves' exact sums up the tree, finalise each
// node's centred covariance, solve the 3x3 symmetric eigenproblem, score each
// node by surface variation x screen coverage, and rebuild the per-frame
// priority queue.
//
// The reference specifies this stage in prose only (wiki/02_KernelPipeline.md:204-224,
// README.md:30-48, plans/01_NoveltyAssessment.md:44-46); there is no kernel to
// follow. Conventions fixed here: eigenvalues are descending, l1 >= l2 >= l3,
// in units of (node size)^2; surface variation = l3 / (l1 + l2 + l3);
// planarity = (l2 - l3) / l1; closure = the node's subtree received no point
// for `closure_margin` batches (lastTouchedBatch plus a batch-age margin,
// wiki/02_KernelPipeline.md:215-221; the Morton watermark is not a closure
// test because no reader emits Morton order).
//
// Arithmetic: the roll-up is exact (64/128-bit integers, children re-based to
// the parent's origin); the centred scatter n*Sxx - Sx*Sx is exact in 128 bits
// and is converted to FP64 once; the eigen-solve is the closed-form
// trigonometric method (O. K. Smith, "Eigenvalues of a symmetric 3x3 matrix",
// CACM 4(4):168, 1961) in FP32, with a cyclic Jacobi in FP64 for near-degenerate
// matrices (l3 < 1e-3 * l1, or a nearly diagonal matrix).
#include <cuda_runtime.h>

#include "rb_analysis.h"
#include "rb_kernels.h"
#include "rb_state.h"

namespace rb {

typedef unsigned __int128 u128;
typedef __int128 i128;

__device__ __forceinline__ bool leafA(const Dev& d, uint32_t node) {
    const int4* row = reinterpret_cast<const int4*>(d.child + node * 8u);
    const int4 a = row[0], b = row[1];
    return (a.x & a.y & a.z & a.w & b.x & b.y & b.z & b.w) == -1;
}

// One level of the roll-up: leaves copy their accumulator; inner nodes add
// their children, each re-based by its offset o (0 or half the parent) in the
// parent's 2^(28 - L) grid: S1 += n o, S2_ab += o_a S1_b + o_b S1_a + n o_a o_b.
__global__ void __launch_bounds__(256) k_roll_level(Dev d, RollSum* roll, uint32_t level) {
    const uint32_t nn = d.ctr->numNodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        if (d.level[i] != level) continue;
        RollSum r;
        if (leafA(d, i)) {
            const AccumI& a = d.accum[i];
            r.n = a.count;
            for (int k = 0; k < 3; k++) r.s1[k] = a.s1[k];
            for (int k = 0; k < 6; k++) {
                r.s2[2 * k] = a.s2lo[k];
                r.s2[2 * k + 1] = a.s2hi[k];
            }
            for (int k = 0; k < 3; k++) {
                r.c1[k] = a.c1[k];
                r.c2[k] = a.c2[k];
            }
            r.lastTouched = a.count ? a.lastTouchedBatch : 0u;
            r.pad = 0;
        } else {
            unsigned long long cc1[3] = {0, 0, 0}, cc2[3] = {0, 0, 0};
            u128 s1[3] = {0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
            u128 n = 0;
            uint32_t lt = 0;
            const uint32_t sh = 28u - (level + 1u);
            for (int c = 0; c < 8; c++) {
                const int32_t ci = d.child[i * 8u + c];
                if (ci < 0) continue;
                const RollSum& cr = roll[ci];
                if (cr.n == 0) continue;
                const u128 cn = cr.n;
                const u128 o[3] = {(u128)((c >> 2) & 1) << sh, (u128)((c >> 1) & 1) << sh, (u128)(c & 1) << sh};
                const u128 c1[3] = {cr.s1[0], cr.s1[1], cr.s1[2]};
                n += cn;
                for (int k = 0; k < 3; k++) s1[k] += c1[k] + cn * o[k];
                const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
                for (int k = 0; k < 6; k++) {
                    const u128 c2 = ((u128)cr.s2[2 * k + 1] << 64) | cr.s2[2 * k];
                    s2[k] += c2 + o[pa[k]] * c1[pb[k]] + o[pb[k]] * c1[pa[k]] + cn * o[pa[k]] * o[pb[k]];
                }
                lt = cr.lastTouched > lt ? cr.lastTouched : lt;
                for (int k = 0; k < 3; k++) {
                    cc1[k] += cr.c1[k];
                    cc2[k] += cr.c2[k];
                }
            }
            for (int k = 0; k < 3; k++) {
                r.c1[k] = cc1[k];
                r.c2[k] = cc2[k];
            }
            r.n = (unsigned long long)n;
            for (int k = 0; k < 3; k++) r.s1[k] = (unsigned long long)s1[k];
            for (int k = 0; k < 6; k++) {
                r.s2[2 * k] = (unsigned long long)s2[k];
                r.s2[2 * k + 1] = (unsigned long long)(s2[k] >> 64);
            }
            r.lastTouched = lt;
            r.pad = 0;
        }
        roll[i] = r;
    }
}

__device__ __forceinline__ double i128ToDouble(i128 v) {
    const bool neg = v < 0;
    const u128 m = neg ? (u128)(-v) : (u128)v;
    const double hi = (double)(unsigned long long)(m >> 64);
    const double lo = (double)(unsigned long long)m;
    const double r = hi * 18446744073709551616.0 + lo;
    return neg ? -r : r;
}

// Cyclic Jacobi on a symmetric 3x3 in FP64; eigenvalues descending, the
// eigenvector of the smallest in vmin.
__device__ void jacobi3(const double ain[6], double eig[3], double vmin[3]) {
    double a[3][3] = {{ain[0], ain[1], ain[2]}, {ain[1], ain[3], ain[4]}, {ain[2], ain[4], ain[5]}};
    double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 32; sweep++) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-36 * diag || off == 0.0) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0.0) continue;
                const double th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    const double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = c * vkp - s * vkq;
                    v[k][q] = s * vkp + c * vkq;
                }
            }
    }
    int o[3] = {0, 1, 2};
    const double dg[3] = {a[0][0], a[1][1], a[2][2]};
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (dg[o[j]] > dg[o[i]]) {
                const int t = o[i];
                o[i] = o[j];
                o[j] = t;
            }
    for (int i = 0; i < 3; i++) eig[i] = dg[o[i]];
    for (int k = 0; k < 3; k++) vmin[k] = v[k][o[2]];
}

// Smith's closed form in FP32. Returns false when the matrix is too close to
// degenerate for it (the caller then takes the FP64 branch).
__device__ bool smith3(const float a[6], float eig[3]) {
    const float p1 = a[1] * a[1] + a[2] * a[2] + a[4] * a[4];
    const float q = (a[0] + a[3] + a[5]) * (1.0f / 3.0f);
    const float b00 = a[0] - q, b11 = a[3] - q, b22 = a[5] - q;
    const float p2 = b00 * b00 + b11 * b11 + b22 * b22 + 2.0f * p1;
    if (!(p2 > 0.0f)) return false;
    const float p = sqrtf(p2 * (1.0f / 6.0f));
    if (p1 < 1e-12f * p2) return false;  // nearly diagonal
    const float ip = 1.0f / p;
    const float c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip;
    const float c01 = a[1] * ip, c02 = a[2] * ip, c12 = a[4] * ip;
    const float det = c00 * (c11 * c22 - c12 * c12) - c01 * (c01 * c22 - c12 * c02) + c02 * (c01 * c12 - c11 * c02);
    float r = 0.5f * det;
    r = fminf(fmaxf(r, -1.0f), 1.0f);
    const float phi = acosf(r) * (1.0f / 3.0f);
    const float l1 = q + 2.0f * p * cosf(phi);
    const float l3 = q + 2.0f * p * cosf(phi + 2.0943951023931953f);
    const float l2 = 3.0f * q - l1 - l3;
    eig[0] = l1;
    eig[1] = l2;
    eig[2] = l3;
    return l3 >= 1e-3f * l1;
}

struct F4a {
    float x, y, z, w;
};

__device__ __forceinline__ F4a mat(const float* m, float x, float y, float z) {
    F4a r;
    r.x = m[0] * x + m[1] * y + m[2] * z + m[3];
    r.y = m[4] * x + m[5] * y + m[6] * z + m[7];
    r.z = m[8] * x + m[9] * y + m[10] * z + m[11];
    r.w = m[12] * x + m[13] * y + m[14] * z + m[15];
    return r;
}

// Per node: covariance, eigen-solve, metrics, screen coverage, score, queue key.
__global__ void __launch_bounds__(256) k_analyze(Dev d, const RollSum* roll, NodeAnalysis* out,
                                                 float* features, AnalysisParams prm, Frame f,
                                                 AnalysisCounters* ac) {
    const uint32_t nn = d.ctr->numNodes;
    const float cube = fmaxf(fmaxf(f.boxMax[0] - f.boxMin[0], f.boxMax[1] - f.boxMin[1]), f.boxMax[2] - f.boxMin[2]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const RollSum r = roll[i];
        NodeAnalysis o;
        o.count = r.n;
        o.lastTouched = r.lastTouched;
        o.flags = 0;
        for (int k = 0; k < 3; k++) {
            o.eig[k] = 0.0f;
            o.normal[k] = 0.0f;
        }
        o.surfaceVariation = 0.0f;
        o.planarity = 0.0f;
        const uint32_t lv = d.level[i];
        if (r.n >= 3) {
            const u128 n = r.n;
            const i128 s1[3] = {(i128)r.s1[0], (i128)r.s1[1], (i128)r.s1[2]};
            const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
            double cov[6];
            const double nd = (double)r.n;
            const double unit = ldexp(1.0, (int)(28u - lv));
            const double scale = 1.0 / (nd * nd * unit * unit);
            for (int k = 0; k < 6; k++) {
                const u128 s2 = ((u128)r.s2[2 * k + 1] << 64) | r.s2[2 * k];
                const i128 c = (i128)(n * s2) - s1[pa[k]] * s1[pb[k]];
                cov[k] = i128ToDouble(c) * scale;
            }
            float cf[6];
            for (int k = 0; k < 6; k++) cf[k] = (float)cov[k];
            float e[3];
            if (smith3(cf, e)) {
                for (int k = 0; k < 3; k++) o.eig[k] = e[k];
                // normal: the row cross product of (A - l3 I) with the largest norm
                const float m00 = cf[0] - e[2], m11 = cf[3] - e[2], m22 = cf[5] - e[2];
                const float r0[3] = {m00, cf[1], cf[2]}, r1[3] = {cf[1], m11, cf[4]}, r2[3] = {cf[2], cf[4], m22};
                float c0[3] = {r0[1] * r1[2] - r0[2] * r1[1], r0[2] * r1[0] - r0[0] * r1[2], r0[0] * r1[1] - r0[1] * r1[0]};
                float c1[3] = {r0[1] * r2[2] - r0[2] * r2[1], r0[2] * r2[0] - r0[0] * r2[2], r0[0] * r2[1] - r0[1] * r2[0]};
                float c2[3] = {r1[1] * r2[2] - r1[2] * r2[1], r1[2] * r2[0] - r1[0] * r2[2], r1[0] * r2[1] - r1[1] * r2[0]};
                const float n0 = c0[0] * c0[0] + c0[1] * c0[1] + c0[2] * c0[2];
                const float n1 = c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2];
                const float n2 = c2[0] * c2[0] + c2[1] * c2[1] + c2[2] * c2[2];
                const float* best = n0 >= n1 && n0 >= n2 ? c0 : (n1 >= n2 ? c1 : c2);
                const float nb = fmaxf(fmaxf(n0, n1), n2);
                const float inv = nb > 0.0f ? rsqrtf(nb) : 0.0f;
                for (int k = 0; k < 3; k++) o.normal[k] = best[k] * inv;
            } else {
                double ed[3], vd[3];
                jacobi3(cov, ed, vd);
                for (int k = 0; k < 3; k++) {
                    o.eig[k] = (float)ed[k];
                    o.normal[k] = (float)vd[k];
                }
                o.flags |= kAnalysisFp64;
                atomicAdd(&ac->fp64Branch, 1u);
            }
            const float tr = o.eig[0] + o.eig[1] + o.eig[2];
            o.surfaceVariation = tr > 0.0f ? fmaxf(o.eig[2], 0.0f) / tr : 0.0f;
            o.planarity = o.eig[0] > 0.0f ? (o.eig[1] - o.eig[2]) / o.eig[0] : 0.0f;
        }
        // screen coverage of the node's box at this frame (projectedExtent, remolod_render.cu:40-70)
        float ext[2][4];
        bool anyv[2] = {false, false};
        for (int which = 0; which < 2; which++) {
            const uint32_t L = which == 0 ? lv : (lv > 0 ? lv - 1u : 0u);
            const uint32_t sh = which == 0 ? 0u : (lv > 0 ? 1u : 0u);
            const float s = cube / __int_as_float((int)((127u + L) << 23));
            const float mn[3] = {f.boxMin[0] + (float)(d.nodeX[i] >> sh) * s, f.boxMin[1] + (float)(d.nodeY[i] >> sh) * s,
                                 f.boxMin[2] + (float)(d.nodeZ[i] >> sh) * s};
            float minX = 1e30f, minY = 1e30f, maxX = -1e30f, maxY = -1e30f;
            for (int corner = 0; corner < 8; corner++) {
                const F4a c = mat(f.transformFrozen, (corner & 1) ? mn[0] + s : mn[0], (corner & 2) ? mn[1] + s : mn[1],
                                  (corner & 4) ? mn[2] + s : mn[2]);
                if (c.w <= 0.0f) continue;
                const float iw = 1.0f / c.w;
                const float sx = (c.x * iw * 0.5f + 0.5f) * f.width, sy = (c.y * iw * 0.5f + 0.5f) * f.height;
                minX = fminf(minX, sx);
                maxX = fmaxf(maxX, sx);
                minY = fminf(minY, sy);
                maxY = fmaxf(maxY, sy);
                anyv[which] = true;
            }
            ext[which][0] = minX;
            ext[which][1] = maxX;
            ext[which][2] = minY;
            ext[which][3] = maxY;
        }
        float cov2d = 0.0f;
        bool large = false, parentLarge = lv == 0;
        if (anyv[0]) {
            const float x0 = fmaxf(ext[0][0], 0.0f), x1 = fminf(ext[0][1], f.width);
            const float y0 = fmaxf(ext[0][2], 0.0f), y1 = fminf(ext[0][3], f.height);
            if (x1 > x0 && y1 > y0) cov2d = (x1 - x0) * (y1 - y0) / (f.width * f.height);
            large = (ext[0][1] - ext[0][0]) > prm.pixelBudget || (ext[0][3] - ext[0][2]) > prm.pixelBudget;
        }
        if (lv > 0 && anyv[1])
            parentLarge = (ext[1][1] - ext[1][0]) > prm.pixelBudget || (ext[1][3] - ext[1][2]) > prm.pixelBudget;
        const bool inner = !leafA(d, i);
        if (large) o.flags |= kAnalysisLarge;
        if (inner && !large && parentLarge) o.flags |= kAnalysisFrontier;
        o.coverage = cov2d;
        o.closed = (prm.currentBatch >= o.lastTouched + prm.closureMargin && r.n > 0) ? 1u : 0u;
        o.score = 0.0f;
        out[i] = o;
        // the learned scorer's inputs (the training-data logger records these)
        float* ft = features + (size_t)i * kNumFeatures;
        const double nd = r.n ? (double)r.n : 1.0;
        const double unit = ldexp(1.0, (int)(28u - lv));
        ft[0] = log2f(1.0f + (float)r.n) * (1.0f / 24.0f);
        ft[1] = (float)lv * (1.0f / 20.0f);
        for (int k = 0; k < 3; k++) ft[2 + k] = r.n ? (float)((double)r.s1[k] / (nd * unit)) : 0.0f;
        {
            // normalised centred second moments (a uniform cube has 1/12 on the diagonal)
            const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
            for (int k = 0; k < 6; k++) {
                float v = 0.0f;
                if (r.n >= 2) {
                    const u128 s2 = ((u128)r.s2[2 * k + 1] << 64) | r.s2[2 * k];
                    const i128 c = (i128)((u128)r.n * s2) - (i128)r.s1[pa[k]] * (i128)r.s1[pb[k]];
                    v = (float)(i128ToDouble(c) / (nd * nd * unit * unit) * 12.0);
                }
                ft[5 + k] = v;
            }
        }
        ft[11] = o.surfaceVariation * 3.0f;
        ft[12] = o.planarity;
        const bool leafNode = !inner;
        const float fill = leafNode ? (float)d.numPoints[i] * (1.0f / 50000.0f) : (float)d.numVoxels[i] * (1.0f / 16384.0f);
        ft[13] = fminf(fill, 4.0f);
        float cvar = 0.0f;
        if (r.n >= 2) {
            for (int k = 0; k < 3; k++) {
                const double m = (double)r.c1[k] / nd;
                cvar += (float)(((double)r.c2[k] / nd - m * m) / (255.0 * 255.0));
            }
        }
        ft[14] = cvar * (4.0f / 3.0f);
        const float age = prm.currentBatch > o.lastTouched ? (float)(prm.currentBatch - o.lastTouched) : 0.0f;
        ft[15] = fminf(age / (float)(prm.closureMargin ? prm.closureMargin : 1u), 2.0f);
    }
}

// Score x coverage, the queue key, per node. In the learned mode an open
// node's surface variation is its partial one plus the network's predicted
// correction (output 0, x 1/300).
__global__ void __launch_bounds__(256) k_score(Dev d, NodeAnalysis* out, const float* pred, unsigned long long* keys,
                                               AnalysisParams prm, AnalysisCounters* ac) {
    const uint32_t nn = d.ctr->numNodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        NodeAnalysis o = out[i];
        float sv = o.surfaceVariation;
        if (prm.scoreMode == kScoreClosed && !o.closed) sv = 0.0f;
        // the network predicts the change from the partial surface variation to the final one
        if (prm.scoreMode == kScoreLearned && !o.closed && pred)
            sv = fminf(fmaxf(sv + pred[2 * i] * (1.0f / 300.0f), 0.0f), 1.0f / 3.0f);
        float score = sv * o.coverage;
        if (o.count < prm.minPoints) score = 0.0f;
        out[i].score = score;
        const bool eligible = score > 0.0f && (prm.frontierOnly == 0u || (o.flags & kAnalysisFrontier));
        keys[i] = eligible ? (((unsigned long long)__float_as_uint(score) << 32) | (0xFFFFFFFFu - i)) : 0ull;
        if (eligible) atomicAdd(&ac->eligible, 1u);
    }
}

// Radix select of the queue: a 65536-bin histogram of the keys' top 16 bits.
__global__ void __launch_bounds__(256) k_queue_hist(const Dev d, const unsigned long long* keys, uint32_t* hist) {
    const uint32_t nn = d.ctr->numNodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        if (k) atomicAdd(&hist[(uint32_t)(k >> 48)], 1u);
    }
}

// One block: the lowest bin b such that the bins >= b hold at least K keys.
__global__ void __launch_bounds__(1024) k_queue_threshold(const uint32_t* hist, uint32_t K, AnalysisCounters* ac) {
    __shared__ uint32_t s_sum[1024];
    // each thread owns 64 consecutive bins, counted from the top
    uint32_t local = 0;
    const uint32_t t = threadIdx.x;
    for (uint32_t j = 0; j < 64; j++) local += hist[65535u - (t * 64u + j)];
    s_sum[t] = local;
    __syncthreads();
    if (t == 0) {
        uint32_t acc = 0;
        uint32_t thr = 0;
        bool found = false;
        for (uint32_t u = 0; u < 1024 && !found; u++) {
            if (acc + s_sum[u] >= K) {
                for (uint32_t j = 0; j < 64; j++) {
                    const uint32_t bin = 65535u - (u * 64u + j);
                    acc += hist[bin];
                    if (acc >= K) {
                        thr = bin;
                        found = true;
                        break;
                    }
                }
            } else {
                acc += s_sum[u];
            }
        }
        ac->thresholdBin = found ? thr : 0u;
        ac->numCandidates = 0;
    }
}

__global__ void __launch_bounds__(256) k_queue_collect(const Dev d, const unsigned long long* keys,
                                                       unsigned long long* cand, uint32_t cap, AnalysisCounters* ac) {
    const uint32_t nn = d.ctr->numNodes;
    const uint32_t thr = ac->thresholdBin;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        if (k && (uint32_t)(k >> 48) >= thr) {
            const uint32_t slot = atomicAdd(&ac->numCandidates, 1u);
            if (slot < cap) cand[slot] = k;
        }
    }
}

// One block: descending bitonic sort of the candidates in shared memory; the
// first K become the queue (node ids).
__global__ void __launch_bounds__(1024) k_queue_sort(const unsigned long long* cand, uint32_t cap, uint32_t K,
                                                     uint32_t* queue, AnalysisCounters* ac) {
    extern __shared__ unsigned long long s_k[];
    uint32_t n = ac->numCandidates;
    if (n > cap) {
        if (threadIdx.x == 0) ac->overflow = 1;
        n = cap;
    }
    uint32_t m = 1;
    while (m < n) m <<= 1;
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) s_k[i] = i < n ? cand[i] : 0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= m; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const unsigned long long a = s_k[i], b = s_k[l];
                    const bool desc = (i & k) == 0;
                    if ((a < b) == desc) {
                        s_k[i] = b;
                        s_k[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    const uint32_t q = n < K ? n : K;
    for (uint32_t i = threadIdx.x; i < q; i += blockDim.x)
        queue[i] = 0xFFFFFFFFu - (uint32_t)(s_k[i] & 0xFFFFFFFFull);
    if (threadIdx.x == 0) ac->queueLength = q;
}

// Refinement's budgeted pass: the first `budget` queue entries become forced
// splits of the LOD cut (rb_render's force-large mask).
__global__ void __launch_bounds__(256) k_refine_mask(const Dev d, uint8_t* mask) {
    const uint32_t nn = d.ctr->numNodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) mask[i] = 0;
}

__global__ void __launch_bounds__(256) k_refine_set(const uint32_t* queue, const AnalysisCounters* ac,
                                                    uint32_t budget, uint8_t* mask) {
    const uint32_t q = ac->queueLength < budget ? ac->queueLength : budget;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += gridDim.x * blockDim.x) mask[queue[i]] = 1;
}

void launchRollLevel(const Dev& d, RollSum* roll, uint32_t level, int grid, cudaStream_t s) {
    k_roll_level<<<grid, 256, 0, s>>>(d, roll, level);
}
void launchAnalyze(const Dev& d, const RollSum* roll, NodeAnalysis* out, float* features,
                   const AnalysisParams& p, const Frame& f, AnalysisCounters* ac, int grid, cudaStream_t s) {
    k_analyze<<<grid, 256, 0, s>>>(d, roll, out, features, p, f, ac);
}
void launchScore(const Dev& d, NodeAnalysis* out, const float* predictions, unsigned long long* keys,
                 const AnalysisParams& p, AnalysisCounters* ac, int grid, cudaStream_t s) {
    k_score<<<grid, 256, 0, s>>>(d, out, predictions, keys, p, ac);
}
void launchQueue(const Dev& d, const unsigned long long* keys, uint32_t* hist, unsigned long long* cand,
                 uint32_t candCap, uint32_t K, uint32_t* queue, AnalysisCounters* ac, int grid, cudaStream_t s) {
    k_queue_hist<<<grid, 256, 0, s>>>(d, keys, hist);
    k_queue_threshold<<<1, 1024, 0, s>>>(hist, K, ac);
    k_queue_collect<<<grid, 256, 0, s>>>(d, keys, cand, candCap, ac);
    uint32_t m = 1;
    while (m < candCap) m <<= 1;
    k_queue_sort<<<1, 1024, (size_t)m * 8, s>>>(cand, candCap, K, queue, ac);
}
void launchRefineMask(const Dev& d, const uint32_t* queue, const AnalysisCounters* ac, uint32_t budget,
                      uint8_t* mask, int grid, cudaStream_t s) {
    k_refine_mask<<<grid, 256, 0, s>>>(d, mask);
    k_refine_set<<<grid, 256, 0, s>>>(queue, ac, budget, mask);
}
cudaError_t configureQueueSort(uint32_t candCap) {
    uint32_t m = 1;
    while (m < candCap) m <<= 1;
    return cudaFuncSetAttribute(k_queue_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(m * 8));
}

}  // namespace rb
