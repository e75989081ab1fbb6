/*
 * Seeded synthetic lidar scenes: see synth.h for the contract.
 *
 * Geometry is evaluated in double precision and stored as float32 at the end,
 * relative to the scene box minimum -- the reference's readers translate the
 * same way (src/io/PointSource.cpp:355-365 sets translation = -boxMin and the
 * uniforms' box becomes [0, boxSize], src/shell/App.cpp:228-229).
 *
 * RNG: splitmix64 (Steele, Lea, Flood 2014) seeds; PCG32 XSH-RR (O'Neill 2014)
 * per-batch streams; Box-Muller for Gaussian range noise.
 */
#define _GNU_SOURCE
#include "synth.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define RB_PI 3.14159265358979323846

/* ------------------------------------------------------------------ RNG */

static uint64_t splitmix64(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct pcg32 {
    uint64_t state;
    uint64_t inc;
} pcg32;

static uint32_t pcg32_next(pcg32* r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ull + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
}

static void pcg32_seed(pcg32* r, uint64_t initstate, uint64_t stream) {
    r->state = 0u;
    r->inc = (stream << 1u) | 1u;
    pcg32_next(r);
    r->state += initstate;
    pcg32_next(r);
}

/* uniform in [0, 1) with 53 random bits */
static double pcg_unit(pcg32* r) {
    uint64_t hi = pcg32_next(r) >> 5;  /* 27 bits */
    uint64_t lo = pcg32_next(r) >> 6;  /* 26 bits */
    return (double)((hi << 26) | lo) * (1.0 / 9007199254740992.0);
}

static double pcg_range(pcg32* r, double a, double b) { return a + (b - a) * pcg_unit(r); }

static double pcg_gauss(pcg32* r) {
    double u1 = pcg_unit(r);
    double u2 = pcg_unit(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(2.0 * RB_PI * u2);
}

/* ---------------------------------------------------------------- scene */

typedef struct box_obj {
    double x0, y0, z0, x1, y1, z1;
} box_obj;

typedef struct pole_obj {
    double cx, cy, r, z0, z1;
} pole_obj;

typedef struct scene {
    double tile;
    double amp[4], kx[4], ky[4], phase[4];
    double lipschitz;
    uint32_t num_boxes, num_poles;
    box_obj* boxes;
    pole_obj* poles;
    /* 2D uniform grid of object ids (boxes first, then poles offset by num_boxes) */
    double cell;
    int gn;
    uint32_t* cell_start; /* gn*gn + 1 */
    uint32_t* cell_items;
    double zlo, zhi;
    uint32_t lanes;
    double sensor_height;
    double path_len;
} scene;

static double ground_h(const scene* s, double x, double y) {
    double h = 0.0;
    for (int i = 0; i < 4; i++) h += s->amp[i] * sin(s->kx[i] * x + s->ky[i] * y + s->phase[i]);
    return h;
}

static void scene_free(scene* s) {
    free(s->boxes);
    free(s->poles);
    free(s->cell_start);
    free(s->cell_items);
    memset(s, 0, sizeof(*s));
}

static int scene_build(const rb_synth_config* cfg, scene* s) {
    memset(s, 0, sizeof(*s));
    uint64_t sm = cfg->seed;
    pcg32 r;
    pcg32_seed(&r, splitmix64(&sm), 0xA5A5A5A5ull);

    s->tile = cfg->tile;
    s->lipschitz = 0.0;
    double amp_sum = 0.0;
    for (int i = 0; i < 4; i++) {
        double a = pcg_range(&r, 0.5, 2.0);
        double wl = pcg_range(&r, 10.0, 80.0);
        double th = pcg_range(&r, 0.0, 2.0 * RB_PI);
        double ph = pcg_range(&r, 0.0, 2.0 * RB_PI);
        double k = 2.0 * RB_PI / wl;
        s->amp[i] = a;
        s->kx[i] = k * cos(th);
        s->ky[i] = k * sin(th);
        s->phase[i] = ph;
        s->lipschitz += a * k;
        amp_sum += a;
    }

    double ztop = amp_sum;
    s->num_boxes = cfg->num_boxes;
    s->num_poles = cfg->num_poles;
    s->boxes = (box_obj*)calloc(s->num_boxes ? s->num_boxes : 1, sizeof(box_obj));
    s->poles = (pole_obj*)calloc(s->num_poles ? s->num_poles : 1, sizeof(pole_obj));
    if (!s->boxes || !s->poles) return -1;
    for (uint32_t i = 0; i < s->num_boxes; i++) {
        double cx = pcg_range(&r, 0.0, s->tile);
        double cy = pcg_range(&r, 0.0, s->tile);
        double sx = pcg_range(&r, 5.0, 30.0);
        double sy = pcg_range(&r, 5.0, 30.0);
        double hgt = pcg_range(&r, 3.0, 40.0);
        double x0 = cx - 0.5 * sx, x1 = cx + 0.5 * sx;
        double y0 = cy - 0.5 * sy, y1 = cy + 0.5 * sy;
        double base = ground_h(s, cx, cy);
        double c[4] = {ground_h(s, x0, y0), ground_h(s, x1, y0), ground_h(s, x0, y1),
                       ground_h(s, x1, y1)};
        for (int k = 0; k < 4; k++)
            if (c[k] < base) base = c[k];
        base -= 0.2;
        box_obj b = {x0, y0, base, x1, y1, base + hgt};
        s->boxes[i] = b;
        if (b.z1 > ztop) ztop = b.z1;
    }
    for (uint32_t i = 0; i < s->num_poles; i++) {
        double cx = pcg_range(&r, 0.0, s->tile);
        double cy = pcg_range(&r, 0.0, s->tile);
        double rad = pcg_range(&r, 0.1, 0.5);
        double hgt = pcg_range(&r, 4.0, 12.0);
        double base = ground_h(s, cx, cy) - 0.2;
        pole_obj p = {cx, cy, rad, base, base + hgt};
        s->poles[i] = p;
        if (p.z1 > ztop) ztop = p.z1;
    }
    s->zlo = -amp_sum - 1.0;
    s->zhi = ztop + 1.0;

    /* object grid */
    s->cell = 8.0;
    s->gn = (int)ceil(s->tile / s->cell);
    if (s->gn < 1) s->gn = 1;
    size_t ncell = (size_t)s->gn * (size_t)s->gn;
    s->cell_start = (uint32_t*)calloc(ncell + 1, sizeof(uint32_t));
    if (!s->cell_start) return -1;
    uint32_t nobj = s->num_boxes + s->num_poles;
    /* pass 1: counts; pass 2: fill */
    for (int pass = 0; pass < 2; pass++) {
        uint32_t* cursor = NULL;
        if (pass == 1) {
            uint32_t total = 0;
            for (size_t c = 0; c < ncell; c++) {
                uint32_t n = s->cell_start[c];
                s->cell_start[c] = total;
                total += n;
            }
            s->cell_start[ncell] = total;
            s->cell_items = (uint32_t*)malloc((total ? total : 1) * sizeof(uint32_t));
            cursor = (uint32_t*)malloc(ncell * sizeof(uint32_t));
            if (!s->cell_items || !cursor) return -1;
            memcpy(cursor, s->cell_start, ncell * sizeof(uint32_t));
        }
        for (uint32_t o = 0; o < nobj; o++) {
            double x0, y0, x1, y1;
            if (o < s->num_boxes) {
                x0 = s->boxes[o].x0; x1 = s->boxes[o].x1;
                y0 = s->boxes[o].y0; y1 = s->boxes[o].y1;
            } else {
                const pole_obj* p = &s->poles[o - s->num_boxes];
                x0 = p->cx - p->r; x1 = p->cx + p->r;
                y0 = p->cy - p->r; y1 = p->cy + p->r;
            }
            int i0 = (int)floor(x0 / s->cell), i1 = (int)floor(x1 / s->cell);
            int j0 = (int)floor(y0 / s->cell), j1 = (int)floor(y1 / s->cell);
            if (i0 < 0) i0 = 0;
            if (j0 < 0) j0 = 0;
            if (i1 >= s->gn) i1 = s->gn - 1;
            if (j1 >= s->gn) j1 = s->gn - 1;
            for (int j = j0; j <= j1; j++)
                for (int i = i0; i <= i1; i++) {
                    size_t c = (size_t)j * s->gn + i;
                    if (pass == 0) s->cell_start[c]++;
                    else s->cell_items[cursor[c]++] = o;
                }
        }
        free(cursor);
    }

    s->lanes = (uint32_t)floor(s->tile / 200.0 + 0.5);
    if (s->lanes < 1) s->lanes = 1;
    s->sensor_height = 2.0;
    s->path_len = (double)s->lanes * s->tile;
    return 0;
}

/* ray vs. axis-aligned box (slab test); returns entry distance in (tmin, tmax) or -1 */
static double hit_box(const box_obj* b, const double o[3], const double d[3], double tmax) {
    double t0 = 1e-4, t1 = tmax;
    const double lo[3] = {b->x0, b->y0, b->z0};
    const double hi[3] = {b->x1, b->y1, b->z1};
    for (int a = 0; a < 3; a++) {
        if (fabs(d[a]) < 1e-12) {
            if (o[a] < lo[a] || o[a] > hi[a]) return -1.0;
            continue;
        }
        double inv = 1.0 / d[a];
        double ta = (lo[a] - o[a]) * inv, tb = (hi[a] - o[a]) * inv;
        if (ta > tb) { double t = ta; ta = tb; tb = t; }
        if (ta > t0) t0 = ta;
        if (tb < t1) t1 = tb;
        if (t0 > t1) return -1.0;
    }
    return t0;
}

/* ray vs. vertical cylinder side and top cap */
static double hit_pole(const pole_obj* p, const double o[3], const double d[3], double tmax) {
    double best = -1.0;
    double ox = o[0] - p->cx, oy = o[1] - p->cy;
    double a = d[0] * d[0] + d[1] * d[1];
    if (a > 1e-14) {
        double b = 2.0 * (ox * d[0] + oy * d[1]);
        double c = ox * ox + oy * oy - p->r * p->r;
        double disc = b * b - 4.0 * a * c;
        if (disc >= 0.0) {
            double sq = sqrt(disc);
            double t = (-b - sq) / (2.0 * a);
            if (t > 1e-4 && t < tmax) {
                double z = o[2] + t * d[2];
                if (z >= p->z0 && z <= p->z1) best = t;
            }
        }
    }
    if (fabs(d[2]) > 1e-12) {
        double t = (p->z1 - o[2]) / d[2];
        if (t > 1e-4 && t < tmax && (best < 0.0 || t < best)) {
            double x = ox + t * d[0], y = oy + t * d[1];
            if (x * x + y * y <= p->r * p->r) best = t;
        }
    }
    return best;
}

/* nearest object hit along the ray within tmax, by 2D DDA over the object grid */
static double hit_objects(const scene* s, const double o[3], const double d[3], double tmax) {
    if (s->num_boxes + s->num_poles == 0) return -1.0;
    double best = -1.0;
    double limit = tmax;
    double dx = d[0], dy = d[1];
    int ix = (int)floor(o[0] / s->cell), iy = (int)floor(o[1] / s->cell);
    int stepx = dx > 0 ? 1 : -1, stepy = dy > 0 ? 1 : -1;
    double tdx = fabs(dx) > 1e-12 ? s->cell / fabs(dx) : 1e300;
    double tdy = fabs(dy) > 1e-12 ? s->cell / fabs(dy) : 1e300;
    double nx = (dx > 0 ? (ix + 1) * s->cell - o[0] : o[0] - ix * s->cell);
    double ny = (dy > 0 ? (iy + 1) * s->cell - o[1] : o[1] - iy * s->cell);
    double tmx = fabs(dx) > 1e-12 ? nx / fabs(dx) : 1e300;
    double tmy = fabs(dy) > 1e-12 ? ny / fabs(dy) : 1e300;
    double tcell = 0.0;
    for (int guard = 0; guard < 4096; guard++) {
        if (ix >= 0 && iy >= 0 && ix < s->gn && iy < s->gn) {
            size_t c = (size_t)iy * s->gn + ix;
            for (uint32_t k = s->cell_start[c]; k < s->cell_start[c + 1]; k++) {
                uint32_t obj = s->cell_items[k];
                double t = obj < s->num_boxes ? hit_box(&s->boxes[obj], o, d, limit)
                                              : hit_pole(&s->poles[obj - s->num_boxes], o, d, limit);
                if (t > 0.0 && (best < 0.0 || t < best)) {
                    best = t;
                    limit = t;
                }
            }
        } else if ((ix < 0 && stepx < 0) || (iy < 0 && stepy < 0) ||
                   (ix >= s->gn && stepx > 0) || (iy >= s->gn && stepy > 0)) {
            break;
        }
        if (tcell > limit) break;
        if (tmx < tmy) {
            tcell = tmx;
            tmx += tdx;
            ix += stepx;
        } else {
            tcell = tmy;
            tmy += tdy;
            iy += stepy;
        }
        if (tcell > limit) break;
    }
    return best;
}

/* Ground hit: march along the ray with the larger of the Lipschitz-safe step
 * and a secant-predicted step, then bisect the first sign change. A secant
 * step can jump a crest the ray only grazes; that costs a little occlusion
 * realism and nothing else. */
static double hit_ground(const scene* s, const double o[3], const double d[3], double tmax) {
    double dxy = sqrt(d[0] * d[0] + d[1] * d[1]);
    double bound = fabs(d[2]) + s->lipschitz * dxy;
    if (bound < 1e-9) return -1.0;
    double tp = 0.0;
    double fp = o[2] - ground_h(s, o[0], o[1]);
    if (fp <= 0.0) return -1.0;
    double slope = 0.0;
    int have_slope = 0;
    for (int it = 0; it < 600; it++) {
        double step = fp / bound;
        if (have_slope && slope < 0.0) {
            double pred = 0.7 * fp / (-slope);
            if (pred > step) step = pred;
        }
        if (step < 0.02) step = 0.02;
        if (step > 10.0) step = 10.0;
        double t = tp + step;
        if (t > tmax) return -1.0;
        double f = o[2] + t * d[2] - ground_h(s, o[0] + t * d[0], o[1] + t * d[1]);
        if (f <= 0.0) {
            double a = tp, b = t;
            for (int k = 0; k < 24; k++) {
                double m = 0.5 * (a + b);
                double fm = o[2] + m * d[2] - ground_h(s, o[0] + m * d[0], o[1] + m * d[1]);
                if (fm > 0.0) a = m;
                else b = m;
            }
            return 0.5 * (a + b);
        }
        slope = (f - fp) / (t - tp);
        have_slope = 1;
        tp = t;
        fp = f;
    }
    return -1.0;
}

static void sensor_pose(const scene* s, double progress, double o[3]) {
    if (progress < 0.0) progress = 0.0;
    if (progress >= s->path_len) progress = s->path_len - 1e-6;
    uint32_t lane = (uint32_t)floor(progress / s->tile);
    if (lane >= s->lanes) lane = s->lanes - 1;
    double u = progress - lane * s->tile;
    double x = (lane & 1u) ? s->tile - u : u;
    double y = (lane + 0.5) * s->tile / s->lanes;
    o[0] = x;
    o[1] = y;
    o[2] = ground_h(s, x, y) + s->sensor_height;
}

static uint32_t colormap(double v, pcg32* r) {
    /* five-stop terrain gradient: deep blue, green, yellow, red, white */
    static const double stops[5][3] = {
        {30, 60, 160}, {40, 150, 60}, {220, 210, 60}, {200, 60, 40}, {245, 245, 245}};
    if (v < 0.0) v = 0.0;
    if (v > 1.0) v = 1.0;
    double f = v * 4.0;
    int i = (int)f;
    if (i > 3) i = 3;
    double t = f - i;
    uint32_t out = 0;
    for (int c = 0; c < 3; c++) {
        double val = stops[i][c] + (stops[i + 1][c] - stops[i][c]) * t;
        int n = (int)(pcg32_next(r) % 21u) - 10;
        int q = (int)floor(val + 0.5) + n;
        if (q < 0) q = 0;
        if (q > 255) q = 255;
        out |= (uint32_t)q << (8 * c);
    }
    return out | (255u << 24);
}

typedef struct gen_point {
    double x, y, z;
    uint32_t color;
} gen_point;

static void gen_one(const scene* s, const rb_synth_config* cfg, uint64_t index, uint64_t total,
                    pcg32* r, gen_point* out) {
    double zspan = s->zhi - s->zlo;
    if (cfg->outlier_fraction > 0.0 && pcg_unit(r) < cfg->outlier_fraction) {
        out->x = pcg_range(r, 0.0, s->tile);
        out->y = pcg_range(r, 0.0, s->tile);
        out->z = pcg_range(r, s->zlo + 0.5, s->zhi - 0.5);
        out->color = colormap((out->z - s->zlo) / zspan, r);
        return;
    }
    const uint32_t channels = 32, steps_per_rev = 360;
    uint64_t steps = (total + channels - 1) / channels;
    uint64_t a = index / channels;
    uint32_t ch = (uint32_t)(index % channels);
    double progress = ((double)a + 0.5) * (s->path_len / (double)steps);
    double o[3];
    sensor_pose(s, progress, o);
    double az = 2.0 * RB_PI * ((double)(a % steps_per_rev) + pcg_range(r, -0.5, 0.5)) / steps_per_rev;
    double el = (-30.0 + ch * (40.0 / (channels - 1)) + pcg_range(r, -0.3, 0.3)) * (RB_PI / 180.0);
    const double tmax = 120.0;
    for (int attempt = 0; attempt < 24; attempt++) {
        if (attempt > 0) {
            az = pcg_range(r, 0.0, 2.0 * RB_PI);
            el = pcg_range(r, -30.0, -2.0) * (RB_PI / 180.0);
        }
        if (attempt == 23) el = -60.0 * (RB_PI / 180.0);
        double d[3] = {cos(el) * cos(az), cos(el) * sin(az), sin(el)};
        double tg = hit_ground(s, o, d, tmax);
        double to = hit_objects(s, o, d, tg > 0.0 ? tg : tmax);
        double t = to > 0.0 ? to : tg;
        if (t <= 0.0) continue;
        t += cfg->range_noise * pcg_gauss(r);
        double x = o[0] + t * d[0], y = o[1] + t * d[1], z = o[2] + t * d[2];
        if (!(x >= 0.0 && x < s->tile && y >= 0.0 && y < s->tile)) continue;
        if (z < s->zlo) z = s->zlo;
        if (z > s->zhi) z = s->zhi;
        out->x = x;
        out->y = y;
        out->z = z;
        out->color = colormap((z - s->zlo) / zspan, r);
        return;
    }
    /* a ray straight down at the sensor always lands in the tile */
    out->x = o[0];
    out->y = o[1];
    out->z = o[2] - s->sensor_height;
    out->color = colormap((out->z - s->zlo) / zspan, r);
}

int rb_synth_default_config(int config_id, rb_synth_config* cfg) {
    if (!cfg) return -1;
    memset(cfg, 0, sizeof(*cfg));
    cfg->seed = 1;
    cfg->range_noise = 0.02;
    switch (config_id) {
        case 1:
            cfg->num_points = 8ull * 262144ull;
            cfg->batch_size = 262144;
            cfg->tile = 200.0;
            cfg->num_boxes = 40;
            break;
        case 2:
            cfg->num_points = 100000000ull;
            cfg->batch_size = 1000000;
            cfg->tile = 2000.0;
            cfg->num_boxes = 2000;
            cfg->num_poles = 20000;
            break;
        case 3:
            cfg->num_points = 200000000ull;
            cfg->batch_size = 1000000;
            cfg->tile = 2000.0;
            cfg->num_boxes = 2000;
            cfg->num_poles = 20000;
            cfg->origin_x = 500000.0;
            cfg->origin_y = 4000000.0;
            cfg->quantum = 0.001;
            break;
        case 5:
            cfg->num_points = 1000000000ull;
            cfg->batch_size = 4000000;
            cfg->tile = 4000.0;
            cfg->num_boxes = 8000;
            cfg->num_poles = 80000;
            cfg->outlier_fraction = 0.05;
            break;
        default:
            return -1;
    }
    return 0;
}

int rb_synth_scene_info_get(const rb_synth_config* cfg, rb_synth_scene_info* info) {
    if (!cfg || !info) return -1;
    scene s;
    if (scene_build(cfg, &s) != 0) {
        scene_free(&s);
        return -1;
    }
    info->box_min[0] = cfg->origin_x;
    info->box_min[1] = cfg->origin_y;
    info->box_min[2] = s.zlo;
    info->box_max[0] = cfg->origin_x + s.tile;
    info->box_max[1] = cfg->origin_y + s.tile;
    info->box_max[2] = s.zhi;
    info->num_lanes = s.lanes;
    info->sensor_height = s.sensor_height;
    scene_free(&s);
    return 0;
}

typedef struct job {
    const scene* s;
    const rb_synth_config* cfg;
    uint64_t first, count;
    int relative;
    rb_synth_point* out32;
    double* out64;
    uint32_t* color64;
    uint64_t next_batch; /* shared cursor, in batches */
    uint64_t num_batches;
    pthread_mutex_t mu;
} job;

static void snap(const rb_synth_config* cfg, double* w) {
    if (cfg->quantum > 0.0) *w = floor(*w / cfg->quantum + 0.5) * cfg->quantum;
}

static void* worker(void* arg) {
    job* j = (job*)arg;
    const uint64_t bs = j->cfg->batch_size;
    const uint64_t first_batch = j->first / bs;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        uint64_t b = j->next_batch++;
        pthread_mutex_unlock(&j->mu);
        if (b >= j->num_batches) break;
        uint64_t gb = first_batch + b;
        uint64_t sm = j->cfg->seed ^ 0x5EEDBA7C4ull;
        uint64_t init = splitmix64(&sm);
        pcg32 r;
        pcg32_seed(&r, init, gb);
        uint64_t lo = gb * bs;
        uint64_t hi = lo + bs;
        if (hi > j->cfg->num_points) hi = j->cfg->num_points;
        for (uint64_t i = lo; i < hi; i++) {
            if (i < j->first || i >= j->first + j->count) continue;
            gen_point p;
            gen_one(j->s, j->cfg, i, j->cfg->num_points, &r, &p);
            double wx = p.x + j->cfg->origin_x, wy = p.y + j->cfg->origin_y, wz = p.z;
            snap(j->cfg, &wx);
            snap(j->cfg, &wy);
            snap(j->cfg, &wz);
            uint64_t k = i - j->first;
            if (j->out32) {
                rb_synth_point q;
                if (j->relative) {
                    q.x = (float)(wx - j->cfg->origin_x);
                    q.y = (float)(wy - j->cfg->origin_y);
                    q.z = (float)(wz - j->s->zlo);
                } else {
                    q.x = (float)wx;
                    q.y = (float)wy;
                    q.z = (float)wz;
                }
                q.color = p.color;
                j->out32[k] = q;
            } else {
                j->out64[3 * k + 0] = wx;
                j->out64[3 * k + 1] = wy;
                j->out64[3 * k + 2] = wz;
                j->color64[k] = p.color;
            }
        }
    }
    return NULL;
}

static int run(const rb_synth_config* cfg, uint64_t first, uint64_t count, int relative,
               rb_synth_point* out32, double* out64, uint32_t* color64) {
    if (!cfg || cfg->batch_size == 0 || cfg->tile <= 0.0) return -1;
    if (first % cfg->batch_size != 0) return -1;
    if (first + count > cfg->num_points) return -1;
    if (count == 0) return 0;
    scene s;
    if (scene_build(cfg, &s) != 0) {
        scene_free(&s);
        return -1;
    }
    job j;
    memset(&j, 0, sizeof(j));
    j.s = &s;
    j.cfg = cfg;
    j.first = first;
    j.count = count;
    j.relative = relative;
    j.out32 = out32;
    j.out64 = out64;
    j.color64 = color64;
    j.num_batches = (count + cfg->batch_size - 1) / cfg->batch_size;
    pthread_mutex_init(&j.mu, NULL);
    long hw = sysconf(_SC_NPROCESSORS_ONLN);
    uint32_t nt = cfg->num_threads ? cfg->num_threads : (uint32_t)(hw > 0 ? hw : 1);
    if (nt > j.num_batches) nt = (uint32_t)j.num_batches;
    if (nt > 256) nt = 256;
    pthread_t th[256];
    uint32_t started = 0;
    for (uint32_t t = 0; t < nt; t++)
        if (pthread_create(&th[t], NULL, worker, &j) == 0) started++;
    if (started == 0) worker(&j);
    for (uint32_t t = 0; t < started; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&j.mu);
    scene_free(&s);
    return 0;
}

int rb_synth_generate(const rb_synth_config* cfg, uint64_t first, uint64_t count, int relative,
                      rb_synth_point* out) {
    if (!out) return -1;
    return run(cfg, first, count, relative, out, NULL, NULL);
}

int rb_synth_generate_f64(const rb_synth_config* cfg, uint64_t first, uint64_t count,
                          double* xyz, uint32_t* color) {
    if (!xyz || !color) return -1;
    return run(cfg, first, count, 0, NULL, xyz, color);
}
