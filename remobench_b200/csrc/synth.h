/*
 * Seeded synthetic lidar scenes for the progressive LOD path.
 *
 * A scene is a tile of ground (sum of four sinusoids), axis-aligned boxes and
 * vertical cylinder poles, scanned by a 32-channel spinning sensor that rides
 * 2 m above the ground along straight lanes. Points come out in acquisition
 * order, so a batch is a contiguous stretch of the sensor path -- the same
 * spatial coherence a lidar file has, which is what the reference's readers
 * hand to the device (src/io/LasReader.cpp reads in file order).
 *
 * Reproducibility: splitmix64(seed) seeds the scene; batch b draws only from
 * its own PCG32 stream (stream id b), so any batch can be regenerated alone and
 * the output does not depend on the number of threads.
 *
 * Point layout matches the reference's 16-byte point
 * (include/remo/HostDeviceCommon.h:15-18): float x, y, z; uint32 rgba with
 * r in the low byte (kernels/shared/remo_prelude.cuh:228-230).
 */
#ifndef RB_SYNTH_H
#define RB_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rb_synth_point {
    float x, y, z;
    uint32_t color;
} rb_synth_point;

typedef struct rb_synth_config {
    uint64_t seed;
    uint64_t num_points;
    uint32_t batch_size;     /* points per batch (acquisition-order stretch) */
    uint32_t num_boxes;
    uint32_t num_poles;
    uint32_t num_threads;    /* 0 = all hardware threads */
    double tile;             /* tile side in metres; the tile spans [0, tile)^2 */
    double origin_x;         /* world offset added before storing (UTM-like runs) */
    double origin_y;
    double outlier_fraction; /* share of points replaced by uniform noise in the tile volume */
    double range_noise;      /* sigma of the Gaussian range noise, metres (0.02) */
    double quantum;          /* >0: world coordinates snapped to this step (1 mm runs) */
} rb_synth_config;

typedef struct rb_synth_scene_info {
    double box_min[3];
    double box_max[3];
    uint32_t num_lanes;
    double sensor_height;
} rb_synth_scene_info;

/* Fills cfg with the defaults of a named configuration:
 *   1 = 2M points, 8 x 256K batches, 200 m tile, 40 boxes
 *   2 = 100M points, 1M batches, 2 km tile, 2000 boxes, 20000 poles
 *   3 = 200M points, 1M batches, 2 km tile at a UTM-like origin, 1 mm quantum
 *   5 = 1B points, 4M batches, 4 km tile, 5% uniform outliers
 * Returns 0, or -1 for an unknown id. */
int rb_synth_default_config(int config_id, rb_synth_config* cfg);

/* Scene bounding box (the cloud's declared box) for cfg. */
int rb_synth_scene_info_get(const rb_synth_config* cfg, rb_synth_scene_info* info);

/* Writes points [first, first+count) of the cloud into out, as float32
 * coordinates relative to the scene box minimum when relative != 0 (the
 * reference's readers translate to the box minimum in double precision), or as
 * float32 world coordinates otherwise. first must be a multiple of
 * cfg->batch_size. Returns 0 on success. */
int rb_synth_generate(const rb_synth_config* cfg, uint64_t first, uint64_t count,
                      int relative, rb_synth_point* out);

/* Same points as float64 world coordinates (x, y, z interleaved) plus colours. */
int rb_synth_generate_f64(const rb_synth_config* cfg, uint64_t first, uint64_t count,
                          double* xyz, uint32_t* color);

#ifdef __cplusplus
}
#endif

#endif
