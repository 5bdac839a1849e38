/*
 * CPU oracle for the foveated HTGS forward rasterizer — TEST INFRASTRUCTURE ONLY.
 *
 * A restatement, in plain C++ on the host, of the reference's forward path
 * (TrueKuehli/FoveatedHTGSCudaBackend, rasterization/src/inference.cu:49-472 and the
 * kernels it launches).  Every stage is templated on the arithmetic type: the FP64
 * instantiation is the accuracy oracle, the FP32 one is the host-core baseline.  Only the
 * test-suite, the smoke check and the CPU leg of the benchmark may call it; the product
 * (foveatedhtgscudabackend_b200) never links, loads or falls back to it.
 *
 * Parity pin: the stages are checked against outputs of the reference itself (built from
 * its own sources by oracle/build_ref.sh and oracle/ref_harness.cu, run on a B200, stored
 * as fixtures under tests/golden/ by tests/golden/make_golden.py).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One camera, as the reference's Pose/Intrinsics/Masks (rasterization_utils.h:88-109). */
typedef struct {
    int width, height;
    float focal_x, focal_y, center_x, center_y;
    float near_plane, far_plane;
    float M[12];          /* 3 rows x float4, world -> view                          */
    float VPM[16];        /* 4 rows x float4, world -> screen                        */
    float VPR_inv[16];    /* 4 rows x float4, screen -> world direction              */
    float cam_position[3];
    float gaze[2];        /* pixels, un-clamped (clamped as inference.cu:79-82)      */
    const uint32_t* visibility_mask;            /* bit per large tile            */
    const uint32_t* visibility_mask_area_table; /* (gx+1)*(gy+1)                 */
    const uint32_t* fovea_mask_area_table;      /* 49*49                         */
} oracle_view;

/* Gaussians, activated, fp32 as the reference consumes them. */
typedef struct {
    const float* positions;  /* [N,3] */
    const float* scales;     /* [N,3] */
    const float* rotations;  /* [N,4] (w,x,y,z) */
    const float* opacities;  /* [N]   */
    const float* sh_0;       /* [N,3] */
    const float* sh_rest;    /* [N,S,3] */
    int n;
    int total_sh_bases;      /* S = sh_rest.size(1) (inference_api.cu:76) */
} oracle_scene;

typedef struct {
    int K;
    int active_sh_bases;
    float scale_modifier;
    int to_chw, blur_periphery, anti_aliasing;
    int background_type;             /* 0 none, 1 SH, 2 texture, 3 raw texture */
    const float* background_data;    /* SH: [16,3]; texture: [3,h,w]            */
    int texture_width, texture_height;
    int precision;                   /* 32 or 64 */
    int n_threads;                   /* OpenMP threads, <=0: default            */
    /* Foveation (as fhtgs_settings.foveation of the product): 0 the reference's; 1 rings
     * (full resolution for NDC distance < ring_full from the gaze, stride 2 below ring_half,
     * stride 4 beyond); 2 none (all tiles full resolution).  Modes 1 and 2 have no
     * counterpart in the reference. */
    int foveation;
    float ring_full, ring_half;
} oracle_settings;

/* Per-primitive results of the preprocess stage (inference.cuh:42-136). */
typedef struct {
    uint32_t* n_touched;     /* [N]      */
    uint16_t* screen_bounds; /* [N,4]  x_min,x_max,y_min,y_max (large tiles) */
    float* vpmt;             /* [N,12] VPMT1,VPMT2,VPMT4 */
    float* rgba;             /* [N,4]  */
} oracle_primitives;

/* Tile classification (shared_kernels.cuh:155-238, inference.cu:131-188). */
typedef struct {
    uint32_t* tile_index_map_partitioned; /* [T] (first n_active valid) */
    uint8_t* tile_type_partitioned;       /* [T] */
    uint32_t* partition_ranges;           /* [6] fovea, periphery, blended (x,y) */
    uint32_t* n_active_tiles;             /* [1] */
} oracle_tiles;

/* Instance lists: keys widened to uint32 (sentinel 0xFFFF for 16-bit keys). */
typedef struct {
    uint32_t* keys;           /* [capacity] */
    uint32_t* values;         /* [capacity] */
    int64_t capacity;
    int64_t* n_instances;     /* [1] M = inclusive_scan(n_touched)[N-1] */
    uint32_t* instance_ranges;/* [2*T] */
} oracle_instances;

/* Derived sizes for a view: grid of large tiles, small-tile count, key end bit. */
void oracle_view_geometry(const oracle_view* v, int* grid_large_w, int* grid_large_h,
                          int* n_tiles_small, int* end_bit, int* gaze_tile_x, int* gaze_tile_y);

int oracle_classify_tiles(const oracle_view* v, oracle_tiles* out);
int oracle_preprocess(const oracle_scene* s, const oracle_view* v, const oracle_settings* st,
                      oracle_primitives* out);
/* Instance creation from given per-primitive bounds/counts, then stable sort + ranges. */
int oracle_instances_from_primitives(const oracle_view* v, int n, const uint32_t* n_touched,
                                     const uint16_t* screen_bounds, oracle_instances* out,
                                     uint32_t* unsorted_keys, uint32_t* unsorted_values);
/* K-buffer blend + periphery upsampling/composition from given intermediates. */
int oracle_blend_compose(const oracle_view* v, const oracle_settings* st, int n,
                         const float* vpmt, const float* rgba,
                         const uint32_t* tile_index_map_partitioned,
                         const uint32_t* partition_ranges,
                         const uint32_t* sorted_values, const uint32_t* instance_ranges,
                         float* image);
/* Whole view: all stages chained; any intermediate pointer may be NULL. */
int oracle_render_view(const oracle_scene* s, const oracle_view* v, const oracle_settings* st,
                       float* image, oracle_primitives* prim, oracle_tiles* tiles,
                       oracle_instances* inst);
/* Timing helper for the CPU baseline: renders n_views views, returns wall seconds. */
double oracle_time_views(const oracle_scene* s, const oracle_view* views, int n_views,
                         const oracle_settings* st, float* const* images);
/* Seconds per stage of the last oracle_time_views call (std::chrono, summed over its views):
 * [0] preprocess, [1] tile classification, [2] instance creation + sort + ranges,
 * [3] blend + composition. */
void oracle_stage_seconds(double* out4);

#ifdef __cplusplus
}
#endif
