/*
 * fhtgs — B200-native forward renderer for foveated hybrid-transparency Gaussian splatting.
 *
 * C ABI of libfhtgs.so.  Plain pointers and sizes only; no torch types.  All pointers marked
 * "device" must point to CUDA device memory of the context's device; "host" values are read
 * during the call.  Calls are asynchronous on the given stream unless the name ends in
 * `_sync`.  A context is not thread-safe: use one context per host thread (contexts may
 * share a device).
 *
 * Reference interfaces replaced (paths relative to the reference's FoveatedHTGSCudaBackend/
 * package directory):
 *   fhtgs_render_mono       <- _C.render            = inference_wrapper
 *                              (rasterization/src/inference_api.cu:13-43, torch_bindings/bindings.cpp:8)
 *   fhtgs_benchmark_mono    <- _C_benchmarking.benchmark = fast_inference_wrapper
 *                              (rasterization/src/fast_inference_api.cu:12-43, torch_bindings/bindings_benchmarking.cpp:7)
 *   fhtgs_render_stereo     <- _C_stereo.render     = inference_stereo_wrapper
 *                              (rasterization/src/inference_stereo_api.cu:13-67, torch_bindings/bindings_stereo.cpp:8)
 *   fhtgs_render_views      <- inference() / inference_stereo() generalised to n views
 *                              (rasterization/src/inference.cu:49-472, inference_stereo.cu:49-828)
 */
#ifndef FHTGS_H_
#define FHTGS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FHTGS_ABI_VERSION 4

typedef enum {
    FHTGS_OK = 0,
    FHTGS_ERR_INVALID_ARGUMENT = 1, /* bad shape, null pointer, unsupported option       */
    FHTGS_ERR_CUDA = 2,             /* a CUDA runtime call failed (see fhtgs_last_error) */
    FHTGS_ERR_OUT_OF_MEMORY = 3,    /* device arena could not grow                        */
    FHTGS_ERR_CAPACITY = 4,         /* instance count exceeded the arena; re-run (the
                                       _sync entry points grow and retry by themselves)   */
    FHTGS_ERR_NOT_READY = 5         /* no completed frame to inspect                      */
} fhtgs_status;

/* Background models, as the reference's BackgroundModelType (rasterization_utils.h:6-11). */
typedef enum {
    FHTGS_BACKGROUND_NONE = 0,
    FHTGS_BACKGROUND_SH = 1,          /* data: device float[16*3]                           */
    FHTGS_BACKGROUND_TEXTURE = 2,     /* data: device float[3*h*w], equirectangular         */
    FHTGS_BACKGROUND_TEXTURE_RAW = 3  /* as TEXTURE, sigmoid applied after interpolation   */
} fhtgs_background_type;

typedef struct fhtgs_context_s* fhtgs_context;

/* Storage formats of the Gaussian attributes (fhtgs_primitives.storage).  Either way every
 * attribute is widened to float32 when read and all arithmetic is float32. */
typedef enum {
    FHTGS_STORAGE_FP32 = 0,  /* all attributes float32 (the reference's format)            */
    FHTGS_STORAGE_HALF = 1   /* positions float32; scales, rotations, opacities IEEE fp16;
                                sh_0 and sh_rest bfloat16 (124 instead of 236 B per SH3
                                Gaussian)                                                  */
} fhtgs_storage;

/* Gaussians (device, contiguous, activated parameters; element type per `storage`).  The
 * pointers are typed float for the FP32 format; for FHTGS_STORAGE_HALF pass the 16-bit arrays
 * cast to these pointer types. */
typedef struct {
    const float* positions;  /* [N,3]                                   */
    const float* scales;     /* [N,3] linear                            */
    const float* rotations;  /* [N,4] (w,x,y,z), used as given          */
    const float* opacities;  /* [N] post-sigmoid                        */
    const float* sh_0;       /* [N,3]                                   */
    const float* sh_rest;    /* [N,S,3], may be NULL when S == 0        */
    int32_t n_primitives;    /* N                                       */
    int32_t total_sh_bases;  /* S = sh_rest.size(1)                     */
    int32_t storage;         /* fhtgs_storage; 0 = FP32                 */
} fhtgs_primitives;

/* One camera and its output image. */
typedef struct {
    const float* M;        /* device [3,4] world -> view                       */
    const float* VPM;      /* device [4,4] world -> screen                     */
    const float* VPR_inv;  /* device [4,4] screen -> world direction           */
    const float* cam_position;   /* device [3]                                 */
    float gaze_x, gaze_y;        /* host: gaze in pixels                       */
    const uint32_t* visibility_mask;            /* device, 1 bit per 16x16 tile   */
    const uint32_t* visibility_mask_area_table; /* device, (gx+1)*(gy+1)          */
    const uint32_t* fovea_mask_area_table;      /* device, 49*49                  */
    int32_t width, height;
    float focal_x, focal_y, center_x, center_y;
    float* image;          /* device output, [3,H,W] (to_chw) or [H,W,3]         */
    /* per-view foveation (no counterpart in the reference): 0 = the frame's settings;
     * 1 + fhtgs_foveation = this view's own mode, with its own ring radii */
    int32_t foveation;
    float ring_full, ring_half;
} fhtgs_view;

typedef struct {
    int32_t K;                 /* core size; rounded down to a power of two <= 32   */
    int32_t active_sh_bases;   /* 1, 4, 9 or 16                                     */
    float near_plane, far_plane, scale_modifier;
    int32_t to_chw, blur_periphery, anti_aliasing;
    int32_t background_type;   /* fhtgs_background_type                             */
    const float* background_data;
    int32_t texture_width, texture_height;
    int32_t fast_math;         /* 1: arithmetic of _C_benchmarking/_C_stereo
                                  (-use_fast_math); 0: IEEE arithmetic of _C         */
    int32_t foveation;         /* fhtgs_foveation; 0 = the reference's                */
    float ring_full, ring_half;/* FHTGS_FOVEATION_RINGS: NDC radii (see below)        */
} fhtgs_settings;

/* Foveation modes (fhtgs_settings.foveation).
 *   REFERENCE: the reference's fixed layout (config.h:30-35): 16x16 tiles whose centre lies
 *     within 15 tiles (240 px) of the gaze tile at full resolution, up to 24 tiles (375 px)
 *     at full resolution cross-faded into the periphery, the rest sampled at stride 2 and
 *     upsampled bilinearly.  The only mode the reference has; the drop-in calls use it.
 *   RINGS: no counterpart in the reference.  A tile whose centre lies at NDC distance
 *     r < ring_full from the gaze (x and y each scaled by half the image size) is rendered at
 *     full resolution, r < ring_half at stride 2, the rest at stride 4; strided tiles are
 *     upsampled bilinearly from their own samples and the first row/column of their right and
 *     lower neighbours (a 2x tile does not sample a 4x neighbour; masked neighbours are
 *     clamped into the tile).  Ring boundaries are hard tile edges (no cross-fade).
 *     blur_periphery is not available in this mode.
 *   NONE: every visible tile at full resolution. */
typedef enum {
    FHTGS_FOVEATION_REFERENCE = 0,
    FHTGS_FOVEATION_RINGS = 1,
    FHTGS_FOVEATION_NONE = 2
} fhtgs_foveation;

/* Per-view facts of the last frame rendered by a context (read after it completed). */
typedef struct {
    int64_t n_instances;       /* reference's M = sum of touched-tile counts (sub-tile copies
                                  of fovea tiles and over-counted sentinel slots included);
                                  in the RINGS / NONE foveation modes the stored count      */
    int64_t instance_capacity; /* stored-instance slots available per view                 */
    uint32_t n_active_tiles;   /* small-tile entries in the tile index map                 */
    uint32_t partition_ranges[6]; /* fovea, periphery, blended [begin,end)                 */
    int32_t overflow;          /* 1 when n_instances_stored > instance_capacity             */
    int32_t end_bit;           /* reference key bits (bit width of small tiles + 1)         */
    int64_t n_instances_stored;/* instances actually stored and sorted: one per (Gaussian,
                                  visible 16x16 tile)                                      */
} fhtgs_frame_info;

/* Intermediates of one view of the last frame, copied to HOST buffers (any may be NULL), in
 * the reference's layout: keys are small-tile ids widened to uint32, the list of a fovea-circle
 * tile appears once per sub-tile, and over-counted slots follow as sentinel keys (0xFFFF for
 * 16-bit keys, else 0xFFFFFFFF) with value 0xFFFFFFFF.  The renderer itself stores each list
 * once; these arrays are expanded from it exactly. */
/* In the RINGS / NONE foveation modes there is no reference layout: keys, values and ranges
 * hold each stored list once, keyed by its large tile's first sub-tile (4 * tile). */
typedef struct {
    uint32_t* n_touched;      /* [N]           */
    uint16_t* screen_bounds;  /* [N,4]         */
    float* vpmt;              /* [N,12] VPMT1, VPMT2, VPMT4 */
    float* rgba;              /* [N,4]         */
    uint32_t* tile_index_map_partitioned; /* [n_active_tiles] */
    uint8_t* tile_type_partitioned;       /* [n_active_tiles] */
    uint32_t* keys;           /* [n_instances] sorted */
    uint32_t* values;         /* [n_instances] sorted */
    uint32_t* instance_ranges;/* [2*T], T = 4 * ceil(W/16) * ceil(H/16) */
} fhtgs_intermediates;

/* ---- context ---- */
fhtgs_status fhtgs_context_create(int32_t device, fhtgs_context* out);
fhtgs_status fhtgs_context_destroy(fhtgs_context ctx);
/* Reserve arena space for up to n_views views of n_primitives Gaussians with the given
 * instance capacity per view (0: estimate).  Optional; rendering grows the arena. */
fhtgs_status fhtgs_context_reserve(fhtgs_context ctx, int32_t n_primitives, int32_t n_views,
                                   int32_t max_width, int32_t max_height, int64_t instances_per_view);
size_t fhtgs_context_arena_bytes(fhtgs_context ctx);
/* Total kernels this context has launched (all frames). */
int64_t fhtgs_context_launch_count(fhtgs_context ctx);

/* ---- stage timing ----
 * With profiling on, every frame records CUDA events on its stream between the stages:
 *   0 setup (status reset, camera gather), 1 preprocess (the tile classification runs beside
 *   it on a second stream of the context), 2 scan+create instances, 3 sort,
 *   4 tile ranges + blend work order, 5 blend (all tiles), 6 compose.
 * fhtgs_get_stage_times waits for the last frame and returns the milliseconds per stage. */
#define FHTGS_N_STAGES 7
fhtgs_status fhtgs_context_set_profiling(fhtgs_context ctx, int32_t enable);
fhtgs_status fhtgs_get_stage_times(fhtgs_context ctx, float* ms, int32_t n);
/* Stage times of up to the last 64 profiled frames, oldest first: ms[f*FHTGS_N_STAGES + s]. */
fhtgs_status fhtgs_get_stage_history(fhtgs_context ctx, float* ms, int32_t max_frames, int32_t* n_frames);

/* ---- rendering ---- */
/* Renders n_views views of one scene, asynchronously on `stream` (cudaStream_t).
 * Returns FHTGS_OK once queued; instance overflow is reported by fhtgs_get_frame_info after the
 * stream has completed the frame. */
fhtgs_status fhtgs_render_views(fhtgs_context ctx, const fhtgs_primitives* prims,
                                const fhtgs_view* views, int32_t n_views,
                                const fhtgs_settings* settings, void* stream);
/* As fhtgs_render_views, then waits for the frame; on instance overflow it grows the arena
 * and renders again, so the images are always complete on FHTGS_OK. */
fhtgs_status fhtgs_render_views_sync(fhtgs_context ctx, const fhtgs_primitives* prims,
                                     const fhtgs_view* views, int32_t n_views,
                                     const fhtgs_settings* settings, void* stream);
/* Waits for the last frame and reports one view of it.  FHTGS_ERR_CUDA if the frame is
 * incomplete because one of its bounded device-side waits gave up (the sort's look-back over
 * earlier tiles, or the preprocess's bulk-copy barrier). */
fhtgs_status fhtgs_get_frame_info(fhtgs_context ctx, int32_t view, fhtgs_frame_info* out);
fhtgs_status fhtgs_copy_intermediates(fhtgs_context ctx, int32_t view, fhtgs_intermediates* out);

/* ---- tests of the bounded device-side waits ----
 * No counterpart in the reference, whose kernels neither wait on one another nor report errors.
 * Two stages of a frame wait on the device, each with an iteration limit after which the kernel
 * records an error bit and returns instead of hanging: the sort's decoupled look-back over the
 * counts that earlier tiles publish, and the preprocess's wait for the bulk copies that stage a
 * block's Gaussians in shared memory.  A view whose wait gave up renders background only and
 * fhtgs_get_frame_info (and the _sync calls) return FHTGS_ERR_CUDA naming the stage; the next
 * frame is unaffected.  This call arms the next frame `ctx` renders (fhtgs_frame_graph_create
 * renders one eagerly first, which consumes it) so that one wait runs out, without any fault:
 *   FHTGS_WAIT_TEST_SORT_LOOKBACK: tile 0 of the first sort pass is never handed out, so its
 *     counts are never published; tile 1's look-back gives up after `limit` reads
 *     (0 <= limit <= 4194304, the default).  Needs more than one sort tile (4096 instances).
 *   FHTGS_WAIT_TEST_STAGING: the preprocess declares its staging late after `limit` polls
 *     (0 <= limit <= 1048576, the default; 0 = at once), then drains the copies in flight
 *     before the block exits.  Only the fast-math flavour stages (16-byte aligned arrays). */
#define FHTGS_WAIT_TEST_SORT_LOOKBACK 1
#define FHTGS_WAIT_TEST_STAGING 2
fhtgs_status fhtgs_context_test_wait_timeout(fhtgs_context ctx, int32_t which, int32_t limit);

/* ---- drop-in mirrors of the reference's positional entry points (blocking) ----
 * Arguments follow the reference's order; tensors become device pointers (+ the sizes the
 * reference reads from tensor shapes), gaze_position becomes two host floats, and the output
 * image(s) are caller-allocated device buffers. */
fhtgs_status fhtgs_render_mono(
    fhtgs_context ctx,
    const float* positions, const float* scales, const float* rotations, const float* opacities,
    const float* sh_0, const float* sh_rest, int32_t n_primitives, int32_t total_sh_bases,
    const float* M, const float* VPM, const float* VPR_inv, const float* cam_position,
    float gaze_x, float gaze_y,
    const uint32_t* visibility_mask, const uint32_t* visibility_mask_area_table,
    const uint32_t* fovea_mask_area_table,
    const float* background_model_data, int32_t texture_width, int32_t texture_height,
    int32_t background_model_type, int32_t K, int32_t active_sh_bases, int32_t width, int32_t height,
    float focal_x, float focal_y, float center_x, float center_y,
    float near_plane, float far_plane, float scale_modifier,
    int32_t to_chw, int32_t blur_periphery, int32_t anti_aliasing,
    float* image, void* stream);
/* Same arguments; the fast-math arithmetic of the reference's benchmarking module. */
fhtgs_status fhtgs_benchmark_mono(
    fhtgs_context ctx,
    const float* positions, const float* scales, const float* rotations, const float* opacities,
    const float* sh_0, const float* sh_rest, int32_t n_primitives, int32_t total_sh_bases,
    const float* M, const float* VPM, const float* VPR_inv, const float* cam_position,
    float gaze_x, float gaze_y,
    const uint32_t* visibility_mask, const uint32_t* visibility_mask_area_table,
    const uint32_t* fovea_mask_area_table,
    const float* background_model_data, int32_t texture_width, int32_t texture_height,
    int32_t background_model_type, int32_t K, int32_t active_sh_bases, int32_t width, int32_t height,
    float focal_x, float focal_y, float center_x, float center_y,
    float near_plane, float far_plane, float scale_modifier,
    int32_t to_chw, int32_t blur_periphery, int32_t anti_aliasing,
    float* image, void* stream);
/* Stereo: as the reference, K, SH bases, near/far, scale modifier and background model of
 * the LEFT settings apply to both eyes (inference_stereo_api.cu:111-120,180-186). */
fhtgs_status fhtgs_render_stereo(
    fhtgs_context ctx,
    const float* positions, const float* scales, const float* rotations, const float* opacities,
    const float* sh_0, const float* sh_rest, int32_t n_primitives, int32_t total_sh_bases,
    const float* M_left, const float* VPM_left, const float* VPR_inv_left, const float* cam_position_left,
    float gaze_x_left, float gaze_y_left,
    const uint32_t* visibility_mask_left, const uint32_t* visibility_mask_area_table_left,
    const uint32_t* fovea_mask_area_table_left,
    const float* background_model_data_left, int32_t texture_width_left, int32_t texture_height_left,
    int32_t background_model_type_left, int32_t K_left, int32_t active_sh_bases_left,
    int32_t width_left, int32_t height_left,
    float focal_x_left, float focal_y_left, float center_x_left, float center_y_left,
    float near_plane_left, float far_plane_left, float scale_modifier_left,
    const float* M_right, const float* VPM_right, const float* VPR_inv_right, const float* cam_position_right,
    float gaze_x_right, float gaze_y_right,
    const uint32_t* visibility_mask_right, const uint32_t* visibility_mask_area_table_right,
    const uint32_t* fovea_mask_area_table_right,
    int32_t width_right, int32_t height_right,
    float focal_x_right, float focal_y_right, float center_x_right, float center_y_right,
    int32_t to_chw, int32_t blur_periphery, int32_t anti_aliasing,
    float* image_left, float* image_right, void* stream);

/* ---- sorting without device allocation ----
 * No counterpart in the reference.  For callers that must not allocate device memory — a VR
 * compositor or display thread that cannot afford the stall of a cudaMalloc/cudaFree, or a
 * plugin whose host application owns the whole device-memory budget — this runs the
 * renderer's stable instance sort (tile key, primitive index) with working memory in a fixed
 * device array inside libfhtgs.so (about 8.3 MB, held by every GPU that loads the library
 * until the process exits) instead of the context arena.
 *   keys_in/values_in -> keys_out/values_out: n pairs on the current device, keys of key_bytes
 *   (2 or 4) bytes sorted stably by their low end_bit bits alone (higher bits are carried
 *   along and do not affect the order, as cub's end_bit); the inputs are not modified, except
 *   in an in-place call (keys_out == keys_in and/or values_out == values_in).  Any other
 *   overlap between the four buffers fails with FHTGS_ERR_INVALID_ARGUMENT.
 *   n <= 1048576, larger requests fail with FHTGS_ERR_INVALID_ARGUMENT.
 * The array is shared by all calls on a device and keeps the last call's contents (nothing in
 * it needs to start at zero); calls that overlap on the GPU race on it, so serialise them.  The
 * first call on each device looks up the array's address and keeps it; make that call before
 * any stream capture, and do not cudaDeviceReset a device while the library is in use on it.
 * A CUDA error that an earlier call left pending is not consumed: the sort returns
 * FHTGS_ERR_CUDA naming it and does not run.
 * Asynchronous on `stream`; no allocation of any kind. */
fhtgs_status fhtgs_sort_instances_noalloc(const void* keys_in, const uint32_t* values_in,
                                          void* keys_out, uint32_t* values_out, int64_t n,
                                          int32_t key_bytes, int32_t end_bit, void* stream);

/* ---- batched frames: tuning, autotuner, captured frame graphs ----
 * No counterpart in the reference (one view per blocking call, inference.cu:49-472).
 *
 * Tuning knobs of a context; every choice renders identical images (they change which pairs
 * the blend culls as hopeless and how the sort is tiled, never a pixel's arithmetic):
 *   blend_warp_width     pixels per warp row in the blend: 8 (8x4 pixels), 16 (16x2) or 4 (4x8)
 *   blend_blocks_per_sm  persistent blend blocks per SM; 0 = as many as fit
 *   sort_items           keys per thread of a radix-sort tile: 8, 12 or 16 (tile = 256 x items) */
typedef struct fhtgs_tuning {
    int32_t blend_warp_width;
    int32_t blend_blocks_per_sm;
    int32_t sort_items;
} fhtgs_tuning;
fhtgs_status fhtgs_context_set_tuning(fhtgs_context ctx, const fhtgs_tuning* tuning);
fhtgs_status fhtgs_context_get_tuning(fhtgs_context ctx, fhtgs_tuning* tuning);
/* Split blend, a tolerance mode (off by default).  A full-resolution tile's K-buffer walk over its
 * whole list is the serial critical path of a frame; with the mode on, a tile whose list is
 * longer than `segment_share` x (the frame's instances / persistent blend blocks) is blended as
 * up to 8 contiguous segments on different blocks.  Each segment records the fragments that enter
 * its own K-buffer; the last segment to finish replays them in list order, which reproduces every
 * K-buffer insertion and eviction of the serial walk (reference blend_cu, inference.cuh:188-240),
 * so only the float summation order of the tail and of its transmittance changes (images differ
 * from the bit-identical path by rounding only).  `records` (0 = 8 K + 64) bounds the records a
 * segment keeps per pixel (20 bytes each); a tile with a pixel over the bound is blended whole,
 * serially (counted as a fallback).  segment_share: 0 (off) or in [0.05, 8].  Applies from the
 * next frame. */
fhtgs_status fhtgs_context_set_blend_split(fhtgs_context ctx, float segment_share, int32_t records);
/* The exact split blend (exact = 1; 0 returns to the records above): the segments log, per pixel
 * and in list order, the alpha and depth of every Gaussian their warps evaluate (8 bytes each,
 * and each step's Gaussian colour), and the last segment of a tile replays the log with the
 * walk's own K-buffer and tail steps, so the operations and their order are those of the serial
 * walk: images bit-identical to the default path.  The logs share one pool of `log_bytes`
 * (0 = 8 GiB; about 2.2 KB per list entry of a split tile); a tile whose segments do
 * not fit it is blended whole.  The share set by fhtgs_context_set_blend_split applies. */
fhtgs_status fhtgs_context_set_blend_split_exact(fhtgs_context ctx, int32_t exact, int64_t log_bytes);
/* The last frame's split blend: tiles split, segments blended, tiles blended whole after a record
 * overflow, and the most records one pixel of a segment produced.  Waits for the context's last
 * frame. */
fhtgs_status fhtgs_context_get_blend_split_stats(fhtgs_context ctx, int32_t* split_tiles, int32_t* segments,
                                                 int32_t* whole_fallbacks, int32_t* max_records);
/* Autotuner: renders the given frame with each candidate and keeps the fastest.  The blend knobs
 * are chosen first by the blend's CUDA-event time (width x blocks), then sort_items by the
 * sort's; each candidate is timed as the median of `repeats` (1..32) frames after one warm-up
 * frame.  The winner becomes the context's tuning and is returned with its median frame time.
 * Blocks the calling thread; profiling is switched on for the search and restored after. */
fhtgs_status fhtgs_autotune(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views,
                            int32_t n_views, const fhtgs_settings* settings, int32_t repeats,
                            fhtgs_tuning* best, float* best_frame_ms, void* stream);

/* A frame of n views captured once into a CUDA graph and replayed by one launch.  Everything the
 * views point to is baked in by address: the caller updates camera matrices, masks and
 * Gaussians in place between launches and reads the images from the same buffers.  Gaze:
 * `gaze_device` = NULL keeps the host values of views[]; otherwise [n_views][2] floats in device
 * memory are read (clamped and rounded as on the host) at every launch.  Creation renders the
 * frame eagerly first and sizes the instance capacity at `capacity_headroom` (>= 1) times the
 * largest per-view count, so that moving cameras fit; a launch whose instances exceed it sets
 * `overflow` in fhtgs_get_frame_info (create the graph again then).  A graph belongs to its
 * context: launching it after the context's arena moved (a larger eager frame, a reserve, a
 * tuning change that grows it) fails with FHTGS_ERR_NOT_READY.  One frame at a time per context. */
typedef struct fhtgs_frame_graph_s* fhtgs_frame_graph;
fhtgs_status fhtgs_frame_graph_create(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views,
                                      int32_t n_views, const fhtgs_settings* settings, const float* gaze_device,
                                      float capacity_headroom, fhtgs_frame_graph* out, void* stream);
fhtgs_status fhtgs_frame_graph_launch(fhtgs_frame_graph graph, void* stream);
fhtgs_status fhtgs_frame_graph_destroy(fhtgs_frame_graph graph);

/* ---- serving: resident scenes, a request queue and continuous batching ----
 * No counterpart in the reference, which renders one view (_C) or one stereo pair (_C_stereo)
 * per blocking call (inference.cu:49-472, inference_stereo.cu:49-828).
 *
 * A server owns one scheduler thread and `max_in_flight` frame slots (a context, a stream and
 * pinned staging each) on one device.  Scenes stay resident: the caller's device arrays are
 * borrowed until the scene is removed, and their bytes count against the budget.  Requests (one
 * or two eyes of one scene) are submitted from any host thread and queue up.  Whenever a slot is
 * free the scheduler takes the oldest queued request together with every other queued request of
 * the same scene (up to `max_batch_requests`) and renders all their views as ONE frame on that
 * slot's stream: requests that arrive while others are on the GPU join the next frame of their
 * scene as soon as a slot frees up, and the frames of different slots overlap on the device.
 * Nothing in the loop waits for the GPU: a frame's status (instance count) comes back by an
 * asynchronous copy and its completion by a host function on the slot's stream.  A frame whose
 * instances overflowed the slot's capacity is rendered again with a larger capacity (its
 * requests keep their place at the head of the queue).
 *
 * Admission: before a frame is launched, the device memory it needs (the slot's arena for its
 * views and instance capacity, plus server-owned output images) is checked against
 * `hbm_budget_bytes` together with everything already resident (scenes, the other slots' arenas,
 * output images, tables).  A frame that does not fit is shrunk to fewer requests; if one request
 * alone does not fit, idle slots' arenas and unused output buffers are freed, and otherwise the
 * frame waits until running frames complete.  A request that cannot fit even with nothing else
 * running fails with FHTGS_ERR_OUT_OF_MEMORY.
 *
 * Output: an eye whose `image` is a device pointer is rendered into it (the caller keeps it alive
 * until the completion); with `image` NULL the server renders into an output buffer of its own
 * (counted against the budget, recycled) whose address the completion returns; it stays valid
 * until fhtgs_server_release(ticket).
 * Results: every view is rendered exactly as fhtgs_render_views renders it alone — a request's
 * images do not depend on what else shares its frame (with blend_split_permille set, up to the
 * split blend's rounding of the tail sums: which tiles are split depends on the frame). */
typedef struct fhtgs_server_s* fhtgs_server;

typedef struct {
    int32_t device;
    int32_t max_in_flight;       /* frame slots, 1..8; 0 = 2                                  */
    int32_t max_batch_requests;  /* requests fused into one frame, 1..64; 0 = 8                */
    int32_t blend_split_permille; /* split blend of every frame (fhtgs_context_set_blend_split):
                                     segment share x 1000, 50..8000; 0 = off                   */
    int64_t hbm_budget_bytes;    /* device memory the server may account for; 0 = 150 GB      */
} fhtgs_server_config;

/* One eye of a request.  The camera values are host floats, copied at submit. */
typedef struct {
    float M[12];            /* world -> view, row-major [3,4]                                 */
    float VPM[16];          /* world -> screen [4,4]                                          */
    float VPR_inv[16];      /* screen -> world direction [4,4]                                */
    float cam_position[3];
    float gaze_x, gaze_y;   /* pixels                                                         */
    int32_t width, height;
    float focal_x, focal_y, center_x, center_y;
    /* device tile tables as in fhtgs_view; NULL visibility mask and area table = every tile
     * visible (tables built once per resolution by the server); NULL fovea table = the
     * standard 49x49 table */
    const uint32_t* visibility_mask;
    const uint32_t* visibility_mask_area_table;
    const uint32_t* fovea_mask_area_table;
    float* image;           /* device output ([3,H,W] or [H,W,3] per the scene's to_chw), or
                               NULL for a server-owned output buffer                           */
} fhtgs_eye;

typedef struct {
    int32_t scene;          /* id from fhtgs_server_add_scene                                 */
    int32_t n_eyes;         /* 1 or 2                                                         */
    uint64_t tag;           /* returned unchanged in the completion                           */
    /* optional cudaEvent_t recorded after the request's device inputs (mask tables, output
     * images) were produced or last used on the caller's streams; the frame's stream waits
     * for it.  NULL: those buffers are ready at submit.  Keep the event alive until the
     * request completes. */
    void* ready_event;
    fhtgs_eye eyes[2];
} fhtgs_request;

typedef struct {
    int64_t ticket;
    uint64_t tag;
    int32_t status;          /* fhtgs_status of this request                                  */
    int32_t frame_views;     /* views in the frame that rendered it (0 if it never ran)       */
    double submit_ms;        /* server clock (fhtgs_server_clock_ms) at submit                */
    double launch_ms;        /* when its (last) frame was enqueued                            */
    double done_ms;          /* when its frame completed on the GPU                           */
    float* images[2];        /* device images of the eyes (the caller's or server-owned)      */
    char message[96];        /* reason of a failure, empty on FHTGS_OK                        */
} fhtgs_completion;

typedef struct {
    int64_t submitted, completed, failed;
    int64_t frames, views, retries;      /* frames launched, views rendered, overflow re-renders */
    int64_t queued, in_flight;           /* requests waiting / in running frames, right now      */
    int64_t resident_bytes;              /* accounted against the budget, right now             */
    int64_t peak_resident_bytes;
    int64_t admission_waits;             /* times a frame waited for memory to free up          */
    int64_t max_frame_requests;          /* largest number of requests fused into one frame     */
} fhtgs_server_stats;

fhtgs_status fhtgs_server_create(const fhtgs_server_config* config, fhtgs_server* out);
/* Fails queued requests (FHTGS_ERR_NOT_READY), waits for running frames, frees everything the
 * server allocated.  Completions not yet polled are dropped. */
fhtgs_status fhtgs_server_destroy(fhtgs_server server);
/* Registers a resident scene; `prims` (device arrays, complete when this is called: the
 * server's streams do not wait for the caller's) and `settings` (K, SH bases, planes,
 * background, to_chw, blur, math) apply to every request of the scene.  Fails with
 * FHTGS_ERR_OUT_OF_MEMORY if its bytes do not fit the budget beside what is resident. */
fhtgs_status fhtgs_server_add_scene(fhtgs_server server, const fhtgs_primitives* prims,
                                    const fhtgs_settings* settings, int32_t* scene_id);
/* Queued requests of the scene fail; running frames finish; then its bytes leave the budget. */
fhtgs_status fhtgs_server_remove_scene(fhtgs_server server, int32_t scene_id);
fhtgs_status fhtgs_server_submit(fhtgs_server server, const fhtgs_request* request, int64_t* ticket);
/* Moves up to max_completions finished requests (in completion order) into `out`; waits up to
 * wait_ms for the first one when none is ready. */
fhtgs_status fhtgs_server_poll(fhtgs_server server, fhtgs_completion* out, int32_t max_completions,
                               int32_t wait_ms, int32_t* n_out);
/* Returns the server-owned output buffers of a completed request to the server's pool. */
fhtgs_status fhtgs_server_release(fhtgs_server server, int64_t ticket);
/* Paused (1), the server accepts requests but launches no new frame; running frames finish.
 * Resumed (0), it forms frames from everything queued.  For maintenance windows, and to hand a
 * whole burst of requests to the batcher at once. */
fhtgs_status fhtgs_server_set_paused(fhtgs_server server, int32_t paused);
/* Waits until no request is queued or running (FHTGS_ERR_NOT_READY after timeout_ms; < 0 = no
 * limit). */
fhtgs_status fhtgs_server_drain(fhtgs_server server, int32_t timeout_ms);
fhtgs_status fhtgs_server_get_stats(fhtgs_server server, fhtgs_server_stats* out);
double fhtgs_server_clock_ms(fhtgs_server server);   /* ms since the server was created */

/* ---- several GPUs: a replica group of servers ----
 * No counterpart in the reference (one GPU; one view or stereo pair per blocking call).
 * Views are independent once their camera is known, and the K-buffer blend cannot merge partial
 * results over a split of the Gaussians (the core is quantised to RGBA8 as fragments arrive), so
 * several GPUs serve more requests by each holding a REPLICA of every scene and rendering each
 * request, whole, on one of them.  A group owns one server per entry of `devices` (configured by
 * `config`, whose device field is ignored); a device may appear more than once (several
 * replicas on one GPU).  Nothing crosses devices per frame: no collective, no peer traffic.
 *  - add_scene: the caller's arrays (and background data) lie on `home_device`.  The first
 *    replica on that device borrows them; every other replica gets its own copy in its device's
 *    HBM (cudaMemcpyPeerAsync; the call returns once the copies landed), counted in its server's
 *    budget.  Copies are freed when the group is destroyed.
 *  - submit: the request goes, whole, to the replica with the least outstanding work: the
 *    pixels of its eyes times (1 + Gaussians / 262144), summed over the requests routed to it
 *    whose completions have not been polled yet; ties go round robin.  A request whose eyes carry
 *    device buffers (masks, tables, output images) is routed among the replicas on the device of
 *    those buffers; one without any goes to any replica and gets server-owned outputs there.
 *    `replica` (may be NULL) receives the replica's index.
 *  - poll: completions of every replica, in group tickets, with the replica and its device.
 *  - get_stats: one replica's server statistics and its outstanding work. */
typedef struct fhtgs_server_group_s* fhtgs_server_group;

typedef struct {
    fhtgs_completion completion;   /* ticket: the group's ticket                                  */
    int32_t replica;               /* index into the group's devices                              */
    int32_t device;                /* where completion.images lie                                 */
} fhtgs_group_completion;

fhtgs_status fhtgs_server_group_create(const int32_t* devices, int32_t n_devices,
                                       const fhtgs_server_config* config, fhtgs_server_group* out);
/* Destroys every replica's server (running frames finish) and frees the scene copies. */
fhtgs_status fhtgs_server_group_destroy(fhtgs_server_group group);
int32_t fhtgs_server_group_size(fhtgs_server_group group);
fhtgs_status fhtgs_server_group_add_scene(fhtgs_server_group group, int32_t home_device,
                                          const fhtgs_primitives* prims, const fhtgs_settings* settings,
                                          int32_t* scene_id);
fhtgs_status fhtgs_server_group_remove_scene(fhtgs_server_group group, int32_t scene_id);
fhtgs_status fhtgs_server_group_submit(fhtgs_server_group group, const fhtgs_request* request,
                                       int64_t* ticket, int32_t* replica);
fhtgs_status fhtgs_server_group_poll(fhtgs_server_group group, fhtgs_group_completion* out,
                                     int32_t max_completions, int32_t wait_ms, int32_t* n_out);
fhtgs_status fhtgs_server_group_release(fhtgs_server_group group, int64_t ticket);
fhtgs_status fhtgs_server_group_drain(fhtgs_server_group group, int32_t timeout_ms);
fhtgs_status fhtgs_server_group_get_stats(fhtgs_server_group group, int32_t replica, fhtgs_server_stats* out,
                                          int64_t* outstanding_cost);

/* ---- tile masks on the device ----
 * No counterpart in the reference, which takes the three mask tensors precomputed by the
 * calling framework (torch_bindings/rasterization.py:22-43; read at
 * rasterization/include/utils/kernel_utils.cuh:168-210).  Builds them on `stream` from one byte
 * per 16x16 tile of a width x height view (row-major, grid ceil(width/16) x ceil(height/16);
 * non-zero = visible; NULL = every tile visible):
 *   visibility_mask            ceil(tiles/32) words, bit t%32 of word t/32 = tile t visible
 *   visibility_mask_area_table (grid_w+1)*(grid_h+1) summed-area table, leading zero row/column
 *   fovea_mask_area_table      49*49 table counting 3 extra sub-tiles per tile of the 48x48
 *                              window around the gaze whose centre is inside the 24-tile circle
 *                              (gaze-independent; NULL = skip).
 * One launch, no allocation. */
fhtgs_status fhtgs_build_tile_masks(const uint8_t* visible_tiles, int32_t width, int32_t height,
                                    uint32_t* visibility_mask, uint32_t* visibility_mask_area_table,
                                    uint32_t* fovea_mask_area_table, void* stream);

/* ---- display-ready output ----
 * No counterpart in the reference (its images are float32 RGB).  Packs n_views (1..8) float
 * images of width x height (HWC, or CHW when to_chw) into one RGBA8 (BGRA8 when bgra) image of
 * (n_views*width) x height, views side by side left to right (stereo: left | right), alpha 255.
 * Each channel: clamp to [0,1] (NaN -> 0), then trunc(fma(c, 255, 0.5)).  `images` is a host
 * array of device pointers; `out` is device memory of 4*n_views*width*height bytes. */
fhtgs_status fhtgs_pack_display(const float* const* images, int32_t n_views, int32_t width, int32_t height,
                                int32_t to_chw, int32_t bgra, uint8_t* out, void* stream);

/* ---- debug overlays (replace _C_visualization, torch_bindings/bindings_visualization.cpp:8-9) ----
 * fhtgs_visualize_gaze: visualization/src/visualization_api.cu:13-35 + visualization.cu:27-57.
 *   Draws a marker of visualization_size pixels in (r,g,b) at the gaze (host floats, clamped to
 *   the image) into the device image: type 0 circle, 2 cross, any other value < 256 a square.
 * fhtgs_visualize_tile_boundaries: visualization_api.cu:37-64 + visualization.cu:60-236.
 *   Outlines every visible tile of `visibility_mask` (device words as above) by its class for the
 *   gaze: fovea sub-tiles orange (0.902,0.624,0), blended sub-tiles light blue
 *   (0.337,0.706,0.914), periphery tiles green (0,0.620,0.451); nothing when at most one tile
 *   entry is active, as in the reference.  One launch, no host synchronisation.
 * Both asynchronous on `stream`; image is HWC float32 RGB, or CHW when to_chw. */
fhtgs_status fhtgs_visualize_gaze(float* image, int32_t width, int32_t height, float gaze_x, float gaze_y,
                                  float r, float g, float b, int32_t visualization_type,
                                  int32_t visualization_size, int32_t to_chw, void* stream);
fhtgs_status fhtgs_visualize_tile_boundaries(float* image, int32_t width, int32_t height,
                                             const uint32_t* visibility_mask, float gaze_x, float gaze_y,
                                             int32_t to_chw, void* stream);

/* ---- errors / version ---- */
const char* fhtgs_last_error(void);   /* thread-local message of the last failure */
int32_t fhtgs_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FHTGS_H_ */
