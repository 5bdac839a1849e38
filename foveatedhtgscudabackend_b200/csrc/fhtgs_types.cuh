// Shared host/device definitions of the fhtgs renderer: constants, per-view parameters,
// frame buffers and the table of kernel launchers each math flavour exports.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fhtgs {

// Renderer constants; identical values to rasterization/include/config.h:13-45 of the
// reference (thresholds, tile sizes, foveation radius 375 px / blend band 125 px).
constexpr float kTransmittanceThreshold = 1e-4f;
constexpr float kMaxFragmentAlpha = 1.0f;
constexpr float kMinAlphaRcp = 255.0f;
constexpr float kMinAlpha = 1.0f / kMinAlphaRcp;
constexpr float kMaxCutoffSq = 11.0825270903f;
constexpr float kMinAlphaCore = 1.0f / 20.0f;
constexpr int kTileSmall = 8;
constexpr int kTileLarge = 16;
constexpr int kStride = kTileLarge / kTileSmall;      // 2
constexpr int kSubTiles = kStride * kStride;          // 4
constexpr int kFoveaRadiusPx = 375;
constexpr int kFoveaRadiusTiles = (kFoveaRadiusPx + kTileLarge - 1) / kTileLarge;  // 24
constexpr int kBlendWidthPx = 125;
constexpr int kBlendRadiusTiles = (kFoveaRadiusPx - kBlendWidthPx) / kTileLarge;   // 15
constexpr int kBlendRadiusPx = kBlendRadiusTiles * kTileLarge;                     // 240
constexpr int kFoveaTableSide = 2 * kFoveaRadiusTiles + 1;                         // 49

// kQuarter exists only in the ring foveation mode (tiles sampled at stride 4).
enum TileType : uint8_t { kFovea = 0, kPeriphery = 1, kBlended = 2, kMasked = 3, kQuarter = 4 };
constexpr int kQuarterStride = 4;

// Foveation modes (fhtgs_settings.foveation): the reference's fixed fovea/blend/periphery
// tiles; rings by NDC distance from the gaze (full / 2x down / 4x down); none (all full).
enum FoveationMode : int { kFoveationReference = 0, kFoveationRings = 1, kFoveationNone = 2 };

// Per-view parameters, resident in device memory for the whole frame (filled by the
// setup kernel from the caller's device matrices and host scalars).
struct ViewParams {
    float4 M[3];
    float4 VPM[4];
    float4 VPR_inv[4];
    float4 cam;            // xyz
    float2 gaze_px;        // clamped to the image (inference.cu:79-82)
    float2 gaze_tiles;     // float of the int gaze tile (inference.cu:98-105)
    int2 gaze_tiles_i;
    int width, height;
    float focal_x, focal_y, center_x, center_y;
    int glw, glh;          // large-tile grid
    int n_large, n_tiles;  // large tiles, small-tile ids (4 per large tile)
    const uint32_t* vis_mask;
    const uint32_t* vis_sat;
    const uint32_t* fovea_sat;
    float* image;          // final image
    float* work;           // blend target of periphery/blended tiles (temp buffer when blurring)
    int fov_mode;          // FoveationMode of this view
    float ring_full2;      // rings: squared NDC radius of full resolution
    float ring_half2;      // rings: squared NDC radius of 2x-down sampling (4x beyond)
};

// Host-side description of a view before the setup kernel runs.
struct ViewSetup {
    const float* M;
    const float* VPM;
    const float* VPR_inv;
    const float* cam;
    const float* gaze;     // device (x, y) read by the setup kernel, or null: gaze fields of p are used
    ViewParams p;          // scalars filled on the host, matrices gathered on the device
};

// Settings shared by all views of a frame (kernel parameter, by value).
struct FrameParams {
    int n_views;
    int n_prims;
    int total_sh;          // S
    int active_sh;
    int K;
    float near_plane, far_plane, scale_modifier;
    int to_chw, blur, aaa;
    int bg_type;
    const float* bg_data;
    int tex_w, tex_h;
    int key_u32;           // 0: 16-bit keys, 1: 32-bit keys
    int end_bit;           // key bits sorted: bit width of the largest large-tile index
    int64_t cap;           // instance slots per view
    int max_tiles;         // max small-tile ids over views (stride of per-tile arrays)
    int max_large;         // max large tiles over views
    int n_blocks_prim;     // preprocess/create blocks per view
    int blend_rw;          // blend: pixels per warp row (4, 8 or 16; 32 / blend_rw rows)
    int blend_blocks;      // persistent blend blocks per SM (0: as many as fit)
    int sort_key_bits;     // three-kernel sort: > 0 = only key bits below this decide the order
                           // (higher bits are carried along, as cub's end_bit); 0 = all bits of
                           // the sort's 8-bit passes (the renderer's keys have no higher bits)
    // Bounded device waits (set by the host for every frame; see kLookSpinLimit and
    // kStageWaitLimit for the defaults):
    int look_spin_limit;   // onesweep look-back: reads of an unpublished word before giving up
    int stage_wait_limit;  // preprocess: polls of the staging barrier before it is declared late
                           // (0: at once, before any copy can have landed)
    int look_first_ticket; // first ticket of the first sort pass: 0; 1 in the wait test (tile 0
                           // is never handed out, so its look-back words are never published)
};

// Per-view frame status written by the device, read by the host after the frame.
// Instances are stored once per (primitive, visible large tile): `n_instances` counts those;
// `n_instances_ref` is the reference's count (sum of touched-tile counts, with the four
// sub-tiles of a fovea tile and the over-counted slots of masked fovea tiles).
struct FrameStatus {
    unsigned long long n_instances;   // stored instances (sorted, blended)
    unsigned long long n_instances_ref;
    uint32_t n_active;                // entries in the partitioned tile map
    uint32_t ranges[6];               // partition ranges (fovea, periphery, blended)
    uint32_t n_fovea_large, n_blended_large, n_periphery_large, n_masked_large;
    uint32_t overflow;
    uint32_t n_quarter_large;         // ring mode: tiles sampled at stride 4 (after the
                                      // periphery tiles in work_low)
};

// Attribute arrays; with `half` set, scales/rotations/opacities hold fp16 and sh_0/sh_rest
// bfloat16 values behind these pointers (positions stay float32).
struct Gaussians {
    const float* positions;
    const float* scales;
    const float* rotations;
    const float* opacities;
    const float* sh_0;
    const float* sh_rest;
    int half;
};

// All per-frame device buffers (arena carve-up); arrays are [view][...] with the strides
// recorded in FrameParams.
struct FrameBuffers {
    ViewParams* views;
    FrameStatus* status;
    uint32_t* n_touched;      // [V][N] reference touched-tile counts
    uint32_t* n_vis;          // [V][N] visible large tiles in the bounds = stored instances
    ushort4* bounds;          // [V][N]
    float4* rec;              // [V][N][4]: VPMT1, VPMT2, VPMT4, rgba
    uint32_t* block_sums;     // [V][n_blocks_prim]
    void* keys[2];            // [V][cap] uint16 or uint32
    uint32_t* vals[2];        // [V][cap]
    int final_buf;            // which of keys/vals holds the sorted result
    uint32_t* sort_hist;      // [V][256][sort_tiles]
    uint32_t* sort_digit_tot; // [V][256]
    int sort_tiles;           // tiles of the radix sort per view (capacity based)
    int sort_items;           // keys per thread of a sort tile (kSortItemChoices)
    uint2* ranges;            // [V][max_large] instance range per large tile
    uint32_t* tile_map_part;  // [V][max_tiles]
    uint8_t* tile_type_part;  // [V][max_tiles]
    uint8_t* large_type;      // [V][max_large]
    uint32_t* work_full;      // [V][max_large] fovea then blended large tiles
    uint32_t* work_low;       // [V][max_large] periphery large tiles, then quarter tiles
    uint32_t* work_masked;    // [V][max_large] masked large tiles
    uint32_t* counters;       // [kCounterWords]: work counters, then the work-order buckets
    uint32_t* work_order[2];  // [0]: [V*max_large] packed blend items, heaviest first; [1] unused
    // Onesweep sort state (null: the three-kernel sort, which needs sort_hist/sort_digit_tot):
    uint32_t* sort_ghist;     // [V][kSortMaxPasses][256] digit counts of every pass (create fills)
    uint32_t* sort_look;      // [V][kSortMaxPasses][sort_tiles][256] look-back words
    uint32_t* sort_ticket;    // [V][kSortMaxPasses] tiles handed out so far
};

// Work ordering: tiles are bucketed by class and by list length in quarter octaves and
// blended in descending bucket order: full-resolution tiles, then periphery, then quarter
// tiles, the longest lists of each class first (longest-processing-time scheduling).
constexpr int kCostBuckets = 130;                     // per tile class
constexpr int kOrderBuckets = 3 * kCostBuckets;       // full-resolution, periphery, quarter
// counters[0..2]: next full-resolution / periphery / quarter item of the blend; then the split
// blend's words; the work-order histogram and cursors follow from kCtrHist.
constexpr int kCtrSplitNext = 3;      // next split segment of the blend
constexpr int kCtrSplitSegs = 4;      // segments reserved by the work order
constexpr int kCtrSplitTiles = 5;     // tiles split
constexpr int kCtrSplitFallback = 6;  // split tiles blended whole after a record overflow
constexpr int kCtrSplitRecMax = 7;    // most records a pixel of a later segment produced
constexpr int kCtrSplitPool = 8;      // exact mode: 256-byte units of the fragment log reserved
                                      // (64-bit: words 8 and 9)
constexpr int kCtrSplitView = 16;     // [256] tiles split per view
constexpr int kCtrHist = kCtrSplitView + 256;
constexpr int kCounterWords = kCtrHist + 2 * kOrderBuckets;  // counters, histogram, cursors
constexpr int kSplitMaxSegments = 8;

// Persistent blend blocks per SM the register allocation has to allow: the K-buffer (2 K
// registers) dominates for large K.
__host__ __device__ constexpr int blend_min_blocks(int K) { return K >= 32 ? 2 : K >= 16 ? 3 : 4; }

// Split blend (a tolerance mode, off by default; its own kernel argument so that the other
// kernels' parameters keep their layout): a full-resolution tile whose list is longer than
// share x (instances of the frame / blocks) is blended as up to kSplitMaxSegments contiguous
// segments on different blocks, merged by the last of them.
struct SplitArgs {
    float share;           // 0: off
    int blocks;            // persistent blend blocks of the launch
    int cap;               // segments the scratch holds
    int recs;              // records a later segment keeps per pixel
    int stride;            // bytes of scratch per segment
    uint32_t* of;          // [V][max_large] per full-resolution item: first segment | S << 28, or ~0
    uint2* list;           // [cap] per segment: packed item, first segment | S << 28 (~0: unused)
    uint32_t* ctl;         // [cap] per first segment: segments finished
    char* scratch;         // [cap][stride] per-pixel state and records
    // [V] the status the blend of the other tiles reads: the view's, with the split tiles taken
    // out of n_fovea_large + n_blended_large (that kernel reads only this sum, and n_fovea_large,
    // which is kept; n_blended_large is adjusted modulo 2^32)
    FrameStatus* status;
    // Exact mode (bit-identical images): every segment logs, per pixel and in list order, the
    // alpha and depth of each Gaussian its warp evaluates; the last segment of a tile replays the
    // whole log with the walk's own K-buffer and tail steps.
    int exact;
    uint32_t pool_units;   // 256-byte units of the fragment log
    char* pool;
    uint32_t* seg_unit;    // [cap] first unit of each segment's log
};

// Exact split: a segment's log, for a segment of at most `stride` list entries (each warp walks
// at most that many steps): n_steps[8] u32 | rgba[8][stride] float4 (each step's Gaussian colour
// and opacity) | frag[8][stride][32] float2 (alpha, or -1 where the pair is no fragment; depth).
__host__ __device__ inline uint32_t split_log_pos_unit() { return 1u; }
__host__ __device__ inline uint32_t split_log_frag_unit(uint32_t stride) { return 1u + (stride + 1u) / 2u; }
__host__ __device__ inline uint32_t split_log_units(uint32_t stride) { return split_log_frag_unit(stride) + 8u * stride; }

// Split blend scratch of one segment (256 pixels; arrays pixel-fastest):
//   first segment:  depth[K][256] f32 | color[K][256] u32 | tail[256] float4 | T[256] f32
//   later segments: n_rec[256] u32 | tail[256] float4 | T[256] f32 | depth[R][256] f32 |
//                   pm[R][256] float4 (the fragments that entered the segment's K-buffer)
constexpr int kSplitPx = 256;
__host__ __device__ constexpr int split_stride_bytes(int K, int R) {
    return (2 * K + 5 > 6 + 5 * R ? 2 * K + 5 : 6 + 5 * R) * 4 * kSplitPx;
}

// Launchers exported by each math flavour (fast = -use_fast_math, ieee = default).
struct KernelSet {
    // Each launcher returns the number of kernels it launched.
    int (*setup)(const ViewSetup* setups, int n_views, ViewParams* out, cudaStream_t s);
    int (*classify)(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s);
    int (*preprocess)(const FrameParams& fp, const FrameBuffers& fb, const Gaussians& g, cudaStream_t s);
    int (*scan_blocks)(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s);
    int (*create_instances)(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s);
    int (*sort)(const FrameParams& fp, FrameBuffers& fb, cudaStream_t s);
    int (*ranges)(const FrameParams& fp, const FrameBuffers& fb, int n_sms, cudaStream_t s);
    int (*order)(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp, int n_sms, cudaStream_t s);
    // `mid` (may be null) is recorded right after the blend.
    // With the split blend on, the split segments' kernel runs first and the blend of the other
    // tiles follows it as a programmatic dependent launch.
    int (*blend)(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp, int n_sms, cudaStream_t s,
                 cudaEvent_t mid);
    int (*compose)(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s);
};

const KernelSet& kernels_fast();
const KernelSet& kernels_ieee();

constexpr int kPrimBlock = 256;      // preprocess / create-instances block
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;        // default keys per thread per sort tile
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 (default tile)
constexpr int kSortItemsMin = 8;      // smallest tile the autotuner may choose (2048 keys)
// Blend warp rectangles the autotuner may choose: pixels per warp row.
constexpr int kBlendRowChoices[3] = {8, 16, 4};
constexpr int kSortRadixBits = 8;
constexpr int kSortBins = 1 << kSortRadixBits;
constexpr int kSortMaxPasses = 3;     // keys of at most 24 significant bits (tile ids < 2^24)
// Look-back words of the onesweep sort: 2 flag bits over a 30-bit count, so the onesweep path
// needs an instance capacity below 2^30 per view (larger arenas use the three-kernel sort).
constexpr int64_t kOnesweepMaxCap = int64_t(1) << 30;
constexpr uint32_t kFrameErrSortLookback = 2u;  // FrameStatus.overflow bit: look-back gave up
constexpr uint32_t kFrameErrStaging = 4u;   // FrameStatus.overflow bit: attribute staging timed out
constexpr uint32_t kFrameErrWait = kFrameErrSortLookback | kFrameErrStaging;
// Default limits of the bounded device waits (FrameParams.look_spin_limit / stage_wait_limit).
constexpr int kLookSpinLimit = 1 << 22;   // reads of an unpublished look-back word (~0.1-1 s)
constexpr int kStageWaitLimit = 1 << 20;  // polls of the preprocess staging barrier

}  // namespace fhtgs
