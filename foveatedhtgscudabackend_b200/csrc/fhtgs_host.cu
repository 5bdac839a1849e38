// Host side of libfhtgs: context with a growable device arena, frame orchestration (all
// views of a frame in the same launches, no device->host round trip inside a frame) and the
// C ABI declared in include/fhtgs.h.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fhtgs.h"
#include "fhtgs_types.cuh"

using namespace fhtgs;

namespace {

thread_local std::string g_error;

fhtgs_status fail(fhtgs_status code, const std::string& msg) {
    g_error = msg;
    return code;
}

#define FHTGS_CK(call)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return fail(FHTGS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr size_t kAlign = 256;
size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

int end_bit_of(uint32_t n) {
    int b = 0;
    while (n) { ++b; n >>= 1; }
    return b;
}

struct ViewGeom {
    int glw, glh, n_large, n_tiles;
    int end_bit;       // reference key bits: bit width of (small tiles + 1)
    int key_bits;      // stored key bits: bit width of the largest large-tile index
    int gaze_tx, gaze_ty;
    float gaze_px, gaze_py;
};

// Grid sizes, key width and gaze rounding of one view (inference.cu:79-105 of the reference,
// including its clamp of the gaze tile to the small-tile grid).
ViewGeom geometry(const fhtgs_view& v) {
    ViewGeom g;
    g.glw = (v.width + kTileLarge - 1) / kTileLarge;
    g.glh = (v.height + kTileLarge - 1) / kTileLarge;
    g.n_large = g.glw * g.glh;
    g.n_tiles = g.n_large * kSubTiles;
    g.end_bit = end_bit_of(static_cast<uint32_t>(g.n_tiles + 1));
    g.key_bits = std::max(1, end_bit_of(static_cast<uint32_t>(g.n_large - 1)));
    g.gaze_px = std::min(std::max(v.gaze_x, 0.0f), static_cast<float>(v.width - 1));
    g.gaze_py = std::min(std::max(v.gaze_y, 0.0f), static_cast<float>(v.height - 1));
    const int gw = g.glw * kStride, gh = g.glh * kStride;
    g.gaze_tx = std::max(0, std::min(gw - 1, (static_cast<int>(g.gaze_px) + kTileLarge / 2) / kTileLarge));
    g.gaze_ty = std::max(0, std::min(gh - 1, (static_cast<int>(g.gaze_py) + kTileLarge / 2) / kTileLarge));
    return g;
}

}  // namespace

namespace fhtgs {
// Lets other translation units of the library report through fhtgs_last_error().
void set_last_error(const std::string& msg) { g_error = msg; }
}  // namespace fhtgs

namespace {
// NVTX ranges of a frame in the "fhtgs" domain: one "frame" range around the enqueue and one
// range per pipeline stage (the stages of the profiling events), so that a timeline tool shows
// the stages and, through CUDA correlation, their kernels.  Without a tool attached each call is
// a check of a null function pointer.
const char* const kStageNames[FHTGS_N_STAGES] = {"setup", "preprocess+classify", "scan+create instances", "sort",
                                                 "ranges+work order", "blend", "compose"};
nvtxDomainHandle_t nvtx_domain() {
    static nvtxDomainHandle_t d = nvtxDomainCreateA("fhtgs");
    return d;
}
void nvtx_push(const char* name) {
    nvtxEventAttributes_t a{};
    a.version = NVTX_VERSION;
    a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
    a.messageType = NVTX_MESSAGE_TYPE_ASCII;
    a.message.ascii = name;
    nvtxDomainRangePushEx(nvtx_domain(), &a);
}
void nvtx_pop() { nvtxDomainRangePop(nvtx_domain()); }
}  // namespace

// Stage boundaries recorded when profiling: start | setup | preprocess (classification beside it) |
// scan+create | sort | ranges+work order | blend | compose.
constexpr int kStageEvents = FHTGS_N_STAGES + 1;
constexpr int kStageRing = 64;   // frames whose stage events are kept

struct fhtgs_context_s {
    int device = 0;
    int n_sms = 148;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    long long arena_generation = 0;   // bumped whenever the arena moves (captured graphs go stale)
    bool capturing = false;           // a frame graph is being captured: no profiling events
    fhtgs_tuning tuning{8, 0, kSortItems};
    float split_share = 0.0f;     // split blend: 0 = off (bit-identical blend)
    int split_exact = 0;          // 1: the exact split (fragment logs, bit-identical images)
    int64_t split_pool = 0;       // bytes of the exact split's fragment log
    bool split_active = false;    // the last frame ran the split blend
    int split_recs = 0;           // records per pixel of a later segment; 0 = 8 K + 64
    int64_t cap = 0;              // instance slots per view
    FrameStatus* h_status = nullptr;  // pinned
    int h_status_n = 0;
    // last frame
    bool have_frame = false;
    FrameParams fp{};
    FrameBuffers fb{};
    std::vector<ViewGeom> geo;
    std::vector<fhtgs_view> views;
    int frame_foveation = 0;          // the settings' foveation of the last frame
    cudaStream_t stream = nullptr;
    // tile classification runs on a second stream beside the preprocess (forked and joined
    // with these events inside every frame)
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // armed by fhtgs_context_test_wait_timeout: the next frame's wait test and its limit
    int wait_test = 0;
    int wait_test_limit = 0;
    // profiling: events around the stages of the last frame, and a launch counter
    bool profile = false;
    cudaEvent_t ev[kStageRing][kStageEvents] = {};
    long long frames_profiled = 0;
    long long launches = 0;
};

namespace {

struct Layout {
    size_t total = 0;
    size_t off_views, off_status, off_nt, off_nvis, off_bounds, off_rec, off_bsums, off_keys0, off_keys1, off_vals0, off_vals1;
    size_t off_hist, off_dtot, off_ranges, off_map, off_type, off_ltype, off_wf, off_wl, off_wm, off_ctr, off_temp;
    size_t off_order0, off_order1;
    size_t off_ghist, off_look, off_ticket;
    size_t off_split_of = 0, off_split_list = 0, off_split_ctl = 0, off_split_scratch = 0, off_split_status = 0;
    size_t off_split_units = 0, off_split_pool = 0;
    std::vector<size_t> temp_offsets;
};

// Split blend sizes of a frame (all zero when the mode is off).
struct SplitPlan {
    float share = 0.0f;
    int blocks = 0, cap = 0, recs = 0, stride = 0, exact = 0;
    uint32_t pool_units = 0;
};

constexpr int64_t kSplitPoolDefault = int64_t(8) << 30;  // exact split: fragment log bytes

SplitPlan split_plan(float share, int recs, int exact, int64_t pool, int K, int blend_blocks_per_sm, int n_sms, int V,
                     int max_large) {
    SplitPlan sp;
    if (!(share > 0.0f)) return sp;
    sp.exact = exact;
    if (exact) sp.pool_units = static_cast<uint32_t>((pool > 0 ? pool : kSplitPoolDefault) / 256);
    const int Ki = K >= 32 ? 32 : K >= 16 ? 16 : K >= 8 ? 8 : K >= 4 ? 4 : K >= 2 ? 2 : 1;  // the blend's K
    const int per_sm = blend_blocks_per_sm > 0 ? std::min(blend_blocks_per_sm, blend_min_blocks(Ki)) : blend_min_blocks(Ki);
    sp.share = share;
    sp.blocks = n_sms * per_sm;
    sp.recs = exact ? 0 : recs > 0 ? recs : 8 * Ki + 64;  // 20 bytes each
    sp.stride = exact ? 0 : split_stride_bytes(Ki, sp.recs);
    // Segments of about the threshold's length cover at most instances / threshold = blocks /
    // share list entries; tiles whose reservation does not fit are blended whole.
    const int64_t bound = static_cast<int64_t>(std::ceil(sp.blocks / static_cast<double>(share))) + 8 * kSplitMaxSegments;
    sp.cap = static_cast<int>(std::min<int64_t>(bound, static_cast<int64_t>(kSplitMaxSegments) * V * max_large));
    return sp;
}

Layout plan(int V, int64_t N, int nbp, int64_t cap, int key_bytes, int sort_tiles, int max_tiles, int max_large,
            const std::vector<int64_t>& temp_floats, const SplitPlan& sp) {
    Layout L;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o = align_up(o + std::max<size_t>(bytes, 1)); return at; };
    L.off_views = take(sizeof(ViewParams) * V);
    L.off_status = take(sizeof(FrameStatus) * V);
    L.off_nt = take(4ull * V * N);
    L.off_nvis = take(4ull * V * N);
    L.off_bounds = take(8ull * V * N);
    L.off_rec = take(64ull * V * N);
    L.off_bsums = take(4ull * V * nbp);
    L.off_keys0 = take(static_cast<size_t>(key_bytes) * V * cap);
    L.off_keys1 = take(static_cast<size_t>(key_bytes) * V * cap);
    L.off_vals0 = take(4ull * V * cap);
    L.off_vals1 = take(4ull * V * cap);
    L.off_hist = take(4ull * V * kSortBins * sort_tiles);
    L.off_dtot = take(4ull * V * kSortBins);
    L.off_ranges = take(8ull * V * max_large);
    L.off_map = take(4ull * V * max_tiles);
    L.off_type = take(1ull * V * max_tiles);
    L.off_ltype = take(1ull * V * max_large);
    L.off_wf = take(4ull * V * max_large);
    L.off_wl = take(4ull * V * max_large);
    L.off_wm = take(4ull * V * max_large);
    L.off_ctr = take(4ull * kCounterWords);
    L.off_order0 = take(4ull * V * max_large);
    L.off_order1 = take(4);
    L.off_ghist = take(4ull * V * kSortMaxPasses * kSortBins);
    L.off_look = take(4ull * V * kSortMaxPasses * sort_tiles * kSortBins);
    L.off_ticket = take(4ull * V * kSortMaxPasses);
    for (int64_t f : temp_floats) L.temp_offsets.push_back(f > 0 ? take(4ull * f) : 0);
    if (sp.cap > 0) {
        L.off_split_of = take(4ull * V * max_large);
        L.off_split_list = take(8ull * sp.cap);
        L.off_split_ctl = take(4ull * sp.cap);
        L.off_split_scratch = take(static_cast<size_t>(sp.stride) * sp.cap);
        L.off_split_status = take(sizeof(FrameStatus) * V);
        L.off_split_units = take(4ull * sp.cap);
        L.off_split_pool = take(256ull * sp.pool_units);
    }
    L.total = o;
    return L;
}

fhtgs_status ensure_arena(fhtgs_context ctx, size_t bytes) {
    if (bytes <= ctx->arena_bytes) return FHTGS_OK;
    if (ctx->arena) {
        FHTGS_CK(cudaDeviceSynchronize());
        cudaFree(ctx->arena);
        ctx->arena = nullptr;
        ctx->arena_bytes = 0;
    }
    const size_t want = align_up(bytes + bytes / 8);
    cudaError_t e = cudaMalloc(&ctx->arena, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->arena = nullptr;
        return fail(FHTGS_ERR_OUT_OF_MEMORY, "arena allocation of " + std::to_string(want) + " bytes failed: " +
                                                 cudaGetErrorString(e));
    }
    ctx->arena_bytes = want;
    ++ctx->arena_generation;
    return FHTGS_OK;
}

fhtgs_status validate(const fhtgs_primitives* p, const fhtgs_view* views, int n_views, const fhtgs_settings* s) {
    if (!p || !views || !s) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (n_views <= 0 || n_views > 255) return fail(FHTGS_ERR_INVALID_ARGUMENT, "n_views must be in [1, 255]");
    if (p->n_primitives < 0) return fail(FHTGS_ERR_INVALID_ARGUMENT, "n_primitives must be >= 0");
    if (p->total_sh_bases < 0) return fail(FHTGS_ERR_INVALID_ARGUMENT, "total_sh_bases must be >= 0");
    if (p->storage != FHTGS_STORAGE_FP32 && p->storage != FHTGS_STORAGE_HALF)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown storage format");
    if (p->n_primitives > 0 && (!p->positions || !p->scales || !p->rotations || !p->opacities || !p->sh_0))
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "null Gaussian attribute pointer");
    if (s->active_sh_bases > 1 && s->active_sh_bases > p->total_sh_bases + 1)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "active_sh_bases exceeds 1 + sh_rest.size(1)");
    if (s->active_sh_bases > 1 && p->n_primitives > 0 && !p->sh_rest)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "sh_rest is null but higher SH bands are active");
    if (s->background_type < 0 || s->background_type > 3) return fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown background model");
    if (s->background_type != 0 && !s->background_data) return fail(FHTGS_ERR_INVALID_ARGUMENT, "background data is null");
    if ((s->background_type == 2 || s->background_type == 3) && (s->texture_width <= 0 || s->texture_height <= 0))
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "texture background needs positive texture size");
    if (s->foveation < FHTGS_FOVEATION_REFERENCE || s->foveation > FHTGS_FOVEATION_NONE)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown foveation mode");
    if (s->foveation == FHTGS_FOVEATION_RINGS) {
        if (!(s->ring_full >= 0.0f) || !(s->ring_half >= s->ring_full) || !std::isfinite(s->ring_half))
            return fail(FHTGS_ERR_INVALID_ARGUMENT, "ring radii must satisfy 0 <= ring_full <= ring_half < inf");
        if (s->blur_periphery) return fail(FHTGS_ERR_INVALID_ARGUMENT, "blur_periphery is not available with ring foveation");
    }
    for (int i = 0; i < n_views; ++i) {
        const fhtgs_view& v = views[i];
        if (v.width <= 0 || v.height <= 0) return fail(FHTGS_ERR_INVALID_ARGUMENT, "view size must be positive");
        if (static_cast<int64_t>(v.width) * v.height > (1ll << 28))
            return fail(FHTGS_ERR_INVALID_ARGUMENT, "view larger than 2^28 pixels");
        const int64_t gl = (static_cast<int64_t>(v.width) + 15) / 16 * ((static_cast<int64_t>(v.height) + 15) / 16);
        if (gl * kSubTiles + 1 >= (1ll << 31)) return fail(FHTGS_ERR_INVALID_ARGUMENT, "tile grid too large");
        if ((v.width + 15) / 16 > 65535 || (v.height + 15) / 16 > 65535)
            return fail(FHTGS_ERR_INVALID_ARGUMENT, "tile grid exceeds 16-bit bounds");
        if (!v.M || !v.VPM || !v.VPR_inv || !v.cam_position || !v.visibility_mask || !v.visibility_mask_area_table ||
            !v.fovea_mask_area_table || !v.image)
            return fail(FHTGS_ERR_INVALID_ARGUMENT, "null view pointer");
        if (v.foveation < 0 || v.foveation > FHTGS_FOVEATION_NONE + 1)
            return fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown per-view foveation");
        if (v.foveation == FHTGS_FOVEATION_RINGS + 1) {
            if (!(v.ring_full >= 0.0f) || !(v.ring_half >= v.ring_full) || !std::isfinite(v.ring_half))
                return fail(FHTGS_ERR_INVALID_ARGUMENT, "view ring radii must satisfy 0 <= ring_full <= ring_half < inf");
            if (s->blur_periphery) return fail(FHTGS_ERR_INVALID_ARGUMENT, "blur_periphery is not available with ring foveation");
        }
    }
    return FHTGS_OK;
}

int64_t estimate_capacity(int64_t n_prims) {
    int64_t c = std::max<int64_t>(int64_t(1) << 20, 12 * n_prims);
    return (c + kSortTile - 1) / kSortTile * kSortTile;
}

int sort_tiles_for(int64_t cap, int sort_items) {
    const int64_t tile = static_cast<int64_t>(kSortThreads) * sort_items;
    return static_cast<int>((cap + tile - 1) / tile);
}

// Grid sizes of every view of a frame and the arena carve-up it needs at instance capacity `cap`.
struct FramePlan {
    std::vector<ViewGeom> geo;
    int max_tiles = 0, max_large = 0, end_bit = 0, key_u32 = 0, nbp = 0, sort_tiles = 0;
    SplitPlan split;
    Layout L;
};

FramePlan frame_plan(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int V,
                     const fhtgs_settings* s, int64_t cap) {
    const int sort_items = ctx->tuning.sort_items;
    FramePlan P;
    const int64_t N = prims->n_primitives;
    P.geo.resize(V);
    for (int i = 0; i < V; ++i) {
        P.geo[i] = geometry(views[i]);
        P.max_tiles = std::max(P.max_tiles, P.geo[i].n_tiles);
        P.max_large = std::max(P.max_large, P.geo[i].n_large);
        P.end_bit = std::max(P.end_bit, P.geo[i].key_bits);
    }
    P.key_u32 = P.max_large > 65536 ? 1 : 0;
    P.nbp = static_cast<int>((N + kPrimBlock - 1) / kPrimBlock);
    P.sort_tiles = sort_tiles_for(cap, sort_items);
    std::vector<int64_t> temp_floats(V, 0);
    if (s->blur_periphery)
        for (int i = 0; i < V; ++i) temp_floats[i] = 3ll * views[i].width * views[i].height;
    P.split = split_plan(ctx->split_share, ctx->split_recs, ctx->split_exact, ctx->split_pool, s->K,
                         ctx->tuning.blend_blocks_per_sm, ctx->n_sms, V, P.max_large);
    P.L = plan(V, N, P.nbp, cap, P.key_u32 ? 4 : 2, P.sort_tiles, P.max_tiles, P.max_large, temp_floats, P.split);
    return P;
}

// Enqueues one frame on `stream` (no host synchronisation).  `gaze_dev` (null or [n_views][2]
// floats in device memory) replaces the views' host gaze values at run time.
fhtgs_status render_impl(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int n_views,
                         const fhtgs_settings* s, cudaStream_t stream, const float* gaze_dev = nullptr) {
    fhtgs_status st = validate(prims, views, n_views, s);
    if (st != FHTGS_OK) return st;
    FHTGS_CK(cudaSetDevice(ctx->device));
    const int V = n_views;
    const int64_t N = prims->n_primitives;
    if (ctx->cap <= 0) ctx->cap = estimate_capacity(N);
    const int64_t cap = ctx->cap;
    FramePlan P = frame_plan(ctx, prims, views, V, s, cap);
    const std::vector<ViewGeom>& geo = P.geo;
    const int max_tiles = P.max_tiles, max_large = P.max_large, end_bit = P.end_bit, key_u32 = P.key_u32;
    const int nbp = P.nbp, sort_tiles = P.sort_tiles;
    const Layout& L = P.L;
    st = ensure_arena(ctx, L.total);
    if (st != FHTGS_OK) return st;
    char* A = ctx->arena;

    FrameParams fp{};
    fp.n_views = V;
    fp.n_prims = static_cast<int>(N);
    fp.total_sh = prims->total_sh_bases;
    fp.active_sh = s->active_sh_bases;
    fp.K = s->K;
    fp.near_plane = s->near_plane;
    fp.far_plane = s->far_plane;
    fp.scale_modifier = s->scale_modifier;
    fp.to_chw = s->to_chw ? 1 : 0;
    fp.blur = s->blur_periphery ? 1 : 0;
    fp.aaa = s->anti_aliasing ? 1 : 0;
    fp.bg_type = s->background_type;
    fp.bg_data = s->background_data;
    fp.tex_w = s->texture_width;
    fp.tex_h = s->texture_height;
    fp.key_u32 = key_u32;
    fp.end_bit = end_bit;
    fp.cap = cap;
    fp.max_tiles = max_tiles;
    fp.max_large = max_large;
    fp.n_blocks_prim = nbp;
    fp.blend_rw = ctx->tuning.blend_warp_width;
    fp.blend_blocks = ctx->tuning.blend_blocks_per_sm;
    fp.look_spin_limit = kLookSpinLimit;
    fp.stage_wait_limit = kStageWaitLimit;
    fp.look_first_ticket = 0;
    if (ctx->wait_test == FHTGS_WAIT_TEST_SORT_LOOKBACK) {
        fp.look_spin_limit = ctx->wait_test_limit;
        fp.look_first_ticket = 1;
    } else if (ctx->wait_test == FHTGS_WAIT_TEST_STAGING) {
        fp.stage_wait_limit = ctx->wait_test_limit;
    }
    ctx->wait_test = 0;  // one frame only

    FrameBuffers fb{};
    fb.views = reinterpret_cast<ViewParams*>(A + L.off_views);
    fb.status = reinterpret_cast<FrameStatus*>(A + L.off_status);
    fb.n_touched = reinterpret_cast<uint32_t*>(A + L.off_nt);
    fb.n_vis = reinterpret_cast<uint32_t*>(A + L.off_nvis);
    fb.bounds = reinterpret_cast<ushort4*>(A + L.off_bounds);
    fb.rec = reinterpret_cast<float4*>(A + L.off_rec);
    fb.block_sums = reinterpret_cast<uint32_t*>(A + L.off_bsums);
    fb.keys[0] = A + L.off_keys0;
    fb.keys[1] = A + L.off_keys1;
    fb.vals[0] = reinterpret_cast<uint32_t*>(A + L.off_vals0);
    fb.vals[1] = reinterpret_cast<uint32_t*>(A + L.off_vals1);
    fb.final_buf = 0;
    fb.sort_hist = reinterpret_cast<uint32_t*>(A + L.off_hist);
    fb.sort_digit_tot = reinterpret_cast<uint32_t*>(A + L.off_dtot);
    fb.sort_tiles = N > 0 ? sort_tiles : 0;
    fb.sort_items = ctx->tuning.sort_items;
    fb.ranges = reinterpret_cast<uint2*>(A + L.off_ranges);
    fb.tile_map_part = reinterpret_cast<uint32_t*>(A + L.off_map);
    fb.tile_type_part = reinterpret_cast<uint8_t*>(A + L.off_type);
    fb.large_type = reinterpret_cast<uint8_t*>(A + L.off_ltype);
    fb.work_full = reinterpret_cast<uint32_t*>(A + L.off_wf);
    fb.work_low = reinterpret_cast<uint32_t*>(A + L.off_wl);
    fb.work_masked = reinterpret_cast<uint32_t*>(A + L.off_wm);
    fb.counters = reinterpret_cast<uint32_t*>(A + L.off_ctr);
    fb.work_order[0] = reinterpret_cast<uint32_t*>(A + L.off_order0);
    fb.work_order[1] = reinterpret_cast<uint32_t*>(A + L.off_order1);
    if (cap < kOnesweepMaxCap) {  // onesweep sort (look-back counts are 30-bit)
        fb.sort_ghist = reinterpret_cast<uint32_t*>(A + L.off_ghist);
        fb.sort_look = reinterpret_cast<uint32_t*>(A + L.off_look);
        fb.sort_ticket = reinterpret_cast<uint32_t*>(A + L.off_ticket);
    }
    SplitArgs sa{};
    if (P.split.cap > 0) {
        sa.share = P.split.share;
        sa.blocks = P.split.blocks;
        sa.cap = P.split.cap;
        sa.recs = P.split.recs;
        sa.stride = P.split.stride;
        sa.of = reinterpret_cast<uint32_t*>(A + L.off_split_of);
        sa.list = reinterpret_cast<uint2*>(A + L.off_split_list);
        sa.ctl = reinterpret_cast<uint32_t*>(A + L.off_split_ctl);
        sa.scratch = A + L.off_split_scratch;
        sa.status = reinterpret_cast<FrameStatus*>(A + L.off_split_status);
        sa.exact = P.split.exact;
        sa.pool_units = P.split.pool_units;
        sa.seg_unit = reinterpret_cast<uint32_t*>(A + L.off_split_units);
        sa.pool = A + L.off_split_pool;
    }

    std::vector<ViewSetup> setups(V);
    for (int i = 0; i < V; ++i) {
        const fhtgs_view& v = views[i];
        const ViewGeom& g = geo[i];
        ViewSetup& su = setups[i];
        su.M = v.M;
        su.VPM = v.VPM;
        su.VPR_inv = v.VPR_inv;
        su.cam = v.cam_position;
        su.gaze = gaze_dev ? gaze_dev + 2 * i : nullptr;
        ViewParams& p = su.p;
        std::memset(&p, 0, sizeof(p));
        p.gaze_px = make_float2(g.gaze_px, g.gaze_py);
        p.gaze_tiles = make_float2(static_cast<float>(g.gaze_tx), static_cast<float>(g.gaze_ty));
        p.gaze_tiles_i = make_int2(g.gaze_tx, g.gaze_ty);
        p.width = v.width;
        p.height = v.height;
        p.focal_x = v.focal_x;
        p.focal_y = v.focal_y;
        p.center_x = v.center_x;
        p.center_y = v.center_y;
        p.glw = g.glw;
        p.glh = g.glh;
        p.n_large = g.n_large;
        p.n_tiles = g.n_tiles;
        p.vis_mask = v.visibility_mask;
        p.vis_sat = v.visibility_mask_area_table;
        p.fovea_sat = v.fovea_mask_area_table;
        p.image = v.image;
        p.work = s->blur_periphery ? reinterpret_cast<float*>(A + L.temp_offsets[i]) : v.image;
        // foveation: the view's own when it sets one, else the frame's
        const bool own = v.foveation > 0;
        const float rf = own ? v.ring_full : s->ring_full, rh = own ? v.ring_half : s->ring_half;
        p.fov_mode = own ? v.foveation - 1 : s->foveation;
        p.ring_full2 = rf * rf;
        p.ring_half2 = rh * rh;
    }
    Gaussians gs{prims->positions, prims->scales, prims->rotations, prims->opacities, prims->sh_0, prims->sh_rest,
                 prims->storage == FHTGS_STORAGE_HALF ? 1 : 0};
    const KernelSet& ks = s->fast_math ? kernels_fast() : kernels_ieee();

    const bool prof = ctx->profile && !ctx->capturing;
    cudaEvent_t* ev = ctx->ev[ctx->frames_profiled % kStageRing];
    // NVTX: the frame's range and the current stage's, closed on every exit path
    struct Ranges {
        int open = 0;
        Ranges() { nvtx_push("frame"); open = 1; }
        void stage(int i) {
            if (open > 1) { nvtx_pop(); --open; }
            if (i < FHTGS_N_STAGES) { nvtx_push(kStageNames[i]); ++open; }
        }
        ~Ranges() { while (open-- > 0) nvtx_pop(); }
    } ranges;
    // stage boundary i: profiling event; the range of stage i - 1 ends and that of stage i starts
    auto mark = [&](int i) {
        if (prof) cudaEventRecord(ev[i], stream);
        ranges.stage(i);
    };
    long long n = 0;
    mark(0);
    FHTGS_CK(cudaMemsetAsync(fb.counters, 0, 4ull * kCounterWords, stream));
    // the per-view status words start at zero (counts, error bits): the preprocess and the
    // classification write into them concurrently
    FHTGS_CK(cudaMemsetAsync(fb.status, 0, sizeof(FrameStatus) * V, stream));
    n += ks.setup(setups.data(), V, fb.views, stream);
    mark(1);
    // tile classification (one block per view, latency-bound) beside the preprocess: nothing
    // reads its outputs before the range and work-order stage, where the side stream joins
    FHTGS_CK(cudaEventRecord(ctx->fork_ev, stream));
    FHTGS_CK(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
    n += ks.classify(fp, fb, ctx->side);
    FHTGS_CK(cudaEventRecord(ctx->join_ev, ctx->side));
    n += ks.preprocess(fp, fb, gs, stream);
    mark(2);
    if (nbp > 0) {
        n += ks.scan_blocks(fp, fb, stream);
        n += ks.create_instances(fp, fb, stream);
    }
    mark(3);
    n += ks.sort(fp, fb, stream);
    mark(4);
    FHTGS_CK(cudaStreamWaitEvent(stream, ctx->join_ev, 0));
    n += ks.ranges(fp, fb, ctx->n_sms, stream);
    n += ks.order(fp, fb, sa, ctx->n_sms, stream);
    mark(5);
    n += ks.blend(fp, fb, sa, ctx->n_sms, stream, nullptr);
    mark(6);
    n += ks.compose(fp, fb, stream);
    mark(7);
    FHTGS_CK(cudaGetLastError());
    ctx->launches += n;
    if (prof) ++ctx->frames_profiled;

    ctx->have_frame = true;
    ctx->fp = fp;
    ctx->fb = fb;
    ctx->split_active = sa.cap > 0;
    ctx->geo = geo;
    ctx->views.assign(views, views + V);
    ctx->frame_foveation = s->foveation;
    ctx->stream = stream;
    return FHTGS_OK;
}

// Foveation mode a view of the last frame was rendered with.
int view_mode(fhtgs_context ctx, int view) {
    const fhtgs_view& v = ctx->views[view];
    return v.foveation > 0 ? v.foveation - 1 : ctx->frame_foveation;
}

fhtgs_status read_status(fhtgs_context ctx) {
    const int V = ctx->fp.n_views;
    if (ctx->h_status_n < V) {
        if (ctx->h_status) cudaFreeHost(ctx->h_status);
        ctx->h_status = nullptr;
        FHTGS_CK(cudaMallocHost(&ctx->h_status, sizeof(FrameStatus) * V));
        ctx->h_status_n = V;
    }
    FHTGS_CK(cudaMemcpyAsync(ctx->h_status, ctx->fb.status, sizeof(FrameStatus) * V, cudaMemcpyDeviceToHost, ctx->stream));
    FHTGS_CK(cudaStreamSynchronize(ctx->stream));
    return FHTGS_OK;
}

fhtgs_status render_sync_impl(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int n_views,
                              const fhtgs_settings* s, cudaStream_t stream) {
    for (int attempt = 0; attempt < 4; ++attempt) {
        fhtgs_status st = render_impl(ctx, prims, views, n_views, s, stream);
        if (st != FHTGS_OK) return st;
        st = read_status(ctx);
        if (st != FHTGS_OK) return st;
        unsigned long long need = 0;
        bool overflow = false;
        for (int i = 0; i < n_views; ++i) {
            need = std::max(need, ctx->h_status[i].n_instances);
            overflow = overflow || ctx->h_status[i].n_instances > static_cast<unsigned long long>(ctx->cap);
            if (ctx->h_status[i].overflow & kFrameErrSortLookback)
                return fail(FHTGS_ERR_CUDA, "instance sort: a look-back wait gave up (view " + std::to_string(i) + ")");
            if (ctx->h_status[i].overflow & kFrameErrStaging)
                return fail(FHTGS_ERR_CUDA, "preprocess: attribute staging did not complete (view " + std::to_string(i) + ")");
        }
        if (!overflow) return FHTGS_OK;
        int64_t grown = static_cast<int64_t>(need + need / 4 + kSortTile);
        ctx->cap = (grown + kSortTile - 1) / kSortTile * kSortTile;
    }
    return fail(FHTGS_ERR_CAPACITY, "instance capacity still insufficient after regrowth");
}

}  // namespace

// Internal interface used by the request server (fhtgs_server.cu), declared in fhtgs_internal.h.
namespace fhtgs {

fhtgs_status enqueue_frame(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int n_views,
                           const fhtgs_settings* s, cudaStream_t stream, FrameStatus* host_status) {
    fhtgs_status st = render_impl(ctx, prims, views, n_views, s, stream);
    if (st != FHTGS_OK || !host_status) return st;
    FHTGS_CK(cudaMemcpyAsync(host_status, ctx->fb.status, sizeof(FrameStatus) * n_views, cudaMemcpyDeviceToHost, stream));
    return FHTGS_OK;
}

size_t frame_arena_need(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int n_views,
                        const fhtgs_settings* s, int64_t cap) {
    const size_t total = frame_plan(ctx, prims, views, n_views, s, cap).L.total;
    if (total <= ctx->arena_bytes) return ctx->arena_bytes;
    return align_up(total + total / 8);  // what ensure_arena allocates
}

int64_t default_instance_capacity(int64_t n_prims) { return estimate_capacity(n_prims); }

int64_t context_capacity(fhtgs_context ctx) { return ctx->cap; }

void set_context_capacity(fhtgs_context ctx, int64_t cap) {
    ctx->cap = (std::max<int64_t>(cap, 1) + kSortTile - 1) / kSortTile * kSortTile;
}

fhtgs_status release_arena(fhtgs_context ctx) {
    if (!ctx->arena) return FHTGS_OK;
    FHTGS_CK(cudaSetDevice(ctx->device));
    FHTGS_CK(cudaFree(ctx->arena));
    ctx->arena = nullptr;
    ctx->arena_bytes = 0;
    ++ctx->arena_generation;
    ctx->have_frame = false;
    return FHTGS_OK;
}

fhtgs_status validate_frame(const fhtgs_primitives* p, const fhtgs_view* views, int n_views, const fhtgs_settings* s) {
    return validate(p, views, n_views, s);
}

}  // namespace fhtgs

extern "C" {

int32_t fhtgs_abi_version(void) { return FHTGS_ABI_VERSION; }
const char* fhtgs_last_error(void) { return g_error.c_str(); }

fhtgs_status fhtgs_context_create(int32_t device, fhtgs_context* out) {
    if (!out) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    int n = 0;
    FHTGS_CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(FHTGS_ERR_INVALID_ARGUMENT, "no such CUDA device");
    FHTGS_CK(cudaSetDevice(device));
    auto* c = new fhtgs_context_s();
    c->device = device;
    cudaDeviceGetAttribute(&c->n_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        fhtgs_context_destroy(c);
        return fail(FHTGS_ERR_CUDA, "context stream/events");
    }
    *out = c;
    return FHTGS_OK;
}

fhtgs_status fhtgs_context_destroy(fhtgs_context ctx) {
    if (!ctx) return FHTGS_OK;
    cudaSetDevice(ctx->device);
    for (auto& set : ctx->ev)
        for (auto& e : set)
            if (e) cudaEventDestroy(e);
    if (ctx->arena) {
        cudaDeviceSynchronize();
        cudaFree(ctx->arena);
    }
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->side) {
        cudaStreamSynchronize(ctx->side);
        cudaStreamDestroy(ctx->side);
    }
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
    delete ctx;
    return FHTGS_OK;
}

fhtgs_status fhtgs_context_reserve(fhtgs_context ctx, int32_t n_primitives, int32_t n_views, int32_t max_width,
                                   int32_t max_height, int64_t instances_per_view) {
    if (!ctx || n_primitives < 0 || n_views <= 0 || max_width <= 0 || max_height <= 0)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "invalid reserve request");
    FHTGS_CK(cudaSetDevice(ctx->device));
    int64_t cap = instances_per_view > 0 ? instances_per_view : estimate_capacity(n_primitives);
    cap = (cap + kSortTile - 1) / kSortTile * kSortTile;
    ctx->cap = std::max(ctx->cap, cap);
    const int glw = (max_width + 15) / 16, glh = (max_height + 15) / 16;
    const int n_large = glw * glh, n_tiles = 4 * n_large;
    const int nbp = (n_primitives + kPrimBlock - 1) / kPrimBlock;
    std::vector<int64_t> temp(n_views, 3ll * max_width * max_height);
    Layout L = plan(n_views, n_primitives, nbp, ctx->cap, end_bit_of(n_tiles + 1) > 16 ? 4 : 2,
                    sort_tiles_for(ctx->cap, kSortItemsMin), n_tiles, n_large, temp,
                    split_plan(ctx->split_share, ctx->split_recs, ctx->split_exact, ctx->split_pool, 32,
                               ctx->tuning.blend_blocks_per_sm, ctx->n_sms, n_views, n_large));
    return ensure_arena(ctx, L.total);
}

size_t fhtgs_context_arena_bytes(fhtgs_context ctx) { return ctx ? ctx->arena_bytes : 0; }

fhtgs_status fhtgs_context_set_profiling(fhtgs_context ctx, int32_t enable) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null context");
    FHTGS_CK(cudaSetDevice(ctx->device));
    if (enable && !ctx->ev[0][0])
        for (auto& set : ctx->ev)
            for (auto& e : set) FHTGS_CK(cudaEventCreate(&e));
    ctx->profile = enable != 0;
    return FHTGS_OK;
}

fhtgs_status fhtgs_context_test_wait_timeout(fhtgs_context ctx, int32_t which, int32_t limit) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null context");
    if (which != FHTGS_WAIT_TEST_SORT_LOOKBACK && which != FHTGS_WAIT_TEST_STAGING)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "which must be FHTGS_WAIT_TEST_SORT_LOOKBACK or FHTGS_WAIT_TEST_STAGING");
    const int max_limit = which == FHTGS_WAIT_TEST_SORT_LOOKBACK ? kLookSpinLimit : kStageWaitLimit;
    if (limit < 0 || limit > max_limit)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "limit must be in [0, " + std::to_string(max_limit) + "]");
    ctx->wait_test = which;
    ctx->wait_test_limit = limit;
    return FHTGS_OK;
}

fhtgs_status fhtgs_get_stage_times(fhtgs_context ctx, float* ms, int32_t n) {
    if (!ctx || !ms || n < FHTGS_N_STAGES) return fail(FHTGS_ERR_INVALID_ARGUMENT, "need a buffer of FHTGS_N_STAGES floats");
    if (!ctx->profile || ctx->frames_profiled == 0) return fail(FHTGS_ERR_NOT_READY, "profiling off or no frame rendered");
    cudaEvent_t* ev = ctx->ev[(ctx->frames_profiled - 1) % kStageRing];
    FHTGS_CK(cudaEventSynchronize(ev[kStageEvents - 1]));
    for (int i = 0; i < FHTGS_N_STAGES; ++i) FHTGS_CK(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
    return FHTGS_OK;
}

fhtgs_status fhtgs_get_stage_history(fhtgs_context ctx, float* ms, int32_t max_frames, int32_t* n_frames) {
    if (!ctx || !ms || !n_frames || max_frames <= 0) return fail(FHTGS_ERR_INVALID_ARGUMENT, "bad history request");
    if (!ctx->profile || ctx->frames_profiled == 0) return fail(FHTGS_ERR_NOT_READY, "profiling off or no frame rendered");
    const long long have = std::min<long long>(ctx->frames_profiled, kStageRing);
    const int n = static_cast<int>(std::min<long long>(have, max_frames));
    for (int f = 0; f < n; ++f) {
        cudaEvent_t* ev = ctx->ev[(ctx->frames_profiled - n + f) % kStageRing];
        FHTGS_CK(cudaEventSynchronize(ev[kStageEvents - 1]));
        for (int i = 0; i < FHTGS_N_STAGES; ++i)
            FHTGS_CK(cudaEventElapsedTime(&ms[f * FHTGS_N_STAGES + i], ev[i], ev[i + 1]));
    }
    *n_frames = n;
    return FHTGS_OK;
}

int64_t fhtgs_context_launch_count(fhtgs_context ctx) { return ctx ? ctx->launches : 0; }

fhtgs_status fhtgs_render_views(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views,
                                int32_t n_views, const fhtgs_settings* settings, void* stream) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null context");
    return render_impl(ctx, prims, views, n_views, settings, static_cast<cudaStream_t>(stream));
}

fhtgs_status fhtgs_render_views_sync(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views,
                                     int32_t n_views, const fhtgs_settings* settings, void* stream) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null context");
    return render_sync_impl(ctx, prims, views, n_views, settings, static_cast<cudaStream_t>(stream));
}

fhtgs_status fhtgs_get_frame_info(fhtgs_context ctx, int32_t view, fhtgs_frame_info* out) {
    if (!ctx || !out) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (!ctx->have_frame) return fail(FHTGS_ERR_NOT_READY, "no frame rendered yet");
    if (view < 0 || view >= ctx->fp.n_views) return fail(FHTGS_ERR_INVALID_ARGUMENT, "view index out of range");
    fhtgs_status st = read_status(ctx);
    if (st != FHTGS_OK) return st;
    const FrameStatus& s = ctx->h_status[view];
    if (s.overflow & kFrameErrWait)
        return fail(FHTGS_ERR_CUDA, std::string("the frame is incomplete: a bounded device wait gave up (") +
                                        ((s.overflow & kFrameErrSortLookback) ? "instance sort look-back" : "") +
                                        ((s.overflow & kFrameErrSortLookback) && (s.overflow & kFrameErrStaging) ? ", " : "") +
                                        ((s.overflow & kFrameErrStaging) ? "preprocess attribute staging" : "") +
                                        "); the view rendered background only");
    // the reference's count has a meaning only in its own foveation layout
    out->n_instances = static_cast<int64_t>(view_mode(ctx, view) == kFoveationReference ? s.n_instances_ref : s.n_instances);
    out->instance_capacity = ctx->fp.cap;
    out->n_active_tiles = s.n_active;
    for (int k = 0; k < 6; ++k) out->partition_ranges[k] = s.ranges[k];
    out->overflow = s.n_instances > static_cast<unsigned long long>(ctx->fp.cap) ? 1 : 0;
    out->end_bit = ctx->geo[view].end_bit;
    out->n_instances_stored = static_cast<int64_t>(s.n_instances);
    return FHTGS_OK;
}

fhtgs_status fhtgs_copy_intermediates(fhtgs_context ctx, int32_t view, fhtgs_intermediates* out) {
    if (!ctx || !out) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (!ctx->have_frame) return fail(FHTGS_ERR_NOT_READY, "no frame rendered yet");
    if (view < 0 || view >= ctx->fp.n_views) return fail(FHTGS_ERR_INVALID_ARGUMENT, "view index out of range");
    fhtgs_status st = read_status(ctx);
    if (st != FHTGS_OK) return st;
    const FrameParams& fp = ctx->fp;
    const FrameBuffers& fb = ctx->fb;
    const FrameStatus& s = ctx->h_status[view];
    const size_t N = static_cast<size_t>(fp.n_prims);
    const size_t vo = static_cast<size_t>(view) * N;
    if (out->n_touched && N) FHTGS_CK(cudaMemcpy(out->n_touched, fb.n_touched + vo, 4 * N, cudaMemcpyDeviceToHost));
    if (out->screen_bounds && N) FHTGS_CK(cudaMemcpy(out->screen_bounds, fb.bounds + vo, 8 * N, cudaMemcpyDeviceToHost));
    if ((out->vpmt || out->rgba) && N) {
        std::vector<float4> rec(4 * N);
        FHTGS_CK(cudaMemcpy(rec.data(), fb.rec + 4 * vo, 64 * N, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < N; ++i) {
            if (out->vpmt) std::memcpy(out->vpmt + 12 * i, &rec[4 * i], 48);
            if (out->rgba) std::memcpy(out->rgba + 4 * i, &rec[4 * i + 3], 16);
        }
    }
    const size_t T = static_cast<size_t>(ctx->geo[view].n_tiles);
    const size_t na = s.n_active;
    if (out->tile_index_map_partitioned && na)
        FHTGS_CK(cudaMemcpy(out->tile_index_map_partitioned, fb.tile_map_part + static_cast<size_t>(view) * fp.max_tiles,
                            4 * na, cudaMemcpyDeviceToHost));
    if (out->tile_type_partitioned && na)
        FHTGS_CK(cudaMemcpy(out->tile_type_partitioned, fb.tile_type_part + static_cast<size_t>(view) * fp.max_tiles, na,
                            cudaMemcpyDeviceToHost));
    // Stored instances: one per (primitive, visible large tile), sorted by large tile.
    const ViewGeom& g = ctx->geo[view];
    const size_t Ms = static_cast<size_t>(std::min<unsigned long long>(s.n_instances, static_cast<unsigned long long>(fp.cap)));
    std::vector<uint32_t> vals(Ms);
    std::vector<uint2> lr(static_cast<size_t>(g.n_large));
    if (Ms) FHTGS_CK(cudaMemcpy(vals.data(), fb.vals[fb.final_buf] + static_cast<size_t>(view) * fp.cap, 4 * Ms,
                                cudaMemcpyDeviceToHost));
    FHTGS_CK(cudaMemcpy(lr.data(), fb.ranges + static_cast<size_t>(view) * fp.max_large, 8 * lr.size(),
                        cudaMemcpyDeviceToHost));
    std::vector<uint8_t> lt(static_cast<size_t>(g.n_large));
    FHTGS_CK(cudaMemcpy(lt.data(), fb.large_type + static_cast<size_t>(view) * fp.max_large, lt.size(),
                        cudaMemcpyDeviceToHost));
    // The reference's arrays (create_instances_cu + SortPairs + extract_instance_ranges_cu):
    // keys are small-tile ids 4*t+i, the list of a fovea-circle tile (type fovea or blended) is
    // repeated for its four sub-tiles, other visible tiles carry key 4*t once; the slots its
    // area tables over-count follow as sentinel keys, up to its instance count.
    // Other foveation modes have no reference layout: each stored list appears once, keyed by
    // its large tile's first sub-tile, without sentinel slots.
    const bool ref_layout = view_mode(ctx, view) == kFoveationReference;
    const uint64_t m_ref = ref_layout ? s.n_instances_ref : Ms;
    const uint32_t sentinel = g.end_bit <= 16 ? 0xFFFFu : 0xFFFFFFFFu;
    uint64_t pos = 0;
    std::vector<uint2> rr(T, make_uint2(0, 0));
    for (int t = 0; t < g.n_large; ++t) {
        const uint2 r = lr[t];
        if (r.y <= r.x) continue;
        const uint32_t len = r.y - r.x;
        const int reps = ref_layout && (lt[t] == kFovea || lt[t] == kBlended) ? kSubTiles : 1;
        for (int i = 0; i < reps; ++i) {
            const uint32_t key = static_cast<uint32_t>(t) * kSubTiles + i;
            if (pos + len > m_ref) return fail(FHTGS_ERR_CAPACITY, "stored instances exceed the reference count");
            for (uint32_t j = 0; j < len; ++j) {
                if (out->keys) out->keys[pos + j] = key;
                if (out->values) out->values[pos + j] = vals[r.x + j];
            }
            rr[key] = make_uint2(static_cast<uint32_t>(pos), static_cast<uint32_t>(pos + len));
            pos += len;
        }
    }
    for (; pos < m_ref; ++pos) {
        if (out->keys) out->keys[pos] = sentinel;
        if (out->values) out->values[pos] = 0xFFFFFFFFu;
    }
    if (out->instance_ranges && T) std::memcpy(out->instance_ranges, rr.data(), 8 * T);
    return FHTGS_OK;
}

// ---- tuning, autotuner, frame graphs ----------------------------------------------------

fhtgs_status fhtgs_context_set_tuning(fhtgs_context ctx, const fhtgs_tuning* t) {
    if (!ctx || !t) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (t->blend_warp_width != 4 && t->blend_warp_width != 8 && t->blend_warp_width != 16)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "blend_warp_width must be 4, 8 or 16");
    if (t->blend_blocks_per_sm < 0 || t->blend_blocks_per_sm > 8)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "blend_blocks_per_sm must be in [0, 8]");
    if (t->sort_items != 8 && t->sort_items != 12 && t->sort_items != 16)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "sort_items must be 8, 12 or 16");
    ctx->tuning = *t;
    return FHTGS_OK;
}

fhtgs_status fhtgs_context_set_blend_split(fhtgs_context ctx, float segment_share, int32_t records) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (!(segment_share == 0.0f || (segment_share >= 0.05f && segment_share <= 8.0f)))
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "segment_share must be 0 (off) or in [0.05, 8]");
    if (records < 0 || records > 256) return fail(FHTGS_ERR_INVALID_ARGUMENT, "records must be in [0, 256]");
    ctx->split_share = segment_share;
    ctx->split_recs = records;
    return FHTGS_OK;
}

fhtgs_status fhtgs_context_set_blend_split_exact(fhtgs_context ctx, int32_t exact, int64_t log_bytes) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (exact != 0 && exact != 1) return fail(FHTGS_ERR_INVALID_ARGUMENT, "exact must be 0 or 1");
    if (log_bytes != 0 && (log_bytes < (int64_t(1) << 20) || log_bytes > (int64_t(64) << 30)))
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "log_bytes must be 0 (8 GiB) or in [1 MiB, 64 GiB]");
    ctx->split_exact = exact;
    ctx->split_pool = log_bytes;
    return FHTGS_OK;
}

fhtgs_status fhtgs_context_get_blend_split_stats(fhtgs_context ctx, int32_t* split_tiles, int32_t* segments,
                                                 int32_t* whole_fallbacks, int32_t* max_records) {
    if (!ctx || !split_tiles || !segments || !whole_fallbacks || !max_records)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (!ctx->have_frame) return fail(FHTGS_ERR_NOT_READY, "no frame rendered yet");
    *split_tiles = *segments = *whole_fallbacks = *max_records = 0;
    if (!ctx->split_active) return FHTGS_OK;
    FHTGS_CK(cudaSetDevice(ctx->device));
    uint32_t c[kCtrHist];
    FHTGS_CK(cudaMemcpyAsync(c, ctx->fb.counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    FHTGS_CK(cudaStreamSynchronize(ctx->stream));
    *split_tiles = static_cast<int32_t>(c[kCtrSplitTiles]);
    *segments = static_cast<int32_t>(c[kCtrSplitSegs]);
    *whole_fallbacks = static_cast<int32_t>(c[kCtrSplitFallback]);
    *max_records = static_cast<int32_t>(c[kCtrSplitRecMax]);
    return FHTGS_OK;
}

fhtgs_status fhtgs_context_get_tuning(fhtgs_context ctx, fhtgs_tuning* t) {
    if (!ctx || !t) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    *t = ctx->tuning;
    return FHTGS_OK;
}

namespace {

float median_of(std::vector<float> v) {
    if (v.empty()) return 0.0f;
    std::sort(v.begin(), v.end());
    const size_t n = v.size();
    return n % 2 ? v[n / 2] : 0.5f * (v[n / 2 - 1] + v[n / 2]);
}

// Renders `repeats` frames with tuning `t` after one warm-up frame; medians of one stage's time
// and of the whole frame (CUDA events between the stages).
fhtgs_status time_candidate(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int n_views,
                            const fhtgs_settings* s, cudaStream_t stream, const fhtgs_tuning& t, int repeats, int stage,
                            float* stage_ms, float* frame_ms) {
    ctx->tuning = t;
    for (int r = 0; r <= repeats; ++r) {
        fhtgs_status st = render_impl(ctx, prims, views, n_views, s, stream);
        if (st != FHTGS_OK) return st;
    }
    FHTGS_CK(cudaStreamSynchronize(stream));
    std::vector<float> st_ms, fr_ms;
    for (int f = 0; f < repeats; ++f) {
        cudaEvent_t* ev = ctx->ev[(ctx->frames_profiled - repeats + f) % kStageRing];
        float a = 0.0f, b = 0.0f;
        FHTGS_CK(cudaEventElapsedTime(&a, ev[stage], ev[stage + 1]));
        FHTGS_CK(cudaEventElapsedTime(&b, ev[0], ev[kStageEvents - 1]));
        st_ms.push_back(a);
        fr_ms.push_back(b);
    }
    *stage_ms = median_of(st_ms);
    *frame_ms = median_of(fr_ms);
    return FHTGS_OK;
}

}  // namespace

fhtgs_status fhtgs_autotune(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int32_t n_views,
                            const fhtgs_settings* settings, int32_t repeats, fhtgs_tuning* best, float* best_frame_ms,
                            void* stream_) {
    if (!ctx || !best) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (repeats < 1 || repeats > 32) return fail(FHTGS_ERR_INVALID_ARGUMENT, "repeats must be in [1, 32]");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const bool was_profiling = ctx->profile;
    fhtgs_status st = fhtgs_context_set_profiling(ctx, 1);
    if (st != FHTGS_OK) return st;
    const fhtgs_tuning start = ctx->tuning;
    auto finish = [&](fhtgs_status r) {
        ctx->profile = was_profiling;
        if (r != FHTGS_OK) ctx->tuning = start;
        return r;
    };
    st = render_sync_impl(ctx, prims, views, n_views, settings, stream);  // sizes the capacity
    if (st != FHTGS_OK) return finish(st);
    constexpr int kStageSort = 3, kStageBlend = 5;
    fhtgs_tuning cur = start;
    float best_stage = 3.4e38f, frame = 0.0f, stage = 0.0f;
    // blend: warp rectangle x persistent blocks per SM
    fhtgs_tuning win = cur;
    for (int w : kBlendRowChoices) {
        for (int b : {0, 3, 2}) {
            fhtgs_tuning t = cur;
            t.blend_warp_width = w;
            t.blend_blocks_per_sm = b;
            st = time_candidate(ctx, prims, views, n_views, settings, stream, t, repeats, kStageBlend, &stage, &frame);
            if (st != FHTGS_OK) return finish(st);
            if (stage < best_stage) { best_stage = stage; win = t; }
        }
    }
    cur = win;
    // sort: keys per thread of a tile
    best_stage = 3.4e38f;
    for (int items : {16, 12, 8}) {
        fhtgs_tuning t = cur;
        t.sort_items = items;
        st = time_candidate(ctx, prims, views, n_views, settings, stream, t, repeats, kStageSort, &stage, &frame);
        if (st != FHTGS_OK) return finish(st);
        if (stage < best_stage) { best_stage = stage; win = t; }
    }
    cur = win;
    st = time_candidate(ctx, prims, views, n_views, settings, stream, cur, repeats, kStageBlend, &stage, &frame);
    if (st != FHTGS_OK) return finish(st);
    ctx->tuning = cur;
    *best = cur;
    if (best_frame_ms) *best_frame_ms = frame;
    return finish(FHTGS_OK);
}

struct fhtgs_frame_graph_s {
    fhtgs_context ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long generation = 0;
    long long launches_per_frame = 0;
    FrameParams fp{};
    FrameBuffers fb{};
    std::vector<ViewGeom> geo;
    std::vector<fhtgs_view> views;
    int frame_foveation = 0;
    bool split_active = false;
};

fhtgs_status fhtgs_frame_graph_create(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views,
                                      int32_t n_views, const fhtgs_settings* settings, const float* gaze_device,
                                      float capacity_headroom, fhtgs_frame_graph* out, void* stream_) {
    if (!ctx || !out) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (!(capacity_headroom >= 1.0f) || capacity_headroom > 16.0f)
        return fail(FHTGS_ERR_INVALID_ARGUMENT, "capacity_headroom must be in [1, 16]");
    fhtgs_status st = validate(prims, views, n_views, settings);
    if (st != FHTGS_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    // 1) an eager frame measures the instance counts; the capacity gets the headroom
    st = render_sync_impl(ctx, prims, views, n_views, settings, stream);
    if (st != FHTGS_OK) return st;
    unsigned long long need = 0;
    for (int i = 0; i < n_views; ++i) need = std::max(need, ctx->h_status[i].n_instances);
    const int64_t want = static_cast<int64_t>(static_cast<double>(need) * capacity_headroom) + kSortTile;
    if (want > ctx->cap) ctx->cap = (want + kSortTile - 1) / kSortTile * kSortTile;
    // 2) a frame at the final capacity places the arena (nothing may allocate while capturing)
    st = render_impl(ctx, prims, views, n_views, settings, stream, gaze_device);
    if (st != FHTGS_OK) return st;
    FHTGS_CK(cudaStreamSynchronize(stream));
    // 3) capture the same frame on a private stream
    cudaStream_t cs = nullptr;
    FHTGS_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    const long long launches0 = ctx->launches;
    const long long generation = ctx->arena_generation;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        ctx->capturing = true;
        st = render_impl(ctx, prims, views, n_views, settings, cs, gaze_device);
        ctx->capturing = false;
        e = cudaStreamEndCapture(cs, &graph);
    }
    cudaStreamDestroy(cs);
    ctx->stream = stream;  // the capture stream is gone; inspection reads follow the caller's
    const long long per_frame = ctx->launches - launches0;
    ctx->launches = launches0;
    if (st != FHTGS_OK || e != cudaSuccess || ctx->arena_generation != generation) {
        if (graph) cudaGraphDestroy(graph);
        if (st != FHTGS_OK) return st;
        if (e != cudaSuccess) return fail(FHTGS_ERR_CUDA, std::string("frame capture: ") + cudaGetErrorString(e));
        return fail(FHTGS_ERR_CUDA, "the arena moved during the capture");
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(FHTGS_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    auto* g = new fhtgs_frame_graph_s();
    g->ctx = ctx;
    g->graph = graph;
    g->exec = exec;
    g->generation = generation;
    g->launches_per_frame = per_frame;
    g->fp = ctx->fp;
    g->fb = ctx->fb;
    g->split_active = ctx->split_active;
    g->geo = ctx->geo;
    g->views = ctx->views;
    g->frame_foveation = ctx->frame_foveation;
    *out = g;
    return FHTGS_OK;
}

fhtgs_status fhtgs_frame_graph_launch(fhtgs_frame_graph g, void* stream_) {
    if (!g) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null graph");
    fhtgs_context ctx = g->ctx;
    if (ctx->arena_generation != g->generation)
        return fail(FHTGS_ERR_NOT_READY, "the context's arena moved since the capture; create the graph again");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    FHTGS_CK(cudaSetDevice(ctx->device));
    FHTGS_CK(cudaGraphLaunch(g->exec, stream));
    ctx->have_frame = true;
    ctx->fp = g->fp;
    ctx->fb = g->fb;
    ctx->split_active = g->split_active;
    ctx->geo = g->geo;
    ctx->views = g->views;
    ctx->frame_foveation = g->frame_foveation;
    ctx->stream = stream;
    ctx->launches += g->launches_per_frame;
    return FHTGS_OK;
}

fhtgs_status fhtgs_frame_graph_destroy(fhtgs_frame_graph g) {
    if (!g) return FHTGS_OK;
    cudaSetDevice(g->ctx->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return FHTGS_OK;
}

static fhtgs_status mono_common(fhtgs_context ctx, int fast, const float* positions, const float* scales,
                                const float* rotations, const float* opacities, const float* sh_0, const float* sh_rest,
                                int32_t n_primitives, int32_t total_sh_bases, const float* M, const float* VPM,
                                const float* VPR_inv, const float* cam_position, float gaze_x, float gaze_y,
                                const uint32_t* visibility_mask, const uint32_t* visibility_mask_area_table,
                                const uint32_t* fovea_mask_area_table, const float* background_model_data,
                                int32_t texture_width, int32_t texture_height, int32_t background_model_type, int32_t K,
                                int32_t active_sh_bases, int32_t width, int32_t height, float focal_x, float focal_y,
                                float center_x, float center_y, float near_plane, float far_plane, float scale_modifier,
                                int32_t to_chw, int32_t blur_periphery, int32_t anti_aliasing, float* image,
                                void* stream) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null context");
    fhtgs_primitives p{positions, scales, rotations, opacities, sh_0, sh_rest, n_primitives, total_sh_bases,
                       FHTGS_STORAGE_FP32};
    fhtgs_view v{};
    v.M = M; v.VPM = VPM; v.VPR_inv = VPR_inv; v.cam_position = cam_position;
    v.gaze_x = gaze_x; v.gaze_y = gaze_y;
    v.visibility_mask = visibility_mask; v.visibility_mask_area_table = visibility_mask_area_table;
    v.fovea_mask_area_table = fovea_mask_area_table;
    v.width = width; v.height = height; v.focal_x = focal_x; v.focal_y = focal_y; v.center_x = center_x; v.center_y = center_y;
    v.image = image;
    fhtgs_settings s{};
    s.K = K; s.active_sh_bases = active_sh_bases; s.near_plane = near_plane; s.far_plane = far_plane;
    s.scale_modifier = scale_modifier; s.to_chw = to_chw; s.blur_periphery = blur_periphery; s.anti_aliasing = anti_aliasing;
    s.background_type = background_model_type; s.background_data = background_model_data;
    s.texture_width = texture_width; s.texture_height = texture_height; s.fast_math = fast;
    return render_sync_impl(ctx, &p, &v, 1, &s, static_cast<cudaStream_t>(stream));
}

fhtgs_status fhtgs_render_mono(fhtgs_context ctx, const float* positions, const float* scales, const float* rotations,
                               const float* opacities, const float* sh_0, const float* sh_rest, int32_t n_primitives,
                               int32_t total_sh_bases, const float* M, const float* VPM, const float* VPR_inv,
                               const float* cam_position, float gaze_x, float gaze_y, const uint32_t* visibility_mask,
                               const uint32_t* visibility_mask_area_table, const uint32_t* fovea_mask_area_table,
                               const float* background_model_data, int32_t texture_width, int32_t texture_height,
                               int32_t background_model_type, int32_t K, int32_t active_sh_bases, int32_t width,
                               int32_t height, float focal_x, float focal_y, float center_x, float center_y,
                               float near_plane, float far_plane, float scale_modifier, int32_t to_chw,
                               int32_t blur_periphery, int32_t anti_aliasing, float* image, void* stream) {
    return mono_common(ctx, 0, positions, scales, rotations, opacities, sh_0, sh_rest, n_primitives, total_sh_bases, M,
                       VPM, VPR_inv, cam_position, gaze_x, gaze_y, visibility_mask, visibility_mask_area_table,
                       fovea_mask_area_table, background_model_data, texture_width, texture_height,
                       background_model_type, K, active_sh_bases, width, height, focal_x, focal_y, center_x, center_y,
                       near_plane, far_plane, scale_modifier, to_chw, blur_periphery, anti_aliasing, image, stream);
}

fhtgs_status fhtgs_benchmark_mono(fhtgs_context ctx, const float* positions, const float* scales, const float* rotations,
                                  const float* opacities, const float* sh_0, const float* sh_rest, int32_t n_primitives,
                                  int32_t total_sh_bases, const float* M, const float* VPM, const float* VPR_inv,
                                  const float* cam_position, float gaze_x, float gaze_y, const uint32_t* visibility_mask,
                                  const uint32_t* visibility_mask_area_table, const uint32_t* fovea_mask_area_table,
                                  const float* background_model_data, int32_t texture_width, int32_t texture_height,
                                  int32_t background_model_type, int32_t K, int32_t active_sh_bases, int32_t width,
                                  int32_t height, float focal_x, float focal_y, float center_x, float center_y,
                                  float near_plane, float far_plane, float scale_modifier, int32_t to_chw,
                                  int32_t blur_periphery, int32_t anti_aliasing, float* image, void* stream) {
    return mono_common(ctx, 1, positions, scales, rotations, opacities, sh_0, sh_rest, n_primitives, total_sh_bases, M,
                       VPM, VPR_inv, cam_position, gaze_x, gaze_y, visibility_mask, visibility_mask_area_table,
                       fovea_mask_area_table, background_model_data, texture_width, texture_height,
                       background_model_type, K, active_sh_bases, width, height, focal_x, focal_y, center_x, center_y,
                       near_plane, far_plane, scale_modifier, to_chw, blur_periphery, anti_aliasing, image, stream);
}

fhtgs_status fhtgs_render_stereo(
    fhtgs_context ctx, const float* positions, const float* scales, const float* rotations, const float* opacities,
    const float* sh_0, const float* sh_rest, int32_t n_primitives, int32_t total_sh_bases, const float* M_left,
    const float* VPM_left, const float* VPR_inv_left, const float* cam_position_left, float gaze_x_left,
    float gaze_y_left, const uint32_t* visibility_mask_left, const uint32_t* visibility_mask_area_table_left,
    const uint32_t* fovea_mask_area_table_left, const float* background_model_data_left, int32_t texture_width_left,
    int32_t texture_height_left, int32_t background_model_type_left, int32_t K_left, int32_t active_sh_bases_left,
    int32_t width_left, int32_t height_left, float focal_x_left, float focal_y_left, float center_x_left,
    float center_y_left, float near_plane_left, float far_plane_left, float scale_modifier_left, const float* M_right,
    const float* VPM_right, const float* VPR_inv_right, const float* cam_position_right, float gaze_x_right,
    float gaze_y_right, const uint32_t* visibility_mask_right, const uint32_t* visibility_mask_area_table_right,
    const uint32_t* fovea_mask_area_table_right, int32_t width_right, int32_t height_right, float focal_x_right,
    float focal_y_right, float center_x_right, float center_y_right, int32_t to_chw, int32_t blur_periphery,
    int32_t anti_aliasing, float* image_left, float* image_right, void* stream) {
    if (!ctx) return fail(FHTGS_ERR_INVALID_ARGUMENT, "null context");
    fhtgs_primitives p{positions, scales, rotations, opacities, sh_0, sh_rest, n_primitives, total_sh_bases,
                       FHTGS_STORAGE_FP32};
    fhtgs_view v[2] = {};
    v[0].M = M_left; v[0].VPM = VPM_left; v[0].VPR_inv = VPR_inv_left; v[0].cam_position = cam_position_left;
    v[0].gaze_x = gaze_x_left; v[0].gaze_y = gaze_y_left;
    v[0].visibility_mask = visibility_mask_left; v[0].visibility_mask_area_table = visibility_mask_area_table_left;
    v[0].fovea_mask_area_table = fovea_mask_area_table_left;
    v[0].width = width_left; v[0].height = height_left; v[0].focal_x = focal_x_left; v[0].focal_y = focal_y_left;
    v[0].center_x = center_x_left; v[0].center_y = center_y_left; v[0].image = image_left;
    v[1].M = M_right; v[1].VPM = VPM_right; v[1].VPR_inv = VPR_inv_right; v[1].cam_position = cam_position_right;
    v[1].gaze_x = gaze_x_right; v[1].gaze_y = gaze_y_right;
    v[1].visibility_mask = visibility_mask_right; v[1].visibility_mask_area_table = visibility_mask_area_table_right;
    v[1].fovea_mask_area_table = fovea_mask_area_table_right;
    v[1].width = width_right; v[1].height = height_right; v[1].focal_x = focal_x_right; v[1].focal_y = focal_y_right;
    v[1].center_x = center_x_right; v[1].center_y = center_y_right; v[1].image = image_right;
    fhtgs_settings s{};
    s.K = K_left; s.active_sh_bases = active_sh_bases_left; s.near_plane = near_plane_left; s.far_plane = far_plane_left;
    s.scale_modifier = scale_modifier_left; s.to_chw = to_chw; s.blur_periphery = blur_periphery;
    s.anti_aliasing = anti_aliasing; s.background_type = background_model_type_left;
    s.background_data = background_model_data_left; s.texture_width = texture_width_left;
    s.texture_height = texture_height_left; s.fast_math = 1;
    return render_sync_impl(ctx, &p, v, 2, &s, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
