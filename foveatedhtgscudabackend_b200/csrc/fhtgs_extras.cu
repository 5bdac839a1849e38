// Kernels around the rendering path: the tile masks and area tables the renderer consumes,
// display packing of the float images, and the reference's two debug overlays.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/fhtgs.h"
#include "fhtgs_types.cuh"

namespace fhtgs {
void set_last_error(const std::string& msg);  // fhtgs_host.cu
}

using namespace fhtgs;

namespace {

fhtgs_status extras_fail(fhtgs_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

fhtgs_status launch_status(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return extras_fail(FHTGS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return FHTGS_OK;
}

// ------------------------------------------------------------------------------------------
// tile masks and area tables
// ------------------------------------------------------------------------------------------
// One 1024-thread block: bit words (a warp's ballot = one word), then the (gw+1) x (gh+1)
// summed-area table (row prefix, then column prefix), then the 49 x 49 fovea table (3 extra
// sub-tiles for every window tile whose centre lies inside the 24-tile circle, the float test
// of the renderer's fovea classification).
__global__ void __launch_bounds__(1024) build_masks_kernel(const uint8_t* __restrict__ visible, int gw, int gh,
                                                           uint32_t* __restrict__ words, uint32_t* __restrict__ sat,
                                                           uint32_t* __restrict__ fovea_sat) {
    const int n = gw * gh;
    const int lane = threadIdx.x & 31;
    for (int base = (threadIdx.x & ~31); base < n; base += blockDim.x) {  // warp-uniform bound
        const int t = base + lane;
        const bool vis = t < n && (visible == nullptr || visible[t] != 0);
        const uint32_t w = __ballot_sync(0xffffffffu, vis);
        if (lane == 0) words[base / 32] = w;
    }
    const int W1 = gw + 1;
    for (int x = threadIdx.x; x < W1; x += blockDim.x) sat[x] = 0;  // leading zero row
    for (int y = threadIdx.x; y < gh; y += blockDim.x) {
        uint32_t acc = 0;
        sat[(y + 1) * W1] = 0;  // leading zero column
        for (int x = 0; x < gw; ++x) {
            acc += (visible == nullptr || visible[y * gw + x] != 0) ? 1u : 0u;
            sat[(y + 1) * W1 + x + 1] = acc;
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < W1; x += blockDim.x) {
        uint32_t acc = 0;
        for (int y = 1; y <= gh; ++y) {
            acc += sat[y * W1 + x];
            sat[y * W1 + x] = acc;
        }
    }
    if (fovea_sat == nullptr) return;
    constexpr int D = 2 * kFoveaRadiusTiles, F1 = D + 1;
    constexpr float r2 = static_cast<float>(kFoveaRadiusTiles * kFoveaRadiusTiles);
    __shared__ uint32_t cnt[D * D];
    for (int k = threadIdx.x; k < D * D; k += blockDim.x) {
        const float dx = static_cast<float>(k % D - kFoveaRadiusTiles) + 0.5f;
        const float dy = static_cast<float>(k / D - kFoveaRadiusTiles) + 0.5f;
        cnt[k] = dx * dx + dy * dy < r2 ? static_cast<uint32_t>(kSubTiles - 1) : 0u;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < F1; x += blockDim.x) fovea_sat[x] = 0;
    for (int y = threadIdx.x; y < D; y += blockDim.x) {
        uint32_t acc = 0;
        fovea_sat[(y + 1) * F1] = 0;
        for (int x = 0; x < D; ++x) {
            acc += cnt[y * D + x];
            fovea_sat[(y + 1) * F1 + x + 1] = acc;
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < F1; x += blockDim.x) {
        uint32_t acc = 0;
        for (int y = 1; y <= D; ++y) {
            acc += fovea_sat[y * F1 + x];
            fovea_sat[y * F1 + x] = acc;
        }
    }
}

// ------------------------------------------------------------------------------------------
// display packing
// ------------------------------------------------------------------------------------------
struct PackArgs {
    const float* images[8];
    int n_views, width, height, chw, bgra;
};

// Clamp to [0, 1] (NaN -> 0), scale by 255 and round half up: trunc(fma(x, 255, 0.5)).
__device__ __forceinline__ uint32_t to_u8(float x) {
    return static_cast<uint32_t>(__fmaf_rn(fminf(fmaxf(x, 0.0f), 1.0f), 255.0f, 0.5f));
}

// out[y][v * width + x] = RGBA8 (or BGRA8) of view v's pixel (x, y), alpha 255.
__global__ void pack_display_kernel(const __grid_constant__ PackArgs a, uint32_t* __restrict__ out) {
    const int row_len = a.n_views * a.width;
    const int64_t n = static_cast<int64_t>(row_len) * a.height;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(i / row_len), xx = static_cast<int>(i % row_len);
        const int v = xx / a.width, x = xx % a.width;
        const float* img = a.images[v];
        const int64_t p = static_cast<int64_t>(y) * a.width + x;
        float r, g, b;
        if (a.chw) {
            const int64_t np = static_cast<int64_t>(a.width) * a.height;
            r = img[p]; g = img[np + p]; b = img[2 * np + p];
        } else {
            r = img[3 * p]; g = img[3 * p + 1]; b = img[3 * p + 2];
        }
        const uint32_t c0 = to_u8(a.bgra ? b : r), c1 = to_u8(g), c2 = to_u8(a.bgra ? r : b);
        out[i] = c0 | (c1 << 8) | (c2 << 16) | (255u << 24);
    }
}

// ------------------------------------------------------------------------------------------
// debug overlays (restate visualize_gaze_cu and visualize_tile_boundaries_cu,
// visualization/include/kernels/visualization.cuh:11-111, and their launch logic,
// visualization/src/visualization.cu)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void put_rgb(float* img, int W, int H, int x, int y, bool chw, float3 c) {
    const int p = W * y + x;
    if (chw) {
        const int n = W * H;
        img[p] = c.x; img[n + p] = c.y; img[2 * n + p] = c.z;
    } else {
        img[3 * p] = c.x; img[3 * p + 1] = c.y; img[3 * p + 2] = c.z;
    }
}

// Marker of `size` pixels around the clamped gaze: 0 circle, 2 cross, any other type a square.
// Offsets are computed in float from the block/thread position minus size/2 and truncated, as
// the reference does (so odd sizes draw a doubled centre row/column).
__global__ void gaze_marker_kernel(float* img, int W, int H, float gx, float gy, float3 color, float size, int type,
                                   int chw) {
    const int x_off = static_cast<int>(static_cast<float>(blockIdx.x * kTileSmall + threadIdx.x) - size / 2);
    const int y_off = static_cast<int>(static_cast<float>(blockIdx.y * kTileSmall + threadIdx.y) - size / 2);
    if (static_cast<float>(x_off) > size / 2 || static_cast<float>(y_off) > size / 2) return;
    if (type == 0) {
        if (static_cast<float>(x_off * x_off + y_off * y_off) > (size / 2) * (size / 2)) return;
    } else if (type == 2) {
        if (abs(x_off) > 1 && abs(y_off) > 1) return;
    }
    const int x = static_cast<int>(gx) + x_off, y = static_cast<int>(gy) + y_off;
    if (x < 0 || x >= W || y < 0 || y >= H) return;
    put_rgb(img, W, H, x, y, chw != 0, color);
}

// Border pixel k of a tw x th rectangle: top row, bottom row, left column, right column.
__device__ __forceinline__ void border_pixel(int k, int tw, int th, int& x, int& y) {
    if (k < tw) { x = k; y = 0; }
    else if (k < 2 * tw) { x = k - tw; y = th - 1; }
    else if (k < 2 * tw + th - 2) { x = 0; y = k - 2 * tw + 1; }
    else { x = tw - 1; y = k - (2 * tw + th - 2) + 1; }
}

__device__ __forceinline__ bool in_circle(uint32_t tx, uint32_t ty, float gx, float gy, int r) {
    const float dx = (__uint2float_rn(tx) + 0.5f) - gx, dy = (__uint2float_rn(ty) + 0.5f) - gy;
    return dx * dx + dy * dy < static_cast<float>(r * r);
}

// Fovea sub-tiles orange, blended sub-tiles light blue (8x8 borders), periphery tiles green
// (16x16 borders), masked tiles untouched.  The reference draws nothing when at most one
// small-tile entry is active, because its partition ranges stay empty then: every block decides
// that from the mask itself (a fovea tile alone is 4 entries, a periphery tile alone 1).  Then a
// warp per large tile, grid-stride.
__global__ void __launch_bounds__(256) tile_borders_kernel(float* img, int W, int H, const uint32_t* vis, float gtx,
                                                          float gty, int chw) {
    const int glw = (W + kTileLarge - 1) / kTileLarge, glh = (H + kTileLarge - 1) / kTileLarge;
    const int n_large = glw * glh, n_words = (n_large + 31) / 32;
    __shared__ uint32_t s_visible, s_draw;
    if (threadIdx.x == 0) { s_visible = 0; s_draw = 0; }
    __syncthreads();
    uint32_t mine = 0;
    for (int w = threadIdx.x; w < n_words; w += blockDim.x) {
        const uint32_t valid = (w == n_words - 1 && (n_large & 31)) ? ((1u << (n_large & 31)) - 1) : 0xffffffffu;
        mine += __popc(vis[w] & valid);
    }
    atomicAdd(&s_visible, mine);
    __syncthreads();
    if (s_visible == 0) return;
    if (s_visible == 1) {
        for (int w = threadIdx.x; w < n_words; w += blockDim.x) {
            const uint32_t valid = (w == n_words - 1 && (n_large & 31)) ? ((1u << (n_large & 31)) - 1) : 0xffffffffu;
            const uint32_t bits = vis[w] & valid;
            if (bits) {
                const int t = 32 * w + __ffs(bits) - 1;
                s_draw = in_circle(t % glw, t / glw, gtx, gty, kFoveaRadiusTiles) ? 1u : 0u;
            }
        }
        __syncthreads();
        if (s_draw == 0) return;
    }
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), n_warps = gridDim.x * (blockDim.x >> 5);
    const float3 orange = make_float3(0.902f, 0.624f, 0.0f), blue = make_float3(0.337f, 0.706f, 0.914f),
                 green = make_float3(0.0f, 0.620f, 0.451f);
    for (int t = warp; t < n_large; t += n_warps) {
        if ((vis[t / 32] & (1u << (t % 32))) == 0) continue;
        const uint32_t tx = t % glw, ty = t / glw;
        const int ox = static_cast<int>(tx) * kTileLarge, oy = static_cast<int>(ty) * kTileLarge;
        if (in_circle(tx, ty, gtx, gty, kFoveaRadiusTiles)) {
            const float3 c = in_circle(tx, ty, gtx, gty, kBlendRadiusTiles) ? orange : blue;
            constexpr int nb = 2 * kTileSmall + 2 * kTileSmall - 4;  // 28
            for (int k = lane; k < kSubTiles * nb; k += 32) {
                const int sub = k / nb;
                int bx, by;
                border_pixel(k % nb, kTileSmall, kTileSmall, bx, by);
                const int x = ox + (sub % kStride) * kTileSmall + bx, y = oy + (sub / kStride) * kTileSmall + by;
                if (x < W && y < H) put_rgb(img, W, H, x, y, chw != 0, c);
            }
        } else {
            constexpr int nb = 2 * kTileLarge + 2 * kTileLarge - 4;  // 60
            for (int k = lane; k < nb; k += 32) {
                int bx, by;
                border_pixel(k, kTileLarge, kTileLarge, bx, by);
                const int x = ox + bx, y = oy + by;
                if (x < W && y < H) put_rgb(img, W, H, x, y, chw != 0, green);
            }
        }
    }
}

}  // namespace

extern "C" {

fhtgs_status fhtgs_build_tile_masks(const uint8_t* visible_tiles, int32_t width, int32_t height,
                                    uint32_t* visibility_mask, uint32_t* visibility_mask_area_table,
                                    uint32_t* fovea_mask_area_table, void* stream) {
    if (width <= 0 || height <= 0) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "view size must be positive");
    if (!visibility_mask || !visibility_mask_area_table) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "null output");
    const int gw = (width + kTileLarge - 1) / kTileLarge, gh = (height + kTileLarge - 1) / kTileLarge;
    if (static_cast<int64_t>(gw) * gh > (1 << 24)) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "tile grid too large");
    build_masks_kernel<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(visible_tiles, gw, gh, visibility_mask,
                                                                          visibility_mask_area_table,
                                                                          fovea_mask_area_table);
    return launch_status("build_masks_kernel");
}

fhtgs_status fhtgs_pack_display(const float* const* images, int32_t n_views, int32_t width, int32_t height,
                                int32_t to_chw, int32_t bgra, uint8_t* out, void* stream) {
    if (!images || !out) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (n_views <= 0 || n_views > 8) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "n_views must be in [1, 8]");
    if (width <= 0 || height <= 0) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "view size must be positive");
    PackArgs a{};
    for (int v = 0; v < n_views; ++v) {
        if (!images[v]) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "null image");
        a.images[v] = images[v];
    }
    a.n_views = n_views; a.width = width; a.height = height; a.chw = to_chw ? 1 : 0; a.bgra = bgra ? 1 : 0;
    const int64_t n = static_cast<int64_t>(n_views) * width * height;
    const int blocks = static_cast<int>(n / 256 + 1 < 148 * 16 ? n / 256 + 1 : 148 * 16);
    pack_display_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(a, reinterpret_cast<uint32_t*>(out));
    return launch_status("pack_display_kernel");
}

fhtgs_status fhtgs_visualize_gaze(float* image, int32_t width, int32_t height, float gaze_x, float gaze_y, float r,
                                  float g, float b, int32_t visualization_type, int32_t visualization_size,
                                  int32_t to_chw, void* stream) {
    if (!image || width <= 0 || height <= 0) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "bad image");
    if (visualization_type < 0 || visualization_type > 255) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "marker type must fit in 8 bits");
    if (visualization_size <= 0) return FHTGS_OK;
    const float gx = fminf(fmaxf(gaze_x, 0.0f), static_cast<float>(width - 1));
    const float gy = fminf(fmaxf(gaze_y, 0.0f), static_cast<float>(height - 1));
    const int nb = (visualization_size + kTileSmall - 1) / kTileSmall;
    gaze_marker_kernel<<<dim3(nb, nb), dim3(kTileSmall, kTileSmall), 0, static_cast<cudaStream_t>(stream)>>>(
        image, width, height, gx, gy, make_float3(r, g, b), static_cast<float>(visualization_size), visualization_type,
        to_chw);
    return launch_status("gaze_marker_kernel");
}

fhtgs_status fhtgs_visualize_tile_boundaries(float* image, int32_t width, int32_t height,
                                             const uint32_t* visibility_mask, float gaze_x, float gaze_y,
                                             int32_t to_chw, void* stream) {
    if (!image || !visibility_mask || width <= 0 || height <= 0) return extras_fail(FHTGS_ERR_INVALID_ARGUMENT, "bad argument");
    const float gx = fminf(fmaxf(gaze_x, 0.0f), static_cast<float>(width - 1));
    const float gy = fminf(fmaxf(gaze_y, 0.0f), static_cast<float>(height - 1));
    const int gw = ((width + kTileLarge - 1) / kTileLarge) * kStride, gh = ((height + kTileLarge - 1) / kTileLarge) * kStride;
    const int gtx = max(0, min(gw - 1, (static_cast<int>(gx) + kTileLarge / 2) / kTileLarge));
    const int gty = max(0, min(gh - 1, (static_cast<int>(gy) + kTileLarge / 2) / kTileLarge));
    const int n_large = (gw / kStride) * (gh / kStride);
    const int blocks = std::min((n_large + 7) / 8, 148 * 8);
    tile_borders_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(image, width, height, visibility_mask,
                                                                             static_cast<float>(gtx),
                                                                             static_cast<float>(gty), to_chw);
    return launch_status("tile_borders_kernel");
}

}  // extern "C"
