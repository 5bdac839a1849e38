// fhtgs device kernels.  Included by kernels_fast.cu (-use_fast_math, the arithmetic of the
// reference's _C_benchmarking / _C_stereo modules) and kernels_ieee.cu (the arithmetic of the
// reference's _C module) with FHTGS_FLAVOR naming the namespace.
//
// Pipeline of one frame, all views of the frame in the same launches, no host round trip:
//   setup      gather per-view camera matrices into ViewParams
//   classify   large-tile classification + compaction (one block per view)
//   preprocess one thread per Gaussian for all views: cull, project, bounds, SH colour
//   scan       exclusive scan of the preprocess blocks' instance sums -> M per view
//   create     one (large-tile key, primitive) instance per visible tile of the bounds
//   sort       stable LSD radix sort of (key, value) pairs, 8-bit digits
//   ranges     [begin, end) per large tile from key boundaries
// The reference stores the four sub-tiles of every fovea tile as separate instances with
// identical lists, plus sentinel slots for masked fovea tiles; here each list is stored once
// and the reference's arrays are reproduced exactly on request (fhtgs_copy_intermediates).
//   blend      K-buffer blend; full-res 16x16 tiles (fovea, blended) and 2x-down 16x16
//              tiles (periphery), persistent blocks pulling tiles from a work counter
//   compose    periphery bilinear upsampling / blur and blended-ring cross-fade
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fhtgs_math.cuh"
#include "fhtgs_types.cuh"

#ifndef FHTGS_FLAVOR
#error "FHTGS_FLAVOR must name the math flavour namespace"
#endif

namespace fhtgs {
namespace FHTGS_FLAVOR {
using namespace fhtgs::vm;

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Block-wide exclusive scan (blockDim.x multiple of 32, <= 1024).  `total` receives the sum.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T x, T& total, T* s_warp /* >= 32 entries */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T incl = warp_incl_scan(x);
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nw ? s_warp[lane] : T(0);
        T wi = warp_incl_scan(w);
        if (lane < nw) s_warp[lane] = wi - w;
        if (lane == nw - 1) s_warp[32] = wi;
    }
    __syncthreads();
    T res = incl - x + s_warp[warp];
    total = s_warp[32];
    __syncthreads();
    return res;
}

__device__ __forceinline__ bool tile_visible(const uint32_t* mask, uint32_t tile) {
    return (mask[tile / 32u] & (1u << (tile % 32u))) != 0;
}

// Tile-centre-in-circle test of the foveation (shared_kernels.cuh:155-220 and
// kernel_utils.cuh:43-73 of the reference use the same float arithmetic).
template <int radius>
__device__ __forceinline__ bool in_fovea(uint32_t tx, uint32_t ty, float2 gaze_tiles) {
    constexpr float r2 = static_cast<float>(radius * radius);
    const float2 d = make_float2(__uint2float_rn(tx) + 0.5f, __uint2float_rn(ty) + 0.5f) - gaze_tiles;
    return dot(d, d) < r2;
}

__device__ __forceinline__ float4 ld4(const float* p) { return make_float4(p[0], p[1], p[2], p[3]); }

// ------------------------------------------------------------------------------------------
// setup
// ------------------------------------------------------------------------------------------
constexpr int kSetupChunk = 32;
struct SetupChunk {
    ViewSetup v[kSetupChunk];
    int n, first;
};

// Gaze clamp and rounding of the host path (fhtgs_host.cu: geometry(), after inference.cu:79-105
// of the reference), for a gaze read from device memory: std::max/std::min as comparisons.
__device__ __forceinline__ void gaze_from_device(ViewParams& p, const float* g) {
    const float wm1 = static_cast<float>(p.width - 1), hm1 = static_cast<float>(p.height - 1);
    float gx = g[0] < 0.0f ? 0.0f : g[0];
    float gy = g[1] < 0.0f ? 0.0f : g[1];
    gx = wm1 < gx ? wm1 : gx;
    gy = hm1 < gy ? hm1 : gy;
    const int gw = p.glw * kStride, gh = p.glh * kStride;
    const int tx = max(0, min(gw - 1, (static_cast<int>(gx) + kTileLarge / 2) / kTileLarge));
    const int ty = max(0, min(gh - 1, (static_cast<int>(gy) + kTileLarge / 2) / kTileLarge));
    p.gaze_px = make_float2(gx, gy);
    p.gaze_tiles = make_float2(static_cast<float>(tx), static_cast<float>(ty));
    p.gaze_tiles_i = make_int2(tx, ty);
}

__global__ void setup_kernel(const __grid_constant__ SetupChunk c, ViewParams* __restrict__ out) {
    const int i = threadIdx.x;
    if (i >= c.n) return;
    ViewParams p = c.v[i].p;
    if (c.v[i].gaze) gaze_from_device(p, c.v[i].gaze);
    for (int r = 0; r < 3; ++r) p.M[r] = ld4(c.v[i].M + 4 * r);
    for (int r = 0; r < 4; ++r) p.VPM[r] = ld4(c.v[i].VPM + 4 * r);
    for (int r = 0; r < 4; ++r) p.VPR_inv[r] = ld4(c.v[i].VPR_inv + 4 * r);
    p.cam = make_float4(c.v[i].cam[0], c.v[i].cam[1], c.v[i].cam[2], 0.0f);
    out[c.first + i] = p;
}

int launch_setup(const ViewSetup* setups, int n_views, ViewParams* out, cudaStream_t s) {
    int n = 0;
    for (int first = 0; first < n_views; first += kSetupChunk) {
        SetupChunk c;
        c.n = n_views - first < kSetupChunk ? n_views - first : kSetupChunk;
        c.first = first;
        for (int i = 0; i < c.n; ++i) c.v[i] = setups[first + i];
        setup_kernel<<<1, kSetupChunk, 0, s>>>(c, out);
        ++n;
    }
    return n;
}

// ------------------------------------------------------------------------------------------
// tile classification + compaction (replaces fill_tile_index_num_tiles, the scan,
// build_tile_index_map, the 2-bit type sort and get_partition_ranges_cu of the reference,
// shared_kernels.cuh:155-238, inference.cu:131-188, with one block per view)
// ------------------------------------------------------------------------------------------
// Ring level of a large tile: squared NDC distance of the tile centre from the (clamped) gaze,
// x and y each scaled by half the image size, in explicitly rounded IEEE steps (the CPU
// oracle evaluates the same sequence, so both agree on every tile).
__device__ __forceinline__ uint8_t ring_tile_type(const ViewParams& vp, uint32_t tx, uint32_t ty) {
    const float cx = static_cast<float>(tx * kTileLarge + kTileLarge / 2);
    const float cy = static_cast<float>(ty * kTileLarge + kTileLarge / 2);
    const float dx = __fdiv_rn(__fsub_rn(cx, vp.gaze_px.x), __fmul_rn(0.5f, static_cast<float>(vp.width)));
    const float dy = __fdiv_rn(__fsub_rn(cy, vp.gaze_px.y), __fmul_rn(0.5f, static_cast<float>(vp.height)));
    const float r2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    return r2 < vp.ring_full2 ? kFovea : r2 < vp.ring_half2 ? kPeriphery : kQuarter;
}

__device__ __forceinline__ uint8_t large_tile_type(const ViewParams& vp, const FrameParams& fp, uint32_t tile) {
    if (!tile_visible(vp.vis_mask, tile)) return kMasked;
    if (vp.fov_mode == kFoveationNone) return kFovea;
    const uint32_t tx = tile % static_cast<uint32_t>(vp.glw), ty = tile / static_cast<uint32_t>(vp.glw);
    if (vp.fov_mode == kFoveationRings) return ring_tile_type(vp, tx, ty);
    if (in_fovea<kFoveaRadiusTiles>(tx, ty, vp.gaze_tiles))
        return in_fovea<kBlendRadiusTiles>(tx, ty, vp.gaze_tiles) ? kFovea : kBlended;
    return kPeriphery;
}

__global__ void __launch_bounds__(1024) classify_kernel(FrameParams fp, FrameBuffers fb) {
    __shared__ unsigned long long s_warp[33];
    const int v = blockIdx.x;
    const ViewParams& vp = fb.views[v];
    const int TL = vp.n_large;
    const int seg = (TL + blockDim.x - 1) / blockDim.x;
    const int b0 = min(TL, static_cast<int>(threadIdx.x) * seg), b1 = min(TL, b0 + seg);
    uint32_t cnt[5] = {0, 0, 0, 0, 0};
    for (int t = b0; t < b1; ++t) cnt[large_tile_type(vp, fp, t)]++;
    // packed 64-bit scans: (fovea | periphery << 32), (blended | masked << 32), quarter
    unsigned long long tot0, tot1, tot2;
    unsigned long long e0 = block_excl_scan<unsigned long long>(cnt[0] | (static_cast<unsigned long long>(cnt[1]) << 32), tot0, s_warp);
    unsigned long long e1 = block_excl_scan<unsigned long long>(cnt[2] | (static_cast<unsigned long long>(cnt[3]) << 32), tot1, s_warp);
    unsigned long long e2 = block_excl_scan<unsigned long long>(cnt[4], tot2, s_warp);
    const uint32_t nF = static_cast<uint32_t>(tot0), nP = static_cast<uint32_t>(tot0 >> 32);
    const uint32_t nB = static_cast<uint32_t>(tot1), nM = static_cast<uint32_t>(tot1 >> 32);
    const uint32_t nQ = static_cast<uint32_t>(tot2);
    uint32_t oF = static_cast<uint32_t>(e0), oP = static_cast<uint32_t>(e0 >> 32);
    uint32_t oB = static_cast<uint32_t>(e1), oM = static_cast<uint32_t>(e1 >> 32);
    uint32_t oQ = static_cast<uint32_t>(e2);
    // quarter tiles appear in the partitioned map as periphery entries (after the others)
    const uint32_t n_active = kSubTiles * nF + nP + nQ + kSubTiles * nB;
    // The reference renders nothing when exactly one small-tile entry is active (its
    // partition-range kernel starts at index 1, shared_kernels.cuh:222-238); that tile is then
    // cleared instead of blended, which matches the zero-initialised output of _C.  The other
    // foveation modes have no counterpart there and no such rule.
    const bool none = vp.fov_mode == kFoveationReference && n_active <= 1;
    uint32_t* map = fb.tile_map_part + static_cast<size_t>(v) * fp.max_tiles;
    uint8_t* typ = fb.tile_type_part + static_cast<size_t>(v) * fp.max_tiles;
    uint8_t* lt = fb.large_type + static_cast<size_t>(v) * fp.max_large;
    uint32_t* wf = fb.work_full + static_cast<size_t>(v) * fp.max_large;
    uint32_t* wl = fb.work_low + static_cast<size_t>(v) * fp.max_large;
    uint32_t* wm = fb.work_masked + static_cast<size_t>(v) * fp.max_large;
    for (int t = b0; t < b1; ++t) {
        const uint8_t ty = large_tile_type(vp, fp, t);
        lt[t] = ty;
        const uint32_t sub0 = static_cast<uint32_t>(t) * kSubTiles;
        if (ty == kFovea) {
            for (int i = 0; i < kSubTiles; ++i) { map[kSubTiles * oF + i] = sub0 + i; typ[kSubTiles * oF + i] = kFovea; }
            wf[oF++] = t;
        } else if (ty == kPeriphery) {
            map[kSubTiles * nF + oP] = sub0; typ[kSubTiles * nF + oP] = kPeriphery;
            if (none) wm[nM] = t; else wl[oP] = t;
            ++oP;
        } else if (ty == kBlended) {
            const uint32_t base = kSubTiles * nF + nP + nQ + kSubTiles * oB;
            for (int i = 0; i < kSubTiles; ++i) { map[base + i] = sub0 + i; typ[base + i] = kBlended; }
            wf[nF + oB++] = t;
        } else if (ty == kQuarter) {
            map[kSubTiles * nF + nP + oQ] = sub0; typ[kSubTiles * nF + nP + oQ] = kPeriphery;
            wl[nP + oQ++] = t;
        } else {
            wm[oM++] = t;
        }
    }
    if (threadIdx.x == 0) {
        FrameStatus& st = fb.status[v];
        st.n_active = n_active;
        for (int k = 0; k < 6; ++k) st.ranges[k] = 0;
        if (!none) {
            if (nF) { st.ranges[0] = 0; st.ranges[1] = kSubTiles * nF; }
            if (nP + nQ) { st.ranges[2] = kSubTiles * nF; st.ranges[3] = kSubTiles * nF + nP + nQ; }
            if (nB) { st.ranges[4] = kSubTiles * nF + nP + nQ; st.ranges[5] = n_active; }
        }
        st.n_fovea_large = nF;
        st.n_blended_large = nB;
        st.n_periphery_large = none ? 0 : nP;
        st.n_quarter_large = nQ;
        st.n_masked_large = none ? nM + nP : nM;
        // overflow and the instance counts were zeroed before the frame: the preprocess,
        // running beside this kernel, adds to them
    }
}

int launch_classify(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s) {
    classify_kernel<<<fp.n_views, 1024, 0, s>>>(fp, fb);
    return 1;
}

// ------------------------------------------------------------------------------------------
// preprocess (restates preprocess_cu / transform_and_cull / convert_sh_to_color of the
// reference, inference.cuh:42-136, kernel_utils.cuh:76-213, sh_utils.cuh:8-69, with the same
// expression structure; one thread per Gaussian, all views per thread)
// ------------------------------------------------------------------------------------------
struct Mat3 { float r11, r12, r13, r21, r22, r23, r31, r32, r33; };

// Quaternion (w,x,y,z), not normalised, to rotation matrix (kernel_utils.cuh:76-88 of the
// reference).  Which product of each sum is fused into an FMA decides the last bit of the
// result; the choice below is the one the reference's build makes (established from its
// outputs: tests/golden and the live comparison), written with explicit intrinsics so that
// it no longer depends on the compiler's contraction heuristics.
__device__ __forceinline__ Mat3 quat_to_rot(const float4 q) {
    const float r = q.x, x = q.y, y = q.z, z = q.w;
    const float xx = __fmul_rn(x, x), yy = __fmul_rn(y, y), zz = __fmul_rn(z, z);
    const float xy = __fmul_rn(x, y), xz = __fmul_rn(x, z), yz = __fmul_rn(y, z);
    const float rx = __fmul_rn(r, x), ry = __fmul_rn(r, y), rz = __fmul_rn(r, z);
    return {__fmaf_rn(-2.0f, __fadd_rn(yy, zz), 1.0f), 2.0f * __fmaf_rn(x, y, -rz), 2.0f * __fmaf_rn(r, y, xz),
            2.0f * __fmaf_rn(x, y, rz), __fmaf_rn(-2.0f, __fmaf_rn(x, x, zz), 1.0f), 2.0f * __fmaf_rn(y, z, -rx),
            2.0f * __fmaf_rn(-r, y, xz), 2.0f * __fmaf_rn(y, z, rx), __fmaf_rn(-2.0f, __fmaf_rn(x, x, yy), 1.0f)};
}

// n . a with the left-to-right fused evaluation ((n.x a.x) + n.y a.y) + n.z a.z.
__device__ __forceinline__ float dot3_lr(const float3 n, const float3 a) {
    return __fmaf_rn(n.z, a.z, __fmaf_rn(n.y, a.y, __fmul_rn(n.x, a.x)));
}

// Real spherical-harmonics basis constants (degree <= 3).
constexpr float kC0 = 0.28209479177387814f, kC1 = 0.48860251190291987f;
constexpr float kC2a = 1.0925484305920792f, kC2b = 0.94617469575755997f, kC2c = 0.31539156525251999f,
                kC2d = 0.54627421529603959f;
constexpr float kC3a = 0.59004358992664352f, kC3b = 1.7701307697799304f, kC3c = 2.8906114426405538f,
                kC3d = 0.45704579946446572f, kC3e = 2.2852289973223288f, kC3f = 1.865881662950577f,
                kC3g = 1.1195289977703462f, kC3h = 1.4453057213202769f;

// Attribute loads of the two storage formats, widened to float32 (exact conversions).
__device__ __forceinline__ float ldf(const float* p) { return *p; }
__device__ __forceinline__ float ldf(const __half* p) { return __half2float(*p); }
__device__ __forceinline__ float ldf(const __nv_bfloat16* p) { return __bfloat162float(*p); }
template <typename T>
__device__ __forceinline__ float3 ld3t(const T* p) { return make_float3(ldf(p), ldf(p + 1), ldf(p + 2)); }
template <typename T>
__device__ __forceinline__ float4 ld4t(const T* p) { return make_float4(ldf(p), ldf(p + 1), ldf(p + 2), ldf(p + 3)); }

template <typename ShT>
__device__ __forceinline__ float3 sh_to_rgb(const ShT* __restrict__ sh0, const ShT* __restrict__ rest,
                                            float3 pos, float3 cam, int active) {
    auto ld3 = [](const ShT* p) { return ld3t(p); };
    float3 res = 0.5f + kC0 * ld3(sh0);
    if (active > 1) {
        const float3 d = normalize(pos - cam);
        const float x = d.x, y = d.y, z = d.z;
        res = res - kC1 * y * ld3(rest + 0) + kC1 * z * ld3(rest + 3) - kC1 * x * ld3(rest + 6);
        if (active > 4) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, xz = x * z, yz = y * z;
            res = res + kC2a * xy * ld3(rest + 9) - kC2a * yz * ld3(rest + 12) + (kC2b * zz - kC2c) * ld3(rest + 15)
                      - kC2a * xz * ld3(rest + 18) + kC2d * (xx - yy) * ld3(rest + 21);
            if (active > 9) {
                res = res + y * (kC3a * yy - kC3b * xx) * ld3(rest + 24) + kC3c * xy * z * ld3(rest + 27)
                          + y * (kC3d - kC3e * zz) * ld3(rest + 30) + z * (kC3f * zz - kC3g) * ld3(rest + 33)
                          + x * (kC3d - kC3e * zz) * ld3(rest + 36) + kC3h * z * (xx - yy) * ld3(rest + 39)
                          + x * (kC3b * yy - kC3a * xx) * ld3(rest + 42);
            }
        }
    }
    return res;
}

// Touched-tile count of the reference (visible tiles of the bounds from the visibility SAT,
// plus 3 per fovea-window tile from the fovea SAT); `vis` receives the first part alone.
__device__ __forceinline__ uint32_t touched_from_bounds(const ViewParams& vp, const uint4 b, uint32_t& vis) {
    const int diam = 2 * kFoveaRadiusTiles;
    const int tlx = vp.gaze_tiles_i.x - kFoveaRadiusTiles, tly = vp.gaze_tiles_i.y - kFoveaRadiusTiles;
    const uint4 fb = make_uint4(min(diam, max(0, static_cast<int>(b.x) - tlx)), min(diam, max(0, static_cast<int>(b.y) - tlx)),
                                min(diam, max(0, static_cast<int>(b.z) - tly)), min(diam, max(0, static_cast<int>(b.w) - tly)));
    const uint32_t W1 = static_cast<uint32_t>(vp.glw) + 1u;
    const uint32_t* sat = vp.vis_sat;
    uint32_t n = sat[b.y + W1 * b.w] + sat[b.x + W1 * b.z] - sat[b.y + W1 * b.z] - sat[b.x + W1 * b.w];
    vis = n;
    if (fb.y != fb.x && fb.w != fb.z) {
        const uint32_t F1 = static_cast<uint32_t>(diam) + 1u;
        const uint32_t* f = vp.fovea_sat;
        n += f[fb.y + F1 * fb.w] + f[fb.x + F1 * fb.z] - f[fb.y + F1 * fb.z] - f[fb.x + F1 * fb.w];
    }
    return n;
}

__device__ __forceinline__ float4 xform_row(const float4 P, float3 u, float3 v, float3 w, float3 pos) {
    const float3 n = xyz(P);
    return make_float4(dot3_lr(n, u), dot3_lr(n, v), dot3_lr(n, w), __fadd_rn(dot3_lr(n, pos), P.w));
}

// Column c of R scaled by s then by the scale modifier: ((R_ic * s) * m).
__device__ __forceinline__ float3 scaled_axis(float a, float b, float c, float s, float m) {
    return make_float3(__fmul_rn(__fmul_rn(a, s), m), __fmul_rn(__fmul_rn(b, s), m), __fmul_rn(__fmul_rn(c, s), m));
}

// Standard (non anti-aliased) transform and cull.  Returns true when culled.
__device__ __forceinline__ bool transform_and_cull(const ViewParams& vp, const FrameParams& fp, float3 pos,
                                                   float3 scale, float4 quat, float opacity, float4& P1,
                                                   float4& P2, float4& P4, uint4& b, uint32_t& n, uint32_t& vis) {
    const float4 M3 = vp.M[2];
    const float z = dot(xyz(M3), pos) + M3.w;
    if (z < fp.near_plane || z > fp.far_plane) return true;
    const Mat3 R = quat_to_rot(quat);
    const float3 u = scaled_axis(R.r11, R.r21, R.r31, scale.x, fp.scale_modifier);
    const float3 v = scaled_axis(R.r12, R.r22, R.r32, scale.y, fp.scale_modifier);
    const float3 w = scaled_axis(R.r13, R.r23, R.r33, scale.z, fp.scale_modifier);
    P4 = xform_row(vp.VPM[3], u, v, w, pos);
    const float rho_cutoff = 2.0f * logf(opacity * kMinAlphaRcp);
    const float4 d = make_float4(rho_cutoff, rho_cutoff, rho_cutoff, -1.0f);
    const float s = dot(d, P4 * P4);
    if (s == 0.0f) return true;
    const float4 f = (1.0f / s) * d;
    const float4 P3 = xform_row(vp.VPM[2], u, v, w, pos);
    const float cz = dot(f, P3 * P4);
    const float ez = sqrtf(fmaxf(cz * cz - dot(f, P3 * P3), 0.0f));
    if (cz - ez < -1.0f || cz + ez > 1.0f) return true;
    P1 = xform_row(vp.VPM[0], u, v, w, pos);
    const float cx = dot(f, P1 * P4);
    const float ex = sqrtf(fmaxf(cx * cx - dot(f, P1 * P1), 0.0f));
    P2 = xform_row(vp.VPM[1], u, v, w, pos);
    const float cy = dot(f, P2 * P4);
    const float ey = sqrtf(fmaxf(cy * cy - dot(f, P2 * P2), 0.0f));
    const uint32_t gw = static_cast<uint32_t>(vp.glw), gh = static_cast<uint32_t>(vp.glh);
    const float tw = static_cast<float>(kTileLarge);
    b = make_uint4(min(gw, static_cast<uint32_t>(max(0, __float2int_rd((cx - ex + 0.5f) / tw)))),
                   min(gw, static_cast<uint32_t>(max(0, __float2int_ru((cx + ex + 0.5f) / tw)))),
                   min(gh, static_cast<uint32_t>(max(0, __float2int_rd((cy - ey + 0.5f) / tw)))),
                   min(gh, static_cast<uint32_t>(max(0, __float2int_ru((cy + ey + 0.5f) / tw)))));
    n = touched_from_bounds(vp, b, vis);
    return n == 0;
}

// ---- anti-aliased variant (restates kernel_utils_aaa.cuh:9-363) ----
__device__ __forceinline__ float max_contrib_plane(float4 plane, float4 P1, float4 P2, float4 P3, float4 P4, float4& out) {
    const float norm = plane.w / (plane.x * plane.x + plane.y * plane.y + plane.z * plane.z);
    const float4 mp = -norm * plane;
    out.x = dot(xyz(P1), xyz(mp)) + P1.w;
    out.y = dot(xyz(P2), xyz(mp)) + P2.w;
    out.z = dot(xyz(P3), xyz(mp)) + P3.w;
    out.w = dot(xyz(P4), xyz(mp)) + P4.w;
    return -mp.w;
}
__device__ __forceinline__ float max_contrib_ray(float4 a, float4 b, float4 P1, float4 P2, float4 P3, float4 P4, float4& out) {
    const float3 d = make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
    const float3 m = make_float3(a.w * b.x - a.x * b.w, a.w * b.y - a.y * b.w, a.w * b.z - a.z * b.w);
    const float dd = dot(d, d);
    const float3 mdd = make_float3(m.x / dd, m.y / dd, m.z / dd);
    const float3 mp = cross(d, mdd);
    out.x = dot(xyz(P1), mp) + P1.w;
    out.y = dot(xyz(P2), mp) + P2.w;
    out.z = dot(xyz(P3), mp) + P3.w;
    out.w = dot(xyz(P4), mp) + P4.w;
    return dot(m, mdd);
}
__device__ __forceinline__ bool in_screen_range(float p, float from, float ext, float ph) {
    const float d = p - from * ph;
    return d > 0.0f && d < ext * ph;
}
__device__ float max_contrib_frustum(float4 P1, float4 P2, float4 P3, float4 P4, float width, float height) {
    float best = 3.402823466e+38f;
    const float3 from = make_float3(0.0f, 0.0f, -1.0f);
    const float3 ext = make_float3(width - 1.0f, height - 1.0f, 2.0f);
    const float3 d = make_float3(P1.w - from.x * P4.w, P2.w - from.y * P4.w, P3.w - from.z * P4.w);
    const bool bx = d.x > 0.0f && d.x < ext.x * P4.w;
    const bool by = d.y > 0.0f && d.y < ext.y * P4.w;
    const bool bz = d.z > 0.0f && d.z < ext.z * P4.w;
    if (bx && by && bz) return 0.0f;
    const float dx = copysignf(ext.x * 0.5f, d.x - (ext.x * 0.5f * P4.w));
    const float dy = copysignf(ext.y * 0.5f, d.y - (ext.y * 0.5f * P4.w));
    const float4 cpx = P1 - P4 * (from.x + ext.x * 0.5f + dx);
    const float4 cpy = P2 - P4 * (from.y + ext.y * 0.5f + dy);
    float4 ps;
    float c = max_contrib_plane(cpx, P1, P2, P3, P4, ps);
    if (c < best && in_screen_range(ps.y, from.y, ext.y, ps.w) && in_screen_range(ps.z, from.z, ext.z, ps.w)) best = c;
    c = max_contrib_plane(cpy, P1, P2, P3, P4, ps);
    if (c < best && in_screen_range(ps.x, from.x, ext.x, ps.w) && in_screen_range(ps.z, from.z, ext.z, ps.w)) best = c;
    c = max_contrib_ray(cpx, cpy, P1, P2, P3, P4, ps);
    if (c < best && in_screen_range(ps.z, from.z, ext.z, ps.w)) best = c;
    const float4 opy = P2 - P4 * (from.y + ext.y * 0.5f - dy);
    c = max_contrib_ray(cpx, opy, P1, P2, P3, P4, ps);
    if (c < best && in_screen_range(ps.z, from.z, ext.z, ps.w)) best = c;
    const float4 opx = P1 - P4 * (from.x + ext.x * 0.5f - dx);
    c = max_contrib_ray(opx, cpy, P1, P2, P3, P4, ps);
    if (c < best && in_screen_range(ps.z, from.z, ext.z, ps.w)) best = c;
    return best;
}
__device__ __forceinline__ float normalize_angle(float th) {
    constexpr float pi = 3.141592654f;
    constexpr float two_pi = 2.0f * pi;
    th = fmodf(th, two_pi);
    if (th > pi) th -= two_pi;
    if (th <= -pi) th += two_pi;
    return th;
}
__device__ __forceinline__ float2 aabb_theta(float4 MT_axis, float4 MT3, float4 t, float theta_mu) {
    constexpr float pi = 3.141592654f;
    constexpr float two_pi = 2.0f * pi;
    constexpr float max_theta = 0.5f * pi - 1e-5f;
    const float sq_axis = dot(t, MT_axis * MT_axis);
    const float sq_z = dot(t, MT3 * MT3);
    const float mid = dot(t, MT_axis * MT3);
    const float inside = mid * mid - sq_z * sq_axis;
    float2 r = make_float2(-max_theta, max_theta);
    if (inside > 0.0f) {
        float2 th = make_float2(atan2f(-(mid + sqrtf(inside)), -sq_z), atan2f(-(mid - sqrtf(inside)), -sq_z));
        while (th.x > theta_mu) th.x -= pi;
        while (th.x < (theta_mu - pi)) th.x += pi;
        while (th.y < theta_mu) th.y += pi;
        while (th.y > (theta_mu + pi)) th.y -= pi;
        const float2 tn = make_float2(normalize_angle(th.x), normalize_angle(th.y));
        if (theta_mu < 0.0f && fabsf(tn.x) < fabsf(tn.y)) { th.x += two_pi; th.y += two_pi; }
        else if (theta_mu > 0.0f && fabsf(tn.y) < fabsf(tn.x)) { th.x -= two_pi; th.y -= two_pi; }
        r = make_float2(fmaxf(r.x, th.x), fminf(r.y, th.y));
    }
    return make_float2(tanf(r.x), tanf(r.y));
}

__device__ __forceinline__ bool transform_and_cull_aaa(const ViewParams& vp, const FrameParams& fp, float3 pos,
                                                       float3 osc, float4 quat, float& opacity, float4& P1,
                                                       float4& P2, float4& P4, uint4& b, uint32_t& n, uint32_t& vis) {
    const Mat3 R = quat_to_rot(quat);
    const float4 M3 = vp.M[2];
    const float z = dot(xyz(M3), pos) + M3.w;
    constexpr float kernel_size = 0.3f;
    const float max_focal = fmaxf(vp.focal_x, vp.focal_y);
    const float fsv = z / max_focal;
    const float fvar = fsv * fsv * kernel_size;
    const float3 ovar = osc * osc;
    const float3 var = make_float3(ovar.x + fvar, ovar.y + fvar, ovar.z + fvar);
    const float3 sc = make_float3(sqrtf(var.x), sqrtf(var.y), sqrtf(var.z));
    const float3 cam = xyz(vp.cam);
    const float3 vdw = normalize(pos - cam);
    const float3 vdg = make_float3(R.r11 * vdw.x + R.r21 * vdw.y + R.r31 * vdw.z,
                                   R.r12 * vdw.x + R.r22 * vdw.y + R.r32 * vdw.z,
                                   R.r13 * vdw.x + R.r23 * vdw.y + R.r33 * vdw.z);
    const float3 r = vdg * vdg;
    const float det_o = dot(r, make_float3(ovar.y * ovar.z, ovar.z * ovar.x, ovar.x * ovar.y));
    const float det_d = dot(r, make_float3(var.y * var.z, var.z * var.x, var.x * var.y));
    const float dil = sqrtf(__saturatef(det_o / det_d));
    opacity *= dil;
    if (opacity < kMinAlpha) return true;
    const float rho_cutoff = 2.0f * logf(opacity * kMinAlphaRcp);
    const float3 cs = cam - pos;
    const float3 cg = make_float3(R.r11 * cs.x + R.r21 * cs.y + R.r31 * cs.z, R.r12 * cs.x + R.r22 * cs.y + R.r32 * cs.z,
                                  R.r13 * cs.x + R.r23 * cs.y + R.r33 * cs.z) / sc;
    if (dot(cg, cg) < rho_cutoff) return true;
    const float3 u = scaled_axis(R.r11, R.r21, R.r31, sc.x, fp.scale_modifier);
    const float3 v = scaled_axis(R.r12, R.r22, R.r32, sc.y, fp.scale_modifier);
    const float3 w = scaled_axis(R.r13, R.r23, R.r33, sc.z, fp.scale_modifier);
    P1 = xform_row(vp.VPM[0], u, v, w, pos);
    P2 = xform_row(vp.VPM[1], u, v, w, pos);
    const float4 P3 = xform_row(vp.VPM[2], u, v, w, pos);
    P4 = xform_row(vp.VPM[3], u, v, w, pos);
    const float mc = max_contrib_frustum(P1, P2, P3, P4, static_cast<float>(vp.width), static_cast<float>(vp.height));
    if (mc > rho_cutoff) return true;
    const float4 MT1 = xform_row(vp.M[0], u, v, w, pos);
    const float4 MT2 = xform_row(vp.M[1], u, v, w, pos);
    const float4 t = make_float4(rho_cutoff, rho_cutoff, rho_cutoff, -1.0f);
    const float3 viewdir = normalize(make_float3(MT1.w, MT2.w, P4.w));
    const float2 tx = aabb_theta(MT1, P4, t, atan2f(viewdir.x, viewdir.z));
    const float2 ty = aabb_theta(MT2, P4, t, atan2f(viewdir.y, viewdir.z));
    const float2 bxx = make_float2(vp.center_x + vp.focal_x * tx.x, vp.center_x + vp.focal_x * tx.y);
    const float2 byy = make_float2(vp.center_y + vp.focal_y * ty.x, vp.center_y + vp.focal_y * ty.y);
    const float2 ctr = make_float2((bxx.y + bxx.x) / 2.0f, (byy.y + byy.x) / 2.0f);
    const float2 ext = make_float2((bxx.y - bxx.x) / 2.0f, (byy.y - byy.x) / 2.0f);
    const uint32_t gw = static_cast<uint32_t>(vp.glw), gh = static_cast<uint32_t>(vp.glh);
    const float tw = static_cast<float>(kTileLarge);
    b = make_uint4(min(gw, static_cast<uint32_t>(max(0, __float2int_rd((ctr.x - ext.x) / tw)))),
                   min(gw, static_cast<uint32_t>(max(0, __float2int_ru((ctr.x + ext.x) / tw)))),
                   min(gh, static_cast<uint32_t>(max(0, __float2int_rd((ctr.y - ext.y) / tw)))),
                   min(gh, static_cast<uint32_t>(max(0, __float2int_ru((ctr.y + ext.y) / tw)))));
    n = touched_from_bounds(vp, b, vis);
    return n == 0;
}

// ---- bulk-copy (TMA) staging of a block's Gaussian attributes into shared memory ----------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// One contiguous global -> shared copy by the bulk-copy engine, completing on `bar` (no
// multicast: this CTA's own shared memory).  dst, src and bytes are multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Bounded wait for the staging barrier: true when the copies landed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit) {
    for (int k = 0; k < limit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Drain after a late staging: a block must not exit while bulk copies still write into its
// shared memory, so it waits for them, backing off, for up to kStageDrainLimit polls (seconds:
// a copy of under 72 KB that has not landed by then means the memory system has failed, and
// the block gives up so that the kernel still ends).
constexpr int kStageDrainLimit = 1 << 24;
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity) {
    for (int k = 0; k < kStageDrainLimit; ++k) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(256);
    }
    return false;
}

// Bytes of one block's staged attributes (kPrimBlock Gaussians, each array 16-byte padded).
template <typename AttrT, typename ShT>
__host__ __device__ __forceinline__ uint32_t staged_bytes(int total_sh) {
    return kPrimBlock * (12u + 3u * sizeof(AttrT) + 4u * sizeof(AttrT) + sizeof(AttrT) + 3u * sizeof(ShT) +
                         3u * static_cast<uint32_t>(total_sh) * sizeof(ShT));
}
constexpr uint32_t kMaxStagedBytes = 72 * 1024;  // 3 blocks per SM

// AttrT: element type of scales/rotations/opacities; ShT: of sh_0/sh_rest.
// `staged`: full blocks copy their attributes into shared memory with the bulk-copy engine
// (the arrays are contiguous per block: kPrimBlock x {12, 3, 4, 1, 3, 3S} elements) and every
// thread then reads its Gaussian from there; the last partial block, and launches whose arrays
// are not 16-byte aligned, read global memory directly.  Same values either way.
template <typename AttrT, typename ShT, bool STAGED>
__global__ void __launch_bounds__(kPrimBlock, 3) preprocess_kernel(FrameParams fp, FrameBuffers fb, Gaussians g) {
    extern __shared__ __align__(128) unsigned char s_stage[];
    __shared__ uint32_t s_warp[33];
    __shared__ uint64_t s_bar;
    const int i0 = blockIdx.x * kPrimBlock;
    const int i = i0 + threadIdx.x;
    const bool valid = i < fp.n_prims;
    const int ii = valid ? i : 0;
    const float* positions = g.positions;
    const AttrT* scales = reinterpret_cast<const AttrT*>(g.scales);
    const AttrT* rotations = reinterpret_cast<const AttrT*>(g.rotations);
    const AttrT* opacities = reinterpret_cast<const AttrT*>(g.opacities);
    const ShT* sh_0 = reinterpret_cast<const ShT*>(g.sh_0);
    const ShT* sh_rest = reinterpret_cast<const ShT*>(g.sh_rest);
    size_t li = static_cast<size_t>(ii);  // index into the arrays read below
    if (STAGED && i0 + kPrimBlock <= fp.n_prims) {
        const uint32_t S3 = 3u * static_cast<uint32_t>(fp.total_sh);
        const uint32_t b_pos = kPrimBlock * 12u, b_sc = kPrimBlock * 3u * sizeof(AttrT),
                       b_rot = kPrimBlock * 4u * sizeof(AttrT), b_op = kPrimBlock * sizeof(AttrT),
                       b_sh0 = kPrimBlock * 3u * sizeof(ShT), b_shr = kPrimBlock * S3 * sizeof(ShT);
        unsigned char* d_pos = s_stage;
        unsigned char* d_sc = d_pos + b_pos;
        unsigned char* d_rot = d_sc + b_sc;
        unsigned char* d_op = d_rot + b_rot;
        unsigned char* d_sh0 = d_op + b_op;
        unsigned char* d_shr = d_sh0 + b_sh0;
        if (threadIdx.x == 0) mbar_init(&s_bar, 1u);
        __syncthreads();
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(&s_bar, b_pos + b_sc + b_rot + b_op + b_sh0 + b_shr);
            bulk_g2s(d_pos, positions + 3 * static_cast<size_t>(i0), b_pos, &s_bar);
            bulk_g2s(d_sc, scales + 3 * static_cast<size_t>(i0), b_sc, &s_bar);
            bulk_g2s(d_rot, rotations + 4 * static_cast<size_t>(i0), b_rot, &s_bar);
            bulk_g2s(d_op, opacities + static_cast<size_t>(i0), b_op, &s_bar);
            bulk_g2s(d_sh0, sh_0 + 3 * static_cast<size_t>(i0), b_sh0, &s_bar);
            if (b_shr) bulk_g2s(d_shr, sh_rest + static_cast<size_t>(S3) * i0, b_shr, &s_bar);
        }
        const bool late = __syncthreads_or(!mbar_wait_bounded(&s_bar, 0u, fp.stage_wait_limit));
        if (late) {
            // flag the frame (the host reports it as failed and the range stage skips its
            // views), give this block's Gaussians no instances, and drain the copies still in
            // flight before the block exits
            const size_t N = static_cast<size_t>(fp.n_prims);
            for (int v = 0; v < fp.n_views; ++v) {
                const size_t o = static_cast<size_t>(v) * N + i;
                fb.n_touched[o] = 0u;
                fb.n_vis[o] = 0u;
                if (threadIdx.x == 0) {
                    fb.block_sums[static_cast<size_t>(v) * fp.n_blocks_prim + blockIdx.x] = 0u;
                    atomicOr(&fb.status[v].overflow, kFrameErrStaging);
                }
            }
            __syncthreads_or(!mbar_drain(&s_bar, 0u));
            return;
        }
        positions = reinterpret_cast<const float*>(d_pos);
        scales = reinterpret_cast<const AttrT*>(d_sc);
        rotations = reinterpret_cast<const AttrT*>(d_rot);
        opacities = reinterpret_cast<const AttrT*>(d_op);
        sh_0 = reinterpret_cast<const ShT*>(d_sh0);
        sh_rest = reinterpret_cast<const ShT*>(d_shr);
        li = threadIdx.x;
    }
    float3 pos = make_float3(0.f, 0.f, 0.f), scale = pos;
    float4 quat = make_float4(1.f, 0.f, 0.f, 0.f);
    float op = 0.0f;
    if (valid) {
        pos = ld3(positions + 3 * li);
        scale = ld3t(scales + 3 * li);
        quat = ld4t(rotations + 4 * li);
        op = ldf(opacities + li);
    }
    const size_t N = static_cast<size_t>(fp.n_prims);
    for (int v = 0; v < fp.n_views; ++v) {
        const ViewParams& vp = fb.views[v];
        uint32_t n = 0, vis = 0;
        if (valid) {
            float4 P1, P2, P4;
            uint4 b;
            float opacity = op;
            const bool culled = fp.aaa ? transform_and_cull_aaa(vp, fp, pos, scale, quat, opacity, P1, P2, P4, b, n, vis)
                                       : transform_and_cull(vp, fp, pos, scale, quat, opacity, P1, P2, P4, b, n, vis);
            if (culled) n = vis = 0;
            const size_t o = static_cast<size_t>(v) * N + ii;
            fb.n_touched[o] = n;
            fb.n_vis[o] = vis;
            if (!culled) {
                fb.bounds[o] = make_ushort4(static_cast<unsigned short>(b.x), static_cast<unsigned short>(b.y),
                                            static_cast<unsigned short>(b.z), static_cast<unsigned short>(b.w));
                const float3 rgb = sh_to_rgb(sh_0 + 3 * li, sh_rest + static_cast<size_t>(3) * fp.total_sh * li, pos,
                                             xyz(vp.cam), fp.active_sh);
                float4* r = fb.rec + 4 * o;
                r[0] = P1;
                r[1] = P2;
                r[2] = P4;
                r[3] = make_float4(rgb.x, rgb.y, rgb.z, opacity);
            }
        }
        uint32_t tot_vis, tot_ref;
        block_excl_scan<uint32_t>(vis, tot_vis, s_warp);
        block_excl_scan<uint32_t>(n, tot_ref, s_warp);
        if (threadIdx.x == 0) {
            fb.block_sums[static_cast<size_t>(v) * fp.n_blocks_prim + blockIdx.x] = tot_vis;
            atomicAdd(&fb.status[v].n_instances_ref, static_cast<unsigned long long>(tot_ref));
        }
    }
}

// Staging is used by the fast-math flavour only: the IEEE flavour (the reference's _C) keeps
// direct loads, whose compiled arithmetic is the one pinned bit for bit against the reference.
template <typename AttrT, typename ShT>
void launch_preprocess_t(const FrameParams& fp, const FrameBuffers& fb, const Gaussians& g, cudaStream_t s) {
    const uint32_t bytes = staged_bytes<AttrT, ShT>(fp.total_sh);
    auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    const bool staged = kStagedPreprocess && bytes <= kMaxStagedBytes && aligned(g.positions) && aligned(g.scales) &&
                        aligned(g.rotations) && aligned(g.opacities) && aligned(g.sh_0) &&
                        (fp.total_sh == 0 || aligned(g.sh_rest));
    if (!staged) {
        preprocess_kernel<AttrT, ShT, false><<<fp.n_blocks_prim, kPrimBlock, 0, s>>>(fp, fb, g);
        return;
    }
    static bool configured = false;  // per instantiation: allow the staging buffer's size
    if (!configured) {
        cudaFuncSetAttribute(preprocess_kernel<AttrT, ShT, kStagedPreprocess>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kMaxStagedBytes));
        configured = true;
    }
    preprocess_kernel<AttrT, ShT, kStagedPreprocess><<<fp.n_blocks_prim, kPrimBlock, bytes, s>>>(fp, fb, g);
}

int launch_preprocess(const FrameParams& fp, const FrameBuffers& fb, const Gaussians& g, cudaStream_t s) {
    if (fp.n_blocks_prim == 0) return 0;
    if (g.half) launch_preprocess_t<__half, __nv_bfloat16>(fp, fb, g, s);
    else launch_preprocess_t<float, float>(fp, fb, g, s);
    return 1;
}

// ------------------------------------------------------------------------------------------
// scan of block sums -> block prefixes (in place) and M per view
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) scan_blocks_kernel(FrameParams fp, FrameBuffers fb) {
    __shared__ unsigned long long s_warp[33];
    const int v = blockIdx.x;
    uint32_t* bs = fb.block_sums + static_cast<size_t>(v) * fp.n_blocks_prim;
    const int nb = fp.n_blocks_prim;
    unsigned long long carry = 0;
    for (int base = 0; base < nb; base += blockDim.x) {
        const int k = base + threadIdx.x;
        const unsigned long long x = k < nb ? bs[k] : 0ull;
        unsigned long long tot;
        const unsigned long long e = block_excl_scan<unsigned long long>(x, tot, s_warp);
        if (k < nb) bs[k] = static_cast<uint32_t>(carry + e);  // 32-bit offsets, as the reference
        carry += tot;
    }
    if (threadIdx.x == 0) {
        fb.status[v].n_instances = static_cast<uint32_t>(carry);
        // OR: the preprocess may already have flagged a late staging in this word
        fb.status[v].overflow |= static_cast<uint32_t>(carry) > static_cast<unsigned long long>(fp.cap) ? 1u : 0u;
    }
    if (fb.sort_ghist) {  // onesweep sort: digit counts (filled by create) and tile tickets start at 0
        for (int k = threadIdx.x; k < kSortMaxPasses * kSortBins; k += blockDim.x)
            fb.sort_ghist[static_cast<size_t>(v) * kSortMaxPasses * kSortBins + k] = 0u;
        if (threadIdx.x < kSortMaxPasses)
            fb.sort_ticket[v * kSortMaxPasses + threadIdx.x] =
                threadIdx.x == 0 ? static_cast<uint32_t>(fp.look_first_ticket) : 0u;
    }
}

int launch_scan_blocks(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s) {
    scan_blocks_kernel<<<fp.n_views, 1024, 0, s>>>(fp, fb);
    return 1;
}

// ------------------------------------------------------------------------------------------
// instance creation: one (large-tile key, primitive index) pair per visible large tile of a
// primitive's bounds, in row-major bounds order (the emission order of create_instances_cu,
// shared_kernels.cuh:15-130, with the reference's four sub-tile copies of a fovea tile folded
// into one and no sentinel slots: the count per primitive is the visibility-SAT part of the
// reference's touched-tile count)
// ------------------------------------------------------------------------------------------
constexpr uint32_t kSeqTiles = 16;   // bounds tiles handled by the owning thread
constexpr uint32_t kNoPrimitive = 0xFFFFFFFFu;  // value of a sentinel instance slot
constexpr int kBigList = kPrimBlock;

// Stored instances the sort and the later stages see: the count, capped at the capacity.
__device__ __forceinline__ uint64_t view_count(const FrameParams& fp, const FrameBuffers& fb, int v) {
    const unsigned long long m = fb.status[v].n_instances;
    return m < static_cast<unsigned long long>(fp.cap) ? m : static_cast<unsigned long long>(fp.cap);
}

__host__ __device__ __forceinline__ int sort_passes(const FrameParams& fp) {
    return (fp.end_bit + kSortRadixBits - 1) / kSortRadixBits;
}

// Onesweep sort support in the creation kernel: every key written is counted into the block's
// digit histogram of each pass (added to fb.sort_ghist at the end), and the view's look-back
// words of the tiles the sort will use are cleared (the sort runs after this kernel).
__device__ __forceinline__ void count_key(uint32_t* s_hist, int passes, uint32_t key) {
    for (int p = 0; p < passes; ++p) atomicAdd(&s_hist[p * kSortBins + ((key >> (p * kSortRadixBits)) & (kSortBins - 1))], 1u);
}

template <typename KeyT>
__global__ void __launch_bounds__(kPrimBlock) create_instances_kernel(FrameParams fp, FrameBuffers fb) {
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_dhist[kSortMaxPasses * kSortBins];
    __shared__ uint32_t s_big_n;
    __shared__ uint32_t s_big_prim[kBigList];
    __shared__ uint32_t s_big_off[kBigList];
    __shared__ ushort4 s_big_b[kBigList];
    const int v = blockIdx.y;
    const ViewParams& vp = fb.views[v];
    const int i = blockIdx.x * kPrimBlock + threadIdx.x;
    const size_t N = static_cast<size_t>(fp.n_prims);
    const size_t o = static_cast<size_t>(v) * N + i;
    const uint32_t nv = i < fp.n_prims ? fb.n_vis[o] : 0u;
    uint32_t tot;
    const uint32_t local = block_excl_scan<uint32_t>(nv, tot, s_warp);
    const uint32_t off = fb.block_sums[static_cast<size_t>(v) * fp.n_blocks_prim + blockIdx.x] + local;
    const uint64_t lim = static_cast<uint64_t>(fp.cap);
    KeyT* keys = reinterpret_cast<KeyT*>(fb.keys[0]) + static_cast<size_t>(v) * fp.cap;
    uint32_t* vals = fb.vals[0] + static_cast<size_t>(v) * fp.cap;
    const uint32_t glw = static_cast<uint32_t>(vp.glw);
    const bool onesweep = fb.sort_ghist != nullptr;
    const int passes = sort_passes(fp);
    if (threadIdx.x == 0) s_big_n = 0;
    if (onesweep) {
        for (int k = threadIdx.x; k < kSortMaxPasses * kSortBins; k += kPrimBlock) s_dhist[k] = 0u;
        // look-back words of this view's tiles: [pass][tile][digit], tiles of the stored count
        const uint64_t m = view_count(fp, fb, v);
        const uint64_t tile = static_cast<uint64_t>(kSortThreads) * fb.sort_items;
        const uint64_t per_pass = ((m + tile - 1) / tile) * kSortBins;
        const uint64_t pass_stride = static_cast<uint64_t>(fb.sort_tiles) * kSortBins;
        uint32_t* look = fb.sort_look + static_cast<size_t>(v) * kSortMaxPasses * pass_stride;
        for (int p = 0; p < passes; ++p)
            for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * kPrimBlock + threadIdx.x; k < per_pass;
                 k += static_cast<uint64_t>(gridDim.x) * kPrimBlock)
                look[p * pass_stride + k] = 0u;
    }
    __syncthreads();
    if (nv > 0) {
        const ushort4 b = fb.bounds[o];
        const uint32_t bw = static_cast<uint32_t>(b.y - b.x);
        const uint32_t cnt = static_cast<uint32_t>(b.w - b.z) * bw;
        if (cnt <= kSeqTiles) {
            uint64_t w = off;
            const uint64_t end = static_cast<uint64_t>(off) + nv;
            for (uint32_t ty = b.z; ty < b.w && w < end; ++ty) {  // row-major over the bounds
                const uint32_t row = ty * glw;
                for (uint32_t tx = b.x; tx < b.y && w < end; ++tx) {
                    const uint32_t tile = row + tx;
                    if (!tile_visible(vp.vis_mask, tile)) continue;
                    if (w < lim) {
                        keys[w] = static_cast<KeyT>(tile);
                        vals[w] = static_cast<uint32_t>(i);
                        if (onesweep) count_key(s_dhist, passes, tile);
                    }
                    ++w;
                }
            }
            // a visibility area table that counts more tiles than the mask holds leaves slots
            // over: they get sentinels that the range and blend stages skip
            for (; w < end && w < lim; ++w) {
                keys[w] = static_cast<KeyT>(~KeyT(0));
                vals[w] = kNoPrimitive;
                if (onesweep) count_key(s_dhist, passes, static_cast<KeyT>(~KeyT(0)));
            }
        } else {
            const uint32_t slot = atomicAdd(&s_big_n, 1u);
            s_big_prim[slot] = static_cast<uint32_t>(i);
            s_big_off[slot] = off;
            s_big_b[slot] = b;
        }
    }
    __syncthreads();
    // Large bounds: one warp per Gaussian (eight at a time), 32 tiles per step in row-major
    // bounds order, a ballot of the per-tile visibility giving each visible tile its slot; no
    // block barrier, so the warps do not wait for one another's Gaussians.
    const uint32_t n_big = s_big_n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lanemask_lt = (1u << lane) - 1u;
    for (uint32_t q = warp; q < n_big; q += kPrimBlock / 32) {
        const uint32_t prim = s_big_prim[q];
        const ushort4 bb = s_big_b[q];
        const uint32_t bw = static_cast<uint32_t>(bb.y - bb.x);
        const uint32_t cnt = static_cast<uint32_t>(bb.w - bb.z) * bw;
        uint64_t w0 = s_big_off[q];
        const uint64_t end = w0 + fb.n_vis[static_cast<size_t>(v) * N + prim];
        for (uint32_t base = 0; base < cnt; base += 32) {
            const uint32_t k = base + lane;
            uint32_t tile = 0;
            bool c = false;
            if (k < cnt) {
                tile = (bb.z + k / bw) * glw + bb.x + k % bw;
                c = tile_visible(vp.vis_mask, tile);
            }
            const uint32_t vote = __ballot_sync(0xffffffffu, c);
            const uint64_t w = w0 + __popc(vote & lanemask_lt);
            if (c && w < lim && w < end) {
                keys[w] = static_cast<KeyT>(tile);
                vals[w] = prim;
                if (onesweep) count_key(s_dhist, passes, tile);
            }
            w0 += __popc(vote);
        }
        for (uint64_t w = w0 + lane; w < end && w < lim; w += 32) {  // see above
            keys[w] = static_cast<KeyT>(~KeyT(0));
            vals[w] = kNoPrimitive;
            if (onesweep) count_key(s_dhist, passes, static_cast<KeyT>(~KeyT(0)));
        }
    }
    if (onesweep) {
        __syncthreads();
        uint32_t* gh = fb.sort_ghist + static_cast<size_t>(v) * kSortMaxPasses * kSortBins;
        for (int k = threadIdx.x; k < passes * kSortBins; k += kPrimBlock)
            if (s_dhist[k]) atomicAdd(&gh[k], s_dhist[k]);
    }
}

int launch_create(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s) {
    if (fp.n_blocks_prim == 0) return 0;
    dim3 grid(fp.n_blocks_prim, fp.n_views);
    if (fp.key_u32) create_instances_kernel<uint32_t><<<grid, kPrimBlock, 0, s>>>(fp, fb);
    else create_instances_kernel<uint16_t><<<grid, kPrimBlock, 0, s>>>(fp, fb);
    return 1;
}

// ------------------------------------------------------------------------------------------
// stable LSD radix sort of (key, value) pairs per view (replaces cub::DeviceRadixSort::
// SortPairs over bits [0, end_bit), inference.cu:267-274).  Three-kernel form (capacities of
// 2^30 pairs and more, and the no-allocation entry point): digit ranking with __match_any_sync
// per warp; counts per (digit, tile) scanned digit-major; the scatter goes through shared
// memory so that global stores run along digit runs.  Smaller capacities use the onesweep
// pass below.
// ------------------------------------------------------------------------------------------

// Key bits that decide the order in the three-kernel form (FrameParams.sort_key_bits).
__device__ __forceinline__ uint32_t sort_key_mask(const FrameParams& fp) {
    return fp.sort_key_bits > 0 && fp.sort_key_bits < 32 ? (1u << fp.sort_key_bits) - 1u : 0xFFFFFFFFu;
}

template <typename KeyT, int ITEMS>
__global__ void __launch_bounds__(kSortThreads) sort_upsweep_kernel(FrameParams fp, FrameBuffers fb, int buf, int shift) {
    constexpr int TILE = kSortThreads * ITEMS;
    __shared__ uint32_t s_hist[kSortThreads / 32][kSortBins];
    const int v = blockIdx.y;
    const uint64_t M = view_count(fp, fb, v);
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * TILE;
    if (t0 >= M) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < (kSortThreads / 32) * kSortBins; k += kSortThreads) (&s_hist[0][0])[k] = 0;
    __syncthreads();
    const uint32_t n_here = static_cast<uint32_t>(M - t0 < static_cast<uint64_t>(TILE) ? M - t0 : TILE);
    const KeyT* keys = reinterpret_cast<const KeyT*>(fb.keys[buf]) + static_cast<size_t>(v) * fp.cap + t0;
    const uint32_t wbase = static_cast<uint32_t>(warp) * 32 * ITEMS + lane;
    const uint32_t kmask = sort_key_mask(fp);
#pragma unroll 4
    for (int it = 0; it < ITEMS; ++it) {
        const uint32_t idx = wbase + it * 32;
        const bool ok = idx < n_here;
        const uint32_t d = ok ? ((static_cast<uint32_t>(keys[idx]) & kmask) >> shift) & (kSortBins - 1) : kSortBins;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (ok && lane == __ffs(peers) - 1) s_hist[warp][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    const int d = threadIdx.x;  // kSortThreads == kSortBins
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) c += s_hist[w][d];
    fb.sort_hist[(static_cast<size_t>(v) * kSortBins + d) * fb.sort_tiles + blockIdx.x] = c;
}

__global__ void __launch_bounds__(256) sort_scan_kernel(FrameParams fp, FrameBuffers fb) {
    __shared__ uint32_t s_warp[33];
    const int d = blockIdx.x, v = blockIdx.y;
    const uint64_t M = view_count(fp, fb, v);
    const int tile = kSortThreads * fb.sort_items;
    const int ntiles = static_cast<int>((M + tile - 1) / tile);
    uint32_t* row = fb.sort_hist + (static_cast<size_t>(v) * kSortBins + d) * fb.sort_tiles;
    uint32_t carry = 0;
    for (int base = 0; base < ntiles; base += blockDim.x) {
        const int k = base + threadIdx.x;
        const uint32_t x = k < ntiles ? row[k] : 0u;
        uint32_t tot;
        const uint32_t e = block_excl_scan<uint32_t>(x, tot, s_warp);
        if (k < ntiles) row[k] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0) fb.sort_digit_tot[static_cast<size_t>(v) * kSortBins + d] = carry;
}

template <typename KeyT, int ITEMS>
__global__ void __launch_bounds__(kSortThreads, 3) sort_scatter_kernel(FrameParams fp, FrameBuffers fb, int buf, int shift) {
    constexpr int TILE = kSortThreads * ITEMS;
    __shared__ uint32_t s_whist[kSortThreads / 32][kSortBins];  // per-warp counts, then running slots
    __shared__ uint32_t s_local_start[kSortBins];
    __shared__ uint32_t s_global_start[kSortBins];
    __shared__ uint32_t s_warp[33];
    __shared__ KeyT s_keys[TILE];
    __shared__ uint32_t s_vals[TILE];
    const int v = blockIdx.y;
    const uint64_t M = view_count(fp, fb, v);
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * TILE;
    if (t0 >= M) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lanemask_lt = (1u << lane) - 1u;
    for (int k = threadIdx.x; k < (kSortThreads / 32) * kSortBins; k += kSortThreads) (&s_whist[0][0])[k] = 0;
    __syncthreads();
    const uint32_t n_here = static_cast<uint32_t>(M - t0 < static_cast<uint64_t>(TILE) ? M - t0 : TILE);
    const KeyT* keys = reinterpret_cast<const KeyT*>(fb.keys[buf]) + static_cast<size_t>(v) * fp.cap + t0;
    const uint32_t* vals = fb.vals[buf] + static_cast<size_t>(v) * fp.cap + t0;
    KeyT* okeys = reinterpret_cast<KeyT*>(fb.keys[buf ^ 1]) + static_cast<size_t>(v) * fp.cap;
    uint32_t* ovals = fb.vals[buf ^ 1] + static_cast<size_t>(v) * fp.cap;
    // Each warp owns 32 * ITEMS consecutive keys, visited warp-striped (coalesced loads);
    // the visit order is the key order, which makes the ranking stable.
    const uint32_t wbase = static_cast<uint32_t>(warp) * 32 * ITEMS + lane;
    const uint32_t kmask = sort_key_mask(fp);
    KeyT k_reg[ITEMS];
    uint32_t v_reg[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        const uint32_t idx = wbase + it * 32;
        const bool ok = idx < n_here;
        k_reg[it] = ok ? keys[idx] : static_cast<KeyT>(0);
        v_reg[it] = ok ? vals[idx] : 0u;
        const uint32_t d = ok ? ((static_cast<uint32_t>(k_reg[it]) & kmask) >> shift) & (kSortBins - 1) : kSortBins;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (ok && lane == __ffs(peers) - 1) s_whist[warp][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // digit d (thread d): counts of the warps -> exclusive prefix, tile count, starts
    const int d = threadIdx.x;
    uint32_t cnt = 0, wpre[kSortThreads / 32];
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
        wpre[w] = cnt;
        cnt += s_whist[w][d];
    }
    uint32_t tile_total;
    const uint32_t lstart = block_excl_scan<uint32_t>(cnt, tile_total, s_warp);
    s_local_start[d] = lstart;
    const uint32_t dtot = fb.sort_digit_tot[static_cast<size_t>(v) * kSortBins + d];
    uint32_t all_total;
    const uint32_t dbase = block_excl_scan<uint32_t>(dtot, all_total, s_warp);
    s_global_start[d] = dbase + fb.sort_hist[(static_cast<size_t>(v) * kSortBins + d) * fb.sort_tiles + blockIdx.x];
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) s_whist[w][d] = lstart + wpre[w];  // first slot of warp w
    __syncthreads();
    // second visit: stable slot of every key inside the tile
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        const bool ok = wbase + it * 32 < n_here;
        const uint32_t dd = ok ? ((static_cast<uint32_t>(k_reg[it]) & kmask) >> shift) & (kSortBins - 1) : kSortBins;
        const uint32_t peers = __match_any_sync(0xffffffffu, dd);
        const uint32_t base = ok ? s_whist[warp][dd] : 0u;
        __syncwarp();
        if (ok) {
            const uint32_t p = base + __popc(peers & lanemask_lt);
            s_keys[p] = k_reg[it];
            s_vals[p] = v_reg[it];
            if (lane == __ffs(peers) - 1) s_whist[warp][dd] = base + __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < n_here; j += kSortThreads) {
        const KeyT kk = s_keys[j];
        const uint32_t dd = ((static_cast<uint32_t>(kk) & kmask) >> shift) & (kSortBins - 1);
        const uint32_t gpos = s_global_start[dd] + (j - s_local_start[dd]);
        okeys[gpos] = kk;
        ovals[gpos] = s_vals[j];
    }
}

// Onesweep pass (one kernel per 8-bit digit, after Adinets & Merrill, "Onesweep: a faster
// least significant digit radix sort for GPUs", 2022): a block takes the next tile of the view
// from a ticket counter (so every earlier tile belongs to a block that already runs), ranks
// each key within its warp by the lanes holding the same digit (digit_peers: eight ballots;
// stable: warps own consecutive key runs, visited in key order), publishes its digit counts,
// and finds the counts of all earlier tiles by
// decoupled look-back over their published words: flag kLookAggregate = this tile's own
// count, kLookPrefix = the inclusive count of every tile up to it.  The digit's global start
// is the exclusive sum of the pass's digit histogram (filled by the creation kernel).  The
// look-back wait is bounded: a word that stays unpublished for fp.look_spin_limit reads sets
// kFrameErrSortLookback in the frame status and the pass goes on (the host reports the error
// and the range stage skips the view).
constexpr uint32_t kLookAggregate = 1u, kLookPrefix = 2u;
constexpr uint32_t kLookCountMask = (1u << 30) - 1u;

__device__ __forceinline__ uint32_t ld_look(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_look(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Lanes of the warp whose 8-bit digit equals this lane's (the mask __match_any_sync returns),
// from eight ballots over the digit bits; lanes without an item (ok false) match no lane.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, bool ok) {
    uint32_t peers = __ballot_sync(0xffffffffu, ok);
#pragma unroll
    for (int b = 0; b < kSortRadixBits; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t m = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? m : ~m;
    }
    return peers;
}

template <typename KeyT, int ITEMS>
__global__ void __launch_bounds__(kSortThreads, 4) sort_onesweep_kernel(FrameParams fp, FrameBuffers fb, int buf, int pass) {
    constexpr int TILE = kSortThreads * ITEMS;
    static_assert(32 * ITEMS < 65536, "a warp's ranks are packed as 16-bit fields");
    __shared__ uint32_t s_whist[kSortThreads / 32][kSortBins];  // per-warp counts, then warp starts
    __shared__ uint32_t s_local_start[kSortBins];
    __shared__ uint32_t s_global_start[kSortBins];
    __shared__ uint32_t s_warp[33];
    __shared__ uint32_t s_tile, s_err;
    __shared__ KeyT s_keys[TILE];
    __shared__ uint32_t s_vals[TILE];
    const int v = blockIdx.y;
    const int shift = pass * kSortRadixBits;
    const uint64_t M = view_count(fp, fb, v);
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(&fb.sort_ticket[v * kSortMaxPasses + pass], 1u);
        s_err = 0u;
    }
    for (int k = threadIdx.x; k < (kSortThreads / 32) * kSortBins; k += kSortThreads) (&s_whist[0][0])[k] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t t0 = static_cast<uint64_t>(tile) * TILE;
    if (t0 >= M) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lanemask_lt = (1u << lane) - 1u;
    const uint32_t n_here = static_cast<uint32_t>(M - t0 < static_cast<uint64_t>(TILE) ? M - t0 : TILE);
    const KeyT* keys = reinterpret_cast<const KeyT*>(fb.keys[buf]) + static_cast<size_t>(v) * fp.cap + t0;
    const uint32_t* vals = fb.vals[buf] + static_cast<size_t>(v) * fp.cap + t0;
    KeyT* okeys = reinterpret_cast<KeyT*>(fb.keys[buf ^ 1]) + static_cast<size_t>(v) * fp.cap;
    uint32_t* ovals = fb.vals[buf ^ 1] + static_cast<size_t>(v) * fp.cap;
    const uint32_t wbase = static_cast<uint32_t>(warp) * 32 * ITEMS + lane;
    KeyT k_reg[ITEMS];
    uint32_t v_reg[ITEMS];
    // same-digit keys of this warp before the key, two 16-bit ranks per word (a warp ranks at
    // most 32 x ITEMS keys)
    uint32_t rank2[(ITEMS + 1) / 2] = {};
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        const uint32_t idx = wbase + it * 32;
        const bool ok = idx < n_here;
        k_reg[it] = ok ? keys[idx] : static_cast<KeyT>(0);
        v_reg[it] = ok ? vals[idx] : 0u;
    }
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        const bool ok = wbase + it * 32 < n_here;
        const uint32_t d = ok ? (static_cast<uint32_t>(k_reg[it]) >> shift) & (kSortBins - 1) : kSortBins;
        const uint32_t peers = digit_peers(d, ok);
        const uint32_t base = ok ? s_whist[warp][d] : 0u;
        __syncwarp();
        rank2[it >> 1] |= (base + __popc(peers & lanemask_lt)) << (16 * (it & 1));
        if (ok && lane == __ffs(peers) - 1) s_whist[warp][d] = base + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // digit d (thread d): warp starts and the tile's count
    const int d = threadIdx.x;
    uint32_t cnt = 0, wpre[kSortThreads / 32];
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
        wpre[w] = cnt;
        cnt += s_whist[w][d];
    }
    uint32_t tile_total;
    const uint32_t lstart = block_excl_scan<uint32_t>(cnt, tile_total, s_warp);
    // publish this tile's count, then look back over the earlier tiles for this digit
    uint32_t* look = fb.sort_look + (static_cast<size_t>(v) * kSortMaxPasses + pass) * fb.sort_tiles * kSortBins;
    st_look(look + static_cast<size_t>(tile) * kSortBins + d, ((tile == 0 ? kLookPrefix : kLookAggregate) << 30) | cnt);
    uint32_t excl = 0;
    if (tile > 0) {
        int64_t t = static_cast<int64_t>(tile) - 1;
        int spins = 0;
        while (t >= 0) {
            const uint32_t w = ld_look(look + static_cast<size_t>(t) * kSortBins + d);
            const uint32_t flag = w >> 30;
            if (flag == 0u) {
                if (++spins > fp.look_spin_limit) {
                    atomicOr(&fb.status[v].overflow, kFrameErrSortLookback);
                    s_err = 1u;
                    break;
                }
                __nanosleep(32);
                continue;
            }
            excl += w & kLookCountMask;
            if (flag == kLookPrefix) break;
            --t;
        }
        st_look(look + static_cast<size_t>(tile) * kSortBins + d, (kLookPrefix << 30) | ((excl + cnt) & kLookCountMask));
    }
    uint32_t all_total;
    const uint32_t dbase = block_excl_scan<uint32_t>(
        fb.sort_ghist[(static_cast<size_t>(v) * kSortMaxPasses + pass) * kSortBins + d], all_total, s_warp);
    s_local_start[d] = lstart;
    s_global_start[d] = dbase + excl;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) s_whist[w][d] = lstart + wpre[w];  // first slot of warp w
    __syncthreads();
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
        if (wbase + it * 32 < n_here) {
            const uint32_t dd = (static_cast<uint32_t>(k_reg[it]) >> shift) & (kSortBins - 1);
            const uint32_t p = s_whist[warp][dd] + ((rank2[it >> 1] >> (16 * (it & 1))) & 0xffffu);
            s_keys[p] = k_reg[it];
            s_vals[p] = v_reg[it];
        }
    }
    __syncthreads();
    if (s_err) return;  // a look-back gave up: no position of this tile can be trusted
    for (uint32_t j = threadIdx.x; j < n_here; j += kSortThreads) {
        const KeyT kk = s_keys[j];
        const uint32_t dd = (static_cast<uint32_t>(kk) >> shift) & (kSortBins - 1);
        const uint32_t gpos = s_global_start[dd] + (j - s_local_start[dd]);
        if (gpos < M) {
            okeys[gpos] = kk;
            ovals[gpos] = s_vals[j];
        }
    }
}

// fb.sort_tiles must be ceil(cap / (kSortThreads * ITEMS)).
template <typename KeyT, int ITEMS>
int sort_t(const FrameParams& fp, FrameBuffers& fb, cudaStream_t s) {
    if (fb.sort_look) {  // onesweep: one kernel per pass
        const int passes = sort_passes(fp);
        dim3 gt(fb.sort_tiles, fp.n_views);
        int buf = 0;
        for (int p = 0; p < passes; ++p) {
            sort_onesweep_kernel<KeyT, ITEMS><<<gt, kSortThreads, 0, s>>>(fp, fb, buf, p);
            buf ^= 1;
        }
        fb.final_buf = buf;
        return passes;
    }
    const int passes = (fp.end_bit + kSortRadixBits - 1) / kSortRadixBits;
    int buf = 0;
    dim3 gt(fb.sort_tiles, fp.n_views), gd(kSortBins, fp.n_views);
    for (int p = 0; p < passes; ++p) {
        const int shift = p * kSortRadixBits;
        sort_upsweep_kernel<KeyT, ITEMS><<<gt, kSortThreads, 0, s>>>(fp, fb, buf, shift);
        sort_scan_kernel<<<gd, 256, 0, s>>>(fp, fb);
        sort_scatter_kernel<KeyT, ITEMS><<<gt, kSortThreads, 0, s>>>(fp, fb, buf, shift);
        buf ^= 1;
    }
    fb.final_buf = buf;
    return 3 * passes;
}

template <typename KeyT>
int sort_items_t(const FrameParams& fp, FrameBuffers& fb, cudaStream_t s) {
    switch (fb.sort_items) {
        case 8: return sort_t<KeyT, 8>(fp, fb, s);
        case 12: return sort_t<KeyT, 12>(fp, fb, s);
        default: return sort_t<KeyT, 16>(fp, fb, s);
    }
}

int launch_sort(const FrameParams& fp, FrameBuffers& fb, cudaStream_t s) {
    if (fb.sort_tiles == 0) { fb.final_buf = 0; return 0; }
    return fp.key_u32 ? sort_items_t<uint32_t>(fp, fb, s) : sort_items_t<uint16_t>(fp, fb, s);
}

// ------------------------------------------------------------------------------------------
// per-large-tile instance ranges from the boundaries of the sorted keys (the boundary rule of
// extract_instance_ranges_cu, shared_kernels.cuh:133-152; ranges are zeroed beforehand)
// ------------------------------------------------------------------------------------------
// Each thread reads 16 bytes of sorted keys at a time (8 u16 or 4 u32 keys; a view's keys start
// 16-byte aligned: the capacity is a whole number of 4096-key sort tiles) and the key before them.
template <typename KeyT>
__global__ void __launch_bounds__(256) ranges_kernel(FrameParams fp, FrameBuffers fb) {
    constexpr int PER = 16 / static_cast<int>(sizeof(KeyT));
    const int v = blockIdx.y;
    // a view whose sort or staging gave up keeps empty ranges: its sorted values may come from
    // slots that nothing wrote in this frame, and the blend must not read them
    if (fb.status[v].overflow & kFrameErrWait) return;
    const uint64_t M = view_count(fp, fb, v);
    const KeyT* keys = reinterpret_cast<const KeyT*>(fb.keys[fb.final_buf]) + static_cast<size_t>(v) * fp.cap;
    uint2* r = fb.ranges + static_cast<size_t>(v) * fp.max_large;
    const uint32_t n_large = static_cast<uint32_t>(fb.views[v].n_large);
    for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c * PER < M;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t i0 = c * PER;
        KeyT k[PER];
        if (i0 + PER <= M) {
            const uint4 q = *reinterpret_cast<const uint4*>(keys + i0);
            memcpy(k, &q, sizeof(q));
        } else {
#pragma unroll
            for (int j = 0; j < PER; ++j) k[j] = i0 + j < M ? keys[i0 + j] : static_cast<KeyT>(0);
        }
        KeyT prev = i0 > 0 ? keys[i0 - 1] : static_cast<KeyT>(0);
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const uint64_t i = i0 + j;
            if (i >= M) break;
            const KeyT kk = k[j];
            const bool k_ok = static_cast<uint32_t>(kk) < n_large;  // sentinels are no tile
            if (i == 0) {
                if (k_ok) r[kk].x = 0;
            } else if (kk != prev) {
                if (static_cast<uint32_t>(prev) < n_large) r[prev].y = static_cast<uint32_t>(i);
                if (k_ok) r[kk].x = static_cast<uint32_t>(i);
            }
            if (i == M - 1 && k_ok) r[kk].y = static_cast<uint32_t>(M);
            prev = kk;
        }
    }
}

int launch_ranges(const FrameParams& fp, const FrameBuffers& fb, int n_sms, cudaStream_t s) {
    cudaMemsetAsync(fb.ranges, 0, sizeof(uint2) * static_cast<size_t>(fp.max_large) * fp.n_views, s);
    if (fb.sort_tiles == 0) return 0;
    const int64_t per_thread = fp.key_u32 ? 4 : 8;  // keys of one 16-byte load
    const int64_t want = (fp.cap + 256 * per_thread - 1) / (256 * per_thread);
    const unsigned nb = static_cast<unsigned>(want < 8 * n_sms ? (want > 0 ? want : 1) : 8 * n_sms);
    dim3 grid(nb, fp.n_views);
    if (fp.key_u32) ranges_kernel<uint32_t><<<grid, 256, 0, s>>>(fp, fb);
    else ranges_kernel<uint16_t><<<grid, 256, 0, s>>>(fp, fb);
    return 1;
}

// ------------------------------------------------------------------------------------------
// work ordering for the persistent blend (bucketed longest-processing-time first)
// One list holds both kinds of tile: full-resolution (fovea + blended, 8 warps of pixels) and
// periphery (8 x 8 samples at stride 2, 2 warps).  An item is packed as
//   view << 24 | periphery << 23 | index into the view's work_full / work_low list.
// Its cost is (warps x list length); items are bucketed by cost in quarter octaves and the
// buckets are served heaviest first, so that long serial per-pixel chains start early.
// ------------------------------------------------------------------------------------------
constexpr uint32_t kItemLowres = 1u << 23;

__device__ __forceinline__ int items_of_view(const FrameStatus& st) {
    return static_cast<int>(st.n_fovea_large + st.n_blended_large + st.n_periphery_large + st.n_quarter_large);
}

__device__ __forceinline__ int cost_bucket(uint32_t cost) {
    return cost == 0 ? 0 : min(kCostBuckets - 1, 1 + __float2int_rd(4.0f * __log2f(static_cast<float>(cost))));
}

// Maps flat item g to (view, index within the view); `pre` holds the exclusive prefix of the
// per-view item counts.
__device__ __forceinline__ void item_of(int g, const int* pre, int n_views, int& v, int& j) {
    int lo = 0, hi = n_views - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= g) lo = mid; else hi = mid - 1;
    }
    v = lo;
    j = g - pre[lo];
}

// Packed item and cost of the view's j-th item (full-resolution tiles first).
__device__ __forceinline__ uint32_t item_cost(const FrameParams& fp, const FrameBuffers& fb, int v, int j,
                                              uint32_t& packed) {
    const FrameStatus& st = fb.status[v];
    const int n_full = static_cast<int>(st.n_fovea_large + st.n_blended_large);
    const bool low = j >= n_full;
    const int idx = low ? j - n_full : j;
    const uint32_t lt = low ? fb.work_low[static_cast<size_t>(v) * fp.max_large + idx]
                            : fb.work_full[static_cast<size_t>(v) * fp.max_large + idx];
    const uint2 r = fb.ranges[static_cast<size_t>(v) * fp.max_large + lt];
    packed = (static_cast<uint32_t>(v) << 24) | (low ? kItemLowres : 0u) | static_cast<uint32_t>(idx);
    const uint32_t len = r.y > r.x ? r.y - r.x : 0u;
    const bool quarter = low && static_cast<uint32_t>(idx) >= st.n_periphery_large;
    return len * (quarter ? 1u : low ? 2u : 8u);
}

// Work-list bucket of an item: its class (full resolution 2, periphery 1, quarter 0) above its
// cost bucket, so that the descending scatter lists every full-resolution tile first (all 8
// warps of a block busy), then the periphery tiles, then the quarter tiles, each class heaviest
// first; a strided tile then never holds a block that full-resolution work is waiting for.
__device__ __forceinline__ int item_bucket(const FrameParams& fp, const FrameBuffers& fb, int v, int j, uint32_t& packed,
                                           uint32_t& cost) {
    cost = item_cost(fp, fb, v, j, packed);
    const FrameStatus& st = fb.status[v];
    const int n_full = static_cast<int>(st.n_fovea_large + st.n_blended_large);
    const int cls = j < n_full ? 2 : (j - n_full) < static_cast<int>(st.n_periphery_large) ? 1 : 0;
    return cls * kCostBuckets + cost_bucket(cost);
}

// Split blend: the list length above which a full-resolution tile is split, share x the
// frame's instances per blend block (0 when the mode is off).
__device__ __forceinline__ uint32_t split_threshold(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp) {
    if (!(sp.share > 0.0f) || sp.of == nullptr) return 0u;
    uint64_t m = 0;
    for (int v = 0; v < fp.n_views; ++v) m += view_count(fp, fb, v);
    const double t = static_cast<double>(sp.share) * static_cast<double>(m) / static_cast<double>(sp.blocks);
    return t < 256.0 ? 256u : t > 4.0e9 ? 4000000000u : static_cast<uint32_t>(t);
}

// Reserves S consecutive segments for a split tile of `len` list entries (one atomic; in the
// exact mode a second one for the segments' fragment logs).  A reservation that does not fit
// fails and marks the segment slots it reached below the capacity unused.
__device__ __forceinline__ bool split_reserve(const FrameBuffers& fb, const SplitArgs& sp, uint32_t S, uint32_t len,
                                              uint32_t& seg0) {
    seg0 = atomicAdd(&fb.counters[kCtrSplitSegs], S);
    bool ok = seg0 + S <= static_cast<uint32_t>(sp.cap);
    if (ok && sp.exact) {
        const uint32_t units = split_log_units((len + S - 1) / S);
        const unsigned long long want = static_cast<unsigned long long>(units) * S;
        // a 64-bit count (words kCtrSplitPool, +1), so that failed reservations cannot wrap it
        unsigned long long* pool_used = reinterpret_cast<unsigned long long*>(&fb.counters[kCtrSplitPool]);
        const unsigned long long u0 = want <= sp.pool_units ? atomicAdd(pool_used, want) : sp.pool_units;
        ok = want <= sp.pool_units && u0 + want <= sp.pool_units;
        if (ok)
            for (uint32_t k = 0; k < S; ++k) sp.seg_unit[seg0 + k] = static_cast<uint32_t>(u0) + k * units;
    }
    if (ok) return true;
    for (uint32_t k = seg0; k < seg0 + S && k < static_cast<uint32_t>(sp.cap); ++k) sp.list[k] = make_uint2(0u, ~0u);
    return false;
}

constexpr int kMaxOrderViews = 1024;

// Per-view prefix of the item counts into shared memory; returns the total.
__device__ __forceinline__ int items_prefix(const FrameParams& fp, const FrameBuffers& fb, int* pre) {
    __shared__ int s_total;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int v = 0; v < fp.n_views; ++v) {
            pre[v] = acc;
            acc += items_of_view(fb.status[v]);
        }
        s_total = acc;
    }
    __syncthreads();
    return s_total;
}

// Also decides which full-resolution tiles the split blend splits (they leave the work list,
// their segments go to the split list) and clears the split tickets.
__global__ void __launch_bounds__(256) order_hist_kernel(FrameParams fp, FrameBuffers fb, SplitArgs sp) {
    __shared__ int pre[kMaxOrderViews];
    __shared__ uint32_t hist[kOrderBuckets];
    __shared__ uint32_t s_split_len;
    const int total = items_prefix(fp, fb, pre);
    for (int k = threadIdx.x; k < kOrderBuckets; k += blockDim.x) hist[k] = 0;
    if (threadIdx.x == 0) s_split_len = split_threshold(fp, fb, sp);
    __syncthreads();
    const uint32_t split_len = s_split_len;
    if (split_len > 0)
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < sp.cap; k += gridDim.x * blockDim.x) sp.ctl[k] = 0u;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        int v, j;
        item_of(g, pre, fp.n_views, v, j);
        uint32_t packed, cost;
        const int b = item_bucket(fp, fb, v, j, packed, cost);
        if (split_len > 0 && b >= 2 * kCostBuckets) {  // a full-resolution tile: cost = 8 x length
            const uint32_t len = cost / 8u;
            uint32_t tag = ~0u, seg0;
            if (len > split_len) {
                const uint32_t S = min(static_cast<uint32_t>(kSplitMaxSegments), (len + split_len - 1) / split_len);
                if (split_reserve(fb, sp, S, len, seg0)) {
                    tag = seg0 | (S << 28);
                    atomicAdd(&fb.counters[kCtrSplitTiles], 1u);
                    atomicAdd(&fb.counters[kCtrSplitView + v], 1u);
                }
            }
            sp.of[static_cast<size_t>(v) * fp.max_large + j] = tag;
            if (tag != ~0u) continue;
        }
        atomicAdd(&hist[b], 1u);
    }
    __syncthreads();
    uint32_t* gh = fb.counters + kCtrHist;
    for (int k = threadIdx.x; k < kOrderBuckets; k += blockDim.x)
        if (hist[k]) atomicAdd(&gh[k], hist[k]);
}

// Items go to their bucket's run of the work list in rounds of blockDim.x: a block counts its
// round's items per bucket in shared memory (each item's rank among them), reserves one
// contiguous place per bucket with a single global atomic, and writes its items there.  (One
// global atomic per item made the few heavily used buckets' cursors a serial bottleneck.)  The
// order inside a bucket follows the reservations; it changes the schedule, never a pixel.
__global__ void __launch_bounds__(256) order_scatter_kernel(FrameParams fp, FrameBuffers fb, SplitArgs sp) {
    __shared__ int pre[kMaxOrderViews];
    __shared__ uint32_t base[kOrderBuckets];
    __shared__ uint32_t s_cnt[kOrderBuckets];
    __shared__ uint32_t s_warp[33];
    const int total = items_prefix(fp, fb, pre);
    if (sp.status != nullptr && sp.share > 0.0f && blockIdx.x == 0)
        for (int v = threadIdx.x; v < fp.n_views; v += blockDim.x) {
            FrameStatus c = fb.status[v];
            c.n_blended_large -= fb.counters[kCtrSplitView + v];
            sp.status[v] = c;
        }
    const uint32_t* gh = fb.counters + kCtrHist;
    uint32_t* cursor = fb.counters + kCtrHist + kOrderBuckets;
    {  // each bucket's first place in descending bucket order: a block scan, two buckets a thread
        static_assert(kOrderBuckets <= 2 * 256, "two buckets per thread of a 256-thread block");
        const int p0 = 2 * static_cast<int>(threadIdx.x), p1 = p0 + 1;  // places in descending order
        const uint32_t c0 = p0 < kOrderBuckets ? gh[kOrderBuckets - 1 - p0] : 0u;
        const uint32_t c1 = p1 < kOrderBuckets ? gh[kOrderBuckets - 1 - p1] : 0u;
        uint32_t all;
        const uint32_t e = block_excl_scan<uint32_t>(c0 + c1, all, s_warp);
        if (p0 < kOrderBuckets) base[kOrderBuckets - 1 - p0] = e;
        if (p1 < kOrderBuckets) base[kOrderBuckets - 1 - p1] = e + c0;
    }
    uint32_t* out = fb.work_order[0];
    for (int g0 = blockIdx.x * blockDim.x; g0 < total; g0 += gridDim.x * blockDim.x) {
        for (int k = threadIdx.x; k < kOrderBuckets; k += blockDim.x) s_cnt[k] = 0;
        __syncthreads();
        const int g = g0 + static_cast<int>(threadIdx.x);
        int b = -1;
        uint32_t packed = 0, local = 0;
        if (g < total) {
            int v, j;
            item_of(g, pre, fp.n_views, v, j);
            uint32_t cost;
            b = item_bucket(fp, fb, v, j, packed, cost);
            if (sp.of != nullptr && sp.share > 0.0f && b >= 2 * kCostBuckets) {
                const uint32_t tag = sp.of[static_cast<size_t>(v) * fp.max_large + j];
                if (tag != ~0u) {  // a split tile: its segments go to the split list
                    const uint32_t seg0 = tag & 0x0fffffffu, S = tag >> 28;
                    for (uint32_t k = 0; k < S; ++k) sp.list[seg0 + k] = make_uint2(packed, tag);
                    b = -1;
                }
            }
            if (b >= 0) local = atomicAdd(&s_cnt[b], 1u);
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kOrderBuckets; k += blockDim.x)
            if (s_cnt[k]) s_cnt[k] = atomicAdd(&cursor[k], s_cnt[k]);
        __syncthreads();
        if (b >= 0) out[base[b] + s_cnt[b] + local] = packed;
        __syncthreads();  // the counts are cleared for the next round
    }
}

int launch_order(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp, int n_sms, cudaStream_t s) {
    const int per_view = fp.max_large;
    int blocks = (fp.n_views * per_view + 255) / 256;
    blocks = blocks < 2 * n_sms ? (blocks > 0 ? blocks : 1) : 2 * n_sms;
    order_hist_kernel<<<blocks, 256, 0, s>>>(fp, fb, sp);
    order_scatter_kernel<<<blocks, 256, 0, s>>>(fp, fb, sp);
    return 2;
}

// ------------------------------------------------------------------------------------------
// K-buffer blend (restates blend_cu and FragmentInfo, inference.cuh:16-286, and the
// background models, background_model.cuh:8-117).  Per pixel the arithmetic and the order of
// Gaussians are the reference's; a Gaussian is skipped for a whole warp when the warp's pixel
// rectangle lies outside the Gaussian's cutoff ellipse bounding box (+1 px), where every pixel
// would fail the alpha >= 1/255 test anyway.
// ------------------------------------------------------------------------------------------
struct Frag {
    float depth;
    uint32_t color;
};

__device__ __forceinline__ uint32_t pack_channel(const float x) {
    return static_cast<uint32_t>(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f + 0.5f);
}
__device__ __forceinline__ uint32_t pack_rgba(const float4 c) {
    return pack_channel(c.x) | (pack_channel(c.y) << 8) | (pack_channel(c.z) << 16) | (pack_channel(c.w) << 24);
}
__device__ __forceinline__ float4 unpack_rgba(const uint32_t c) {
    return make_float4(static_cast<float>((c >> 0) & 0xff), static_cast<float>((c >> 8) & 0xff),
                       static_cast<float>((c >> 16) & 0xff), static_cast<float>((c >> 24) & 0xff)) * (1.0f / 255.0f);
}

__device__ __forceinline__ float3 background_dir(const ViewParams& vp, float px, float py) {
    const float4 pc = make_float4(px, py, 1.0f, 1.0f);
    return normalize(make_float3(dot(vp.VPR_inv[0], pc), dot(vp.VPR_inv[1], pc), dot(vp.VPR_inv[2], pc)));
}

__device__ float3 eval_sh_background(const ViewParams& vp, const float* __restrict__ c, float px, float py) {
    const float3 t = background_dir(vp, px, py);
    if (t.y > 0.1f) return make_float3(0.0f, 0.0f, 0.0f);
    const float3 n = normalize(t);
    const float x = n.x, y = n.y, z = n.z;
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, xz = x * z, yz = y * z;
    const float3 e = 0.5f + kC0 * ld3(c + 0) - kC1 * y * ld3(c + 3) + kC1 * z * ld3(c + 6) - kC1 * x * ld3(c + 9)
                     + kC2a * xy * ld3(c + 12) - kC2a * yz * ld3(c + 15) + (kC2b * zz - kC2c) * ld3(c + 18)
                     - kC2a * xz * ld3(c + 21) + kC2d * (xx - yy) * ld3(c + 24)
                     + y * (kC3a * yy - kC3b * xx) * ld3(c + 27) + kC3c * xy * z * ld3(c + 30)
                     + y * (kC3d - kC3e * zz) * ld3(c + 33) + z * (kC3f * zz - kC3g) * ld3(c + 36)
                     + x * (kC3d - kC3e * zz) * ld3(c + 39) + kC3h * z * (xx - yy) * ld3(c + 42)
                     + x * (kC3b * yy - kC3a * xx) * ld3(c + 45);
    const float3 col = make_float3(__saturatef(tanhf(e.x) * 0.5f + 0.5f), __saturatef(tanhf(e.y) * 0.5f + 0.5f),
                                   __saturatef(tanhf(e.z) * 0.5f + 0.5f));
    return t.y > 0.0f ? (1.0f - t.y / 0.1f) * col : col;
}

__device__ float3 eval_tex_background(const ViewParams& vp, const float* __restrict__ tex, int W, int H, bool act,
                                      float px, float py) {
    const float3 t = background_dir(vp, px, py);
    if (t.y > 0.1f) return make_float3(0.0f, 0.0f, 0.0f);
    constexpr float kPi = 3.14159265358979323846f;
    const float2 eq = make_float2(atan2f(t.x, t.z) / kPi * 0.5f + 0.5f, asinf(t.y) / (0.5f * kPi) * 0.5f + 0.5f);
    const float tx = eq.x * W - 0.5f;
    const float ty = eq.y * H - 0.5f;
    const int x0 = __float2int_rd(tx), y0 = __float2int_rd(ty);
    const int x1 = x0 + 1, y1 = y0 + 1;
    const float fx = tx - x0, fy = ty - y0;
    const int x0w = x0 < 0 ? x0 + W : x0, x1w = x1 >= W ? x1 - W : x1;
    const int y0c = max(0, min(H - 1, y0)), y1c = max(0, min(H - 1, y1));
    const int i00 = x0w + y0c * W, i10 = x1w + y0c * W, i01 = x0w + y1c * W, i11 = x1w + y1c * W;
    const int nt = W * H;
    float3 col = make_float3(0.0f, 0.0f, 0.0f);
    for (int ch = 0; ch < 3; ++ch) {
        const int off = ch * nt;
        const float c00 = tex[i00 + off], c10 = tex[i10 + off], c01 = tex[i01 + off], c11 = tex[i11 + off];
        const float c0 = c00 * (1.0f - fx) + c10 * fx;
        const float c1 = c01 * (1.0f - fx) + c11 * fx;
        float cc = c0 * (1.0f - fy) + c1 * fy;
        if (act) cc = 1.0f / (1.0f + __expf(-cc));
        if (ch == 0) col.x = cc; else if (ch == 1) col.y = cc; else col.z = cc;
    }
    return t.y > 0.0f ? (1.0f - t.y / 0.1f) * col : col;
}

__device__ __forceinline__ void store_rgb(float* img, int W, int H, int x, int y, bool chw, float r, float g, float b) {
    const int p = W * y + x;
    if (chw) {
        const int n = W * H;
        img[p] = r;
        img[n + p] = g;
        img[2 * n + p] = b;
    } else {
        img[3 * p] = r;
        img[3 * p + 1] = g;
        img[3 * p + 2] = b;
    }
}

// Pixel-space bounding box of a Gaussian's cutoff ellipse, evaluated about the projected
// mean (x0 = P1.w / P4.w) so that no large terms cancel.  Returns false when the box is
// unbounded (camera inside the cutoff quadric or mean behind it): no culling then.
__device__ __forceinline__ bool cutoff_box(const float4 P1, const float4 P2, const float4 P4, float opacity,
                                           float4& box, bool& never) {
    never = false;
    const float rc = 2.0f * __logf(opacity * kMinAlphaRcp);
    if (rc < 0.0f) { never = true; return true; }  // alpha <= opacity < 1/255 everywhere
    if (!(P4.w > 0.0f) || !(rc > 0.0f)) return false;
    const float3 n4 = xyz(P4);
    const float a = P4.w * P4.w - rc * dot(n4, n4);
    if (!(a > 0.0f)) return false;
    const float ia = 1.0f / a;
    const float x0 = P1.w / P4.w, y0 = P2.w / P4.w;
    const float3 q1 = xyz(P1) - x0 * n4, q2 = xyz(P2) - y0 * n4;
    const float cx = -rc * dot(q1, n4) * ia, cy = -rc * dot(q2, n4) * ia;
    const float ex = sqrtf(fmaxf(cx * cx + rc * dot(q1, q1) * ia, 0.0f));
    const float ey = sqrtf(fmaxf(cy * cy + rc * dot(q2, q2) * ia, 0.0f));
    if (!(isfinite(ex) && isfinite(ey) && isfinite(x0) && isfinite(y0))) return false;
    const float mx = 1.0f + 1e-4f * (fabsf(x0) + ex), my = 1.0f + 1e-4f * (fabsf(y0) + ey);
    box = make_float4(x0 + cx - ex - mx, x0 + cx + ex + mx, y0 + cy - ey - my, y0 + cy + ey + my);
    return true;
}

// The cutoff ellipse of a Gaussian as a conic F(x', y') <= 0 about its projected mean
// (x' = x - x0, y' = y - y0).  With Q1 = VPMT1 - x0 VPMT4 and Q2 = VPMT2 - y0 VPMT4 (both with
// zero w) the blend's moment vector is m = w4 (y' q1 - x' q2) and its direction vector
// d = q1 x q2 + x' (q2 x n4) + y' (n4 x q1), so rho^2 <= rc  <=>
//   w4^2 |y' q1 - x' q2|^2 - rc |d|^2 <= 0.
// rc is inflated by kCullRcInflation and the rectangles by kCullPixelMargin, so that a
// rectangle reported empty holds no pixel the blend could accept.  Measured on B200 over 1.8 G
// accepted fragments of five scenes (1M-Gaussian stereo 2064x2208, 100k SH0 1280x720, a camera
// inside a 300k cloud, 20k Gaussians 25x the benchmark size, 4096x1024): evaluated at the
// accepted pixel with rc not inflated, this conic rejects 3,052 of them (float rounding of the
// blend's plane arithmetic); inflated by 0.1 % it rejects none.  0.5 % keeps 5x that margin; the
// 0.02 px covers the rounding of the rectangle edges for sub-pixel ellipses.
constexpr float kCullRcInflation = 1.005f;
constexpr float kCullPixelMargin = 0.02f;

struct Conic {
    float x0, y0, A, B, C, D, E, F0, det;
};

__device__ __forceinline__ bool cutoff_conic(const float4 P1, const float4 P2, const float4 P4, float opacity, Conic& q) {
    const float rc = 2.0f * __logf(opacity * kMinAlphaRcp) * kCullRcInflation;
    const float3 n4 = xyz(P4);
    const float w4 = P4.w;
    if (!(rc > 0.0f) || !(w4 > 0.0f)) return false;
    q.x0 = P1.w / w4;
    q.y0 = P2.w / w4;
    const float3 q1 = xyz(P1) - q.x0 * n4, q2 = xyz(P2) - q.y0 * n4;
    const float3 c0 = cross(q1, q2), cx = cross(q2, n4), cy = cross(n4, q1);
    const float ww = w4 * w4;
    q.A = ww * dot(q2, q2) - rc * dot(cx, cx);
    q.C = ww * dot(q1, q1) - rc * dot(cy, cy);
    q.B = -2.0f * (ww * dot(q1, q2) + rc * dot(cx, cy));
    q.D = -2.0f * rc * dot(c0, cx);
    q.E = -2.0f * rc * dot(c0, cy);
    q.F0 = -rc * dot(c0, c0);
    q.det = 4.0f * q.A * q.C - q.B * q.B;
    // an ellipse, clearly: positive definite quadratic part
    return q.A > 0.0f && q.C > 0.0f && q.det > 1e-4f * (4.0f * q.A * q.C) && isfinite(q.det) && isfinite(q.F0) &&
           isfinite(q.D) && isfinite(q.E) && isfinite(q.x0) && isfinite(q.y0);
}

// Does the ellipse F <= 0 meet the pixel rectangle [ax0, ax1] x [ay0, ay1]?  Minimum of the
// convex F over the rectangle: the free minimum if it lies inside, else the best edge point.
__device__ __forceinline__ bool conic_meets_rect(const Conic& q, float ax0, float ax1, float ay0, float ay1) {
    const float X0 = ax0 - q.x0 - kCullPixelMargin, X1 = ax1 - q.x0 + kCullPixelMargin,
                Y0 = ay0 - q.y0 - kCullPixelMargin, Y1 = ay1 - q.y0 + kCullPixelMargin;
    const float xc = (q.B * q.E - 2.0f * q.C * q.D) / q.det, yc = (q.B * q.D - 2.0f * q.A * q.E) / q.det;
    if (xc >= X0 && xc <= X1 && yc >= Y0 && yc <= Y1) return true;
    auto F = [&](float x, float y) { return (q.A * x + q.B * y + q.D) * x + (q.C * y + q.E) * y + q.F0; };
    const float i2a = 0.5f / q.A, i2c = 0.5f / q.C;
    const float yl = fminf(fmaxf(-(q.B * X0 + q.E) * i2c, Y0), Y1);
    const float yr = fminf(fmaxf(-(q.B * X1 + q.E) * i2c, Y0), Y1);
    const float xt = fminf(fmaxf(-(q.B * Y0 + q.D) * i2a, X0), X1);
    const float xb = fminf(fmaxf(-(q.B * Y1 + q.D) * i2a, X0), X1);
    const float m = fminf(fminf(F(X0, yl), F(X1, yr)), fminf(F(xt, Y0), F(xb, Y1)));
    return !(m > 0.0f);
}

// Shared memory of a blend block: one batch of 256 staged Gaussian records (the three VPMT rows
// and rgba), each Gaussian's warp-culling mask, and each warp's compacted list of batch positions.

struct BlendSmem {
    float4* p1;
    float4* p2;
    float4* p4;
    float4* rgba;
    uint32_t* mask;
    uint8_t (*list)[256];
};

// A segment of a split tile's list (SEG instantiations only).  SEG 1, the records mode: mode 0,
// the whole list, resolved as usual (a split tile blended whole); mode 1, the first segment, whose
// K-buffer, tail and transmittance go to its scratch; mode 2, a later segment, walked from an
// empty K-buffer: every fragment that enters it is recorded (depth, premultiplied colour) instead
// of being blended, and the tail holds only the fragments that never entered it.  SEG 3, the exact
// split: the segment is walked without a K-buffer and every pair is logged (`recs` = the steps a
// warp can take, the log's stride).
struct SegWalk {
    uint32_t s, S;
    int mode;
    int recs;  // SEG 1 mode 2: records kept per pixel; SEG 3: the log's stride in steps
    char* scratch;
};

// Resolves one pixel from its K-buffer, tail and tail transmittance: the split blend's merge
// (the same steps as the end of blend_tile).
template <int K>
__device__ __forceinline__ void blend_resolve(const FrameParams& fp, const ViewParams& vp, const Frag (&core)[K],
                                              const float4 tail, const float tail_T, float pixel_x, float pixel_y,
                                              float* out, int px_i, int py_i) {
    float3 rgb = make_float3(0.0f, 0.0f, 0.0f);
    float Tc = 1.0f;
#pragma unroll
    for (int k = 0; k < K && Tc >= kTransmittanceThreshold; ++k) {
        const float4 c = unpack_rgba(core[k].color);
        rgb += Tc * xyz(c);
        Tc *= 1.0f - c.w;
    }
    if (Tc >= kTransmittanceThreshold && tail.w >= kMinAlpha) {
        const float wt = Tc * (1.0f - tail_T);
        rgb += wt * (1.0f / tail.w) * xyz(tail);
    }
    if (fp.bg_type != 0) {
        const float wb = Tc * tail_T;
        if (wb >= kTransmittanceThreshold) {
            if (fp.bg_type == 1) rgb += wb * eval_sh_background(vp, fp.bg_data, pixel_x, pixel_y);
            else rgb += wb * eval_tex_background(vp, fp.bg_data, fp.tex_w, fp.tex_h, fp.bg_type == 3, pixel_x, pixel_y);
        }
    }
    store_rgb(out, vp.width, vp.height, px_i, py_i, fp.to_chw != 0, __saturatef(rgb.x), __saturatef(rgb.y),
              __saturatef(rgb.z));
}

// Renders one 16x16 work item with the whole 256-thread block: CLS 0 a full-resolution tile with
// its 8 warps (each RW x 32/RW pixels: 8 x 4 laid out 2 x 4, 16 x 2 stacked, or 4 x 8 laid out
// 4 x 2); CLS 1 a periphery tile sampled at stride 2 with warps 0-1 (each min(RW, 8) wide); CLS 2
// a ring-mode quarter tile sampled at stride 4 with lanes 0-15 of warp 0.  The Gaussians of the
// tile's list are staged in shared memory 256 at a time; each thread culls one of them against
// the warp rectangles, and every warp then walks only its own compacted list, in list order.
// The warp shape only changes which pairs are culled (pairs that cannot pass the alpha test),
// never a pixel's arithmetic.  The tile layout is a compile-time constant of each class.
template <int K, int RW, int CLS, int SEG = 0>
__device__ __forceinline__ void blend_tile(const FrameParams& fp, const FrameBuffers& fb, uint32_t packed,
                                        const BlendSmem& sm, const SegWalk sw = SegWalk{0u, 1u, 0, 0, nullptr}) {
    constexpr int NT = 256;
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lanemask_lt = (1u << lane) - 1u;
    const int v = static_cast<int>(packed >> 24);
    const int item = static_cast<int>(packed & (kItemLowres - 1u));
    const ViewParams& vp = fb.views[v];
    const FrameStatus& st = fb.status[v];
    const uint32_t lt = CLS != 0 ? fb.work_low[static_cast<size_t>(v) * fp.max_large + item]
                            : fb.work_full[static_cast<size_t>(v) * fp.max_large + item];
    const bool is_fovea = CLS == 0 && static_cast<uint32_t>(item) < st.n_fovea_large;
    constexpr int S = CLS == 0 ? 1 : CLS == 1 ? kStride : kQuarterStride;
    // warp rectangle rw x rh (powers of two); warps laid out 2^wx_bits per row
    constexpr int RW_LOW = RW > 8 ? 8 : RW;  // the periphery sample grid is 8 wide
    constexpr int RW_BITS = RW == 4 ? 2 : RW == 8 ? 3 : 4, RW_LOW_BITS = RW_LOW == 4 ? 2 : 3;
    constexpr int rw_bits = CLS == 2 ? 2 : CLS == 1 ? RW_LOW_BITS : RW_BITS;
    constexpr int rw = 1 << rw_bits, rh = 32 >> rw_bits;
    constexpr int rh_used = CLS == 2 ? 4 : rh;  // sample rows of a warp that lie in the tile
    constexpr int wx_bits = CLS == 2 ? 0 : (CLS == 1 ? 3 : 4) - rw_bits;
    constexpr int n_warps = CLS == 2 ? 1 : CLS == 1 ? 2 : NW;
    const int ox = static_cast<int>(lt % static_cast<uint32_t>(vp.glw)) * kTileLarge;
    const int oy = static_cast<int>(lt / static_cast<uint32_t>(vp.glw)) * kTileLarge;
    const int lx = (warp & ((1 << wx_bits) - 1)) * rw + (lane & (rw - 1));
    const int ly = (warp >> wx_bits) * rh + (lane >> rw_bits);
    const int px_i = ox + lx * S, py_i = oy + ly * S;
    const bool inside = warp < n_warps && (lane >> rw_bits) < rh_used && px_i < vp.width && py_i < vp.height;
    const float pixel_x = __uint2float_rn(static_cast<uint32_t>(px_i));
    const float pixel_y = __uint2float_rn(static_cast<uint32_t>(py_i));
    uint2 range = fb.ranges[static_cast<size_t>(v) * fp.max_large + lt];
    if constexpr (SEG != 0) {  // segment s of S equal parts of the list
        const uint64_t len = range.y > range.x ? range.y - range.x : 0u;
        const uint32_t lo = range.x + static_cast<uint32_t>(len * sw.s / sw.S);
        const uint32_t hi = range.x + static_cast<uint32_t>(len * (sw.s + 1u) / sw.S);
        range = make_uint2(lo, hi);
    }
    const uint32_t* vals = fb.vals[fb.final_buf] + static_cast<size_t>(v) * fp.cap;
    const float4* rec = fb.rec + 4 * static_cast<size_t>(v) * fp.n_prims;
    uint32_t n_rec = 0;     // SEG mode 2: fragments that entered the K-buffer
    uint32_t n_logged = 0;  // SEG mode 3: steps of this warp logged so far
    constexpr bool log_mode = SEG == 3;  // the exact split's segment: log the fragments only

    float tail_T = 1.0f;
    float4 tail = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    Frag core[K];
#pragma unroll
    for (int k = 0; k < K; ++k) { core[k].depth = 3.402823466e+38f; core[k].color = 0u; }

    for (uint32_t start = range.x; start < range.y; start += NT) {
        const uint32_t n_batch = min(static_cast<uint32_t>(NT), range.y - start);
        __syncthreads();
        if (static_cast<uint32_t>(tid) < n_batch && vals[start + tid] >= static_cast<uint32_t>(fp.n_prims)) {
            sm.mask[tid] = 0u;  // a sentinel slot: no primitive to blend
        } else if (static_cast<uint32_t>(tid) < n_batch) {
            const uint32_t p = vals[start + tid];
            const float4* r = rec + 4 * static_cast<size_t>(p);
            const float4 P1 = r[0], P2 = r[1], P4 = r[2], c = r[3];
            sm.p1[tid] = P1;
            sm.p2[tid] = P2;
            sm.p4[tid] = P4;
            sm.rgba[tid] = c;
            float4 box;
            bool never;
            uint32_t m = (1u << n_warps) - 1u;
            if (cutoff_box(P1, P2, P4, c.w, box, never)) {
                if (never) m = 0u;
                else {
                    Conic q;
                    const bool ell = cutoff_conic(P1, P2, P4, c.w, q);
                    m = 0u;
                    for (int w = 0; w < n_warps; ++w) {
                        const float ax0 = static_cast<float>(ox + (w & ((1 << wx_bits) - 1)) * rw * S);
                        const float ax1 = ax0 + static_cast<float>((rw - 1) * S);
                        const float ay0 = static_cast<float>(oy + (w >> wx_bits) * rh * S);
                        const float ay1 = ay0 + static_cast<float>((rh_used - 1) * S);
                        if (box.y >= ax0 && box.x <= ax1 && box.w >= ay0 && box.z <= ay1 &&
                            (!ell || conic_meets_rect(q, ax0, ax1, ay0, ay1)))
                            m |= 1u << w;
                    }
                }
            }
            sm.mask[tid] = m;
        }
        __syncthreads();
        // this warp's list: the batch positions whose mask has its bit, in order
        int n_mine = 0;
        for (uint32_t c0 = 0; c0 < n_batch; c0 += 32) {
            const uint32_t j = c0 + lane;
            const bool hit = j < n_batch && ((sm.mask[j] >> warp) & 1u);
            const uint32_t b = __ballot_sync(0xffffffffu, hit);
            if (hit) sm.list[warp][n_mine + __popc(b & lanemask_lt)] = static_cast<uint8_t>(j);
            if constexpr (log_mode) {
                if (hit)  // each step's Gaussian colour and opacity
                    reinterpret_cast<float4*>(sw.scratch + 256u * split_log_pos_unit())
                        [static_cast<uint32_t>(warp) * sw.recs + n_logged + n_mine + __popc(b & lanemask_lt)] = sm.rgba[j];
            }
            n_mine += __popc(b);
        }
        __syncwarp();
        uint32_t step0 = 0;
        if constexpr (SEG != 0) {
            step0 = n_logged;
            n_logged += static_cast<uint32_t>(n_mine);
        }
        if (!inside) continue;
        for (int t = 0; t < n_mine; ++t) {
            const int j = sm.list[warp][t];
            const float4 VPMT1 = sm.p1[j], VPMT2 = sm.p2[j], VPMT4 = sm.p4[j];
            const float4 plane_x = VPMT1 - VPMT4 * pixel_x;
            const float4 plane_y = VPMT2 - VPMT4 * pixel_y;
            const float3 nx = xyz(plane_x), ny = xyz(plane_y);
            const float3 m = plane_x.w * ny - nx * plane_y.w;
            const float3 d = cross(nx, ny);
            const float num = dot(m, m);
            const float den = dot(d, d);
            // In almost every warp step some lane passes both tests, so the fragment is
            // evaluated for every lane and the tests only gate its effects (no divergent
            // exits; a lane that failed cannot contribute: its `frag` is false whatever
            // rcp/exp return for it).
            const bool live = !(num > kMaxCutoffSq * den);
            const float den_rcp = 1.0f / den;
            const float G = expf(-0.5f * num * den_rcp);
            const float4 c = sm.rgba[j];
            const float alpha = fminf(c.w * G, kMaxFragmentAlpha);
            const bool frag = live && !(alpha < kMinAlpha);
            float4 pm = make_float4(c.x * alpha, c.y * alpha, c.z * alpha, alpha);
            // the depth matters only to a fragment that may enter the core (alpha >= 1/20):
            // evaluated when some lane of the warp has such a fragment (a warp-uniform branch,
            // so that warps whose fragments are all faint skip it without reconvergence work)
            const bool cand = frag && alpha >= kMinAlphaCore;
            float logged_depth = 0.0f;
            if (__any_sync(__activemask(), cand)) {
                const float3 ep = cross(d, m) * den_rcp;
                const float depth = dot(xyz(VPMT4), ep) + VPMT4.w;
                if constexpr (log_mode) logged_depth = depth;
                if (cand && depth < core[K - 1].depth && !log_mode) {
                    if constexpr (SEG == 1) {
                        if (sw.mode == 2) {  // recorded; the merge decides what it does
                            if (n_rec < static_cast<uint32_t>(sw.recs)) {
                                reinterpret_cast<float*>(sw.scratch + 6 * 4 * NT)[n_rec * NT + tid] = depth;
                                reinterpret_cast<float4*>(sw.scratch + (6 + sw.recs) * 4 * NT)[n_rec * NT + tid] = pm;
                            }
                            ++n_rec;
                        }
                    }
                    Frag f;
                    f.depth = depth;
                    f.color = pack_rgba(pm);
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        if (f.depth < core[k].depth) {
                            const Frag tf = core[k];
                            core[k] = f;
                            f = tf;
                        }
                    }
                    pm = unpack_rgba(f.color);
                    if constexpr (SEG == 1) {
                        if (sw.mode == 2) pm = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // adds nothing below
                    }
                }
            }
            if constexpr (log_mode) {
                {  // the pair's alpha (-1: no fragment) and depth, for the replay
                    reinterpret_cast<float2*>(sw.scratch + 256u * split_log_frag_unit(sw.recs))
                        [(static_cast<uint32_t>(warp) * sw.recs + step0 + t) * 32u + lane] =
                        make_float2(frag ? alpha : -1.0f, logged_depth);
                    continue;
                }
            }
            if (frag) {
                const float pt = 1.0f - pm.w;
                tail += pm;
                tail_T *= pt;
            }
        }
    }
    if constexpr (SEG == 1) {
        if (sw.mode == 1) {
            float* cd = reinterpret_cast<float*>(sw.scratch);
            uint32_t* cc = reinterpret_cast<uint32_t*>(sw.scratch + K * 4 * NT);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                cd[k * NT + tid] = core[k].depth;
                cc[k * NT + tid] = core[k].color;
            }
            reinterpret_cast<float4*>(sw.scratch + 2 * K * 4 * NT)[tid] = tail;
            reinterpret_cast<float*>(sw.scratch + (2 * K + 4) * 4 * NT)[tid] = tail_T;
            return;
        }
        if (sw.mode == 2) {
            reinterpret_cast<uint32_t*>(sw.scratch)[tid] = n_rec;
            reinterpret_cast<float4*>(sw.scratch + 4 * NT)[tid] = tail;
            reinterpret_cast<float*>(sw.scratch + 5 * 4 * NT)[tid] = tail_T;
            return;
        }
    }
    if constexpr (log_mode) {
        if (lane == 0) reinterpret_cast<uint32_t*>(sw.scratch)[warp] = n_logged;
        return;
    }
    if (inside) {
        float3 rgb = make_float3(0.0f, 0.0f, 0.0f);
        float Tc = 1.0f;
#pragma unroll
        for (int k = 0; k < K && Tc >= kTransmittanceThreshold; ++k) {
            const float4 c = unpack_rgba(core[k].color);
            rgb += Tc * xyz(c);
            Tc *= 1.0f - c.w;
        }
        if (Tc >= kTransmittanceThreshold && tail.w >= kMinAlpha) {
            const float wt = Tc * (1.0f - tail_T);
            rgb += wt * (1.0f / tail.w) * xyz(tail);
        }
        if (fp.bg_type != 0) {
            const float wb = Tc * tail_T;
            if (wb >= kTransmittanceThreshold) {
                if (fp.bg_type == 1) rgb += wb * eval_sh_background(vp, fp.bg_data, pixel_x, pixel_y);
                else rgb += wb * eval_tex_background(vp, fp.bg_data, fp.tex_w, fp.tex_h, fp.bg_type == 3, pixel_x, pixel_y);
            }
        }
        float* out = is_fovea ? vp.image : vp.work;
        store_rgb(out, vp.width, vp.height, px_i, py_i, fp.to_chw != 0, __saturatef(rgb.x), __saturatef(rgb.y),
                  __saturatef(rgb.z));
    }
}

// Exact split: the merge.  Each pixel replays, segment by segment and step by step, the
// fragments its warp evaluated, with the walk's own K-buffer insertion and tail accumulation, so
// the operations and their order are those of the serial walk over the whole list.
template <int K, int RW>
__device__ __forceinline__ void split_replay(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp,
                                             uint32_t packed, uint32_t seg0, uint32_t S, uint32_t log_stride) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int v = static_cast<int>(packed >> 24);
    const int item = static_cast<int>(packed & (kItemLowres - 1u));
    const ViewParams& vp = fb.views[v];
    const uint32_t lt = fb.work_full[static_cast<size_t>(v) * fp.max_large + item];
    const bool is_fovea = static_cast<uint32_t>(item) < fb.status[v].n_fovea_large;
    constexpr int rw_bits = RW == 4 ? 2 : RW == 8 ? 3 : 4;
    constexpr int rw = 1 << rw_bits, rh = 32 >> rw_bits;
    constexpr int wx_bits = 4 - rw_bits;
    const int px_i = static_cast<int>(lt % static_cast<uint32_t>(vp.glw)) * kTileLarge + (warp & ((1 << wx_bits) - 1)) * rw + (lane & (rw - 1));
    const int py_i = static_cast<int>(lt / static_cast<uint32_t>(vp.glw)) * kTileLarge + (warp >> wx_bits) * rh + (lane >> rw_bits);
    if (px_i >= vp.width || py_i >= vp.height) return;
    float tail_T = 1.0f;
    float4 tail = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    Frag core[K];
#pragma unroll
    for (int k = 0; k < K; ++k) { core[k].depth = 3.402823466e+38f; core[k].color = 0u; }
    constexpr uint32_t kChunk = 4;  // steps whose log entries are loaded before any is replayed
    for (uint32_t k = 0; k < S; ++k) {
        const char* b = sp.pool + 256ull * sp.seg_unit[seg0 + k];
        const uint32_t n = __ldcg(reinterpret_cast<const uint32_t*>(b) + warp);
        const float4* col = reinterpret_cast<const float4*>(b + 256u * split_log_pos_unit()) +
                            static_cast<size_t>(warp) * log_stride;
        const float2* fr = reinterpret_cast<const float2*>(b + 256u * split_log_frag_unit(log_stride)) +
                           static_cast<size_t>(warp) * log_stride * 32u + lane;
        for (uint32_t t0 = 0; t0 < n; t0 += kChunk) {
            float2 ads[kChunk];
            float4 cs[kChunk];
#pragma unroll
            for (uint32_t i = 0; i < kChunk; ++i) {
                const bool ok = t0 + i < n;
                ads[i] = ok ? __ldcg(fr + (t0 + i) * 32u) : make_float2(-1.0f, 0.0f);
                cs[i] = ok ? __ldcg(col + t0 + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
#pragma unroll
            for (uint32_t i = 0; i < kChunk; ++i) {
            const float2 ad = ads[i];
            if (ad.x < 0.0f) continue;  // not a fragment
            const float alpha = ad.x;
            const float4 c = cs[i];
            float4 pm = make_float4(c.x * alpha, c.y * alpha, c.z * alpha, alpha);
            const bool cand = alpha >= kMinAlphaCore;
            if (cand && ad.y < core[K - 1].depth) {
                Frag f;
                f.depth = ad.y;
                f.color = pack_rgba(pm);
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    if (f.depth < core[q].depth) {
                        const Frag tf = core[q];
                        core[q] = f;
                        f = tf;
                    }
                }
                pm = unpack_rgba(f.color);
            }
            const float pt = 1.0f - pm.w;
            tail += pm;
            tail_T *= pt;
            }
        }
    }
    blend_resolve<K>(fp, vp, core, tail, tail_T, __uint2float_rn(static_cast<uint32_t>(px_i)),
                     __uint2float_rn(static_cast<uint32_t>(py_i)), is_fovea ? vp.image : vp.work, px_i, py_i);
}

// The records mode's segment and merge.  The last of the tile's segments to finish merges them:
// per pixel it starts from the first segment's K-buffer and tail, and replays every later
// segment's records in list order with the K-buffer's own insertion rule.  A fragment that never
// entered its segment's (initially empty) K-buffer can never enter the true one, whose K-th
// depth is never larger, so the replay reproduces every insertion and eviction of the serial
// walk exactly; only the tail sums and the transmittance products are combined in a different
// order.  If some pixel recorded more fragments than the scratch holds, the merging block blends
// the whole tile serially instead.
template <int K, int RW>
__device__ __forceinline__ void blend_split_records(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp,
                                                    uint32_t g, const BlendSmem& sm, uint32_t packed, uint32_t seg0,
                                                    uint32_t S, uint32_t s, size_t stride) {
    constexpr int NT = 256;
    __shared__ int s_last;
    const int tid = threadIdx.x;
    blend_tile<K, RW, 0, 1>(fp, fb, packed, sm, SegWalk{s, S, s == 0 ? 1 : 2, sp.recs, sp.scratch + g * stride});
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(&sp.ctl[seg0], 1u) == S - 1u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const char* base = sp.scratch + seg0 * stride;
    const int R = sp.recs;
    uint32_t most = 0;
    for (uint32_t k = 1; k < S; ++k) most = max(most, __ldcg(reinterpret_cast<const uint32_t*>(base + k * stride) + tid));
    const uint32_t warp_most = __reduce_max_sync(0xffffffffu, most);
    if ((tid & 31) == 0 && warp_most > 0) atomicMax(&fb.counters[kCtrSplitRecMax], warp_most);
    if (__syncthreads_or(most > static_cast<uint32_t>(R))) {
        if (tid == 0) atomicAdd(&fb.counters[kCtrSplitFallback], 1u);
        blend_tile<K, RW, 0, 1>(fp, fb, packed, sm, SegWalk{0u, 1u, 0, 0, nullptr});
        return;
    }
    // this thread's pixel (the full-resolution layout of blend_tile)
    const int lane = tid & 31, warp = tid >> 5;
    const int v = static_cast<int>(packed >> 24);
    const int item = static_cast<int>(packed & (kItemLowres - 1u));
    const ViewParams& vp = fb.views[v];
    const uint32_t lt = fb.work_full[static_cast<size_t>(v) * fp.max_large + item];
    const bool is_fovea = static_cast<uint32_t>(item) < fb.status[v].n_fovea_large;
    constexpr int rw_bits = RW == 4 ? 2 : RW == 8 ? 3 : 4;
    constexpr int rw = 1 << rw_bits, rh = 32 >> rw_bits;
    constexpr int wx_bits = 4 - rw_bits;
    const int px_i = static_cast<int>(lt % static_cast<uint32_t>(vp.glw)) * kTileLarge + (warp & ((1 << wx_bits) - 1)) * rw + (lane & (rw - 1));
    const int py_i = static_cast<int>(lt / static_cast<uint32_t>(vp.glw)) * kTileLarge + (warp >> wx_bits) * rh + (lane >> rw_bits);
    if (px_i >= vp.width || py_i >= vp.height) return;
    Frag core[K];
    const float* cd = reinterpret_cast<const float*>(base);
    const uint32_t* cc = reinterpret_cast<const uint32_t*>(base + K * 4 * NT);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        core[k].depth = __ldcg(cd + k * NT + tid);
        core[k].color = __ldcg(cc + k * NT + tid);
    }
    float4 tail = __ldcg(reinterpret_cast<const float4*>(base + 2 * K * 4 * NT) + tid);
    float tail_T = __ldcg(reinterpret_cast<const float*>(base + (2 * K + 4) * 4 * NT) + tid);
    for (uint32_t k = 1; k < S; ++k) {
        const char* b = base + k * stride;
        const uint32_t n = __ldcg(reinterpret_cast<const uint32_t*>(b) + tid);
        tail += __ldcg(reinterpret_cast<const float4*>(b + 4 * NT) + tid);
        tail_T *= __ldcg(reinterpret_cast<const float*>(b + 5 * 4 * NT) + tid);
        const float* rd = reinterpret_cast<const float*>(b + 6 * 4 * NT);
        const float4* rp = reinterpret_cast<const float4*>(b + (6 + R) * 4 * NT);
#pragma unroll 4
        for (uint32_t r = 0; r < n; ++r) {
            const float depth = __ldcg(rd + r * NT + tid);
            float4 pm = __ldcg(rp + r * NT + tid);
            if (depth < core[K - 1].depth) {
                Frag f;
                f.depth = depth;
                f.color = pack_rgba(pm);
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    if (f.depth < core[q].depth) {
                        const Frag tf = core[q];
                        core[q] = f;
                        f = tf;
                    }
                }
                pm = unpack_rgba(f.color);
            }
            tail += pm;
            tail_T *= 1.0f - pm.w;
        }
    }
    blend_resolve<K>(fp, vp, core, tail, tail_T, __uint2float_rn(static_cast<uint32_t>(px_i)),
                     __uint2float_rn(static_cast<uint32_t>(py_i)), is_fovea ? vp.image : vp.work, px_i, py_i);
}

// One segment of a split full-resolution tile (split list entry g): the exact split's log and
// replay (EXACT), or the records mode's segment and merge.
template <int K, int RW, bool EXACT>
__device__ __forceinline__ void blend_split_segment(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp,
                                                    uint32_t g, const BlendSmem& sm) {
    __shared__ int s_last;
    const int tid = threadIdx.x;
    const uint2 e = sp.list[g];
    if (e.y == ~0u) return;  // a slot of a reservation that did not fit
    const uint32_t packed = e.x, seg0 = e.y & 0x0fffffffu, S = e.y >> 28, s = g - seg0;
    const size_t stride = static_cast<size_t>(sp.stride);
    if constexpr (EXACT) {
        const int v = static_cast<int>(packed >> 24);
        const uint32_t lt = fb.work_full[static_cast<size_t>(v) * fp.max_large + (packed & (kItemLowres - 1u))];
        const uint2 r = fb.ranges[static_cast<size_t>(v) * fp.max_large + lt];
        const uint32_t len = r.y > r.x ? r.y - r.x : 0u;
        const uint32_t log_stride = (len + S - 1u) / S;  // steps a warp of one segment can take
        blend_tile<K, RW, 0, 3>(fp, fb, packed, sm,
                                SegWalk{s, S, 3, static_cast<int>(log_stride), sp.pool + 256ull * sp.seg_unit[g]});
        __threadfence();
        __syncthreads();
        if (tid == 0) s_last = atomicAdd(&sp.ctl[seg0], 1u) == S - 1u;
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        split_replay<K, RW>(fp, fb, sp, packed, seg0, S, log_stride);
        return;
    } else {
        blend_split_records<K, RW>(fp, fb, sp, g, sm, packed, seg0, S, s, stride);
    }
}

// The split segments of a frame, longest lists first, on persistent blocks; it lets the blend of
// the other tiles (launched after it as its programmatic dependent) start at once, so that
// those blocks take the SMs as this kernel's blocks run out of segments.
template <int K, int RW, bool EXACT>
__global__ void __launch_bounds__(256, blend_min_blocks(K)) blend_split_kernel(FrameParams fp, FrameBuffers fb,
                                                                              SplitArgs sp) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    constexpr int NT = 256;
    constexpr int NW = NT / 32;
    __shared__ float4 s_p1[NT], s_p2[NT], s_p4[NT], s_rgba[NT];
    __shared__ uint32_t s_mask[NT];
    __shared__ uint8_t s_list[NW][NT];
    __shared__ int s_item;
    const BlendSmem sm{s_p1, s_p2, s_p4, s_rgba, s_mask, s_list};
    const uint32_t n_seg = min(fb.counters[kCtrSplitSegs], static_cast<uint32_t>(sp.cap));
    for (;;) {
        if (threadIdx.x == 0) s_item = static_cast<int>(atomicAdd(&fb.counters[kCtrSplitNext], 1u));
        __syncthreads();
        const uint32_t g = static_cast<uint32_t>(s_item);
        __syncthreads();
        if (g >= n_seg) break;
        blend_split_segment<K, RW, EXACT>(fp, fb, sp, g, sm);
    }
}

// One persistent kernel blends every tile of every view.  The work list holds the full-resolution
// tiles, then the periphery tiles, then the quarter tiles, each class heaviest first; blocks take
// items class by class, each class with its own compiled tile code.
// SPLIT: launched after blend_split_kernel as its programmatic dependent, with the status whose
// full-resolution counts leave out the split tiles (which the work order left out of its list).
template <int K, int RW, bool SPLIT>
__global__ void __launch_bounds__(256, blend_min_blocks(K)) blend_kernel(FrameParams fp, FrameBuffers fb) {
    constexpr int NT = 256;
    constexpr int NW = NT / 32;
    __shared__ float4 s_p1[NT], s_p2[NT], s_p4[NT], s_rgba[NT];
    __shared__ uint32_t s_mask[NT];
    __shared__ uint8_t s_list[NW][NT];
    __shared__ int s_item;
    const BlendSmem sm{s_p1, s_p2, s_p4, s_rgba, s_mask, s_list};
    const int tid = threadIdx.x;
    int n_full = 0, n_half = 0, n_quarter = 0;
    for (int v = 0; v < fp.n_views; ++v) {
        const FrameStatus& st = fb.status[v];
        n_full += static_cast<int>(st.n_fovea_large + st.n_blended_large);
        n_half += static_cast<int>(st.n_periphery_large);
        n_quarter += static_cast<int>(st.n_quarter_large);
    }
    const uint32_t* order = fb.work_order[0];
    for (;;) {  // full-resolution tiles (listed first)
        if (tid == 0) s_item = static_cast<int>(atomicAdd(&fb.counters[0], 1u));
        __syncthreads();
        const int g = s_item;
        __syncthreads();
        if (g >= n_full) break;
        blend_tile<K, RW, 0>(fp, fb, order[g], sm);
    }
    for (;;) {  // periphery tiles
        if (tid == 0) s_item = static_cast<int>(atomicAdd(&fb.counters[1], 1u));
        __syncthreads();
        const int g = s_item;
        __syncthreads();
        if (g >= n_half) break;
        blend_tile<K, RW, 1>(fp, fb, order[n_full + g], sm);
    }
    for (;;) {  // ring-mode quarter tiles
        if (tid == 0) s_item = static_cast<int>(atomicAdd(&fb.counters[2], 1u));
        __syncthreads();
        const int g = s_item;
        __syncthreads();
        if (g >= n_quarter) break;
        blend_tile<K, RW, 2>(fp, fb, order[n_full + n_half + g], sm);
    }
    // this grid completes only after the split kernel's has
    if constexpr (SPLIT) asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <int K, int RW>
int launch_blend_kr(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp, int n_sms, cudaStream_t s,
                    cudaEvent_t mid) {
    static int occ = -1, occ_split = -1;  // per instantiation, queried once
    if (occ < 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, blend_kernel<K, RW, false>, 256, 0);
    int per_sm = occ > 0 ? occ : 1;
    if (fp.blend_blocks > 0 && fp.blend_blocks < per_sm) per_sm = fp.blend_blocks;
    if (!(sp.share > 0.0f) || sp.of == nullptr) {
        blend_kernel<K, RW, false><<<n_sms * per_sm, 256, 0, s>>>(fp, fb);
        if (mid) cudaEventRecord(mid, s);
        return 1;
    }
    if (occ_split < 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_split, blend_split_kernel<K, RW, false>, 256, 0);
    int per_sm_split = occ_split > 0 ? occ_split : 1;
    if (fp.blend_blocks > 0 && fp.blend_blocks < per_sm_split) per_sm_split = fp.blend_blocks;
    if (sp.exact) blend_split_kernel<K, RW, true><<<n_sms * per_sm_split, 256, 0, s>>>(fp, fb, sp);
    else blend_split_kernel<K, RW, false><<<n_sms * per_sm_split, 256, 0, s>>>(fp, fb, sp);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_sms * per_sm);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FrameBuffers rest = fb;  // the other tiles: the status without the split tiles
    rest.status = sp.status;
    cudaLaunchKernelEx(&cfg, blend_kernel<K, RW, true>, fp, rest);
    if (mid) cudaEventRecord(mid, s);
    return 2;
}

template <int K>
int launch_blend_k(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp, int n_sms, cudaStream_t s,
                   cudaEvent_t mid) {
    switch (fp.blend_rw) {
        case 16: return launch_blend_kr<K, 16>(fp, fb, sp, n_sms, s, mid);
        case 4: return launch_blend_kr<K, 4>(fp, fb, sp, n_sms, s, mid);
        default: return launch_blend_kr<K, 8>(fp, fb, sp, n_sms, s, mid);
    }
}

int launch_blend(const FrameParams& fp, const FrameBuffers& fb, const SplitArgs& sp, int n_sms, cudaStream_t s,
                 cudaEvent_t mid) {
    const int K = fp.K;
    if (K >= 32) return launch_blend_k<32>(fp, fb, sp, n_sms, s, mid);
    if (K >= 16) return launch_blend_k<16>(fp, fb, sp, n_sms, s, mid);
    if (K >= 8) return launch_blend_k<8>(fp, fb, sp, n_sms, s, mid);
    if (K >= 4) return launch_blend_k<4>(fp, fb, sp, n_sms, s, mid);
    if (K >= 2) return launch_blend_k<2>(fp, fb, sp, n_sms, s, mid);
    return launch_blend_k<1>(fp, fb, sp, n_sms, s, mid);
}

// ------------------------------------------------------------------------------------------
// compose: periphery upsampling / blur and blended cross-fade (restates
// bilinear_interpolation, bilinear_interpolation_blended, interpolate_and_blur and
// interpolate_and_blur_blended, interpolation.cuh:11-584), plus clearing of masked tiles.
// One 256-thread block per large tile; blended tiles use four 64-thread groups.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float3 load_rgb(const float* img, int W, int H, int x, int y, bool chw) {
    const int sx = clampi(x, 0, W - 1), sy = clampi(y, 0, H - 1);
    const int p = W * sy + sx;
    if (chw) {
        const int n = W * H;
        return make_float3(img[p], img[n + p], img[2 * n + p]);
    }
    return make_float3(img[3 * p], img[3 * p + 1], img[3 * p + 2]);
}

// Sample (sx, sy) of a stride-2 grid starting at (bx, by); masked-tile samples are clamped
// into the large tile (ltx, lty).  `zero_fovea`: the blend target holds no fovea pixels
// (blur mode), where the reference's zero-initialised temporary buffer reads as 0.
__device__ __forceinline__ float3 grid_sample(const ViewParams& vp, const uint8_t* ltype, const float* src, bool chw,
                                              int bx, int by, int sx, int sy, int max_r, int max_d, int ltx, int lty,
                                              bool zero_fovea) {
    const int px = bx + min(sx, max_r) * kStride;
    const int py = by + min(sy, max_d) * kStride;
    const int tile = py / kTileLarge * vp.glw + px / kTileLarge;
    // a quarter tile (ring mode) holds no stride-2 samples: treated like a masked neighbour
    if ((vp.vis_mask[tile / 32] & (1u << (tile % 32))) == 0 || ltype[tile] == kQuarter) {
        const int cx = clampi(px, ltx * kTileLarge, ltx * kTileLarge + kTileLarge - kStride);
        const int cy = clampi(py, lty * kTileLarge, lty * kTileLarge + kTileLarge - kStride);
        return load_rgb(src, vp.width, vp.height, cx, cy, chw);
    }
    if (zero_fovea) {
        const int qx = clampi(px, 0, vp.width - 1), qy = clampi(py, 0, vp.height - 1);
        if (ltype[(qy / kTileLarge) * vp.glw + qx / kTileLarge] == kFovea) return make_float3(0.0f, 0.0f, 0.0f);
    }
    return load_rgb(src, vp.width, vp.height, px, py, chw);
}

// Sample (sx, sy) of the stride-4 grid of a quarter tile (ring mode) starting at its origin
// (ox, oy): every visible tile holds the stride-4 positions (full, 2x and 4x tiles alike);
// samples in masked tiles are clamped into the tile (ltx, lty), as the periphery grid is.
__device__ __forceinline__ float3 grid_sample4(const ViewParams& vp, const float* src, bool chw, int ox, int oy,
                                               int sx, int sy, int max_r, int max_d, int ltx, int lty) {
    const int px = ox + min(sx, max_r) * kQuarterStride;
    const int py = oy + min(sy, max_d) * kQuarterStride;
    const int tile = py / kTileLarge * vp.glw + px / kTileLarge;
    if ((vp.vis_mask[tile / 32] & (1u << (tile % 32))) == 0) {
        const int cx = clampi(px, ltx * kTileLarge, ltx * kTileLarge + kTileLarge - kQuarterStride);
        const int cy = clampi(py, lty * kTileLarge, lty * kTileLarge + kTileLarge - kQuarterStride);
        return load_rgb(src, vp.width, vp.height, cx, cy, chw);
    }
    return load_rgb(src, vp.width, vp.height, px, py, chw);
}

// Bilinear fill between the samples of an S-strided grid (S = 2: the reference's periphery
// interpolation; S = 4: the ring mode's quarter tiles, same steps).
template <int S = kStride>
__device__ __forceinline__ float3 bilerp(const float3* s, int n, int lx, int ly) {
    const int bx = lx / S, by = ly / S;
    const float xf = static_cast<float>(lx % S) / static_cast<float>(S);
    const float yf = static_cast<float>(ly % S) / static_cast<float>(S);
    float3 r = make_float3(0.0f, 0.0f, 0.0f);
    if (lx % S == 0) {
        r += s[by * n + bx] * (1.0f - yf);
        r += s[(by + 1) * n + bx] * yf;
    } else if (ly % S == 0) {
        r += s[by * n + bx] * (1.0f - xf);
        r += s[by * n + bx + 1] * xf;
    } else {
        r += s[by * n + bx] * (1.0f - xf) * (1.0f - yf);
        r += s[by * n + bx + 1] * xf * (1.0f - yf);
        r += s[(by + 1) * n + bx] * (1.0f - xf) * yf;
        r += s[(by + 1) * n + bx + 1] * xf * yf;
    }
    return r;
}

__device__ __forceinline__ float3 blur5(const float3* s, int n, int lx, int ly, float& factor) {
    const int bx = lx / 2 + 1, by = ly / 2 + 1;
    auto S = [&](int yy, int xx) { return s[yy * n + xx]; };
    float3 r = make_float3(0.0f, 0.0f, 0.0f);
    if ((lx & 1) == 0 && (ly & 1) == 0) {
        factor = 1.0f / 64.0f;
        r += S(by - 1, bx - 1); r += S(by - 1, bx) * 6.0f; r += S(by - 1, bx + 1);
        r += S(by, bx - 1) * 6.0f; r += S(by, bx) * 36.0f; r += S(by, bx + 1) * 6.0f;
        r += S(by + 1, bx - 1); r += S(by + 1, bx) * 6.0f; r += S(by + 1, bx + 1);
    } else if ((lx & 1) == 0 && (ly & 1) == 1) {
        factor = 1.0f / 16.0f;
        r += S(by, bx - 1); r += S(by, bx) * 6.0f; r += S(by, bx + 1);
        r += S(by + 1, bx - 1); r += S(by + 1, bx) * 6.0f; r += S(by + 1, bx + 1);
    } else if ((lx & 1) == 1 && (ly & 1) == 0) {
        factor = 1.0f / 16.0f;
        r += S(by - 1, bx); r += S(by - 1, bx + 1);
        r += S(by, bx) * 6.0f; r += S(by, bx + 1) * 6.0f;
        r += S(by + 1, bx); r += S(by + 1, bx + 1);
    } else {
        factor = 1.0f / 4.0f;
        r += S(by, bx); r += S(by, bx + 1); r += S(by + 1, bx); r += S(by + 1, bx + 1);
    }
    return r;
}

// One 64-thread block per non-fovea large tile; each thread produces 4 of its 256 pixels (or
// one pixel of each of a blended tile's four 8x8 sub-tiles).  Small blocks keep many tiles'
// sample loads in flight per SM: the stage is bound by the latency of those loads.
constexpr int kComposeThreads = 64;

__global__ void __launch_bounds__(kComposeThreads) compose_kernel(FrameParams fp, FrameBuffers fb) {
    __shared__ float3 s_samples[4][10 * 10];
    const int v = blockIdx.y;
    const ViewParams& vp = fb.views[v];
    const FrameStatus& st = fb.status[v];
    const int nP = static_cast<int>(st.n_periphery_large), nB = static_cast<int>(st.n_blended_large),
              nM = static_cast<int>(st.n_masked_large), nQ = static_cast<int>(st.n_quarter_large);
    int item = blockIdx.x;
    if (item >= nP + nQ + nB + nM) return;
    const bool chw = fp.to_chw != 0;
    const bool blur = fp.blur != 0;
    const float* src = vp.work;
    float* dst = vp.image;
    const uint8_t* ltype = fb.large_type + static_cast<size_t>(v) * fp.max_large;
    const int tid = threadIdx.x;
    const int W = vp.width, H = vp.height;
    if (item < nP) {
        const uint32_t lt = fb.work_low[static_cast<size_t>(v) * fp.max_large + item];
        const int ltx = static_cast<int>(lt % static_cast<uint32_t>(vp.glw)), lty = static_cast<int>(lt / static_cast<uint32_t>(vp.glw));
        const int ox = ltx * kTileLarge, oy = lty * kTileLarge;
        const int n = blur ? 10 : 9;
        const int bx = blur ? ox - kStride : ox, by = blur ? oy - kStride : oy;
        const int max_r = static_cast<int>((static_cast<unsigned>(W) - static_cast<unsigned>(bx) - 1u) / static_cast<unsigned>(kStride));
        const int max_d = static_cast<int>((static_cast<unsigned>(H) - static_cast<unsigned>(by) - 1u) / static_cast<unsigned>(kStride));
        float3* s = s_samples[0];
        for (int k = tid; k < n * n; k += kComposeThreads)
            s[k] = grid_sample(vp, ltype, src, chw, bx, by, k % n, k / n, max_r, max_d, ltx, lty, blur);
        __syncthreads();
        for (int q = 0; q < 4; ++q) {
            const int p = tid + kComposeThreads * q;
            const int lx = p & 15, ly = p >> 4;
            const int px = ox + lx, py = oy + ly;
            if (px >= W || py >= H) continue;
            if (!blur) {
                if ((lx % kStride) == 0 && (ly % kStride) == 0) continue;
                const float3 r = bilerp(s, 9, lx, ly);
                store_rgb(dst, W, H, px, py, chw, __saturatef(r.x), __saturatef(r.y), __saturatef(r.z));
            } else {
                float f;
                const float3 r = blur5(s, 10, lx, ly, f);
                store_rgb(dst, W, H, px, py, chw, __saturatef(r.x * f), __saturatef(r.y * f), __saturatef(r.z * f));
            }
        }
        return;
    }
    item -= nP;
    if (item < nQ) {
        // ring mode: 4x-down tile, 5 x 5 samples at stride 4 (its own 4 x 4 and the first
        // row/column of its right and lower neighbours)
        const uint32_t lt = fb.work_low[static_cast<size_t>(v) * fp.max_large + nP + item];
        const int ltx = static_cast<int>(lt % static_cast<uint32_t>(vp.glw)), lty = static_cast<int>(lt / static_cast<uint32_t>(vp.glw));
        const int ox = ltx * kTileLarge, oy = lty * kTileLarge;
        const int max_r = static_cast<int>((static_cast<unsigned>(W) - static_cast<unsigned>(ox) - 1u) / static_cast<unsigned>(kQuarterStride));
        const int max_d = static_cast<int>((static_cast<unsigned>(H) - static_cast<unsigned>(oy) - 1u) / static_cast<unsigned>(kQuarterStride));
        float3* s = s_samples[0];
        if (tid < 25) s[tid] = grid_sample4(vp, src, chw, ox, oy, tid % 5, tid / 5, max_r, max_d, ltx, lty);
        __syncthreads();
        for (int q = 0; q < 4; ++q) {
            const int p = tid + kComposeThreads * q;
            const int lx = p & 15, ly = p >> 4;
            const int px = ox + lx, py = oy + ly;
            if (px >= W || py >= H) continue;
            if ((lx % kQuarterStride) == 0 && (ly % kQuarterStride) == 0) continue;
            const float3 r = bilerp<kQuarterStride>(s, 5, lx, ly);
            store_rgb(dst, W, H, px, py, chw, __saturatef(r.x), __saturatef(r.y), __saturatef(r.z));
        }
        return;
    }
    item -= nQ;
    if (item < nB) {
        const uint32_t lt = fb.work_full[static_cast<size_t>(v) * fp.max_large + st.n_fovea_large + item];
        const int ltx = static_cast<int>(lt % static_cast<uint32_t>(vp.glw)), lty = static_cast<int>(lt / static_cast<uint32_t>(vp.glw));
        const int n = blur ? 6 : 5;
        // the samples of the four 8x8 sub-tiles g (origins (g % 2, g / 2) x 8 in the tile)
        for (int k = tid; k < 4 * n * n; k += kComposeThreads) {
            const int g = k / (n * n), kk = k % (n * n);
            const int ox = ltx * kTileLarge + (g % kStride) * kTileSmall, oy = lty * kTileLarge + (g / kStride) * kTileSmall;
            const int bx = blur ? ox - kStride : ox, by = blur ? oy - kStride : oy;
            const int max_r = static_cast<int>((static_cast<unsigned>(W) - static_cast<unsigned>(bx) - 1u) / static_cast<unsigned>(kStride));
            const int max_d = static_cast<int>((static_cast<unsigned>(H) - static_cast<unsigned>(by) - 1u) / static_cast<unsigned>(kStride));
            s_samples[g][kk] = grid_sample(vp, ltype, src, chw, bx, by, kk % n, kk / n, max_r, max_d, ltx, lty, blur);
        }
        __syncthreads();
        const int lx = tid & 7, ly = tid >> 3;
        for (int g = 0; g < 4; ++g) {
            const int ox = ltx * kTileLarge + (g % kStride) * kTileSmall, oy = lty * kTileLarge + (g / kStride) * kTileSmall;
            const int px = ox + lx, py = oy + ly;
            if (px >= W || py >= H) continue;
            const float3* s = s_samples[g];
            const float2 dg = vp.gaze_px - make_float2(static_cast<float>(px), static_cast<float>(py));
            const float bf = clampf((length(dg) - kBlendRadiusPx - kTileLarge) / (kBlendWidthPx - kTileLarge), 0.0f, 1.0f);
            if (!blur) {
                if ((lx % kStride) == 0 && (ly % kStride) == 0) continue;
                const float3 r = bilerp(s, 5, lx, ly);
                const float3 cc = load_rgb(src, W, H, px, py, chw);
                if (bf > 0.0f)
                    store_rgb(dst, W, H, px, py, chw, __saturatef(r.x * bf + cc.x * (1.0f - bf)),
                              __saturatef(r.y * bf + cc.y * (1.0f - bf)), __saturatef(r.z * bf + cc.z * (1.0f - bf)));
            } else {
                float f;
                const float3 r = blur5(s, 6, lx, ly, f);
                const float3 cc = load_rgb(src, W, H, px, py, chw);
                if (bf > 0.0f)
                    store_rgb(dst, W, H, px, py, chw, __saturatef(cc.x * (1.0f - bf) + r.x * f * bf),
                              __saturatef(cc.y * (1.0f - bf) + r.y * f * bf), __saturatef(cc.z * (1.0f - bf) + r.z * f * bf));
                else
                    store_rgb(dst, W, H, px, py, chw, cc.x, cc.y, cc.z);
            }
        }
        return;
    }
    item -= nB;
    {
        const uint32_t lt = fb.work_masked[static_cast<size_t>(v) * fp.max_large + item];
        const int ox = static_cast<int>(lt % static_cast<uint32_t>(vp.glw)) * kTileLarge;
        const int oy = static_cast<int>(lt / static_cast<uint32_t>(vp.glw)) * kTileLarge;
        for (int q = 0; q < 4; ++q) {
            const int p = tid + kComposeThreads * q;
            const int px = ox + (p & 15), py = oy + (p >> 4);
            if (px < W && py < H) store_rgb(dst, W, H, px, py, chw, 0.0f, 0.0f, 0.0f);
        }
    }
}

int launch_compose(const FrameParams& fp, const FrameBuffers& fb, cudaStream_t s) {
    if (fp.max_large == 0) return 0;
    compose_kernel<<<dim3(fp.max_large, fp.n_views), kComposeThreads, 0, s>>>(fp, fb);
    return 1;
}

const KernelSet& kernel_set() {
    static const KernelSet ks = {launch_setup, launch_classify, launch_preprocess, launch_scan_blocks, launch_create,
                                 launch_sort,  launch_ranges,   launch_order,      launch_blend,       launch_compose};
    return ks;
}

}  // namespace FHTGS_FLAVOR
}  // namespace fhtgs
