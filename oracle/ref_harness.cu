/*
 * Reference harness — TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own CUDA kernels (preprocess_cu, fill_tile_index_num_tiles,
 * build_tile_index_map, get_partition_ranges_cu, create_instances_cu,
 * extract_instance_ranges_cu, included from the reference's headers where they lie) and the
 * same CUB calls, in the order of rasterization/src/inference.cu:74-284, and copies every
 * intermediate to host buffers so the tests can compare them bit for bit with libfhtgs.
 * Built twice by oracle/Makefile: with -use_fast_math (the flags of _C_benchmarking and
 * _C_stereo) and without (the flags of _C).  Output only into oracle/_ref/.
 *
 * Guards that the reference itself lacks, so that no test input can make the harness touch
 * memory out of bounds: no launch for zero primitives or zero active tiles, and the range
 * extraction is skipped when the first sorted key is the sentinel (every slot over-counted).
 */
#include "config.h"
#include "helper_math.h"
#include "utils.h"
#include "kernels/inference.cuh"
#include "kernels/shared_kernels.cuh"
#include "utils/rasterization_utils.h"
#include <cub/cub.cuh>
#include <cstdint>
#include <cstring>
#include <vector>

namespace R = htgs_foveated::rasterization;

extern "C" {

typedef struct {
    const float* positions; const float* scales; const float* rotations; const float* opacities;
    const float* sh_0; const float* sh_rest; int n; int total_sh_bases;
    const float* M; const float* VPM; const float* VPR_inv; const float* cam_position;  /* device */
    float gaze_x, gaze_y;                                                               /* host   */
    const unsigned* visibility_mask; const unsigned* visibility_mask_area_table;
    const unsigned* fovea_mask_area_table;                                              /* device */
    int active_sh_bases, width, height;
    float focal_x, focal_y, center_x, center_y, near_plane, far_plane, scale_modifier;
    int anti_aliasing;
} ref_args;

typedef struct {
    uint32_t* n_touched;       /* [N]   */
    uint16_t* screen_bounds;   /* [N,4] */
    float* vpmt;               /* [N,12] */
    float* rgba;               /* [N,4] */
    uint32_t* offsets;         /* [N] inclusive scan */
    uint32_t* tile_index_map_partitioned; uint8_t* tile_type_partitioned; /* [T] */
    uint32_t* partition_ranges;  /* [6] */
    uint32_t* n_active_tiles;    /* [1] */
    uint32_t* keys_unsorted; uint32_t* values_unsorted; /* [capacity] */
    uint32_t* keys; uint32_t* values;                   /* [capacity] */
    int64_t capacity;
    int64_t* n_instances;        /* [1] */
    uint32_t* instance_ranges;   /* [2*T] */
    int32_t* end_bit;            /* [1] */
} ref_out;

}  // extern "C"

static int check(cudaError_t e) { return e == cudaSuccess ? 0 : static_cast<int>(e); }
#define RK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { return static_cast<int>(e_); } } while (0)

template <typename KeyT>
static int instances_t(const ref_args* a, ref_out* o, int n_instances, int end_bit, uint32_t* d_nt, uint32_t* d_off,
                       ushort4* d_sb, float2 gaze_tiles, int glw, int n_tiles) {
    const int M = n_instances;
    KeyT *k0 = nullptr, *k1 = nullptr;
    uint32_t *v0 = nullptr, *v1 = nullptr;
    uint2* d_ranges = nullptr;
    RK(cudaMalloc(&k0, sizeof(KeyT) * (M + 1)));
    RK(cudaMalloc(&k1, sizeof(KeyT) * (M + 1)));
    RK(cudaMalloc(&v0, sizeof(uint32_t) * (M + 1)));
    RK(cudaMalloc(&v1, sizeof(uint32_t) * (M + 1)));
    RK(cudaMalloc(&d_ranges, sizeof(uint2) * n_tiles));
    RK(cudaMemset(d_ranges, 0, sizeof(uint2) * n_tiles));
    RK(cudaMemset(k0, 255, sizeof(KeyT) * (M + 1)));
    RK(cudaMemset(v0, 255, sizeof(uint32_t) * (M + 1)));
    if (a->n > 0) {
        R::kernels::shared::create_instances_cu<KeyT, config::foveation_radius_tiles, config::num_small_tiles_per_large_tile, 0>
            <<<div_round_up(a->n, config::block_size_create_instances), config::block_size_create_instances>>>(
                d_nt, d_off, d_sb, k0, v0, a->visibility_mask, gaze_tiles, glw, a->n);
        RK(cudaGetLastError());
    }
    const int64_t cnt = M < o->capacity ? M : o->capacity;
    std::vector<KeyT> hk(cnt > 0 ? cnt : 1);
    if (cnt > 0) {
        RK(cudaMemcpy(hk.data(), k0, sizeof(KeyT) * cnt, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < cnt; ++i) o->keys_unsorted[i] = hk[i];
        RK(cudaMemcpy(o->values_unsorted, v0, 4 * cnt, cudaMemcpyDeviceToHost));
    }
    cub::DoubleBuffer<KeyT> keys(k0, k1);
    cub::DoubleBuffer<uint32_t> vals(v0, v1);
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, vals, M, 0, end_bit);
    void* tmp = nullptr;
    RK(cudaMalloc(&tmp, tmp_bytes + 16));
    RK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, vals, M, 0, end_bit));
    if (M > 0) {
        KeyT first;
        RK(cudaMemcpy(&first, keys.Current(), sizeof(KeyT), cudaMemcpyDeviceToHost));
        if (first != static_cast<KeyT>(~KeyT(0))) {
            R::kernels::shared::extract_instance_ranges_cu<KeyT>
                <<<div_round_up(M, config::block_size_extract_instance_ranges), config::block_size_extract_instance_ranges>>>(
                    keys.Current(), d_ranges, M);
            RK(cudaGetLastError());
        }
    }
    RK(cudaDeviceSynchronize());
    if (cnt > 0) {
        RK(cudaMemcpy(hk.data(), keys.Current(), sizeof(KeyT) * cnt, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < cnt; ++i) o->keys[i] = hk[i];
        RK(cudaMemcpy(o->values, vals.Current(), 4 * cnt, cudaMemcpyDeviceToHost));
    }
    RK(cudaMemcpy(o->instance_ranges, d_ranges, sizeof(uint2) * n_tiles, cudaMemcpyDeviceToHost));
    cudaFree(tmp); cudaFree(k0); cudaFree(k1); cudaFree(v0); cudaFree(v1); cudaFree(d_ranges);
    return 0;
}

extern "C" int ref_intermediates(const ref_args* a, ref_out* o) {
    RK(cudaMemcpyToSymbol(c_M, a->M, 3 * sizeof(float4), 0, cudaMemcpyDeviceToDevice));
    RK(cudaMemcpyToSymbol(c_VPM, a->VPM, 4 * sizeof(float4), 0, cudaMemcpyDeviceToDevice));
    RK(cudaMemcpyToSymbol(c_VPR_inv, a->VPR_inv, 4 * sizeof(float4), 0, cudaMemcpyDeviceToDevice));
    RK(cudaMemcpyToSymbol(c_cam_position, a->cam_position, sizeof(float3), 0, cudaMemcpyDeviceToDevice));
    const float2 gz = make_float2(clamp(a->gaze_x, 0.0f, static_cast<float>(a->width - 1)),
                                  clamp(a->gaze_y, 0.0f, static_cast<float>(a->height - 1)));
    RK(cudaMemcpyToSymbol(c_gaze_position_cuda, &gz, sizeof(float2), 0, cudaMemcpyHostToDevice));
    const dim3 gl(div_round_up(a->width, config::tile_width_large), div_round_up(a->height, config::tile_height_large), 1);
    const dim3 g(gl.x * config::tile_stride_x, gl.y * config::tile_stride_y, 1);
    const int n_large = gl.x * gl.y, n_tiles = g.x * g.y;
    const int end_bit = extract_end_bit(n_tiles + 1);
    const int2 gti = make_int2(
        max(0, min(static_cast<int>(g.x - 1), (static_cast<int>(gz.x) + config::tile_width_large / 2) / config::tile_width_large)),
        max(0, min(static_cast<int>(g.y - 1), (static_cast<int>(gz.y) + config::tile_width_large / 2) / config::tile_width_large)));
    const float2 gt = make_float2(static_cast<float>(gti.x), static_cast<float>(gti.y));
    if (o->end_bit) *o->end_bit = end_bit;

    /* tile classification (inference.cu:131-188) */
    uint32_t *d_num = nullptr, *d_toff = nullptr, *d_map = nullptr, *d_map_p = nullptr;
    uint8_t *d_type = nullptr, *d_type_p = nullptr;
    uint2* d_pr = nullptr;
    RK(cudaMalloc(&d_num, 4 * n_large)); RK(cudaMalloc(&d_toff, 4 * n_large));
    RK(cudaMalloc(&d_map, 4 * n_tiles)); RK(cudaMalloc(&d_map_p, 4 * n_tiles));
    RK(cudaMalloc(&d_type, n_tiles)); RK(cudaMalloc(&d_type_p, n_tiles));
    RK(cudaMalloc(&d_pr, sizeof(uint2) * 3)); RK(cudaMemset(d_pr, 0, sizeof(uint2) * 3));
    R::kernels::shared::fill_tile_index_num_tiles<config::foveation_radius_tiles, config::num_small_tiles_per_large_tile, 0>
        <<<div_round_up(n_large, config::block_size_create_tile_index_map), config::block_size_create_tile_index_map>>>(
            d_num, a->visibility_mask, gt, n_large, gl.x);
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, d_num, d_toff, n_large);
    void* t1 = nullptr;
    RK(cudaMalloc(&t1, tb + 16));
    RK(cub::DeviceScan::InclusiveSum(t1, tb, d_num, d_toff, n_large));
    R::kernels::shared::build_tile_index_map<config::num_small_tiles_per_large_tile, config::blend_radius_tiles>
        <<<div_round_up(n_large, config::block_size_create_tile_index_map), config::block_size_create_tile_index_map>>>(
            d_map, reinterpret_cast<R::TileType*>(d_type), d_num, d_toff, gt, gl.x, n_large);
    uint32_t n_active = 0;
    RK(cudaMemcpy(&n_active, d_toff + n_large - 1, 4, cudaMemcpyDeviceToHost));
    if (n_active > 0) {
        size_t tb2 = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb2, d_type, d_type_p, d_map, d_map_p, static_cast<int>(n_active), 0, R::NUM_TILE_TYPE_BITS);
        void* t2 = nullptr;
        RK(cudaMalloc(&t2, tb2 + 16));
        RK(cub::DeviceRadixSort::SortPairs(t2, tb2, d_type, d_type_p, d_map, d_map_p, static_cast<int>(n_active), 0, R::NUM_TILE_TYPE_BITS));
        R::kernels::shared::get_partition_ranges_cu
            <<<div_round_up(static_cast<int>(n_active), config::block_size_get_partition_ranges), config::block_size_get_partition_ranges>>>(
                d_pr, reinterpret_cast<R::TileType*>(d_type_p), n_active);
        RK(cudaDeviceSynchronize());
        cudaFree(t2);
        RK(cudaMemcpy(o->tile_index_map_partitioned, d_map_p, 4 * n_active, cudaMemcpyDeviceToHost));
        RK(cudaMemcpy(o->tile_type_partitioned, d_type_p, n_active, cudaMemcpyDeviceToHost));
    }
    RK(cudaMemcpy(o->partition_ranges, d_pr, sizeof(uint2) * 3, cudaMemcpyDeviceToHost));
    *o->n_active_tiles = n_active;

    /* preprocess + scan (inference.cu:190-236) */
    const int N = a->n;
    uint32_t *d_nt = nullptr, *d_off = nullptr;
    ushort4* d_sb = nullptr;
    float4 *d_v1 = nullptr, *d_v2 = nullptr, *d_v4 = nullptr, *d_rgba = nullptr;
    const size_t nn = N > 0 ? N : 1;
    RK(cudaMalloc(&d_nt, 4 * nn)); RK(cudaMalloc(&d_off, 4 * nn)); RK(cudaMalloc(&d_sb, 8 * nn));
    RK(cudaMalloc(&d_v1, 16 * nn)); RK(cudaMalloc(&d_v2, 16 * nn)); RK(cudaMalloc(&d_v4, 16 * nn)); RK(cudaMalloc(&d_rgba, 16 * nn));
    RK(cudaMemset(d_sb, 0, 8 * nn)); RK(cudaMemset(d_v1, 0, 16 * nn)); RK(cudaMemset(d_v2, 0, 16 * nn));
    RK(cudaMemset(d_v4, 0, 16 * nn)); RK(cudaMemset(d_rgba, 0, 16 * nn));
    int n_instances = 0;
    if (N > 0) {
        const auto pre = a->anti_aliasing ? R::kernels::inference::preprocess_cu<true, 0> : R::kernels::inference::preprocess_cu<false, 0>;
        pre<<<div_round_up(N, config::block_size_preprocess), config::block_size_preprocess>>>(
            reinterpret_cast<const float3*>(a->positions), reinterpret_cast<const float3*>(a->scales),
            reinterpret_cast<const float4*>(a->rotations), a->opacities, reinterpret_cast<const float3*>(a->sh_0),
            reinterpret_cast<const float3*>(a->sh_rest), d_nt, d_sb, d_v1, d_v2, d_v4, d_rgba,
            a->visibility_mask_area_table, a->fovea_mask_area_table, N, gl.x, gl.y, a->active_sh_bases,
            a->total_sh_bases, gti, static_cast<float>(a->width), static_cast<float>(a->height), a->focal_x,
            a->focal_y, a->center_x, a->center_y, a->near_plane, a->far_plane, a->scale_modifier);
        RK(cudaGetLastError());
        size_t tb3 = 0;
        cub::DeviceScan::InclusiveSum(nullptr, tb3, d_nt, d_off, N);
        void* t3 = nullptr;
        RK(cudaMalloc(&t3, tb3 + 16));
        RK(cub::DeviceScan::InclusiveSum(t3, tb3, d_nt, d_off, N));
        RK(cudaDeviceSynchronize());
        cudaFree(t3);
        RK(cudaMemcpy(&n_instances, d_off + N - 1, sizeof(int), cudaMemcpyDeviceToHost));
        RK(cudaMemcpy(o->n_touched, d_nt, 4 * N, cudaMemcpyDeviceToHost));
        RK(cudaMemcpy(o->screen_bounds, d_sb, 8 * N, cudaMemcpyDeviceToHost));
        RK(cudaMemcpy(o->offsets, d_off, 4 * N, cudaMemcpyDeviceToHost));
        std::vector<float4> h1(N), h2(N), h4(N), hc(N);
        RK(cudaMemcpy(h1.data(), d_v1, 16 * N, cudaMemcpyDeviceToHost));
        RK(cudaMemcpy(h2.data(), d_v2, 16 * N, cudaMemcpyDeviceToHost));
        RK(cudaMemcpy(h4.data(), d_v4, 16 * N, cudaMemcpyDeviceToHost));
        RK(cudaMemcpy(hc.data(), d_rgba, 16 * N, cudaMemcpyDeviceToHost));
        for (int i = 0; i < N; ++i) {
            std::memcpy(o->vpmt + 12 * size_t(i), &h1[i], 16);
            std::memcpy(o->vpmt + 12 * size_t(i) + 4, &h2[i], 16);
            std::memcpy(o->vpmt + 12 * size_t(i) + 8, &h4[i], 16);
            std::memcpy(o->rgba + 4 * size_t(i), &hc[i], 16);
        }
    }
    *o->n_instances = n_instances;
    int rc = end_bit <= 16
        ? instances_t<unsigned short>(a, o, n_instances, end_bit, d_nt, d_off, d_sb, gt, gl.x, n_tiles)
        : instances_t<unsigned int>(a, o, n_instances, end_bit, d_nt, d_off, d_sb, gt, gl.x, n_tiles);
    cudaFree(d_num); cudaFree(d_toff); cudaFree(d_map); cudaFree(d_map_p); cudaFree(d_type); cudaFree(d_type_p);
    cudaFree(d_pr); cudaFree(t1); cudaFree(d_nt); cudaFree(d_off); cudaFree(d_sb); cudaFree(d_v1); cudaFree(d_v2);
    cudaFree(d_v4); cudaFree(d_rgba);
    (void)check;
    return rc;
}
