/*
 * CPU oracle for the foveated HTGS forward rasterizer — TEST INFRASTRUCTURE ONLY.
 * See fhtgs_oracle.h.  Each function cites the reference file:line it restates; paths are
 * relative to the reference's FoveatedHTGSCudaBackend/ package directory.
 *
 * The arithmetic follows the reference's expression structure so that the FP32
 * instantiation lands close to the GPU's results; the FP64 instantiation is the accuracy
 * oracle.  Integer outputs that derive from floating point (tile bounds, touched-tile
 * counts) can differ from the GPU's only where a value lies within rounding distance of a
 * tile boundary; the tests account for that with the FP64 margin.
 */
#include "fhtgs_oracle.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <limits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* rasterization/include/config.h:13-45 */
constexpr float kTransmittanceThreshold = 1e-4f;
constexpr float kMaxFragmentAlpha = 1.0f;
constexpr float kMinAlphaRcp = 255.0f;
constexpr float kMinAlpha = 1.0f / kMinAlphaRcp;
constexpr float kMaxCutoffSq = 11.0825270903f;
constexpr float kMinAlphaCore = 1.0f / 20.0f;
constexpr int kTileSmall = 8;
constexpr int kTileLarge = 16;
constexpr int kStride = 2;
constexpr int kSubTiles = 4;
constexpr int kFoveaRadiusTiles = 24;   /* (375 + 15) / 16 */
constexpr int kBlendRadiusTiles = 15;   /* (375 - 125) / 16 */
constexpr int kBlendRadiusPx = 240;     /* 15 * 16 */
constexpr int kBlendWidthPx = 125;

enum TileType : uint8_t { FOVEA = 0, PERIPHERY = 1, BLENDED = 2 };

template <class T> struct V2 { T x, y; };
template <class T> struct V3 { T x, y, z; };
template <class T> struct V4 { T x, y, z, w; };

template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline V3<T> operator+(T s, V3<T> a) { return {s + a.x, s + a.y, s + a.z}; }
template <class T> inline V3<T> operator+(V3<T> a, T s) { return {s + a.x, s + a.y, s + a.z}; }
template <class T> inline V4<T> operator-(V4<T> a, V4<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
template <class T> inline V4<T> operator+(V4<T> a, V4<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class T> inline V4<T> operator*(V4<T> a, V4<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
template <class T> inline V4<T> operator*(V4<T> a, T s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> inline V4<T> operator*(T s, V4<T> a) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline T dot(V4<T> a, V4<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
template <class T> inline V3<T> xyz(V4<T> a) { return {a.x, a.y, a.z}; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline V3<T> normalize(V3<T> v) { T inv = T(1) / std::sqrt(dot(v, v)); return v * inv; }
template <class T> inline T clampT(T x, T lo, T hi) { return std::max(lo, std::min(hi, x)); }
template <class T> inline T saturate(T x) { return std::isnan(x) ? T(0) : clampT(x, T(0), T(1)); }

template <class T> inline V4<T> load4(const float* p) { return {T(p[0]), T(p[1]), T(p[2]), T(p[3])}; }
template <class T> inline V3<T> load3(const float* p) { return {T(p[0]), T(p[1]), T(p[2])}; }

/* __float2int_rd / __float2int_ru semantics: saturating, NaN -> 0. */
template <class T> inline int to_int_rd(T x) {
    if (std::isnan(x)) return 0;
    T f = std::floor(x);
    if (f >= T(INT_MAX)) return INT_MAX;
    if (f <= T(INT_MIN)) return INT_MIN;
    return static_cast<int>(f);
}
template <class T> inline int to_int_ru(T x) {
    if (std::isnan(x)) return 0;
    T f = std::ceil(x);
    if (f >= T(INT_MAX)) return INT_MAX;
    if (f <= T(INT_MIN)) return INT_MIN;
    return static_cast<int>(f);
}

inline bool visible(const uint32_t* mask, uint32_t tile) {
    return (mask[tile / 32u] & (1u << (tile % 32u))) != 0;
}

/* is_in_fovea, kernel_utils.cuh:43-73 (float arithmetic, as on the device). */
inline bool in_fovea(uint32_t tx, uint32_t ty, float gx, float gy, int radius) {
    float dx = (static_cast<float>(tx) + 0.5f) - gx;
    float dy = (static_cast<float>(ty) + 0.5f) - gy;
    return dx * dx + dy * dy < static_cast<float>(radius * radius);
}

struct Geometry {
    int glw, glh;          /* large grid */
    int gw, gh;            /* small grid */
    int n_large, n_tiles;
    int end_bit;
    int gaze_tx, gaze_ty;  /* int gaze tile (clamped to the SMALL grid, inference.cu:98-101) */
    float gaze_px, gaze_py;/* clamped gaze pixels (inference.cu:79-82) */
};

/* extract_end_bit, rasterization_utils.h:50-60 */
int end_bit_of(uint32_t n) { int b = 0; while (n) { ++b; n >>= 1; } return b; }

Geometry geometry(const oracle_view* v) {
    Geometry g;
    g.glw = (v->width + kTileLarge - 1) / kTileLarge;
    g.glh = (v->height + kTileLarge - 1) / kTileLarge;
    g.gw = g.glw * kStride;
    g.gh = g.glh * kStride;
    g.n_large = g.glw * g.glh;
    g.n_tiles = g.gw * g.gh;
    g.end_bit = end_bit_of(static_cast<uint32_t>(g.n_tiles + 1));
    g.gaze_px = std::min(std::max(v->gaze[0], 0.0f), static_cast<float>(v->width - 1));
    g.gaze_py = std::min(std::max(v->gaze[1], 0.0f), static_cast<float>(v->height - 1));
    g.gaze_tx = std::max(0, std::min(g.gw - 1, (static_cast<int>(g.gaze_px) + kTileLarge / 2) / kTileLarge));
    g.gaze_ty = std::max(0, std::min(g.gh - 1, (static_cast<int>(g.gaze_py) + kTileLarge / 2) / kTileLarge));
    return g;
}

/* convert_quaternion_to_rotation_matrix, kernel_utils.cuh:76-88 (no normalisation). */
template <class T> struct Mat3 { T r11, r12, r13, r21, r22, r23, r31, r32, r33; };
template <class T> Mat3<T> quat_to_rot(V4<T> q) {
    T r = q.x, x = q.y, y = q.z, z = q.w;
    T xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
    T rx = r * x, ry = r * y, rz = r * z;
    return {T(1) - T(2) * (yy + zz), T(2) * (xy - rz), T(2) * (xz + ry),
            T(2) * (xy + rz), T(1) - T(2) * (xx + zz), T(2) * (yz - rx),
            T(2) * (xz - ry), T(2) * (yz + rx), T(1) - T(2) * (xx + yy)};
}

/* SH constants and convert_sh_to_color, sh_utils.cuh:8-69 (real SH basis, degree <= 3). */
constexpr double C0 = 0.28209479177387814, C1 = 0.48860251190291987;
constexpr double C2a = 1.0925484305920792, C2b = 0.94617469575755997, C2c = 0.31539156525251999,
                 C2d = 0.54627421529603959;
constexpr double C3a = 0.59004358992664352, C3b = 1.7701307697799304, C3c = 2.8906114426405538,
                 C3d = 0.45704579946446572, C3e = 2.2852289973223288, C3f = 1.865881662950577,
                 C3g = 1.1195289977703462, C3h = 1.4453057213202769;

template <class T> inline T c(double x) { return static_cast<T>(static_cast<float>(x)); }

template <class T>
V3<T> sh_to_rgb(const float* sh0, const float* rest, V3<T> pos, V3<T> cam, int active, int /*total*/) {
    V3<T> res = T(0.5) + c<T>(C0) * load3<T>(sh0);
    if (active > 1) {
        V3<T> d = normalize(pos - cam);
        T x = d.x, y = d.y, z = d.z;
        auto k = [&](int i) { return load3<T>(rest + 3 * i); };
        res = res - c<T>(C1) * y * k(0) + c<T>(C1) * z * k(1) - c<T>(C1) * x * k(2);
        if (active > 4) {
            T xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
            res = res + c<T>(C2a) * xy * k(3) - c<T>(C2a) * yz * k(4) + (c<T>(C2b) * zz - c<T>(C2c)) * k(5)
                      - c<T>(C2a) * xz * k(6) + c<T>(C2d) * (xx - yy) * k(7);
            if (active > 9) {
                res = res + y * (c<T>(C3a) * yy - c<T>(C3b) * xx) * k(8) + c<T>(C3c) * xy * z * k(9)
                          + y * (c<T>(C3d) - c<T>(C3e) * zz) * k(10) + z * (c<T>(C3f) * zz - c<T>(C3g)) * k(11)
                          + x * (c<T>(C3d) - c<T>(C3e) * zz) * k(12) + c<T>(C3h) * z * (xx - yy) * k(13)
                          + x * (c<T>(C3b) * yy - c<T>(C3a) * xx) * k(14);
            }
        }
    }
    return res;
}

template <class T> inline V3<T> operator-(V3<T> a, T s) { return {a.x - s, a.y - s, a.z - s}; }

struct PrimOut {
    uint32_t n_touched = 0;
    uint16_t b[4] = {0, 0, 0, 0};
    float vpmt[12] = {0};
    float rgba[4] = {0};
};

template <class T>
void touched_from_bounds(const oracle_view* v, const Geometry& g, const uint32_t b[4], uint32_t& n) {
    /* kernel_utils.cuh:168-210 */
    const int diam = 2 * kFoveaRadiusTiles;
    const int tlx = g.gaze_tx - kFoveaRadiusTiles, tly = g.gaze_ty - kFoveaRadiusTiles;
    uint32_t fb[4] = {
        static_cast<uint32_t>(std::min(diam, std::max(0, static_cast<int>(b[0]) - tlx))),
        static_cast<uint32_t>(std::min(diam, std::max(0, static_cast<int>(b[1]) - tlx))),
        static_cast<uint32_t>(std::min(diam, std::max(0, static_cast<int>(b[2]) - tly))),
        static_cast<uint32_t>(std::min(diam, std::max(0, static_cast<int>(b[3]) - tly)))};
    const uint32_t W1 = static_cast<uint32_t>(g.glw + 1);
    const uint32_t* sat = v->visibility_mask_area_table;
    n = sat[b[1] + W1 * b[3]] + sat[b[0] + W1 * b[2]] - sat[b[1] + W1 * b[2]] - sat[b[0] + W1 * b[3]];
    if (fb[1] != fb[0] && fb[3] != fb[2]) {
        const uint32_t F1 = diam + 1;
        const uint32_t* f = v->fovea_mask_area_table;
        n += f[fb[1] + F1 * fb[3]] + f[fb[0] + F1 * fb[2]] - f[fb[1] + F1 * fb[2]] - f[fb[0] + F1 * fb[3]];
    }
}

template <class T>
inline uint32_t bound_lo(T x, int grid) { return static_cast<uint32_t>(std::min(grid, std::max(0, to_int_rd<T>(x)))); }
template <class T>
inline uint32_t bound_hi(T x, int grid) { return static_cast<uint32_t>(std::min(grid, std::max(0, to_int_ru<T>(x)))); }

/* transform_and_cull, kernel_utils.cuh:91-213; returns true when culled. */
template <class T>
bool transform_and_cull(const oracle_scene* s, const oracle_view* v, const oracle_settings* st,
                        const Geometry& g, int i, V4<T>& VPMT1, V4<T>& VPMT2, V4<T>& VPMT4,
                        T& opacity, uint32_t b[4], uint32_t& n) {
    V3<T> pos = load3<T>(s->positions + 3 * i);
    V4<T> M3 = load4<T>(v->M + 8);
    T z = dot(xyz(M3), pos) + M3.w;
    if (z < T(v->near_plane) || z > T(v->far_plane)) return true;
    V3<T> sc = load3<T>(s->scales + 3 * i);
    Mat3<T> R = quat_to_rot(load4<T>(s->rotations + 4 * i));
    T sm = T(st->scale_modifier);
    V3<T> u = V3<T>{R.r11 * sc.x, R.r21 * sc.x, R.r31 * sc.x} * sm;
    V3<T> vv = V3<T>{R.r12 * sc.y, R.r22 * sc.y, R.r32 * sc.y} * sm;
    V3<T> w = V3<T>{R.r13 * sc.z, R.r23 * sc.z, R.r33 * sc.z} * sm;
    auto row = [&](int r) { return load4<T>(v->VPM + 4 * r); };
    auto xform = [&](V4<T> P) { return V4<T>{dot(xyz(P), u), dot(xyz(P), vv), dot(xyz(P), w), dot(xyz(P), pos) + P.w}; };
    VPMT4 = xform(row(3));
    T rho_cutoff = T(2) * std::log(opacity * T(kMinAlphaRcp));
    V4<T> d = {rho_cutoff, rho_cutoff, rho_cutoff, T(-1)};
    T ss = dot(d, VPMT4 * VPMT4);
    if (ss == T(0)) return true;
    V4<T> f = (T(1) / ss) * d;
    V4<T> VPMT3 = xform(row(2));
    T cz = dot(f, VPMT3 * VPMT4);
    T ez = std::sqrt(std::max(cz * cz - dot(f, VPMT3 * VPMT3), T(0)));
    if (cz - ez < T(-1) || cz + ez > T(1)) return true;
    VPMT1 = xform(row(0));
    T cx = dot(f, VPMT1 * VPMT4);
    T ex = std::sqrt(std::max(cx * cx - dot(f, VPMT1 * VPMT1), T(0)));
    VPMT2 = xform(row(1));
    T cy = dot(f, VPMT2 * VPMT4);
    T ey = std::sqrt(std::max(cy * cy - dot(f, VPMT2 * VPMT2), T(0)));
    const T tw = T(kTileLarge);
    b[0] = bound_lo<T>((cx - ex + T(0.5)) / tw, g.glw);
    b[1] = bound_hi<T>((cx + ex + T(0.5)) / tw, g.glw);
    b[2] = bound_lo<T>((cy - ey + T(0.5)) / tw, g.glh);
    b[3] = bound_hi<T>((cy + ey + T(0.5)) / tw, g.glh);
    touched_from_bounds<T>(v, g, b, n);
    return n == 0;
}

/* ---- anti-aliased transform ("aaa" mode), kernel_utils_aaa.cuh:9-363 ---- */
template <class T>
T max_contrib_plane(V4<T> plane, V4<T> P1, V4<T> P2, V4<T> P3, V4<T> P4, V4<T>& out) {
    T norm = plane.w / (plane.x * plane.x + plane.y * plane.y + plane.z * plane.z);
    V4<T> mp = (-norm) * plane;
    V3<T> m3 = xyz(mp);
    out = {dot(xyz(P1), m3) + P1.w, dot(xyz(P2), m3) + P2.w, dot(xyz(P3), m3) + P3.w, dot(xyz(P4), m3) + P4.w};
    return -mp.w;
}
template <class T>
T max_contrib_ray(V4<T> a, V4<T> b, V4<T> P1, V4<T> P2, V4<T> P3, V4<T> P4, V4<T>& out) {
    V3<T> d = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    V3<T> m = {a.w * b.x - a.x * b.w, a.w * b.y - a.y * b.w, a.w * b.z - a.z * b.w};
    T dd = dot(d, d);
    V3<T> mdd = {m.x / dd, m.y / dd, m.z / dd};
    V3<T> mp = cross(d, mdd);
    out = {dot(xyz(P1), mp) + P1.w, dot(xyz(P2), mp) + P2.w, dot(xyz(P3), mp) + P3.w, dot(xyz(P4), mp) + P4.w};
    return dot(m, mdd);
}
template <class T> inline bool in_range(T p, T from, T ext, T ph) { T d = p - from * ph; return d > T(0) && d < ext * ph; }
template <class T>
T max_contrib_frustum(V4<T> P1, V4<T> P2, V4<T> P3, V4<T> P4, T width, T height) {
    T best = std::numeric_limits<float>::max();
    const V3<T> from = {T(0), T(0), T(-1)};
    const V3<T> ext = {width - T(1), height - T(1), T(2)};
    V3<T> d = {P1.w - from.x * P4.w, P2.w - from.y * P4.w, P3.w - from.z * P4.w};
    bool bx = d.x > T(0) && d.x < ext.x * P4.w;
    bool by = d.y > T(0) && d.y < ext.y * P4.w;
    bool bz = d.z > T(0) && d.z < ext.z * P4.w;
    if (bx && by && bz) return T(0);
    T dx = std::copysign(ext.x * T(0.5), d.x - (ext.x * T(0.5) * P4.w));
    T dy = std::copysign(ext.y * T(0.5), d.y - (ext.y * T(0.5) * P4.w));
    V4<T> cpx = P1 - P4 * (from.x + ext.x * T(0.5) + dx);
    V4<T> cpy = P2 - P4 * (from.y + ext.y * T(0.5) + dy);
    V4<T> ps;
    T cval = max_contrib_plane(cpx, P1, P2, P3, P4, ps);
    if (cval < best && in_range(ps.y, from.y, ext.y, ps.w) && in_range(ps.z, from.z, ext.z, ps.w)) best = cval;
    cval = max_contrib_plane(cpy, P1, P2, P3, P4, ps);
    if (cval < best && in_range(ps.x, from.x, ext.x, ps.w) && in_range(ps.z, from.z, ext.z, ps.w)) best = cval;
    cval = max_contrib_ray(cpx, cpy, P1, P2, P3, P4, ps);
    if (cval < best && in_range(ps.z, from.z, ext.z, ps.w)) best = cval;
    V4<T> opy = P2 - P4 * (from.y + ext.y * T(0.5) - dy);
    cval = max_contrib_ray(cpx, opy, P1, P2, P3, P4, ps);
    if (cval < best && in_range(ps.z, from.z, ext.z, ps.w)) best = cval;
    V4<T> opx = P1 - P4 * (from.x + ext.x * T(0.5) - dx);
    cval = max_contrib_ray(opx, cpy, P1, P2, P3, P4, ps);
    if (cval < best && in_range(ps.z, from.z, ext.z, ps.w)) best = cval;
    return best;
}
template <class T> T normalize_angle(T th) {
    const T pi = T(3.141592654f), two_pi = T(2) * pi;
    th = std::fmod(th, two_pi);
    if (th > pi) th -= two_pi;
    if (th <= -pi) th += two_pi;
    return th;
}
template <class T>
void aabb_view(V4<T> MT1, V4<T> MT2, V4<T> MT3, T fx, T fy, T cxp, T cyp, T cutoff, V2<T>& center, V2<T>& extent) {
    const T pi = T(3.141592654f), two_pi = T(2) * pi;
    const T max_theta = T(0.5) * pi - T(1e-5f);
    V4<T> t = {cutoff, cutoff, cutoff, T(-1)};
    V3<T> viewdir = normalize(V3<T>{MT1.w, MT2.w, MT3.w});
    auto theta = [&](int axis) {
        bool is_x = axis == 0;
        T theta_mu = std::atan2(is_x ? viewdir.x : viewdir.y, viewdir.z);
        V4<T> MA = is_x ? MT1 : MT2;
        T sq_axis = dot(t, MA * MA), sq_z = dot(t, MT3 * MT3), mid = dot(t, MA * MT3);
        T inside = mid * mid - sq_z * sq_axis;
        V2<T> r = {-max_theta, max_theta};
        if (inside > T(0)) {
            V2<T> th = {std::atan2(-(mid + std::sqrt(inside)), -sq_z), std::atan2(-(mid - std::sqrt(inside)), -sq_z)};
            while (th.x > theta_mu) th.x -= pi;
            while (th.x < (theta_mu - pi)) th.x += pi;
            while (th.y < theta_mu) th.y += pi;
            while (th.y > (theta_mu + pi)) th.y -= pi;
            V2<T> tn = {normalize_angle(th.x), normalize_angle(th.y)};
            if (theta_mu < T(0) && std::fabs(tn.x) < std::fabs(tn.y)) { th.x += two_pi; th.y += two_pi; }
            else if (theta_mu > T(0) && std::fabs(tn.y) < std::fabs(tn.x)) { th.x -= two_pi; th.y -= two_pi; }
            r = {std::max(r.x, th.x), std::min(r.y, th.y)};
        }
        return V2<T>{std::tan(r.x), std::tan(r.y)};
    };
    V2<T> tx = theta(0), ty = theta(1);
    V2<T> bx = {cxp + fx * tx.x, cxp + fx * tx.y};
    V2<T> by = {cyp + fy * ty.x, cyp + fy * ty.y};
    center = {(bx.y + bx.x) / T(2), (by.y + by.x) / T(2)};
    extent = {(bx.y - bx.x) / T(2), (by.y - by.x) / T(2)};
}

template <class T>
bool transform_and_cull_aaa(const oracle_scene* s, const oracle_view* v, const oracle_settings* st,
                            const Geometry& g, int i, V4<T>& VPMT1, V4<T>& VPMT2, V4<T>& VPMT4,
                            T& opacity, uint32_t b[4], uint32_t& n) {
    V3<T> pos = load3<T>(s->positions + 3 * i);
    V3<T> osc = load3<T>(s->scales + 3 * i);
    Mat3<T> R = quat_to_rot(load4<T>(s->rotations + 4 * i));
    V4<T> M3 = load4<T>(v->M + 8);
    T z = dot(xyz(M3), pos) + M3.w;
    const T kernel = T(0.3f);
    T max_focal = std::max(T(v->focal_x), T(v->focal_y));
    T fsv = z / max_focal;
    T fvar = fsv * fsv * kernel;
    V3<T> ovar = osc * osc;
    V3<T> var = ovar + fvar;
    V3<T> sc = {std::sqrt(var.x), std::sqrt(var.y), std::sqrt(var.z)};
    V3<T> cam = load3<T>(v->cam_position);
    V3<T> vdw = normalize(pos - cam);
    V3<T> vdg = {R.r11 * vdw.x + R.r21 * vdw.y + R.r31 * vdw.z, R.r12 * vdw.x + R.r22 * vdw.y + R.r32 * vdw.z,
                 R.r13 * vdw.x + R.r23 * vdw.y + R.r33 * vdw.z};
    V3<T> r = vdg * vdg;
    T det_o = dot(r, V3<T>{ovar.y * ovar.z, ovar.z * ovar.x, ovar.x * ovar.y});
    T det_d = dot(r, V3<T>{var.y * var.z, var.z * var.x, var.x * var.y});
    T dil = std::sqrt(saturate(det_o / det_d));
    opacity *= dil;
    if (opacity < T(kMinAlpha)) return true;
    T rho_cutoff = T(2) * std::log(opacity * T(kMinAlphaRcp));
    V3<T> cs = cam - pos;
    V3<T> cg = V3<T>{R.r11 * cs.x + R.r21 * cs.y + R.r31 * cs.z, R.r12 * cs.x + R.r22 * cs.y + R.r32 * cs.z,
                     R.r13 * cs.x + R.r23 * cs.y + R.r33 * cs.z} / sc;
    if (dot(cg, cg) < rho_cutoff) return true;
    T sm = T(st->scale_modifier);
    V3<T> u = V3<T>{R.r11 * sc.x, R.r21 * sc.x, R.r31 * sc.x} * sm;
    V3<T> vv = V3<T>{R.r12 * sc.y, R.r22 * sc.y, R.r32 * sc.y} * sm;
    V3<T> w = V3<T>{R.r13 * sc.z, R.r23 * sc.z, R.r33 * sc.z} * sm;
    auto xform = [&](const float* P_) { V4<T> P = load4<T>(P_); return V4<T>{dot(xyz(P), u), dot(xyz(P), vv), dot(xyz(P), w), dot(xyz(P), pos) + P.w}; };
    VPMT1 = xform(v->VPM + 0);
    VPMT2 = xform(v->VPM + 4);
    V4<T> VPMT3 = xform(v->VPM + 8);
    VPMT4 = xform(v->VPM + 12);
    T mc = max_contrib_frustum(VPMT1, VPMT2, VPMT3, VPMT4, T(v->width), T(v->height));
    if (mc > rho_cutoff) return true;
    V4<T> MT1 = xform(v->M + 0), MT2 = xform(v->M + 4);
    V2<T> ctr, ext;
    aabb_view(MT1, MT2, VPMT4, T(v->focal_x), T(v->focal_y), T(v->center_x), T(v->center_y), rho_cutoff, ctr, ext);
    const T tw = T(kTileLarge);
    b[0] = bound_lo<T>((ctr.x - ext.x) / tw, g.glw);
    b[1] = bound_hi<T>((ctr.x + ext.x) / tw, g.glw);
    b[2] = bound_lo<T>((ctr.y - ext.y) / tw, g.glh);
    b[3] = bound_hi<T>((ctr.y + ext.y) / tw, g.glh);
    touched_from_bounds<T>(v, g, b, n);
    return n == 0;
}

/* preprocess_cu, inference.cuh:42-136 */
template <class T>
void preprocess_one(const oracle_scene* s, const oracle_view* v, const oracle_settings* st,
                    const Geometry& g, int i, PrimOut& o) {
    o = PrimOut();
    T opacity = T(s->opacities[i]);
    V4<T> P1{}, P2{}, P4{};
    uint32_t b[4] = {0, 0, 0, 0};
    uint32_t n = 0;
    bool culled = st->anti_aliasing
        ? transform_and_cull_aaa<T>(s, v, st, g, i, P1, P2, P4, opacity, b, n)
        : transform_and_cull<T>(s, v, st, g, i, P1, P2, P4, opacity, b, n);
    if (culled) return;
    o.n_touched = n;
    for (int k = 0; k < 4; ++k) o.b[k] = static_cast<uint16_t>(b[k]);
    const V4<T> P[3] = {P1, P2, P4};
    for (int r = 0; r < 3; ++r) {
        o.vpmt[4 * r + 0] = float(P[r].x); o.vpmt[4 * r + 1] = float(P[r].y);
        o.vpmt[4 * r + 2] = float(P[r].z); o.vpmt[4 * r + 3] = float(P[r].w);
    }
    V3<T> rgb = sh_to_rgb<T>(s->sh_0 + 3 * i, s->sh_rest + size_t(3) * s->total_sh_bases * i,
                             load3<T>(s->positions + 3 * i), load3<T>(v->cam_position),
                             st->active_sh_bases, s->total_sh_bases);
    o.rgba[0] = float(rgb.x); o.rgba[1] = float(rgb.y); o.rgba[2] = float(rgb.z); o.rgba[3] = float(opacity);
}

/* ---- tile classification: shared_kernels.cuh:155-238, inference.cu:131-188 ---- */
struct Tiles {
    std::vector<uint32_t> map_part;
    std::vector<uint8_t> type_part;
    uint32_t ranges[6] = {0, 0, 0, 0, 0, 0};
    uint32_t n_active = 0;
};

Tiles classify(const oracle_view* v, const Geometry& g) {
    std::vector<uint32_t> map;
    std::vector<uint8_t> type;
    const float gx = float(g.gaze_tx), gy = float(g.gaze_ty);
    for (int t = 0; t < g.n_large; ++t) {
        if (!visible(v->visibility_mask, t)) continue;
        uint32_t tx = t % g.glw, ty = t / g.glw;
        if (in_fovea(tx, ty, gx, gy, kFoveaRadiusTiles)) {
            uint8_t ty_ = in_fovea(tx, ty, gx, gy, kBlendRadiusTiles) ? FOVEA : BLENDED;
            for (int i = 0; i < kSubTiles; ++i) { map.push_back(t * kSubTiles + i); type.push_back(ty_); }
        } else {
            map.push_back(t * kSubTiles);
            type.push_back(PERIPHERY);
        }
    }
    Tiles out;
    out.n_active = static_cast<uint32_t>(map.size());
    /* stable sort by type (CUB radix sort over 2 bits, inference.cu:167-172) */
    for (uint8_t want = 0; want < 3; ++want)
        for (size_t i = 0; i < map.size(); ++i)
            if (type[i] == want) { out.map_part.push_back(map[i]); out.type_part.push_back(want); }
    /* get_partition_ranges_cu (shared_kernels.cuh:222-238), incl. the n==1 quirk */
    const uint32_t n = out.n_active;
    for (uint32_t i = 1; i < n; ++i) {
        uint8_t cur = out.type_part[i], prev = out.type_part[i - 1];
        if (cur != prev) { out.ranges[2 * cur] = i; out.ranges[2 * prev + 1] = i; }
        if (i == n - 1) out.ranges[2 * cur + 1] = n;
    }
    return out;
}

/* ---- instances: create_instances_cu (shared_kernels.cuh:15-130), stable radix sort over
 *      bits [0,end_bit) (inference.cu:267-274), extract_instance_ranges_cu (:133-152) ---- */
struct Inst {
    std::vector<uint32_t> keys, values, keys_unsorted, values_unsorted;
    std::vector<uint32_t> ranges;  /* 2*T */
    int64_t m = 0;
    uint32_t sentinel = 0;
};

Inst instances(const oracle_view* v, const Geometry& g, int n, const uint32_t* nt, const uint16_t* sb) {
    Inst I;
    I.sentinel = g.end_bit <= 16 ? 0xFFFFu : 0xFFFFFFFFu;
    std::vector<int64_t> off(n + 1, 0);
    for (int i = 0; i < n; ++i) off[i + 1] = off[i] + nt[i];
    /* the reference keeps the scan in 32-bit unsigned (inference.cu:226-236) */
    I.m = n > 0 ? static_cast<int64_t>(static_cast<uint32_t>(off[n])) : 0;
    I.keys_unsorted.assign(I.m, I.sentinel);
    I.values_unsorted.assign(I.m, 0xFFFFFFFFu);
    const float gx = float(g.gaze_tx), gy = float(g.gaze_ty);
    for (int i = 0; i < n; ++i) {
        if (nt[i] == 0) continue;
        int64_t w = off[i];
        const int64_t end = off[i] + nt[i];
        const uint32_t bw = uint32_t(sb[4 * i + 1] - sb[4 * i + 0]);
        const uint32_t cnt = uint32_t(sb[4 * i + 3] - sb[4 * i + 2]) * bw;
        for (uint32_t k = 0; k < cnt; ++k) {
            uint32_t tx = sb[4 * i + 0] + k % bw, ty = sb[4 * i + 2] + k / bw;
            uint32_t tile = ty * g.glw + tx;
            if (!visible(v->visibility_mask, tile)) continue;
            uint32_t key = tile * kSubTiles;
            int reps = in_fovea(tx, ty, gx, gy, kFoveaRadiusTiles) ? kSubTiles : 1;
            for (int r = 0; r < reps; ++r) {
                if (w < end && w < I.m) {  /* the reference writes unchecked; see DESIGN */
                    I.keys_unsorted[w] = (key + r) & I.sentinel;
                    I.values_unsorted[w] = uint32_t(i);
                }
                ++w;
            }
        }
    }
    std::vector<int64_t> idx(I.m);
    std::iota(idx.begin(), idx.end(), 0);
    const uint32_t mask = g.end_bit >= 32 ? 0xFFFFFFFFu : ((1u << g.end_bit) - 1u);
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
        return (I.keys_unsorted[a] & mask) < (I.keys_unsorted[b] & mask);
    });
    I.keys.resize(I.m);
    I.values.resize(I.m);
    for (int64_t k = 0; k < I.m; ++k) { I.keys[k] = I.keys_unsorted[idx[k]]; I.values[k] = I.values_unsorted[idx[k]]; }
    I.ranges.assign(size_t(2) * g.n_tiles, 0);
    for (int64_t k = 0; k < I.m; ++k) {
        uint32_t key = I.keys[k];
        if (k == 0) {
            if (key != I.sentinel) I.ranges[2 * key] = 0;  /* reference writes even for sentinels */
        } else {
            uint32_t prev = I.keys[k - 1];
            if (key != prev) {
                if (prev != I.sentinel) I.ranges[2 * prev + 1] = uint32_t(k);
                if (key != I.sentinel) I.ranges[2 * key] = uint32_t(k);
            }
        }
        if (k == I.m - 1 && key != I.sentinel) I.ranges[2 * key + 1] = uint32_t(I.m);
    }
    return I;
}

/* ---- blend_cu, inference.cuh:16-286; background models, background_model.cuh:8-117 ---- */
inline uint32_t pack_channel(float x) { return static_cast<uint32_t>(std::fmin(std::fmax(x, 0.0f), 1.0f) * 255.0f + 0.5f); }
template <class T> inline uint32_t pack_channel_t(T x) {
    T y = std::min(std::max(x, T(0)), T(1)) * T(255) + T(0.5);
    return static_cast<uint32_t>(y);
}

template <class T> struct Frag {
    T depth;
    uint32_t color;
};

template <class T> inline V4<T> unpack(uint32_t c) {
    const T s = T(1) / T(255);
    return {T(c & 0xff) * s, T((c >> 8) & 0xff) * s, T((c >> 16) & 0xff) * s, T((c >> 24) & 0xff) * s};
}

template <class T>
V3<T> bg_sh(const oracle_view* v, const float* coeff, T px, T py) {
    V4<T> pc = {px, py, T(1), T(1)};
    V3<T> d = normalize(V3<T>{dot(load4<T>(v->VPR_inv + 0), pc), dot(load4<T>(v->VPR_inv + 4), pc), dot(load4<T>(v->VPR_inv + 8), pc)});
    if (d.y > T(0.1f)) return {T(0), T(0), T(0)};
    V3<T> n = normalize(d);
    T x = n.x, y = n.y, z = n.z;
    T xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
    auto k = [&](int i) { return load3<T>(coeff + 3 * i); };
    V3<T> e = T(0.5) + c<T>(C0) * k(0) - c<T>(C1) * y * k(1) + c<T>(C1) * z * k(2) - c<T>(C1) * x * k(3)
              + c<T>(C2a) * xy * k(4) - c<T>(C2a) * yz * k(5) + (c<T>(C2b) * zz - c<T>(C2c)) * k(6)
              - c<T>(C2a) * xz * k(7) + c<T>(C2d) * (xx - yy) * k(8)
              + y * (c<T>(C3a) * yy - c<T>(C3b) * xx) * k(9) + c<T>(C3c) * xy * z * k(10)
              + y * (c<T>(C3d) - c<T>(C3e) * zz) * k(11) + z * (c<T>(C3f) * zz - c<T>(C3g)) * k(12)
              + x * (c<T>(C3d) - c<T>(C3e) * zz) * k(13) + c<T>(C3h) * z * (xx - yy) * k(14)
              + x * (c<T>(C3b) * yy - c<T>(C3a) * xx) * k(15);
    V3<T> col = {saturate(std::tanh(e.x) * T(0.5) + T(0.5)), saturate(std::tanh(e.y) * T(0.5) + T(0.5)),
                 saturate(std::tanh(e.z) * T(0.5) + T(0.5))};
    return d.y > T(0) ? (T(1) - d.y / T(0.1f)) * col : col;
}

template <class T>
V3<T> bg_tex(const oracle_view* v, const float* tex, int W, int H, bool activate, T px, T py) {
    V4<T> pc = {px, py, T(1), T(1)};
    V3<T> d = normalize(V3<T>{dot(load4<T>(v->VPR_inv + 0), pc), dot(load4<T>(v->VPR_inv + 4), pc), dot(load4<T>(v->VPR_inv + 8), pc)});
    if (d.y > T(0.1f)) return {T(0), T(0), T(0)};
    const T pi = T(3.14159265358979323846f);
    T eu = std::atan2(d.x, d.z) / pi * T(0.5) + T(0.5);
    T ev = std::asin(d.y) / (T(0.5) * pi) * T(0.5) + T(0.5);
    T tx = eu * T(W) - T(0.5), ty = ev * T(H) - T(0.5);
    int x0 = to_int_rd<T>(tx), y0 = to_int_rd<T>(ty), x1 = x0 + 1, y1 = y0 + 1;
    T fx = tx - T(x0), fy = ty - T(y0);
    int x0w = x0 < 0 ? x0 + W : x0, x1w = x1 >= W ? x1 - W : x1;
    int y0c = std::max(0, std::min(H - 1, y0)), y1c = std::max(0, std::min(H - 1, y1));
    int i00 = x0w + y0c * W, i10 = x1w + y0c * W, i01 = x0w + y1c * W, i11 = x1w + y1c * W;
    const int n = W * H;
    T out[3];
    for (int ch = 0; ch < 3; ++ch) {
        const float* t = tex + size_t(ch) * n;
        T c0 = T(t[i00]) * (T(1) - fx) + T(t[i10]) * fx;
        T c1 = T(t[i01]) * (T(1) - fx) + T(t[i11]) * fx;
        T cc = c0 * (T(1) - fy) + c1 * fy;
        if (activate) cc = T(1) / (T(1) + std::exp(-cc));
        out[ch] = cc;
    }
    V3<T> col = {out[0], out[1], out[2]};
    return d.y > T(0) ? (T(1) - d.y / T(0.1f)) * col : col;
}

struct ImageRef {
    float* data;
    int W, H;
    bool chw;
    inline void store(int x, int y, float r, float gg, float b) const {
        size_t p = size_t(W) * y + x;
        if (chw) { size_t n = size_t(W) * H; data[p] = r; data[n + p] = gg; data[2 * n + p] = b; }
        else { data[3 * p] = r; data[3 * p + 1] = gg; data[3 * p + 2] = b; }
    }
    inline V3<float> load(int x, int y) const {
        int sx = std::max(0, std::min(W - 1, x)), sy = std::max(0, std::min(H - 1, y));
        size_t p = size_t(W) * sy + sx;
        if (chw) { size_t n = size_t(W) * H; return {data[p], data[n + p], data[2 * n + p]}; }
        return {data[3 * p], data[3 * p + 1], data[3 * p + 2]};
    }
};

template <class T>
void blend_pixel(const oracle_view* v, const oracle_settings* st, const float* vpmt, const float* rgba,
                 const uint32_t* vals, uint32_t begin, uint32_t end, int px, int py, const ImageRef& img) {
    const int K = st->K >= 32 ? 32 : st->K >= 16 ? 16 : st->K >= 8 ? 8 : st->K >= 4 ? 4 : st->K >= 2 ? 2 : 1;
    const T x = T(float(px)), y = T(float(py));
    T tail_T = T(1);
    V4<T> tail = {T(0), T(0), T(0), T(0)};
    Frag<T> core[32];
    for (int k = 0; k < K; ++k) core[k] = {T(std::numeric_limits<float>::max()), 0u};
    for (uint32_t idx = begin; idx < end; ++idx) {
        const uint32_t p = vals[idx];
        const float* q = vpmt + size_t(12) * p;
        V4<T> P1 = load4<T>(q), P2 = load4<T>(q + 4), P4 = load4<T>(q + 8);
        V4<T> a = P1 - P4 * x, b = P2 - P4 * y;
        V3<T> an = xyz(a), bn = xyz(b);
        V3<T> m = a.w * bn - an * b.w;
        V3<T> d = cross(an, bn);
        T num = dot(m, m), den = dot(d, d);
        if (num > T(kMaxCutoffSq) * den) continue;
        T den_rcp = T(1) / den;
        T G = std::exp(T(-0.5) * num * den_rcp);
        T alpha = std::min(T(rgba[4 * p + 3]) * G, T(kMaxFragmentAlpha));
        if (alpha < T(kMinAlpha)) continue;
        V3<T> ep = cross(d, m) * den_rcp;
        T depth = dot(xyz(P4), ep) + P4.w;
        V4<T> pm = {T(rgba[4 * p]) * alpha, T(rgba[4 * p + 1]) * alpha, T(rgba[4 * p + 2]) * alpha, alpha};
        if (depth < core[K - 1].depth && alpha >= T(kMinAlphaCore)) {
            Frag<T> f = {depth, pack_channel_t(pm.x) | (pack_channel_t(pm.y) << 8) | (pack_channel_t(pm.z) << 16) |
                                    (pack_channel_t(pm.w) << 24)};
            for (int k = 0; k < K; ++k)
                if (f.depth < core[k].depth) std::swap(f, core[k]);
            pm = unpack<T>(f.color);
        }
        tail = tail + pm;
        tail_T *= T(1) - pm.w;
    }
    V3<T> rgb = {T(0), T(0), T(0)};
    T Tc = T(1);
    for (int k = 0; k < K && Tc >= T(kTransmittanceThreshold); ++k) {
        V4<T> c4 = unpack<T>(core[k].color);
        rgb = rgb + Tc * xyz(c4);
        Tc *= T(1) - c4.w;
    }
    if (Tc >= T(kTransmittanceThreshold) && tail.w >= T(kMinAlpha)) {
        T wt = Tc * (T(1) - tail_T);
        rgb = rgb + (wt * (T(1) / tail.w)) * xyz(tail);
    }
    if (st->background_type != 0) {
        T wb = Tc * tail_T;
        if (wb >= T(kTransmittanceThreshold)) {
            V3<T> bgc = st->background_type == 1
                ? bg_sh<T>(v, st->background_data, x, y)
                : bg_tex<T>(v, st->background_data, st->texture_width, st->texture_height, st->background_type == 3, x, y);
            rgb = rgb + wb * bgc;
        }
    }
    img.store(px, py, float(saturate(rgb.x)), float(saturate(rgb.y)), float(saturate(rgb.z)));
}

/* ---- interpolation.cuh:11-584 ---- */
/* Samples a stride-2 grid of (n x n) points starting at (bx, by), clamped as the reference:
 * per-axis extent clamp to the image, then masked-tile samples clamped into the large tile. */
void load_samples(const ImageRef& src, const uint32_t* mask, int glw, int bx, int by, int n,
                  int ltx, int lty, std::vector<V3<float>>& s) {
    const int max_r = int((unsigned(src.W) - unsigned(bx) - 1u) / unsigned(kStride));
    const int max_d = int((unsigned(src.H) - unsigned(by) - 1u) / unsigned(kStride));
    s.resize(size_t(n) * n);
    for (int sy = 0; sy < n; ++sy)
        for (int sx = 0; sx < n; ++sx) {
            int px = bx + std::min(sx, max_r) * kStride;
            int py = by + std::min(sy, max_d) * kStride;
            int tile = py / kTileLarge * glw + px / kTileLarge;  /* C truncation, as the device */
            if ((mask[tile / 32] & (1u << (tile % 32))) == 0) {
                int cx = std::max(ltx * kTileLarge, std::min(ltx * kTileLarge + kTileLarge - kStride, px));
                int cy = std::max(lty * kTileLarge, std::min(lty * kTileLarge + kTileLarge - kStride, py));
                s[size_t(sy) * n + sx] = src.load(cx, cy);
            } else {
                s[size_t(sy) * n + sx] = src.load(px, py);
            }
        }
}

inline float sat_f(float x) { return std::isnan(x) ? 0.0f : std::min(std::max(x, 0.0f), 1.0f); }

V3<float> bilinear(const std::vector<V3<float>>& s, int n, int lx, int ly) {
    int bx = lx / kStride, by = ly / kStride;
    float xf = float(lx % kStride) / float(kStride), yf = float(ly % kStride) / float(kStride);
    auto S = [&](int yy, int xx) { return s[size_t(yy) * n + xx]; };
    V3<float> r = {0, 0, 0};
    if (lx % kStride == 0) {
        r = r + S(by, bx) * (1.0f - yf);
        r = r + S(by + 1, bx) * yf;
    } else if (ly % kStride == 0) {
        r = r + S(by, bx) * (1.0f - xf);
        r = r + S(by, bx + 1) * xf;
    } else {
        r = r + S(by, bx) * (1.0f - xf) * (1.0f - yf);
        r = r + S(by, bx + 1) * xf * (1.0f - yf);
        r = r + S(by + 1, bx) * (1.0f - xf) * yf;
        r = r + S(by + 1, bx + 1) * xf * yf;
    }
    return r;
}

/* 5x5 binomial blur on the stride-2 grid, interpolation.cuh:343-399 (base index +1). */
V3<float> blur(const std::vector<V3<float>>& s, int n, int lx, int ly, float& factor) {
    int bx = lx / 2 + 1, by = ly / 2 + 1;
    auto S = [&](int yy, int xx) { return s[size_t(yy) * n + xx]; };
    V3<float> r = {0, 0, 0};
    if ((lx & 1) == 0 && (ly & 1) == 0) {
        factor = 1.0f / 64.0f;
        r = r + S(by - 1, bx - 1); r = r + S(by - 1, bx) * 6.0f; r = r + S(by - 1, bx + 1);
        r = r + S(by, bx - 1) * 6.0f; r = r + S(by, bx) * 36.0f; r = r + S(by, bx + 1) * 6.0f;
        r = r + S(by + 1, bx - 1); r = r + S(by + 1, bx) * 6.0f; r = r + S(by + 1, bx + 1);
    } else if ((lx & 1) == 0 && (ly & 1) == 1) {
        factor = 1.0f / 16.0f;
        r = r + S(by, bx - 1); r = r + S(by, bx) * 6.0f; r = r + S(by, bx + 1);
        r = r + S(by + 1, bx - 1); r = r + S(by + 1, bx) * 6.0f; r = r + S(by + 1, bx + 1);
    } else if ((lx & 1) == 1 && (ly & 1) == 0) {
        factor = 1.0f / 16.0f;
        r = r + S(by - 1, bx); r = r + S(by - 1, bx + 1);
        r = r + S(by, bx) * 6.0f; r = r + S(by, bx + 1) * 6.0f;
        r = r + S(by + 1, bx); r = r + S(by + 1, bx + 1);
    } else {
        factor = 1.0f / 4.0f;
        r = r + S(by, bx); r = r + S(by, bx + 1); r = r + S(by + 1, bx); r = r + S(by + 1, bx + 1);
    }
    return r;
}

inline float blend_factor(float gx, float gy, int px, int py) {
    float dx = gx - float(px), dy = gy - float(py);
    float len = std::sqrt(dx * dx + dy * dy);
    return std::min(std::max((len - float(kBlendRadiusPx) - float(kTileLarge)) / float(kBlendWidthPx - kTileLarge), 0.0f), 1.0f);
}

template <class T>
void blend_compose(const oracle_view* v, const oracle_settings* st, const Geometry& g, const float* vpmt,
                   const float* rgba, const uint32_t* map_part, const uint32_t* pranges,
                   const uint32_t* vals, const uint32_t* iranges, float* image) {
    const bool chw = st->to_chw != 0;
    const size_t npx = size_t(v->width) * v->height * 3;
    std::vector<float> temp;
    float* work = image;
    if (st->blur_periphery) { temp.assign(npx, 0.0f); work = temp.data(); }
    ImageRef fin{image, v->width, v->height, chw}, img{work, v->width, v->height, chw};
    const uint32_t fovea_b = pranges[0], fovea_e = pranges[1];
    const uint32_t per_b = pranges[2], per_e = pranges[3];
    const uint32_t bl_b = pranges[4], bl_e = pranges[5];
    auto tile_origin = [&](uint32_t tg, int& ox, int& oy, int& ltx, int& lty) {
        uint32_t lt = tg / kSubTiles, st_ = tg % kSubTiles;
        ltx = int(lt % g.glw); lty = int(lt / g.glw);
        ox = ltx * kTileLarge + int(st_ % kStride) * kTileSmall;
        oy = lty * kTileLarge + int(st_ / kStride) * kTileSmall;
    };
    /* blends (inference.cu:333-396): blended -> image, periphery (stride 2) -> image,
     * fovea -> image_final */
    auto blend_range = [&](uint32_t b, uint32_t e, bool lowres, const ImageRef& out) {
        #pragma omp parallel for schedule(dynamic, 4)
        for (int64_t gi = b; gi < int64_t(e); ++gi) {
            uint32_t tg = map_part[gi];
            int ox, oy, ltx, lty;
            tile_origin(tg, ox, oy, ltx, lty);
            uint32_t rb = iranges[2 * tg], re = iranges[2 * tg + 1];
            for (int ty = 0; ty < kTileSmall; ++ty)
                for (int tx = 0; tx < kTileSmall; ++tx) {
                    int px = ox + tx * (lowres ? kStride : 1), py = oy + ty * (lowres ? kStride : 1);
                    if (px >= v->width || py >= v->height) continue;
                    blend_pixel<T>(v, st, vpmt, rgba, vals, rb, re, px, py, out);
                }
        }
    };
    blend_range(bl_b, bl_e, false, img);
    blend_range(per_b, per_e, true, img);
    blend_range(fovea_b, fovea_e, false, fin);
    /* periphery: bilinear_interpolation (:41-146) / interpolate_and_blur (:270-413) */
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t gi = per_b; gi < int64_t(per_e); ++gi) {
        uint32_t tg = map_part[gi];
        int ox, oy, ltx, lty;
        tile_origin(tg, ox, oy, ltx, lty);
        std::vector<V3<float>> s;
        if (!st->blur_periphery) {
            load_samples(img, v->visibility_mask, g.glw, ox, oy, 9, ltx, lty, s);
            for (int ly = 0; ly < kTileLarge; ++ly)
                for (int lx = 0; lx < kTileLarge; ++lx) {
                    int px = ox + lx, py = oy + ly;
                    if (px >= v->width || py >= v->height) continue;
                    if (lx % 2 == 0 && ly % 2 == 0) continue;
                    V3<float> r = bilinear(s, 9, lx, ly);
                    fin.store(px, py, sat_f(r.x), sat_f(r.y), sat_f(r.z));
                }
        } else {
            load_samples(img, v->visibility_mask, g.glw, ox - 2, oy - 2, 10, ltx, lty, s);
            for (int ly = 0; ly < kTileLarge; ++ly)
                for (int lx = 0; lx < kTileLarge; ++lx) {
                    int px = ox + lx, py = oy + ly;
                    if (px >= v->width || py >= v->height) continue;
                    float f;
                    V3<float> r = blur(s, 10, lx, ly, f);
                    fin.store(px, py, sat_f(r.x * f), sat_f(r.y * f), sat_f(r.z * f));
                }
        }
    }
    /* blended: bilinear_interpolation_blended (:149-267) / interpolate_and_blur_blended (:416-584) */
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t gi = bl_b; gi < int64_t(bl_e); ++gi) {
        uint32_t tg = map_part[gi];
        int ox, oy, ltx, lty;
        tile_origin(tg, ox, oy, ltx, lty);
        std::vector<V3<float>> s;
        if (!st->blur_periphery) {
            load_samples(img, v->visibility_mask, g.glw, ox, oy, 5, ltx, lty, s);
            for (int ly = 0; ly < kTileSmall; ++ly)
                for (int lx = 0; lx < kTileSmall; ++lx) {
                    int px = ox + lx, py = oy + ly;
                    if (px >= v->width || py >= v->height) continue;
                    if (lx % 2 == 0 && ly % 2 == 0) continue;
                    V3<float> r = bilinear(s, 5, lx, ly);
                    float bf = blend_factor(g.gaze_px, g.gaze_py, px, py);
                    V3<float> cc = img.load(px, py);
                    if (bf > 0.0f)
                        fin.store(px, py, sat_f(r.x * bf + cc.x * (1.0f - bf)), sat_f(r.y * bf + cc.y * (1.0f - bf)),
                                  sat_f(r.z * bf + cc.z * (1.0f - bf)));
                }
        } else {
            load_samples(img, v->visibility_mask, g.glw, ox - 2, oy - 2, 6, ltx, lty, s);
            for (int ly = 0; ly < kTileSmall; ++ly)
                for (int lx = 0; lx < kTileSmall; ++lx) {
                    int px = ox + lx, py = oy + ly;
                    if (px >= v->width || py >= v->height) continue;
                    float f;
                    V3<float> r = blur(s, 6, lx, ly, f);
                    float bf = blend_factor(g.gaze_px, g.gaze_py, px, py);
                    V3<float> cc = img.load(px, py);
                    if (bf > 0.0f)
                        fin.store(px, py, sat_f(cc.x * (1.0f - bf) + r.x * f * bf), sat_f(cc.y * (1.0f - bf) + r.y * f * bf),
                                  sat_f(cc.z * (1.0f - bf) + r.z * f * bf));
                    else
                        fin.store(px, py, cc.x, cc.y, cc.z);
                }
        }
    }
}

/* ---- ring / no foveation: no counterpart in the reference; restates the product's
 *      FHTGS_FOVEATION_RINGS / _NONE modes (fhtgs_kernels.cuh: ring_tile_type, the blend's
 *      stride-4 tiles, grid_sample4 and the stride-4 bilinear fill).  Per-tile lists are the
 *      reference's (primitives in ascending order whose bounds hold the visible tile); each
 *      tile is blended at stride 1, 2 or 4 with the reference's per-pixel arithmetic and
 *      strided tiles are filled bilinearly. ---- */
enum : uint8_t { LVL_FULL = 0, LVL_HALF = 1, LVL_MASKED = 3, LVL_QUARTER = 4 };

uint8_t ring_level(const oracle_view* v, const oracle_settings* st, const Geometry& g, int tx, int ty) {
    if (st->foveation == 2) return LVL_FULL;
    const float cx = float(tx * kTileLarge + kTileLarge / 2), cy = float(ty * kTileLarge + kTileLarge / 2);
    const float hx = 0.5f * float(v->width), hy = 0.5f * float(v->height);
    const float dx = (cx - g.gaze_px) / hx, dy = (cy - g.gaze_py) / hy;
    const float dxx = dx * dx, dyy = dy * dy;
    const float r2 = dxx + dyy;
    const float f2 = st->ring_full * st->ring_full, h2 = st->ring_half * st->ring_half;
    return r2 < f2 ? LVL_FULL : r2 < h2 ? LVL_HALF : LVL_QUARTER;
}

/* (n x n) samples of the S-strided grid from (bx, by); a sample whose tile is masked, or
 * (for the 2x grid) a 4x tile, is clamped into the large tile (ltx, lty). */
void load_samples_rings(const ImageRef& src, const uint32_t* mask, const std::vector<uint8_t>& level, int glw,
                        int bx, int by, int n, int S, int ltx, int lty, std::vector<V3<float>>& s) {
    const int max_r = int((unsigned(src.W) - unsigned(bx) - 1u) / unsigned(S));
    const int max_d = int((unsigned(src.H) - unsigned(by) - 1u) / unsigned(S));
    s.resize(size_t(n) * n);
    for (int sy = 0; sy < n; ++sy)
        for (int sx = 0; sx < n; ++sx) {
            int px = bx + std::min(sx, max_r) * S;
            int py = by + std::min(sy, max_d) * S;
            int tile = py / kTileLarge * glw + px / kTileLarge;
            bool ok = (mask[tile / 32] & (1u << (tile % 32))) != 0 && !(S == kStride && level[tile] == LVL_QUARTER);
            if (!ok) {
                int cx = std::max(ltx * kTileLarge, std::min(ltx * kTileLarge + kTileLarge - S, px));
                int cy = std::max(lty * kTileLarge, std::min(lty * kTileLarge + kTileLarge - S, py));
                s[size_t(sy) * n + sx] = src.load(cx, cy);
            } else {
                s[size_t(sy) * n + sx] = src.load(px, py);
            }
        }
}

V3<float> bilinear_s(const std::vector<V3<float>>& s, int n, int S, int lx, int ly) {
    int bx = lx / S, by = ly / S;
    float xf = float(lx % S) / float(S), yf = float(ly % S) / float(S);
    auto P = [&](int yy, int xx) { return s[size_t(yy) * n + xx]; };
    V3<float> r = {0, 0, 0};
    if (lx % S == 0) {
        r = r + P(by, bx) * (1.0f - yf);
        r = r + P(by + 1, bx) * yf;
    } else if (ly % S == 0) {
        r = r + P(by, bx) * (1.0f - xf);
        r = r + P(by, bx + 1) * xf;
    } else {
        r = r + P(by, bx) * (1.0f - xf) * (1.0f - yf);
        r = r + P(by, bx + 1) * xf * (1.0f - yf);
        r = r + P(by + 1, bx) * (1.0f - xf) * yf;
        r = r + P(by + 1, bx + 1) * xf * yf;
    }
    return r;
}

template <class T>
void render_rings(const oracle_view* v, const oracle_settings* st, const Geometry& g, int n, const uint32_t* nt,
                  const uint16_t* sb, const float* vpmt, const float* rgba, float* image) {
    std::vector<std::vector<uint32_t>> lists(size_t(g.n_large));
    for (int i = 0; i < n; ++i) {
        if (nt[i] == 0) continue;
        for (uint32_t ty = sb[4 * i + 2]; ty < sb[4 * i + 3]; ++ty)
            for (uint32_t tx = sb[4 * i + 0]; tx < sb[4 * i + 1]; ++tx) {
                const uint32_t t = ty * uint32_t(g.glw) + tx;
                if (visible(v->visibility_mask, t)) lists[t].push_back(uint32_t(i));
            }
    }
    std::vector<uint8_t> level(size_t(g.n_large), LVL_MASKED);
    for (int t = 0; t < g.n_large; ++t)
        if (visible(v->visibility_mask, t)) level[t] = ring_level(v, st, g, t % g.glw, t / g.glw);
    ImageRef img{image, v->width, v->height, st->to_chw != 0};
    #pragma omp parallel for schedule(dynamic, 4)
    for (int t = 0; t < g.n_large; ++t) {
        if (level[t] == LVL_MASKED) continue;
        const int S = level[t] == LVL_FULL ? 1 : level[t] == LVL_HALF ? kStride : 4;
        const int ox = (t % g.glw) * kTileLarge, oy = (t / g.glw) * kTileLarge;
        const std::vector<uint32_t>& L = lists[t];
        for (int y = 0; y < kTileLarge; y += S)
            for (int x = 0; x < kTileLarge; x += S) {
                if (ox + x >= v->width || oy + y >= v->height) continue;
                blend_pixel<T>(v, st, vpmt, rgba, L.data(), 0, uint32_t(L.size()), ox + x, oy + y, img);
            }
    }
    #pragma omp parallel for schedule(dynamic, 4)
    for (int t = 0; t < g.n_large; ++t) {
        if (level[t] != LVL_HALF && level[t] != LVL_QUARTER) continue;
        const int S = level[t] == LVL_HALF ? kStride : 4;
        const int ltx = t % g.glw, lty = t / g.glw, ox = ltx * kTileLarge, oy = lty * kTileLarge;
        const int ns = kTileLarge / S + 1;
        std::vector<V3<float>> smp;
        load_samples_rings(img, v->visibility_mask, level, g.glw, ox, oy, ns, S, ltx, lty, smp);
        for (int ly = 0; ly < kTileLarge; ++ly)
            for (int lx = 0; lx < kTileLarge; ++lx) {
                const int px = ox + lx, py = oy + ly;
                if (px >= v->width || py >= v->height) continue;
                if (lx % S == 0 && ly % S == 0) continue;
                V3<float> r = bilinear_s(smp, ns, S, lx, ly);
                img.store(px, py, sat_f(r.x), sat_f(r.y), sat_f(r.z));
            }
    }
}

struct ThreadScope {
    int prev = 0;
    explicit ThreadScope(int n) {
#ifdef _OPENMP
        prev = omp_get_max_threads();
        if (n > 0) omp_set_num_threads(n);
#else
        (void)n;
#endif
    }
    ~ThreadScope() {
#ifdef _OPENMP
        omp_set_num_threads(prev);
#endif
    }
};

template <class T>
void preprocess_all(const oracle_scene* s, const oracle_view* v, const oracle_settings* st, const Geometry& g,
                    std::vector<uint32_t>& nt, std::vector<uint16_t>& sb, std::vector<float>& vpmt, std::vector<float>& rgba) {
    const int n = s->n;
    nt.assign(n, 0); sb.assign(size_t(4) * n, 0); vpmt.assign(size_t(12) * n, 0.0f); rgba.assign(size_t(4) * n, 0.0f);
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        PrimOut o;
        preprocess_one<T>(s, v, st, g, i, o);
        nt[i] = o.n_touched;
        for (int k = 0; k < 4; ++k) sb[4 * size_t(i) + k] = o.b[k];
        std::memcpy(&vpmt[12 * size_t(i)], o.vpmt, sizeof(o.vpmt));
        std::memcpy(&rgba[4 * size_t(i)], o.rgba, sizeof(o.rgba));
    }
}

// Wall seconds per stage (preprocess, tile classification, instance creation + sort + ranges,
// blend + composition), summed over the views of the last oracle_time_views call.
double g_stage_seconds[4];

template <class T>
int render_view_t(const oracle_scene* s, const oracle_view* v, const oracle_settings* st, float* image,
                  oracle_primitives* prim, oracle_tiles* tiles, oracle_instances* inst) {
    using clk = std::chrono::steady_clock;
    auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    const Geometry g = geometry(v);
    std::vector<uint32_t> nt;
    std::vector<uint16_t> sb;
    std::vector<float> vpmt, rgba;
    const auto t0 = clk::now();
    preprocess_all<T>(s, v, st, g, nt, sb, vpmt, rgba);
    const auto t1 = clk::now();
    Tiles tl = classify(v, g);
    const auto t2 = clk::now();
    Inst I = instances(v, g, s->n, nt.data(), sb.data());
    const auto t3 = clk::now();
    if (image) {
        std::memset(image, 0, sizeof(float) * size_t(v->width) * v->height * 3);
        if (st->foveation == 0)
            blend_compose<T>(v, st, g, vpmt.data(), rgba.data(), tl.map_part.data(), tl.ranges, I.values.data(),
                             I.ranges.data(), image);
        else
            render_rings<T>(v, st, g, s->n, nt.data(), sb.data(), vpmt.data(), rgba.data(), image);
    }
    const auto t4 = clk::now();
    g_stage_seconds[0] += secs(t0, t1);
    g_stage_seconds[1] += secs(t1, t2);
    g_stage_seconds[2] += secs(t2, t3);
    g_stage_seconds[3] += secs(t3, t4);
    if (prim) {
        if (prim->n_touched) std::memcpy(prim->n_touched, nt.data(), nt.size() * 4);
        if (prim->screen_bounds) std::memcpy(prim->screen_bounds, sb.data(), sb.size() * 2);
        if (prim->vpmt) std::memcpy(prim->vpmt, vpmt.data(), vpmt.size() * 4);
        if (prim->rgba) std::memcpy(prim->rgba, rgba.data(), rgba.size() * 4);
    }
    if (tiles) {
        if (tiles->tile_index_map_partitioned) std::memcpy(tiles->tile_index_map_partitioned, tl.map_part.data(), tl.map_part.size() * 4);
        if (tiles->tile_type_partitioned) std::memcpy(tiles->tile_type_partitioned, tl.type_part.data(), tl.type_part.size());
        if (tiles->partition_ranges) std::memcpy(tiles->partition_ranges, tl.ranges, sizeof(tl.ranges));
        if (tiles->n_active_tiles) *tiles->n_active_tiles = tl.n_active;
    }
    if (inst) {
        if (inst->n_instances) *inst->n_instances = I.m;
        int64_t cnt = std::min<int64_t>(I.m, inst->capacity);
        if (inst->keys) std::memcpy(inst->keys, I.keys.data(), size_t(cnt) * 4);
        if (inst->values) std::memcpy(inst->values, I.values.data(), size_t(cnt) * 4);
        if (inst->instance_ranges) std::memcpy(inst->instance_ranges, I.ranges.data(), I.ranges.size() * 4);
    }
    return 0;
}

}  // namespace

extern "C" {

void oracle_view_geometry(const oracle_view* v, int* glw, int* glh, int* n_tiles, int* end_bit, int* gtx, int* gty) {
    Geometry g = geometry(v);
    if (glw) *glw = g.glw;
    if (glh) *glh = g.glh;
    if (n_tiles) *n_tiles = g.n_tiles;
    if (end_bit) *end_bit = g.end_bit;
    if (gtx) *gtx = g.gaze_tx;
    if (gty) *gty = g.gaze_ty;
}

int oracle_classify_tiles(const oracle_view* v, oracle_tiles* out) {
    Geometry g = geometry(v);
    Tiles t = classify(v, g);
    if (out->tile_index_map_partitioned) std::memcpy(out->tile_index_map_partitioned, t.map_part.data(), t.map_part.size() * 4);
    if (out->tile_type_partitioned) std::memcpy(out->tile_type_partitioned, t.type_part.data(), t.type_part.size());
    if (out->partition_ranges) std::memcpy(out->partition_ranges, t.ranges, sizeof(t.ranges));
    if (out->n_active_tiles) *out->n_active_tiles = t.n_active;
    return 0;
}

int oracle_preprocess(const oracle_scene* s, const oracle_view* v, const oracle_settings* st, oracle_primitives* out) {
    ThreadScope ts(st->n_threads);
    Geometry g = geometry(v);
    std::vector<uint32_t> nt;
    std::vector<uint16_t> sb;
    std::vector<float> vpmt, rgba;
    if (st->precision == 64) preprocess_all<double>(s, v, st, g, nt, sb, vpmt, rgba);
    else preprocess_all<float>(s, v, st, g, nt, sb, vpmt, rgba);
    if (out->n_touched) std::memcpy(out->n_touched, nt.data(), nt.size() * 4);
    if (out->screen_bounds) std::memcpy(out->screen_bounds, sb.data(), sb.size() * 2);
    if (out->vpmt) std::memcpy(out->vpmt, vpmt.data(), vpmt.size() * 4);
    if (out->rgba) std::memcpy(out->rgba, rgba.data(), rgba.size() * 4);
    return 0;
}

int oracle_instances_from_primitives(const oracle_view* v, int n, const uint32_t* nt, const uint16_t* sb,
                                     oracle_instances* out, uint32_t* uk, uint32_t* uv) {
    Geometry g = geometry(v);
    Inst I = instances(v, g, n, nt, sb);
    if (out->n_instances) *out->n_instances = I.m;
    int64_t cnt = std::min<int64_t>(I.m, out->capacity);
    if (out->keys) std::memcpy(out->keys, I.keys.data(), size_t(cnt) * 4);
    if (out->values) std::memcpy(out->values, I.values.data(), size_t(cnt) * 4);
    if (uk) std::memcpy(uk, I.keys_unsorted.data(), size_t(cnt) * 4);
    if (uv) std::memcpy(uv, I.values_unsorted.data(), size_t(cnt) * 4);
    if (out->instance_ranges) std::memcpy(out->instance_ranges, I.ranges.data(), I.ranges.size() * 4);
    return 0;
}

int oracle_blend_compose(const oracle_view* v, const oracle_settings* st, int n, const float* vpmt, const float* rgba,
                         const uint32_t* map_part, const uint32_t* pranges, const uint32_t* vals,
                         const uint32_t* iranges, float* image) {
    (void)n;
    ThreadScope ts(st->n_threads);
    Geometry g = geometry(v);
    std::memset(image, 0, sizeof(float) * size_t(v->width) * v->height * 3);
    if (st->precision == 64) blend_compose<double>(v, st, g, vpmt, rgba, map_part, pranges, vals, iranges, image);
    else blend_compose<float>(v, st, g, vpmt, rgba, map_part, pranges, vals, iranges, image);
    return 0;
}

int oracle_render_view(const oracle_scene* s, const oracle_view* v, const oracle_settings* st, float* image,
                       oracle_primitives* prim, oracle_tiles* tiles, oracle_instances* inst) {
    ThreadScope ts(st->n_threads);
    if (st->precision == 64) return render_view_t<double>(s, v, st, image, prim, tiles, inst);
    return render_view_t<float>(s, v, st, image, prim, tiles, inst);
}

double oracle_time_views(const oracle_scene* s, const oracle_view* views, int n_views, const oracle_settings* st,
                         float* const* images) {
    for (double& x : g_stage_seconds) x = 0.0;
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < n_views; ++i) oracle_render_view(s, &views[i], st, images[i], nullptr, nullptr, nullptr);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

void oracle_stage_seconds(double* out) {
    for (int i = 0; i < 4; ++i) out[i] = g_stage_seconds[i];
}

}  // extern "C"
