// Per-Gaussian device math of the pinhole 3DGS path: raw activation, EWA
// projection, screen-covariance cap, opacity-aware tile walk, SH colour,
// and their adjoints.
//
// Bit-exact draw lists against the reference need the same floating-point
// rounding sequence in every value that feeds a sort key or a tile decision
// (pixel mean, conic, opacity, depth, tile walk). The expressions below keep
// the reference's association order and operand order for those values, term
// by term, and the library is compiled with the same -use_fast_math flags:
//   activation   third_party/splat_drender/src/device/activation.cuh:13-31
//   projection   third_party/splat_drender/src/device/geometry.cuh:127-277 (pinhole branch)
//   cov cap      third_party/splat_drender/src/device/footprint.cuh:14-35
//   tile walk    third_party/splat_drender/src/device/tiles.cuh:18-179 (non-wrapping walk)
//   SH colour    third_party/splat_drender/src/device/sh.cuh:19-66
//   3x3 algebra  third_party/splat_drender/src/device/matrix.cuh:49-170
// The adjoints (geometry.cuh:317-912 pinhole RGB chain, sh.cuh:76-173) only
// need tolerance-level agreement and are written for registers.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace gsb {

constexpr int kTileW = 16;
constexpr int kTileH = 16;
constexpr int kTilePixels = kTileW * kTileH;
constexpr float kAlphaFloor = 1.0f / 255.0f;
constexpr float kTransmittanceFloor = 1.0e-4f;

// Kernel-parameter camera: everything a launch needs, passed by value so no
// device upload precedes a render.
struct Camera {
    float view[16];  // column-major world-to-camera
    float center[3]; // camera centre, world space
    float fx, fy, cx, cy;
    float near_plane, alpha_clip;
    int width, height;
    int grid_x, grid_y;
    int compensate_2d;
    float kernel_size;
    float scale_modifier;
};

// ------------------------------------------------------------------ 3x3 ----
struct M3 {
    float m[3][3];
};

__device__ __forceinline__ M3 m3_zero() {
    M3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            o.m[i][j] = 0.f;
    return o;
}

__device__ __forceinline__ M3 m3_diag(float x, float y, float z) {
    M3 o = m3_zero();
    o.m[0][0] = x;
    o.m[1][1] = y;
    o.m[2][2] = z;
    return o;
}

// Row-major product; every entry sums k = 0,1,2 left to right.
__device__ __forceinline__ M3 m3_mul(const M3& a, const M3& b) {
    M3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            o.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return o;
}

__device__ __forceinline__ M3 m3_t(const M3& a) {
    M3 o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            o.m[i][j] = a.m[j][i];
    return o;
}

// Scalar-first quaternion to rotation rows.
__device__ __forceinline__ M3 quat_to_rows(float4 q) {
    const float r = q.x, x = q.y, y = q.z, z = q.w;
    M3 o;
    o.m[0][0] = 1.f - 2.f * (y * y + z * z);
    o.m[0][1] = 2.f * (x * y + r * z);
    o.m[0][2] = 2.f * (x * z - r * y);
    o.m[1][0] = 2.f * (x * y - r * z);
    o.m[1][1] = 1.f - 2.f * (x * x + z * z);
    o.m[1][2] = 2.f * (y * z + r * x);
    o.m[2][0] = 2.f * (x * z + r * y);
    o.m[2][1] = 2.f * (y * z - r * x);
    o.m[2][2] = 1.f - 2.f * (x * x + y * y);
    return o;
}

// World point -> camera point with the column-major 4x4 view.
__device__ __forceinline__ float3 to_camera(float3 p, const float* v) {
    return make_float3(v[0] * p.x + v[4] * p.y + v[8] * p.z + v[12],
                       v[1] * p.x + v[5] * p.y + v[9] * p.z + v[13],
                       v[2] * p.x + v[6] * p.y + v[10] * p.z + v[14]);
}

// Camera-frame gradient back to world frame (R^T g).
__device__ __forceinline__ float3 to_world_dir(float3 d, const float* v) {
    return make_float3(v[0] * d.x + v[1] * d.y + v[2] * d.z, v[4] * d.x + v[5] * d.y + v[6] * d.z,
                       v[8] * d.x + v[9] * d.y + v[10] * d.z);
}

// Rotation block of the view with rows = world axes (glm's transposed W).
__device__ __forceinline__ M3 view_rows(const float* v) {
    M3 w;
    w.m[0][0] = v[0];
    w.m[0][1] = v[1];
    w.m[0][2] = v[2];
    w.m[1][0] = v[4];
    w.m[1][1] = v[5];
    w.m[1][2] = v[6];
    w.m[2][0] = v[8];
    w.m[2][1] = v[9];
    w.m[2][2] = v[10];
    return w;
}

// ---------------------------------------------------------- activation ----
struct Activated {
    float3 scale;       // exp(log scale), 3D-filtered
    float3 raw_scale;   // exp(log scale)
    float4 rot;         // normalised quaternion
    float opacity;      // sigmoid(logit) * filter ratio
};

__device__ __forceinline__ Activated activate(const float* __restrict__ log_scales,
                                              const float* __restrict__ quats,
                                              const float* __restrict__ logits,
                                              const float* __restrict__ filter_3d, int i) {
    Activated a;
    float* s = &a.scale.x;
    float ratio = 1.f;
    const float f2 = filter_3d ? filter_3d[i] * filter_3d[i] : 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float v = expf(log_scales[3 * i + k]);
        (&a.raw_scale.x)[k] = v;
        s[k] = sqrtf(v * v + f2);
        ratio *= v / s[k];
    }
    const float4 q = reinterpret_cast<const float4*>(quats)[i];
    const float w = q.x, x = q.y, y = q.z, z = q.w;
    const float inv = rsqrtf(fmaxf(w * w + x * x + y * y + z * z, 1e-20f));
    a.rot = make_float4(w * inv, x * inv, y * inv, z * inv);
    a.opacity = (1.f / (1.f + expf(-logits[i]))) * ratio;
    return a;
}

// ---------------------------------------------------------- projection ----
// 2D screen covariance (kernel-inflated) and the Mip opacity coefficient of
// one Gaussian under the pinhole EWA Jacobian with the +-1.3 tan(fov) clamp.
struct Cov2D {
    float a, b, c; // xx, xy, yy
    float coef;
};

__device__ __forceinline__ Cov2D project_cov(float3 mean, const Camera& K, float3 scale,
                                             float4 rot) {
    float3 t = to_camera(mean, K.view);
    const float tan_fovx = float(K.width) / (2.f * K.fx);
    const float tan_fovy = float(K.height) / (2.f * K.fy);
    const float limx = 1.3f * tan_fovx, limy = 1.3f * tan_fovy;
    const float u = t.x / t.z;
    const float v = t.y / t.z;
    t.x = fminf(limx, fmaxf(-limx, u)) * t.z;
    t.y = fminf(limy, fmaxf(-limy, v)) * t.z;
    M3 J;
    J.m[0][0] = K.fx / t.z;
    J.m[0][1] = 0.f;
    J.m[0][2] = 0.f;
    J.m[1][0] = 0.f;
    J.m[1][1] = K.fy / t.z;
    J.m[1][2] = 0.f;
    J.m[2][0] = -(K.fx * t.x) / (t.z * t.z);
    J.m[2][1] = -(K.fy * t.y) / (t.z * t.z);
    J.m[2][2] = 0.f;
    const M3 W = view_rows(K.view);
    const M3 T = m3_mul(W, J);
    const float sm = K.scale_modifier;
    const M3 S = m3_diag(sm * scale.x, sm * scale.y, sm * scale.z);
    const M3 R = quat_to_rows(rot);
    const M3 SR = m3_mul(S, R);
    const M3 M = m3_mul(SR, T);
    const M3 cov = m3_mul(m3_t(M), M);
    Cov2D o;
    o.a = cov.m[0][0] + K.kernel_size;
    o.b = cov.m[0][1];
    o.c = cov.m[1][1] + K.kernel_size;
    const float det0 = fmaxf(1.0e-6f, cov.m[0][0] * cov.m[1][1] - cov.m[0][1] * cov.m[0][1]);
    const float det1 = fmaxf(1.0e-6f, o.a * o.c - o.b * o.b);
    o.coef = K.compensate_2d ? sqrtf(det0 / det1) : 1.f;
    return o;
}

// --------------------------------------------------- geometry channels ----
// Matrix times column vector, rows summed left to right.
__device__ __forceinline__ float3 m3_vec(const M3& a, float3 v) {
    return make_float3(a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
                       a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
                       a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z);
}

// Ray plane and footprint normal of a Gaussian for the median-depth and
// normal channels (geometry.cuh:255-275, pinhole branch, scale/rotation
// form): along the camera ray through screen offset (dx, dy) from the
// Gaussian's centre, the distance of its density peak is approximately
// plane.x * dx + plane.y * dy + plane.z (plane.z = distance of the centre),
// and plane.w is 1/sigma of the density along the ray at the peak. The normal
// is the camera-space normal of the peak surface. Uses the clamped camera
// point of the EWA projection; the steps and association are the reference's
// (the inverse covariance M^-T M^-1 with M^-1 = S^-1 R W, S^-1 by IEEE
// reciprocals).
__device__ __forceinline__ void ray_plane_normal(float3 mean, const Camera& K, float3 scale,
                                                 float4 rot, float4& plane_out,
                                                 float3& normal_out) {
    float3 t = to_camera(mean, K.view);
    const float tc = norm3df(t.x, t.y, t.z);
    const float tan_fovx = float(K.width) / (2.f * K.fx);
    const float tan_fovy = float(K.height) / (2.f * K.fy);
    const float limx = 1.3f * tan_fovx, limy = 1.3f * tan_fovy;
    float u = t.x / t.z;
    float v = t.y / t.z;
    t.x = fminf(limx, fmaxf(-limx, u)) * t.z;
    t.y = fminf(limy, fmaxf(-limy, v)) * t.z;
    u = t.x / t.z;
    v = t.y / t.z;
    const M3 W = view_rows(K.view);
    const float sm = K.scale_modifier;
    const M3 S_inv =
        m3_diag(__frcp_rn(sm * scale.x), __frcp_rn(sm * scale.y), __frcp_rn(sm * scale.z));
    const M3 R = quat_to_rows(rot);
    const M3 SR_inv = m3_mul(S_inv, R);
    const M3 M_inv = m3_mul(SR_inv, W);
    const M3 cov_cam_inv = m3_mul(m3_t(M_inv), M_inv);
    const float3 uvh = make_float3(u, v, 1.f);
    const float3 uvh_m = m3_vec(cov_cam_inv, uvh);
    const float u2 = u * u, v2 = v * v;
    const float l = norm3df(t.x, t.y, t.z);
    M3 nJ_inv = m3_zero();
    nJ_inv.m[0][0] = v2 + 1.f;
    nJ_inv.m[0][1] = -(u * v);
    nJ_inv.m[0][2] = -u;
    nJ_inv.m[1][0] = -(u * v);
    nJ_inv.m[1][1] = u2 + 1.f;
    nJ_inv.m[1][2] = -v;
    const float vb = uvh_m.x * uvh.x + uvh_m.y * uvh.y + uvh_m.z * uvh.z;
    const float ray_len2 = u2 + v2 + 1.f;
    const float factor_normal = l / ray_len2;
    const float3 plane =
        m3_vec(nJ_inv, make_float3(uvh_m.x / vb, uvh_m.y / vb, uvh_m.z / vb));
    const float rsigmat = sqrtf(vb / ray_len2);
    plane_out = make_float4(plane.x * factor_normal / K.fx, plane.y * factor_normal / K.fy, tc,
                            rsigmat);
    const float3 ray_normal =
        make_float3(-plane.x * factor_normal, -plane.y * factor_normal, -1.f);
    M3 nJ = m3_zero();
    const float iz = 1.f / t.z;
    nJ.m[0][0] = iz;
    nJ.m[0][2] = t.x / l;
    nJ.m[1][1] = iz;
    nJ.m[1][2] = t.y / l;
    nJ.m[2][0] = -t.x * iz * iz;
    nJ.m[2][1] = -t.y * iz * iz;
    nJ.m[2][2] = t.z / l;
    const float3 cam_normal = m3_vec(nJ, ray_normal);
    const float inv = rnorm3df(cam_normal.x, cam_normal.y, cam_normal.z);
    normal_out = make_float3(cam_normal.x * inv, cam_normal.y * inv, cam_normal.z * inv);
}

// Camera-space Z of the unit ray through pixel (px, py) (camera.h:251-300):
// converts a distance along the ray into depth.
__device__ __forceinline__ float pixel_ray_z(float px, float py, const Camera& K) {
    const float x = (px - K.cx) / K.fx;
    const float y = (py - K.cy) / K.fy;
    return rnorm3df(x, y, 1.f);
}

// Screen-covariance cap: lambda_max(C) <= min(1024, W, H)^2 / 8.
struct CovCap {
    float q, lambda, da, db, dc;
};

__device__ __forceinline__ CovCap cov_cap(float a, float b, float c, int width, int height) {
    const float half = .5f * (a - c);
    const float radius = hypotf(half, b);
    const float lambda = .5f * a + .5f * c + radius;
    const float limit = fminf(1024.f, float(min(width, height)));
    const float variance = .125f * limit * limit;
    if (!(lambda > variance) || !isfinite(lambda))
        return {1.f, lambda, 0.f, 0.f, 0.f};
    const float h = radius > 0.f ? half / radius : 0.f;
    return {variance / lambda, lambda, .5f + .5f * h, radius > 0.f ? b / radius : 0.f,
            .5f - .5f * h};
}

// ------------------------------------------------------------- tile walk --
// Opacity-aware tile footprint: the alpha = 1/255 iso-contour ellipse,
// sliced along the shorter screen axis; each slice (column u) covers an exact
// interval [v_min, v_max) on the long axis. Tiles are visited in walk order
// (outer: u, inner: v). TW x TH is the tile shape in pixels (16 x 16 is the
// reference's). The set-up and the per-column interval are separate so a warp
// can share one Gaussian's columns; the expressions are the same either way.
struct TileWalk {
    float cu, cv, av, bu, det, threshold, eu, ev, blk_u, blk_v, arg_v_min, arg_v_max;
    int gu, gv, u_min, u_max, grid_x;
    bool along_x;
};

// False when the footprint reaches no tile.
template <int TW = kTileW, int TH = kTileH>
__device__ __forceinline__ bool walk_setup(float2 mean, float4 co, int grid_x, int grid_y,
                                           TileWalk& w) {
    const float a = co.x, b = co.y, c = co.z;
    const float det = a * c - b * b;
    if (!(a > 0.f && c > 0.f) || !(co.w >= 1.f / 255.f) || !(det > 0.f))
        return false;
    const float threshold = 2.f * logf(co.w * 255.f);
    if (!(threshold >= 0.f))
        return false;
    const float ex = sqrtf(threshold * c / det);
    const float ey = sqrtf(threshold * a / det);
    const bool along_x = (2.f * ex) / TW <= (2.f * ey) / TH;
    const float cu = along_x ? mean.x : mean.y;
    const float cv = along_x ? mean.y : mean.x;
    const float au = along_x ? a : c;
    const float av = along_x ? c : a;
    const float bu = b;
    const int gu = along_x ? grid_x : grid_y;
    const int gv = along_x ? grid_y : grid_x;
    const float blk_u = along_x ? float(TW) : float(TH);
    const float blk_v = along_x ? float(TH) : float(TW);
    const float eu = sqrtf(threshold * av / det);
    const float ev = sqrtf(threshold * au / det);
    const int u_min = max(0, min(gu, int(floorf((cu - eu) / blk_u))));
    const int u_max = min(gu, min(gu, int(floorf((cu + eu) / blk_u)) + 1));
    if (u_min >= u_max)
        return false;
    w.cu = cu;
    w.cv = cv;
    w.av = av;
    w.bu = bu;
    w.det = det;
    w.threshold = threshold;
    w.eu = eu;
    w.ev = ev;
    w.blk_u = blk_u;
    w.blk_v = blk_v;
    w.arg_v_min = cu + bu * ev / au;
    w.arg_v_max = cu - bu * ev / au;
    w.gu = gu;
    w.gv = gv;
    w.u_min = u_min;
    w.u_max = u_max;
    w.grid_x = grid_x;
    w.along_x = along_x;
    return true;
}

// [v_min, v_max) of column tu (empty when v_min >= v_max).
__device__ __forceinline__ void walk_column(const TileWalk& w, int tu, int& v_min, int& v_max) {
    const float cu = w.cu, cv = w.cv, av = w.av, bu = w.bu, det = w.det;
    const float s0 = fmaxf(cu - w.eu, tu * w.blk_u);
    const float s1 = fminf(cu + w.eu, (tu + 1) * w.blk_u);
    const float d0 = s0 - cu, d1 = s1 - cu;
    const float r0 = sqrtf(fmaxf(0.f, av * w.threshold - det * d0 * d0));
    const float r1 = sqrtf(fmaxf(0.f, av * w.threshold - det * d1 * d1));
    const float lo0 = cv + (-bu * d0 - r0) / av;
    const float lo1 = cv + (-bu * d1 - r1) / av;
    const float hi0 = cv + (-bu * d0 + r0) / av;
    const float hi1 = cv + (-bu * d1 + r1) / av;
    const float sv_min = (w.arg_v_min >= s0 && w.arg_v_min <= s1) ? cv - w.ev : fminf(lo0, lo1);
    const float sv_max = (w.arg_v_max >= s0 && w.arg_v_max <= s1) ? cv + w.ev : fmaxf(hi0, hi1);
    v_min = max(0, min(w.gv, int(floorf(sv_min / w.blk_v))));
    v_max = min(w.gv, min(w.gv, int(floorf(sv_max / w.blk_v)) + 1));
}

__device__ __forceinline__ unsigned walk_tile_id(const TileWalk& w, int tu, int tv) {
    const int tx = w.along_x ? tu : tv;
    const int ty = w.along_x ? tv : tu;
    return unsigned(ty) * unsigned(w.grid_x) + unsigned(tx);
}

// ------------------------------------------------------------ tile spans --
// The preprocess's walk in 16 bytes, so the instance emit expands it without
// walking again (emit.cuh lists a Gaussian's columns from it):
//  x: bits 0-11 first column u_min, 12-23 base row v_base (the least v_min
//     of the non-empty columns), 24-26 column count u_max - u_min,
//     27 along_x, 31 (kSpanWalk) set when the walk does not fit and the emit
//     walks it again;
//  y, z, w: column c < kSpanCols in bits [16 (c & 1), 16 (c & 1) + 16) of
//     word c / 2: low byte v_min - v_base, high byte the column's tile count.
// Instance k of a Gaussian is the k-th tile in walk order (u, then v).
constexpr int kSpanCols = 6;
constexpr unsigned kSpanWalk = 1u << 31;

// walk_tiles' count, with the walk recorded in `spans`.
template <int TW = kTileW, int TH = kTileH>
__device__ __forceinline__ unsigned walk_count_spans(float2 mean, float4 co, int grid_x,
                                                     int grid_y, uint4& spans) {
    spans = make_uint4(kSpanWalk, 0u, 0u, 0u);
    TileWalk w;
    if (!walk_setup<TW, TH>(mean, co, grid_x, grid_y, w))
        return 0;
    int lo[kSpanCols], len[kSpanCols];
    unsigned count = 0;
#pragma unroll
    for (int c = 0; c < kSpanCols; ++c) {
        lo[c] = 0;
        len[c] = 0;
        if (w.u_min + c < w.u_max) {
            int v_min, v_max;
            walk_column(w, w.u_min + c, v_min, v_max);
            lo[c] = v_min;
            len[c] = v_max > v_min ? v_max - v_min : 0;
            count += unsigned(len[c]);
        }
    }
    for (int tu = w.u_min + kSpanCols; tu < w.u_max; ++tu) {
        int v_min, v_max;
        walk_column(w, tu, v_min, v_max);
        if (v_max > v_min)
            count += unsigned(v_max - v_min);
    }
    const int ncol = w.u_max - w.u_min;
    int base = 0xfff;
#pragma unroll
    for (int c = 0; c < kSpanCols; ++c)
        if (len[c] > 0)
            base = min(base, lo[c]);
    bool fits = ncol <= kSpanCols && w.u_min < 0x1000 && count > 0;
    unsigned packed[3] = {0u, 0u, 0u};
#pragma unroll
    for (int c = 0; c < kSpanCols; ++c) {
        const int off = len[c] > 0 ? lo[c] - base : 0;
        fits = fits && off < 256 && len[c] < 256;
        packed[c >> 1] |= (unsigned(off & 0xff) | (unsigned(len[c] & 0xff) << 8)) << (16 * (c & 1));
    }
    if (fits)
        spans = make_uint4(unsigned(w.u_min) | (unsigned(base) << 12) | (unsigned(ncol) << 24) |
                               (w.along_x ? 1u << 27 : 0u),
                           packed[0], packed[1], packed[2]);
    return count;
}

// ------------------------------------------------------------------- SH --
__device__ constexpr float kSH0 = 0.28209479177387814f;
__device__ constexpr float kSH1 = 0.4886025119029199f;
__device__ constexpr float kSH2[5] = {1.0925484305920792f, -1.0925484305920792f,
                                      0.31539156525252005f, -1.0925484305920792f,
                                      0.5462742152960396f};
__device__ constexpr float kSH3[7] = {-0.5900435899266435f, 2.890611442640554f,
                                      -0.4570457994644658f, 0.3731763325901154f,
                                      -0.4570457994644658f, 1.445305721320277f,
                                      -0.5900435899266435f};

// View-dependent colour of one Gaussian from its SH row `c` (RGB triples).
// clamp_bits receives bit k set when channel k was negative before max(.,0).
__device__ __forceinline__ float3 sh_color(const float3* c, int degree, float3 pos, float3 campos,
                                           unsigned& clamp_bits) {
    float3 dir = make_float3(pos.x - campos.x, pos.y - campos.y, pos.z - campos.z);
    const float inv = rnorm3df(dir.x, dir.y, dir.z);
    dir = make_float3(dir.x * inv, dir.y * inv, dir.z * inv);
    float3 r = make_float3(kSH0 * c[0].x, kSH0 * c[0].y, kSH0 * c[0].z);
    const float x = dir.x, y = dir.y, z = dir.z;
    if (degree > 0) {
        r.x += -kSH1 * y * c[1].x + kSH1 * z * c[2].x - kSH1 * x * c[3].x;
        r.y += -kSH1 * y * c[1].y + kSH1 * z * c[2].y - kSH1 * x * c[3].y;
        r.z += -kSH1 * y * c[1].z + kSH1 * z * c[2].z - kSH1 * x * c[3].z;
        if (degree > 1) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, yz = y * z, xz = x * z;
            const float q2[5] = {xy, yz, 2.f * zz - xx - yy, xz, xx - yy};
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                r.x += kSH2[k] * q2[k] * c[4 + k].x;
                r.y += kSH2[k] * q2[k] * c[4 + k].y;
                r.z += kSH2[k] * q2[k] * c[4 + k].z;
            }
            if (degree > 2) {
                const float q3[7] = {y * (3.f * xx - yy),      xy * z,
                                     y * (4.f * zz - xx - yy), z * (2.f * zz - 3.f * xx - 3.f * yy),
                                     x * (4.f * zz - xx - yy), z * (xx - yy),
                                     x * (xx - 3.f * yy)};
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    r.x += kSH3[k] * q3[k] * c[9 + k].x;
                    r.y += kSH3[k] * q3[k] * c[9 + k].y;
                    r.z += kSH3[k] * q3[k] * c[9 + k].z;
                }
            }
        }
    }
    r.x += 0.5f;
    r.y += 0.5f;
    r.z += 0.5f;
    clamp_bits = (r.x < 0.f ? 1u : 0u) | (r.y < 0.f ? 2u : 0u) | (r.z < 0.f ? 4u : 0u);
    return make_float3(fmaxf(r.x, 0.f), fmaxf(r.y, 0.f), fmaxf(r.z, 0.f));
}

// Adjoint of sh_color: writes dL/dcoefficients of the row into g (RGB triples,
// `bases` entries, zero beyond the active degree) and returns the view-direction
// part of dL/dmean.
template <bool kBasis = false>
__device__ __forceinline__ float3 sh_color_backward(const float3* c, int degree, int bases,
                                                    float3 pos, float3 campos, unsigned clamp_bits,
                                                    float3 dl, float3* g, float* wdl = nullptr) {
    const float3 d0 = make_float3(pos.x - campos.x, pos.y - campos.y, pos.z - campos.z);
    const float inv = rnorm3df(d0.x, d0.y, d0.z);
    const float x = d0.x * inv, y = d0.y * inv, z = d0.z * inv;
    if (clamp_bits & 1u) dl.x = 0.f;
    if (clamp_bits & 2u) dl.y = 0.f;
    if (clamp_bits & 4u) dl.z = 0.f;
    // Every base up to the active degree is written below; only the inactive
    // ones are zeroed here. kBasis: instead of the coefficient gradients
    // g[k] = w_k * dl, the basis values w_k go to wdl[k] and the clamped colour
    // gradient dl to wdl[16..18] (the gradient of coefficient (k, channel) is
    // then the single product w_k * dl.channel, the same rounding as g).
    auto put = [&](int k, float w) {
        if constexpr (kBasis)
            wdl[k] = w;
        else
            g[k] = make_float3(w * dl.x, w * dl.y, w * dl.z);
    };
    if constexpr (kBasis) {
        wdl[16] = dl.x;
        wdl[17] = dl.y;
        wdl[18] = dl.z;
    }
    for (int k = (degree + 1) * (degree + 1); k < bases; ++k)
        put(k, 0.f);
    put(0, kSH0);
    float3 gx = make_float3(0.f, 0.f, 0.f), gy = gx, gz = gx; // d colour / d dir
    if (degree > 0) {
        const float e1 = -kSH1 * y, e2 = kSH1 * z, e3 = -kSH1 * x;
        put(1, e1);
        put(2, e2);
        put(3, e3);
        gx = make_float3(-kSH1 * c[3].x, -kSH1 * c[3].y, -kSH1 * c[3].z);
        gy = make_float3(-kSH1 * c[1].x, -kSH1 * c[1].y, -kSH1 * c[1].z);
        gz = make_float3(kSH1 * c[2].x, kSH1 * c[2].y, kSH1 * c[2].z);
        if (degree > 1) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, yz = y * z, xz = x * z;
            const float q2[5] = {xy, yz, 2.f * zz - xx - yy, xz, xx - yy};
            const float q2x[5] = {y, 0.f, -2.f * x, z, 2.f * x};
            const float q2y[5] = {x, z, -2.f * y, 0.f, -2.f * y};
            const float q2z[5] = {0.f, y, 4.f * z, x, 0.f};
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const float w = kSH2[k] * q2[k];
                put(4 + k, w);
                const float3 ck = c[4 + k];
                gx.x += kSH2[k] * q2x[k] * ck.x; gx.y += kSH2[k] * q2x[k] * ck.y; gx.z += kSH2[k] * q2x[k] * ck.z;
                gy.x += kSH2[k] * q2y[k] * ck.x; gy.y += kSH2[k] * q2y[k] * ck.y; gy.z += kSH2[k] * q2y[k] * ck.z;
                gz.x += kSH2[k] * q2z[k] * ck.x; gz.y += kSH2[k] * q2z[k] * ck.y; gz.z += kSH2[k] * q2z[k] * ck.z;
            }
            if (degree > 2) {
                const float q3[7] = {y * (3.f * xx - yy),      xy * z,
                                     y * (4.f * zz - xx - yy), z * (2.f * zz - 3.f * xx - 3.f * yy),
                                     x * (4.f * zz - xx - yy), z * (xx - yy),
                                     x * (xx - 3.f * yy)};
                const float q3x[7] = {6.f * xy, yz, -2.f * xy, -6.f * xz,
                                      -3.f * xx + 4.f * zz - yy, 2.f * xz, 3.f * (xx - yy)};
                const float q3y[7] = {3.f * (xx - yy), xz, -3.f * yy + 4.f * zz - xx, -6.f * yz,
                                      -2.f * xy, -2.f * yz, -6.f * xy};
                const float q3z[7] = {0.f, xy, 8.f * yz, 3.f * (2.f * zz - xx - yy), 8.f * xz,
                                      xx - yy, 0.f};
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    const float w = kSH3[k] * q3[k];
                    put(9 + k, w);
                    const float3 ck = c[9 + k];
                    gx.x += kSH3[k] * q3x[k] * ck.x; gx.y += kSH3[k] * q3x[k] * ck.y; gx.z += kSH3[k] * q3x[k] * ck.z;
                    gy.x += kSH3[k] * q3y[k] * ck.x; gy.y += kSH3[k] * q3y[k] * ck.y; gy.z += kSH3[k] * q3y[k] * ck.z;
                    gz.x += kSH3[k] * q3z[k] * ck.x; gz.y += kSH3[k] * q3z[k] * ck.y; gz.z += kSH3[k] * q3z[k] * ck.z;
                }
            }
        }
    }
    // dL/ddir, then through dir = d0 / |d0|.
    const float ddx = gx.x * dl.x + gx.y * dl.y + gx.z * dl.z;
    const float ddy = gy.x * dl.x + gy.y * dl.y + gy.z * dl.z;
    const float ddz = gz.x * dl.x + gz.y * dl.y + gz.z * dl.z;
    const float dot = x * ddx + y * ddy + z * ddz;
    return make_float3((ddx - x * dot) * inv, (ddy - y * dot) * inv, (ddz - z * dot) * inv);
}

// Per-pixel Gaussian exponent with a fixed rounding sequence, so forward,
// backward and every re-evaluation agree bit for bit
// (third_party/splat_drender/src/device/geometry.cuh:26-33).
__device__ __forceinline__ float gaussian_power(float4 co, float dx, float dy) {
    const float xx = __fmul_rn(co.x, dx);
    const float yy = __fmul_rn(__fmul_rn(co.z, dy), dy);
    const float xy = __fmul_rn(__fmul_rn(co.y, dx), dy);
    return __fsub_rn(__fmul_rn(-0.5f, __fmaf_rn(dx, xx, yy)), xy);
}

} // namespace gsb
