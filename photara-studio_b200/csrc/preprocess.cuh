// Per-Gaussian preprocess for one camera: world-to-camera projection, EWA
// screen covariance with the reference's cap, conic and opacity, tile-walk
// count, SH colour, radial depth and the alpha >= 1/255 pixel box.
//
// Reference behaviour followed:
//   preprocess_gaussians  third_party/splat_drender/src/render_forward.cu:30-139
// Shared by the single-view kernel (reference 16x16 tiles) and the batched
// kernel over (view, Gaussian) pairs (any tile shape of the batch schedule).
#pragma once

#include "common.cuh"

namespace gsb {

struct PreResult {
    unsigned touched;    // tiles overlapped (0: culled)
    unsigned depth_bits; // radial depth as ordered float bits (visible only)
    int radius;          // conservative pixel radius (0: culled)
};

// Writes the forward state of Gaussian i into slot `slot` of st when it is
// visible (touched > 0); st.touched / radii are left to the caller. kGeometry
// also writes the ray plane and normal of the median-depth channel.
template <int TW, int TH, bool kGeometry = false>
__device__ __forceinline__ PreResult preprocess_one(
    int i, size_t slot, const float* __restrict__ means, const float* __restrict__ log_scales,
    const float* __restrict__ quats, const float* __restrict__ logits,
    const float* __restrict__ filter_3d, const float* __restrict__ sh,
    const float* __restrict__ colors, int sh_degree, int sh_bases, const Camera& K,
    const GaussianState& st) {
    unsigned touched = 0;
    unsigned depth_bits = 0;
    int radius_out = 0;
    const float3 mean = make_float3(means[3 * i], means[3 * i + 1], means[3 * i + 2]);
    const float3 t = to_camera(mean, K.view);
    if (t.z > K.near_plane) {
        const Activated act = activate(log_scales, quats, logits, filter_3d, i);
        Cov2D cv = project_cov(mean, K, act.scale, act.rot);
        const CovCap cap = cov_cap(cv.a, cv.b, cv.c, K.width, K.height);
        if (cap.q < 1.f) {
            cv.a *= cap.q;
            cv.b *= cap.q;
            cv.c *= cap.q;
        }
        // Pixel centre from the unclamped camera point.
        const float iz = 1.f / t.z;
        const float px = t.x * iz * K.fx + K.cx;
        const float py = t.y * iz * K.fy + K.cy;
        const float det = cv.a * cv.c - cv.b * cv.b;
        if (det != 0.f) {
            const float det_inv = 1.f / det;
            const float4 co = make_float4(cv.c * det_inv, -cv.b * det_inv, cv.a * det_inv,
                                          act.opacity * cv.coef);
            const float mid = 0.5f * (cv.a + cv.c);
            const float root = sqrtf(fmaxf(0.1f, mid * mid - det));
            const float radius = ceilf(3.f * sqrtf(fmaxf(mid + root, mid - root)));
            const float2 m2 = make_float2(px, py);
            uint4 spans;
            touched = walk_count_spans<TW, TH>(m2, co, K.grid_x, K.grid_y, spans);
            if (touched > 0) {
                float3 rgb;
                unsigned clamp_bits = 0;
                const float3 campos = make_float3(K.center[0], K.center[1], K.center[2]);
                if (sh && sh_bases == 16 && (reinterpret_cast<uintptr_t>(sh) & 15) == 0) {
                    // Degree-3 row (192 bytes, 16-byte aligned): twelve 16-byte
                    // loads in flight at once instead of 48 scalar ones.
                    const float4* row = reinterpret_cast<const float4*>(sh) + size_t(i) * 12;
                    float4 q[12];
#pragma unroll
                    for (int k = 0; k < 12; ++k)
                        q[k] = __ldg(row + k);
                    float3 c[16];
                    const float* f = reinterpret_cast<const float*>(q);
#pragma unroll
                    for (int k = 0; k < 16; ++k)
                        c[k] = make_float3(f[3 * k], f[3 * k + 1], f[3 * k + 2]);
                    rgb = sh_color(c, sh_degree, mean, campos, clamp_bits);
                } else if (sh) {
                    rgb = sh_color(reinterpret_cast<const float3*>(sh) + size_t(i) * sh_bases,
                                   sh_degree, mean, campos, clamp_bits);
                } else {
                    rgb = make_float3(colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]);
                }
                st.mean2d[slot] = m2;
                st.conic[slot] = co;
                if constexpr (kGeometry) {
                    float4 pl;
                    float3 nm;
                    ray_plane_normal(mean, K, act.scale, act.rot, pl, nm);
                    st.plane[slot] = pl;
                    st.normal[slot] = make_float4(nm.x, nm.y, nm.z, 0.f);
                }
                st.rgb[slot] = make_float4(rgb.x, rgb.y, rgb.z, __uint_as_float(clamp_bits));
                depth_bits = __float_as_uint(norm3df(t.x, t.y, t.z));
                st.depth[slot] = depth_bits;
                radius_out = int(radius);
                const float threshold = 2.f * logf(co.w / kAlphaFloor);
                const float ex = sqrtf(fmaxf(0.f, threshold * cv.a));
                const float ey = sqrtf(fmaxf(0.f, threshold * cv.c));
                const ushort4 box = make_ushort4(
                    static_cast<unsigned short>(fmaxf(0.f, fminf(65535.f, floorf(px - ex)))),
                    static_cast<unsigned short>(fmaxf(0.f, fminf(65535.f, floorf(px + ex) + 1.f))),
                    static_cast<unsigned short>(fmaxf(0.f, fminf(65535.f, floorf(py - ey)))),
                    static_cast<unsigned short>(fmaxf(0.f, fminf(65535.f, floorf(py + ey) + 1.f))));
                st.bounds[slot] = box;
                if (st.rec) {
                    SplatRec r;
                    r.co = co;
                    r.rgb = make_float4(rgb.x, rgb.y, rgb.z, __uint_as_float(clamp_bits));
                    r.xy = m2;
                    r.bounds = box;
                    r.spans = spans;
                    st.rec[slot] = r;
                } else if (st.spans) {
                    st.spans[slot] = spans;
                }
            }
        }
    }
    return {touched, depth_bits, radius_out};
}

} // namespace gsb
