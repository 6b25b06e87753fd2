// Per-Gaussian projection adjoint (pinhole RGB EWA chain: conic, covariance
// cap, 3D covariance, Jacobian, pixel mean) and the chain to raw parameters,
// shared by the single-view and the batched per-Gaussian backward kernels.
//
// Reference behaviour followed:
//   splat_backward  third_party/splat_drender/src/device/geometry.cuh:317-912
//                   (ray-plane / normal chain :617-757)
//   raw chain       third_party/splat_drender/src/render_backward.cu:525-706
//                   (log scale with the 3D filter, quaternion normalisation,
//                   sigmoid logit)
#pragma once

#include "common.cuh"

namespace gsb {

// ----------------------------------------------------- projection adjoint --
struct ProjGrad {
    float3 d_mean;
    float3 d_scale; // w.r.t. activated scale
    float4 d_rot;   // w.r.t. normalised quaternion
    float d_opac;   // w.r.t. activated opacity
};

__device__ __forceinline__ float3 conic_cap_backward(float a, float b, float c, const CovCap& cap,
                                                     float4 dco) {
    const float x = a * cap.q, y = b * cap.q, z = c * cap.q;
    const float det = x * z - y * y;
    const float u = z / det, v = -y / det, w = x / det;
    const float ga = -(u * u * dco.x + 2.f * u * v * dco.y + v * v * dco.z);
    const float gb = -2.f * (u * v * dco.x + (u * w + v * v) * dco.y + v * w * dco.z);
    const float gc = -(v * v * dco.x + 2.f * v * w * dco.y + w * w * dco.z);
    const float pull = (ga * a + gb * b + gc * c) / cap.lambda;
    return make_float3(cap.q * (ga - pull * cap.da), cap.q * (gb - pull * cap.db),
                       cap.q * (gc - pull * cap.dc));
}

// Geometry-channel part of the projection adjoint (geometry.cuh:617-757,
// scale parameterisation, always well conditioned): the gradients of the ray
// plane (x, y: screen slopes stored divided by the focal lengths, z: peak
// distance |t|, w: 1/sigma along the ray) and of the footprint normal, back to
// the projected centre (u, v), the camera z and the world covariance V. The
// steps are the reference's, in its order; t is the clamped camera point,
// u = t.x / t.z, v = t.y / t.z.
struct GeoChain {
    float du, dv, dz;
    float dV[6]; // symmetric V gradient in the (00, 01, 02, 11, 12, 22) cov-local layout
};

__device__ __forceinline__ GeoChain geometry_chain(float3 t, float u, float v, const M3& W,
                                                   const M3& R, float3 sl, float4 dplane,
                                                   float3 dnormal, float fx, float fy) {
    GeoChain o;
    const float dpx = dplane.x / fx, dpy = dplane.y / fy, drs = dplane.w;
    const M3 S_inv = m3_diag(__frcp_rn(sl.x), __frcp_rn(sl.y), __frcp_rn(sl.z));
    const M3 SR_inv = m3_mul(S_inv, R);
    const M3 M_inv = m3_mul(SR_inv, W);
    const M3 cov_cam_inv = m3_mul(m3_t(M_inv), M_inv);
    const M3 V_inv = m3_mul(m3_t(SR_inv), SR_inv);
    const float3 uvh = make_float3(u, v, 1.f);
    const float3 uvh_m = m3_vec(cov_cam_inv, uvh);
    const float u2 = u * u, v2 = v * v;
    const float vb = uvh_m.x * uvh.x + uvh_m.y * uvh.y + uvh_m.z * uvh.z;
    const float l = norm3df(t.x, t.y, t.z);
    M3 nJ = m3_zero();
    const float iz = 1.f / t.z;
    nJ.m[0][0] = iz;
    nJ.m[0][2] = t.x / l;
    nJ.m[1][1] = iz;
    nJ.m[1][2] = t.y / l;
    nJ.m[2][0] = -t.x * iz * iz;
    nJ.m[2][1] = -t.y * iz * iz;
    nJ.m[2][2] = t.z / l;
    M3 nJ_inv = m3_zero();
    nJ_inv.m[0][0] = v2 + 1.f;
    nJ_inv.m[0][1] = -(u * v);
    nJ_inv.m[0][2] = -u;
    nJ_inv.m[1][0] = -(u * v);
    nJ_inv.m[1][1] = u2 + 1.f;
    nJ_inv.m[1][2] = -v;
    const float clamp_vb = fmaxf(vb, 1.0e-7f);
    const float ray_len2 = u2 + v2 + 1.f;
    const float ray_len_inv = rsqrtf(ray_len2);
    const float factor = l / ray_len2;
    const float3 q = make_float3(uvh_m.x / clamp_vb, uvh_m.y / clamp_vb, uvh_m.z / clamp_vb);
    const float3 plane = m3_vec(nJ_inv, q);
    const float3 rn = make_float3(-plane.x * factor, -plane.y * factor, -1.f);
    const float3 cn = m3_vec(nJ, rn);
    const float inv = rnorm3df(cn.x, cn.y, cn.z);
    const float3 nrm = make_float3(cn.x * inv, cn.y * inv, cn.z * inv);
    // normalisation adjoint of the pre-normalised camera normal
    const float ndl = nrm.x * dnormal.x + nrm.y * dnormal.y + nrm.z * dnormal.z;
    const float3 dcn = make_float3((dnormal.x - nrm.x * ndl) * inv, (dnormal.y - nrm.y * ndl) * inv,
                                   (dnormal.z - nrm.z * ndl) * inv);
    const float3 drn = m3_vec(m3_t(nJ), dcn);
    // dL/dnJ = dcn rn^T (element [r][c] = dcn_r rn_c)
    const float dfactor = plane.x * (-drn.x + dpx) + plane.y * (-drn.y + dpy);
    const float dplx = (-drn.x + dpx) * factor;
    const float dply = (-drn.y + dpy) * factor;
    const float3 dpa = make_float3(dplx, dply, 0.f);
    const float aux = dplx * plane.x + dply * plane.y;
    const float3 W_uvh = m3_vec(W, uvh);
    const float3 tmp = m3_vec(m3_t(nJ_inv), dpa);
    const float3 numer = make_float3(
        (cov_cam_inv.m[0][0] * tmp.x + cov_cam_inv.m[0][1] * tmp.y + cov_cam_inv.m[0][2] * tmp.z) /
            clamp_vb,
        (cov_cam_inv.m[1][0] * tmp.x + cov_cam_inv.m[1][1] * tmp.y + cov_cam_inv.m[1][2] * tmp.z) /
            clamp_vb,
        (cov_cam_inv.m[2][0] * tmp.x + cov_cam_inv.m[2][1] * tmp.y + cov_cam_inv.m[2][2] * tmp.z) /
            clamp_vb);
    const float3 duvh = make_float3(2.f * (-aux) * q.x + numer.x, 2.f * (-aux) * q.y + numer.y,
                                    2.f * (-aux) * q.z + numer.z);
    // rsigma = sqrt(vb / ray_len2): both depend on (u, v)
    const float rsigmat = sqrtf(vb / ray_len2);
    const float dlen2_x2 = -drs * rsigmat / ray_len2;
    const float du_sigma = dlen2_x2 * u + drs * rsigmat * q.x;
    const float dv_sigma = dlen2_x2 * v + drs * rsigmat * q.y;
    // nJ's dependence on (u, v, z) through t = z (u, v, 1)
    const float nj20 = dcn.x * rn.z, nj21 = dcn.y * rn.z, nj22 = dcn.z * rn.z; // at(2, c)
    const float nj02 = dcn.z * rn.x, nj12 = dcn.z * rn.y;                       // at(c, 2)
    const float nj00 = dcn.x * rn.x, nj11 = dcn.y * rn.y;
    const float aux_nJ = (-nj20 * u - nj21 * v - nj22) / ray_len2 * ray_len_inv;
    const float du_nJ = -nj02 / t.z + nj20 * ray_len_inv + aux_nJ * u;
    const float dv_nJ = -nj12 / t.z + nj21 * ray_len_inv + aux_nJ * v;
    const float dz_nJ = (nj00 + nj11 - nj02 * u - nj12 * v) / (-t.z * t.z);
    // nJ_inv's dependence on (u, v): dL/dnJ_inv = dpa q^T
    const float ni01 = dpa.y * q.x, ni10 = dpa.x * q.y; // at(0, 1), at(1, 0)
    const float ni11 = dpa.y * q.y, ni00 = dpa.x * q.x;
    const float ni20 = dpa.x * q.z, ni21 = dpa.y * q.z; // at(2, 0), at(2, 1)
    const float du_plane = duvh.x + (ni01 + ni10) * (-v) + 2.f * ni11 * u - ni20;
    const float dv_plane = duvh.y + (ni01 + ni10) * (-u) + 2.f * ni00 * v - ni21;
    const float aux_factor = dfactor * (-t.z / ray_len2 * ray_len_inv);
    o.du = du_nJ + du_plane + aux_factor * u + du_sigma;
    o.dv = dv_nJ + dv_plane + aux_factor * v + dv_sigma;
    o.dz = dz_nJ + dfactor * ray_len_inv;
    // world covariance through V^-1: dL/dV = -(V^-1 W uvh) (V^-1 rhs)^T / vb
    const float dvb_xvb = -aux + drs * 0.5f * rsigmat;
    const float3 rhs1 = m3_vec(W, tmp);
    const float3 rhs = make_float3(rhs1.x + W_uvh.x * dvb_xvb, rhs1.y + W_uvh.y * dvb_xvb,
                                   rhs1.z + W_uvh.z * dvb_xvb);
    const float3 lhs = m3_vec(V_inv, W_uvh);
    const float3 vr = m3_vec(V_inv, rhs);
    float dV[3][3];
    const float lh[3] = {lhs.x, lhs.y, lhs.z}, vv[3] = {-vr.x, -vr.y, -vr.z};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            dV[i][j] = lh[i] * vv[j] / vb;
    o.dV[0] = dV[0][0];
    o.dV[3] = dV[1][1];
    o.dV[5] = dV[2][2];
    o.dV[1] = dV[0][1] + dV[1][0];
    o.dV[2] = dV[0][2] + dV[2][0];
    o.dV[4] = dV[1][2] + dV[2][1];
    return o;
}

// kGeo: also differentiates the ray plane (dplane) and footprint normal
// (dnormal) of the median-depth / normal channels.
template <bool kGeo = false>
__device__ __forceinline__ ProjGrad projection_backward(float3 mean, const Camera& K, float3 scale,
                                                        float4 rot, float4 dco, float2 dm2,
                                                        float4 dplane = float4{},
                                                        float3 dnormal = float3{}) {
    ProjGrad o;
    const float fx = K.fx, fy = K.fy;
    float3 t = to_camera(mean, K.view);
    // the peak distance |t| of the ray plane, on the unclamped camera point
    float3 dt_tc = make_float3(0.f, 0.f, 0.f);
    if constexpr (kGeo) {
        const float rtc = rnorm3df(t.x, t.y, t.z);
        dt_tc = make_float3(t.x * rtc * dplane.z, t.y * rtc * dplane.z, t.z * rtc * dplane.z);
    }
    const float tan_fovx = float(K.width) / (2.f * fx);
    const float tan_fovy = float(K.height) / (2.f * fy);
    const float limx = 1.3f * tan_fovx, limy = 1.3f * tan_fovy;
    const float u0 = t.x / t.z, v0 = t.y / t.z;
    t.x = fminf(limx, fmaxf(-limx, u0)) * t.z;
    t.y = fminf(limy, fmaxf(-limy, v0)) * t.z;
    const float x_mul = (u0 < -limx || u0 > limx) ? 0.f : 1.f;
    const float y_mul = (v0 < -limy || v0 > limy) ? 0.f : 1.f;
    M3 J = m3_zero();
    J.m[0][0] = fx / t.z;
    J.m[1][1] = fy / t.z;
    J.m[2][0] = -(fx * t.x) / (t.z * t.z);
    J.m[2][1] = -(fy * t.y) / (t.z * t.z);
    const M3 W = view_rows(K.view);
    const M3 T = m3_mul(W, J);
    const float sm = K.scale_modifier;
    const float3 sl = make_float3(sm * scale.x, sm * scale.y, sm * scale.z);
    const M3 R = quat_to_rows(rot);
    const M3 SR = m3_mul(m3_diag(sl.x, sl.y, sl.z), R);
    const M3 M = m3_mul(SR, T);
    const M3 cov = m3_mul(m3_t(M), M);
    const M3 V = m3_mul(m3_t(SR), SR); // world covariance
    const float det0 = fmaxf(1.0e-6f, cov.m[0][0] * cov.m[1][1] - cov.m[0][1] * cov.m[0][1]);
    const float det1 = fmaxf(1.0e-6f, (cov.m[0][0] + K.kernel_size) * (cov.m[1][1] + K.kernel_size) -
                                          cov.m[0][1] * cov.m[0][1]);
    const float coef = K.compensate_2d ? sqrtf(det0 / det1) : 1.f;

    // Conic -> screen covariance (+ cap), opacity through the Mip coefficient.
    const float a = cov.m[0][0] + K.kernel_size, b = cov.m[0][1], c = cov.m[1][1] + K.kernel_size;
    const float denom = a * c - b * b;
    const float denom2inv = 1.f / (denom * denom + 1.0e-7f);
    float da = 0.f, db = 0.f, dc = 0.f;
    float dcl[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    o.d_opac = 0.f;
    const CovCap cap = cov_cap(a, b, c, K.width, K.height);
    // Columns of T as the rows of the 2x3 screen Jacobian: A = d(px)/d(world), B = d(py)/d(world).
    const float A0 = T.m[0][0], A1 = T.m[1][0], A2 = T.m[2][0];
    const float B0 = T.m[0][1], B1 = T.m[1][1], B2 = T.m[2][1];
    if (denom2inv != 0.f || cap.q < 1.f) {
        da = denom2inv * (-c * c * dco.x + 2.f * b * c * dco.y + (denom - a * c) * dco.z);
        dc = denom2inv * (-a * a * dco.z + 2.f * a * b * dco.y + (denom - a * c) * dco.x);
        db = denom2inv * 2.f * (b * c * dco.x - (denom + 2.f * b * b) * dco.y + a * b * dco.z);
        if (cap.q < 1.f) {
            const float3 g = conic_cap_backward(a, b, c, cap, dco);
            da = g.x;
            db = g.y;
            dc = g.z;
        }
        // Mip coefficient stays detached from the covariance gradient.
        o.d_opac = dco.w * coef;
        dcl[0] = A0 * A0 * da + A0 * B0 * db + B0 * B0 * dc;
        dcl[3] = A1 * A1 * da + A1 * B1 * db + B1 * B1 * dc;
        dcl[5] = A2 * A2 * da + A2 * B2 * db + B2 * B2 * dc;
        dcl[1] = 2.f * A0 * A1 * da + (A0 * B1 + A1 * B0) * db + 2.f * B0 * B1 * dc;
        dcl[2] = 2.f * A0 * A2 * da + (A0 * B2 + A2 * B0) * db + 2.f * B0 * B2 * dc;
        dcl[4] = 2.f * A2 * A1 * da + (A1 * B2 + A2 * B1) * db + 2.f * B1 * B2 * dc;
    }
    float geo_du = 0.f, geo_dv = 0.f, geo_dz = 0.f;
    if constexpr (kGeo) {
        // an unused geometry branch is exactly zero: skip its algebra (a very
        // thin splat could turn it into 0 * inf)
        if (dnormal.x != 0.f || dnormal.y != 0.f || dnormal.z != 0.f || dplane.x != 0.f ||
            dplane.y != 0.f || dplane.z != 0.f || dplane.w != 0.f) {
            const GeoChain gc = geometry_chain(t, t.x / t.z, t.y / t.z, W, R, sl, dplane,
                                               dnormal, fx, fy);
            geo_du = gc.du;
            geo_dv = gc.dv;
            geo_dz = gc.dz;
#pragma unroll
            for (int k = 0; k < 6; ++k)
                dcl[k] += gc.dV[k];
        }
    }

    // World covariance V = (S R)^T (S R) -> scale / rotation.
    {
        const float g00 = dcl[0], g11 = dcl[3], g22 = dcl[5];
        const float g01 = 0.5f * dcl[1], g02 = 0.5f * dcl[2], g12 = 0.5f * dcl[4];
        const float Gs[3][3] = {{g00, g01, g02}, {g01, g11, g12}, {g02, g12, g22}};
        // dL/dM = 2 M G with M = S R (rows scaled).
        float dM[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                dM[i][j] = 2.f * (SR.m[i][0] * Gs[0][j] + SR.m[i][1] * Gs[1][j] + SR.m[i][2] * Gs[2][j]);
        o.d_scale = make_float3(R.m[0][0] * dM[0][0] + R.m[0][1] * dM[0][1] + R.m[0][2] * dM[0][2],
                                R.m[1][0] * dM[1][0] + R.m[1][1] * dM[1][1] + R.m[1][2] * dM[1][2],
                                R.m[2][0] * dM[2][0] + R.m[2][1] * dM[2][1] + R.m[2][2] * dM[2][2]);
        o.d_scale = make_float3(o.d_scale.x * sm, o.d_scale.y * sm, o.d_scale.z * sm);
        // dL/dR = S dL/dM; Q[i][j] = dL/dR[i][j].
        float Q[3][3];
        const float s3[3] = {sl.x, sl.y, sl.z};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                Q[i][j] = s3[i] * dM[i][j];
        const float r = rot.x, x = rot.y, y = rot.z, z = rot.w;
        // R rows (quat_to_rows) differentiated w.r.t. (r, x, y, z).
        o.d_rot.x = 2.f * z * (Q[0][1] - Q[1][0]) + 2.f * y * (Q[2][0] - Q[0][2]) +
                    2.f * x * (Q[1][2] - Q[2][1]);
        o.d_rot.y = 2.f * y * (Q[0][1] + Q[1][0]) + 2.f * z * (Q[0][2] + Q[2][0]) +
                    2.f * r * (Q[1][2] - Q[2][1]) - 4.f * x * (Q[2][2] + Q[1][1]);
        o.d_rot.z = 2.f * x * (Q[0][1] + Q[1][0]) + 2.f * r * (Q[2][0] - Q[0][2]) +
                    2.f * z * (Q[1][2] + Q[2][1]) - 4.f * y * (Q[2][2] + Q[0][0]);
        o.d_rot.w = 2.f * r * (Q[0][1] - Q[1][0]) + 2.f * x * (Q[0][2] + Q[2][0]) +
                    2.f * y * (Q[1][2] + Q[2][1]) - 4.f * z * (Q[1][1] + Q[0][0]);
    }

    // Screen covariance -> T = W J -> J -> camera point.
    float dT0[3], dT1[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float va = A0 * V.m[0][j] + A1 * V.m[1][j] + A2 * V.m[2][j];
        const float vb = B0 * V.m[0][j] + B1 * V.m[1][j] + B2 * V.m[2][j];
        dT0[j] = 2.f * va * da + vb * db;
        dT1[j] = 2.f * vb * dc + va * db;
    }
    const float dJ00 = W.m[0][0] * dT0[0] + W.m[1][0] * dT0[1] + W.m[2][0] * dT0[2];
    const float dJ02 = W.m[0][2] * dT0[0] + W.m[1][2] * dT0[1] + W.m[2][2] * dT0[2];
    const float dJ11 = W.m[0][1] * dT1[0] + W.m[1][1] * dT1[1] + W.m[2][1] * dT1[2];
    const float dJ12 = W.m[0][2] * dT1[0] + W.m[1][2] * dT1[1] + W.m[2][2] * dT1[2];
    const float tz = 1.f / t.z, tz2 = tz * tz, tz3 = tz2 * tz;
    float3 gm;
    if constexpr (kGeo) {
        const float dtx = x_mul * (-fx * tz2 * dJ02 + geo_du * tz);
        const float dty = y_mul * (-fy * tz2 * dJ12 + geo_dv * tz);
        const float dtz = -fx * tz2 * dJ00 - fy * tz2 * dJ11 +
                          ((1.f + x_mul) * fx * t.x) * tz3 * dJ02 +
                          ((1.f + y_mul) * fy * t.y) * tz3 * dJ12 -
                          (x_mul * geo_du * t.x + y_mul * geo_dv * t.y) * tz2 + geo_dz;
        gm = to_world_dir(make_float3(dtx + dt_tc.x, dty + dt_tc.y, dtz + dt_tc.z), K.view);
    } else {
        const float dtx = x_mul * (-fx * tz2 * dJ02);
        const float dty = y_mul * (-fy * tz2 * dJ12);
        const float dtz = -fx * tz2 * dJ00 - fy * tz2 * dJ11 +
                          ((1.f + x_mul) * fx * t.x) * tz3 * dJ02 +
                          ((1.f + y_mul) * fy * t.y) * tz3 * dJ12;
        gm = to_world_dir(make_float3(dtx, dty, dtz), K.view);
    }

    // Pixel centre -> mean.
    {
        const float* v = K.view;
        const float3 pv = to_camera(mean, v);
        const float rz = 1.f / (pv.z + 1.0e-7f);
        const float sx = pv.x * rz, sy = pv.y * rz;
        gm.x += (fx * (v[0] - sx * v[2]) * dm2.x + fy * (v[1] - sy * v[2]) * dm2.y) * rz;
        gm.y += (fx * (v[4] - sx * v[6]) * dm2.x + fy * (v[5] - sy * v[6]) * dm2.y) * rz;
        gm.z += (fx * (v[8] - sx * v[10]) * dm2.x + fy * (v[9] - sy * v[10]) * dm2.y) * rz;
    }
    o.d_mean = gm;
    return o;
}

// Activated-space gradients -> raw parameter gradients (log scale with the 3D
// filter, quaternion normalisation Jacobian, sigmoid logit).
struct RawGrad {
    float log_s[3];
    float quat[4];
    float logit;
};

__device__ __forceinline__ RawGrad chain_to_raw(const ProjGrad& g, const Activated& act,
                                                const float* __restrict__ quats,
                                                const float* __restrict__ logits,
                                                const float* __restrict__ filter_3d, int i) {
    RawGrad r;
    const float f2 = filter_3d ? filter_3d[i] * filter_3d[i] : 0.f;
    const float ds[3] = {g.d_scale.x, g.d_scale.y, g.d_scale.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float raw = (&act.raw_scale.x)[k];
        const float s = (&act.scale.x)[k];
        r.log_s[k] = ds[k] * raw * raw / s + g.d_opac * act.opacity * f2 / (s * s);
    }
    const float4 q4 = reinterpret_cast<const float4*>(quats)[i];
    const float qw = q4.x, qx = q4.y, qy = q4.z, qz = q4.w;
    const float inv = rsqrtf(fmaxf(qw * qw + qx * qx + qy * qy + qz * qz, 1e-20f));
    const float q[4] = {qw * inv, qx * inv, qy * inv, qz * inv};
    const float dr[4] = {g.d_rot.x, g.d_rot.y, g.d_rot.z, g.d_rot.w};
    const float qdot = q[0] * dr[0] + q[1] * dr[1] + q[2] * dr[2] + q[3] * dr[3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        r.quat[k] = inv * (dr[k] - q[k] * qdot);
    const float sig = 1.f / (1.f + expf(-logits[i]));
    r.logit = g.d_opac * act.opacity * (1.f - sig);
    return r;
}

} // namespace gsb
