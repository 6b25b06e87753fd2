// Per-Gaussian projection adjoint (pinhole RGB EWA chain: conic, covariance
// cap, 3D covariance, Jacobian, pixel mean) and the chain to raw parameters,
// shared by the single-view and the batched per-Gaussian backward kernels.
//
// Reference behaviour followed:
//   splat_backward  third_party/splat_drender/src/device/geometry.cuh:317-912
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

__device__ __forceinline__ ProjGrad projection_backward(float3 mean, const Camera& K, float3 scale,
                                                        float4 rot, float4 dco, float2 dm2) {
    ProjGrad o;
    const float fx = K.fx, fy = K.fy;
    float3 t = to_camera(mean, K.view);
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
    const float dtx = x_mul * (-fx * tz2 * dJ02);
    const float dty = y_mul * (-fy * tz2 * dJ12);
    const float dtz = -fx * tz2 * dJ00 - fy * tz2 * dJ11 + ((1.f + x_mul) * fx * t.x) * tz3 * dJ02 +
                      ((1.f + y_mul) * fy * t.y) * tz3 * dJ12;
    float3 gm = to_world_dir(make_float3(dtx, dty, dtz), K.view);

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
