// Per-tile front-to-back compositing and its reverse-order adjoint.
//
// Forward numerics follow blend_tile pass 1
// (third_party/splat_drender/src/render_forward.cu:341-416, :508-525):
//   power = gaussian_power(conic, mean - pixel); skip power > 0;
//   alpha = min(alpha_clip, o * exp(power)); skip alpha < 1/255;
//   T' = T (1 - alpha); T' < 1e-4 ends the pixel WITHOUT blending;
//   C += rgb * alpha * T;  out = C + T * bg, alpha_out = 1 - T.
// B200 organisation: one 256-thread CTA per 16x16 tile, Gaussian batches
// staged in shared memory; each warp (two pixel rows) rejects a Gaussian
// whose alpha >= 1/255 box (widened by one pixel, so the test can only drop
// work the per-pixel test would drop) misses its rows, and stops as soon as
// all of its 32 pixels are saturated.
//
// Backward: the reference restarts from stored 32-instance snapshots
// (render_backward.cu:156-519). Here each tile walks its list back to front
// from every pixel's last contributor, recovering T by T_i = T_{i+1}/(1-a_i)
// from the stored final transmittance (no per-pixel lists or snapshots), and
// reduces each Gaussian's 12 partial gradients across the warp with a
// 13-shuffle reduce-scatter before shared-memory accumulation and one set of
// float4 global atomics per (Gaussian, tile).
#include "common.cuh"
#include "kernels.h"

namespace gsb {

struct TileStage {
    unsigned id[kTilePixels];
    float2 xy[kTilePixels];
    float4 co[kTilePixels];
    float4 rgb[kTilePixels];
    ushort4 bnd[kTilePixels];
};

__device__ __forceinline__ bool warp_rect_hit(ushort4 b, int x0, int y0) {
    // Warp pixels: x in [x0, x0+16), y in [y0, y0+2); box widened by 1 px.
    return int(b.x) - 1 < x0 + kTileW && int(b.y) + 1 > x0 && int(b.z) - 1 < y0 + 2 &&
           int(b.w) + 1 > y0;
}

__global__ void __launch_bounds__(kTilePixels) composite_forward_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, float* __restrict__ out_color, float* __restrict__ out_alpha,
    float* __restrict__ pix_T, unsigned* __restrict__ pix_last, float* __restrict__ visibility) {
    __shared__ TileStage s;
    __shared__ unsigned char s_vis[kTilePixels];
    const int tile = blockIdx.x;
    const int tx = tile % K.grid_x, ty = tile / K.grid_x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int px = tx * kTileW + (tid & 15);
    const int py = ty * kTileH + (tid >> 4);
    const int wx0 = tx * kTileW, wy0 = ty * kTileH + 2 * warp;
    const bool inside = px < K.width && py < K.height;
    const float fx = float(px), fy = float(py);
    const uint2 range = ranges[tile];
    const int n = int(range.y - range.x);
    const float clip = K.alpha_clip;

    float T = 1.f;
    float c0 = 0.f, c1 = 0.f, c2 = 0.f;
    unsigned last = 0;
    bool done = !inside;
    s_vis[tid] = 0;

    for (int base = 0; base < n; base += kTilePixels) {
        if (__syncthreads_count(!done) == 0)
            break;
        const int idx = base + tid;
        if (idx < n) {
            const unsigned g = order[range.x + idx];
            s.id[tid] = g;
            s.xy[tid] = st.mean2d[g];
            s.co[tid] = st.conic[g];
            s.rgb[tid] = st.rgb[g];
            s.bnd[tid] = st.bounds[g];
        }
        __syncthreads();
        const int cnt = min(kTilePixels, n - base);
        if (!__all_sync(0xffffffffu, done)) {
            for (int j = 0; j < cnt; ++j) {
                if (!warp_rect_hit(s.bnd[j], wx0, wy0))
                    continue;
                if (!done) {
                    const float2 m = s.xy[j];
                    const float4 co = s.co[j];
                    const float dx = m.x - fx, dy = m.y - fy;
                    const float power = gaussian_power(co, dx, dy);
                    if (power <= 0.f) {
                        const float alpha = fminf(clip, co.w * expf(power));
                        if (alpha >= kAlphaFloor) {
                            const float test_t = T * (1.f - alpha);
                            if (test_t < kTransmittanceFloor) {
                                done = true;
                            } else {
                                const float w = alpha * T;
                                const float4 c = s.rgb[j];
                                c0 += c.x * w;
                                c1 += c.y * w;
                                c2 += c.z * w;
                                T = test_t;
                                last = unsigned(base + j + 1);
                                s_vis[j] = 1;
                            }
                        }
                    }
                }
                if (__all_sync(0xffffffffu, done))
                    break;
            }
        }
        __syncthreads();
        if (visibility && idx < n && s_vis[tid]) {
            visibility[s.id[tid]] = 1.f;
        }
        s_vis[tid] = 0;
    }
    if (inside) {
        const size_t P = size_t(K.width) * K.height;
        const size_t pid = size_t(py) * K.width + px;
        out_color[pid] = c0 + T * bg.x;
        out_color[P + pid] = c1 + T * bg.y;
        out_color[2 * P + pid] = c2 + T * bg.z;
        out_alpha[pid] = 1.f - T;
        if (pix_T) {
            pix_T[pid] = T;
            pix_last[pid] = last;
        }
    }
}

// Reduce 12 per-lane values across the warp; returns the summed value of
// slot `slot` (or slot = -1 for lanes that hold nothing).
__device__ __forceinline__ float reduce_scatter12(const float (&v)[12], int& slot) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
    float u[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float send = b4 ? v[k] : v[k + 6];
        const float keep = b4 ? v[k + 6] : v[k];
        u[k] = keep + __shfl_xor_sync(full, send, 16);
    }
    float w[4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float send = b3 ? u[k] : u[k + 3];
        const float keep = b3 ? u[k + 3] : u[k];
        w[k] = keep + __shfl_xor_sync(full, send, 8);
    }
    w[3] = 0.f;
    float x[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float send = b2 ? w[k] : w[k + 2];
        const float keep = b2 ? w[k + 2] : w[k];
        x[k] = keep + __shfl_xor_sync(full, send, 4);
    }
    const float send = b1 ? x[0] : x[1];
    const float keep = b1 ? x[1] : x[0];
    float y = keep + __shfl_xor_sync(full, send, 2);
    y += __shfl_xor_sync(full, y, 1);
    const int idx = b2 ? (b1 ? -1 : 2) : (b1 ? 1 : 0);
    slot = (idx < 0 || (lane & 1)) ? -1 : (b4 ? 6 : 0) + (b3 ? 3 : 0) + idx;
    return y;
}

__global__ void __launch_bounds__(kTilePixels) composite_backward_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, const float* __restrict__ pix_T,
    const unsigned* __restrict__ pix_last, const float* __restrict__ dL_color,
    const float* __restrict__ dL_alpha, const float* __restrict__ densify_map, int want_refine) {
    __shared__ TileStage s;
    __shared__ float s_acc[kTilePixels][12];
    __shared__ unsigned s_wmax[8];
    const int tile = blockIdx.x;
    const int tx = tile % K.grid_x, ty = tile / K.grid_x;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int px = tx * kTileW + (tid & 15);
    const int py = ty * kTileH + (tid >> 4);
    const int wx0 = tx * kTileW, wy0 = ty * kTileH + 2 * warp;
    const bool inside = px < K.width && py < K.height;
    const float fx = float(px), fy = float(py);
    const uint2 range = ranges[tile];
    const float clip = K.alpha_clip;
    const size_t P = size_t(K.width) * K.height;
    const size_t pid = inside ? size_t(py) * K.width + px : 0;

    float T_final = 1.f, gx = 0.f, gy = 0.f, gz = 0.f, dfin = 0.f, dmap = 0.f;
    unsigned last = 0;
    if (inside) {
        T_final = pix_T[pid];
        last = pix_last[pid];
        gx = dL_color[pid];
        gy = dL_color[P + pid];
        gz = dL_color[2 * P + pid];
        dfin = bg.x * gx + bg.y * gy + bg.z * gz - (dL_alpha ? dL_alpha[pid] : 0.f);
        dmap = densify_map ? densify_map[pid] : 0.f;
    }
    const float refine_scale = want_refine ? 1.f / fmaxf(1.f - T_final, 1.0e-5f) : 0.f;
    const float fin_term = T_final * dfin;
    unsigned wlast = last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        wlast = max(wlast, __shfl_xor_sync(0xffffffffu, wlast, o));
    if ((tid & 31) == 0)
        s_wmax[warp] = wlast;
#pragma unroll
    for (int k = 0; k < 12; ++k)
        s_acc[tid][k] = 0.f;
    __syncthreads();
    unsigned tile_last = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w)
        tile_last = max(tile_last, s_wmax[w]);
    tile_last = min(tile_last, range.y - range.x);

    float T = T_final;
    float sdot = 0.f; // sum over later Gaussians of alpha*T*(c . g)
    const float Wf = float(K.width), Hf = float(K.height);
    const int batches = int((tile_last + kTilePixels - 1) / kTilePixels);
    for (int b = batches - 1; b >= 0; --b) {
        const int base = b * kTilePixels;
        const int cnt = min(kTilePixels, int(tile_last) - base);
        if (tid < cnt) {
            const unsigned g = order[range.x + base + tid];
            s.id[tid] = g;
            s.xy[tid] = st.mean2d[g];
            s.co[tid] = st.conic[g];
            s.rgb[tid] = st.rgb[g];
            s.bnd[tid] = st.bounds[g];
        }
        __syncthreads();
        const int jtop = min(cnt, int(wlast) - base) - 1;
        for (int j = jtop; j >= 0; --j) {
            if (!warp_rect_hit(s.bnd[j], wx0, wy0))
                continue;
            const unsigned pos = unsigned(base + j);
            bool hit = false;
            float dx = 0.f, dy = 0.f, G = 0.f, alpha = 0.f;
            float4 co = make_float4(0.f, 0.f, 0.f, 0.f);
            if (pos < last) {
                const float2 m = s.xy[j];
                co = s.co[j];
                dx = m.x - fx;
                dy = m.y - fy;
                const float power = gaussian_power(co, dx, dy);
                if (power <= 0.f) {
                    G = expf(power);
                    alpha = fminf(clip, co.w * G);
                    hit = alpha >= kAlphaFloor;
                }
            }
            if (!__any_sync(0xffffffffu, hit))
                continue;
            float v[12];
#pragma unroll
            for (int k = 0; k < 12; ++k)
                v[k] = 0.f;
            if (hit) {
                const float inv_1ma = 1.f / (1.f - alpha);
                T = T * inv_1ma;
                const float w = alpha * T;
                const float4 c = s.rgb[j];
                const float cdot = c.x * gx + c.y * gy + c.z * gz;
                const float dL_da = T * cdot - (sdot + fin_term) * inv_1ma;
                sdot += w * cdot;
                const float dL_dG = co.w * dL_da;
                const float gdx = G * dx, gdy = G * dy;
                const float dG_ddx = -gdx * co.x - gdy * co.y;
                const float dG_ddy = -gdy * co.z - gdx * co.y;
                const float dmx = dL_dG * dG_ddx;
                const float dmy = dL_dG * dG_ddy;
                v[0] = -0.5f * gdx * dx * dL_dG;
                v[1] = -0.5f * gdx * dy * dL_dG;
                v[2] = -0.5f * gdy * dy * dL_dG;
                v[3] = G * dL_da;
                v[4] = dmx;
                v[5] = dmy;
                if (want_refine) {
                    const float rx = dmx * Wf, ry = dmy * Hf;
                    v[6] = sqrtf(rx * rx + ry * ry) * refine_scale;
                }
                v[7] = dmap * w;
                v[8] = w * gx;
                v[9] = w * gy;
                v[10] = w * gz;
                v[11] = w;
            }
            int slot;
            const float r = reduce_scatter12(v, slot);
            if (slot >= 0 && r != 0.f)
                atomicAdd(&s_acc[j][slot], r);
        }
        __syncthreads();
        if (tid < cnt) {
            float* a = s_acc[tid];
            bool any = false;
#pragma unroll
            for (int k = 0; k < 12; ++k)
                any |= a[k] != 0.f;
            if (any) {
                float4* dst = st.grad + size_t(s.id[tid]) * kGradSlots;
                atomicAdd(dst + 0, make_float4(a[0], a[1], a[2], a[3]));
                atomicAdd(dst + 1, make_float4(a[4], a[5], a[6], a[7]));
                atomicAdd(dst + 2, make_float4(a[8], a[9], a[10], densify_map ? a[11] : 0.f));
#pragma unroll
                for (int k = 0; k < 12; ++k)
                    a[k] = 0.f;
            }
        }
        __syncthreads();
    }
}

void launch_composite_forward(cudaStream_t s, int tiles, const uint2* ranges,
                              const unsigned* order, const GaussianState& st, const Camera& K,
                              float3 bg, float* color, float* alpha, float* pix_T,
                              unsigned* pix_last, float* visibility) {
    composite_forward_kernel<<<tiles, kTilePixels, 0, s>>>(ranges, order, st, K, bg, color, alpha,
                                                           pix_T, pix_last, visibility);
}

void launch_composite_backward(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, const float* pix_T, const unsigned* pix_last,
                               const float* dL_color, const float* dL_alpha,
                               const float* densify_map, int want_refine) {
    composite_backward_kernel<<<tiles, kTilePixels, 0, s>>>(ranges, order, st, K, bg, pix_T,
                                                            pix_last, dL_color, dL_alpha,
                                                            densify_map, want_refine);
}

} // namespace gsb
