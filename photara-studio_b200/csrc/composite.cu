// Per-tile front-to-back compositing and its reverse-order adjoint.
//
// Forward numerics follow blend_tile pass 1
// (third_party/splat_drender/src/render_forward.cu:341-416, :508-525):
//   power = gaussian_power(conic, mean - pixel); skip power > 0;
//   alpha = min(alpha_clip, o * exp(power)); skip alpha < 1/255;
//   T' = T (1 - alpha); T' < 1e-4 ends the pixel WITHOUT blending;
//   C += rgb * alpha * T;  out = C + T * bg, alpha_out = 1 - T.
// B200 organisation: one 128-thread CTA per 16x16 tile (two pixels per
// thread), Gaussian batches staged in shared memory; each warp (four pixel
// rows) rejects a Gaussian whose alpha >= 1/255 box (widened by one pixel, so
// the test can only drop work the per-pixel test would drop) misses its rows,
// and stops as soon as all of its 64 pixels are saturated.
//
// Backward: the reference restarts from stored 32-instance snapshots
// (render_backward.cu:156-519). Here each tile walks its list back to front
// from every pixel's last contributor, recovering T by T_i = T_{i+1}/(1-a_i)
// from the stored final transmittance (no per-pixel lists or snapshots), and
// reduces each Gaussian's 12 partial gradients (summed over the thread's two
// pixels) across the warp with a 13-shuffle reduce-scatter before
// shared-memory accumulation and one set of float4 global atomics per
// (Gaussian, tile).
#include "common.cuh"
#include "kernels.h"

namespace gsb {

// Two vertically adjacent pixels per thread: a 16x16 tile is 128 threads,
// warp w covers tile rows 4w..4w+3, lane l owns column (l & 15) and rows
// 4w + 2(l >> 4) + {0, 1}. Shared loads, warp culling and (in the backward)
// the warp reduction are amortised over 64 pixels instead of 32.
constexpr int kCompositeThreads = kTilePixels / 2;
constexpr int kBatch = 256; // Gaussians staged per round

struct TileStage {
    unsigned id[kBatch];
    float2 xy[kBatch];
    float4 co[kBatch];
    float4 rgb[kBatch];
    ushort4 bnd[kBatch];
};

__device__ __forceinline__ bool band_hit(ushort4 b, int x0, int y0) {
    // Warp pixels: x in [x0, x0+16), y in [y0, y0+4); box widened by 1 px so
    // the test can only drop Gaussians whose alpha is below 1/255 there.
    return int(b.x) - 1 < x0 + kTileW && int(b.y) + 1 > x0 && int(b.z) - 1 < y0 + 4 &&
           int(b.w) + 1 > y0;
}

__device__ __forceinline__ void stage_batch(TileStage& s, const unsigned* __restrict__ order,
                                            unsigned first, int cnt, const GaussianState& st,
                                            int tid) {
    for (int k = tid; k < cnt; k += kCompositeThreads) {
        const unsigned g = order[first + k];
        s.id[k] = g;
        s.xy[k] = st.mean2d[g];
        s.co[k] = st.conic[g];
        s.rgb[k] = st.rgb[g];
        s.bnd[k] = st.bounds[g];
    }
}

__global__ void __launch_bounds__(kCompositeThreads) composite_forward_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, float* __restrict__ out_color, float* __restrict__ out_alpha,
    float* __restrict__ pix_T, unsigned* __restrict__ pix_last, float* __restrict__ visibility) {
    __shared__ TileStage s;
    __shared__ unsigned char s_vis[kBatch];
    const int tile = blockIdx.x;
    const int tx = tile % K.grid_x, ty = tile / K.grid_x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int px = tx * kTileW + (lane & 15);
    const int py0 = ty * kTileH + 4 * warp + 2 * (lane >> 4);
    const int wx0 = tx * kTileW, wy0 = ty * kTileH + 4 * warp;
    const bool in0 = px < K.width && py0 < K.height;
    const bool in1 = px < K.width && py0 + 1 < K.height;
    const float fx = float(px), fy0 = float(py0), fy1 = float(py0 + 1);
    const uint2 range = ranges[tile];
    const int n = int(range.y - range.x);
    const float clip = K.alpha_clip;

    float T0 = 1.f, T1 = 1.f;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, b0 = 0.f, b1 = 0.f, b2 = 0.f;
    unsigned last0 = 0, last1 = 0;
    bool done0 = !in0, done1 = !in1;
    for (int k = tid; k < kBatch; k += kCompositeThreads)
        s_vis[k] = 0;

    for (int base = 0; base < n; base += kBatch) {
        if (__syncthreads_count(!(done0 && done1)) == 0)
            break;
        const int cnt = min(kBatch, n - base);
        stage_batch(s, order, range.x + base, cnt, st, tid);
        __syncthreads();
        if (!__all_sync(0xffffffffu, done0 && done1)) {
            for (int j = 0; j < cnt; ++j) {
                if (!band_hit(s.bnd[j], wx0, wy0))
                    continue;
                const float2 m = s.xy[j];
                const float4 co = s.co[j];
                const float dx = m.x - fx;
                bool blended = false;
                if (!done0) {
                    const float dy = m.y - fy0;
                    const float power = gaussian_power(co, dx, dy);
                    if (power <= 0.f) {
                        const float alpha = fminf(clip, co.w * expf(power));
                        if (alpha >= kAlphaFloor) {
                            const float test_t = T0 * (1.f - alpha);
                            if (test_t < kTransmittanceFloor) {
                                done0 = true;
                            } else {
                                const float w = alpha * T0;
                                const float4 c = s.rgb[j];
                                a0 += c.x * w;
                                a1 += c.y * w;
                                a2 += c.z * w;
                                T0 = test_t;
                                last0 = unsigned(base + j + 1);
                                blended = true;
                            }
                        }
                    }
                }
                if (!done1) {
                    const float dy = m.y - fy1;
                    const float power = gaussian_power(co, dx, dy);
                    if (power <= 0.f) {
                        const float alpha = fminf(clip, co.w * expf(power));
                        if (alpha >= kAlphaFloor) {
                            const float test_t = T1 * (1.f - alpha);
                            if (test_t < kTransmittanceFloor) {
                                done1 = true;
                            } else {
                                const float w = alpha * T1;
                                const float4 c = s.rgb[j];
                                b0 += c.x * w;
                                b1 += c.y * w;
                                b2 += c.z * w;
                                T1 = test_t;
                                last1 = unsigned(base + j + 1);
                                blended = true;
                            }
                        }
                    }
                }
                if (blended)
                    s_vis[j] = 1;
                if (__all_sync(0xffffffffu, done0 && done1))
                    break;
            }
        }
        __syncthreads();
        for (int k = tid; k < cnt; k += kCompositeThreads) {
            if (visibility && s_vis[k])
                visibility[s.id[k]] = 1.f;
            s_vis[k] = 0;
        }
    }
    const size_t P = size_t(K.width) * K.height;
    if (in0) {
        const size_t pid = size_t(py0) * K.width + px;
        out_color[pid] = a0 + T0 * bg.x;
        out_color[P + pid] = a1 + T0 * bg.y;
        out_color[2 * P + pid] = a2 + T0 * bg.z;
        out_alpha[pid] = 1.f - T0;
        if (pix_T) {
            pix_T[pid] = T0;
            pix_last[pid] = last0;
        }
    }
    if (in1) {
        const size_t pid = size_t(py0 + 1) * K.width + px;
        out_color[pid] = b0 + T1 * bg.x;
        out_color[P + pid] = b1 + T1 * bg.y;
        out_color[2 * P + pid] = b2 + T1 * bg.z;
        out_alpha[pid] = 1.f - T1;
        if (pix_T) {
            pix_T[pid] = T1;
            pix_last[pid] = last1;
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

// Per-pixel backward state.
struct PixBack {
    float T, sdot, T_final, gx, gy, gz, fin_term, refine_scale, dmap;
    unsigned last;
};

__device__ __forceinline__ void pixel_backward_init(PixBack& p, bool inside, size_t pid, size_t P,
                                                    float3 bg, const float* __restrict__ pix_T,
                                                    const unsigned* __restrict__ pix_last,
                                                    const float* __restrict__ dL_color,
                                                    const float* __restrict__ dL_alpha,
                                                    const float* __restrict__ densify_map,
                                                    int want_refine) {
    p.T_final = 1.f;
    p.gx = p.gy = p.gz = 0.f;
    p.dmap = 0.f;
    p.last = 0;
    float dfin = 0.f;
    if (inside) {
        p.T_final = pix_T[pid];
        p.last = pix_last[pid];
        p.gx = dL_color[pid];
        p.gy = dL_color[P + pid];
        p.gz = dL_color[2 * P + pid];
        dfin = bg.x * p.gx + bg.y * p.gy + bg.z * p.gz - (dL_alpha ? dL_alpha[pid] : 0.f);
        p.dmap = densify_map ? densify_map[pid] : 0.f;
    }
    p.refine_scale = want_refine ? 1.f / fmaxf(1.f - p.T_final, 1.0e-5f) : 0.f;
    p.fin_term = p.T_final * dfin;
    p.T = p.T_final;
    p.sdot = 0.f;
}

// Adds this pixel's contribution of Gaussian (m, co, c) to v; returns whether
// the Gaussian was blended at the pixel.
__device__ __forceinline__ bool pixel_backward_step(PixBack& p, unsigned pos, float2 m, float4 co,
                                                    float4 c, float fx, float fy, float clip,
                                                    float Wf, float Hf, int want_refine,
                                                    float (&v)[12]) {
    if (pos >= p.last)
        return false;
    const float dx = m.x - fx, dy = m.y - fy;
    const float power = gaussian_power(co, dx, dy);
    if (power > 0.f)
        return false;
    const float G = expf(power);
    const float alpha = fminf(clip, co.w * G);
    if (alpha < kAlphaFloor)
        return false;
    const float inv_1ma = 1.f / (1.f - alpha);
    p.T = p.T * inv_1ma;
    const float w = alpha * p.T;
    const float cdot = c.x * p.gx + c.y * p.gy + c.z * p.gz;
    const float dL_da = p.T * cdot - (p.sdot + p.fin_term) * inv_1ma;
    p.sdot += w * cdot;
    const float dL_dG = co.w * dL_da;
    const float gdx = G * dx, gdy = G * dy;
    const float dmx = dL_dG * (-gdx * co.x - gdy * co.y);
    const float dmy = dL_dG * (-gdy * co.z - gdx * co.y);
    v[0] += -0.5f * gdx * dx * dL_dG;
    v[1] += -0.5f * gdx * dy * dL_dG;
    v[2] += -0.5f * gdy * dy * dL_dG;
    v[3] += G * dL_da;
    v[4] += dmx;
    v[5] += dmy;
    if (want_refine) {
        const float rx = dmx * Wf, ry = dmy * Hf;
        v[6] += sqrtf(rx * rx + ry * ry) * p.refine_scale;
    }
    v[7] += p.dmap * w;
    v[8] += w * p.gx;
    v[9] += w * p.gy;
    v[10] += w * p.gz;
    v[11] += w;
    return true;
}

__global__ void __launch_bounds__(kCompositeThreads) composite_backward_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, const float* __restrict__ pix_T,
    const unsigned* __restrict__ pix_last, const float* __restrict__ dL_color,
    const float* __restrict__ dL_alpha, const float* __restrict__ densify_map, int want_refine) {
    __shared__ TileStage s;
    __shared__ float s_acc[kBatch][12];
    __shared__ unsigned s_wmax[4];
    const int tile = blockIdx.x;
    const int tx = tile % K.grid_x, ty = tile / K.grid_x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int px = tx * kTileW + (lane & 15);
    const int py0 = ty * kTileH + 4 * warp + 2 * (lane >> 4);
    const int wx0 = tx * kTileW, wy0 = ty * kTileH + 4 * warp;
    const bool in0 = px < K.width && py0 < K.height;
    const bool in1 = px < K.width && py0 + 1 < K.height;
    const float fx = float(px), fy0 = float(py0), fy1 = float(py0 + 1);
    const uint2 range = ranges[tile];
    const float clip = K.alpha_clip;
    const size_t P = size_t(K.width) * K.height;
    PixBack p0, p1;
    pixel_backward_init(p0, in0, in0 ? size_t(py0) * K.width + px : 0, P, bg, pix_T, pix_last,
                        dL_color, dL_alpha, densify_map, want_refine);
    pixel_backward_init(p1, in1, in1 ? size_t(py0 + 1) * K.width + px : 0, P, bg, pix_T,
                        pix_last, dL_color, dL_alpha, densify_map, want_refine);
    unsigned wlast = max(p0.last, p1.last);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        wlast = max(wlast, __shfl_xor_sync(0xffffffffu, wlast, o));
    if (lane == 0)
        s_wmax[warp] = wlast;
    for (int k = tid; k < kBatch * 12; k += kCompositeThreads)
        (&s_acc[0][0])[k] = 0.f;
    __syncthreads();
    unsigned tile_last = max(max(s_wmax[0], s_wmax[1]), max(s_wmax[2], s_wmax[3]));
    tile_last = min(tile_last, range.y - range.x);
    const float Wf = float(K.width), Hf = float(K.height);
    const int batches = int((tile_last + kBatch - 1) / kBatch);
    for (int b = batches - 1; b >= 0; --b) {
        const int base = b * kBatch;
        const int cnt = min(kBatch, int(tile_last) - base);
        stage_batch(s, order, range.x + base, cnt, st, tid);
        __syncthreads();
        const int jtop = min(cnt, int(wlast) - base) - 1;
        for (int j = jtop; j >= 0; --j) {
            if (!band_hit(s.bnd[j], wx0, wy0))
                continue;
            const unsigned pos = unsigned(base + j);
            const float2 m = s.xy[j];
            const float4 co = s.co[j];
            const float4 c = s.rgb[j];
            float v[12];
#pragma unroll
            for (int k = 0; k < 12; ++k)
                v[k] = 0.f;
            bool hit = pixel_backward_step(p0, pos, m, co, c, fx, fy0, clip, Wf, Hf, want_refine, v);
            hit |= pixel_backward_step(p1, pos, m, co, c, fx, fy1, clip, Wf, Hf, want_refine, v);
            const unsigned hits = __ballot_sync(0xffffffffu, hit);
            if (hits == 0)
                continue;
            if (__popc(hits) == 1) {
                // A single contributing lane adds its partials directly.
                if (hit) {
#pragma unroll
                    for (int k = 0; k < 12; ++k)
                        if (v[k] != 0.f)
                            atomicAdd(&s_acc[j][k], v[k]);
                }
                continue;
            }
            int slot;
            const float r = reduce_scatter12(v, slot);
            if (slot >= 0 && r != 0.f)
                atomicAdd(&s_acc[j][slot], r);
        }
        __syncthreads();
        for (int k = tid; k < cnt; k += kCompositeThreads) {
            float* a = s_acc[k];
            bool any = false;
#pragma unroll
            for (int q = 0; q < 12; ++q)
                any |= a[q] != 0.f;
            if (any) {
                float4* dst = st.grad + size_t(s.id[k]) * kGradSlots;
                atomicAdd(dst + 0, make_float4(a[0], a[1], a[2], a[3]));
                atomicAdd(dst + 1, make_float4(a[4], a[5], a[6], a[7]));
                atomicAdd(dst + 2, make_float4(a[8], a[9], a[10], densify_map ? a[11] : 0.f));
#pragma unroll
                for (int q = 0; q < 12; ++q)
                    a[q] = 0.f;
            }
        }
        __syncthreads();
    }
}

void launch_composite_forward(cudaStream_t s, int tiles, const uint2* ranges,
                              const unsigned* order, const GaussianState& st, const Camera& K,
                              float3 bg, float* color, float* alpha, float* pix_T,
                              unsigned* pix_last, float* visibility) {
    composite_forward_kernel<<<tiles, kCompositeThreads, 0, s>>>(ranges, order, st, K, bg, color,
                                                                 alpha, pix_T, pix_last,
                                                                 visibility);
}

void launch_composite_backward(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, const float* pix_T, const unsigned* pix_last,
                               const float* dL_color, const float* dL_alpha,
                               const float* densify_map, int want_refine) {
    composite_backward_kernel<<<tiles, kCompositeThreads, 0, s>>>(
        ranges, order, st, K, bg, pix_T, pix_last, dL_color, dL_alpha, densify_map, want_refine);
}

} // namespace gsb
