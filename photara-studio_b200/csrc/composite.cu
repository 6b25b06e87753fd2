// Single-view compositing kernels: one CTA per reference 16x16 tile running
// the per-tile forward / adjoint of composite.cuh (numerics and organisation
// described there; reference: third_party/splat_drender/src/render_forward.cu
// :341-416, :508-525 and render_backward.cu:156-519).
#include "composite.cuh"
#include "kernels.h"

namespace gsb {

// Single view: one CTA per reference 16x16 tile.
template <int PX>
__global__ void __launch_bounds__(TileGeom<kTileW, kTileH, PX>::kThreads) composite_forward_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, float* __restrict__ out_color, float* __restrict__ out_alpha,
    float* __restrict__ pix_T, unsigned* __restrict__ pix_last, float* __restrict__ visibility) {
    using G = TileGeom<kTileW, kTileH, PX>;
    __shared__ TileStage<G::kBatch> s;
    __shared__ unsigned char s_vis[G::kBatch];
    for (int k = threadIdx.x; k < G::kBatch; k += G::kThreads)
        s_vis[k] = 0;
    const int tile = blockIdx.x;
    const ViewTarget o{K.width, K.height, K.alpha_clip, bg, out_color, out_alpha, pix_T, pix_last};
    composite_forward_tile<kTileW, kTileH, PX>(s, s_vis, tile % K.grid_x, tile / K.grid_x,
                                               ranges[tile], order, st, o, visibility);
}

// Four pixels per thread: capped at 96 registers (no spills) for 10 resident
// CTAs per SM instead of 8 (0.700 -> 0.684 ms at 1M Gaussians, 1080p; the
// 80-register cap for 12 CTAs spills and measured slower).
template <int PX, bool kRefine, bool kDensify>
__global__ void __launch_bounds__(TileGeom<kTileW, kTileH, PX>::kThreads, PX == 4 ? 10 : 1)
    composite_backward_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, const float* __restrict__ pix_T,
    const unsigned* __restrict__ pix_last, const float* __restrict__ dL_color,
    const float* __restrict__ dL_alpha, const float* __restrict__ densify_map) {
    using G = TileGeom<kTileW, kTileH, PX>;
    __shared__ BackStage<G::kBatch> sb;
    __shared__ unsigned s_wmax[G::kWarps];
    for (int k = threadIdx.x; k < G::kBatch * 12; k += G::kThreads)
        (&sb.acc[0][0])[k] = 0.f;
    const int tile = blockIdx.x;
    const ViewGrads o{K.width, K.height, K.alpha_clip, bg, pix_T, pix_last, dL_color, dL_alpha,
                      densify_map};
    composite_backward_tile<kTileW, kTileH, PX, kRefine, kDensify>(
        sb, s_wmax, tile % K.grid_x, tile / K.grid_x, ranges[tile], order, st, o);
}

// ------------------------------------------------- geometry channels ----
// Forward with the median-depth and normal channels (render_forward.cu
// :274-525, blend_tile<GEOMETRY = true>): one thread per pixel of a 16x16
// tile. Pass 1 is the colour forward (the same per-pixel arithmetic as the
// colour kernels, so colour, alpha, final transmittance and last contributor
// are bit-identical to them) plus the alpha-weighted footprint normal and the
// depth seed (the ray-plane depth of the last Gaussian blended while the
// transmittance was above 0.5). Pass 2 finds the depth at which the
// transmittance along the ray crosses 0.5: each Gaussian is a 1D Gaussian
// along the ray around its plane depth, and the pixel's transmittance at a
// probe depth is the product of the Gaussians' partial opacities there; 8
// probes over a +-0.4 window around the seed, refined 5 times (every
// refinement walks the tile's list up to the pixel's last contributor again),
// then linear interpolation inside the final bracket.
constexpr int kDepthSplit = 8;
constexpr int kDepthRefinements = 5;
constexpr float kDepthSeedWindow = 0.4f;
constexpr float kDepthMinTransmittance = 0.45f;
constexpr int kGeoThreads = kTileW * kTileH;

__global__ void __launch_bounds__(kGeoThreads) composite_geometry_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, float* __restrict__ out_color, float* __restrict__ out_alpha,
    float* __restrict__ pix_T, unsigned* __restrict__ pix_last, float* __restrict__ visibility,
    float* __restrict__ out_depth, float* __restrict__ out_normal) {
    __shared__ unsigned s_id[kGeoThreads];
    __shared__ float2 s_xy[kGeoThreads];
    __shared__ float4 s_co[kGeoThreads];
    __shared__ float4 s_rgb[kGeoThreads];
    __shared__ float4 s_plane[kGeoThreads];
    __shared__ float4 s_nrm[kGeoThreads];
    __shared__ unsigned s_warp[kGeoThreads / 32];
    const int tile = blockIdx.x;
    const int tx = tile % K.grid_x, ty = tile / K.grid_x;
    const int tid = threadIdx.x;
    const int px = tx * kTileW + tid % kTileW, py = ty * kTileH + tid / kTileW;
    const bool inside = px < K.width && py < K.height;
    const float fx = float(px), fy = float(py);
    const uint2 range = ranges[tile];
    const int n = int(range.y - range.x);
    const float clip = K.alpha_clip;

    // ---- pass 1: colour, alpha, normal, depth seed ----
    float T = 1.f, cr = 0.f, cg = 0.f, cb = 0.f;
    float nx = 0.f, ny = 0.f, nz = 0.f, seed = 0.f;
    unsigned last = 0;
    bool done = !inside;
    for (int base = 0; base < n; base += kGeoThreads) {
        if (__syncthreads_and(done))
            break;
        if (base + tid < n) {
            const unsigned g = order[range.x + base + tid];
            s_id[tid] = g;
            s_xy[tid] = st.mean2d[g];
            s_co[tid] = st.conic[g];
            s_rgb[tid] = st.rgb[g];
            s_plane[tid] = st.plane[g];
            s_nrm[tid] = st.normal[g];
        }
        __syncthreads();
        const int cnt = min(kGeoThreads, n - base);
        for (int j = 0; !done && j < cnt; ++j) {
            const float dx = s_xy[j].x - fx, dy = s_xy[j].y - fy;
            const float4 co = s_co[j];
            const float power = gaussian_power(co, dx, dy);
            if (power > 0.f)
                continue;
            const float alpha = fminf(clip, co.w * expf(power));
            if (alpha < kAlphaFloor)
                continue;
            const float test_t = T * (1.f - alpha);
            if (test_t < kTransmittanceFloor) {
                done = true;
                continue;
            }
            const float w = alpha * T;
            const float4 c = s_rgb[j];
            cr += c.x * w;
            cg += c.y * w;
            cb += c.z * w;
            const float4 rp = s_plane[j];
            const float4 nm = s_nrm[j];
            const float t = rp.x * dx + rp.y * dy + rp.z;
            nx += nm.x * w;
            ny += nm.y * w;
            nz += nm.z * w;
            seed = T > 0.5f ? t : seed;
            if (visibility)
                visibility[s_id[j]] = 1.f;
            T = test_t;
            last = unsigned(base + j + 1);
        }
    }
    // the tile's furthest last contributor bounds pass 2
    unsigned wmax = last;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, off));
    if ((tid & 31) == 0)
        s_warp[tid >> 5] = wmax;
    __syncthreads();
    unsigned block_max = 0;
#pragma unroll
    for (int w = 0; w < kGeoThreads / 32; ++w)
        block_max = max(block_max, s_warp[w]);

    // ---- pass 2: median-depth bisection ----
    constexpr int S = kDepthSplit;
    float depth_min = fmaxf(seed - kDepthSeedWindow, 0.f);
    float depth_max = fmaxf(seed + kDepthSeedWindow, 0.f);
    bool in_range = T <= kDepthMinTransmittance;
    float Tp[S + 1];
#pragma unroll
    for (int r = 0; r < kDepthRefinements; ++r) {
        const bool first = r == 0;
#pragma unroll
        for (int k = 0; k <= S; ++k)
            if (first || (k > 0 && k < S))
                Tp[k] = 1.f;
        const float interval = (depth_max - depth_min) * (1.f / float(S));
        bool ldone = !in_range;
        unsigned seen = 0;
        for (int base = 0; base < int(block_max); base += kGeoThreads) {
            if (__syncthreads_and(ldone))
                break;
            if (base + tid < int(block_max)) {
                const unsigned g = order[range.x + base + tid];
                s_xy[tid] = st.mean2d[g];
                s_co[tid] = st.conic[g];
                s_plane[tid] = st.plane[g];
            }
            __syncthreads();
            const int cnt = min(kGeoThreads, int(block_max) - base);
            for (int j = 0; !ldone && j < cnt; ++j) {
                ++seen;
                ldone = seen >= last;
                const float dx = s_xy[j].x - fx, dy = s_xy[j].y - fy;
                const float4 co = s_co[j];
                const float power = gaussian_power(co, dx, dy);
                if (power > 0.f)
                    continue;
                const float alpha = fminf(clip, co.w * expf(power));
                if (alpha < kAlphaFloor)
                    continue;
                const float4 rp = s_plane[j];
                const float t_peak = rp.x * dx + rp.y * dy + rp.z;
                const float rsigma = rp.w;
                const bool ball = rsigma > 0.f;
                // Beyond 8 sigma of the peak a probe's Gaussian factor is
                // exactly 0 in the product (alpha g < 2^-25, so 1 - alpha g
                // rounds to 1 and its inverse square root is 1): the probe
                // takes (1 - alpha) behind the peak and 1 in front of it. A
                // Gaussian whose peak is over 8 sigma behind every probe
                // changes nothing; one over 8 sigma in front scales all.
                const int k0 = first ? 0 : 1, k1 = first ? S : S - 1;
                const float d_lo = (depth_min + interval * float(k0) - t_peak) * rsigma;
                const float d_hi = (depth_min + interval * float(k1) - t_peak) * rsigma;
                if (ball && d_hi < -8.f)
                    continue;
                const float oma = 1.f - alpha;
                if (!ball || d_lo > 8.f) {
#pragma unroll
                    for (int k = 0; k <= S; ++k) {
                        if (!(first || (k > 0 && k < S)))
                            continue;
                        const float ts = depth_min + interval * float(k);
                        Tp[k] *= ts > t_peak ? oma : 1.f;
                    }
                    continue;
                }
#pragma unroll
                for (int k = 0; k <= S; ++k) {
                    if (!(first || (k > 0 && k < S)))
                        continue;
                    const float ts = depth_min + interval * float(k);
                    const float delta = (ts - t_peak) * rsigma;
                    if (delta * delta > 64.f) {
                        Tp[k] *= ts > t_peak ? oma : 1.f;
                        continue;
                    }
                    const float gk = expf(-0.5f * delta * delta);
                    const float omg = 1.f - alpha * gk;
                    const float rv = rsqrtf(omg);
                    Tp[k] *= (ts > t_peak ? oma : omg) * rv;
                }
            }
        }
        if (first)
            in_range = Tp[0] >= 0.5f && Tp[S] <= 0.5f && in_range;
        int start = 0;
#pragma unroll
        for (int k = 1; k < S; ++k)
            start = Tp[k] >= 0.5f ? k : start;
        // Tp indices are compile-time after unrolling: pick the bracket ends
        // with selects.
        float lo_T = Tp[0], hi_T = Tp[1];
#pragma unroll
        for (int k = 1; k < S; ++k) {
            lo_T = start == k ? Tp[k] : lo_T;
            hi_T = start == k ? Tp[k + 1] : hi_T;
        }
        depth_max = depth_min + float(start + 1) * interval;
        depth_min = depth_min + float(start + 0) * interval;
        Tp[0] = lo_T;
        Tp[S] = hi_T;
    }
    const float w_max = __saturatef((Tp[0] - 0.5f) / (Tp[0] - Tp[S]));
    const float w_min = 1.f - w_max;
    const float median = in_range ? w_max * depth_max + w_min * depth_min : 0.f;

    if (inside) {
        const size_t P = size_t(K.width) * K.height;
        const size_t pid = size_t(py) * K.width + px;
        out_color[pid] = cr + T * bg.x;
        out_color[P + pid] = cg + T * bg.y;
        out_color[2 * P + pid] = cb + T * bg.z;
        out_alpha[pid] = 1.f - T;
        if (pix_T) {
            pix_T[pid] = T;
            pix_last[pid] = last;
        }
        out_depth[pid] = median * pixel_ray_z(fx, fy, K);
        const float len = 1.f - T;
        out_normal[pid] = last ? nx / len : 0.f;
        out_normal[P + pid] = last ? ny / len : 0.f;
        out_normal[2 * P + pid] = last ? nz / len : 0.f;
    }
}

void launch_composite_geometry(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, float* color, float* alpha, float* pix_T,
                               unsigned* pix_last, float* visibility, float* median_depth,
                               float* normal) {
    composite_geometry_kernel<<<tiles, kGeoThreads, 0, s>>>(ranges, order, st, K, bg, color,
                                                            alpha, pix_T, pix_last, visibility,
                                                            median_depth, normal);
}

void launch_composite_forward(cudaStream_t s, int tiles, const uint2* ranges,
                              const unsigned* order, const GaussianState& st, const Camera& K,
                              float3 bg, float* color, float* alpha, float* pix_T,
                              unsigned* pix_last, float* visibility, int pixels_per_thread) {
    if (pixels_per_thread == 2)
        composite_forward_kernel<2><<<tiles, TileGeom<kTileW, kTileH, 2>::kThreads, 0, s>>>(
            ranges, order, st, K, bg, color, alpha, pix_T, pix_last, visibility);
    else if (pixels_per_thread == 8)
        composite_forward_kernel<8><<<tiles, TileGeom<kTileW, kTileH, 8>::kThreads, 0, s>>>(
            ranges, order, st, K, bg, color, alpha, pix_T, pix_last, visibility);
    else
        composite_forward_kernel<4><<<tiles, TileGeom<kTileW, kTileH, 4>::kThreads, 0, s>>>(
            ranges, order, st, K, bg, color, alpha, pix_T, pix_last, visibility);
}

template <int PX>
static void launch_backward_px(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, const float* pix_T, const unsigned* pix_last,
                               const float* dL_color, const float* dL_alpha,
                               const float* densify_map, int want_refine) {
    const int T = TileGeom<kTileW, kTileH, PX>::kThreads;
#define GSB_BWD(R, D)                                                                            \
    composite_backward_kernel<PX, R, D><<<tiles, T, 0, s>>>(ranges, order, st, K, bg, pix_T,     \
                                                            pix_last, dL_color, dL_alpha,        \
                                                            densify_map)
    if (want_refine && densify_map) GSB_BWD(true, true);
    else if (want_refine) GSB_BWD(true, false);
    else if (densify_map) GSB_BWD(false, true);
    else GSB_BWD(false, false);
#undef GSB_BWD
}

void launch_composite_backward(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, const float* pix_T, const unsigned* pix_last,
                               const float* dL_color, const float* dL_alpha,
                               const float* densify_map, int want_refine, int pixels_per_thread) {
    if (pixels_per_thread == 2)
        launch_backward_px<2>(s, tiles, ranges, order, st, K, bg, pix_T, pix_last, dL_color,
                              dL_alpha, densify_map, want_refine);
    else if (pixels_per_thread == 8)
        launch_backward_px<8>(s, tiles, ranges, order, st, K, bg, pix_T, pix_last, dL_color,
                              dL_alpha, densify_map, want_refine);
    else
        launch_backward_px<4>(s, tiles, ranges, order, st, K, bg, pix_T, pix_last, dL_color,
                              dL_alpha, densify_map, want_refine);
}

} // namespace gsb
