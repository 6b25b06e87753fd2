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
