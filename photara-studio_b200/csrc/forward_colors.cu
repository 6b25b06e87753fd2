// Colour reuse (splat_drender Rasterizer::forward_colors,
// third_party/splat_drender/src/pipeline.cu:617-649): after a training
// forward of a model with precomputed colours, blend new colours over the
// same draw list. Alpha, termination and the draw order do not depend on the
// colours, so projection, sorting and the per-pixel state are reused; only the
// per-Gaussian colour slots are rewritten (no SH clamp bits) before the
// compositing kernel runs again.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace gsb {

namespace {

__global__ void __launch_bounds__(256) set_colors_kernel(int n, const float* __restrict__ colors,
                                                        float4* __restrict__ rgb,
                                                        SplatRec* __restrict__ rec) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i < n) {
        const float4 c = make_float4(colors[3 * size_t(i)], colors[3 * size_t(i) + 1],
                                     colors[3 * size_t(i) + 2], __uint_as_float(0u));
        rgb[i] = c;
        if (rec)
            rec[i].rgb = c;
    }
}

} // namespace

cudaError_t launch_set_colors(cudaStream_t s, int n, const float* colors, float4* rgb,
                              SplatRec* rec) {
    if (n > 0)
        set_colors_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, colors, rgb, rec);
    return cudaGetLastError();
}

} // namespace gsb
