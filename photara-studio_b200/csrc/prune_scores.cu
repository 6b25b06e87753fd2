// Speedy-Splat pruning scores (photara/src/splat/rasterizer.cu:93-146,
// CudaRasterizer::pruning_scores :450-490): per Gaussian, the sum over the
// pixels it was blended into of the squared sensitivity of the pixel's
// colour sum to its opacity, d = o (T c - R / (1 - a)), with R the colour
// left behind it (the rendered colour, background included, minus what the
// Gaussians up to it added), c its colour sum; or, with gaussian_pop, the
// squared norm of the per-channel a (T c_k - R_k / (1 - a)).
//
// B200 organisation: the reference adds every (pixel, Gaussian) value to the
// Gaussian's score with a global atomic. Here a CTA owns a 16 x 16 tile,
// stages each batch of the tile's draw list in shared memory, reduces each
// entry's values over a warp with shuffles and over the CTA in shared
// memory, and issues one global atomic per (tile, Gaussian). The per-pixel
// walk follows the forward's draw order up to the pixel's last blended entry
// and repeats the reference's per-pixel arithmetic expression for expression.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "splat_math.cuh"

namespace gsb {

namespace {

constexpr int kTile = 16;
constexpr int kThreads = kTile * kTile;
constexpr int kWarps = kThreads / 32;

__global__ void __launch_bounds__(kThreads) pruning_scores_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order,
    const float2* __restrict__ mean2d, const float4* __restrict__ conic,
    const float4* __restrict__ rgb, const unsigned* __restrict__ pix_last,
    const float* __restrict__ image, int width, int height, int grid_x, float alpha_clip,
    int gaussian_pop, float* __restrict__ scores) {
    __shared__ float2 s_xy[kThreads];
    __shared__ float4 s_co[kThreads];
    __shared__ float4 s_rgb[kThreads];
    __shared__ unsigned s_id[kThreads];
    __shared__ float s_part[kWarps][kThreads];
    __shared__ unsigned s_max[kWarps];
    const int tile = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x = (tile % grid_x) * kTile + (tid % kTile);
    const int y = (tile / grid_x) * kTile + (tid / kTile);
    const bool inside = x < width && y < height;
    const uint2 range = ranges[tile];
    const unsigned len = range.y - range.x;
    const size_t pixels = size_t(width) * height;
    const size_t p = size_t(y) * width + x;
    unsigned limit = 0;
    float residual = 0.f;
    float3 residual_rgb = make_float3(0.f, 0.f, 0.f);
    if (inside) {
        limit = min(len, pix_last[p]);
        residual = image[p] + image[p + pixels] + image[p + 2 * pixels];
        residual_rgb = make_float3(image[p], image[p + pixels], image[p + 2 * pixels]);
    }
    float transmittance = 1.f;
    // the tile's walk ends at its pixels' largest last entry
    unsigned m = limit;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0)
        s_max[warp] = m;
    __syncthreads();
    unsigned tile_max = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w)
        tile_max = max(tile_max, s_max[w]);
    for (unsigned base = 0; base < tile_max; base += kThreads) {
        const int n = int(min(unsigned(kThreads), tile_max - base));
        __syncthreads(); // the previous batch's flush has read s_id and s_part
        if (tid < n) {
            const unsigned g = order[range.x + base + tid];
            s_id[tid] = g;
            s_xy[tid] = mean2d[g];
            s_co[tid] = conic[g];
            s_rgb[tid] = rgb[g];
        }
        __syncthreads();
        // warp-uniform walk; lanes past their last entry contribute zero
        for (int k = 0; k < n; ++k) {
            const unsigned j = base + unsigned(k);
            if (__all_sync(0xffffffffu, j >= limit))
                break;
            float value = 0.f;
            if (j < limit) {
                const float dx = s_xy[k].x - x;
                const float dy = s_xy[k].y - y;
                const float4 co = s_co[k];
                const float power = -.5f * (co.x * dx * dx + co.z * dy * dy) - co.y * dx * dy;
                if (!(power > 0.f)) {
                    const float alpha = fminf(alpha_clip, co.w * expf(power));
                    if (!(alpha < kAlphaFloor)) {
                        const float4 c = s_rgb[k];
                        const float colour = c.x + c.y + c.z;
                        residual -= transmittance * alpha * colour;
                        const float derivative =
                            co.w * (transmittance * colour - residual / (1.f - alpha));
                        value = derivative * derivative;
                        if (gaussian_pop) {
                            residual_rgb.x -= transmittance * alpha * c.x;
                            residual_rgb.y -= transmittance * alpha * c.y;
                            residual_rgb.z -= transmittance * alpha * c.z;
                            const float ex =
                                alpha * (transmittance * c.x - residual_rgb.x / (1.f - alpha));
                            const float ey =
                                alpha * (transmittance * c.y - residual_rgb.y / (1.f - alpha));
                            const float ez =
                                alpha * (transmittance * c.z - residual_rgb.z / (1.f - alpha));
                            value = ex * ex + ey * ey + ez * ez;
                        }
                        transmittance *= 1.f - alpha;
                    }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                value += __shfl_xor_sync(0xffffffffu, value, off);
            if (lane == 0)
                s_part[warp][k] = value;
        }
        __syncthreads();
        // one global atomic per (tile, Gaussian); warps that stopped early
        // wrote nothing past their stop, so read only what each wrote
        if (tid < n) {
            float sum = 0.f;
            const unsigned j = base + unsigned(tid);
#pragma unroll
            for (int w = 0; w < kWarps; ++w)
                sum += j < s_max[w] ? s_part[w][tid] : 0.f;
            if (sum != 0.f)
                atomicAdd(scores + s_id[tid], sum);
        }
    }
}

} // namespace

cudaError_t launch_pruning_scores(cudaStream_t s, int tiles, const uint2* ranges,
                                  const unsigned* order, const GaussianState& st, const Camera& K,
                                  const unsigned* pix_last, const float* image, int gaussian_pop,
                                  float* scores) {
    if (tiles > 0)
        pruning_scores_kernel<<<tiles, kThreads, 0, s>>>(
            ranges, order, st.mean2d, st.conic, st.rgb, pix_last, image, K.width, K.height,
            K.grid_x, K.alpha_clip, gaussian_pop, scores);
    return cudaGetLastError();
}

} // namespace gsb
