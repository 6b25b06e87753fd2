// C entry points onto the reference's own fused L1 + SSIM kernels
// (photara/src/splat/fused_ssim.cu), compiled from that file where it lies.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed reference arm of the
// loss): built by oracle/Makefile into oracle/_ref/libssim_ref.so. The
// launches restate cuda_backend::fused_l1_ssim_loss (fused_ssim.cu:473-555)
// and cuda_backend::fused_ssim_metric (fused_ssim.cu:557-607) with scratch
// that this harness allocates once instead of per call.
#include "fused_ssim.cu"

#include <cstdio>
#include <stdexcept>

// The reference's tinytensor wrappers are compiled with the file but never
// called here; these definitions satisfy the linker only.
namespace tinytensor {
Tensor Tensor::empty(TensorShape, Device, DataType, bool) {
    throw std::runtime_error("not available in the SSIM harness");
}
void Tensor::materialize_if_deferred() {}
Tensor::~Tensor() {}
Tensor& Tensor::operator=(Tensor&&) noexcept { return *this; }
std::vector<float> Tensor::to_vector() const {
    throw std::runtime_error("not available in the SSIM harness");
}
} // namespace tinytensor

namespace {
struct Scratch {
    float* p = nullptr;
    size_t n = 0;
    float* get(size_t floats) {
        if (floats > n) {
            if (p)
                cudaFree(p);
            if (cudaMalloc(&p, floats * sizeof(float)) != cudaSuccess)
                return nullptr;
            n = floats;
        }
        return p;
    }
};
Scratch g_scratch;
} // namespace

using namespace photara::splat::detail;

extern "C" int ref_fused_l1_ssim(const float* prediction, const float* target, const float* mask,
                                 float ssim_weight, float photometric_weight, float* gradient,
                                 float* scalar_terms, int width, int height, void* stream_ptr) {
    if (width <= k_halo2 || height <= k_halo2)
        return 1;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    constexpr int channels = 3;
    const size_t count = size_t(channels) * width * height;
    const dim3 block(k_block_x, k_block_y);
    const dim3 grid((width + k_block_x - 1) / k_block_x, (height + k_block_y - 1) / k_block_y, 1);
    const size_t blocks = size_t(grid.x) * grid.y;
    float* s = g_scratch.get(5 * count + blocks);
    if (!s)
        return 2;
    float* dm_dmu1 = s;
    float* dm_dsigma1_sq = s + count;
    float* dm_dsigma12 = s + 2 * count;
    float* masked_prediction = s + 3 * count;
    float* masked_target = s + 4 * count;
    float* loss_blocks = s + 5 * count;
    const float* image1 = prediction;
    const float* image2 = target;
    if (mask) {
        apply_mask_kernel<<<(count + 255) / 256, 256, 0, stream>>>(
            prediction, target, mask, masked_prediction, masked_target, channels, height, width,
            true);
        image1 = masked_prediction;
        image2 = masked_target;
    }
    const float normalization =
        photometric_weight / float(channels * (width - k_halo2) * (height - k_halo2));
    fused_l1_ssim_forward_kernel<true, false><<<grid, block, 0, stream>>>(
        ssim_weight, height, width, channels, 0.01F * 0.01F, 0.03F * 0.03F, image1, image2,
        dm_dmu1, dm_dsigma1_sq, dm_dsigma12, scalar_terms ? loss_blocks : nullptr, normalization,
        nullptr, false, nullptr, nullptr);
    if (scalar_terms)
        reduce_loss_blocks_kernel<<<1, 256, 0, stream>>>(loss_blocks, blocks, scalar_terms);
    fused_l1_ssim_backward_kernel<<<grid, block, 0, stream>>>(
        ssim_weight, height, width, channels, image1, image2, normalization, gradient, dm_dmu1,
        dm_dsigma1_sq, dm_dsigma12, mask, mask != nullptr);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

extern "C" int ref_ssim_metric(const float* prediction, const float* target, const float* mask,
                               int width, int height, float* out, void* stream_ptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    if (width <= k_halo2 || height <= k_halo2)
        return cudaMemsetAsync(out, 0, sizeof(float), stream) == cudaSuccess ? 0 : 3;
    constexpr int channels = 3;
    const size_t count = size_t(channels) * width * height;
    const dim3 block(k_block_x, k_block_y);
    const dim3 grid((width + k_block_x - 1) / k_block_x, (height + k_block_y - 1) / k_block_y, 1);
    const size_t blocks = size_t(grid.x) * grid.y;
    float* s = g_scratch.get(2 * count + 2 * blocks);
    if (!s)
        return 2;
    const float* image1 = prediction;
    const float* image2 = target;
    if (mask) {
        apply_mask_kernel<<<(count + 255) / 256, 256, 0, stream>>>(
            prediction, target, mask, s, s + count, channels, height, width, true);
        image1 = s;
        image2 = s + count;
    }
    float* sum = s + 2 * count;
    float* cnt = sum + blocks;
    fused_l1_ssim_forward_kernel<false, true><<<grid, block, 0, stream>>>(
        1.F, height, width, channels, 0.01F * 0.01F, 0.03F * 0.03F, image1, image2, nullptr,
        nullptr, nullptr, nullptr, 0.F, mask, mask != nullptr, sum, cnt);
    reduce_ssim_metric_kernel<<<1, 256, 0, stream>>>(sum, cnt, blocks, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
