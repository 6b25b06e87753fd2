// C entry points onto the reference's own training-loss kernels
// (photara/src/splat/cuda_ops.cu: loss_kernel, depth_normal_consistency_kernel),
// compiled from that file where it lies.
//
// TEST INFRASTRUCTURE ONLY (the checker): built by oracle/Makefile into
// oracle/_ref/libloss_ref.so. The launches follow
// cuda_backend::compute_training_loss (cuda_ops.cu:2731-2822): loss_kernel,
// then (by the caller, through libssim_ref.so) the fused SSIM kernels, then
// the consistency kernel.
#include "cuda_ops.cu"

#include <stdexcept>

// The reference's tinytensor wrappers are compiled with the file but never
// called here; these definitions satisfy the linker only.
namespace tinytensor {
namespace {
[[noreturn]] void unavailable() { throw std::runtime_error("not available in the loss harness"); }
} // namespace
Tensor Tensor::empty(TensorShape, Device, DataType, bool) { unavailable(); }
Tensor Tensor::zeros(TensorShape, Device, DataType) { unavailable(); }
Tensor Tensor::zeros_bool(TensorShape, Device) { unavailable(); }
Tensor Tensor::from_vector(const std::vector<float>&, TensorShape, Device) { unavailable(); }
Tensor::Tensor(Tensor&&) noexcept { std::abort(); }
Tensor::~Tensor() {}
Tensor& Tensor::operator=(Tensor&&) noexcept { return *this; }
void Tensor::materialize_if_deferred() {}
size_t Tensor::count_nonzero() const { unavailable(); }
Tensor Tensor::to(DataType) const { unavailable(); }
Tensor Tensor::clone() const { unavailable(); }
Tensor Tensor::nonzero() const { unavailable(); }
Tensor Tensor::movement(MovementOp, const MovementArgs&) const { unavailable(); }
std::vector<float> Tensor::to_vector() const { unavailable(); }
} // namespace tinytensor

// The fused SSIM kernels live in their own harness (libssim_ref.so).
void photara::splat::detail::cuda_backend::fused_l1_ssim_loss(
    const tinytensor::Tensor&, const tinytensor::Tensor&, const tinytensor::Tensor&, bool, float,
    float, tinytensor::Tensor&, float*, std::uint32_t, std::uint32_t) {
    throw std::runtime_error("not available in the loss harness");
}

using namespace photara::splat::detail;

extern "C" int ref_loss_kernel(const float* color, const float* alpha, const float* depth,
                               const float* normal, const float* target_color,
                               const float* target_depth, const float* target_normal,
                               const float* mask, float* grad_color, float* grad_alpha,
                               float* grad_depth, float* grad_normal, float* terms, size_t pixels,
                               float photo_weight, float depth_weight, float normal_weight,
                               int mask_enabled, int alpha_mode, float match_alpha_weight,
                               float geometry_epsilon, int ai_prior, void* stream) {
    loss_kernel<<<(pixels + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        color, alpha, depth, normal, target_color, target_depth, target_normal, mask, grad_color,
        grad_alpha, grad_depth, grad_normal, terms, pixels, photo_weight, depth_weight,
        normal_weight, mask_enabled != 0, alpha_mode, match_alpha_weight, 1.F, geometry_epsilon,
        ai_prior != 0);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

extern "C" int ref_depth_normal(const float* depth, const float* normal, float* grad_depth,
                                float* grad_normal, float* terms, unsigned width, unsigned height,
                                float fx, float fy, float cx, float cy, float weight,
                                void* stream) {
    const size_t pixels = size_t(width) * height;
    depth_normal_consistency_kernel<<<(pixels + 255) / 256, 256, 0,
                                      static_cast<cudaStream_t>(stream)>>>(
        depth, normal, grad_depth, grad_normal, terms, width, height, fx, fy, cx, cy, weight);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

extern "C" int ref_split_gaussians(float* parent_means, float* parent_log_scales,
                                   float* parent_opacity_logits, const float* parent_quaternions,
                                   float* child_means, float* child_log_scales,
                                   float* child_opacity_logits, const int* parent_indices,
                                   const float* random_samples, const float* screen_sizes,
                                   size_t count, int mode, float minimum_opacity,
                                   float split_at_screen_size, float split_opacity_k,
                                   void* stream) {
    // the clamps of cuda_backend::split_gaussians (cuda_ops.cu:3105-3122)
    split_gaussians_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        parent_means, parent_log_scales, parent_opacity_logits, parent_quaternions, child_means,
        child_log_scales, child_opacity_logits, parent_indices, random_samples, screen_sizes,
        count, static_cast<SplitMode>(mode), std::clamp(minimum_opacity, 1e-8F, 0.49F),
        std::max(split_at_screen_size, 0.F), std::clamp(split_opacity_k, 1e-4F, 1.F - 1e-4F));
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

extern "C" int ref_adc_decay(float* log_scales, float* opacity_logits, size_t count,
                             float opacity_decay, float scale_decay, void* stream) {
    // the host arithmetic of cuda_backend::apply_adc_decay (cuda_ops.cu:3388-3400)
    const float scale_factor = std::max(1.F - scale_decay, 1e-6F);
    adc_decay_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        log_scales, opacity_logits, count, std::max(opacity_decay, 0.F), std::log(scale_factor));
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

// accumulate_densification_kernel (cuda_ops.cu:1548-1606) with every argument,
// launched as cuda_backend::accumulate_densification_stats_cuda does
// (cuda_ops.cu:3061-3083).
extern "C" int ref_accumulate_densification(
    const float* refine_weight, const float* visibility, const int* radii, float* gradient,
    float* count, float* max_screen_radius, float* priority, size_t n, float inverse_resolution,
    int use_maximum, int require_visibility, float step_score_power,
    float oversize_screen_threshold, const float* geometry_gradient,
    float* max_geometry_gradient, int* first_view, float* view_support, int view_index,
    const float* image_error, float* accumulated_error, const float* normalized_size,
    void* stream) {
    accumulate_densification_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        refine_weight, visibility, radii, gradient, count, max_screen_radius, priority, n,
        inverse_resolution, use_maximum != 0, require_visibility != 0, step_score_power,
        oversize_screen_threshold, geometry_gradient, max_geometry_gradient, first_view,
        view_support, view_index, image_error, accumulated_error, normalized_size);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
