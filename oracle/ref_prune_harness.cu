// C entry point onto the reference's own Speedy-Splat score kernel
// (photara/src/splat/rasterizer.cu:93-146, sensitivity_scores), compiled from
// that file where it lies, run over the reference rasterizer's workspace after
// a forward through oracle/_ref/libsplat_ref.so (ref_forward_state gives the
// pools), the way CudaRasterizer::pruning_scores (:450-490) launches it.
//
// TEST INFRASTRUCTURE ONLY (the checker): built by oracle/Makefile into
// oracle/_ref/libprune_ref.so, linked against libsplat_ref.so for the
// splat_drender symbols rasterizer.cu refers to.
#include "rasterizer.cu"

#include <stdexcept>

// photara / tinytensor functions the file refers to but the score kernel
// never reaches; defined here so the object links.
namespace tinytensor {
namespace {
[[noreturn]] void unavailable() { throw std::runtime_error("not available in the prune harness"); }
} // namespace
Tensor Tensor::empty(TensorShape, Device, DataType, bool) { unavailable(); }
Tensor Tensor::zeros(TensorShape, Device, DataType) { unavailable(); }
Tensor::Tensor(Tensor&&) noexcept { std::abort(); }
Tensor::Tensor(const Tensor&) { std::abort(); }
Tensor::~Tensor() {}
Tensor& Tensor::operator=(Tensor&&) noexcept { return *this; }
Tensor& Tensor::operator=(const Tensor&) { return *this; }
void Tensor::materialize_if_deferred() {}
std::vector<float> Tensor::to_vector() const { unavailable(); }
VramScope::VramScope(std::string_view) {}
VramScope::~VramScope() {}
} // namespace tinytensor

namespace photara::splat::detail {
ActivatedParameters activate_parameters(const GaussianModel&) {
    throw std::runtime_error("not available in the prune harness");
}
void chain_parameter_gradients(const GaussianModel&, const ActivatedParameters&,
                               const tinytensor::Tensor&, const tinytensor::Tensor&,
                               const tinytensor::Tensor&, ModelGradients&) {
    throw std::runtime_error("not available in the prune harness");
}
} // namespace photara::splat::detail

extern "C" int ref_sensitivity_scores(int width, int height, void* gaussian_pool, size_t n,
                                      void* tile_pool, const unsigned* ids,
                                      const unsigned* contributors, const float* image,
                                      float* scores, float alpha_clip, int gaussian_pop,
                                      void* stream) {
    namespace ws = splat_drender::ws;
    const auto gs = ws::GaussianState::from_pool(static_cast<char*>(gaussian_pool), n, 0, false);
    const auto ts = ws::TileState::from_pool(static_cast<char*>(tile_pool),
                                             size_t((width + 15) / 16) * ((height + 15) / 16), 0);
    photara::splat::sensitivity_scores<<<dim3((width + 15) / 16, (height + 15) / 16),
                                         dim3(16, 16), 0,
                         static_cast<cudaStream_t>(stream)>>>(
        width, height, 0, gs, ids, ts.range, contributors, image, scores, alpha_clip,
        gaussian_pop != 0);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
