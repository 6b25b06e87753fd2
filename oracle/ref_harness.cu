// Checker-side harness around the reference rasterizer (splat_drender), built
// from the reference's own sources by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links or calls
// this file; tests and bench.py's reference arm load the resulting
// libsplat_ref.so through ctypes to obtain the reference's own outputs on the
// same device inputs.
//
// The harness drives the public static API of the reference exactly like
// photara's CudaRasterizer bridge does (photara/src/splat/rasterizer.cu:340-402
// for forward, :495-686 for backward): raw activation inputs
// (log_scales/quaternions/opacity_logits), SH colour, cudaMalloc-backed
// grow-only workspace pools kept alive between forward and backward
// (rasterizer.cu:177-185), outputs pre-zeroed by the caller.
#include "splat_drender/api.h"
#include "splat_drender/buffers.h"

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>

namespace {

struct Pool {
    char* base = nullptr;
    std::size_t bytes = 0;
    char* grow(std::size_t need) {
        if (need > bytes) {
            if (base)
                cudaFree(base);
            base = nullptr;
            std::size_t cap = need + need / 4 + 4096;
            if (cudaMalloc(&base, cap) != cudaSuccess)
                throw std::runtime_error("ref harness: pool cudaMalloc failed");
            bytes = cap;
        }
        return base;
    }
};

struct Context {
    Pool gaussian, grad, instance, pixel, tile, point, compact;
    splat_drender::ForwardResult fwd{};
    splat_drender::Gaussians g{};
    splat_drender::CameraView cam{};
    splat_drender::RenderSettings s{};
    float* view_dev = nullptr; // 16 view floats + 3 centre floats
    bool have_forward = false;
    std::string error;
};

Context& ctx() {
    static Context c;
    return c;
}

splat_drender::WorkspacePools pools_of(Context& c) {
    splat_drender::WorkspacePools p;
    p.gaussian = [&c](std::size_t n) { return c.gaussian.grow(n); };
    p.grad = [&c](std::size_t n) { return c.grad.grow(n); };
    p.instance = [&c](std::size_t n) { return c.instance.grow(n); };
    p.pixel = [&c](std::size_t n) { return c.pixel.grow(n); };
    p.tile = [&c](std::size_t n) { return c.tile.grow(n); };
    p.point = [&c](std::size_t n) { return c.point.grow(n); };
    // No compact_instance pool: the sorted draw list stays in the instance
    // pool so the harness can export it for bit-exact comparison.
    return p;
}

} // namespace

extern "C" {

const char* ref_last_error() { return ctx().error.c_str(); }

// 1 (default): forward and backward wait for the device before returning, as
// the tests want. 0: they return once their work is enqueued on the legacy
// default stream (the reference's own forward still waits for its draw
// counts), so a timed loop measures the reference without extra host waits.
static int g_synchronous = 1;
void ref_set_synchronous(int on) { g_synchronous = on != 0; }

static int finish() {
    if (g_synchronous)
        return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Forward over device inputs. view_host: 16 column-major world-to-camera
// floats; center_host: 3 floats. Output buffers are device pointers that the
// caller zeroed. counts_out (host) receives {instances, visible}. need_depth
// renders the median-depth and normal channels into out_median_depth [H,W]
// and out_normal [3,H,W] (blend_tile<GEOMETRY = true>).
// As ref_forward, with the Mip-Splatting 3D filter (RawActivation::filter_3d,
// [N] or NULL) and precomputed view colours ([N,3] in place of sh, or NULL).
int ref_forward_ex(int n, const float* means, const float* log_scales, const float* quats,
                   const float* opacity_logits, const float* sh, int sh_degree, int sh_bases,
                   const float* view_host, const float* center_host, int width, int height,
                   float fx, float fy, float cx, float cy, float near_plane, float alpha_clip,
                   int compensate_2d, float kernel_size, const float* background_host,
                   float* out_color, float* out_alpha, int* out_radii, float* out_visibility,
                   int* counts_out, int need_depth, float* out_median_depth, float* out_normal,
                   const float* filter_3d, const float* colors);

int ref_forward(int n, const float* means, const float* log_scales, const float* quats,
                const float* opacity_logits, const float* sh, int sh_degree, int sh_bases,
                const float* view_host, const float* center_host, int width, int height, float fx,
                float fy, float cx, float cy, float near_plane, float alpha_clip,
                int compensate_2d, float kernel_size, const float* background_host,
                float* out_color, float* out_alpha, int* out_radii, float* out_visibility,
                int* counts_out, int need_depth, float* out_median_depth, float* out_normal) {
    return ref_forward_ex(n, means, log_scales, quats, opacity_logits, sh, sh_degree, sh_bases,
                          view_host, center_host, width, height, fx, fy, cx, cy, near_plane,
                          alpha_clip, compensate_2d, kernel_size, background_host, out_color,
                          out_alpha, out_radii, out_visibility, counts_out, need_depth,
                          out_median_depth, out_normal, nullptr, nullptr);
}

int ref_forward_ex(int n, const float* means, const float* log_scales, const float* quats,
                   const float* opacity_logits, const float* sh, int sh_degree, int sh_bases,
                   const float* view_host, const float* center_host, int width, int height,
                   float fx, float fy, float cx, float cy, float near_plane, float alpha_clip,
                   int compensate_2d, float kernel_size, const float* background_host,
                   float* out_color, float* out_alpha, int* out_radii, float* out_visibility,
                   int* counts_out, int need_depth, float* out_median_depth, float* out_normal,
                   const float* filter_3d, const float* colors) {
    Context& c = ctx();
    try {
        if (!c.view_dev && cudaMalloc(&c.view_dev, 19 * sizeof(float)) != cudaSuccess)
            throw std::runtime_error("ref harness: camera cudaMalloc failed");
        float host[19];
        std::memcpy(host, view_host, 16 * sizeof(float));
        std::memcpy(host + 16, center_host, 3 * sizeof(float));
        if (cudaMemcpy(c.view_dev, host, sizeof(host), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("ref harness: camera upload failed");
        splat_drender::Gaussians g;
        g.count = n;
        g.means = means;
        g.raw = {log_scales, quats, opacity_logits, filter_3d};
        if (colors) {
            g.colors = colors;
        } else {
            g.sh = sh;
            g.sh_degree = sh_degree;
            g.sh_bases = sh_bases;
        }
        splat_drender::CameraView cam;
        cam.width = width;
        cam.height = height;
        cam.fx = fx;
        cam.fy = fy;
        cam.cx = cx;
        cam.cy = cy;
        cam.near_plane = near_plane;
        cam.alpha_clip = alpha_clip;
        cam.compensate_2d = compensate_2d != 0;
        cam.world_to_camera = c.view_dev;
        cam.center = c.view_dev + 16;
        splat_drender::RenderSettings s;
        for (int k = 0; k < 3; ++k)
            s.background[k] = background_host[k];
        s.kernel_size = kernel_size;
        s.need_depth = need_depth != 0;
        splat_drender::RenderOutputs out;
        out.color = out_color;
        out.alpha = out_alpha;
        out.radii = out_radii;
        out.visibility = out_visibility;
        if (need_depth) {
            out.median_depth = out_median_depth;
            out.normal = out_normal;
        }
        c.fwd = splat_drender::Rasterizer::forward(pools_of(c), g, cam, s, out);
        c.g = g;
        c.cam = cam;
        c.s = s;
        c.have_forward = true;
        if (counts_out) {
            counts_out[0] = c.fwd.instance_count;
            counts_out[1] = c.fwd.visible_count;
        }
        return finish();
    } catch (const std::exception& e) {
        c.error = e.what();
        return 1;
    }
}

// Copies the sorted draw list (Gaussian ids in composite order) and the
// per-tile [start, end) ranges of the last forward into device buffers.
int ref_draw_list(unsigned* values_out, unsigned* ranges_out) {
    Context& c = ctx();
    if (!c.have_forward) {
        c.error = "ref harness: no forward";
        return 1;
    }
    const int grid_x = (c.cam.width + 15) / 16;
    const int grid_y = (c.cam.height + 15) / 16;
    const std::size_t tiles = std::size_t(grid_x) * grid_y;
    const std::size_t inst = std::size_t(c.fwd.instance_count);
    // Re-derive the instance pool layout the same way the library does: the
    // tile pool starts with the ranges; the instance values sit after the
    // five visible-sized arrays and two key arrays (buffers.h InstanceState).
    namespace ws = splat_drender::ws;
    auto* tile_state = c.tile.base;
    if (cudaMemcpy(ranges_out, tile_state, tiles * sizeof(uint2), cudaMemcpyDeviceToDevice) !=
        cudaSuccess) {
        c.error = "ref harness: range copy";
        return 2;
    }
    if (inst == 0)
        return 0;
    const std::size_t vis = std::size_t(c.fwd.visible_count);
    std::size_t offset = ws::align_up(vis * sizeof(unsigned)) * 5 +
                         ws::align_up(ws::InstanceState::key_bytes(inst)) * 2;
    if (c.fwd.instance_selector == 1)
        offset += ws::align_up(inst * sizeof(unsigned));
    if (cudaMemcpy(values_out, c.instance.base + offset, inst * sizeof(unsigned),
                   cudaMemcpyDeviceToDevice) != cudaSuccess) {
        c.error = "ref harness: value copy";
        return 2;
    }
    return 0;
}

// Workspace of the last forward, for the reference's Speedy-Splat score
// kernel (oracle/ref_prune_harness.cu): the Gaussian and tile pools, the
// per-pixel contributor counts (first array of the pixel pool) and the sorted
// draw list, located as ref_draw_list locates it.
int ref_forward_state(void** gaussian_pool, void** tile_pool, void** contributors,
                      void** ids, int* instances) {
    Context& c = ctx();
    if (!c.have_forward) {
        c.error = "ref harness: no forward";
        return 1;
    }
    namespace ws = splat_drender::ws;
    const std::size_t inst = std::size_t(c.fwd.instance_count);
    const std::size_t vis = std::size_t(c.fwd.visible_count);
    std::size_t offset = ws::align_up(vis * sizeof(unsigned)) * 5 +
                         ws::align_up(ws::InstanceState::key_bytes(inst)) * 2;
    if (c.fwd.instance_selector == 1)
        offset += ws::align_up(inst * sizeof(unsigned));
    *gaussian_pool = c.gaussian.base;
    *tile_pool = c.tile.base;
    *contributors = c.pixel.base;
    *ids = c.instance.base + offset;
    *instances = int(inst);
    return 0;
}

// Backward of the last forward. Forward outputs (alpha, radii) are passed
// back in. Gradient outputs are device buffers zeroed by the caller; the
// reference accumulates into them. Without fused Adam the scale/rotation/
// opacity gradients are with respect to the ACTIVATED values (exp scale,
// normalised quaternion, sigmoid opacity), as the reference produces them for
// photara's host-side chain rule.
// Optional fused Adam: when adam_means != nullptr the structure Adam runs in
// the reference's gaussian_backward; when sh_param != nullptr the quantized
// SH Adam runs there too.
struct RefAdam {
    float* means;
    float* log_scales;
    float* quaternions;
    float* opacity_logits;
    float* means_first;
    float* means_second;
    float* scales_first;
    float* scales_second;
    float* rotations_first;
    float* rotations_second;
    float* opacity_first;
    float* opacity_second;
    float means_lr, scales_lr, quaternions_lr, opacities_lr;
    float beta1, beta2, correction1, correction2, epsilon;
    float* sh_param;
    void* sh_first;
    unsigned char* sh_packed;
    float* sh_bounds;
    float sh_lr, sh_rest_lr, sh_epsilon, sh_regularization;
    int sh_stride;
    // structure Adam priors and clamps (StructureAdam, api.h:138-164)
    const float* filter_3d;
    float minimum_log_scale, maximum_log_scale;
    float opacity_reg, scale_reg, shape_erank_reg, shape_erank_s3_reg, shape_quat_norm_reg;
    float shape_axis_ratio_reg, shape_max_axis_ratio;
    float* opacity_gradient;
};

int ref_backward_ex(const float* fwd_alpha, const int* fwd_radii, const float* dL_color,
                    const float* dL_alpha, float* grad_means, float* grad_sh,
                    float* grad_opacity, float* grad_scales, float* grad_rotations,
                    float* refine_weight, const RefAdam* adam, float* grad_colors);

int ref_backward_full(const float* fwd_alpha, const int* fwd_radii, const float* dL_color,
                      const float* dL_alpha, float* grad_means, float* grad_sh,
                      float* grad_opacity, float* grad_scales, float* grad_rotations,
                      float* refine_weight, const RefAdam* adam) {
    return ref_backward_ex(fwd_alpha, fwd_radii, dL_color, dL_alpha, grad_means, grad_sh,
                           grad_opacity, grad_scales, grad_rotations, refine_weight, adam,
                           nullptr);
}

// As ref_backward_full, with the gradient of precomputed colours ([N,3], or
// NULL) for a forward rendered from colours.
int ref_backward_ex(const float* fwd_alpha, const int* fwd_radii, const float* dL_color,
                    const float* dL_alpha, float* grad_means, float* grad_sh,
                    float* grad_opacity, float* grad_scales, float* grad_rotations,
                    float* refine_weight, const RefAdam* adam, float* grad_colors) {
    Context& c = ctx();
    try {
        if (!c.have_forward)
            throw std::runtime_error("ref harness: no forward");
        splat_drender::ForwardOutputsView fo;
        fo.alpha = fwd_alpha;
        fo.radii = fwd_radii;
        splat_drender::LossGradients dL;
        dL.color = dL_color;
        dL.alpha = dL_alpha;
        splat_drender::ModelGradients grads;
        grads.means = grad_means;
        grads.sh = grad_sh;
        grads.opacities = grad_opacity;
        grads.scales = grad_scales;
        grads.rotations = grad_rotations;
        grads.refine_weight = refine_weight;
        grads.colors = grad_colors;
        if (adam && adam->means) {
            auto& a = grads.structure_adam;
            a.means = adam->means;
            a.log_scales = adam->log_scales;
            a.quaternions = adam->quaternions;
            a.opacity_logits = adam->opacity_logits;
            a.means_first = adam->means_first;
            a.means_second = adam->means_second;
            a.scales_first = adam->scales_first;
            a.scales_second = adam->scales_second;
            a.rotations_first = adam->rotations_first;
            a.rotations_second = adam->rotations_second;
            a.opacity_first = adam->opacity_first;
            a.opacity_second = adam->opacity_second;
            a.means_lr = adam->means_lr;
            a.scales_lr = adam->scales_lr;
            a.quaternions_lr = adam->quaternions_lr;
            a.opacities_lr = adam->opacities_lr;
            a.beta1 = adam->beta1;
            a.beta2 = adam->beta2;
            a.correction1 = adam->correction1;
            a.correction2 = adam->correction2;
            a.epsilon = adam->epsilon;
            a.filter_3d = adam->filter_3d;
            a.minimum_log_scale = adam->minimum_log_scale;
            a.maximum_log_scale = adam->maximum_log_scale;
            a.opacity_reg = adam->opacity_reg;
            a.scale_reg = adam->scale_reg;
            a.shape_erank_reg = adam->shape_erank_reg;
            a.shape_erank_s3_reg = adam->shape_erank_s3_reg;
            a.shape_quat_norm_reg = adam->shape_quat_norm_reg;
            a.shape_axis_ratio_reg = adam->shape_axis_ratio_reg;
            a.shape_max_axis_ratio = adam->shape_max_axis_ratio;
            a.opacity_gradient = adam->opacity_gradient;
            grads.means = nullptr;
            grads.opacities = nullptr;
            grads.scales = nullptr;
            grads.rotations = nullptr;
        }
        if (adam && adam->sh_param) {
            auto& s = grads.sh_adam;
            s.parameter = adam->sh_param;
            s.lr = adam->sh_lr;
            s.rest_lr = adam->sh_rest_lr;
            s.beta1 = adam->beta1;
            s.beta2 = adam->beta2;
            s.correction1 = adam->correction1;
            s.correction2 = adam->correction2;
            s.epsilon = adam->sh_epsilon;
            s.regularization_factor = adam->sh_regularization;
            s.first = adam->sh_first;
            s.packed = adam->sh_packed;
            s.bounds = adam->sh_bounds;
            s.stride = adam->sh_stride;
            grads.sh = nullptr;
        }
        splat_drender::Rasterizer::backward(pools_of(c), c.g, c.cam, c.s, c.fwd, fo, dL, grads);
        return finish();
    } catch (const std::exception& e) {
        c.error = e.what();
        return 1;
    }
}

// Rasterizer::forward_colors (pipeline.cu:617-649): re-blends new
// precomputed colours [N,3] over the draw list of the last forward, which must
// have been rendered from colours. Outputs zeroed by the caller.
int ref_forward_colors(const float* colors, float* out_color, float* out_alpha,
                       float* out_visibility) {
    Context& c = ctx();
    try {
        if (!c.have_forward || !c.g.colors)
            throw std::runtime_error("ref harness: colour reuse needs a forward from colours");
        splat_drender::Gaussians g = c.g;
        g.colors = colors;
        splat_drender::RenderOutputs out;
        out.color = out_color;
        out.alpha = out_alpha;
        out.visibility = out_visibility;
        splat_drender::Rasterizer::forward_colors(pools_of(c), g, c.cam, c.s, c.fwd, out);
        c.g = g;
        return finish();
    } catch (const std::exception& e) {
        c.error = e.what();
        return 1;
    }
}

// Backward of the last forward (rendered with need_depth) with gradients of
// the median-depth and normal outputs as well (splat_drender LossGradients
// median_depth / normal: median_scale_walk, blend_bucket_backward<GEOMETRY>,
// the ray-plane and normal chain). Activated-space parameter gradients, as
// ref_backward_full without Adam; buffers zeroed by the caller.
// The geometry backward reads the forward's median-depth and normal outputs
// (ForwardOutputsView, api.h:102-107), so both are required here.
int ref_backward_geometry(const float* fwd_alpha, const int* fwd_radii,
                          const float* fwd_median_depth, const float* fwd_normal,
                          const float* dL_color, const float* dL_alpha,
                          const float* dL_median_depth, const float* dL_normal,
                          float* grad_means, float* grad_sh, float* grad_opacity,
                          float* grad_scales, float* grad_rotations) {
    Context& c = ctx();
    try {
        if (!c.have_forward)
            throw std::runtime_error("ref harness: no forward");
        if (!c.s.need_depth || !fwd_median_depth || !fwd_normal)
            throw std::runtime_error(
                "ref harness: the geometry backward needs a need_depth forward and its "
                "median-depth and normal outputs");
        splat_drender::ForwardOutputsView fo;
        fo.alpha = fwd_alpha;
        fo.radii = fwd_radii;
        fo.median_depth = fwd_median_depth;
        fo.normal = fwd_normal;
        splat_drender::LossGradients dL;
        dL.color = dL_color;
        dL.alpha = dL_alpha;
        dL.median_depth = dL_median_depth;
        dL.normal = dL_normal;
        splat_drender::ModelGradients grads;
        grads.means = grad_means;
        grads.sh = grad_sh;
        grads.opacities = grad_opacity;
        grads.scales = grad_scales;
        grads.rotations = grad_rotations;
        splat_drender::Rasterizer::backward(pools_of(c), c.g, c.cam, c.s, c.fwd, fo, dL, grads);
        if (finish() != 0)
            throw std::runtime_error("ref harness: backward failed");
    } catch (const std::exception& e) {
        c.error = e.what();
        return 1;
    }
    return 0;
}

} // extern "C"
