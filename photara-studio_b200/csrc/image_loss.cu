// Per-pixel training-loss terms around the fused L1 + SSIM kernel: the
// reference's compute_training_loss (photara/src/splat/cuda_ops.cu:2731-2822)
// for pinhole cameras, i.e. loss_kernel (cuda_ops.cu:846-966: the L1 colour
// term when the image is too small for SSIM, the relative robust depth term,
// the normal-prior term, the transparent-mode alpha BCE, and the zeroing of
// the gradient images) and depth_normal_consistency_kernel
// (cuda_ops.cu:999-1071: the rendered normal against the normal of the
// median-depth surface, backpropagated into both).
//
// B200 organisation: one pass over the pixels does both kernels' work. The
// reference scatters the consistency term's depth gradient into the four
// neighbours with atomics; here every pixel gathers what its four neighbours
// would scatter into it (their depth normals are recomputed from depths that
// the neighbouring threads read anyway), so the gradient images are written
// once, without atomics, and the result is deterministic. The loss terms are
// reduced per block and then in one fixed-order pass (double), instead of
// one global atomic per pixel and term. Per-pixel arithmetic is the
// reference's, expression for expression.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace gsb {

namespace {

constexpr int kThreads = 256;

struct LossArgs {
    ImageLossImages im;
    ImageLossOptions o;
    ImageLossOutputs out;
    float photo_weight; // 0 when the fused SSIM kernel owns the colour term
    float* partial;     // [blocks][4]
};

__device__ __forceinline__ float3 sub3(float3 a, float3 b) {
    return make_float3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot3(float3 a, float3 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
__device__ __forceinline__ float3 scale3(float3 v, float s) {
    return make_float3(v.x * s, v.y * s, v.z * s);
}

// Depth-normal consistency at pixel (x, y): whether it applies, its loss,
// the unit normal of the surface through the four neighbours' depths, and
// the gradients with respect to the vertical and horizontal differences.
struct DepthNormal {
    bool ok;
    float loss;
    float3 normal;
    float3 grad_dy, grad_dx;
};

__device__ __forceinline__ DepthNormal depth_normal_at(const LossArgs& a, int x, int y,
                                                       float normalization) {
    DepthNormal r;
    r.ok = false;
    const int W = a.im.width, H = a.im.height;
    if (x <= 0 || y <= 0 || x + 1 >= W || y + 1 >= H)
        return r;
    const size_t pixels = size_t(W) * H;
    const size_t pixel = size_t(y) * W + x;
    const float* depth = a.im.median_depth;
    const float d = depth[pixel], dt = depth[pixel - W], db = depth[pixel + W],
                dl = depth[pixel - 1], dr = depth[pixel + 1];
    if (!(d > 0.f && dt > 0.f && db > 0.f && dl > 0.f && dr > 0.f))
        return r;
    const float fx = a.im.fx, fy = a.im.fy, cx = a.im.cx, cy = a.im.cy;
    const auto point = [&](int px, int py, float dd) {
        return make_float3((float(px) - cx) / fx * dd, (float(py) - cy) / fy * dd, dd);
    };
    const float3 dy = sub3(point(x, y + 1, db), point(x, y - 1, dt));
    const float3 dx = sub3(point(x + 1, y, dr), point(x - 1, y, dl));
    const float3 c = cross3(dy, dx);
    const float length_squared = dot3(c, c);
    if (!(length_squared > 1e-20f) || !isfinite(length_squared))
        return r;
    const float inverse_length = rsqrtf(length_squared);
    const float3 dn = scale3(c, inverse_length);
    const float* n = a.im.normal;
    const float3 raster = make_float3(n[pixel], n[pixels + pixel], n[2 * pixels + pixel]);
    r.ok = true;
    r.normal = dn;
    r.loss = normalization * (1.f - dot3(raster, dn));
    const float3 grad_unit = scale3(raster, -normalization);
    const float projection = dot3(dn, grad_unit);
    const float3 grad_cross = scale3(sub3(grad_unit, scale3(dn, projection)), inverse_length);
    r.grad_dy = cross3(dx, grad_cross);
    r.grad_dx = cross3(grad_cross, dy);
    return r;
}

__global__ void __launch_bounds__(kThreads) image_loss_kernel(LossArgs a) {
    __shared__ float s_terms[kThreads / 32][4];
    const size_t pixels = size_t(a.im.width) * a.im.height;
    const size_t pixel = size_t(blockIdx.x) * kThreads + threadIdx.x;
    float t_rgb = 0.f, t_depth = 0.f, t_normal = 0.f, t_alpha = 0.f;
    if (pixel < pixels) {
        const ImageLossOptions& o = a.o;
        const float valid = o.mask_enabled ? a.im.mask[pixel] : 1.f;
        const float inverse_pixels = 1.f / float(pixels);
        // colour L1 (its value only when the fused SSIM kernel does not run)
        float rgb_loss = 0.f;
        for (int channel = 0; channel < 3; ++channel) {
            const size_t offset = size_t(channel) * pixels + pixel;
            const float difference = a.im.color[offset] - a.im.target_color[offset];
            rgb_loss += fabsf(difference);
            a.out.grad_color[offset] = a.photo_weight * 1.f * valid * inverse_pixels / 3.f *
                                       float((difference > 0.f) - (difference < 0.f));
        }
        if (a.photo_weight != 0.f)
            t_rgb = a.photo_weight * 1.f * valid * rgb_loss * inverse_pixels / 3.f;
        // relative robust depth term
        float grad_depth = 0.f;
        const float geometry_mask = o.ai_prior ? valid : 1.f;
        const bool has_depth = o.depth_weight > 0.f && a.im.target_depth[pixel] > 0.f &&
                               a.im.median_depth[pixel] > 0.f;
        if (has_depth && valid > 0.f) {
            const float target = a.im.target_depth[pixel];
            const float scale = fmaxf(target, 1e-4f);
            const float difference = (a.im.median_depth[pixel] - target) / scale;
            const float robust = sqrtf(difference * difference +
                                       o.geometry_epsilon * o.geometry_epsilon);
            grad_depth =
                geometry_mask * o.depth_weight * inverse_pixels * difference / (robust * scale);
            t_depth = geometry_mask * o.depth_weight * robust * inverse_pixels;
        }
        // normal prior
        float3 grad_normal = make_float3(0.f, 0.f, 0.f);
        float tx = 0.f, ty = 0.f, tz = 0.f, target_length2 = 0.f;
        if (o.normal_weight > 0.f) {
            tx = a.im.target_normal[pixel];
            ty = a.im.target_normal[pixels + pixel];
            tz = a.im.target_normal[2 * pixels + pixel];
            target_length2 = tx * tx + ty * ty + tz * tz;
        }
        if (target_length2 > 0.25f && valid > 0.f) {
            const float inverse_target_length = rsqrtf(target_length2);
            const float* n = a.im.normal;
            const float dot = n[pixel] * tx * inverse_target_length +
                              n[pixels + pixel] * ty * inverse_target_length +
                              n[2 * pixels + pixel] * tz * inverse_target_length;
            t_normal = geometry_mask * o.normal_weight * (1.f - dot) * inverse_pixels;
            grad_normal.x = -geometry_mask * o.normal_weight * tx * inverse_target_length *
                            inverse_pixels;
            grad_normal.y = -geometry_mask * o.normal_weight * ty * inverse_target_length *
                            inverse_pixels;
            grad_normal.z = -geometry_mask * o.normal_weight * tz * inverse_target_length *
                            inverse_pixels;
        }
        // transparent mode: BCE of alpha against the mask
        float grad_alpha = 0.f;
        if (o.mask_enabled && o.alpha_mode == 1 && o.match_alpha_weight > 0.f) {
            constexpr float clamp_epsilon = 1e-7f;
            const float raw = a.im.alpha[pixel];
            const float prediction = fminf(fmaxf(raw, clamp_epsilon), 1.f - clamp_epsilon);
            const bool inside = raw > clamp_epsilon && raw < 1.f - clamp_epsilon;
            const float background = 1.f - valid;
            grad_alpha = inside ? o.match_alpha_weight * inverse_pixels *
                                      (background * prediction - valid * (1.f - prediction)) /
                                      (prediction * (1.f - prediction))
                                : 0.f;
            t_alpha = -o.match_alpha_weight * inverse_pixels *
                      (valid * logf(prediction) + background * logf(1.f - prediction));
        }
        // depth-normal consistency: this pixel's own term and what its four
        // neighbours' terms send to its depth
        const bool consistency = o.depth_normal_weight > 0.f && a.out.grad_depth &&
                                 a.out.grad_normal;
        if (consistency) {
            const int W = a.im.width;
            const int x = int(pixel % W), y = int(pixel / W);
            const float normalization = o.depth_normal_weight / float(pixels);
            const DepthNormal self = depth_normal_at(a, x, y, normalization);
            if (self.ok) {
                t_normal += self.loss;
                grad_normal.x += -normalization * self.normal.x;
                grad_normal.y += -normalization * self.normal.y;
                grad_normal.z += -normalization * self.normal.z;
            }
            const float fx = a.im.fx, fy = a.im.fy, cx = a.im.cx, cy = a.im.cy;
            const float3 ray = make_float3((float(x) - cx) / fx, (float(y) - cy) / fy, 1.f);
            const DepthNormal above = depth_normal_at(a, x, y - 1, normalization); // we are its bottom
            if (above.ok)
                grad_depth += dot3(above.grad_dy, ray);
            const DepthNormal below = depth_normal_at(a, x, y + 1, normalization); // we are its top
            if (below.ok)
                grad_depth += -dot3(below.grad_dy, ray);
            const DepthNormal left = depth_normal_at(a, x - 1, y, normalization); // we are its right
            if (left.ok)
                grad_depth += dot3(left.grad_dx, ray);
            const DepthNormal right = depth_normal_at(a, x + 1, y, normalization); // we are its left
            if (right.ok)
                grad_depth += -dot3(right.grad_dx, ray);
        }
        a.out.grad_alpha[pixel] = grad_alpha;
        if (a.out.grad_depth)
            a.out.grad_depth[pixel] = grad_depth;
        if (a.out.grad_normal) {
            a.out.grad_normal[pixel] = grad_normal.x;
            a.out.grad_normal[pixels + pixel] = grad_normal.y;
            a.out.grad_normal[2 * pixels + pixel] = grad_normal.z;
        }
    }
    if (!a.partial)
        return;
    float t[4] = {t_rgb, t_depth, t_normal, t_alpha};
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            t[k] += __shfl_xor_sync(0xffffffffu, t[k], off);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            s_terms[threadIdx.x >> 5][k] = t[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        float s = 0.f;
        for (int w = 0; w < kThreads / 32; ++w)
            s += s_terms[w][threadIdx.x];
        a.partial[size_t(blockIdx.x) * 4 + threadIdx.x] = s;
    }
}

// terms[k] += sum over blocks of partial[block][k], in a fixed order (double).
__global__ void reduce_terms_kernel(const float* __restrict__ partial, int blocks,
                                    float* __restrict__ terms) {
    __shared__ double s[4][64];
    const int k = threadIdx.x >> 6, lane = threadIdx.x & 63;
    double v = 0.0;
    for (int b = lane; b < blocks; b += 64)
        v += partial[size_t(b) * 4 + k];
    s[k][lane] = v;
    __syncthreads();
    for (int w = 32; w > 0; w >>= 1) {
        if (lane < w)
            s[k][lane] += s[k][lane + w];
        __syncthreads();
    }
    if (lane == 0)
        terms[k] += float(s[k][0]);
}

} // namespace

size_t image_loss_partial_floats(int width, int height) {
    return 4 * ((size_t(width) * height + kThreads - 1) / kThreads);
}

cudaError_t launch_image_loss(cudaStream_t s, const ImageLossImages& im,
                              const ImageLossOptions& o, const ImageLossOutputs& out,
                              float photo_weight, float* partial) {
    const size_t pixels = size_t(im.width) * im.height;
    const int blocks = int((pixels + kThreads - 1) / kThreads);
    LossArgs a{im, o, out, photo_weight, out.terms ? partial : nullptr};
    image_loss_kernel<<<blocks, kThreads, 0, s>>>(a);
    if (out.terms)
        reduce_terms_kernel<<<1, 256, 0, s>>>(partial, blocks, out.terms);
    return cudaGetLastError();
}

} // namespace gsb
