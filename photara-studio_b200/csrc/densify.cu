// Densification kernels: per-step statistics, the plain adaptive-density
// control (ADC) decision rule, the learned-proposal policy, MLP features and
// the covariance-preserving split.
//
// Reference behaviour followed:
//   statistics  photara/src/splat/cuda_ops.cu:1548-1606 (accumulate_densification_kernel:
//               refine weight averaged over the views that see a Gaussian, max
//               screen radius; the error map accumulation of render_backward.cu:487-490)
//   split       photara/src/splat/cuda_ops.cu:1720-1845 (SplitMode::adc_covariance:
//               rank-one offset along the major axis, that axis shrunk by 1/sqrt(2),
//               opacity 1 - (1 - a)^(1/sqrt(2)) so the pair composites to the parent)
//   opacity reset photara/src/splat/trainer.cpp (opacity_reset_every)
// The decision rule is the classic ADC: prune below the opacity floor or when
// too large; otherwise a Gaussian whose averaged screen-space gradient passes
// the threshold is cloned when small and split when large.
#include "common.cuh"
#include "kernels.h"

namespace gsb {

__device__ __forceinline__ float sigmoidf_(float x) { return 1.f / (1.f + expf(-x)); }

__global__ void densify_accumulate_kernel(int n, const float* __restrict__ refine_weight,
                                          const int* __restrict__ radii,
                                          const float* __restrict__ densify_weight,
                                          const float* __restrict__ densify_weight_den,
                                          float inv_resolution,
                                          const float* __restrict__ means, float r0, float r1,
                                          float r2, float t2, DensifyStatsArgs s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || radii[i] <= 0)
        return;
    s.depth_acc[i] += r0 * means[3 * i] + r1 * means[3 * i + 1] + r2 * means[3 * i + 2] + t2;
    const float w = refine_weight ? refine_weight[i] : 0.f;
    s.grad_acc[i] += isfinite(w) ? fmaxf(w, 0.f) : 0.f;
    s.count[i] += 1.f;
    s.max_screen[i] = fmaxf(s.max_screen[i], float(radii[i]) * inv_resolution);
    if (densify_weight && densify_weight_den) {
        s.err_num[i] += densify_weight[i];
        s.err_den[i] += densify_weight_den[i];
    }
}

// One view's densification statistics with the reference kernel's full
// semantics (accumulate_densification_kernel, cuda_ops.cu:1548-1606): the
// step score (refine weight, clamped at 0, to step_score_power) summed or
// kept as a running max, the view count, the max screen size, the running max
// of a geometry score, the first view and two-view support, the summed image
// error, and the priority: accumulated log2 oversize evidence over the screen
// threshold (IGS), or score x (1 + screen).
__global__ void accumulate_densification_kernel(DensifyAccumArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n || a.radii[i] <= 0 || (a.require_visibility && a.visibility[i] <= 0.f))
        return;
    const float rw = a.refine_weight[i];
    const float raw = isfinite(rw) ? fmaxf(rw, 0.f) : 0.f;
    if (a.geometry_gradient && isfinite(a.geometry_gradient[i]))
        a.max_geometry_gradient[i] = fmaxf(a.max_geometry_gradient[i], a.geometry_gradient[i]);
    const float score = a.step_score_power == 1.f ? raw : powf(raw, a.step_score_power);
    a.gradient[i] = a.use_maximum ? fmaxf(a.gradient[i], score) : a.gradient[i] + score;
    a.count[i] += 1.f;
    if (a.image_error && isfinite(a.image_error[i]))
        a.accumulated_error[i] += fmaxf(a.image_error[i], 0.f);
    if (a.view_index >= 0) {
        const int first = a.first_view[i];
        if (first == 0) {
            a.first_view[i] = a.view_index + 1;
            a.view_support[i] = 1.f;
        } else if (first != a.view_index + 1) {
            a.view_support[i] = 2.f;
        }
    }
    const float screen =
        a.normalized_size ? a.normalized_size[i] : float(a.radii[i]) * a.inverse_resolution;
    a.max_screen_radius[i] = fmaxf(a.max_screen_radius[i], screen);
    a.priority[i] += a.oversize_screen_threshold > 0.f
                         ? fmaxf(log2f(screen / a.oversize_screen_threshold), 0.f)
                         : score * (1.f + screen);
}

cudaError_t launch_accumulate_densification(cudaStream_t st, const DensifyAccumArgs& a) {
    if (a.n > 0)
        accumulate_densification_kernel<<<(a.n + kBlock - 1) / kBlock, kBlock, 0, st>>>(a);
    return cudaGetLastError();
}

// Eight per-Gaussian features, standardised with (mean, inv_std):
//  0 log averaged screen gradient   1 max log-scale   2 min log-scale
//  3 opacity                        4 log(1 + views seen)
//  5 SH DC norm                     6 log(mean view depth / extent); for a
//                                      Gaussian no view saw: distance to the centre
//  7 age (refinement rounds since creation)
__global__ void densify_features_kernel(int n, const float* __restrict__ means,
                                        const float* __restrict__ log_scales,
                                        const float* __restrict__ logits,
                                        const float* __restrict__ sh, int sh_stride,
                                        DensifyStatsArgs s, float cx, float cy, float cz,
                                        float extent, const float* __restrict__ norm,
                                        float* __restrict__ feats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float cnt = s.count[i];
    const float grad = s.grad_acc[i] / fmaxf(cnt, 1.f);
    const float l0 = log_scales[3 * i], l1 = log_scales[3 * i + 1], l2 = log_scales[3 * i + 2];
    const float dx = means[3 * i] - cx, dy = means[3 * i + 1] - cy, dz = means[3 * i + 2] - cz;
    const float* dc = sh + size_t(i) * sh_stride;
    float f[8];
    f[0] = logf(grad + 1e-8f);
    f[1] = fmaxf(l0, fmaxf(l1, l2));
    f[2] = fminf(l0, fminf(l1, l2));
    f[3] = sigmoidf_(logits[i]);
    f[4] = log1pf(cnt);
    f[5] = sqrtf(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
    const float depth = cnt > 0.f ? s.depth_acc[i] / cnt : sqrtf(dx * dx + dy * dy + dz * dz);
    f[6] = logf(fmaxf(depth, 0.f) / extent + 1e-6f);
    f[7] = s.age[i];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        feats[size_t(i) * 8 + k] = norm ? (f[k] - norm[k]) * norm[8 + k] : f[k];
}

// Plain ADC decision: 0 keep, 1 split, 2 clone, 3 prune.
__global__ void adc_decide_kernel(int n, const float* __restrict__ log_scales,
                                  const float* __restrict__ logits, DensifyStatsArgs s,
                                  AdcArgs a, int* __restrict__ action) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float opacity = sigmoidf_(logits[i]);
    const float max_log =
        fmaxf(log_scales[3 * i], fmaxf(log_scales[3 * i + 1], log_scales[3 * i + 2]));
    const float max_scale = expf(max_log);
    int act = 0;
    if (!(opacity >= a.prune_opacity) || max_scale > a.prune_world_scale * a.extent ||
        (a.prune_screen > 0.f && s.max_screen[i] > a.prune_screen)) {
        act = 3;
    } else if (a.densify) {
        const float grad = s.grad_acc[i] / fmaxf(s.count[i], 1.f);
        if (grad >= a.grad_threshold)
            act = max_scale > a.percent_dense * a.extent ? 1 : 2;
    }
    action[i] = act;
}

// Learned proposal: argmax of the MLP logits when its softmax confidence
// reaches min_confidence, otherwise the plain heuristic's action (fallback).
// Densify proposals are only honoured for Gaussians the statistics saw.
__global__ void proposal_policy_kernel(int n, const float* __restrict__ logits,
                                       const int* __restrict__ fallback, DensifyStatsArgs s,
                                       float min_confidence, int* __restrict__ action) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float* z = logits + size_t(i) * 4;
    int best = 0;
    float zmax = z[0];
    for (int k = 1; k < 4; ++k)
        if (z[k] > zmax) {
            zmax = z[k];
            best = k;
        }
    float se = 0.f;
    for (int k = 0; k < 4; ++k)
        se += expf(z[k] - zmax);
    const float conf = 1.f / se;
    int act = conf >= min_confidence ? best : fallback[i];
    if ((act == 1 || act == 2) && !(s.count[i] > 0.f))
        act = fallback[i];
    if (fallback[i] == 3)
        act = 3; // hard prune rules (opacity floor, oversize) always apply
    action[i] = act;
}

// Covariance-preserving split of parents[k] into (parent, child k): both move
// by -/+ the rank-one offset along the parent's major axis (rotated to world),
// that axis shrinks by 1/sqrt(2), and both take opacity 1 - (1 - a)^(1/sqrt 2).
// Children rows [child0, child0 + count) already hold a copy of their parent.
__global__ void split_kernel(int count, const int* __restrict__ parents, int child0,
                             float* __restrict__ means, float* __restrict__ log_scales,
                             const float* __restrict__ quats, float* __restrict__ logits) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count)
        return;
    const int p = parents[k];
    const int c = child0 + k;
    float ls[3] = {log_scales[3 * p], log_scales[3 * p + 1], log_scales[3 * p + 2]};
    int major = 0;
    for (int ax = 1; ax < 3; ++ax)
        if (ls[ax] > ls[major]) major = ax;
    const float kk = 0.70710678118654752f;
    float local[3] = {0.f, 0.f, 0.f};
    local[major] = sqrtf(1.f - kk * kk) * expf(ls[major]);
    // rotate by the normalised quaternion (scalar first)
    float w = quats[4 * p], x = quats[4 * p + 1], y = quats[4 * p + 2], z = quats[4 * p + 3];
    const float inv = rsqrtf(fmaxf(w * w + x * x + y * y + z * z, 1e-20f));
    w *= inv; x *= inv; y *= inv; z *= inv;
    // rows of R (quat_to_rows) map world -> local, so world offset = R^T local
    const float R[3][3] = {{1.f - 2.f * (y * y + z * z), 2.f * (x * y + w * z), 2.f * (x * z - w * y)},
                           {2.f * (x * y - w * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z + w * x)},
                           {2.f * (x * z + w * y), 2.f * (y * z - w * x), 1.f - 2.f * (x * x + y * y)}};
    float off[3];
    for (int a = 0; a < 3; ++a)
        off[a] = R[0][a] * local[0] + R[1][a] * local[1] + R[2][a] * local[2];
    for (int a = 0; a < 3; ++a) {
        const float center = means[3 * p + a];
        means[3 * p + a] = center - off[a];
        means[3 * c + a] = center + off[a];
    }
    const float delta = logf(kk);
    log_scales[3 * p + major] = ls[major] + delta;
    log_scales[3 * c + major] = ls[major] + delta;
    const float op = sigmoidf_(logits[p]);
    const float revised =
        fminf(fmaxf(1.f - powf(fmaxf(1.f - op, 0.f), kk), 1e-6f), 1.f - 1e-6f);
    const float rl = logf(revised / (1.f - revised));
    logits[p] = rl;
    logits[c] = rl;
}

void launch_densify_accumulate(cudaStream_t st, int n, const float* refine_weight,
                               const int* radii, const float* dw, const float* dwd,
                               float inv_resolution, const float* means, const float* depth_row,
                               const DensifyStatsArgs& s) {
    if (n > 0)
        densify_accumulate_kernel<<<(n + 255) / 256, 256, 0, st>>>(
            n, refine_weight, radii, dw, dwd, inv_resolution, means, depth_row[0], depth_row[1],
            depth_row[2], depth_row[3], s);
}

void launch_densify_features(cudaStream_t st, int n, const float* means, const float* log_scales,
                             const float* logits, const float* sh, int sh_stride,
                             const DensifyStatsArgs& s, const float* center, float extent,
                             const float* norm, float* feats) {
    if (n > 0)
        densify_features_kernel<<<(n + 255) / 256, 256, 0, st>>>(
            n, means, log_scales, logits, sh, sh_stride, s, center[0], center[1], center[2],
            extent, norm, feats);
}

void launch_adc_decide(cudaStream_t st, int n, const float* log_scales, const float* logits,
                       const DensifyStatsArgs& s, const AdcArgs& a, int* action) {
    if (n > 0)
        adc_decide_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, log_scales, logits, s, a, action);
}

void launch_proposal_policy(cudaStream_t st, int n, const float* logits, const int* fallback,
                            const DensifyStatsArgs& s, float min_confidence, int* action) {
    if (n > 0)
        proposal_policy_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, logits, fallback, s,
                                                                min_confidence, action);
}

void launch_split(cudaStream_t st, int count, const int* parents, int child0, float* means,
                  float* log_scales, const float* quats, float* logits) {
    if (count > 0)
        split_kernel<<<(count + 255) / 256, 256, 0, st>>>(count, parents, child0, means,
                                                          log_scales, quats, logits);
}

} // namespace gsb
