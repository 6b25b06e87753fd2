// Host-visible launchers of the device kernels (internal to the library).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace gsb {

struct Camera;
struct GaussianState;
struct SplatRec;

// Gradient outputs of the per-Gaussian backward (ModelGradients subset).
struct GradOutArgs {
    float* means;
    float* scales;
    float* rotations;
    float* opacities;
    float* sh;
    float* colors;
    float* refine_weight;
    float* densify_weight;
    float* densify_weight_den;
    int activated;
};

struct StructureAdamArgs {
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
    const float* filter_3d;
    float means_lr, scales_lr, quaternions_lr, opacities_lr;
    float beta1, beta2, correction1, correction2, epsilon;
    float minimum_log_scale, maximum_log_scale;
    float opacity_reg, scale_reg;
    float shape_erank_reg, shape_erank_s3_reg, shape_quat_norm_reg;
    float shape_axis_ratio_reg, shape_max_axis_ratio;
    float* opacity_gradient;
};

struct ShAdamArgs {
    float* parameter;
    float lr, rest_lr, beta1, beta2, correction1, correction2, epsilon;
    float regularization;
    void* first;
    uint8_t* packed;
    float* bounds;
    int stride;
};

// Per-Gaussian densification statistics (all [N] float32).
struct DensifyStatsArgs {
    float* grad_acc;   // sum of refine weights over views that saw the Gaussian
    float* count;      // views that saw it
    float* max_screen; // max radius / max(W, H)
    float* err_num;    // sum of error * alpha * T
    float* err_den;    // sum of alpha * T
    float* depth_acc;  // sum of view-space depth over the views that saw it
    float* age;        // refinement rounds since creation
};

struct AdcArgs {
    float grad_threshold, percent_dense, extent;
    float prune_opacity, prune_world_scale, prune_screen;
    int densify; // 0: prune only
};

struct DensifyAccumArgs {
    const float* refine_weight;
    const float* visibility;
    const int* radii;
    float* gradient;
    float* count;
    float* max_screen_radius;
    float* priority;
    const float* geometry_gradient;
    float* max_geometry_gradient;
    int* first_view;
    float* view_support;
    const float* image_error;
    float* accumulated_error;
    const float* normalized_size;
    int n;
    float inverse_resolution;
    int use_maximum;
    int require_visibility;
    float step_score_power;
    float oversize_screen_threshold;
    int view_index;
};
cudaError_t launch_accumulate_densification(cudaStream_t st, const DensifyAccumArgs& a);
void launch_densify_accumulate(cudaStream_t st, int n, const float* refine_weight,
                               const int* radii, const float* dw, const float* dwd,
                               float inv_resolution, const float* means, const float* depth_row,
                               const DensifyStatsArgs& s);
void launch_densify_features(cudaStream_t st, int n, const float* means, const float* log_scales,
                             const float* logits, const float* sh, int sh_stride,
                             const DensifyStatsArgs& s, const float* center, float extent,
                             const float* norm, float* feats);
void launch_adc_decide(cudaStream_t st, int n, const float* log_scales, const float* logits,
                       const DensifyStatsArgs& s, const AdcArgs& a, int* action);
void launch_proposal_policy(cudaStream_t st, int n, const float* logits, const int* fallback,
                            const DensifyStatsArgs& s, float min_confidence, int* action);
void launch_split(cudaStream_t st, int count, const int* parents, int child0, float* means,
                  float* log_scales, const float* quats, float* logits);
int mlp_param_count();
void launch_mlp_forward(cudaStream_t s, int n, const float* feats, const void* w_bf16,
                        float* logits);
void launch_mlp_train(cudaStream_t s, int n, const float* feats, const int* labels,
                      const float* weights, const void* w_bf16, float inv_wsum, float* grad,
                      float* loss);
void launch_mlp_adam(cudaStream_t s, float* master, void* w_bf16, const float* grad, float* m,
                     float* v, float lr, float b1, float b2, float c1, float c2, float eps);

void launch_preprocess(cudaStream_t s, int n, const float* means, const float* log_scales,
                       const float* quats, const float* logits, const float* filter_3d,
                       const float* sh, const float* colors, int sh_degree, int sh_bases,
                       const Camera& K, const GaussianState& st, int* radii, unsigned* counters);
// Visible Gaussians only, compacted in index order, with the depth sort's
// digit histograms counted into hist (zeroed by the caller). status must hold
// one u64 per 2,048 Gaussians.
// The depth range (and so the key bits counted) is read from the frame
// counters on the device. zeroed: status, tile counter (and hist) were
// zeroed by the caller.
void launch_depth_compact(cudaStream_t s, int n, const GaussianState& st,
                          const unsigned* counters, unsigned* keys, unsigned* values,
                          unsigned* hist, unsigned long long* status, unsigned* tile_counter,
                          unsigned* err, bool zeroed = false);
void launch_frame_counters_init(cudaStream_t s, unsigned* counters);
// emit_keys also counts the following radix sort's digit histograms (key bits
// [0, bits)) into hist, which the caller zeroes. Its warps take the visible
// Gaussians in groups of about 2^group_shift instances: groups[] are the group
// starts from the offset scan (launch_scan with the same group_shift),
// `instances` the total. The group size is 512 instances once there are
// enough groups to fill the GPU (about 32 warps per SM), smaller below that.
inline int emit_group_shift(unsigned instances) {
    int shift = 9;
    while (shift > 5 && (instances >> shift) < 148u * 32u)
        --shift;
    return shift;
}
inline unsigned emit_group_count(unsigned instances, int group_shift) {
    return unsigned((size_t(instances) + (size_t(1) << group_shift) - 1) >> group_shift);
}
void launch_emit_keys(cudaStream_t s, int visible, unsigned instances, const unsigned* groups,
                      int group_shift, const unsigned* order, const GaussianState& st,
                      int grid_x, int grid_y, unsigned* keys, unsigned* values,
                      unsigned capacity, int bits, unsigned* hist);
void launch_tile_ranges(cudaStream_t s, int count, const unsigned* keys, uint2* ranges,
                        int tiles);
void launch_compose_keys(cudaStream_t s, int count, const unsigned* tiles,
                         const unsigned* values, const unsigned* depth,
                         unsigned long long* out);

// Elements per look-back tile of the single-pass scan (256 threads x 8).
constexpr int kScanItems = 8;
constexpr int kScanTile = 256 * kScanItems;
size_t scan_status_bytes(int n);
// Bytes of device scratch launch_lookback_probe needs.
size_t lookback_probe_bytes();
// Runs one look-back wait (which: 0 scan, 1 onesweep pass) whose predecessor
// is never published, so it gives up after spin_limit re-reads and sets
// kDevLookbackTimeout in *err (for tests of the bounded waits).
void launch_lookback_probe(cudaStream_t s, int which, unsigned spin_limit, char* scratch,
                           unsigned* err);
// groups (optional, group_cap entries, at most (total >> group_shift) + 1 of
// them written): see scan_kernel.
void launch_scan(cudaStream_t s, int n, const unsigned* in, const unsigned* index, unsigned* out,
                 unsigned long long* status, unsigned* tile_counter, unsigned* total,
                 unsigned* err, bool zeroed = false, unsigned* groups = nullptr,
                 int group_shift = 0, unsigned group_cap = 0);
int radix_passes(int bits);
size_t sort_status_bytes(size_t count, int passes);
template <typename Key>
int launch_radix_sort(cudaStream_t s, Key* keys[2], unsigned* vals[2], size_t count,
                      const unsigned* count_dev, int begin_bit, int end_bit, unsigned* hist,
                      unsigned* status, unsigned* tile_counters, unsigned* err,
                      bool hist_ready = false, bool zeroed = false);

// TMA staging of the single-view colour compositing kernels: the tensor map
// of the Gaussians' 64-byte records (GaussianState::rec as [rows][16] floats,
// a box of one row, for tile::gather4) and the device error word their
// bounded waits report to.
struct RecStaging {
    CUtensorMap map;
    unsigned* err;
};

// One CTA whose staging wait (the compositing kernels' mbarrier wait) is never
// satisfied: gives up after `limit` suspended waits of ~1 us and sets
// kDevStageTimeout in *err.
void launch_stage_probe(cudaStream_t s, unsigned limit, unsigned* err);

void launch_composite_forward(cudaStream_t s, int tiles, const uint2* ranges,
                              const unsigned* order, const GaussianState& st, const Camera& K,
                              float3 bg, float* color, float* alpha, float* pix_T,
                              unsigned* pix_last, float* visibility, int pixels_per_thread,
                              const RecStaging& rs, unsigned* tile_work = nullptr);
// Tiles by descending adjoint work (tile_work from launch_composite_forward,
// zeroed before it): a permutation of [0, tiles) into order.
void launch_tile_order(cudaStream_t s, const unsigned* work, int tiles, unsigned* order);
// Fused L1 + SSIM loss: grad += dL/dpred, *loss_out (may be NULL) = L;
// Training-loss terms of one view (image_loss.cu); field meanings as the
// C ABI's gs_loss_images / gs_loss_options / gs_loss_outputs.
struct ImageLossImages {
    const float* color;
    const float* alpha;
    const float* median_depth;
    const float* normal;
    const float* target_color;
    const float* target_depth;
    const float* target_normal;
    const float* mask;
    int width, height;
    float fx, fy, cx, cy;
};
struct ImageLossOptions {
    float depth_weight, normal_weight, depth_normal_weight, match_alpha_weight,
        geometry_epsilon;
    int mask_enabled, alpha_mode, ai_prior;
};
struct ImageLossOutputs {
    float* grad_color;
    float* grad_alpha;
    float* grad_depth;
    float* grad_normal;
    float* terms;
};
size_t image_loss_partial_floats(int width, int height);
cudaError_t launch_image_loss(cudaStream_t s, const ImageLossImages& im,
                              const ImageLossOptions& o, const ImageLossOutputs& out,
                              float photo_weight, float* partial);

// Densification apply (densify_apply.cu). mode: 0 adc_covariance,
// 1 dense_tangent, 2 igs_random, 3 long_axis (photara SplitMode order).
struct SplitModeArgs {
    float* parent_means;
    float* parent_log_scales;
    float* parent_opacity_logits;
    const float* parent_quaternions;
    float* child_means;
    float* child_log_scales; // hold the parents' values; the split adds its delta
    float* child_opacity_logits;
    const int* parents;
    const float* random_samples; // [count][3]
    const float* screen_sizes;   // [count] or NULL
    int count;
    int mode;
    float minimum_opacity, split_at_screen_size, split_opacity_k;
};
cudaError_t launch_split_mode(cudaStream_t s, const SplitModeArgs& a);
cudaError_t launch_adc_decay(cudaStream_t s, float* log_scales, float* opacity_logits,
                             size_t count, float opacity_decay, float log_scale_decay);
size_t select_rows_scratch_words(int n);
cudaError_t launch_select_rows(cudaStream_t s, const unsigned char* keep, int n, int* indices,
                               int* count_out, unsigned* scratch);
constexpr int kMaxGatherArrays = 32;
struct GatherArray {
    const void* src;
    void* dst;
    int row_words; // 4-byte words per row
    int vec4;      // rows and bases allow 16-byte words
};
struct GatherRowsArgs {
    const int* indices;
    int count;
    int arrays;
    GatherArray array[kMaxGatherArrays];
};
cudaError_t launch_gather_rows(cudaStream_t s, const GatherRowsArgs& g, int sm_count);

// partial holds ssim_partial_floats(width, height) floats of scratch.
size_t ssim_partial_floats(int width, int height);
cudaError_t launch_fused_l1_ssim(cudaStream_t s, const float* pred, const float* target,
                                 const float* mask, int width, int height, float ssim_weight,
                                 float photometric_weight, float* grad, float* loss_out,
                                 float* partial);
// Mean SSIM over the valid window and the mask's nonzero pixels into *out.
cudaError_t launch_ssim_metric(cudaStream_t s, const float* pred, const float* target,
                               const float* mask, int width, int height, float* out,
                               float* partial);
// The colour forward plus the median-depth and normal channels (st.plane and
// st.normal filled by the preprocess); colour outputs as launch_composite_forward.
// pix_dtdt [H,W] (training forwards; NULL otherwise): dT/dt at the median
// depth, for the geometry-channel backward.
void launch_composite_geometry(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, float* color, float* alpha, float* pix_T,
                               unsigned* pix_last, float* pix_dtdt, float* visibility,
                               float* median_depth, float* normal);
// Evaluated (Gaussian, pixel) pairs of the colour forward (pairs[0]) and its
// adjoint (pairs[1]) for the last forward's draw list; pairs zeroed by the
// caller; color / alpha receive the (identical) re-rendered images.
void launch_composite_count_pairs(cudaStream_t s, int tiles, const uint2* ranges,
                                  const unsigned* order, const GaussianState& st,
                                  const Camera& K, float3 bg, float* color, float* alpha,
                                  const float* pix_T, const unsigned* pix_last,
                                  int pixels_per_thread, unsigned long long* pairs,
                                  const RecStaging& rs);
// Backward of the colour, median-depth and normal channels of a geometry
// forward: adds per-Gaussian partials to st.grad and st.geo_grad. dL_depth /
// dL_normal may be NULL (not both: the colour adjoint serves that case).
void launch_composite_backward_geometry(cudaStream_t s, int tiles, const uint2* ranges,
                                        const unsigned* order, const GaussianState& st,
                                        const Camera& K, float3 bg, const float* pix_T,
                                        const unsigned* pix_last, const float* pix_dtdt,
                                        const float* dL_color, const float* dL_alpha,
                                        const float* densify_map, int want_refine,
                                        const float* dL_depth, const float* dL_normal,
                                        const float* fwd_depth, const float* fwd_normal);
void launch_composite_backward(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, const float* pix_T, const unsigned* pix_last,
                               const float* dL_color, const float* dL_alpha,
                               const float* densify_map, int want_refine,
                               int pixels_per_thread, const RecStaging& rs,
                               const unsigned* tile_order = nullptr);

cudaError_t launch_pruning_scores(cudaStream_t s, int tiles, const uint2* ranges,
                                  const unsigned* order, const GaussianState& st, const Camera& K,
                                  const unsigned* pix_last, const float* image, int gaussian_pop,
                                  float* scores);

cudaError_t launch_set_colors(cudaStream_t s, int n, const float* colors, float4* rgb,
                              SplatRec* rec);

size_t gaussian_backward_smem(bool fused_sh);
void launch_gaussian_backward(cudaStream_t s, int n, const float* means, const float* log_scales,
                              const float* quats, const float* logits, const float* filter_3d,
                              const float* sh, int sh_degree, int sh_bases, const Camera& K,
                              const GaussianState& st, const int* radii, const GradOutArgs& out,
                              const StructureAdamArgs* sa, const ShAdamArgs* sha,
                              bool geometry = false);
void launch_adam(cudaStream_t s, float* p, const float* g, float* m, float* v, size_t n, float lr,
                 float b1, float b2, float c1, float c2, float eps, float lo, float hi);
void launch_l1(cudaStream_t s, const float* img, const float* tgt, size_t n, float scale,
               float* grad, float* loss);

} // namespace gsb
