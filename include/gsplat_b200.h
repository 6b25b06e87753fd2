/*
 * gsplat_b200 — C ABI of the B200 (sm_100a) 3D Gaussian Splatting rasterizer.
 *
 * Drop-in for the reference's splat rasterizer boundary:
 *   splat_drender::Rasterizer::forward   third_party/splat_drender/include/splat_drender/api.h:246
 *   splat_drender::Rasterizer::backward  third_party/splat_drender/include/splat_drender/api.h:264
 * as called by photara's CudaRasterizer (photara/src/splat/rasterizer.cu:390, :681).
 *
 * Conventions (same meaning as the reference POD structs, api.h:19-240):
 *  - every pointer in a struct is a DEVICE pointer unless marked HOST;
 *  - the caller owns every input and output buffer; the context owns the
 *    workspace (what the reference takes through WorkspacePools callbacks);
 *  - forward() writes every pixel of colour/alpha and every radius itself
 *    (no pre-zeroing needed); backward() ACCUMULATES into gradient buffers
 *    (api.h:262-263), except where fused Adam updates parameters in place;
 *  - no C++ exception crosses this boundary: every entry point returns a
 *    gs_status and gs_last_error() holds the message (the reference throws
 *    std::invalid_argument / std::runtime_error / std::logic_error,
 *    third_party/splat_drender/src/pipeline.cu:63-72, :655);
 *  - all work is enqueued on the context's stream (gs_set_stream).
 */
#ifndef GSPLAT_B200_H
#define GSPLAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_ABI_VERSION 3

#if defined(__GNUC__)
#define GS_API __attribute__((visibility("default")))
#else
#define GS_API
#endif

typedef enum {
    GS_OK = 0,
    GS_ERR_INVALID = 1,  /* bad argument   (reference: std::invalid_argument) */
    GS_ERR_CUDA = 2,     /* CUDA failure   (reference: std::runtime_error)    */
    GS_ERR_STATE = 3,    /* call order     (reference: std::logic_error)      */
    GS_ERR_CAPACITY = 4, /* fixed-capacity buffer too small (batched/no-alloc paths) */
    GS_ERR_TIMEOUT = 5   /* a bounded device-side wait gave up                 */
} gs_status;

typedef struct gs_context gs_context;

/* Gaussians (api.h:19-58, raw activation branch api.h:35-40 as photara binds it,
 * photara/src/splat/rasterizer.cu:226-246). Exactly one of sh / colors. */
typedef struct {
    int count;                    /* N */
    const float* means;           /* [N,3] world space */
    const float* log_scales;      /* [N,3] */
    const float* quaternions;     /* [N,4] scalar-first, not necessarily normalised */
    const float* opacity_logits;  /* [N] */
    const float* filter_3d;       /* [N] or NULL (Mip-Splatting 3D filter) */
    const float* sh;              /* [N,sh_bases,3] coefficient-major, RGB inner, or NULL */
    const float* colors;          /* [N,3] precomputed colours, or NULL */
    int sh_degree;                /* active degree 0..3 */
    int sh_bases;                 /* row length of sh in RGB triples (1,4,9,16) */
} gs_gaussians;

/* Pinhole camera (api.h:19-32). The matrix and centre are passed BY VALUE
 * (the reference takes device pointers filled by a 1-block upload kernel,
 * photara/src/splat/rasterizer.cu:152-168; values need no upload and keep the
 * launch graph-capturable). world_to_camera is column-major 4x4. */
typedef struct {
    int width, height;
    float fx, fy, cx, cy;
    float near_plane;             /* default 0.2  */
    float alpha_clip;             /* default 0.99 */
    int compensate_2d;            /* Mip 2D opacity compensation sqrt(det0/det1) */
    float world_to_camera[16];
    float center[3];
} gs_camera;

/* Render settings (api.h:60-90, the fields the pinhole RGB path reads). */
typedef struct {
    float background[3];
    float scale_modifier;         /* default 1 */
    float kernel_size;            /* screen-space dilation added to cov2D */
    int record_backward_state;    /* 0: inference-only render, backward refused */
    int need_depth;               /* 1: also the median depth and normal channels (ABI 2) */
} gs_settings;

/* Forward outputs (api.h:92-99). visibility may be NULL. With need_depth,
 * median_depth and normal are required (ABI 2): the median depth along each
 * pixel ray as camera-space Z (0 where the pixel's transmittance stays above
 * 0.45 or the bisection bracket misses the crossing) and the alpha-normalised
 * camera-space footprint normal (render_forward.cu:421-525). The backward does
 * not differentiate these two channels. */
typedef struct {
    float* color;                 /* [3,H,W] planar */
    float* alpha;                 /* [H,W] 1 - final transmittance */
    float* visibility;            /* [N] 1 where >= 1 blended sample, else untouched */
    int* radii;                   /* [N] pixel radius, 0 = culled */
    float* median_depth;          /* [H,W] with need_depth, else ignored */
    float* normal;                /* [3,H,W] with need_depth, else ignored */
} gs_outputs;

/* What forward() reports (ForwardResult, api.h:214-223). */
typedef struct {
    int instance_count;           /* (Gaussian, tile) pairs drawn */
    int visible_count;            /* Gaussians with >= 1 tile */
    int depth_bits;               /* rebased depth-key bits sorted (visible Gaussians) */
    int tile_bits;                /* tile-id bits sorted (instances) */
    int tiles;                    /* tile grid size */
} gs_forward_info;

/* Per-pixel loss gradients (LossGradients, api.h:108-117). alpha may be NULL.
 * median_depth / normal: gradients of the geometry channels, only after a
 * forward with need_depth (else GS_ERR_STATE); NULL when not differentiated. */
typedef struct {
    const float* color;           /* [3,H,W] dL/dcolor */
    const float* alpha;           /* [H,W] dL/dalpha or NULL */
    const float* densify_map;     /* [H,W] optional error map or NULL */
    const float* median_depth;    /* [H,W] dL/d median depth or NULL */
    const float* normal;          /* [3,H,W] dL/d normal or NULL */
} gs_loss_grads;

/* Gradient outputs (ModelGradients, api.h:192-211). Every pointer may be NULL.
 * activated == 0: scale/rotation/opacity gradients are with respect to the RAW
 *   parameters (log_scales, quaternions, opacity_logits);
 * activated != 0: with respect to the activated values (exp scale, normalised
 *   quaternion, sigmoid opacity), the reference's convention for its
 *   host-side chain rule (photara/src/splat/rasterizer.cu:674-676). */
typedef struct {
    float* means;                 /* [N,3] */
    float* scales;                /* [N,3] */
    float* rotations;             /* [N,4] */
    float* opacities;             /* [N]   */
    float* sh;                    /* [N,sh_bases,3] */
    float* colors;                /* [N,3] when forward used precomputed colours */
    float* refine_weight;         /* [N] sum ||(W,H) * dL/dmean2d|| / max(1-T_final,1e-5) */
    float* densify_weight;        /* [N] sum err * alpha * T   (needs densify_map) */
    float* densify_weight_den;    /* [N] sum alpha * T         (needs densify_map) */
    int activated;
} gs_model_grads;

/* Fused structure Adam (StructureAdam, api.h:122-158): updates means,
 * log_scales, quaternions and opacity logits in place inside the per-Gaussian
 * backward; culled rows still decay their moments. */
typedef struct {
    float* means;          float* log_scales;     float* quaternions;    float* opacity_logits;
    float* means_first;    float* means_second;
    float* scales_first;   float* scales_second;
    float* rotations_first; float* rotations_second;
    float* opacity_first;  float* opacity_second;
    const float* filter_3d;
    float means_lr, scales_lr, quaternions_lr, opacities_lr;
    float beta1, beta2, correction1, correction2, epsilon;
    float minimum_log_scale, maximum_log_scale;
    float opacity_reg, scale_reg;
    float shape_erank_reg, shape_erank_s3_reg, shape_quat_norm_reg;
    float shape_axis_ratio_reg, shape_max_axis_ratio;
    float* opacity_gradient;      /* optional [N] logit gradient capture */
} gs_structure_adam;

/* Fused quantized SH Adam (SHAdam, api.h:107-120; codec
 * include/splat_drender/sh_adam_quant.cuh:1-234): FP16 normalised first
 * moment, uint8 log second moment, per-row float4 bounds (DC / rest). */
typedef struct {
    float* parameter;             /* [N,stride] (the model's SH, updated in place) */
    float lr, rest_lr, beta1, beta2, correction1, correction2, epsilon;
    float regularization_factor;
    void* first;                  /* [N,stride] fp16 */
    uint8_t* packed;              /* [N,stride] u8   */
    float* bounds;                /* [N,4]           */
    int stride;                   /* sh_bases*3, <= 48 */
} gs_sh_adam;

/* ---- context -------------------------------------------------------------- */
/* Creates a context on `device` enqueuing on `stream` (cudaStream_t, may be 0). */
GS_API gs_status gs_create(gs_context** out, int device, void* stream);
GS_API void gs_destroy(gs_context* ctx);
GS_API gs_status gs_set_stream(gs_context* ctx, void* stream);
GS_API const char* gs_last_error(const gs_context* ctx);
GS_API int gs_abi_version(void);
/* Bytes of device workspace currently held by the context. */
GS_API size_t gs_workspace_bytes(const gs_context* ctx);

/* ---- rasterizer boundary (api.h:246, :264) ------------------------------------ */
/* Renders one view (Rasterizer::forward). info may be NULL. The Gaussian and
 * camera inputs must stay alive and unchanged until the matching backward.
 * The host waits once, for the draw counts (pipeline.cu:208-212); the sorts
 * and the compositing are only enqueued. A look-back wait of those sorts that
 * gave up (a broken invariant: every wait is bounded, none hangs) is reported
 * as GS_ERR_TIMEOUT by whatever consumes the draw list next (gs_backward,
 * gs_forward_colors, gs_pruning_scores, gs_debug_draw_list), by
 * gs_device_status, or by the next gs_forward; the forward's images are then
 * not valid. A staging wait of the compositing kernels that gave up (the same
 * kind of broken invariant) is reported by gs_device_status or the next
 * gs_forward. */
GS_API gs_status gs_forward(gs_context* ctx, const gs_gaussians* g, const gs_camera* cam,
                     const gs_settings* s, const gs_outputs* out, gs_forward_info* info);

/* Backward of the last forward on this context (Rasterizer::backward).
 * fwd_alpha/fwd_radii are the forward outputs. adam / sh_adam may be NULL;
 * when given, the update is fused and the matching gradient outputs are not
 * written (as in the reference, photara/src/splat/rasterizer.cu:663-669).
 * With dL->median_depth or dL->normal (render_backward.cu:47-519, the
 * GEOMETRY branches), the forward's median_depth and normal outputs are read
 * again, as the reference reads them (ForwardOutputsView, api.h:102-107):
 * they must be unchanged since the forward. */
GS_API gs_status gs_backward(gs_context* ctx, const float* fwd_alpha, const int* fwd_radii,
                      const gs_loss_grads* dL, const gs_model_grads* grads,
                      const gs_structure_adam* adam, const gs_sh_adam* sh_adam);

/* Waits for the context's stream and reports whether any bounded device-side
 * wait of the work enqueued on this context gave up since the last report
 * (GS_ERR_TIMEOUT, and the word is cleared), e.g. after an inference-only
 * forward that nothing consumes. The reference has no counterpart (its CUB
 * sorts cannot time out). */
GS_API gs_status gs_device_status(gs_context* ctx);

/* Test hook for the bounded waits (no counterpart in the reference): runs ONE
 * look-back wait of the scan kernel (which = 0) or of a onesweep pass
 * (which = 1) whose predecessor tile is never published, with the wait limited
 * to spin_limit re-reads (1 .. 2^20) instead of the library's 2^22, or
 * (which = 2) the compositing kernels' staging wait on an mbarrier phase that
 * no copy completes, limited to spin_limit suspended waits of ~1 us. The wait
 * gives up, sets the device error word and the kernel returns; the call waits
 * for it and returns GS_ERR_TIMEOUT (the expected outcome) with the context
 * still usable. Every access stays inside the probe's own scratch. */
GS_API gs_status gs_debug_lookback_probe(gs_context* ctx, int which, unsigned spin_limit);

/* Measurement hook (no counterpart in the reference): the (Gaussian, pixel)
 * pairs the compositing kernels of the last colour training forward evaluate,
 * pairs_out[0] for the forward (pixel not yet saturated when its warp takes
 * the Gaussian), pairs_out[1] for the adjoint (Gaussian at or before the
 * pixel's last contributor); HOST array of 2. Re-renders the forward into
 * color / alpha (identical images) with counting kernels and waits for them. */
GS_API gs_status gs_debug_composite_pairs(gs_context* ctx, float* color, float* alpha,
                                          unsigned long long* pairs_out);

/* Compositing schedule: pixels per thread of the per-tile forward/backward
 * kernels (1: 256-thread CTAs, 2: 128, 4: 64, 8: 32), or 0 (the default):
 * chosen per frame from the tile count (fewer pixels per thread for frames
 * with too few tiles to fill the GPU). Results are the same either way
 * (forward bit-identical, gradients up to float-atomic order). */
GS_API gs_status gs_set_schedule(gs_context* ctx, int pixels_per_thread);

/* Debug export of the last forward's draw list for bit-exact comparison:
 * sorted 64-bit keys (tile << 32 | depth bits) [instance_count], Gaussian ids
 * in composite order [instance_count], tile ranges [tiles][2]. Any may be NULL. */
GS_API gs_status gs_debug_draw_list(gs_context* ctx, unsigned long long* keys_out,
                             unsigned* values_out, unsigned* ranges_out);

/* Per-stage device times in milliseconds, averaged over the forward+backward
 * steps completed since timing was enabled, measured with CUDA events on the
 * context stream (no extra host synchronisation per step):
 * [0] preprocess [1] depth sort + offset scan [2] duplicate-with-keys
 * [3] tile sort [4] tile ranges [5] composite [6] composite backward
 * [7] gaussian backward (+Adam); [8] (if n > 8) number of steps averaged. */
GS_API gs_status gs_enable_stage_timing(gs_context* ctx, int enable);
GS_API gs_status gs_stage_times(gs_context* ctx, float* ms_out, int n);

/* ---- device-wide primitives (replace the reference's CUB calls,
 *      third_party/splat_drender/src/pipeline.cu:186-311) ------------------------- */
/* Exclusive prefix sum of n u32 (decoupled look-back, one pass). total_out is a
 * device pointer receiving the sum (may be NULL). Scratch comes from the context. */
GS_API gs_status gs_exclusive_scan_u32(gs_context* ctx, const unsigned* in, unsigned* out, int n,
                                       unsigned* total_out);
/* Stable LSD onesweep radix sort of (u64 key, u32 value) pairs on key bits
 * [begin_bit, end_bit): keys_in/vals_in are left unchanged, the sorted pairs
 * are written to keys_out/vals_out. Ping-pong storage comes from the context;
 * the call reuses the context's draw-list buffers, so a backward of an earlier
 * forward on the same context is refused afterwards (GS_ERR_STATE). */
GS_API gs_status gs_sort_pairs_u64(gs_context* ctx, const unsigned long long* keys_in,
                                   const unsigned* vals_in, unsigned long long* keys_out,
                                   unsigned* vals_out, size_t count, int begin_bit, int end_bit);

/* Colour reuse (splat_drender Rasterizer::forward_colors,
 * third_party/splat_drender/src/pipeline.cu:617-649): after a training forward
 * (record_backward_state) of a model with precomputed colours (gs_gaussians
 * colors set, sh NULL), blends `colors` ([N][3], device) over the same draw
 * list into out->color / alpha / visibility (median depth and normal are not
 * rendered). The context's forward state then describes these colours: a
 * gs_backward that follows differentiates this blend. GS_ERR_STATE without
 * such a forward. */
GS_API gs_status gs_forward_colors(gs_context* ctx, const float* colors, const gs_outputs* out);

/* Speedy-Splat pruning scores of the context's last forward
 * (CudaRasterizer::pruning_scores, photara/src/splat/rasterizer.cu:450-490,
 * kernel :93-146): adds to scores[i] (device float [N]) the sum over the
 * pixels Gaussian i was blended into of (o (T c - R / (1 - a)))^2, with c its
 * colour sum and R the colour sum behind it (background included), or with
 * gaussian_pop != 0 the squared norm of the per-channel a (T c_k - R_k / (1 - a)).
 * image is that forward's colour output [3,H,W]; the forward must have
 * recorded backward state (record_backward_state), GS_ERR_STATE otherwise. */
GS_API gs_status gs_pruning_scores(gs_context* ctx, const float* image, int gaussian_pop,
                                   float* scores);

/* Fused L1 + SSIM photometric loss (cuda_backend::fused_l1_ssim_loss,
 * photara/src/splat/fused_ssim.cu, the loss photara's trainer backpropagates
 * into the rasterizer): prediction, target [3,H,W]; mask [H,W] or NULL (both
 * images are multiplied by it, and so is the gradient). Adds dL/dprediction to
 * grad_out [3,H,W]; adds to loss_out (device float, may be NULL)
 *   w / (3 (W-10)(H-10)) * sum over the valid window of
 *   [ssim_weight (1 - SSIM) + (1 - ssim_weight) |a - b|],  w = photometric_weight.
 * GS_ERR_INVALID unless width and height are > 10 (the reference throws). */
GS_API gs_status gs_fused_l1_ssim(gs_context* ctx, const float* prediction, const float* target,
                                  const float* mask, int width, int height, float ssim_weight,
                                  float photometric_weight, float* grad_out, float* loss_out);
/* Mean SSIM over the valid window (and the mask's nonzero pixels) into out
 * (device float); 0 when width or height is <= 10 (cuda_backend::fused_ssim_metric). */
GS_API gs_status gs_ssim_metric(gs_context* ctx, const float* prediction, const float* target,
                                const float* mask, int width, int height, float* out);

/* Training loss of one rendered view (cuda_backend::compute_training_loss,
 * photara/src/splat/cuda_ops.cu:2731-2822, pinhole cameras): the per-pixel
 * terms of loss_kernel (cuda_ops.cu:846-966), the fused L1 + SSIM term when
 * width and height are > 10 (else the plain L1 term), and the depth-normal
 * consistency term (depth_normal_consistency_kernel, cuda_ops.cu:999-1071).
 * All images are device float arrays: colour [3,H,W], alpha [H,W],
 * median_depth [H,W], normal [3,H,W] (gs_forward with need_depth), targets of
 * the same shapes, mask [H,W]. An image may be NULL when no enabled term reads
 * it. */
typedef struct {
    const float* color;
    const float* alpha;
    const float* median_depth;
    const float* normal;
    const float* target_color;
    const float* target_depth;  /* > 0 where a depth observation exists */
    const float* target_normal; /* |n|^2 > 0.25 where a normal observation exists */
    const float* mask;
    int width, height;
    float fx, fy, cx, cy; /* pinhole intrinsics (depth-normal consistency) */
} gs_loss_images;

typedef struct {
    float photometric_weight;
    float ssim_weight;         /* clamped to [0, 1] */
    float depth_weight;        /* resolved weight of the depth term (0: off) */
    float normal_weight;       /* resolved weight of the normal term (0: off) */
    float depth_normal_weight; /* consistency term (0: off; needs both gradient images) */
    float match_alpha_weight;
    float geometry_epsilon;
    int mask_enabled;
    int alpha_mode; /* -1 validity mask, 0 masked (alpha unsupervised), 1 transparent (BCE) */
    int ai_prior;   /* the mask also weights the geometry terms */
} gs_loss_options;

typedef struct {
    float* grad_color;  /* [3,H,W], written */
    float* grad_alpha;  /* [H,W], written */
    float* grad_depth;  /* [H,W] or NULL, written */
    float* grad_normal; /* [3,H,W] or NULL, written */
    float* terms;       /* [4] rgb, depth, normal, alpha, added to; may be NULL */
} gs_loss_outputs;

GS_API gs_status gs_training_loss(gs_context* ctx, const gs_loss_images* images,
                                  const gs_loss_options* options, const gs_loss_outputs* out);

/* Allocation-free variant of gs_exclusive_scan_u32 (no counterpart in the
 * reference). For callers that may not allocate device memory where they scan:
 * cudaMalloc synchronises the device, and it is unavailable to plugins whose
 * host owns all device memory. Needs no context; enqueues on `stream`
 * (cudaStream_t, may be 0).
 *  - n <= 33,554,432 (2^25) elements, else GS_ERR_CAPACITY and nothing runs;
 *  - scratch is a fixed ~128 KiB device array inside the library, kept on every
 *    device that loads it until the process exits; the first call on a device
 *    looks up that array's device address (a one-time set-up with the device
 *    current), so make the first call before any stream capture;
 *  - all calls share that array: calls whose work may overlap on the GPU
 *    (different unordered streams) race and give undefined results; calls
 *    ordered on one stream are safe;
 *  - calls no cudaMalloc / cudaFree and no allocating library routine;
 *  - returns GS_ERR_INVALID for null buffers or n < 0, GS_ERR_CUDA if a CUDA
 *    call fails; GS_OK means the scan was enqueued, not that it finished: a
 *    look-back wait that gave up (a broken invariant) leaves a partial prefix
 *    and is reported by gs_exclusive_scan_u32_noalloc_status. */
GS_API gs_status gs_exclusive_scan_u32_noalloc(const unsigned* in, unsigned* out, int n,
                                               unsigned* total_out, void* stream);
/* Error word of the last allocation-free scan (no counterpart in the
 * reference): enqueues on `stream` a copy of it into *status_out (device or
 * host memory the caller owns): 0 when every look-back wait completed,
 * GS_ERR_TIMEOUT's device bit (1) when one gave up. Order it after the scan
 * (same stream) and read it once the stream has reached it. Allocates nothing. */
GS_API gs_status gs_exclusive_scan_u32_noalloc_status(unsigned* status_out, void* stream);

/* ---- standalone kernels on the training step (photara/src/splat/cuda_ops.cu) -- */
/* L1 photometric loss gradient (cuda_ops.cu:846-891): grad = w/(3P) * sign(img - target),
 * loss_out (device, 1 float, accumulated) = w/(3P) * sum |img - target|. */
GS_API gs_status gs_l1_loss(gs_context* ctx, const float* image, const float* target, int pixels,
                     float weight, float* grad_out, float* loss_out);

/* Standalone Adam over a flat parameter array (cuda_ops.cu:1336, adam_scalar
 * semantics render_backward.cu:525-550): NaN-resetting, clamped. */
GS_API gs_status gs_adam(gs_context* ctx, float* param, const float* grad, float* first, float* second,
                  size_t n, float lr, float beta1, float beta2, float correction1,
                  float correction2, float epsilon, float clamp_min, float clamp_max);

/* ---- densification (photara/src/splat/cuda_ops.cu:1548-1845) --------------------- */
/* Per-Gaussian statistics between refinements, all [N] float32 device arrays. */
typedef struct {
    float* grad_acc;   /* sum of refine weights over the views that saw the Gaussian */
    float* count;      /* number of such views */
    float* max_screen; /* max radius / max(W, H) */
    float* err_num;    /* sum of error * alpha * T (needs a densify map in backward) */
    float* err_den;    /* sum of alpha * T */
    float* depth_acc;  /* sum of view-space depth over the views that saw the Gaussian */
    float* age;        /* refinement rounds since creation */
} gs_densify_stats;

/* Plain adaptive density control thresholds (classic 3DGS rule). */
typedef struct {
    float grad_threshold;    /* averaged refine weight that triggers densification */
    float percent_dense;     /* clone when max scale <= percent_dense * extent, else split */
    float extent;            /* scene extent (world units) */
    float prune_opacity;     /* prune below this opacity */
    float prune_world_scale; /* prune when max scale > prune_world_scale * extent */
    float prune_screen;      /* prune when max screen radius fraction exceeds this (0 = off) */
    int densify;             /* 0: prune only */
} gs_adc_params;

/* Adds one view's backward outputs to the statistics (accumulate_densification_kernel).
 * means [N][3] and depth_row_host = the view matrix's third row (r20 r21 r22 t2)
 * give the view-space depth accumulated into depth_acc. */
GS_API gs_status gs_densify_accumulate(gs_context* ctx, int n, const float* refine_weight,
                                       const int* radii, const float* densify_weight,
                                       const float* densify_weight_den, float inv_resolution,
                                       const float* means, const float* depth_row_host,
                                       const gs_densify_stats* stats);
/* Densification statistics of one view with the reference kernel's full
 * semantics (accumulate_densification_kernel, photara/src/splat/cuda_ops.cu:
 * 1548-1606, the statistics ADC-IGS reads, ops.hpp DensificationStats). Rows
 * with radius 0, or with zero visibility when require_visibility, are left
 * alone. All arrays are [N] device arrays; optional ones may be NULL. */
typedef struct {
    const float* refine_weight;     /* this view's refine weight (backward output) */
    const float* visibility;        /* forward visibility (read when require_visibility) */
    const int* radii;               /* forward radii */
    float* gradient;                /* sum, or running max (use_maximum), of the step score */
    float* count;                   /* views that saw the row */
    float* max_screen_radius;       /* max screen size: radius * inverse_resolution */
    float* priority;                /* IGS: summed log2 oversize; else step score x (1 + screen) */
    const float* geometry_gradient; /* optional per-view score kept as a running max */
    float* max_geometry_gradient;   /* with geometry_gradient */
    int* first_view;                /* with view_index >= 0: 1 + first view seen (0: none) */
    float* view_support;            /* 1 after one view, 2 after a second distinct view */
    const float* image_error;       /* optional per-view error, summed when finite */
    float* accumulated_error;       /* with image_error */
    const float* normalized_size;   /* optional screen size replacing radius * inverse_resolution */
    int count_rows;                 /* N */
    float inverse_resolution;       /* 1 / min(width, height) (adc_ops.cpp:43) */
    int use_maximum;
    int require_visibility;
    float step_score_power;         /* the score is refine_weight^power (1: unchanged) */
    float oversize_screen_threshold;/* > 0: priority adds max(log2(screen / threshold), 0) */
    int view_index;                 /* < 0: no view support tracking */
} gs_densify_accum;

GS_API gs_status gs_accumulate_densification(gs_context* ctx, const gs_densify_accum* args);

/* Eight standardised features per Gaussian ([N][8]) for the proposal MLP;
 * norm = 16 floats (means, inverse stds) or NULL for raw features. */
GS_API gs_status gs_densify_features(gs_context* ctx, int n, const float* means,
                                     const float* log_scales, const float* opacity_logits,
                                     const float* sh, int sh_stride, const gs_densify_stats* stats,
                                     const float* center3_host, float extent, const float* norm,
                                     float* features_out);
/* Plain ADC decision per Gaussian: 0 keep, 1 split, 2 clone, 3 prune. */
GS_API gs_status gs_adc_decide(gs_context* ctx, int n, const float* log_scales,
                               const float* opacity_logits, const gs_densify_stats* stats,
                               const gs_adc_params* params, int* action_out);
/* Learned proposal: MLP argmax where its softmax confidence >= min_confidence,
 * else the plain decision `fallback`; hard prunes of the fallback always apply. */
GS_API gs_status gs_proposal_policy(gs_context* ctx, int n, const float* logits,
                                    const int* fallback, const gs_densify_stats* stats,
                                    float min_confidence, int* action_out);
/* Covariance-preserving split of parents[k] into itself and row child0 + k
 * (which must already hold a copy of the parent). */
GS_API gs_status gs_split_gaussians(gs_context* ctx, int count, const int* parents, int child0,
                                    float* means, float* log_scales, const float* quaternions,
                                    float* opacity_logits);

/* Split operators of photara's densification (cuda_backend::split_gaussians,
 * photara/src/splat/cuda_ops.cu:1720-1845, 3105-3122; SplitMode order):
 * 0 adc_covariance (rank-one offset along the major axis, k = 1/sqrt 2 or
 * tighter where screen_sizes[k] > split_at_screen_size), 1 dense_tangent,
 * 2 igs_random, 3 long_axis. Parent rows parents[k] of the parent arrays move
 * by -offset; child row k of the child arrays is written at +offset (its log
 * scales must hold the parent's, the split adds the same delta to both);
 * both take the mode's opacity. random_samples [count][3] (modes 1, 2),
 * screen_sizes [count] or NULL (mode 0). minimum_opacity, split_at_screen_size
 * and split_opacity_k are clamped as the reference's host function does. */
typedef struct {
    float* parent_means;
    float* parent_log_scales;
    float* parent_opacity_logits;
    const float* parent_quaternions;
    float* child_means;
    float* child_log_scales;
    float* child_opacity_logits;
    const int* parents;
    const float* random_samples;
    const float* screen_sizes;
    int count;
    int mode;
    float minimum_opacity;
    float split_at_screen_size;
    float split_opacity_k;
} gs_split_args;
GS_API gs_status gs_split_gaussians_mode(gs_context* ctx, const gs_split_args* args);
/* ADC decay (cuda_backend::apply_adc_decay, cuda_ops.cu:3388-3400): opacity
 * minus max(opacity_decay, 0), clamped to (1e-12, 1 - 1e-12); every log scale
 * plus log(max(1 - scale_decay, 1e-6)). */
GS_API gs_status gs_adc_decay(gs_context* ctx, size_t count, float* log_scales,
                              float* opacity_logits, float opacity_decay, float scale_decay);
/* Row selection for pruning (select_training_rows_gpu,
 * photara/src/splat/densification_adc_plus.cpp:68-77): gs_select_rows writes
 * the kept rows' indices in increasing order (keep[i] != 0) to indices_out
 * and their number to *count_out (device int); gs_gather_rows then writes
 * dst_a[i] = src_a[indices[i]] for i < count and every array a (the model's
 * parameters, both Adam moments, the quantized SH-Adam rows ...), rows of
 * row_bytes[a] bytes (a multiple of 4), up to 32 arrays per call, sources and
 * destinations distinct; every index must be below the row count of every
 * source (indices from gs_select_rows over the same rows are). */
GS_API gs_status gs_select_rows(gs_context* ctx, int n, const unsigned char* keep,
                                int* indices_out, int* count_out);
GS_API gs_status gs_gather_rows(gs_context* ctx, int count, const int* indices, int arrays,
                                const void* const* src, void* const* dst,
                                const size_t* row_bytes);

/* ---- proposal MLP: 8 -> 64 -> 64 -> 4, BF16 weights, FP32 accumulation ------------- */
GS_API int gs_mlp_param_count(void);
/* logits_out [n][4] from features [n][8]; weights_bf16 [gs_mlp_param_count()]. */
GS_API gs_status gs_mlp_forward(gs_context* ctx, int n, const float* features,
                                const void* weights_bf16, float* logits_out);
/* Accumulates d(loss)/d(weights) into grad_out (FP32, caller-zeroed) and the
 * loss into *loss_out for softmax cross-entropy against labels (0..3) with
 * per-row weights normalised by 1 / weight_sum. */
GS_API gs_status gs_mlp_train_step(gs_context* ctx, int n, const float* features,
                                   const int* labels, const float* row_weights,
                                   const void* weights_bf16, float weight_sum, float* grad_out,
                                   float* loss_out);
/* Adam on the FP32 master weights; rewrites the BF16 image. */
GS_API gs_status gs_mlp_adam(gs_context* ctx, float* master, void* weights_bf16,
                             const float* grad, float* first, float* second, float lr,
                             float beta1, float beta2, float correction1, float correction2,
                             float epsilon);

/* ---- batched multi-view rendering ------------------------------------------------
 * Many views of uneven resolution rendered and differentiated together: every
 * stage is one launch over all views, tiles of every view feed one persistent
 * compositing launch, and after gs_batch_plan nothing allocates or
 * synchronises, so forward + backward capture into one CUDA graph
 * (gs_batch_capture / gs_batch_replay). Per view the results are those of
 * gs_forward / gs_backward on that camera; gradients are summed over views.
 * No reference counterpart: the reference renders one view per call
 * (photara/src/splat/rasterizer.cu:390, :681); this replaces a loop of such calls.
 * Image layout: views concatenated in order, colour planar [3][H_v][W_v] per
 * view, alpha [H_v][W_v]; per-pair arrays (radii) are [views][N]. */
typedef struct gs_batch gs_batch;

typedef struct {
    int tile_w, tile_h;       /* 8x8, 16x16 or 16x32 (width x height) */
    int pixels_per_thread;    /* 1|2 for 8x8, 2|4 for 16x16 and 16x32 */
    int schedule;             /* 0 static stride, 1 dynamic queue, 2 heaviest tiles first */
    int ctas_per_sm;          /* persistent CTAs per SM; 0 = as many as fit */
} gs_batch_schedule;

typedef struct {
    size_t pairs;             /* views * N */
    size_t instance_capacity; /* planned (Gaussian, tile) capacity */
    size_t total_pixels;      /* sum of W*H over views */
    int total_tiles;
    int views;
    long long instances;      /* requested by the last forward (after a sync) */
    int visible;              /* visible (view, Gaussian) pairs of the last forward */
    int overflow;             /* 1: the last forward needed more than the capacity */
    int device_error;         /* device error word of the last step (0 = none) */
} gs_batch_info;

GS_API gs_status gs_batch_create(gs_batch** out, int device, void* stream);
GS_API void gs_batch_destroy(gs_batch* b);
GS_API const char* gs_batch_last_error(const gs_batch* b);
GS_API gs_status gs_batch_set_stream(gs_batch* b, void* stream);
/* Records the Gaussians (pointers, which must stay valid and fixed in size),
 * copies the cameras and allocates every buffer for the schedule (NULL: 16x16,
 * 4 pixels per thread, dynamic). instance_capacity 0 sizes the instances from a
 * counting pass (+25%); a later forward that needs more sets `overflow`. */
GS_API gs_status gs_batch_plan(gs_batch* b, const gs_gaussians* g, const gs_camera* cams,
                               int views, const gs_settings* s, const gs_batch_schedule* sched,
                               size_t instance_capacity);
/* Synchronises the stream and reports sizes and the last forward's counts. */
GS_API gs_status gs_batch_get_info(gs_batch* b, gs_batch_info* out);
/* Enqueues the forward of every view (radii_out [views][N] may be NULL). */
GS_API gs_status gs_batch_forward(gs_batch* b, float* color, float* alpha, int* radii_out);
/* Enqueues the backward of the last forward; gradients (summed over views)
 * ACCUMULATE into grads; dL_alpha may be NULL. */
GS_API gs_status gs_batch_backward(gs_batch* b, const float* dL_color, const float* dL_alpha,
                                   const gs_model_grads* grads);
/* Captures forward (+ backward when dL_color is not NULL) with these buffers
 * into a CUDA graph; gs_batch_replay launches it on the batch stream. */
GS_API gs_status gs_batch_capture(gs_batch* b, float* color, float* alpha, int* radii_out,
                                  const float* dL_color, const float* dL_alpha,
                                  const gs_model_grads* grads);
GS_API gs_status gs_batch_replay(gs_batch* b);
/* Times forward + backward (CUDA events, `iterations` after 2 warm-ups) for
 * every tile shape / pixels-per-thread / schedule candidate, plans the fastest
 * and returns it in *best (*best_ms its time). tried / tried_ms (capacity
 * *n_tried on entry, count on return) receive every candidate; may be NULL. */
GS_API gs_status gs_batch_autotune(gs_batch* b, const gs_gaussians* g, const gs_camera* cams,
                                   int views, const gs_settings* s, int iterations,
                                   gs_batch_schedule* best, float* best_ms,
                                   gs_batch_schedule* tried, float* tried_ms, int* n_tried);

#ifdef __cplusplus
}
#endif
#endif /* GSPLAT_B200_H */
