/*
 * CPU restatement of the reference's pinhole 3DGS rasterizer path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker. Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it; the
 * product library never links or calls it.
 *
 * Follows (reference paths within the photara-studio project):
 *   activation      third_party/splat_drender/src/device/activation.cuh:13-31
 *   projection      third_party/splat_drender/src/device/geometry.cuh:127-277
 *   screen cov cap  third_party/splat_drender/src/device/footprint.cuh:14-48
 *   tile walk       third_party/splat_drender/src/device/tiles.cuh:115-179
 *   SH colour       third_party/splat_drender/src/device/sh.cuh:19-173
 *   preprocess      third_party/splat_drender/src/render_forward.cu:30-139
 *   composite       third_party/splat_drender/src/render_forward.cu:341-416, :508-525
 *   median depth    third_party/splat_drender/src/render_forward.cu:421-525 (GEOMETRY)
 *   ray plane       third_party/splat_drender/src/device/geometry.cuh:255-275
 *   composite bwd   third_party/splat_drender/src/render_backward.cu:156-519 (RGB branch)
 *   gaussian bwd    third_party/splat_drender/src/device/geometry.cuh:317-912 (pinhole RGB)
 *   Adam            third_party/splat_drender/src/render_backward.cu:525-550, :650-706
 *   SH Adam codec   third_party/splat_drender/include/splat_drender/sh_adam_quant.cuh:23-234
 * Every loop takes a [begin, end) range (Gaussians or tiles) so the caller can
 * run disjoint ranges on several host threads (the Python wrapper does, with
 * one private gradient buffer per thread for the compositing adjoint).
 * Precision: the geometry and colour math run in float (no contraction, IEEE
 * division/sqrt, so per-value results sit within a few ulp of the reference's
 * fast-math GPU build); compositing and its adjoint can run in double
 * (`use_double`) as the FP64 scalar oracle.
 */
#ifndef SPLAT_ORACLE_H
#define SPLAT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    float view[16]; /* column-major world-to-camera */
    float center[3];
    float fx, fy, cx, cy;
    float near_plane, alpha_clip;
    int width, height;
    int compensate_2d;
    float kernel_size, scale_modifier;
} orc_camera;

/* Per-Gaussian preprocess. Outputs (length n unless noted): mean2d[2n],
 * conic[4n] (xx, xy, yy, opacity*coef), rgb[3n], clamp[n] (bits), depth[n]
 * (radial distance), radii[n], touched[n], bounds[4n] (x0,x1,y0,y1). */
void orc_preprocess(int n, const float* means, const float* log_scales, const float* quats,
                    const float* logits, const float* sh, int sh_degree, int sh_bases,
                    const orc_camera* cam, float* mean2d, float* conic, float* rgb,
                    uint8_t* clamp, float* depth, int* radii, uint32_t* touched,
                    int32_t* bounds, int begin, int end);

/* Writes the (tile << 32 | float bits of depth) keys and Gaussian ids of every
 * instance of Gaussian i at offsets[i] (exclusive scan of touched). */
void orc_emit(int n, const float* mean2d, const float* conic, const float* depth,
              const uint32_t* touched, const uint64_t* offsets, int grid_x, int grid_y,
              uint64_t* keys, uint32_t* values);

/* Front-to-back compositing of every tile. ranges[2*tiles], order = Gaussian
 * ids in draw order. Outputs color[3P], alpha[P], T_final[P], last[P],
 * visibility[n] (set to 1 where blended). use_double: accumulate in double. */
void orc_composite(int tiles, const uint32_t* ranges, const uint32_t* order, const float* mean2d,
                   const float* conic, const float* rgb, const orc_camera* cam, const float* bg,
                   int use_double, double* color, double* alpha, double* T_final,
                   uint32_t* last, float* visibility, int tile_begin, int tile_end);

/* Ray planes [4n] and footprint normals [3n] of the visible Gaussians
 * (radii > 0), for the median-depth and normal channels. */
void orc_geometry(int n, const float* means, const float* log_scales, const float* quats,
                  const float* logits, const orc_camera* cam, const int* radii, float* plane,
                  float* normal, int begin, int end);

/* Median depth [P] (camera-space Z, 0 outside range) and alpha-normalised
 * normal [3P] of every pixel of tiles [tile_begin, tile_end). FP32. */
void orc_median_depth(int tiles, const uint32_t* ranges, const uint32_t* order,
                      const float* mean2d, const float* conic, const float* plane,
                      const float* normal, const orc_camera* cam, float* depth, float* normal_out,
                      int tile_begin, int tile_end);

/* Reverse-order adjoint of the compositing (RGB + alpha losses). grad12[12n]
 * accumulates per Gaussian: dconic.xyz (xy half), d(opacity*coef), dmean2d.xy,
 * refine magnitude, 0, dcolor.rgb, 0. Uses the stored T_final/last. */
void orc_composite_backward(int tiles, const uint32_t* ranges, const uint32_t* order,
                            const float* mean2d, const float* conic, const float* rgb,
                            const orc_camera* cam, const float* bg, const double* T_final,
                            const uint32_t* last, const float* dL_color, const float* dL_alpha,
                            int n, double* grad12, int tile_begin, int tile_end);

/* Per-Gaussian adjoint. activated != 0: scale/rotation/opacity gradients with
 * respect to activated values (reference convention); else w.r.t. the raw
 * log scale / quaternion / logit. Outputs accumulate. */
void orc_gaussian_backward(int n, const float* means, const float* log_scales,
                           const float* quats, const float* logits, const float* sh,
                           int sh_degree, int sh_bases, const orc_camera* cam, const int* radii,
                           const uint8_t* clamp, const double* grad12, int activated,
                           double* g_means, double* g_scales, double* g_rots, double* g_opac,
                           double* g_sh, int begin, int end);

/* Adam on a flat array with the reference's NaN handling and clamps. */
void orc_adam(float* param, const float* grad, float* m, float* v, long n, float lr, float b1,
              float b2, float c1, float c2, float eps, float lo, float hi);

/* Quantized SH Adam of `rows` rows (codec of sh_adam_quant.cuh). */
void orc_sh_adam_rows(int rows, int stride, int active, float* param, const float* grad,
                      uint16_t* first_half, uint8_t* packed, float* bounds, float lr,
                      float rest_lr, float b1, float b2, float c1, float c2, float eps,
                      float regularization);

#ifdef __cplusplus
}
#endif
#endif
