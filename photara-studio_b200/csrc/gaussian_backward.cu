// Per-Gaussian backward (EWA projection adjoint + SH adjoint) fused with the
// Adam updates, plus the standalone Adam and L1-loss kernels of the step.
//
// Reference behaviour followed:
//   gaussian_backward        third_party/splat_drender/src/render_backward.cu:708-862
//   splat_backward (pinhole RGB chain, conic / cap / cov3D / J / mean2d)
//                            third_party/splat_drender/src/device/geometry.cuh:317-912
//   update_structure_adam_row, adam_scalar, shape regularizers
//                            third_party/splat_drender/src/render_backward.cu:525-706
//   quantized SH Adam codec  third_party/splat_drender/include/splat_drender/sh_adam_quant.cuh:23-234
//   standalone Adam / L1     photara/src/splat/cuda_ops.cu:846-891, :1336
//
// B200 organisation: 128 Gaussians per CTA. Phase 1, one thread per
// Gaussian: the CTA's SH rows (contiguous in HBM) and, with the fused SH Adam,
// their fp16 first moments, u8 codes and code bounds are staged through shared
// memory with coalesced asynchronous copies while the per-Gaussian inputs
// load; then each thread runs its Gaussian's projection and SH adjoints and
// the structure Adam from registers. The SH adjoint leaves the row's basis
// values and clamped colour gradient in shared memory (19 words instead of the
// 48 coefficient gradients: each gradient is one product of the two).
// Phase 2, the quantized SH Adam: degree-3 rows one thread per row (new
// parameters straight to HBM as 16-byte row segments, log-second values in
// the parameters' shared slots, first moments and codes in place and written
// back coalesced); other strides one half-warp per row. 440 bytes of shared
// memory per Gaussian and a 128-register bound give 4 CTAs (16 warps) per SM
// (the thread-per-row layout with a gradient row took 544 bytes: 3 CTAs).
#include <cuda_fp16.h>

#include <algorithm>

#include "adjoint.cuh"
#include "common.cuh"
#include "kernels.h"

namespace gsb {

constexpr int kGBlock = 128;
constexpr int kShStride = 49; // padded float row (odd: conflict-free per-thread walks)

// ------------------------------------------------------------------ Adam --
__device__ __forceinline__ void adam_one(float* param, size_t idx, float grad, float* first,
                                         float* second, float lr, float b1, float b2, float c1,
                                         float c2, float eps, float lo, float hi) {
    const float prev = param[idx];
    if (!isfinite(prev) || !isfinite(grad)) {
        first[idx] = 0.f;
        second[idx] = 0.f;
        param[idx] = isfinite(prev) ? fminf(fmaxf(prev, lo), hi) : fminf(fmaxf(0.f, lo), hi);
        return;
    }
    const float m = b1 * first[idx] + (1.f - b1) * grad;
    const float v = b2 * second[idx] + (1.f - b2) * grad * grad;
    if (!isfinite(m) || !isfinite(v)) {
        first[idx] = 0.f;
        second[idx] = 0.f;
        param[idx] = fminf(fmaxf(prev, lo), hi);
        return;
    }
    first[idx] = m;
    second[idx] = v;
    const float cand = prev - lr * (m / c1) / (sqrtf(v / c2) + eps);
    const float upd = isfinite(cand) ? cand : prev;
    param[idx] = fminf(fmaxf(upd, lo), hi);
}

// Adam on register values (same arithmetic as adam_one); returns the new
// parameter and updates m / v in place.
__device__ __forceinline__ float adam_reg(float prev, float grad, float& m, float& v, float lr,
                                          float b1, float b2, float c1, float c2, float eps,
                                          float lo, float hi) {
    if (!isfinite(prev) || !isfinite(grad)) {
        m = 0.f;
        v = 0.f;
        return isfinite(prev) ? fminf(fmaxf(prev, lo), hi) : fminf(fmaxf(0.f, lo), hi);
    }
    const float mm = b1 * m + (1.f - b1) * grad;
    const float vv = b2 * v + (1.f - b2) * grad * grad;
    if (!isfinite(mm) || !isfinite(vv)) {
        m = 0.f;
        v = 0.f;
        return fminf(fmaxf(prev, lo), hi);
    }
    m = mm;
    v = vv;
    const float cand = prev - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    const float upd = isfinite(cand) ? cand : prev;
    return fminf(fmaxf(upd, lo), hi);
}

// Shape priors on (log scale, quaternion) (render_backward.cu:552-648).
// Works on private copies (dynamic axis indices put them in local memory) and
// adds the result to the caller's register arrays with constant indices.
struct PriorGrad {
    float log_s[3];
    float quat[4];
};

__device__ __noinline__ PriorGrad shape_priors_delta(float ls0, float ls1, float ls2, float q0,
                                                     float q1, float q2, float q3,
                                                     const StructureAdamArgs a) {
    const float ls[3] = {ls0, ls1, ls2};
    const float q[4] = {q0, q1, q2, q3};
    PriorGrad out;
    float* g_log = out.log_s;
    float* g_quat = out.quat;
    for (int k = 0; k < 3; ++k) g_log[k] = 0.f;
    for (int k = 0; k < 4; ++k) g_quat[k] = 0.f;
    if (a.shape_quat_norm_reg > 0.f) {
        const float ns = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        if (ns > 1e-20f) {
            const float nrm = sqrtf(ns);
            const float f = a.shape_quat_norm_reg * (nrm - 1.f) / ns;
            for (int c = 0; c < 4; ++c)
                g_quat[c] += f * q[c];
        }
    }
    if (a.shape_axis_ratio_reg > 0.f) {
        int hi = 0, lo = 0;
        for (int k = 1; k < 3; ++k) {
            if (ls[k] > ls[hi]) hi = k;
            if (ls[k] < ls[lo]) lo = k;
        }
        const float excess = ls[hi] - ls[lo] - logf(a.shape_max_axis_ratio);
        if (excess > 0.f && isfinite(excess)) {
            g_log[hi] += a.shape_axis_ratio_reg * excess;
            g_log[lo] -= a.shape_axis_ratio_reg * excess;
        }
    }
    if (a.shape_erank_reg <= 0.f && a.shape_erank_s3_reg <= 0.f)
        return out;
    float l[3];
    int largest = 0;
    for (int k = 0; k < 3; ++k) {
        l[k] = ls[k];
        if (!(l[k] > -1e4f)) l[k] = -1e4f;
        if (k > 0 && l[k] > l[largest]) largest = k;
    }
    float x[3];
    for (int k = 0; k < 3; ++k)
        x[k] = expf(2.f * (l[k] - l[largest]));
    const float sum = x[0] + x[1] + x[2];
    if (!(sum > 0.f))
        return out;
    int smallest = 0;
    for (int k = 1; k < 3; ++k)
        if (x[k] < x[smallest]) smallest = k;
    const float p_large = x[largest] / sum;
    const float raw_small = x[smallest] / sum;
    const bool small_clamped = !(raw_small > 1e-30f);
    const float p_small = small_clamped ? 1e-30f : raw_small;
    const float mid_c = 1.f - p_large - p_small;
    const bool mid_clamped = !(mid_c > 1e-30f);
    const float p_mid = mid_clamped ? 1e-30f : mid_c;
    const float entropy = -(p_large * logf(p_large) + p_mid * logf(p_mid) + p_small * logf(p_small));
    const float rank = expf(entropy);
    float dshare[3] = {0.f, 0.f, 0.f};
    if (a.shape_erank_reg > 0.f && rank - 0.99999f < 1.f) {
        const float p[3] = {p_large, p_mid, p_small};
        for (int k = 0; k < 3; ++k)
            dshare[k] = a.shape_erank_reg * rank * (logf(p[k]) + 1.f) / (rank - 0.99999f);
    }
    const float d_small_total = dshare[2] + a.shape_erank_s3_reg;
    float dx[3];
    for (int k = 0; k < 3; ++k) {
        const float d_large = k == largest ? (1.f - p_large) / sum : -p_large / sum;
        float d_small = 0.f;
        if (k == smallest) {
            if (!small_clamped) d_small = (1.f - p_small) / sum;
        } else {
            d_small = -p_small / sum;
        }
        const float d_mid = mid_clamped ? 0.f : -(d_large + d_small);
        dx[k] = dshare[0] * d_large + dshare[1] * d_mid + d_small_total * d_small;
    }
    for (int k = 0; k < 3; ++k) {
        if (k == largest) {
            float pull = 0.f;
            for (int o = 0; o < 3; ++o)
                if (o != largest) pull += dx[o] * x[o];
            g_log[k] += -2.f * pull;
        } else {
            g_log[k] += dx[k] * 2.f * x[k];
        }
    }
    return out;
}

// ------------------------------------------------------- SH quant codec --
constexpr float kCodecEps = 1e-15f;

__device__ __forceinline__ float codec_prev_correction(float c, float beta) {
    return beta > 0.f ? fmaxf((c - (1.f - beta)) / beta, 0.f) : 0.f;
}
__device__ __forceinline__ float codec_to_normalized(float m, float v, float c1, float c2,
                                                     float eps) {
    if (c1 <= 0.f || c2 <= 0.f)
        return 0.f;
    return (m / c1) / (sqrtf(fmaxf(v, 0.f) / c2) + eps);
}
// The codec's expm1 / log1p pair (decode / encode of the log second moment)
// runs on the exp / log intrinsics: log values are either 0 (a coefficient
// with no second moment, exact either way) or large (sqrt(v) / 1e-15 >> 1),
// where exp(x) - 1 and log(1 + y) lose nothing; only second moments below
// ~1e-31, far under the update's epsilon, see a difference. With the
// software expm1f / log1pf the kernel took 0.627 ms at 1M Gaussians, with the
// intrinsics 0.568 ms.
__device__ __forceinline__ float codec_log_to_second(float log_s) {
    const float s = kCodecEps * (__expf(log_s) - 1.f);
    return s * s;
}

// One coefficient of one row, on registers. `first` is the stored fp16
// normalised update (as float) on entry and the new one on exit, `param` the
// coefficient before and after; returns the log-second value to re-encode.
__device__ __forceinline__ float sh_adam_column(int col, int active, float& param, float grad_in,
                                                float& first, unsigned code, float lo, float hi,
                                                const ShAdamArgs& a) {
    float log_s = lo + (hi - lo) * (float(code) * (1.f / 255.f));
    const float g2 = codec_log_to_second(log_s);
    const float stored = first;
    const float pc1 = codec_prev_correction(a.correction1, a.beta1);
    const float pc2 = codec_prev_correction(a.correction2, a.beta2);
    float g1 = 0.f;
    if (pc1 > 0.f) {
        const float sv = pc2 > 0.f ? sqrtf(fmaxf(g2, 0.f) / pc2) : 0.f;
        g1 = stored * (sv + a.epsilon) * pc1;
    }
    if (col >= active) {
        if (!isfinite(g1)) g1 = 0.f;
        if (!isfinite(log_s)) {
            log_s = 0.f;
            g1 = 0.f;
        }
        const float enc = codec_to_normalized(g1, codec_log_to_second(log_s), a.correction1,
                                              a.correction2, a.epsilon);
        first = isfinite(enc) ? enc : 0.f;
        return log_s;
    }
    float grad = grad_in;
    const float prev = param;
    if (a.regularization > 0.f && col >= 3 && isfinite(prev))
        grad += a.regularization * prev;
    if (!isfinite(prev) || !isfinite(grad)) {
        first = 0.f;
        param = isfinite(prev) ? prev : 0.f;
        return 0.f;
    }
    const float m = a.beta1 * g1 + (1.f - a.beta1) * grad;
    const float v = a.beta2 * g2 + (1.f - a.beta2) * grad * grad;
    if (!isfinite(m) || !isfinite(v)) {
        first = 0.f;
        return 0.f;
    }
    const float lr = col >= 3 ? a.rest_lr : a.lr;
    const float nrm = codec_to_normalized(m, v, a.correction1, a.correction2, a.epsilon);
    const float cand = prev - lr * nrm;
    param = isfinite(cand) ? cand : prev;
    first = nrm;
    float ls = __logf(1.f + sqrtf(fmaxf(v, 0.f)) * (1.f / kCodecEps));
    if (!isfinite(ls)) ls = 0.f;
    return ls;
}

// inv_range = 1 / max(hi - lo, eps), computed once per row and group (the
// division it replaces is the same reciprocal-multiply under fast math).
__device__ __forceinline__ uint8_t codec_encode(float value, float lo, float inv_range) {
    const float code = fminf(fmaxf(roundf(255.f * (value - lo) * inv_range), 0.f), 255.f);
    return static_cast<uint8_t>(code);
}

// ---------------------------------------------- SH Adam, degree-3 rows --
// The common case (48 coefficients per row, all active) on a shorter
// instruction path with the same arithmetic: launch constants are folded once
// per thread; sqrt(v / c2) is sqrt(v) / sqrt(c2) and sqrt(g2 / pc2) is
// |s| / sqrt(pc2), so one square root per coefficient serves the update and
// the re-encoded log value; the u8 code becomes a float and the re-encode
// rounding becomes an integer without conversion instructions (the special
// function unit was the kernel's busiest pipe); fp16 moments move as half2
// pairs and codes as 32-bit words.
struct ShAdamConsts {
    float pc1, rs_pc2;    // previous-step corrections: pc1 (0: no first moment), 1/sqrt(pc2)
    float b1, ob1, b2, ob2;
    float ic1, rs_c2;     // 1/c1, 1/sqrt(c2)
    float eps, lr, rest_lr, reg;
    bool norm_ok;         // c1 > 0 and c2 > 0
};

__device__ __forceinline__ ShAdamConsts sh_adam_consts(const ShAdamArgs& a) {
    ShAdamConsts k;
    const float pc1 = codec_prev_correction(a.correction1, a.beta1);
    const float pc2 = codec_prev_correction(a.correction2, a.beta2);
    k.pc1 = pc1;
    k.rs_pc2 = pc2 > 0.f ? 1.f / sqrtf(pc2) : 0.f;
    k.b1 = a.beta1;
    k.ob1 = 1.f - a.beta1;
    k.b2 = a.beta2;
    k.ob2 = 1.f - a.beta2;
    k.norm_ok = a.correction1 > 0.f && a.correction2 > 0.f;
    k.ic1 = k.norm_ok ? 1.f / a.correction1 : 0.f;
    k.rs_c2 = k.norm_ok ? 1.f / sqrtf(a.correction2) : 0.f;
    k.eps = a.epsilon;
    k.lr = a.lr;
    k.rest_lr = a.rest_lr;
    k.reg = a.regularization;
    return k;
}

// One active coefficient: code (as float) -> previous moments -> Adam ->
// new parameter, new fp16 normalised first moment, returned log-second value.
__device__ __forceinline__ float sh_adam_coef(bool rest, float& param, float grad, float& first,
                                              float code, float lo, float range,
                                              const ShAdamConsts& k) {
    const float log_s = lo + range * (code * (1.f / 255.f));
    const float s = kCodecEps * (__expf(log_s) - 1.f);
    const float g2 = s * s;
    const float g1 = k.pc1 > 0.f ? first * (fabsf(s) * k.rs_pc2 + k.eps) * k.pc1 : 0.f;
    const float prev = param;
    if (rest && k.reg > 0.f && isfinite(prev))
        grad += k.reg * prev;
    if (!isfinite(prev) || !isfinite(grad)) {
        first = 0.f;
        param = isfinite(prev) ? prev : 0.f;
        return 0.f;
    }
    const float m = k.b1 * g1 + k.ob1 * grad;
    const float v = k.b2 * g2 + k.ob2 * grad * grad;
    if (!isfinite(m) || !isfinite(v)) {
        first = 0.f;
        return 0.f;
    }
    const float sv = sqrtf(fmaxf(v, 0.f));
    const float nrm = k.norm_ok ? __fdividef(m * k.ic1, sv * k.rs_c2 + k.eps) : 0.f;
    const float cand = prev - (rest ? k.rest_lr : k.lr) * nrm;
    param = isfinite(cand) ? cand : prev;
    first = nrm;
    const float ls = __logf(1.f + sv * (1.f / kCodecEps));
    return isfinite(ls) ? ls : 0.f;
}

// sh_adam_coef without its finiteness tests, for the common case: the new
// parameter, first moment and log-second value go to pn, fn and the return
// value, and chk accumulates m, v, the new parameter and the log value. Any
// non-finite input or intermediate the tests would have caught makes chk
// non-finite (inf and NaN propagate through the sums; a finite overflow only
// sends the group to the checked path), and the caller then redoes the group
// with sh_adam_coef; with finite values both give the same results.
__device__ __forceinline__ float sh_adam_coef_fast(bool rest, float prev, float grad, float first,
                                                   float code, float lo, float range,
                                                   const ShAdamConsts& k, float& pn, float& fn,
                                                   float& chk) {
    const float log_s = lo + range * (code * (1.f / 255.f));
    const float s = kCodecEps * (__expf(log_s) - 1.f);
    const float g2 = s * s;
    const float g1 = k.pc1 > 0.f ? first * (fabsf(s) * k.rs_pc2 + k.eps) * k.pc1 : 0.f;
    if (rest && k.reg > 0.f)
        grad += k.reg * prev;
    const float m = k.b1 * g1 + k.ob1 * grad;
    const float v = k.b2 * g2 + k.ob2 * grad * grad;
    const float sv = sqrtf(fmaxf(v, 0.f));
    const float nrm = k.norm_ok ? __fdividef(m * k.ic1, sv * k.rs_c2 + k.eps) : 0.f;
    pn = prev - (rest ? k.rest_lr : k.lr) * nrm;
    fn = nrm;
    const float ls = __logf(1.f + sv * (1.f / kCodecEps));
    chk += (m + v) + (pn + ls);
    return ls;
}

// u8 code (0..255) as a float, exactly, without a conversion instruction.
__device__ __forceinline__ float code_to_float(unsigned code) {
    return __uint_as_float(0x4b000000u | code) - 8388608.f;
}

// roundf(255 * (value - lo) * inv_range) clamped to [0, 255], as an integer:
// adding 2^23 rounds a value in [0, 256) to the nearest integer (ties to
// even) and leaves it in the low mantissa bits; a tie that went down is then
// moved up, which is roundf's ties-away-from-zero for non-negative values.
// Clamping before rounding gives the same integer (the bounds are integers).
__device__ __forceinline__ unsigned codec_encode_int(float value, float lo, float inv_range) {
    const float y = fminf(fmaxf(255.f * (value - lo) * inv_range, 0.f), 255.f);
    const float t = __fadd_rn(y, 8388608.f);
    unsigned q = __float_as_uint(t) & 0xffu;
    if (__fsub_rn(y, __fsub_rn(t, 8388608.f)) == 0.5f)
        ++q;
    return q;
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Calls f(e, r, c) for e = threadIdx.x, + kGBlock, ... < total with
// r = e / stride and c = e % stride, stepping r and c incrementally: one
// integer division per thread instead of one per element (the staging and
// write-back loops run 84 + 48 elements per Gaussian).
template <typename F>
__device__ __forceinline__ void for_row_elements(int total, int stride, F&& f) {
    int e = threadIdx.x;
    int r = e / stride, c = e - r * stride;
    const int dr = kGBlock / stride, dc = kGBlock - dr * stride;
    for (; e < total; e += kGBlock) {
        f(e, r, c);
        r += dr;
        c += dc;
        if (c >= stride) {
            c -= stride;
            ++r;
        }
    }
}

// Staging of a full CTA of degree-3 rows (128 rows of 48 coefficients) and,
// with the fused SH Adam, of their fp16 first moments and u8 codes. Thread t
// copies elements e = t + 128k of the CTA's contiguous block; an element's
// padded shared-memory word is e + e / W (W words per row, rows padded by one
// word), and since 3 * 128 is a multiple of W, k -> k + 3 moves both
// addresses by constants. So every copy is one instruction at a fixed offset
// from three per-thread bases, instead of the general loop's index arithmetic
// per element.
__device__ __forceinline__ void stage_full48(float* s_coef, __half* s_first, uint8_t* s_code,
                                             const float* src, const uint32_t* fsrc,
                                             const uint32_t* csrc, bool fused) {
    const int t = threadIdx.x;
#pragma unroll
    for (int k0 = 0; k0 < 3; ++k0) {
        const int e = t + kGBlock * k0;
        float* sd = s_coef + e + e / 48;
        const float* gs = src + e;
#pragma unroll
        for (int g = 0; g < 16; ++g) // W = 48: + 384 elements, + 392 words
            cp_async4(sd + 392 * g, gs + 384 * g);
    }
    if (!fused)
        return;
    uint32_t* sf = reinterpret_cast<uint32_t*>(s_first);
    uint32_t* sc = reinterpret_cast<uint32_t*>(s_code);
#pragma unroll
    for (int k0 = 0; k0 < 3; ++k0) {
        const int e = t + kGBlock * k0;
#pragma unroll
        for (int g = 0; g < 8; ++g) // fp16 pairs, W = 24: + 384 words, + 400 padded
            cp_async4(sf + e + e / 24 + 400 * g, fsrc + e + 384 * g);
#pragma unroll
        for (int g = 0; g < 4; ++g) // code quads, W = 12: + 384 words, + 416 padded
            cp_async4(sc + e + e / 12 + 416 * g, csrc + e + 384 * g);
    }
}

// --------------------------------------------------------------- kernel --
// Fused SH Adam, phase 2 for rows other than 48 active columns: one half-warp
// per row, lanes over the columns (lane l owns columns l, l + 16, l + 32
// below the row stride), reading the row's optimiser state that phase 1
// staged in shared memory and writing the new state to HBM as coalesced row
// segments. The coefficient gradient is rebuilt
// from the row's SH basis values and clamped colour gradient (wdl, written by
// phase 1): w_k * dl.channel, the product the SH adjoint forms. DC and rest
// columns share one instruction path (their learning rate, regulariser and
// code bounds are selected per column), so the DC lanes do not diverge. The
// per-row code bounds are a min / max over the row's log-second values,
// reduced across the half-warp, so the result does not depend on the thread
// layout.
constexpr int kWdlStride = 19; // per row: SH basis values [16], clamped colour gradient [3]
constexpr int kHalfStride = 50; // padded fp16 row = 25 words
constexpr int kCodeStride = 52; // padded u8 row = 13 words

// One row (ok: the row exists; every lane of the warp calls this, the
// shuffles take the whole warp). kAll48: 48 columns, all active (degree-3
// rows) on the fast coefficient path; otherwise the general column step.
template <bool kAll48>
__device__ __forceinline__ void sh_adam_row_half(bool ok, size_t i, int stride, int active, int l,
                                                 const float* coef, const float* wdl,
                                                 const __half* first_row, const uint8_t* code_row,
                                                 float4 bnd, const ShAdamArgs& a,
                                                 const ShAdamConsts& k) {
    float b0 = bnd.x, b1 = bnd.y, b2 = bnd.z, b3 = bnd.w;
    if (!isfinite(b0) || !isfinite(b1)) b0 = b1 = 0.f;
    if (!isfinite(b2) || !isfinite(b3)) b2 = b3 = 0.f;
    const float drange = b1 - b0, rrange = b3 - b2;
    float dmin = 1e30f, dmax = -1e30f, rmin = 1e30f, rmax = -1e30f;
    float ls[3];
    float* param_out = a.parameter + i * size_t(stride);
    __half* first_out = reinterpret_cast<__half*>(a.first) + i * size_t(stride);
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
        const int c = l + 16 * kk;
        ls[kk] = 0.f;
        if (!ok || c >= stride)
            continue;
        const int b = c / 3, ch = c - 3 * b;
        const float grad = wdl[b] * wdl[16 + ch];
        float param = coef[c];
        float first = __half2float(first_row[c]);
        const bool rest = c >= 3;
        float lv;
        if constexpr (kAll48) {
            const float cf = code_to_float(code_row[c]);
            const float lo = rest ? b2 : b0, range = rest ? rrange : drange;
            float pn, fn, chk = 0.f;
            lv = sh_adam_coef_fast(rest, param, grad, first, cf, lo, range, k, pn, fn, chk);
            if (isfinite(chk)) {
                param = pn;
                first = fn;
            } else {
                lv = sh_adam_coef(rest, param, grad, first, cf, lo, range, k);
            }
        } else {
            lv = sh_adam_column(c, active, param, grad, first, code_row[c], rest ? b2 : b0,
                                rest ? b3 : b1, a);
        }
        param_out[c] = param;
        first_out[c] = __float2half_rn(first);
        ls[kk] = lv;
        if (rest) {
            rmin = fminf(rmin, lv);
            rmax = fmaxf(rmax, lv);
        } else {
            dmin = fminf(dmin, lv);
            dmax = fmaxf(dmax, lv);
        }
    }
#pragma unroll
    for (int off = 8; off > 0; off >>= 1) {
        dmin = fminf(dmin, __shfl_xor_sync(0xffffffffu, dmin, off));
        dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
        rmin = fminf(rmin, __shfl_xor_sync(0xffffffffu, rmin, off));
        rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, off));
    }
    if (!ok)
        return;
    if (stride <= 3) rmin = rmax = 0.f;
    if (l == 0)
        reinterpret_cast<float4*>(a.bounds)[i] = make_float4(dmin, dmax, rmin, rmax);
    const float inv_d = 1.f / fmaxf(dmax - dmin, kCodecEps);
    const float inv_r = 1.f / fmaxf(rmax - rmin, kCodecEps);
    uint8_t* code_out = a.packed + i * size_t(stride);
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
        const int c = l + 16 * kk;
        if (c >= stride)
            continue;
        const bool rest = c >= 3;
        if constexpr (kAll48)
            code_out[c] = uint8_t(codec_encode_int(ls[kk], rest ? rmin : dmin, rest ? inv_r : inv_d));
        else
            code_out[c] = codec_encode(ls[kk], rest ? rmin : dmin, rest ? inv_r : inv_d);
    }
}

// Fused SH Adam, phase 2 for degree-3 rows (48 columns, all active), one
// thread per row: the instruction path with the fewest instructions per
// coefficient (launch constants folded once, groups of four independent
// coefficient chains, no cross-lane reductions). The coefficient gradients
// come from the row's basis values and clamped colour gradient (4 shared
// loads per 12 columns); the new parameters go straight to HBM as 16-byte row
// segments, and the log-second values take the parameters' shared-memory
// slots for the encode pass; the new fp16 first moments and codes are written
// in place and leave with one coalesced write-back per CTA.
template <bool kFirstBlock>
__device__ __forceinline__ void sh_adam_block48(int q, float* prow, __half* frow,
                                                const uint8_t* crow, const float* wdl,
                                                float3 dl, float* pout, float dlo, float drange,
                                                float rlo, float rrange, float& dmin,
                                                float& dmax, float& rmin, float& rmax,
                                                const ShAdamConsts& k) {
    const float w[4] = {wdl[4 * q], wdl[4 * q + 1], wdl[4 * q + 2], wdl[4 * q + 3]};
    const float d[3] = {dl.x, dl.y, dl.z};
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        const int c0 = 12 * q + 4 * g;
        float pv[4], gv[4], fv[4], cf[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            pv[j] = prow[c0 + j];
            gv[j] = w[(4 * g + j) / 3] * d[(4 * g + j) % 3];
        }
        const float2 f01 = __half22float2(*reinterpret_cast<const __half2*>(frow + c0));
        const float2 f23 = __half22float2(*reinterpret_cast<const __half2*>(frow + c0 + 2));
        fv[0] = f01.x;
        fv[1] = f01.y;
        fv[2] = f23.x;
        fv[3] = f23.y;
        const unsigned cw = *reinterpret_cast<const unsigned*>(crow + c0);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            cf[j] = code_to_float((cw >> (8 * j)) & 0xffu);
        float pn[4], fn[4], ln[4], chk = 0.f;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool rest = !(kFirstBlock && g == 0 && j < 3);
            ln[j] = sh_adam_coef_fast(rest, pv[j], gv[j], fv[j], cf[j], rest ? rlo : dlo,
                                      rest ? rrange : drange, k, pn[j], fn[j], chk);
        }
        if (isfinite(chk)) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                pv[j] = pn[j];
                fv[j] = fn[j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool rest = !(kFirstBlock && g == 0 && j < 3);
                ln[j] = sh_adam_coef(rest, pv[j], gv[j], fv[j], cf[j], rest ? rlo : dlo,
                                     rest ? rrange : drange, k);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (kFirstBlock && g == 0 && j < 3) {
                dmin = fminf(dmin, ln[j]);
                dmax = fmaxf(dmax, ln[j]);
            } else {
                rmin = fminf(rmin, ln[j]);
                rmax = fmaxf(rmax, ln[j]);
            }
            prow[c0 + j] = ln[j];
        }
        *reinterpret_cast<float4*>(pout + c0) = make_float4(pv[0], pv[1], pv[2], pv[3]);
        *reinterpret_cast<__half2*>(frow + c0) = __floats2half2_rn(fv[0], fv[1]);
        *reinterpret_cast<__half2*>(frow + c0 + 2) = __floats2half2_rn(fv[2], fv[3]);
    }
}

__device__ __forceinline__ void sh_adam_row48(float* prow, __half* frow, uint8_t* crow,
                                              const float* wdl, float4 bnd, float* pout,
                                              float4* bout, const ShAdamConsts& k) {
    float b0 = bnd.x, b1 = bnd.y, b2 = bnd.z, b3 = bnd.w;
    if (!isfinite(b0) || !isfinite(b1)) b0 = b1 = 0.f;
    if (!isfinite(b2) || !isfinite(b3)) b2 = b3 = 0.f;
    const float drange = b1 - b0, rrange = b3 - b2;
    float dmin = 1e30f, dmax = -1e30f, rmin = 1e30f, rmax = -1e30f;
    const float3 dl = make_float3(wdl[16], wdl[17], wdl[18]);
    sh_adam_block48<true>(0, prow, frow, crow, wdl, dl, pout, b0, drange, b2, rrange, dmin, dmax,
                          rmin, rmax, k);
#pragma unroll 1
    for (int q = 1; q < 4; ++q)
        sh_adam_block48<false>(q, prow, frow, crow, wdl, dl, pout, b0, drange, b2, rrange, dmin,
                               dmax, rmin, rmax, k);
    *bout = make_float4(dmin, dmax, rmin, rmax);
    const float inv_d = 1.f / fmaxf(dmax - dmin, kCodecEps);
    const float inv_r = 1.f / fmaxf(rmax - rmin, kCodecEps);
#pragma unroll 2
    for (int c0 = 0; c0 < 48; c0 += 4) {
        float lv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            lv[j] = prow[c0 + j];
        unsigned w = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool dc = c0 + j < 3;
            w |= codec_encode_int(lv[j], dc ? dmin : rmin, dc ? inv_d : inv_r) << (8 * j);
        }
        *reinterpret_cast<unsigned*>(crow + c0) = w;
    }
}

template <bool kFusedStruct, bool kFusedSH, bool kGeo>
__global__ void __launch_bounds__(kGBlock, 4) gaussian_backward_kernel(
    int n, const float* __restrict__ means, const float* __restrict__ log_scales,
    const float* __restrict__ quats, const float* __restrict__ logits,
    const float* __restrict__ filter_3d, const float* __restrict__ sh, int sh_degree,
    int sh_bases, const Camera K, GaussianState st, const int* __restrict__ radii,
    GradOutArgs out, StructureAdamArgs sa, ShAdamArgs sha) {
    extern __shared__ float smem[];
    // Shared memory: SH rows [kGBlock][kShStride] floats, then with the fused
    // SH Adam the basis / colour-gradient rows [kGBlock][kWdlStride], fp16
    // first moments [kGBlock][kHalfStride], u8 codes [kGBlock][kCodeStride]
    // and code bounds [kGBlock] float4; without it the coefficient gradients
    // [kGBlock][kShStride].
    float* s_coef = smem;
    float* s_aux = smem + kGBlock * kShStride;
    __half* s_first = reinterpret_cast<__half*>(s_aux + kGBlock * kWdlStride);
    uint8_t* s_code = reinterpret_cast<uint8_t*>(s_first + kGBlock * kHalfStride);
    float4* s_bnd = reinterpret_cast<float4*>(s_code + kGBlock * kCodeStride);
    const int tid = threadIdx.x;
    const int row0 = blockIdx.x * kGBlock;
    const int rows = min(kGBlock, n - row0);
    const int stride = sh ? sh_bases * 3 : 0;
    // 1. Asynchronous, coalesced staging of this CTA's SH rows (contiguous),
    //    and with fused SH Adam of their fp16 first moments, u8 codes and code
    //    bounds.
    if (stride == 48 && rows == kGBlock) {
        stage_full48(s_coef, s_first, s_code, sh + size_t(row0) * 48,
                     kFusedSH ? reinterpret_cast<const uint32_t*>(
                                    reinterpret_cast<const __half*>(sha.first) + size_t(row0) * 48)
                              : nullptr,
                     kFusedSH ? reinterpret_cast<const uint32_t*>(sha.packed + size_t(row0) * 48)
                              : nullptr,
                     kFusedSH);
    } else if (sh) {
        const float* src = sh + size_t(row0) * stride;
        const int total = rows * stride;
        for_row_elements(total, stride, [&](int e, int r, int c) {
            cp_async4(s_coef + r * kShStride + c, src + e);
        });
        if constexpr (kFusedSH) {
            const __half* fsrc = reinterpret_cast<const __half*>(sha.first) + size_t(row0) * stride;
            const uint8_t* csrc = sha.packed + size_t(row0) * stride;
            for_row_elements(total, stride, [&](int e, int r, int c) {
                s_first[r * kHalfStride + c] = fsrc[e];
                s_code[r * kCodeStride + c] = csrc[e];
            });
        }
    }
    if constexpr (kFusedSH)
        if (sh && tid < rows)
            s_bnd[tid] = reinterpret_cast<const float4*>(sha.bounds)[row0 + tid];
    // 2. Meanwhile every per-Gaussian input of this thread is loaded up front.
    const int i = row0 + tid;
    const bool valid = tid < rows;
    const bool visible = valid && radii[i] > 0;
    float3 mean = make_float3(0.f, 0.f, 0.f);
    float4 g0 = make_float4(0.f, 0.f, 0.f, 0.f), g1 = g0, g2 = g0;
    unsigned clamp_bits = 0;
    Activated act{};
    if (valid) {
        mean = make_float3(means[3 * i], means[3 * i + 1], means[3 * i + 2]);
        act = activate(log_scales, quats, logits, filter_3d, i);
    }
    float4 gplane = make_float4(0.f, 0.f, 0.f, 0.f), gnorm = gplane;
    if (visible) {
        const float4* gslot = st.grad + size_t(i) * kGradSlots;
        g0 = gslot[0];
        g1 = gslot[1];
        g2 = gslot[2];
        clamp_bits = __float_as_uint(st.rgb[i].w);
        if constexpr (kGeo) {
            gplane = st.geo_grad[size_t(i) * kGeoGradSlots];
            gnorm = st.geo_grad[size_t(i) * kGeoGradSlots + 1];
        }
    }
    // Structure Adam state, loaded before any arithmetic so all requests are
    // in flight together: parameters p*, first moments m*, second moments v*.
    float pm[3], mm_[3], vm[3], pl[3], ml[3], vl[3], pq[4], mq[4], vq[4], po = 0.f, mo = 0.f,
        vo = 0.f;
    if constexpr (kFusedStruct) {
        if (valid) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                pm[k] = sa.means[3 * i + k];
                mm_[k] = sa.means_first[3 * i + k];
                vm[k] = sa.means_second[3 * i + k];
                pl[k] = sa.log_scales[3 * i + k];
                ml[k] = sa.scales_first[3 * i + k];
                vl[k] = sa.scales_second[3 * i + k];
            }
            const float4 q4 = reinterpret_cast<const float4*>(sa.quaternions)[i];
            const float4 mq4 = reinterpret_cast<const float4*>(sa.rotations_first)[i];
            const float4 vq4 = reinterpret_cast<const float4*>(sa.rotations_second)[i];
            pq[0] = q4.x; pq[1] = q4.y; pq[2] = q4.z; pq[3] = q4.w;
            mq[0] = mq4.x; mq[1] = mq4.y; mq[2] = mq4.z; mq[3] = mq4.w;
            vq[0] = vq4.x; vq[1] = vq4.y; vq[2] = vq4.z; vq[3] = vq4.w;
            po = sa.opacity_logits[i];
            mo = sa.opacity_first[i];
            vo = sa.opacity_second[i];
        }
    }
    // Rows of visible Gaussians are written whole by the SH adjoint below.
    float* wdl = s_aux + tid * kWdlStride;
    float* grow = s_aux + tid * kShStride;
    if (!visible) {
        if constexpr (kFusedSH)
            for (int c = 0; c < kWdlStride; ++c)
                wdl[c] = 0.f;
        else
            for (int c = 0; c < stride; ++c)
                grow[c] = 0.f;
    }
    if (sh)
        cp_async_wait_all();
    __syncthreads();

    // 3. Adjoints.
    ProjGrad pg;
    pg.d_mean = make_float3(0.f, 0.f, 0.f);
    pg.d_scale = make_float3(0.f, 0.f, 0.f);
    pg.d_rot = make_float4(0.f, 0.f, 0.f, 0.f);
    pg.d_opac = 0.f;
    if (visible) {
        float4* gslot = st.grad + size_t(i) * kGradSlots;
        gslot[0] = make_float4(0.f, 0.f, 0.f, 0.f);
        gslot[1] = make_float4(0.f, 0.f, 0.f, 0.f);
        gslot[2] = make_float4(0.f, 0.f, 0.f, 0.f);
        if constexpr (kGeo) {
            st.geo_grad[size_t(i) * kGeoGradSlots] = make_float4(0.f, 0.f, 0.f, 0.f);
            st.geo_grad[size_t(i) * kGeoGradSlots + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
            pg = projection_backward<true>(mean, K, act.scale, act.rot, g0,
                                           make_float2(g1.x, g1.y), gplane,
                                           make_float3(gnorm.x, gnorm.y, gnorm.z));
        } else {
            pg = projection_backward(mean, K, act.scale, act.rot, g0, make_float2(g1.x, g1.y));
        }
        const float3 dcol = make_float3(g2.x, g2.y, g2.z);
        if (sh) {
            const float3* crow = reinterpret_cast<const float3*>(s_coef + tid * kShStride);
            const float3 campos = make_float3(K.center[0], K.center[1], K.center[2]);
            float3 dm;
            if constexpr (kFusedSH)
                dm = sh_color_backward<true>(crow, sh_degree, sh_bases, mean, campos, clamp_bits,
                                             dcol, nullptr, wdl);
            else
                dm = sh_color_backward(crow, sh_degree, sh_bases, mean, campos, clamp_bits, dcol,
                                       reinterpret_cast<float3*>(grow));
            pg.d_mean.x += dm.x;
            pg.d_mean.y += dm.y;
            pg.d_mean.z += dm.z;
        } else if (out.colors) {
            out.colors[3 * i + 0] += dcol.x;
            out.colors[3 * i + 1] += dcol.y;
            out.colors[3 * i + 2] += dcol.z;
        }
        if (out.refine_weight) out.refine_weight[i] += g1.z;
        if (out.densify_weight) out.densify_weight[i] += g1.w;
        if (out.densify_weight_den) out.densify_weight_den[i] += g2.w;
    }

    // 4. Structure: fused Adam or gradient outputs.
    if (valid) {
        if constexpr (kFusedStruct) {
            // Chain to raw parameters (update_structure_adam_row), priors, Adam.
            RawGrad rg;
            {
                const float f2 = sa.filter_3d ? sa.filter_3d[i] * sa.filter_3d[i] : 0.f;
                const float ds[3] = {pg.d_scale.x, pg.d_scale.y, pg.d_scale.z};
    #pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float raw = (&act.raw_scale.x)[k];
                    const float sc = (&act.scale.x)[k];
                    rg.log_s[k] = ds[k] * raw * raw / sc + pg.d_opac * act.opacity * f2 / (sc * sc);
                }
                const float inv = rsqrtf(fmaxf(pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2] +
                                                   pq[3] * pq[3], 1e-20f));
                const float q[4] = {pq[0] * inv, pq[1] * inv, pq[2] * inv, pq[3] * inv};
                const float dr[4] = {pg.d_rot.x, pg.d_rot.y, pg.d_rot.z, pg.d_rot.w};
                const float qdot = q[0] * dr[0] + q[1] * dr[1] + q[2] * dr[2] + q[3] * dr[3];
    #pragma unroll
                for (int k = 0; k < 4; ++k)
                    rg.quat[k] = inv * (dr[k] - q[k] * qdot);
            }
            const float sig = 1.f / (1.f + expf(-po));
            float g_log[3] = {rg.log_s[0], rg.log_s[1], rg.log_s[2]};
            float g_quat[4] = {rg.quat[0], rg.quat[1], rg.quat[2], rg.quat[3]};
            float g_logit = pg.d_opac * act.opacity * (1.f - sig);
            if (isfinite(po) && sa.opacity_reg > 0.f)
                g_logit += sa.opacity_reg * sig * (1.f - sig);
            if (sa.scale_reg > 0.f)
    #pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (isfinite(pl[k]) && pl[k] > -40.f) g_log[k] += sa.scale_reg * expf(pl[k]);
            if (sa.shape_quat_norm_reg > 0.f || sa.shape_axis_ratio_reg > 0.f ||
                sa.shape_erank_reg > 0.f || sa.shape_erank_s3_reg > 0.f) {
                const PriorGrad pr =
                    shape_priors_delta(pl[0], pl[1], pl[2], pq[0], pq[1], pq[2], pq[3], sa);
    #pragma unroll
                for (int k = 0; k < 3; ++k) g_log[k] += pr.log_s[k];
    #pragma unroll
                for (int k = 0; k < 4; ++k) g_quat[k] += pr.quat[k];
            }
            if (sa.opacity_gradient) sa.opacity_gradient[i] = g_logit;
            const float inf = 1.e30f;
            const float gm[3] = {pg.d_mean.x, pg.d_mean.y, pg.d_mean.z};
            float nm[3], nl[3], nq[4];
    #pragma unroll
            for (int c = 0; c < 3; ++c) {
                nm[c] = adam_reg(pm[c], gm[c], mm_[c], vm[c], sa.means_lr, sa.beta1, sa.beta2,
                                 sa.correction1, sa.correction2, sa.epsilon, -inf, inf);
                nl[c] = adam_reg(pl[c], g_log[c], ml[c], vl[c], sa.scales_lr, sa.beta1, sa.beta2,
                                 sa.correction1, sa.correction2, sa.epsilon, sa.minimum_log_scale,
                                 sa.maximum_log_scale);
            }
    #pragma unroll
            for (int c = 0; c < 4; ++c)
                nq[c] = adam_reg(pq[c], g_quat[c], mq[c], vq[c], sa.quaternions_lr, sa.beta1,
                                 sa.beta2, sa.correction1, sa.correction2, sa.epsilon, -inf, inf);
            const float no = adam_reg(po, g_logit, mo, vo, sa.opacities_lr, sa.beta1, sa.beta2,
                                      sa.correction1, sa.correction2, sa.epsilon, -12.f, 12.f);
    #pragma unroll
            for (int c = 0; c < 3; ++c) {
                sa.means[3 * i + c] = nm[c];
                sa.means_first[3 * i + c] = mm_[c];
                sa.means_second[3 * i + c] = vm[c];
                sa.log_scales[3 * i + c] = nl[c];
                sa.scales_first[3 * i + c] = ml[c];
                sa.scales_second[3 * i + c] = vl[c];
            }
            reinterpret_cast<float4*>(sa.quaternions)[i] = make_float4(nq[0], nq[1], nq[2], nq[3]);
            reinterpret_cast<float4*>(sa.rotations_first)[i] = make_float4(mq[0], mq[1], mq[2], mq[3]);
            reinterpret_cast<float4*>(sa.rotations_second)[i] = make_float4(vq[0], vq[1], vq[2], vq[3]);
            sa.opacity_logits[i] = no;
            sa.opacity_first[i] = mo;
            sa.opacity_second[i] = vo;
        } else if (visible) {
            if (out.means) {
                out.means[3 * i + 0] += pg.d_mean.x;
                out.means[3 * i + 1] += pg.d_mean.y;
                out.means[3 * i + 2] += pg.d_mean.z;
            }
            if (out.activated) {
                if (out.scales) {
                    out.scales[3 * i + 0] += pg.d_scale.x;
                    out.scales[3 * i + 1] += pg.d_scale.y;
                    out.scales[3 * i + 2] += pg.d_scale.z;
                }
                if (out.rotations) {
                    out.rotations[4 * i + 0] += pg.d_rot.x;
                    out.rotations[4 * i + 1] += pg.d_rot.y;
                    out.rotations[4 * i + 2] += pg.d_rot.z;
                    out.rotations[4 * i + 3] += pg.d_rot.w;
                }
                if (out.opacities) out.opacities[i] += pg.d_opac;
            } else {
                const RawGrad rg = chain_to_raw(pg, act, quats, logits, filter_3d, i);
                if (out.scales)
                    for (int k = 0; k < 3; ++k) out.scales[3 * i + k] += rg.log_s[k];
                if (out.rotations)
                    for (int k = 0; k < 4; ++k) out.rotations[4 * i + k] += rg.quat[k];
                if (out.opacities) out.opacities[i] += rg.logit;
            }
        }
    }

    // 5. SH: the fused quantized Adam (phase 2, one half-warp per row) or the
    //    coalesced accumulation of the coefficient gradients.
    if constexpr (kFusedSH) {
        if (!sh)
            return;
        __syncthreads();
        const int active = (sh_degree + 1) * (sh_degree + 1) * 3;
        const ShAdamConsts kc = sh_adam_consts(sha);
        const bool aligned = ((reinterpret_cast<uintptr_t>(sha.parameter) & 15) |
                              (reinterpret_cast<uintptr_t>(sha.first) & 7) |
                              (reinterpret_cast<uintptr_t>(sha.packed) & 3)) == 0;
        if (stride == 48 && active == 48 && aligned) {
            // one thread per row, then the coalesced write-back of the new
            // fp16 first moments and codes (four columns per thread and step)
            if (valid)
                sh_adam_row48(s_coef + tid * kShStride, s_first + tid * kHalfStride,
                              s_code + tid * kCodeStride, s_aux + tid * kWdlStride, s_bnd[tid],
                              sha.parameter + size_t(i) * 48,
                              reinterpret_cast<float4*>(sha.bounds) + i, kc);
            __syncthreads();
            uint2* fdst = reinterpret_cast<uint2*>(reinterpret_cast<__half*>(sha.first) +
                                                   size_t(row0) * 48);
            unsigned* cdst = reinterpret_cast<unsigned*>(sha.packed + size_t(row0) * 48);
            for_row_elements(rows * 12, 12, [&](int e, int r, int cq) {
                const unsigned* f =
                    reinterpret_cast<const unsigned*>(s_first + r * kHalfStride + 4 * cq);
                fdst[e] = make_uint2(f[0], f[1]);
                cdst[e] = *reinterpret_cast<const unsigned*>(s_code + r * kCodeStride + 4 * cq);
            });
            return;
        }
        // other strides and degrees: one half-warp per row
        const int l = tid & 15, hw = tid >> 4;
        constexpr int kHalves = kGBlock / 16;       // half-warps per CTA
        constexpr int kPerHalf = kGBlock / kHalves; // rows per half-warp
        for (int k = 0; k < kPerHalf; ++k) {
            const int r = hw + kHalves * k;
            const bool ok = r < rows;
            const float* coef = s_coef + r * kShStride;
            const float* w = s_aux + r * kWdlStride;
            const __half* fr = s_first + r * kHalfStride;
            const uint8_t* cr = s_code + r * kCodeStride;
            const float4 bnd = ok ? s_bnd[r] : make_float4(0.f, 0.f, 0.f, 0.f);
            if (stride == 48 && active == 48)
                sh_adam_row_half<true>(ok, size_t(row0 + r), stride, active, l, coef, w, fr, cr,
                                       bnd, sha, kc);
            else
                sh_adam_row_half<false>(ok, size_t(row0 + r), stride, active, l, coef, w, fr, cr,
                                        bnd, sha, kc);
        }
    } else {
        __syncthreads();
        if (sh && out.sh) {
            float* dst = out.sh + size_t(row0) * stride;
            for_row_elements(rows * stride, stride, [&](int e, int r, int c) {
                dst[e] += s_aux[r * kShStride + c];
            });
        }
    }
}

size_t gaussian_backward_smem(bool fused_sh) {
    if (!fused_sh)
        return size_t(kGBlock) * 2 * kShStride * sizeof(float);
    return size_t(kGBlock) * ((kShStride + kWdlStride) * sizeof(float) +
                              kHalfStride * sizeof(__half) + kCodeStride + sizeof(float4));
}

void launch_gaussian_backward(cudaStream_t s, int n, const float* means, const float* log_scales,
                              const float* quats, const float* logits, const float* filter_3d,
                              const float* sh, int sh_degree, int sh_bases, const Camera& K,
                              const GaussianState& st, const int* radii, const GradOutArgs& out,
                              const StructureAdamArgs* sa, const ShAdamArgs* sha, bool geometry) {
    const int blocks = (n + kGBlock - 1) / kGBlock;
    StructureAdamArgs sa0{};
    ShAdamArgs sha0{};
    const bool fs = sa != nullptr, fh = sha != nullptr && sh != nullptr;
    const size_t smem = gaussian_backward_smem(fh);
#define GSB_LAUNCH(FS, FH, GEO)                                                                  \
    do {                                                                                         \
        auto kfn = gaussian_backward_kernel<FS, FH, GEO>;                                        \
        static bool attr_set = false;                                                            \
        if (!attr_set) {                                                                         \
            cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));   \
            attr_set = true;                                                                     \
        }                                                                                        \
        kfn<<<blocks, kGBlock, smem, s>>>(n, means, log_scales, quats, logits, filter_3d, sh,    \
                                          sh_degree, sh_bases, K, st, radii, out,                \
                                          sa ? *sa : sa0, sha ? *sha : sha0);                    \
    } while (0)
    if (geometry) {
        if (fs && fh) GSB_LAUNCH(true, true, true);
        else if (fs) GSB_LAUNCH(true, false, true);
        else if (fh) GSB_LAUNCH(false, true, true);
        else GSB_LAUNCH(false, false, true);
    } else {
        if (fs && fh) GSB_LAUNCH(true, true, false);
        else if (fs) GSB_LAUNCH(true, false, false);
        else if (fh) GSB_LAUNCH(false, true, false);
        else GSB_LAUNCH(false, false, false);
    }
#undef GSB_LAUNCH
}

// ------------------------------------------------------ standalone kernels --
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, size_t n, float lr,
                            float b1, float b2, float c1, float c2, float eps, float lo, float hi) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
         i += size_t(gridDim.x) * blockDim.x)
        adam_one(p, i, g[i], m, v, lr, b1, b2, c1, c2, eps, lo, hi);
}

void launch_adam(cudaStream_t s, float* p, const float* g, float* m, float* v, size_t n, float lr,
                 float b1, float b2, float c1, float c2, float eps, float lo, float hi) {
    if (n == 0) return;
    const int blocks = int(std::min<size_t>((n + kBlock - 1) / kBlock, size_t(148) * 16));
    adam_kernel<<<blocks, kBlock, 0, s>>>(p, g, m, v, n, lr, b1, b2, c1, c2, eps, lo, hi);
}

// L1 over [3,P] images: grad = w/(3P) sign(d), loss += w/(3P) sum |d|.
__device__ __forceinline__ float l1_grad(float d, float scale) {
    return d > 0.f ? scale : (d < 0.f ? -scale : 0.f);
}

// Four elements per thread and step with 16-byte accesses (the images are
// streamed once: HBM-bound), then a scalar tail; one atomic per warp.
__global__ void __launch_bounds__(kBlock) l1_kernel(const float* __restrict__ img,
                                                    const float* __restrict__ tgt, size_t n,
                                                    float scale, float* __restrict__ grad,
                                                    float* __restrict__ loss, bool vec) {
    float acc = 0.f;
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    const size_t first = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    size_t done = 0;
    if (vec) {
        const size_t n4 = n / 4;
        const float4* a4 = reinterpret_cast<const float4*>(img);
        const float4* b4 = reinterpret_cast<const float4*>(tgt);
        float4* g4 = reinterpret_cast<float4*>(grad);
#pragma unroll 2
        for (size_t i = first; i < n4; i += stride) {
            const float4 a = __ldcs(a4 + i), b = __ldcs(b4 + i);
            const float4 d = make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
            __stcs(g4 + i, make_float4(l1_grad(d.x, scale), l1_grad(d.y, scale),
                                       l1_grad(d.z, scale), l1_grad(d.w, scale)));
            acc += (fabsf(d.x) + fabsf(d.y)) + (fabsf(d.z) + fabsf(d.w));
        }
        done = n4 * 4;
    }
    for (size_t i = done + first; i < n; i += stride) {
        const float d = img[i] - tgt[i];
        grad[i] = l1_grad(d, scale);
        acc += fabsf(d);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    // One global atomic per block (per-warp atomics on one address serialise).
    __shared__ float s_warp[kBlock / 32];
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (loss && threadIdx.x == 0) {
        float sum = 0.f;
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w) sum += s_warp[w];
        atomicAdd(loss, sum * scale);
    }
}

void launch_l1(cudaStream_t s, const float* img, const float* tgt, size_t n, float scale,
               float* grad, float* loss) {
    if (n == 0) return;
    const bool vec = ((reinterpret_cast<uintptr_t>(img) | reinterpret_cast<uintptr_t>(tgt) |
                       reinterpret_cast<uintptr_t>(grad)) & 15) == 0;
    const size_t work = vec ? (n + 3) / 4 : n;
    const int blocks = int(std::min<size_t>((work + kBlock - 1) / kBlock, size_t(148) * 8));
    l1_kernel<<<blocks, kBlock, 0, s>>>(img, tgt, n, scale, grad, loss, vec);
}

} // namespace gsb
