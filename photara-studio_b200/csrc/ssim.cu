// Fused L1 + SSIM photometric loss and its gradient in one kernel (the loss
// photara trains with: photara/src/splat/fused_ssim.cu, called from
// photometric_loss.cpp:8-20), and the SSIM metric.
//
// Loss (SSIM of Wang et al. 2004: 11 x 11 separable Gaussian window of sigma
// 1.5, zero padding outside the image, C1 = 0.01^2, C2 = 0.03^2):
//   L = w / (3 (W - 10) (H - 10)) * sum over channels and over the pixels whose
//       window lies inside the image of [lambda (1 - SSIM) + (1 - lambda)|a - b|]
// with a, b = prediction, target (each times the mask when one is given);
// dL/d prediction (times the mask) is added to grad.
//
// B200 organisation: one kernel, no intermediate maps in HBM. A CTA (512
// threads, two per SM in 101 KB of shared memory each) owns a 32 x 32 output
// tile; per channel it stages the two images with a 10-pixel halo in shared
// memory, filters the five moments separably (rows, then columns) over the
// tile plus a 5-pixel halo, turns them into SSIM and its three partial
// derivatives (d/d mean, d/d variance, d/d covariance, the mean-subtraction
// terms folded into d/d mean) there, and filters those back (rows, then
// columns) onto the tile's pixels: the gradient at a pixel needs the
// derivative maps of its whole window, which the halo holds. Recomputing the
// moments on the halo (1.72x the tile) replaces a 75 MB write and read of
// the derivative maps at 1080p. Loss partials are reduced per CTA and then in
// one deterministic pass (double), as the reference does.
// Float32 throughout, in the reference's expression order and with its
// fast-math division (both are built with -use_fast_math): near-constant
// windows make the derivative terms cancel, and the float32 residue is part
// of the gradient the reference's tests pin (fused_ssim.cu:262-267).
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace gsb {

namespace {

__constant__ float c_window[11] = {
    0.001028380123898387f, 0.0075987582094967365f, 0.036000773310661316f,
    0.10936068743467331f,  0.21300552785396576f,   0.26601171493530273f,
    0.21300552785396576f,  0.10936068743467331f,   0.036000773310661316f,
    0.0075987582094967365f, 0.001028380123898387f};

constexpr int kHalo = 5;
constexpr int kTaps = 2 * kHalo + 1;
constexpr int kT = 32;                   // output tile: kT x kT pixels
constexpr int kI = kT + 4 * kHalo;       // staged images: 52 x 52 (10-pixel halo)
constexpr int kD = kT + 2 * kHalo;       // moment / derivative maps: 42 x 42 (5-pixel halo)
constexpr int kThreads = 512;
constexpr int kLoadIters = (kI * kI + kThreads - 1) / kThreads;
constexpr float kC1 = 0.01f * 0.01f;
constexpr float kC2 = 0.03f * 0.03f;

// Shared-memory planes (floats). Row strides keep the 8-byte loads aligned
// and the column walks of consecutive threads on distinct banks.
constexpr int kImgStride = 2 * (kI + 1);   // s_img [kI][kI + 1] float2 (prediction, target)
constexpr int kRowStride = kD + 2;         // s_row [5][kI][kD + 2]: moments filtered along rows
constexpr int kMomStride = kD;             // s_mom [5][kD][kD]: filtered moments
constexpr int kBwdStride = kT;             // s_bwd [3][kD][kT]: derivative maps filtered along rows
constexpr int kImgFloats = kI * kImgStride;
constexpr int kRowFloats = 5 * kI * kRowStride;
constexpr int kMomFloats = 5 * kD * kMomStride;
// Phases 4-6 reuse s_row for s_dm [3][kD / 2][kD] float2 (two rows
// interleaved), the tile's gradient and mask rows and its two images; s_bwd
// reuses s_mom.
constexpr int kDmFloats = 3 * kD * kD;
static_assert(kDmFloats + 4 * kT * kT <= kRowFloats && 3 * kD * kBwdStride <= kMomFloats);
static_assert(kT * kT % kThreads == 0);
static_assert(kD % 2 == 0 && kT % 2 == 0);

// Work split of each phase over the CTA (tasks <= kThreads each).
constexpr int kRowSeg = 6;                        // row pass: 6 moment columns per task
constexpr int kRowTasks = kI * (kD / kRowSeg);    // 52 rows x 7 segments = 364
constexpr int kColSeg = 14;                       // column pass: 14 rows x 2 columns
constexpr int kColTasks = 5 * (kD / 2) * (kD / kColSeg); // 5 moments x 21 x 3 = 315
constexpr int kBRowSeg = 8;                       // derivative rows: 2 rows x 8 columns
constexpr int kBRowTasks = 3 * (kD / 2) * (kT / kBRowSeg); // 3 maps x 21 x 4 = 252
constexpr int kBColTasks = (kT / 2) * (kT / 2);   // gradient: 2 x 2 pixels per task = 256
static_assert(kD % kRowSeg == 0 && kD % kColSeg == 0 && kT % kBRowSeg == 0);
static_assert(kRowTasks <= kThreads && kColTasks <= kThreads && kBRowTasks <= kThreads &&
              kBColTasks <= kThreads);

struct SsimArgs {
    const float* pred;
    const float* target;
    const float* mask; // [H,W] or NULL
    int width, height;
    float lambda;      // ssim weight
    float norm;        // photometric weight / (3 (W-10) (H-10))
    float* grad;       // [3,H,W], added to (kMetric: unused)
    float* partial;    // per CTA: loss (or SSIM sum, then count)
};

// The SSIM value and its three derivative maps from the five filtered moments.
struct SsimTerms {
    float ssim, d_mu1, d_s11, d_s12;
};

__device__ __forceinline__ SsimTerms ssim_terms(float m0, float m1, float m2, float m3,
                                                float m4) {
    const float mu1 = m0, mu2 = m2;
    const float mu1_sq = mu1 * mu1, mu2_sq = mu2 * mu2;
    const float s11 = m1 - mu1_sq, s22 = m3 - mu2_sq, s12 = m4 - mu1 * mu2;
    const float a = mu1_sq + mu2_sq + kC1;
    const float b = s11 + s22 + kC2;
    const float c = 2.f * mu1 * mu2 + kC1;
    const float d = 2.f * s12 + kC2;
    SsimTerms t;
    t.ssim = c * d / (a * b);
    t.d_mu1 = (2.f * mu2 * d) / (a * b) - (2.f * mu2 * c) / (a * b) -
              (2.f * mu1 * c * d) / (a * a * b) + (2.f * mu1 * c * d) / (a * b * b);
    t.d_s11 = -c * d / (a * b * b);
    t.d_s12 = 2.f * c / (a * b);
    return t;
}

__device__ __forceinline__ float2 wpair(int d) {
    return make_float2(c_window[d], c_window[d]);
}

// Every filter below is a sliding window held in registers: a task streams
// its inputs once, in order, into the accumulators of the outputs whose
// window covers them, so each output sums its taps in window order (the
// reference's order, fused multiply-adds from zero). Pairs of independent
// sums (prediction and target moments, two columns, two rows) share one
// paired FP32 multiply-add.
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                     static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int kPending>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(kPending) : "memory");
}

// Asynchronous copies of one channel's two images into s_img (in-image
// positions only: the zero padding written for the first channel stays).
__device__ __forceinline__ void stage_images_async(float* s_img, const float* A, const float* B,
                                                   int ox0, int oy0, int W, int H, int tid) {
#pragma unroll
    for (int it = 0; it < kLoadIters; ++it) {
        const int k = tid + it * kThreads;
        const int r = k / kI, c = k - r * kI;
        const int y = oy0 + r - 2 * kHalo, x = ox0 + c - 2 * kHalo;
        if (k < kI * kI && x >= 0 && x < W && y >= 0 && y < H) {
            const size_t q = size_t(y) * W + x;
            float* d = s_img + r * kImgStride + 2 * c;
            cp_async4(d, A + q);
            cp_async4(d + 1, B + q);
        }
    }
}

// kMasked: images are multiplied by the mask as they are staged (registers);
// without a mask the next channel's images are copied asynchronously into
// shared memory while the current channel's derivative filters run.
template <bool kMetric, bool kMasked>
__global__ void __launch_bounds__(kThreads, 2) fused_l1_ssim_kernel(SsimArgs p) {
    extern __shared__ float4 smem4[];
    float* smem = reinterpret_cast<float*>(smem4);
    float* s_img = smem;                   // [kI][kI + 1] float2
    float* s_row = s_img + kImgFloats;     // [5][kI][kRowStride]
    float* s_mom = s_row + kRowFloats;     // [5][kD][kD]
    float* s_dm = s_row;                   // [3][kD / 2][kD] float2 (phases 4-5)
    float* s_gr = s_row + kDmFloats;       // [kT][kT] gradient tile (phases 4-6)
    float* s_mk = s_gr + kT * kT;          // [kT][kT] mask tile (phases 4-6)
    float* s_ctr = s_mk + kT * kT;         // [kT][kT] float2 tile images (phases 4-6)
    float* s_bwd = s_mom;                  // [3][kD][kT] (phases 5-6)
    __shared__ float s_red[kThreads / 32][2];
    const int tid = threadIdx.x;
    const int W = p.width, H = p.height;
    const int ox0 = blockIdx.x * kT, oy0 = blockIdx.y * kT;
    const size_t P = size_t(W) * H;
    float acc = 0.f, cnt = 0.f;
    if constexpr (!kMasked) {
        // zero padding (never rewritten) and the first channel's images
        for (int k = tid; k < kI * kI; k += kThreads) {
            const int r = k / kI, c = k - r * kI;
            const int y = oy0 + r - 2 * kHalo, x = ox0 + c - 2 * kHalo;
            if (!(x >= 0 && x < W && y >= 0 && y < H))
                *reinterpret_cast<float2*>(s_img + r * kImgStride + 2 * c) = make_float2(0.f, 0.f);
        }
        stage_images_async(s_img, p.pred, p.target, ox0, oy0, W, H, tid);
        cp_async_commit();
    }
    for (int ch = 0; ch < 3; ++ch) {
        // 1. both images with a 10-pixel halo, zero outside
        if constexpr (kMasked) {
            const float* A = p.pred + ch * P;
            const float* B = p.target + ch * P;
            float2 v[kLoadIters];
#pragma unroll
            for (int it = 0; it < kLoadIters; ++it) {
                const int k = tid + it * kThreads;
                const int r = k / kI, c = k - r * kI;
                const int y = oy0 + r - 2 * kHalo, x = ox0 + c - 2 * kHalo;
                v[it] = make_float2(0.f, 0.f);
                if (k < kI * kI && x >= 0 && x < W && y >= 0 && y < H) {
                    const size_t q = size_t(y) * W + x;
                    const float m = __ldg(p.mask + q);
                    v[it] = make_float2(__ldg(A + q) * m, __ldg(B + q) * m);
                }
            }
#pragma unroll
            for (int it = 0; it < kLoadIters; ++it) {
                const int k = tid + it * kThreads;
                const int r = k / kI, c = k - r * kI;
                if (k < kI * kI)
                    *reinterpret_cast<float2*>(s_img + r * kImgStride + 2 * c) = v[it];
            }
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        // 2. row pass: moments (x, x^2, y, y^2, xy) of every staged row onto
        //    the 42 moment columns (moment column c covers image columns c..c+10)
        if (tid < kRowTasks) {
            const int seg = tid % (kD / kRowSeg), r = tid / (kD / kRowSeg);
            const int c0 = seg * kRowSeg;
            const float2* in = reinterpret_cast<const float2*>(s_img + r * kImgStride) + c0;
            float2 s1[kRowSeg], s2[kRowSeg];
            float sp[kRowSeg];
#pragma unroll
            for (int o = 0; o < kRowSeg; ++o) {
                s1[o] = make_float2(0.f, 0.f);
                s2[o] = make_float2(0.f, 0.f);
                sp[o] = 0.f;
            }
#pragma unroll
            for (int i = 0; i < kRowSeg + kTaps - 1; ++i) {
                const float2 v = in[i];
                const float2 sq = __fmul2_rn(v, v);
                const float pr = __fmul_rn(v.x, v.y);
#pragma unroll
                for (int o = 0; o < kRowSeg; ++o) {
                    const int d = i - o;
                    if (d >= 0 && d < kTaps) {
                        s1[o] = __ffma2_rn(v, wpair(d), s1[o]);
                        s2[o] = __ffma2_rn(sq, wpair(d), s2[o]);
                        sp[o] = __fmaf_rn(pr, c_window[d], sp[o]);
                    }
                }
            }
            float* out = s_row + r * kRowStride + c0;
#pragma unroll
            for (int o = 0; o < kRowSeg; o += 2) {
                *reinterpret_cast<float2*>(out + 0 * kI * kRowStride + o) = make_float2(s1[o].x, s1[o + 1].x);
                *reinterpret_cast<float2*>(out + 1 * kI * kRowStride + o) = make_float2(s2[o].x, s2[o + 1].x);
                *reinterpret_cast<float2*>(out + 2 * kI * kRowStride + o) = make_float2(s1[o].y, s1[o + 1].y);
                *reinterpret_cast<float2*>(out + 3 * kI * kRowStride + o) = make_float2(s2[o].y, s2[o + 1].y);
                *reinterpret_cast<float2*>(out + 4 * kI * kRowStride + o) = make_float2(sp[o], sp[o + 1]);
            }
        }
        __syncthreads();
        // 3. column pass: one moment, two adjacent columns, 14 rows per task
        if (tid < kColTasks) {
            const int cp = tid % (kD / 2);
            const int rest = tid / (kD / 2);
            const int seg = rest % (kD / kColSeg), q = rest / (kD / kColSeg);
            const int r0 = seg * kColSeg;
            const float* in = s_row + (q * kI + r0) * kRowStride + 2 * cp;
            float2 m[kColSeg];
#pragma unroll
            for (int o = 0; o < kColSeg; ++o)
                m[o] = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < kColSeg + kTaps - 1; ++i) {
                const float2 v = *reinterpret_cast<const float2*>(in + i * kRowStride);
#pragma unroll
                for (int o = 0; o < kColSeg; ++o) {
                    const int d = i - o;
                    if (d >= 0 && d < kTaps)
                        m[o] = __ffma2_rn(v, wpair(d), m[o]);
                }
            }
            float* out = s_mom + (q * kD + r0) * kMomStride + 2 * cp;
#pragma unroll
            for (int o = 0; o < kColSeg; ++o)
                *reinterpret_cast<float2*>(out + o * kMomStride) = m[o];
        }
        __syncthreads();
        if constexpr (kMetric) {
            // s_img is free: the next channel's images load during the terms
            if (!kMasked && ch < 2) {
                stage_images_async(s_img, p.pred + (ch + 1) * P, p.target + (ch + 1) * P, ox0,
                                   oy0, W, H, tid);
                cp_async_commit();
            }
        } else {
            // the tile's gradient (and mask) rows, read back in phase 6
#pragma unroll
            for (int it = 0; it < kT * kT / kThreads; ++it) {
                const int k = tid + it * kThreads;
                const int y = oy0 + k / kT, x = ox0 + k % kT;
                if (y < H && x < W) {
                    const size_t q = size_t(y) * W + x;
                    cp_async4(s_gr + k, p.grad + ch * P + q);
                    if constexpr (kMasked)
                        cp_async4(s_mk + k, p.mask + q);
                }
                // the tile's own images, kept for phases 4 and 6
                *reinterpret_cast<float2*>(s_ctr + 2 * k) = *reinterpret_cast<const float2*>(
                    s_img + (k / kT + 2 * kHalo) * kImgStride + 2 * (k % kT + 2 * kHalo));
            }
            cp_async_commit();
        }
        // 4. SSIM and its derivative maps (times the valid-window chain) on
        //    the tile and its 5-pixel halo; loss or metric on the tile
        for (int k = tid; k < kD * kD; k += kThreads) {
            const int r = k / kD, c = k - r * kD;
            const float* mp = s_mom + r * kMomStride + c;
            const SsimTerms t = ssim_terms(mp[0], mp[kD * kMomStride], mp[2 * kD * kMomStride],
                                           mp[3 * kD * kMomStride], mp[4 * kD * kMomStride]);
            const int y = oy0 + r - kHalo, x = ox0 + c - kHalo;
            const bool valid = x >= kHalo && x < W - kHalo && y >= kHalo && y < H - kHalo;
            const bool own = r >= kHalo && r < kHalo + kT && c >= kHalo && c < kHalo + kT;
            if constexpr (kMetric) {
                if (own && valid && (!kMasked || p.mask[size_t(y) * W + x] > 0.f)) {
                    acc += t.ssim;
                    cnt += 1.f;
                }
            } else {
                const float chain = valid ? p.norm : 0.f;
                float* o = s_dm + (r >> 1) * (2 * kD) + 2 * c + (r & 1);
                o[0] = -p.lambda * t.d_mu1 * chain;
                o[kD * kD] = -p.lambda * t.d_s11 * chain;
                o[2 * kD * kD] = -p.lambda * t.d_s12 * chain;
                if (own && valid) {
                    const float2 ab = *reinterpret_cast<const float2*>(
                        s_img + (r + kHalo) * kImgStride + 2 * (c + kHalo));
                    const float l1 = fabsf(ab.x - ab.y);
                    acc += p.norm * (p.lambda * (1.f - t.ssim) + (1.f - p.lambda) * l1);
                }
            }
        }
        __syncthreads();
        if constexpr (!kMetric) {
            // s_img is free (phase 6 reads s_ctr): the next channel's images
            // load during the derivative filters
            const bool next = !kMasked && ch < 2;
            if (next) {
                stage_images_async(s_img, p.pred + (ch + 1) * P, p.target + (ch + 1) * P, ox0,
                                   oy0, W, H, tid);
                cp_async_commit();
            }
            // 5. derivative maps along rows onto the tile's columns: one map,
            //    two rows (interleaved pair), 8 columns per task
            if (tid < kBRowTasks) {
                const int seg = tid % (kT / kBRowSeg);
                const int rest = tid / (kT / kBRowSeg);
                const int rp = rest % (kD / 2), mi = rest / (kD / 2);
                const int c0 = seg * kBRowSeg;
                const float2* in =
                    reinterpret_cast<const float2*>(s_dm + mi * kD * kD + rp * 2 * kD) + c0;
                float2 g[kBRowSeg];
#pragma unroll
                for (int o = 0; o < kBRowSeg; ++o)
                    g[o] = make_float2(0.f, 0.f);
#pragma unroll
                for (int i = 0; i < kBRowSeg + kTaps - 1; ++i) {
                    const float2 v = in[i];
#pragma unroll
                    for (int o = 0; o < kBRowSeg; ++o) {
                        const int d = i - o;
                        if (d >= 0 && d < kTaps)
                            g[o] = __ffma2_rn(v, wpair(d), g[o]);
                    }
                }
                float* out = s_bwd + (mi * kD + 2 * rp) * kBwdStride + c0;
#pragma unroll
                for (int o = 0; o < kBRowSeg; o += 2) {
                    *reinterpret_cast<float2*>(out + o) = make_float2(g[o].x, g[o + 1].x);
                    *reinterpret_cast<float2*>(out + kBwdStride + o) = make_float2(g[o].y, g[o + 1].y);
                }
            }
            // the gradient (and mask) tile has landed once every thread's
            // earlier group is complete
            if (next)
                cp_async_wait<1>();
            else
                cp_async_wait<0>();
            __syncthreads();
            // 6. along columns, and the gradient of 2 x 2 tile pixels per task
            if (tid < kBColTasks) {
                const int cp = tid % (kT / 2), rp = tid / (kT / 2);
                float2 g[3][2];
#pragma unroll
                for (int mi = 0; mi < 3; ++mi) {
                    g[mi][0] = g[mi][1] = make_float2(0.f, 0.f);
                    const float* in = s_bwd + (mi * kD + 2 * rp) * kBwdStride + 2 * cp;
#pragma unroll
                    for (int i = 0; i < kTaps + 1; ++i) {
                        const float2 v = *reinterpret_cast<const float2*>(in + i * kBwdStride);
                        if (i < kTaps)
                            g[mi][0] = __ffma2_rn(v, wpair(i), g[mi][0]);
                        if (i >= 1)
                            g[mi][1] = __ffma2_rn(v, wpair(i - 1), g[mi][1]);
                    }
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int ty = 2 * rp + j, y = oy0 + ty;
                    if (y >= H)
                        continue;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int tc = 2 * cp + e, x = ox0 + tc;
                        if (x >= W)
                            continue;
                        const float2 ab = *reinterpret_cast<const float2*>(s_ctr + 2 * (ty * kT + tc));
                        const float a = ab.x, b = ab.y;
                        const float s0 = e ? g[0][j].y : g[0][j].x;
                        const float s1 = e ? g[1][j].y : g[1][j].x;
                        const float s2 = e ? g[2][j].y : g[2][j].x;
                        const bool valid =
                            x >= kHalo && x < W - kHalo && y >= kHalo && y < H - kHalo;
                        const float chain = valid ? p.norm : 0.f;
                        const float sign = a == b ? 0.f : copysignf(1.f, a - b);
                        const float m = kMasked ? s_mk[ty * kT + tc] : 1.f;
                        p.grad[ch * P + size_t(y) * W + x] =
                            s_gr[ty * kT + tc] +
                            (s0 + 2.f * a * s1 + b * s2 + (1.f - p.lambda) * sign * chain) * m;
                    }
                }
            }
        }
        __syncthreads();
    }
    // per-CTA partial: warp sums, then one thread
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, off);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    }
    if ((tid & 31) == 0) {
        s_red[tid >> 5][0] = acc;
        s_red[tid >> 5][1] = cnt;
    }
    __syncthreads();
    if (tid == 0) {
        float s = 0.f, n = 0.f;
        for (int w = 0; w < kThreads / 32; ++w) {
            s += s_red[w][0];
            n += s_red[w][1];
        }
        const int blk = blockIdx.y * gridDim.x + blockIdx.x;
        if constexpr (kMetric) {
            p.partial[2 * blk] = s;
            p.partial[2 * blk + 1] = n;
        } else {
            p.partial[blk] = s;
        }
    }
}

// Deterministic final reduction of the per-CTA partials (double): the loss
// is added to *out, the metric (sum / count) written.
__global__ void reduce_partials_kernel(const float* __restrict__ partial, int blocks, int stride,
                                       bool ratio, float* __restrict__ out) {
    __shared__ double s0[256], s1[256];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < blocks; i += 256) {
        a += partial[size_t(i) * stride];
        if (ratio)
            b += partial[size_t(i) * stride + 1];
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = b;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            s0[threadIdx.x] += s0[threadIdx.x + k];
            s1[threadIdx.x] += s1[threadIdx.x + k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (ratio)
            *out = s1[0] > 0.0 ? float(s0[0] / s1[0]) : 0.f;
        else
            *out += float(s0[0]); // the loss adds into the caller's scalar, as the gradient does
    }
}

constexpr size_t kSmemBytes = sizeof(float) * (kImgFloats + kRowFloats + kMomFloats);

template <bool kMetric, bool kMasked>
void launch_ssim_kernel(cudaStream_t s, dim3 grid, const SsimArgs& a) {
    cudaFuncSetAttribute(fused_l1_ssim_kernel<kMetric, kMasked>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes));
    fused_l1_ssim_kernel<kMetric, kMasked><<<grid, kThreads, kSmemBytes, s>>>(a);
}

} // namespace

size_t ssim_partial_floats(int width, int height) {
    const size_t blocks = size_t((width + kT - 1) / kT) * ((height + kT - 1) / kT);
    return 2 * blocks;
}

cudaError_t launch_fused_l1_ssim(cudaStream_t s, const float* pred, const float* target,
                                 const float* mask, int width, int height, float ssim_weight,
                                 float photometric_weight, float* grad, float* loss_out,
                                 float* partial) {
    const dim3 grid((width + kT - 1) / kT, (height + kT - 1) / kT);
    SsimArgs a{pred, target, mask, width, height, ssim_weight,
               photometric_weight / float(3 * (width - 2 * kHalo) * (height - 2 * kHalo)),
               grad, partial};
    if (mask)
        launch_ssim_kernel<false, true>(s, grid, a);
    else
        launch_ssim_kernel<false, false>(s, grid, a);
    if (loss_out)
        reduce_partials_kernel<<<1, 256, 0, s>>>(partial, int(grid.x * grid.y), 1, false,
                                                 loss_out);
    return cudaGetLastError();
}

cudaError_t launch_ssim_metric(cudaStream_t s, const float* pred, const float* target,
                               const float* mask, int width, int height, float* out,
                               float* partial) {
    const dim3 grid((width + kT - 1) / kT, (height + kT - 1) / kT);
    SsimArgs a{pred, target, mask, width, height, 1.f, 0.f, nullptr, partial};
    if (mask)
        launch_ssim_kernel<true, true>(s, grid, a);
    else
        launch_ssim_kernel<true, false>(s, grid, a);
    reduce_partials_kernel<<<1, 256, 0, s>>>(partial, int(grid.x * grid.y), 2, true, out);
    return cudaGetLastError();
}

} // namespace gsb
