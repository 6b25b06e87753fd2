// Per-tile front-to-back compositing and its reverse-order adjoint, as device
// functions over one tile, shared by the single-view kernels (one CTA per
// tile) and the batched persistent kernels (each CTA loops over tiles of many
// views).
//
// Forward numerics follow blend_tile pass 1
// (third_party/splat_drender/src/render_forward.cu:341-416, :508-525):
//   power = gaussian_power(conic, mean - pixel); skip power > 0;
//   alpha = min(alpha_clip, o * exp(power)); skip alpha < 1/255;
//   T' = T (1 - alpha); T' < 1e-4 ends the pixel WITHOUT blending;
//   C += rgb * alpha * T;  out = C + T * bg, alpha_out = 1 - T.
// B200 organisation: a TW x TH tile with PX vertically adjacent pixels per
// thread; lane l owns column l % TW and PX rows of row group l / TW, so a warp
// covers a band of (32 / TW) * PX rows. Gaussian batches are staged in shared
// memory; each warp rejects a Gaussian whose alpha >= 1/255 box (widened by
// one pixel, so the test can only drop work the per-pixel test would drop)
// misses its band, and stops as soon as all of its 32*PX pixels saturate.
//
// Backward: the reference restarts from stored 32-instance snapshots
// (render_backward.cu:156-519). Here each tile walks its list back to front
// from every pixel's last contributor, recovering T by T_i = T_{i+1}/(1-a_i)
// from the stored final transmittance (no per-pixel lists or snapshots), and
// reduces each Gaussian's 12 partial gradients (summed over the thread's PX
// pixels) across the warp with a 13-shuffle reduce-scatter before
// shared-memory accumulation and one set of float4 global atomics per
// (Gaussian, tile).
//
// The per-pixel arithmetic does not depend on the tile shape: a pixel blends
// the same Gaussians in the same order whatever TW x TH is, because a
// Gaussian reaches a pixel only inside its alpha = 1/255 contour, which the
// tile walk covers exactly.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace gsb {

constexpr int kMaxBatch = 256;

template <int TW, int TH, int PX> struct TileGeom {
    static_assert(TW == 8 || TW == 16 || TW == 32, "tile width must be 8, 16 or 32");
    static constexpr int kPixels = TW * TH;
    static constexpr int kThreads = kPixels / PX;
    static_assert(kThreads % 32 == 0 && kThreads >= 32 && kThreads <= 1024,
                  "tile / pixels-per-thread give a whole number of warps");
    static constexpr int kWarps = kThreads / 32;
    static_assert(kWarps <= 8, "the staged band mask holds one bit per warp");
    static constexpr int kRowGroups = 32 / TW;          // row groups per warp
    static constexpr int kBandRows = kRowGroups * PX;   // rows per warp
    static_assert(kBandRows * kWarps == TH, "warps tile the rows exactly");
    static constexpr int kBatch = kThreads * 2 > kMaxBatch ? kMaxBatch : kThreads * 2;
};

// A staged batch of a tile's Gaussians, one array per field (plain loads).
template <int B> struct TileStage {
    unsigned id[B];
    float2 xy[B];
    float4 co[B];
    float4 rgb[B];
    unsigned char band[B]; // bit w: the Gaussian's pixel box reaches warp w's rows
    __device__ __forceinline__ float2 xy_of(int j) const { return xy[j]; }
    __device__ __forceinline__ float4 co_of(int j) const { return co[j]; }
    __device__ __forceinline__ float4 rgb_of(int j) const { return rgb[j]; }
};

// A staged batch as 64-byte records, filled by TMA gathers (tile::gather4:
// four records, at four Gaussian ids, per copy) that complete on `bar`.
template <int B> struct __align__(128) RecStage {
    SplatRec rec[B];       // TMA destination (128-byte aligned)
    unsigned id[B];
    unsigned char band[B]; // bit w: the Gaussian's pixel box reaches warp w's rows
    unsigned long long bar;
    __device__ __forceinline__ float2 xy_of(int j) const { return rec[j].xy; }
    __device__ __forceinline__ float4 co_of(int j) const { return rec[j].co; }
    __device__ __forceinline__ float4 rgb_of(int j) const { return rec[j].rgb; }
};
static_assert(kMaxBatch % 4 == 0, "gathers of four records fill a batch exactly");

// TMA staging state of one CTA: the record array's tensor map (rows of 16
// floats, one row per Gaussian), the device error word, and the parity of the
// mbarrier phase the next batch completes.
struct TmaGather {
    const CUtensorMap* map = nullptr;
    unsigned* err = nullptr;
    unsigned phase = 0;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// One wait for the phase of `parity`: the thread is suspended until the phase
// completes or about `suspend_ns` pass (a hint, in nanoseconds), instead of
// spinning on issue slots the working warps need. True if it completed.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity,
                                              unsigned suspend_ns) {
    unsigned done;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity), "r"(suspend_ns)
                 : "memory");
    return done != 0;
}
// Waits for the phase of `parity`, at most `limit` suspended waits of about a
// microsecond each; false if the phase did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned limit) {
    for (unsigned k = 0; k < limit; ++k)
        if (mbar_try_wait(bar, parity, 1000u))
            return true;
    return false;
}
constexpr unsigned kStageWaitLimit = 1u << 18; // ~0.26 s at most

// Four 64-byte rows (Gaussian ids r0..r3) of the record tensor into dst
// (256 contiguous bytes), completing on bar. The column coordinate is 0, so
// the copy's innermost offset is 16-byte aligned by construction.
__device__ __forceinline__ void tma_gather4(void* dst, const CUtensorMap* map, int r0, int r1,
                                            int r2, int r3, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_u32(bar)), "r"(0), "r"(r0),
        "r"(r1), "r"(r2), "r"(r3)
        : "memory");
}

template <int TW, int kRows>
__device__ __forceinline__ bool band_hit(ushort4 b, int x0, int y0) {
    // Warp pixels: x in [x0, x0+TW), y in [y0, y0+kRows); box widened by 1 px
    // so the test can only drop Gaussians whose alpha is below 1/255 there.
    return int(b.x) - 1 < x0 + TW && int(b.y) + 1 > x0 && int(b.z) - 1 < y0 + kRows &&
           int(b.w) + 1 > y0;
}

// Stages a batch of the tile's Gaussians; the band test of every warp of the
// tile (origin x0, y0) is done here once per Gaussian, so the blend loops
// test one bit instead of the box.
template <int TW, int TH, int PX, int B>
__device__ __forceinline__ void stage_batch(TileStage<B>& s, const unsigned* __restrict__ order,
                                            unsigned first, int cnt, const GaussianState& st,
                                            int tid, int x0, int y0) {
    using G = TileGeom<TW, TH, PX>;
    for (int k = tid; k < cnt; k += G::kThreads) {
        const unsigned g = order[first + k];
        s.id[k] = g;
        s.xy[k] = st.mean2d[g];
        s.co[k] = st.conic[g];
        s.rgb[k] = st.rgb[g];
        const ushort4 b = st.bounds[g];
        unsigned m = 0;
#pragma unroll
        for (int w = 0; w < G::kWarps; ++w)
            if (band_hit<TW, G::kBandRows>(b, x0, y0 + G::kBandRows * w))
                m |= 1u << w;
        s.band[k] = static_cast<unsigned char>(m);
    }
}


template <int TW, int TH, int PX, int B>
__device__ __forceinline__ bool stage_any(TileStage<B>& s, const unsigned* __restrict__ order,
                                          unsigned first, int cnt, const GaussianState& st,
                                          int tid, int x0, int y0, TmaGather&) {
    stage_batch<TW, TH, PX>(s, order, first, cnt, st, tid, x0, y0);
    return true;
}

// TMA staging of a batch: the first warp reads the batch's Gaussian ids
// (coalesced) and issues one tile::gather4 copy per four records after one
// lane has announced the batch's bytes on the mbarrier; every thread waits
// for the phase (bounded), then the band masks are computed from the staged
// boxes. The caller synchronises the CTA afterwards, and before the next
// batch overwrites this one. A wait that gives up (which only a broken
// invariant could cause) sets kDevStageTimeout, waits once more for the
// copies in flight and returns false in every thread.
template <int TW, int TH, int PX, int B>
__device__ __forceinline__ bool stage_any(RecStage<B>& s, const unsigned* __restrict__ order,
                                          unsigned first, int cnt, const GaussianState&, int tid,
                                          int x0, int y0, TmaGather& g) {
    using G = TileGeom<TW, TH, PX>;
    const int ops = (cnt + 3) >> 2;
    if (tid < 32) {
        if (tid == 0)
            mbar_arrive_expect_tx(&s.bar, unsigned(ops) * 4u * unsigned(sizeof(SplatRec)));
        __syncwarp();
        // the previous batch's shared-memory reads (ordered before this point
        // by the caller's barrier) come before this batch's asynchronous writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int op = tid; op < ops; op += 32) {
            int r[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int k = 4 * op + q;
                r[q] = int(order[first + unsigned(min(k, cnt - 1))]);
                if (k < cnt)
                    s.id[k] = unsigned(r[q]);
            }
            tma_gather4(&s.rec[4 * op], g.map, r[0], r[1], r[2], r[3], &s.bar);
        }
    }
    const bool ok = mbar_wait_bounded(&s.bar, g.phase, kStageWaitLimit);
    if (__syncthreads_or(!ok)) {
        if (tid == 0)
            atomicOr(g.err, kDevStageTimeout);
        mbar_wait_bounded(&s.bar, g.phase, kStageWaitLimit);
        return false;
    }
    g.phase ^= 1u;
    for (int k = tid; k < cnt; k += G::kThreads) {
        const ushort4 b = s.rec[k].bounds;
        unsigned m = 0;
#pragma unroll
        for (int w = 0; w < G::kWarps; ++w)
            if (band_hit<TW, G::kBandRows>(b, x0, y0 + G::kBandRows * w))
                m |= 1u << w;
        s.band[k] = static_cast<unsigned char>(m);
    }
    return true;
}

// One view's image constants and buffers, already offset to that view.
struct ViewTarget {
    int width, height;
    float clip;
    float3 bg;
    float* color;        // [3][H][W]
    float* alpha;        // [H][W]
    float* pix_T;        // [H][W] final transmittance (NULL: inference only)
    unsigned* pix_last;  // [H][W] 1 + position of the last blended instance
};

struct ViewGrads {
    int width, height;
    float clip;
    float3 bg;
    const float* pix_T;
    const unsigned* pix_last;
    const float* dL_color;
    const float* dL_alpha;    // may be NULL
    const float* densify_map; // may be NULL
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }

// The forward blend of one Gaussian at two vertically adjacent pixels (rows
// fya, fyb of one column). Same expressions as the scalar step, in the same
// rounding (gaussian_power's explicit round-to-nearest products and sums, the
// pair on sm_100 f32x2 instructions), so both pixels take the scalar path's
// decisions; the decisions become selects instead of branches. Returns
// whether either pixel blended.
__device__ __forceinline__ bool pixel_forward_pair(float4 co, float dx, float my, float fya,
                                                   float fyb, float clip, float4 c,
                                                   unsigned pos, float2& T, float2& r, float2& g,
                                                   float2& b, unsigned& la, unsigned& lb,
                                                   bool& da, bool& db) {
    if (da && db)
        return false;
    const float xx = __fmul_rn(co.x, dx);
    const float nxy = -__fmul_rn(co.y, dx);
    const float2 dy = __fadd2_rn(f2s(my), f2(-fya, -fyb));
    const float2 yy = __fmul2_rn(__fmul2_rn(f2s(co.z), dy), dy);
    const float2 power = __fadd2_rn(__fmul2_rn(f2s(-0.5f), __ffma2_rn(f2s(dx), f2s(xx), yy)),
                                    __fmul2_rn(f2s(nxy), dy));
    const float2 og = __fmul2_rn(f2s(co.w), f2(expf(power.x), expf(power.y)));
    const float aa = fminf(clip, og.x), ab = fminf(clip, og.y);
    const bool va = !da && !(power.x > 0.f) && !(aa < kAlphaFloor);
    const bool vb = !db && !(power.y > 0.f) && !(ab < kAlphaFloor);
    const float2 tt = __fmul2_rn(T, __fadd2_rn(f2s(1.f), f2(-aa, -ab)));
    const bool sa = tt.x < kTransmittanceFloor, sb = tt.y < kTransmittanceFloor;
    da = da || (va && sa);
    db = db || (vb && sb);
    const bool bla = va && !sa, blb = vb && !sb;
    const float aea = bla ? aa : 0.f, aeb = blb ? ab : 0.f;
    const float2 w = __fmul2_rn(f2(aea, aeb), T);
    r = __ffma2_rn(f2s(c.x), w, r);
    g = __ffma2_rn(f2s(c.y), w, g);
    b = __ffma2_rn(f2s(c.z), w, b);
    // T (1 - 0) = T exactly, and T (1 - alpha) = tt when blending: the update
    // runs on the FMA pipe (the ALU pipe, with the decisions, is the busier).
    T = __fmul2_rn(T, __fadd2_rn(f2s(1.f), f2(-aea, -aeb)));
    la = bla ? pos : la;
    lb = blb ? pos : lb;
    return bla || blb;
}

// Adds a per-lane count to *out with one atomic per warp.
__device__ __forceinline__ void warp_count_add(unsigned long long v, unsigned long long* out) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v)
        atomicAdd(out, v);
}

// Forward of tile (tx, ty) over instances [range.x, range.y) of `order`.
// s_vis must be zero on entry and is zero on exit. kCount: also adds to
// *pairs the (Gaussian, pixel) pairs whose alpha test runs (the pixel not yet
// saturated when its warp takes the Gaussian), for the roofline figures.
// work (may be NULL): receives the tile's adjoint work estimate (the sum over
// warps of their pixels' largest last-contributor position).
template <int TW, int TH, int PX, bool kCount = false, typename Stage>
__device__ __forceinline__ void composite_forward_tile(
    Stage& s, unsigned char* s_vis, int tx, int ty,
    uint2 range, const unsigned* __restrict__ order, const GaussianState& st,
    const ViewTarget& o, float* __restrict__ visibility,
    unsigned long long* __restrict__ pairs = nullptr, TmaGather* tma = nullptr,
    unsigned* __restrict__ work = nullptr) {
    using G = TileGeom<TW, TH, PX>;
    constexpr int B = G::kBatch;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int px = tx * TW + (lane % TW);
    const int wx0 = tx * TW, wy0 = ty * TH + G::kBandRows * warp;
    const int py0 = wy0 + PX * (lane / TW);
    const float fx = float(px);
    const int n = int(range.y - range.x);
    const float clip = o.clip;

    // Pixel pairs keep their state in float2 registers (the f32x2 operands);
    // the scalar path (odd PX) in plain arrays.
    constexpr int NP = PX % 2 == 0 ? PX / 2 : 1;
    constexpr int NS = PX % 2 == 0 ? 1 : PX;
    float2 T2[NP], r2[NP], g2[NP], b2[NP];
    float T[NS], cr[NS], cg[NS], cb[NS];
    unsigned last[PX];
    bool done[PX];
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        T2[q] = f2s(1.f);
        r2[q] = g2[q] = b2[q] = f2s(0.f);
    }
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        T[q] = 1.f;
        cr[q] = cg[q] = cb[q] = 0.f;
    }
#pragma unroll
    for (int p = 0; p < PX; ++p) {
        last[p] = 0;
        done[p] = !(px < o.width && py0 + p < o.height);
    }
    auto all_done = [&]() {
        bool d = true;
#pragma unroll
        for (int p = 0; p < PX; ++p) d = d && done[p];
        return d;
    };
    unsigned long long evaluated = 0;
    TmaGather no_tma;

    for (int base = 0; base < n; base += B) {
        if (__syncthreads_count(!all_done()) == 0)
            break;
        const int cnt = min(B, n - base);
        if (!stage_any<TW, TH, PX>(s, order, range.x + base, cnt, st, tid, tx * TW, ty * TH,
                                   tma ? *tma : no_tma))
            return;
        __syncthreads();
        if constexpr (PX == 1 && !kCount) {
            // One pixel per thread (the schedule of frames with few tiles,
            // where a tile's serial walk is the kernel's time): two Gaussians
            // per step. Their exponents and opacities are independent and
            // computed together; the blend decisions then run in order, the
            // second on the transmittance the first left (the same decisions
            // and arithmetic as one Gaussian per step).
            int j = 0;
            // every loop condition is warp-uniform (band bits are per warp)
            for (;;) {
                if (__all_sync(0xffffffffu, done[0]))
                    break;
                while (j < cnt && !((s.band[j] >> warp) & 1u))
                    ++j;
                if (j >= cnt)
                    break;
                int j2 = j + 1;
                while (j2 < cnt && !((s.band[j2] >> warp) & 1u))
                    ++j2;
                const bool two = j2 < cnt;
                const float py = float(py0);
                const float2 m0 = s.xy_of(j);
                const float4 co0 = s.co_of(j);
                const float2 m1 = two ? s.xy_of(j2) : m0;
                const float4 co1 = two ? s.co_of(j2) : co0;
                const float pw0 = gaussian_power(co0, m0.x - fx, m0.y - py);
                const float pw1 = gaussian_power(co1, m1.x - fx, m1.y - py);
                const float a0 = fminf(clip, co0.w * expf(pw0));
                const float a1 = fminf(clip, co1.w * expf(pw1));
                bool bl0 = false, bl1 = false;
                if (!done[0] && !(pw0 > 0.f) && !(a0 < kAlphaFloor)) {
                    const float test_t = T[0] * (1.f - a0);
                    if (test_t < kTransmittanceFloor) {
                        done[0] = true;
                    } else {
                        const float w = a0 * T[0];
                        const float4 c = s.rgb_of(j);
                        cr[0] += c.x * w;
                        cg[0] += c.y * w;
                        cb[0] += c.z * w;
                        T[0] = test_t;
                        last[0] = unsigned(base + j + 1);
                        bl0 = true;
                    }
                }
                if (two && !done[0] && !(pw1 > 0.f) && !(a1 < kAlphaFloor)) {
                    const float test_t = T[0] * (1.f - a1);
                    if (test_t < kTransmittanceFloor) {
                        done[0] = true;
                    } else {
                        const float w = a1 * T[0];
                        const float4 c = s.rgb_of(j2);
                        cr[0] += c.x * w;
                        cg[0] += c.y * w;
                        cb[0] += c.z * w;
                        T[0] = test_t;
                        last[0] = unsigned(base + j2 + 1);
                        bl1 = true;
                    }
                }
                if (bl0)
                    s_vis[j] = 1;
                if (bl1)
                    s_vis[j2] = 1;
                j = j2 + 1;
            }
        } else if (!__all_sync(0xffffffffu, all_done())) {
            for (int j = 0; j < cnt; ++j) {
                if (!((s.band[j] >> warp) & 1u))
                    continue;
                const float2 m = s.xy_of(j);
                const float4 co = s.co_of(j);
                const float dx = m.x - fx;
                bool blended = false;
                if constexpr (PX % 2 == 0) {
                    const float4 c = s.rgb_of(j);
                    const unsigned pos = unsigned(base + j + 1);
                    if constexpr (kCount) {
#pragma unroll
                        for (int p = 0; p < PX; ++p)
                            evaluated += done[p] ? 0u : 1u;
                    }
#pragma unroll
                    for (int p = 0; p < PX; p += 2)
                        blended |= pixel_forward_pair(co, dx, m.y, float(py0 + p),
                                                      float(py0 + p + 1), clip, c, pos,
                                                      T2[p / 2], r2[p / 2], g2[p / 2],
                                                      b2[p / 2], last[p], last[p + 1], done[p],
                                                      done[p + 1]);
                    if (blended)
                        s_vis[j] = 1;
                    // saturation is checked every fourth Gaussian: a pixel
                    // pair past its last one returns at its first test
                    // (1M / 1080p: 0.323 ms voting every Gaussian, 0.316
                    // every other, 0.312 every fourth)
                    if ((j & 3) == 3 && __all_sync(0xffffffffu, all_done()))
                        break;
                    continue;
                } else {
#pragma unroll
                for (int p = 0; p < PX; ++p) {
                    if (done[p])
                        continue;
                    if constexpr (kCount)
                        ++evaluated;
                    const float dy = m.y - float(py0 + p);
                    const float power = gaussian_power(co, dx, dy);
                    if (power > 0.f)
                        continue;
                    const float alpha = fminf(clip, co.w * expf(power));
                    if (alpha < kAlphaFloor)
                        continue;
                    const float test_t = T[p] * (1.f - alpha);
                    if (test_t < kTransmittanceFloor) {
                        done[p] = true;
                        continue;
                    }
                    const float w = alpha * T[p];
                    const float4 c = s.rgb_of(j);
                    cr[p] += c.x * w;
                    cg[p] += c.y * w;
                    cb[p] += c.z * w;
                    T[p] = test_t;
                    last[p] = unsigned(base + j + 1);
                    blended = true;
                }
                if (blended)
                    s_vis[j] = 1;
                if (__all_sync(0xffffffffu, all_done()))
                    break;
                }
            }
        }
        __syncthreads();
        for (int k = tid; k < cnt; k += G::kThreads) {
            if (visibility && s_vis[k])
                visibility[s.id[k]] = 1.f;
            s_vis[k] = 0;
        }
    }
    if constexpr (kCount)
        warp_count_add(evaluated, pairs);
    if (work) {
        // the adjoint's work on this tile: each warp walks back from its
        // pixels' last contributor, so the sum of the warps' maxima
        unsigned wl = 0;
#pragma unroll
        for (int p = 0; p < PX; ++p)
            wl = max(wl, last[p]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            wl = max(wl, __shfl_xor_sync(0xffffffffu, wl, off));
        if (lane == 0 && wl)
            atomicAdd(work, wl);
    }
    const size_t P = size_t(o.width) * o.height;
#pragma unroll
    for (int p = 0; p < PX; ++p) {
        if (!(px < o.width && py0 + p < o.height))
            continue;
        float t, r, g, b;
        if constexpr (PX % 2 == 0) {
            const bool hi = p & 1;
            t = hi ? T2[p / 2].y : T2[p / 2].x;
            r = hi ? r2[p / 2].y : r2[p / 2].x;
            g = hi ? g2[p / 2].y : g2[p / 2].x;
            b = hi ? b2[p / 2].y : b2[p / 2].x;
        } else {
            t = T[p];
            r = cr[p];
            g = cg[p];
            b = cb[p];
        }
        const size_t pid = size_t(py0 + p) * o.width + px;
        o.color[pid] = r + t * o.bg.x;
        o.color[P + pid] = g + t * o.bg.y;
        o.color[2 * P + pid] = b + t * o.bg.z;
        o.alpha[pid] = 1.f - t;
        if (o.pix_T) {
            o.pix_T[pid] = t;
            o.pix_last[pid] = last[p];
        }
    }
}

// Reduce 12 per-lane values across the warp; returns the summed value of
// slot `slot` (or slot = -1 for lanes that hold nothing).
__device__ __forceinline__ float reduce_scatter12(const float (&v)[12], int& slot) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
    float u[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float send = b4 ? v[k] : v[k + 6];
        const float keep = b4 ? v[k + 6] : v[k];
        u[k] = keep + __shfl_xor_sync(full, send, 16);
    }
    float w[4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float send = b3 ? u[k] : u[k + 3];
        const float keep = b3 ? u[k + 3] : u[k];
        w[k] = keep + __shfl_xor_sync(full, send, 8);
    }
    w[3] = 0.f;
    float x[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float send = b2 ? w[k] : w[k + 2];
        const float keep = b2 ? w[k + 2] : w[k];
        x[k] = keep + __shfl_xor_sync(full, send, 4);
    }
    const float send = b1 ? x[0] : x[1];
    const float keep = b1 ? x[1] : x[0];
    float y = keep + __shfl_xor_sync(full, send, 2);
    y += __shfl_xor_sync(full, y, 1);
    const int idx = b2 ? (b1 ? -1 : 2) : (b1 ? 1 : 0);
    slot = (idx < 0 || (lane & 1)) ? -1 : (b4 ? 6 : 0) + (b3 ? 3 : 0) + idx;
    return y;
}

// reduce_scatter12 for the ten partials that are not densify terms (slots 7
// and 11 are zero without a densify map): the same butterfly over ten values,
// one shuffle and four selects fewer per Gaussian and warp. Returns the sum
// for partial slot `slot` (-1: nothing) in reduce_scatter12's numbering.
__device__ __forceinline__ float reduce_scatter10(const float (&v)[12], int& slot) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
    // packed order: partials 0-6, 8, 9, 10
    const float p[10] = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[8], v[9], v[10]};
    float u[6];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const float send = b4 ? p[k] : p[k + 5];
        const float keep = b4 ? p[k + 5] : p[k];
        u[k] = keep + __shfl_xor_sync(full, send, 16);
    }
    u[5] = 0.f;
    float w[4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float send = b3 ? u[k] : u[k + 3];
        const float keep = b3 ? u[k + 3] : u[k];
        w[k] = keep + __shfl_xor_sync(full, send, 8);
    }
    w[3] = 0.f;
    float x[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float send = b2 ? w[k] : w[k + 2];
        const float keep = b2 ? w[k + 2] : w[k];
        x[k] = keep + __shfl_xor_sync(full, send, 4);
    }
    const float send = b1 ? x[0] : x[1];
    const float keep = b1 ? x[1] : x[0];
    float y = keep + __shfl_xor_sync(full, send, 2);
    y += __shfl_xor_sync(full, y, 1);
    // element of the lane's group of five: the group of three (b3) it ended
    // in, and its place there (b2, b1; the fourth place is padding)
    const int idx3 = b2 ? (b1 ? -1 : 2) : (b1 ? 1 : 0);
    const int e5 = idx3 < 0 ? -1 : (b3 ? 3 : 0) + idx3;
    const int packed = (b4 ? 5 : 0) + e5;
    slot = (e5 < 0 || e5 >= 5 || (lane & 1)) ? -1 : (packed < 7 ? packed : packed + 1);
    return y;
}

// Per-pixel backward state.
struct PixBack {
    float T, sdot, gx, gy, gz, fin_term, refine_scale, dmap;
    unsigned last;
};

__device__ __forceinline__ void pixel_backward_init(PixBack& p, bool inside, size_t pid, size_t P,
                                                    float3 bg, const float* __restrict__ pix_T,
                                                    const unsigned* __restrict__ pix_last,
                                                    const float* __restrict__ dL_color,
                                                    const float* __restrict__ dL_alpha,
                                                    const float* __restrict__ densify_map) {
    float T_final = 1.f;
    p.gx = p.gy = p.gz = 0.f;
    p.dmap = 0.f;
    p.last = 0;
    float dfin = 0.f;
    if (inside) {
        T_final = pix_T[pid];
        p.last = pix_last[pid];
        p.gx = dL_color[pid];
        p.gy = dL_color[P + pid];
        p.gz = dL_color[2 * P + pid];
        dfin = bg.x * p.gx + bg.y * p.gy + bg.z * p.gz - (dL_alpha ? dL_alpha[pid] : 0.f);
        p.dmap = densify_map ? densify_map[pid] : 0.f;
    }
    p.refine_scale = 1.f / fmaxf(1.f - T_final, 1.0e-5f);
    p.fin_term = T_final * dfin;
    p.T = T_final;
    p.sdot = 0.f;
}

// The forward's blend decision of Gaussian (m, co) at a pixel, evaluated on
// its own (no pixel state needed) so two Gaussians' can be in flight at once.
struct BlendEval {
    float dx, dy, G, alpha;
    bool ok; // the Gaussian lies before the pixel's last contributor and blended there
};

__device__ __forceinline__ BlendEval blend_eval(unsigned pos, unsigned last, float2 m, float4 co,
                                                float fx, float fy, float clip) {
    BlendEval e;
    e.dx = m.x - fx;
    e.dy = m.y - fy;
    const float power = gaussian_power(co, e.dx, e.dy);
    e.G = expf(power);
    e.alpha = fminf(clip, co.w * e.G);
    e.ok = pos < last && !(power > 0.f) && !(e.alpha < kAlphaFloor);
    return e;
}

// The adjoint of one blended Gaussian at a pixel: recovers T, adds the
// pixel's contribution of Gaussian (co, c) to v.
template <bool kRefine, bool kDensify>
__device__ __forceinline__ void pixel_backward_finish(PixBack& p, const BlendEval& e, float4 co,
                                                      float4 c, float Wf, float Hf,
                                                      float (&v)[12]) {
    const float alpha = e.alpha, G = e.G, dx = e.dx, dy = e.dy;
    const float inv_1ma = 1.f / (1.f - alpha);
    p.T = p.T * inv_1ma;
    const float w = alpha * p.T;
    const float cdot = c.x * p.gx + c.y * p.gy + c.z * p.gz;
    const float dL_da = p.T * cdot - (p.sdot + p.fin_term) * inv_1ma;
    p.sdot += w * cdot;
    const float dL_dG = co.w * dL_da;
    const float gdx = G * dx, gdy = G * dy;
    const float dmx = dL_dG * (-gdx * co.x - gdy * co.y);
    const float dmy = dL_dG * (-gdy * co.z - gdx * co.y);
    v[0] += -0.5f * gdx * dx * dL_dG;
    v[1] += -0.5f * gdx * dy * dL_dG;
    v[2] += -0.5f * gdy * dy * dL_dG;
    v[3] += G * dL_da;
    v[4] += dmx;
    v[5] += dmy;
    if constexpr (kRefine) {
        const float rx = dmx * Wf, ry = dmy * Hf;
        v[6] += sqrtf(rx * rx + ry * ry) * p.refine_scale;
    }
    if constexpr (kDensify) {
        v[7] += p.dmap * w;
        v[11] += w;
    }
    v[8] += w * p.gx;
    v[9] += w * p.gy;
    v[10] += w * p.gz;
}

// Adds this pixel's contribution of Gaussian (m, co, c) to v; returns whether
// the Gaussian was blended at the pixel.
template <bool kRefine, bool kDensify>
__device__ __forceinline__ bool pixel_backward_step(PixBack& p, unsigned pos, float2 m, float4 co,
                                                    float4 c, float fx, float fy, float clip,
                                                    float Wf, float Hf, float (&v)[12]) {
    if (pos >= p.last)
        return false;
    const BlendEval e = blend_eval(pos, p.last, m, co, fx, fy, clip);
    if (!e.ok)
        return false;
    pixel_backward_finish<kRefine, kDensify>(p, e, co, c, Wf, Hf, v);
    return true;
}

// Per-pixel backward state of a vertical pixel pair, as float2 registers
// (the f32x2 operands of the pair adjoint).
struct PixPair {
    float2 T, sdot, gx, gy, gz, fin, rscale, dmap;
    unsigned la, lb;
};

__device__ __forceinline__ PixPair pix_pair(const PixBack& a, const PixBack& b) {
    PixPair p;
    p.T = f2(a.T, b.T);
    p.sdot = f2(a.sdot, b.sdot);
    p.gx = f2(a.gx, b.gx);
    p.gy = f2(a.gy, b.gy);
    p.gz = f2(a.gz, b.gz);
    p.fin = f2(a.fin_term, b.fin_term);
    p.rscale = f2(a.refine_scale, b.refine_scale);
    p.dmap = f2(a.dmap, b.dmap);
    p.la = a.last;
    p.lb = b.last;
    return p;
}

// pixel_backward_step for two vertically adjacent pixels at once: the
// per-pixel blend decisions (power, exp, alpha, floors) are the forward's
// scalar expressions, so both pixels skip exactly the Gaussians the forward
// skipped; the adjoint arithmetic then runs on float pairs (sm_100 f32x2
// instructions: one issue for both pixels). A pixel that does not blend the
// Gaussian takes G = alpha = 0 and 1 / (1 - alpha) = 1, which leaves its T and
// running sum unchanged and adds zero to every partial. acc holds per-pixel
// partial sums (x: first pixel, y: second).
template <bool kRefine, bool kDensify>
__device__ __forceinline__ bool pixel_backward_pair(PixPair& p, unsigned pos, float2 m, float4 co,
                                                    float4 c, float fx, float fya, float fyb,
                                                    float clip, float Wf, float Hf,
                                                    float2 (&acc)[12]) {
    if (pos >= p.la && pos >= p.lb)
        return false;
    const float dx = m.x - fx;
    const float xx = __fmul_rn(co.x, dx);
    const float nxy = -__fmul_rn(co.y, dx);
    const float2 dy = __fadd2_rn(f2s(m.y), f2(-fya, -fyb));
    const float2 yy = __fmul2_rn(__fmul2_rn(f2s(co.z), dy), dy);
    const float2 power = __fadd2_rn(__fmul2_rn(f2s(-0.5f), __ffma2_rn(f2s(dx), f2s(xx), yy)),
                                    __fmul2_rn(f2s(nxy), dy));
    const float Ea = expf(power.x), Eb = expf(power.y);
    const float2 og = __fmul2_rn(f2s(co.w), f2(Ea, Eb));
    const float a0 = fminf(clip, og.x), b0 = fminf(clip, og.y);
    const bool ha = pos < p.la && !(power.x > 0.f) && !(a0 < kAlphaFloor);
    const bool hb = pos < p.lb && !(power.y > 0.f) && !(b0 < kAlphaFloor);
    if (!(ha || hb))
        return false;
    const float2 G = f2(ha ? Ea : 0.f, hb ? Eb : 0.f);
    const float2 al = f2(ha ? a0 : 0.f, hb ? b0 : 0.f);
    // alpha = 0 (no blend) gives 1 / (1 - 0) = 1 exactly: no select needed.
    const float2 oma = __fadd2_rn(f2s(1.f), f2(-al.x, -al.y));
    const float2 inv = f2(1.f / oma.x, 1.f / oma.y);
    const float2 T = __fmul2_rn(p.T, inv);
    const float2 w = __fmul2_rn(al, T);
    const float2 cdot =
        __ffma2_rn(f2s(c.z), p.gz, __ffma2_rn(f2s(c.y), p.gy, __fmul2_rn(f2s(c.x), p.gx)));
    const float2 sf = __fadd2_rn(p.sdot, p.fin);
    const float2 dL_da = __ffma2_rn(T, cdot, __fmul2_rn(sf, f2(-inv.x, -inv.y)));
    p.sdot = __ffma2_rn(w, cdot, p.sdot);
    const float2 dL_dG = __fmul2_rn(f2s(co.w), dL_da);
    const float2 ddx = f2s(dx), ddy = dy;
    const float2 gdx = __fmul2_rn(G, ddx), gdy = __fmul2_rn(G, ddy);
    const float2 dmx =
        __fmul2_rn(dL_dG, __ffma2_rn(gdy, f2s(-co.y), __fmul2_rn(gdx, f2s(-co.x))));
    const float2 dmy =
        __fmul2_rn(dL_dG, __ffma2_rn(gdx, f2s(-co.y), __fmul2_rn(gdy, f2s(-co.z))));
    const float2 h = __fmul2_rn(dL_dG, f2s(-0.5f));
    acc[0] = __ffma2_rn(__fmul2_rn(gdx, ddx), h, acc[0]);
    acc[1] = __ffma2_rn(__fmul2_rn(gdx, ddy), h, acc[1]);
    acc[2] = __ffma2_rn(__fmul2_rn(gdy, ddy), h, acc[2]);
    acc[3] = __ffma2_rn(G, dL_da, acc[3]);
    acc[4] = __fadd2_rn(acc[4], dmx);
    acc[5] = __fadd2_rn(acc[5], dmy);
    if constexpr (kRefine) {
        const float2 rx = __fmul2_rn(dmx, f2s(Wf)), ry = __fmul2_rn(dmy, f2s(Hf));
        const float2 q = __ffma2_rn(ry, ry, __fmul2_rn(rx, rx));
        acc[6] = __ffma2_rn(f2(sqrtf(q.x), sqrtf(q.y)), p.rscale, acc[6]);
    }
    if constexpr (kDensify) {
        acc[7] = __ffma2_rn(p.dmap, w, acc[7]);
        acc[11] = __fadd2_rn(acc[11], w);
    }
    acc[8] = __ffma2_rn(w, p.gx, acc[8]);
    acc[9] = __ffma2_rn(w, p.gy, acc[9]);
    acc[10] = __ffma2_rn(w, p.gz, acc[10]);
    p.T = T;
    return true;
}

template <int B, typename S = TileStage<B>> struct BackStage {
    S s;
    float acc[B][12];
};

// Backward of tile (tx, ty). s_acc must be zero on entry and is zero on
// exit; s_wmax holds kWarps words. Per-instance gradients go to st.grad.
// kCount: counts into *pairs the (Gaussian, pixel) pairs the adjoint
// evaluates (the pixel's last contributor lies at or behind the Gaussian)
// and does nothing else.
template <int TW, int TH, int PX, bool kRefine, bool kDensify, bool kCount = false,
          typename Stage = TileStage<TileGeom<TW, TH, PX>::kBatch>>
__device__ __forceinline__ void composite_backward_tile(
    BackStage<TileGeom<TW, TH, PX>::kBatch, Stage>& sb, unsigned* s_wmax, int tx, int ty,
    uint2 range,
    const unsigned* __restrict__ order, const GaussianState& st, const ViewGrads& o,
    unsigned long long* __restrict__ pairs = nullptr, TmaGather* tma = nullptr) {
    using G = TileGeom<TW, TH, PX>;
    constexpr int B = G::kBatch;
    Stage& s = sb.s;
    TmaGather no_tma;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int px = tx * TW + (lane % TW);
    const int wx0 = tx * TW, wy0 = ty * TH + G::kBandRows * warp;
    const int py0 = wy0 + PX * (lane / TW);
    const float fx = float(px);
    const float clip = o.clip;
    const size_t P = size_t(o.width) * o.height;
    // Pixel pairs (even PX) keep their state as float2 registers.
    constexpr int NP = PX % 2 == 0 ? PX / 2 : 1;
    constexpr int NS = PX % 2 == 0 ? 1 : PX;
    PixBack pb[NS];
    PixPair pp[NP];
    unsigned wlast = 0;
#pragma unroll
    for (int p = 0; p < PX; ++p) {
        const bool inside = px < o.width && py0 + p < o.height;
        PixBack x;
        pixel_backward_init(x, inside, inside ? size_t(py0 + p) * o.width + px : 0, P, o.bg,
                            o.pix_T, o.pix_last, o.dL_color, o.dL_alpha, o.densify_map);
        wlast = max(wlast, x.last);
        if constexpr (PX % 2 == 0) {
            if (p & 1)
                pp[p / 2] = pix_pair(pb[0], x);
            else
                pb[0] = x;
        } else {
            pb[p] = x;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        wlast = max(wlast, __shfl_xor_sync(0xffffffffu, wlast, off));
    if (lane == 0)
        s_wmax[warp] = wlast;
    __syncthreads();
    unsigned tile_last = 0;
#pragma unroll
    for (int w = 0; w < G::kWarps; ++w)
        tile_last = max(tile_last, s_wmax[w]);
    tile_last = min(tile_last, range.y - range.x);
    const float Wf = float(o.width), Hf = float(o.height);
    const int batches = int((tile_last + B - 1) / B);
    unsigned long long evaluated = 0;
    for (int b = batches - 1; b >= 0; --b) {
        const int base = b * B;
        const int cnt = min(B, int(tile_last) - base);
        if (!stage_any<TW, TH, PX>(s, order, range.x + base, cnt, st, tid, tx * TW, ty * TH,
                                   tma ? *tma : no_tma))
            return;
        __syncthreads();
        const int jtop = min(cnt, int(wlast) - base) - 1;
        // Adds one Gaussian's partials (per lane) to its shared accumulator.
        auto reduce_add = [&](int j, bool hit, const float (&v)[12]) {
            const unsigned hits = __ballot_sync(0xffffffffu, hit);
            if (hits == 0)
                return;
            if (__popc(hits) == 1) {
                // A single contributing lane adds its partials directly.
                if (hit) {
#pragma unroll
                    for (int k = 0; k < 12; ++k)
                        if (v[k] != 0.f)
                            atomicAdd(&sb.acc[j][k], v[k]);
                }
                return;
            }
            int slot;
            const float r = kDensify ? reduce_scatter12(v, slot) : reduce_scatter10(v, slot);
            if (slot >= 0 && r != 0.f)
                atomicAdd(&sb.acc[j][slot], r);
        };
        if constexpr (PX == 1 && !kCount) {
            // One pixel per thread (frames with few tiles): two Gaussians per
            // step, back to front. Their blend evaluations (exponent,
            // opacity, floors) are independent and computed together; the
            // adjoints then run in order, the second on the transmittance the
            // first recovered (the same arithmetic as one per step).
            int j = jtop;
            for (;;) { // every loop condition is warp-uniform
                while (j >= 0 && !((s.band[j] >> warp) & 1u))
                    --j;
                if (j < 0)
                    break;
                int j2 = j - 1;
                while (j2 >= 0 && !((s.band[j2] >> warp) & 1u))
                    --j2;
                const bool two = j2 >= 0;
                const int jb = two ? j2 : j;
                const float fy = float(py0);
                const float2 m0 = s.xy_of(j), m1 = s.xy_of(jb);
                const float4 co0 = s.co_of(j), co1 = s.co_of(jb);
                const BlendEval e0 =
                    blend_eval(unsigned(base + j), pb[0].last, m0, co0, fx, fy, clip);
                const BlendEval e1 =
                    blend_eval(unsigned(base + jb), pb[0].last, m1, co1, fx, fy, clip);
                float v0[12], v1[12];
#pragma unroll
                for (int k = 0; k < 12; ++k)
                    v0[k] = v1[k] = 0.f;
                const bool hit0 = e0.ok, hit1 = two && e1.ok;
                if (hit0)
                    pixel_backward_finish<kRefine, kDensify>(pb[0], e0, co0, s.rgb_of(j), Wf,
                                                             Hf, v0);
                if (hit1)
                    pixel_backward_finish<kRefine, kDensify>(pb[0], e1, co1, s.rgb_of(jb), Wf,
                                                             Hf, v1);
                reduce_add(j, hit0, v0);
                if (two)
                    reduce_add(jb, hit1, v1);
                j = jb - 1;
            }
        } else
        for (int j = jtop; j >= 0; --j) {
            if (!((s.band[j] >> warp) & 1u))
                continue;
            const unsigned pos = unsigned(base + j);
            if constexpr (kCount) {
                if constexpr (PX % 2 == 0) {
#pragma unroll
                    for (int q = 0; q < NP; ++q)
                        evaluated += (pos < pp[q].la ? 1u : 0u) + (pos < pp[q].lb ? 1u : 0u);
                } else {
#pragma unroll
                    for (int p = 0; p < PX; ++p)
                        evaluated += pos < pb[p].last ? 1u : 0u;
                }
                continue;
            }
            const float2 m = s.xy_of(j);
            const float4 co = s.co_of(j);
            const float4 c = s.rgb_of(j);
            float v[12];
            bool hit = false;
            if constexpr (PX % 2 == 0) {
                float2 acc[12];
#pragma unroll
                for (int k = 0; k < 12; ++k)
                    acc[k] = f2s(0.f);
#pragma unroll
                for (int p = 0; p < PX; p += 2)
                    hit |= pixel_backward_pair<kRefine, kDensify>(
                        pp[p / 2], pos, m, co, c, fx, float(py0 + p), float(py0 + p + 1), clip,
                        Wf, Hf, acc);
#pragma unroll
                for (int k = 0; k < 12; ++k)
                    v[k] = acc[k].x + acc[k].y;
            } else {
#pragma unroll
                for (int k = 0; k < 12; ++k)
                    v[k] = 0.f;
#pragma unroll
                for (int p = 0; p < PX; ++p)
                    hit |= pixel_backward_step<kRefine, kDensify>(pb[p], pos, m, co, c, fx,
                                                                  float(py0 + p), clip, Wf, Hf,
                                                                  v);
            }
            reduce_add(j, hit, v);
        }
        __syncthreads();
        for (int k = tid; k < cnt; k += G::kThreads) {
            float* a = sb.acc[k];
            bool any = false;
#pragma unroll
            for (int q = 0; q < 12; ++q)
                any |= a[q] != 0.f;
            if (any) {
                float4* dst = st.grad + size_t(s.id[k]) * kGradSlots;
                atomicAdd(dst + 0, make_float4(a[0], a[1], a[2], a[3]));
                atomicAdd(dst + 1, make_float4(a[4], a[5], a[6], a[7]));
                atomicAdd(dst + 2, make_float4(a[8], a[9], a[10], a[11]));
#pragma unroll
                for (int q = 0; q < 12; ++q)
                    a[q] = 0.f;
            }
        }
        __syncthreads();
    }
    if constexpr (kCount)
        warp_count_add(evaluated, pairs);
}

} // namespace gsb
