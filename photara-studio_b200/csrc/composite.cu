// Single-view compositing kernels: one CTA per reference 16x16 tile running
// the per-tile forward / adjoint of composite.cuh (numerics and organisation
// described there; reference: third_party/splat_drender/src/render_forward.cu
// :341-416, :508-525 and render_backward.cu:156-519).
#include "composite.cuh"
#include "kernels.h"

namespace gsb {

// Single view: one CTA per reference 16x16 tile. kCount: the same forward
// that also counts its evaluated pairs into *pairs.
// The Gaussians of each batch are staged by TMA gathers of their 64-byte
// records (`map`: the record array as a [rows][16] float tensor).
template <int PX, bool kCount = false>
__global__ void __launch_bounds__(TileGeom<kTileW, kTileH, PX>::kThreads) composite_forward_kernel(
    const __grid_constant__ CUtensorMap map, unsigned* __restrict__ err,
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, float* __restrict__ out_color, float* __restrict__ out_alpha,
    float* __restrict__ pix_T, unsigned* __restrict__ pix_last, float* __restrict__ visibility,
    unsigned* __restrict__ tile_work, unsigned long long* __restrict__ pairs = nullptr) {
    using G = TileGeom<kTileW, kTileH, PX>;
    __shared__ RecStage<G::kBatch> s;
    __shared__ unsigned char s_vis[G::kBatch];
    for (int k = threadIdx.x; k < G::kBatch; k += G::kThreads)
        s_vis[k] = 0;
    if (threadIdx.x == 0)
        mbar_init(&s.bar, 1);
    __syncthreads();
    TmaGather g{&map, err, 0u};
    const int tile = blockIdx.x;
    const ViewTarget o{K.width, K.height, K.alpha_clip, bg, out_color, out_alpha, pix_T, pix_last};
    composite_forward_tile<kTileW, kTileH, PX, kCount>(s, s_vis, tile % K.grid_x,
                                                       tile / K.grid_x, ranges[tile], order, st,
                                                       o, visibility, pairs, &g,
                                                       tile_work ? tile_work + tile : nullptr);
}

// Four pixels per thread: capped at 96 registers (no spills) for 10 resident
// CTAs per SM instead of 8 (0.700 -> 0.684 ms at 1M Gaussians, 1080p; the
// 80-register cap for 12 CTAs spills and measured slower).
template <int PX, bool kRefine, bool kDensify, bool kCount = false>
__global__ void __launch_bounds__(TileGeom<kTileW, kTileH, PX>::kThreads, PX == 4 ? 10 : 1)
    composite_backward_kernel(
    const __grid_constant__ CUtensorMap map, unsigned* __restrict__ err,
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, const float* __restrict__ pix_T,
    const unsigned* __restrict__ pix_last, const float* __restrict__ dL_color,
    const float* __restrict__ dL_alpha, const float* __restrict__ densify_map,
    const unsigned* __restrict__ tile_order, unsigned long long* __restrict__ pairs = nullptr) {
    using G = TileGeom<kTileW, kTileH, PX>;
    using Stage = RecStage<G::kBatch>;
    __shared__ BackStage<G::kBatch, Stage> sb;
    __shared__ unsigned s_wmax[G::kWarps];
    for (int k = threadIdx.x; k < G::kBatch * 12; k += G::kThreads)
        (&sb.acc[0][0])[k] = 0.f;
    if (threadIdx.x == 0)
        mbar_init(&sb.s.bar, 1);
    __syncthreads();
    TmaGather g{&map, err, 0u};
    // heaviest tiles first (tile_order: tiles by descending adjoint work),
    // so the kernel's tail is made of the shortest tiles
    const int tile = tile_order ? int(tile_order[blockIdx.x]) : int(blockIdx.x);
    const ViewGrads o{K.width, K.height, K.alpha_clip, bg, pix_T, pix_last, dL_color, dL_alpha,
                      densify_map};
    composite_backward_tile<kTileW, kTileH, PX, kRefine, kDensify, kCount, Stage>(
        sb, s_wmax, tile % K.grid_x, tile / K.grid_x, ranges[tile], order, st, o, pairs, &g);
}

// Tiles by descending adjoint work (a permutation of [0, tiles) whatever the
// work values): one block, a counting sort on the work clamped to 4095.
__global__ void __launch_bounds__(1024) tile_order_kernel(const unsigned* __restrict__ work,
                                                          int tiles,
                                                          unsigned* __restrict__ order) {
    constexpr int kKeys = 4096;
    __shared__ unsigned s_cnt[kKeys];
    for (int k = threadIdx.x; k < kKeys; k += 1024)
        s_cnt[k] = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < tiles; t += 1024)
        atomicAdd(&s_cnt[kKeys - 1 - min(work[t], unsigned(kKeys - 1))], 1u);
    __syncthreads();
    // exclusive scan of the 4096 counts (descending work first), four per thread
    __shared__ unsigned s_warp[32];
    unsigned v[4], sum = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        v[q] = s_cnt[4 * threadIdx.x + q];
        sum += v[q];
    }
    const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= unsigned(off))
            incl += y;
    }
    if (lane == 31)
        s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        unsigned x = s_warp[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= unsigned(off))
                x += y;
        }
        s_warp[lane] = x;
    }
    __syncthreads();
    unsigned run = incl - sum + (w ? s_warp[w - 1] : 0u);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        s_cnt[4 * threadIdx.x + q] = run;
        run += v[q];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < tiles; t += 1024)
        order[atomicAdd(&s_cnt[kKeys - 1 - min(work[t], unsigned(kKeys - 1))], 1u)] = unsigned(t);
}

void launch_tile_order(cudaStream_t s, const unsigned* work, int tiles, unsigned* order) {
    if (tiles > 0)
        tile_order_kernel<<<1, 1024, 0, s>>>(work, tiles, order);
}

// Test hook for the staging wait: one CTA announces 256 bytes on its
// mbarrier that no copy delivers, waits at most `limit` suspended waits
// (as stage_any does), and reports the timeout as stage_any does.
__global__ void stage_probe_kernel(unsigned limit, unsigned* __restrict__ err) {
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0)
        mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0)
        mbar_arrive_expect_tx(&bar, 256u);
    const bool ok = mbar_wait_bounded(&bar, 0u, limit);
    if (__syncthreads_or(!ok) && threadIdx.x == 0)
        atomicOr(err, kDevStageTimeout);
}

void launch_stage_probe(cudaStream_t s, unsigned limit, unsigned* err) {
    stage_probe_kernel<<<1, 64, 0, s>>>(limit, err);
}

// Evaluated (Gaussian, pixel) pairs of the colour compositing forward and its
// adjoint for the last forward's draw list: pairs[0] forward, pairs[1]
// adjoint (zeroed by the caller). The forward pass re-renders into color /
// alpha (identical images); the adjoint count needs only the per-pixel last
// contributors.
void launch_composite_count_pairs(cudaStream_t s, int tiles, const uint2* ranges,
                                  const unsigned* order, const GaussianState& st,
                                  const Camera& K, float3 bg, float* color, float* alpha,
                                  const float* pix_T, const unsigned* pix_last,
                                  int pixels_per_thread, unsigned long long* pairs,
                                  const RecStaging& rs) {
    // the forward writes pix_T / pix_last again with identical values; the
    // count run leaves them as they were only if given the same buffers, so
    // it writes no per-pixel state (NULL) and no visibility
    auto count = [&]<int PX>() {
        constexpr int T = TileGeom<kTileW, kTileH, PX>::kThreads;
        composite_forward_kernel<PX, true><<<tiles, T, 0, s>>>(
            rs.map, rs.err, ranges, order, st, K, bg, color, alpha, nullptr, nullptr, nullptr,
            nullptr, pairs);
        composite_backward_kernel<PX, false, false, true><<<tiles, T, 0, s>>>(
            rs.map, rs.err, ranges, order, st, K, bg, pix_T, pix_last, color, nullptr, nullptr,
            nullptr, pairs + 1);
    };
    if (pixels_per_thread == 1)
        count.template operator()<1>();
    else if (pixels_per_thread == 2)
        count.template operator()<2>();
    else
        count.template operator()<4>();
}

// ------------------------------------------------- geometry channels ----
// Forward with the median-depth and normal channels (render_forward.cu
// :274-525, blend_tile<GEOMETRY = true>): one thread per pixel of a 16x16
// tile. Pass 1 is the colour forward (the same per-pixel arithmetic as the
// colour kernels, so colour, alpha, final transmittance and last contributor
// are bit-identical to them) plus the alpha-weighted footprint normal and the
// depth seed (the ray-plane depth of the last Gaussian blended while the
// transmittance was above 0.5). Pass 2 finds the depth at which the
// transmittance along the ray crosses 0.5: each Gaussian is a 1D Gaussian
// along the ray around its plane depth, and the pixel's transmittance at a
// probe depth is the product of the Gaussians' partial opacities there; 8
// probes over a +-0.4 window around the seed, refined 5 times (every
// refinement walks the tile's list up to the pixel's last contributor again),
// then linear interpolation inside the final bracket.
constexpr int kDepthSplit = 8;
constexpr int kDepthRefinements = 5;
constexpr float kDepthSeedWindow = 0.4f;
constexpr float kDepthMinTransmittance = 0.45f;
constexpr int kGeoThreads = kTileW * kTileH;

__global__ void __launch_bounds__(kGeoThreads) composite_geometry_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, float* __restrict__ out_color, float* __restrict__ out_alpha,
    float* __restrict__ pix_T, unsigned* __restrict__ pix_last, float* __restrict__ pix_dtdt,
    float* __restrict__ visibility, float* __restrict__ out_depth,
    float* __restrict__ out_normal) {
    __shared__ unsigned s_id[kGeoThreads];
    __shared__ float2 s_xy[kGeoThreads];
    __shared__ float4 s_co[kGeoThreads];
    __shared__ float4 s_rgb[kGeoThreads];
    __shared__ float4 s_plane[kGeoThreads];
    __shared__ float4 s_nrm[kGeoThreads];
    __shared__ unsigned s_warp[kGeoThreads / 32];
    const int tile = blockIdx.x;
    const int tx = tile % K.grid_x, ty = tile / K.grid_x;
    const int tid = threadIdx.x;
    const int px = tx * kTileW + tid % kTileW, py = ty * kTileH + tid / kTileW;
    const bool inside = px < K.width && py < K.height;
    const float fx = float(px), fy = float(py);
    const uint2 range = ranges[tile];
    const int n = int(range.y - range.x);
    const float clip = K.alpha_clip;

    // ---- pass 1: colour, alpha, normal, depth seed ----
    float T = 1.f, cr = 0.f, cg = 0.f, cb = 0.f;
    float nx = 0.f, ny = 0.f, nz = 0.f, seed = 0.f;
    unsigned last = 0;
    bool done = !inside;
    for (int base = 0; base < n; base += kGeoThreads) {
        if (__syncthreads_and(done))
            break;
        if (base + tid < n) {
            const unsigned g = order[range.x + base + tid];
            s_id[tid] = g;
            s_xy[tid] = st.mean2d[g];
            s_co[tid] = st.conic[g];
            s_rgb[tid] = st.rgb[g];
            s_plane[tid] = st.plane[g];
            s_nrm[tid] = st.normal[g];
        }
        __syncthreads();
        const int cnt = min(kGeoThreads, n - base);
        for (int j = 0; !done && j < cnt; ++j) {
            const float dx = s_xy[j].x - fx, dy = s_xy[j].y - fy;
            const float4 co = s_co[j];
            const float power = gaussian_power(co, dx, dy);
            if (power > 0.f)
                continue;
            const float alpha = fminf(clip, co.w * expf(power));
            if (alpha < kAlphaFloor)
                continue;
            const float test_t = T * (1.f - alpha);
            if (test_t < kTransmittanceFloor) {
                done = true;
                continue;
            }
            const float w = alpha * T;
            const float4 c = s_rgb[j];
            cr += c.x * w;
            cg += c.y * w;
            cb += c.z * w;
            const float4 rp = s_plane[j];
            const float4 nm = s_nrm[j];
            const float t = rp.x * dx + rp.y * dy + rp.z;
            nx += nm.x * w;
            ny += nm.y * w;
            nz += nm.z * w;
            seed = T > 0.5f ? t : seed;
            if (visibility)
                visibility[s_id[j]] = 1.f;
            T = test_t;
            last = unsigned(base + j + 1);
        }
    }
    // the tile's furthest last contributor bounds pass 2
    unsigned wmax = last;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, off));
    if ((tid & 31) == 0)
        s_warp[tid >> 5] = wmax;
    __syncthreads();
    unsigned block_max = 0;
#pragma unroll
    for (int w = 0; w < kGeoThreads / 32; ++w)
        block_max = max(block_max, s_warp[w]);

    // ---- pass 2: median-depth bisection ----
    constexpr int S = kDepthSplit;
    float depth_min = fmaxf(seed - kDepthSeedWindow, 0.f);
    float depth_max = fmaxf(seed + kDepthSeedWindow, 0.f);
    bool in_range = T <= kDepthMinTransmittance;
    float Tp[S + 1];
#pragma unroll
    for (int r = 0; r < kDepthRefinements; ++r) {
        const bool first = r == 0;
#pragma unroll
        for (int k = 0; k <= S; ++k)
            if (first || (k > 0 && k < S))
                Tp[k] = 1.f;
        const float interval = (depth_max - depth_min) * (1.f / float(S));
        bool ldone = !in_range;
        unsigned seen = 0;
        for (int base = 0; base < int(block_max); base += kGeoThreads) {
            if (__syncthreads_and(ldone))
                break;
            if (base + tid < int(block_max)) {
                const unsigned g = order[range.x + base + tid];
                s_xy[tid] = st.mean2d[g];
                s_co[tid] = st.conic[g];
                s_plane[tid] = st.plane[g];
            }
            __syncthreads();
            const int cnt = min(kGeoThreads, int(block_max) - base);
            for (int j = 0; !ldone && j < cnt; ++j) {
                ++seen;
                ldone = seen >= last;
                const float dx = s_xy[j].x - fx, dy = s_xy[j].y - fy;
                const float4 co = s_co[j];
                const float power = gaussian_power(co, dx, dy);
                if (power > 0.f)
                    continue;
                const float alpha = fminf(clip, co.w * expf(power));
                if (alpha < kAlphaFloor)
                    continue;
                const float4 rp = s_plane[j];
                const float t_peak = rp.x * dx + rp.y * dy + rp.z;
                const float rsigma = rp.w;
                const bool ball = rsigma > 0.f;
                // Beyond 8 sigma of the peak a probe's Gaussian factor is
                // exactly 0 in the product (alpha g < 2^-25, so 1 - alpha g
                // rounds to 1 and its inverse square root is 1): the probe
                // takes (1 - alpha) behind the peak and 1 in front of it. A
                // Gaussian whose peak is over 8 sigma behind every probe
                // changes nothing; one over 8 sigma in front scales all.
                const int k0 = first ? 0 : 1, k1 = first ? S : S - 1;
                const float d_lo = (depth_min + interval * float(k0) - t_peak) * rsigma;
                const float d_hi = (depth_min + interval * float(k1) - t_peak) * rsigma;
                if (ball && d_hi < -8.f)
                    continue;
                const float oma = 1.f - alpha;
                if (!ball || d_lo > 8.f) {
#pragma unroll
                    for (int k = 0; k <= S; ++k) {
                        if (!(first || (k > 0 && k < S)))
                            continue;
                        const float ts = depth_min + interval * float(k);
                        Tp[k] *= ts > t_peak ? oma : 1.f;
                    }
                    continue;
                }
#pragma unroll
                for (int k = 0; k <= S; ++k) {
                    if (!(first || (k > 0 && k < S)))
                        continue;
                    const float ts = depth_min + interval * float(k);
                    const float delta = (ts - t_peak) * rsigma;
                    if (delta * delta > 64.f) {
                        Tp[k] *= ts > t_peak ? oma : 1.f;
                        continue;
                    }
                    const float gk = expf(-0.5f * delta * delta);
                    const float omg = 1.f - alpha * gk;
                    const float rv = rsqrtf(omg);
                    Tp[k] *= (ts > t_peak ? oma : omg) * rv;
                }
            }
        }
        if (first)
            in_range = Tp[0] >= 0.5f && Tp[S] <= 0.5f && in_range;
        int start = 0;
#pragma unroll
        for (int k = 1; k < S; ++k)
            start = Tp[k] >= 0.5f ? k : start;
        // Tp indices are compile-time after unrolling: pick the bracket ends
        // with selects.
        float lo_T = Tp[0], hi_T = Tp[1];
#pragma unroll
        for (int k = 1; k < S; ++k) {
            lo_T = start == k ? Tp[k] : lo_T;
            hi_T = start == k ? Tp[k + 1] : hi_T;
        }
        depth_max = depth_min + float(start + 1) * interval;
        depth_min = depth_min + float(start + 0) * interval;
        Tp[0] = lo_T;
        Tp[S] = hi_T;
    }
    const float w_max = __saturatef((Tp[0] - 0.5f) / (Tp[0] - Tp[S]));
    const float w_min = 1.f - w_max;
    const float median = in_range ? w_max * depth_max + w_min * depth_min : 0.f;
    const float rln = pixel_ray_z(fx, fy, K);
    const float depth_out = median * rln;

    // ---- pass 3 (training forward only): dT/dt at the median depth ----
    // The derivative of the ray transmittance with respect to the median
    // distance, summed over the pixel's blended Gaussians:
    // -1/4 G_t / (1 - G_t) |delta| / sigma (render_backward.cu:47-151,
    // median_scale_walk, here evaluated where the median is found, at the
    // distance the backward recovers from the written depth). The backward
    // turns it into dL/dt with the depth gradient.
    float dTdt = 0.f;
    if (pix_dtdt) {
        const float mD = depth_out / fmaxf(rln, 1.0e-8f);
        bool ldone = !(inside && mD != 0.f && last != 0);
        unsigned seen = 0;
        for (int base = 0; base < int(block_max); base += kGeoThreads) {
            if (__syncthreads_and(ldone))
                break;
            if (base + tid < int(block_max)) {
                const unsigned g = order[range.x + base + tid];
                s_xy[tid] = st.mean2d[g];
                s_co[tid] = st.conic[g];
                s_plane[tid] = st.plane[g];
            }
            __syncthreads();
            const int cnt = min(kGeoThreads, int(block_max) - base);
            for (int j = 0; !ldone && j < cnt; ++j) {
                ++seen;
                ldone = seen >= last;
                const float dx = s_xy[j].x - fx, dy = s_xy[j].y - fy;
                const float4 co = s_co[j];
                const float power = gaussian_power(co, dx, dy);
                if (power > 0.f)
                    continue;
                const float alpha = fminf(clip, co.w * expf(power));
                if (alpha < kAlphaFloor)
                    continue;
                const float4 rp = s_plane[j];
                const float t_peak = rp.x * dx + rp.y * dy + rp.z;
                const float rsigma = rp.w;
                const float t_delta = (mD - t_peak) * rsigma;
                const float g_exp = expf(-0.5f * t_delta * t_delta);
                const float gt = alpha * g_exp;
                dTdt += -0.25f * gt / (1.f - gt) * fabsf(t_delta) * rsigma;
            }
        }
    }

    if (inside) {
        const size_t P = size_t(K.width) * K.height;
        const size_t pid = size_t(py) * K.width + px;
        out_color[pid] = cr + T * bg.x;
        out_color[P + pid] = cg + T * bg.y;
        out_color[2 * P + pid] = cb + T * bg.z;
        out_alpha[pid] = 1.f - T;
        if (pix_T) {
            pix_T[pid] = T;
            pix_last[pid] = last;
        }
        if (pix_dtdt)
            pix_dtdt[pid] = dTdt;
        out_depth[pid] = depth_out;
        const float len = 1.f - T;
        out_normal[pid] = last ? nx / len : 0.f;
        out_normal[P + pid] = last ? ny / len : 0.f;
        out_normal[2 * P + pid] = last ? nz / len : 0.f;
    }
}

void launch_composite_geometry(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, float* color, float* alpha, float* pix_T,
                               unsigned* pix_last, float* pix_dtdt, float* visibility,
                               float* median_depth, float* normal) {
    composite_geometry_kernel<<<tiles, kGeoThreads, 0, s>>>(ranges, order, st, K, bg, color,
                                                            alpha, pix_T, pix_last, pix_dtdt,
                                                            visibility, median_depth, normal);
}

// ------------------------------------------- geometry-channel adjoint ----
// Backward of the colour, median-depth and normal channels together
// (render_backward.cu:156-519, blend_bucket_backward<GEOMETRY = true>): one
// thread per pixel of a 16x16 tile walks its list back to front from its last
// contributor, recovering T by T_i = T_{i+1} / (1 - a_i) as the colour
// adjoint does. Per pixel it also carries the normal-output gradient divided
// by the rendered alpha (the normal output is the alpha-normalised sum), the
// running sum of the normals blended behind the current Gaussian projected on
// it, the median distance and dL/dt (the depth gradient over -dT/dt from the
// forward). Per (Gaussian, pixel) it adds, besides the colour terms: to
// dL/d opacity the normal term and the median term, to dL/d mean2d the ray
// plane's screen slope times dL/dt, and the gradients of the footprint normal
// (3) and of the ray plane (4). The refine weight takes the colour part of
// the mean2d gradient only, as the reference's. Twelve colour partials and
// seven geometry partials per Gaussian are reduced across the warp (two
// reduce-scatters), summed per tile in shared memory and added with five
// float4 atomics per (Gaussian, tile).
constexpr int kGeoBatch = kGeoThreads;

struct GeoBackStage {
    unsigned id[kGeoBatch];
    float2 xy[kGeoBatch];
    float4 co[kGeoBatch];
    float4 rgb[kGeoBatch];
    float4 plane[kGeoBatch];
    float4 nrm[kGeoBatch];
    unsigned char band[kGeoBatch];
    float acc[kGeoBatch][20]; // [0, 12) colour slots, [12, 16) ray plane, [16, 19) normal
};

// Reduce 8 per-lane values across the warp; returns the sum of slot `slot`
// (slot = -1 for lanes that hold a duplicate).
__device__ __forceinline__ float reduce_scatter8(const float (&v)[8], int& slot) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
    float u[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float send = b4 ? v[k] : v[k + 4];
        const float keep = b4 ? v[k + 4] : v[k];
        u[k] = keep + __shfl_xor_sync(full, send, 16);
    }
    float w[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float send = b3 ? u[k] : u[k + 2];
        const float keep = b3 ? u[k + 2] : u[k];
        w[k] = keep + __shfl_xor_sync(full, send, 8);
    }
    const float send = b2 ? w[0] : w[1];
    const float keep = b2 ? w[1] : w[0];
    float x = keep + __shfl_xor_sync(full, send, 4);
    x += __shfl_xor_sync(full, x, 2);
    x += __shfl_xor_sync(full, x, 1);
    slot = (lane & 3) ? -1 : (b4 ? 4 : 0) + (b3 ? 2 : 0) + (b2 ? 1 : 0);
    return x;
}

template <bool kRefine, bool kDensify>
__global__ void __launch_bounds__(kGeoThreads) composite_backward_geometry_kernel(
    const uint2* __restrict__ ranges, const unsigned* __restrict__ order, GaussianState st,
    const Camera K, float3 bg, const float* __restrict__ pix_T,
    const unsigned* __restrict__ pix_last, const float* __restrict__ pix_dtdt,
    const float* __restrict__ dL_color, const float* __restrict__ dL_alpha,
    const float* __restrict__ densify_map, const float* __restrict__ dL_depth,
    const float* __restrict__ dL_normal, const float* __restrict__ fwd_depth,
    const float* __restrict__ fwd_normal) {
    __shared__ GeoBackStage s;
    __shared__ unsigned s_wmax[kGeoThreads / 32];
    for (int k = threadIdx.x; k < kGeoBatch * 20; k += kGeoThreads)
        (&s.acc[0][0])[k] = 0.f;
    const int tile = blockIdx.x;
    const int tx = tile % K.grid_x, ty = tile / K.grid_x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int px = tx * kTileW + tid % kTileW, py = ty * kTileH + tid / kTileW;
    const bool inside = px < K.width && py < K.height;
    const float fx = float(px), fy = float(py);
    const uint2 range = ranges[tile];
    const float clip = K.alpha_clip;
    const size_t P = size_t(K.width) * K.height;
    const size_t pid = inside ? size_t(py) * K.width + px : 0;
    const bool with_depth = dL_depth != nullptr, with_normal = dL_normal != nullptr;

    // ---- per-pixel state ----
    float T_final = 1.f, gx = 0.f, gy = 0.f, gz = 0.f, gnx = 0.f, gny = 0.f, gnz = 0.f;
    float fin_r = 0.f, fin = 0.f, dmap = 0.f, mD = 0.f, dmt = 0.f;
    unsigned last = 0;
    if (inside) {
        T_final = pix_T[pid];
        last = pix_last[pid];
        gx = dL_color[pid];
        gy = dL_color[P + pid];
        gz = dL_color[2 * P + pid];
        const float dfin_r = bg.x * gx + bg.y * gy + bg.z * gz - (dL_alpha ? dL_alpha[pid] : 0.f);
        float dfin = dfin_r;
        if (with_normal) {
            // the normal output is the blended normal sum over alpha = 1 - T
            const float wf = 1.f - T_final;
            const float inv_w = wf > 0.f ? 1.f / wf : 0.f;
            gnx = dL_normal[pid] * inv_w;
            gny = dL_normal[P + pid] * inv_w;
            gnz = dL_normal[2 * P + pid] * inv_w;
            dfin += gnx * fwd_normal[pid] + gny * fwd_normal[P + pid] + gnz * fwd_normal[2 * P + pid];
        }
        if (with_depth) {
            const float rln = pixel_ray_z(fx, fy, K);
            mD = fwd_depth[pid] / fmaxf(rln, 1.0e-8f);
            dmt = dL_depth[pid] * rln / fmaxf(-pix_dtdt[pid], 1.0e-7f);
        }
        fin_r = T_final * dfin_r;
        fin = T_final * dfin;
        dmap = densify_map ? densify_map[pid] : 0.f;
    }
    const float refine_scale = 1.f / fmaxf(1.f - T_final, 1.0e-5f);
    float T = T_final, sdot = 0.f, ndot = 0.f;
    const float Wf = float(K.width), Hf = float(K.height);

    unsigned wlast = last;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        wlast = max(wlast, __shfl_xor_sync(0xffffffffu, wlast, off));
    if (lane == 0)
        s_wmax[warp] = wlast;
    __syncthreads();
    unsigned tile_last = 0;
#pragma unroll
    for (int w = 0; w < kGeoThreads / 32; ++w)
        tile_last = max(tile_last, s_wmax[w]);
    tile_last = min(tile_last, range.y - range.x);
    const int batches = int((tile_last + kGeoBatch - 1) / kGeoBatch);
    for (int b = batches - 1; b >= 0; --b) {
        const int base = b * kGeoBatch;
        const int cnt = min(kGeoBatch, int(tile_last) - base);
        if (tid < cnt) {
            const unsigned g = order[range.x + base + tid];
            s.id[tid] = g;
            s.xy[tid] = st.mean2d[g];
            s.co[tid] = st.conic[g];
            s.rgb[tid] = st.rgb[g];
            s.plane[tid] = st.plane[g];
            s.nrm[tid] = st.normal[g];
            const ushort4 bx = st.bounds[g];
            unsigned m = 0;
#pragma unroll
            for (int w = 0; w < kGeoThreads / 32; ++w)
                if (band_hit<kTileW, 2>(bx, tx * kTileW, ty * kTileH + 2 * w))
                    m |= 1u << w;
            s.band[tid] = static_cast<unsigned char>(m);
        }
        __syncthreads();
        const int jtop = min(cnt, int(wlast) - base) - 1;
        for (int j = jtop; j >= 0; --j) {
            if (!((s.band[j] >> warp) & 1u))
                continue;
            const unsigned pos = unsigned(base + j);
            float va[12], vg[8];
#pragma unroll
            for (int k = 0; k < 12; ++k)
                va[k] = 0.f;
#pragma unroll
            for (int k = 0; k < 8; ++k)
                vg[k] = 0.f;
            bool hit = false;
            if (pos < last) {
                const float2 m = s.xy[j];
                const float4 co = s.co[j];
                const float dx = m.x - fx, dy = m.y - fy;
                const float power = gaussian_power(co, dx, dy);
                const float G = expf(power);
                const float alpha = fminf(clip, co.w * G);
                hit = !(power > 0.f) && !(alpha < kAlphaFloor);
                if (hit) {
                    const float4 c = s.rgb[j];
                    const float inv_1ma = 1.f / (1.f - alpha);
                    T = T * inv_1ma; // transmittance in front of this Gaussian
                    const float w = alpha * T;
                    const float cdot = c.x * gx + c.y * gy + c.z * gz;
                    const float dL_da_r = T * cdot - (sdot + fin_r) * inv_1ma;
                    float dL_da = T * cdot - (sdot + fin) * inv_1ma;
                    sdot += w * cdot;
                    if (with_normal) {
                        const float4 n = s.nrm[j];
                        const float nd = n.x * gnx + n.y * gny + n.z * gnz;
                        dL_da += T * nd - ndot * inv_1ma;
                        ndot += w * nd;
                        vg[4] = w * gnx;
                        vg[5] = w * gny;
                        vg[6] = w * gnz;
                    }
                    const float4 rp = s.plane[j];
                    float dt = 0.f;
                    if (with_depth) {
                        const float t_peak = rp.x * dx + rp.y * dy + rp.z;
                        const float rsigma = rp.w;
                        const float t_delta = (mD - t_peak) * rsigma;
                        const float g_exp = expf(-0.5f * t_delta * t_delta);
                        const float gt = alpha * g_exp;
                        float dgt = dmt * 0.25f / (1.f - gt);
                        dgt = mD > t_peak ? dgt : -dgt;
                        dgt = rsigma > 0.f ? dgt : 0.f;
                        dL_da += dgt * g_exp - dmt * (t_delta > 0.f ? 0.5f * inv_1ma : 0.f);
                        const float ddelta = -dgt * gt * t_delta;
                        vg[3] = ddelta * (mD - t_peak);
                        dt = -ddelta * rsigma;
                        vg[0] = dt * dx;
                        vg[1] = dt * dy;
                        vg[2] = dt;
                    }
                    const float dL_dG = co.w * dL_da;
                    const float gdx = G * dx, gdy = G * dy;
                    const float dgx = -gdx * co.x - gdy * co.y;
                    const float dgy = -gdy * co.z - gdx * co.y;
                    va[0] = -0.5f * gdx * dx * dL_dG;
                    va[1] = -0.5f * gdx * dy * dL_dG;
                    va[2] = -0.5f * gdy * dy * dL_dG;
                    va[3] = G * dL_da;
                    va[4] = dL_dG * dgx + dt * rp.x;
                    va[5] = dL_dG * dgy + dt * rp.y;
                    if constexpr (kRefine) {
                        const float dL_dG_r = co.w * dL_da_r;
                        const float rx = dL_dG_r * dgx * Wf, ry = dL_dG_r * dgy * Hf;
                        va[6] = sqrtf(rx * rx + ry * ry) * refine_scale;
                    }
                    if constexpr (kDensify) {
                        va[7] = dmap * w;
                        va[11] = w;
                    }
                    va[8] = w * gx;
                    va[9] = w * gy;
                    va[10] = w * gz;
                }
            }
            const unsigned hits = __ballot_sync(0xffffffffu, hit);
            if (hits == 0)
                continue;
            if (__popc(hits) == 1) {
                if (hit) {
#pragma unroll
                    for (int k = 0; k < 12; ++k)
                        if (va[k] != 0.f)
                            atomicAdd(&s.acc[j][k], va[k]);
#pragma unroll
                    for (int k = 0; k < 7; ++k)
                        if (vg[k] != 0.f)
                            atomicAdd(&s.acc[j][12 + k], vg[k]);
                }
                continue;
            }
            int slot;
            const float ra = reduce_scatter12(va, slot);
            if (slot >= 0 && ra != 0.f)
                atomicAdd(&s.acc[j][slot], ra);
            const float rg = reduce_scatter8(vg, slot);
            if (slot >= 0 && slot < 7 && rg != 0.f)
                atomicAdd(&s.acc[j][12 + slot], rg);
        }
        __syncthreads();
        if (tid < cnt) {
            float* a = s.acc[tid];
            bool any = false;
#pragma unroll
            for (int q = 0; q < 19; ++q)
                any |= a[q] != 0.f;
            if (any) {
                const size_t g = s.id[tid];
                float4* dst = st.grad + g * kGradSlots;
                atomicAdd(dst + 0, make_float4(a[0], a[1], a[2], a[3]));
                atomicAdd(dst + 1, make_float4(a[4], a[5], a[6], a[7]));
                atomicAdd(dst + 2, make_float4(a[8], a[9], a[10], a[11]));
                float4* gdst = st.geo_grad + g * kGeoGradSlots;
                atomicAdd(gdst + 0, make_float4(a[12], a[13], a[14], a[15]));
                atomicAdd(gdst + 1, make_float4(a[16], a[17], a[18], 0.f));
#pragma unroll
                for (int q = 0; q < 19; ++q)
                    a[q] = 0.f;
            }
        }
        __syncthreads();
    }
}

void launch_composite_backward_geometry(cudaStream_t s, int tiles, const uint2* ranges,
                                        const unsigned* order, const GaussianState& st,
                                        const Camera& K, float3 bg, const float* pix_T,
                                        const unsigned* pix_last, const float* pix_dtdt,
                                        const float* dL_color, const float* dL_alpha,
                                        const float* densify_map, int want_refine,
                                        const float* dL_depth, const float* dL_normal,
                                        const float* fwd_depth, const float* fwd_normal) {
#define GSB_GEO_BWD(R, D)                                                                        \
    composite_backward_geometry_kernel<R, D><<<tiles, kGeoThreads, 0, s>>>(                      \
        ranges, order, st, K, bg, pix_T, pix_last, pix_dtdt, dL_color, dL_alpha, densify_map,    \
        dL_depth, dL_normal, fwd_depth, fwd_normal)
    if (want_refine && densify_map) GSB_GEO_BWD(true, true);
    else if (want_refine) GSB_GEO_BWD(true, false);
    else if (densify_map) GSB_GEO_BWD(false, true);
    else GSB_GEO_BWD(false, false);
#undef GSB_GEO_BWD
}

void launch_composite_forward(cudaStream_t s, int tiles, const uint2* ranges,
                              const unsigned* order, const GaussianState& st, const Camera& K,
                              float3 bg, float* color, float* alpha, float* pix_T,
                              unsigned* pix_last, float* visibility, int pixels_per_thread,
                              const RecStaging& rs, unsigned* tile_work) {
    auto fwd = [&]<int PX>() {
        composite_forward_kernel<PX><<<tiles, TileGeom<kTileW, kTileH, PX>::kThreads, 0, s>>>(
            rs.map, rs.err, ranges, order, st, K, bg, color, alpha, pix_T, pix_last, visibility,
            tile_work);
    };
    if (pixels_per_thread == 1)
        fwd.template operator()<1>();
    else if (pixels_per_thread == 2)
        fwd.template operator()<2>();
    else if (pixels_per_thread == 8)
        fwd.template operator()<8>();
    else
        fwd.template operator()<4>();
}

template <int PX>
static void launch_backward_px(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, const float* pix_T, const unsigned* pix_last,
                               const float* dL_color, const float* dL_alpha,
                               const float* densify_map, int want_refine,
                               const RecStaging& rs, const unsigned* tile_order) {
    const int T = TileGeom<kTileW, kTileH, PX>::kThreads;
#define GSB_BWD(R, D)                                                                            \
    composite_backward_kernel<PX, R, D><<<tiles, T, 0, s>>>(rs.map, rs.err, ranges, order, st,   \
                                                            K, bg, pix_T, pix_last, dL_color,    \
                                                            dL_alpha, densify_map, tile_order)
    if (want_refine && densify_map) GSB_BWD(true, true);
    else if (want_refine) GSB_BWD(true, false);
    else if (densify_map) GSB_BWD(false, true);
    else GSB_BWD(false, false);
#undef GSB_BWD
}

void launch_composite_backward(cudaStream_t s, int tiles, const uint2* ranges,
                               const unsigned* order, const GaussianState& st, const Camera& K,
                               float3 bg, const float* pix_T, const unsigned* pix_last,
                               const float* dL_color, const float* dL_alpha,
                               const float* densify_map, int want_refine, int pixels_per_thread,
                               const RecStaging& rs, const unsigned* tile_order) {
    if (pixels_per_thread == 1)
        launch_backward_px<1>(s, tiles, ranges, order, st, K, bg, pix_T, pix_last, dL_color,
                              dL_alpha, densify_map, want_refine, rs,
                              tile_order);
    else if (pixels_per_thread == 2)
        launch_backward_px<2>(s, tiles, ranges, order, st, K, bg, pix_T, pix_last, dL_color,
                              dL_alpha, densify_map, want_refine, rs,
                              tile_order);
    else if (pixels_per_thread == 8)
        launch_backward_px<8>(s, tiles, ranges, order, st, K, bg, pix_T, pix_last, dL_color,
                              dL_alpha, densify_map, want_refine, rs,
                              tile_order);
    else
        launch_backward_px<4>(s, tiles, ranges, order, st, K, bg, pix_T, pix_last, dL_color,
                              dL_alpha, densify_map, want_refine, rs,
                              tile_order);
}

} // namespace gsb
