// Batched multi-view rasterization: many camera views of uneven resolution in
// one launch per stage, the whole forward + backward capturable into one CUDA
// graph (no host synchronisation and no allocation after planning).
//
// Per-view semantics are those of the single-view path (preprocess, draw
// order (tile, depth, index), front-to-back compositing, reverse adjoint); the
// per-Gaussian gradients are the sums over views. Layout in HBM:
//   pair (v, i) -> slot v * N + i of every per-Gaussian state array;
//   global tile id = tile_base[v] + local tile; images concatenated per view
//   (colour planar [3][H_v][W_v] at 3 * pix_base[v], alpha at pix_base[v]).
// Stages (each one launch over all views):
//   1 preprocess over (view, Gaussian) pairs, depth keys in the same pass;
//   2 onesweep sort of the pairs by depth bits (one global order: within a
//     view it is that view's depth order, ties by index);
//   3 look-back scan of tile counts in depth order;
//   4 duplicate-with-keys in depth order with global tile ids as keys;
//   5 onesweep sort of the instances on the tile-id bits (stable), instance
//     count read on the device (capacity-sized grids);
//   6 tile ranges; optional tile ordering by cost (heaviest first);
//   7 persistent compositing kernel: each CTA pulls tiles of any view
//     (static stride, a dynamic queue, or the cost order) and runs the shared
//     per-tile body of composite.cuh for the planned tile shape;
//   8 persistent compositing adjoint, same schedule;
//   9 per-Gaussian adjoint looping over the views in registers (one write of
//     each summed gradient, no atomics).
// The tile shape (8x8, 16x16, 16x32), pixels per thread and schedule are plan
// parameters; gs_batch_autotune times the candidates and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/gsplat_b200.h"
#include "adjoint.cuh"
#include "composite.cuh"
#include "emit.cuh"
#include "host.h"
#include "kernels.h"
#include "preprocess.cuh"

using namespace gsb;
using namespace gsb::host;

namespace gsb {

struct BatchView {
    Camera K;           // grid_x / grid_y in the batch tile shape
    unsigned tile_base; // first global tile of the view
    unsigned pix_base;  // first pixel of the view in the concatenated images
};

enum BatchCounter : int {
    kBcInstances = 0, // unused (the instance count is the 64-bit word kBcInstances64)
    kBcVisible = 1,
    kBcErr = 2,
    kBcWork = 3,      // dynamic tile queue (forward)
    kBcWorkBack = 4,  // dynamic tile queue (backward)
    kBcPairs = 5,     // V * N (count for the depth sort)
    kBcTotal = 6,     // scan total
    kBcSorted = 7,    // min(instances, capacity): count for the tile sort
    kBcTiles = 8,     // total tiles (count for the cost sort)
    kBcInstances64 = 10, // words 10-11: instances requested by the preprocess (u64)
    kBcWords = 16
};

// ------------------------------------------------------------- stage 1 --
template <int TW, int TH>
__global__ void __launch_bounds__(kBlock) batch_preprocess_kernel(
    int n, const float* __restrict__ means, const float* __restrict__ log_scales,
    const float* __restrict__ quats, const float* __restrict__ logits,
    const float* __restrict__ filter_3d, const float* __restrict__ sh,
    const float* __restrict__ colors, int sh_degree, int sh_bases,
    const BatchView* __restrict__ views, GaussianState st, int* __restrict__ radii,
    unsigned* __restrict__ dkeys, unsigned* __restrict__ dvals, unsigned* __restrict__ counters) {
    __shared__ Camera sK;
    const int v = blockIdx.y;
    constexpr int kWords = int(sizeof(Camera) / 4);
    for (int k = threadIdx.x; k < kWords; k += blockDim.x)
        reinterpret_cast<unsigned*>(&sK)[k] = reinterpret_cast<const unsigned*>(&views[v].K)[k];
    // Frame totals: per warp, then per block in shared memory, then one pair
    // of global atomics per block (same-address atomics per warp serialise).
    __shared__ unsigned long long s_inst;
    __shared__ unsigned s_vis;
    if (threadIdx.x == 0) {
        s_inst = 0;
        s_vis = 0;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned touched = 0;
    if (i < n) {
        const size_t slot = size_t(v) * size_t(n) + size_t(i);
        const PreResult r = preprocess_one<TW, TH>(i, slot, means, log_scales, quats, logits,
                                                   filter_3d, sh, colors, sh_degree, sh_bases, sK,
                                                   st);
        touched = r.touched;
        st.touched[slot] = r.touched;
        radii[slot] = r.radius;
        dkeys[slot] = r.touched > 0 ? r.depth_bits : 0xffffffffu;
        dvals[slot] = unsigned(slot);
    }
    const unsigned w_inst = __reduce_add_sync(0xffffffffu, touched);
    const unsigned w_vis = __popc(__ballot_sync(0xffffffffu, touched > 0));
    if (lane_id() == 0 && w_vis) {
        atomicAdd(&s_inst, static_cast<unsigned long long>(w_inst));
        atomicAdd(&s_vis, w_vis);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_vis) {
        atomicAdd(reinterpret_cast<unsigned long long*>(counters + kBcInstances64), s_inst);
        atomicAdd(&counters[kBcVisible], s_vis);
    }
}

// Device-side counts for the sorts: the pairs and tiles (fixed by the plan)
// and the instance count clamped to the capacity (flagging an overflow), so
// every later stage sizes itself on the device.
__global__ void batch_counts_kernel(unsigned* __restrict__ counters, unsigned capacity,
                                    unsigned pairs, unsigned tiles) {
    const unsigned long long want =
        *reinterpret_cast<const unsigned long long*>(counters + kBcInstances64);
    counters[kBcSorted] = want < capacity ? unsigned(want) : capacity;
    counters[kBcPairs] = pairs;
    counters[kBcTiles] = tiles;
    if (want > capacity)
        atomicOr(&counters[kBcErr], kDevCapacity);
}

// ------------------------------------------------------------- stage 4 --
// Duplicate-with-keys as the single-view emit: warps take the visible pairs
// in depth order in groups of about 2^group_shift instances (cut by the
// offset scan) and expand their span records (emit_warp_range), with global
// tile ids as keys. The group count comes from the scan total and the range
// of the last group ends at the visible count, both on the device.
constexpr int kBatchEmitBlock = 256;

template <int TW, int TH>
__global__ void __launch_bounds__(kBatchEmitBlock) batch_emit_kernel(
    int n, const unsigned* __restrict__ counters, const unsigned* __restrict__ groups,
    int group_shift, unsigned group_cap, const unsigned* __restrict__ order, GaussianState st,
    const BatchView* __restrict__ views, unsigned* __restrict__ keys, unsigned* __restrict__ vals,
    unsigned capacity) {
    __shared__ uint4 s_col[kBatchEmitBlock / 32][32 * kSpanCols];
    const int warp = int(threadIdx.x >> 5);
    const unsigned total = counters[kBcTotal];
    const int visible = int(counters[kBcVisible]);
    const unsigned group_count =
        min(unsigned((size_t(total) + (size_t(1) << group_shift) - 1) >> group_shift), group_cap);
    const unsigned g = blockIdx.x * (kBatchEmitBlock / 32) + unsigned(warp);
    if (g >= group_count)
        return; // warp-uniform; the kernel has no block-wide barrier
    const int r_begin = int(groups[g]);
    const int r_end = g + 1 < group_count ? int(groups[g + 1]) : visible;
    emit_warp_range<TW, TH>(
        r_begin, r_end, order, st, [&](unsigned p) { return __ldg(&st.spans[p]); },
        [&](unsigned p) {
            const BatchView& v = views[p / unsigned(n)];
            return EmitView{v.K.grid_x, v.K.grid_y, v.tile_base};
        },
        keys, vals, capacity, s_col[warp], [](unsigned) {});
}

// ------------------------------------------------------------- stage 6 --
__global__ void __launch_bounds__(kBlock) batch_ranges_kernel(const unsigned* __restrict__ counters,
                                                              const unsigned* __restrict__ keys,
                                                              uint2* __restrict__ ranges,
                                                              unsigned tiles) {
    const unsigned count = counters[kBcSorted];
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    const unsigned tile = keys[i];
    if (i == 0) {
        if (tile < tiles)
            ranges[tile].x = 0;
    } else {
        const unsigned prev = keys[i - 1];
        if (tile != prev) {
            if (prev < tiles)
                ranges[prev].y = i;
            if (tile < tiles)
                ranges[tile].x = i;
        }
    }
    if (i == count - 1 && tile < tiles)
        ranges[tile].y = count;
}

// Heaviest-first order: 16-bit inverted instance counts, sorted stably.
__global__ void __launch_bounds__(kBlock) batch_tile_cost_kernel(unsigned tiles,
                                                                 const uint2* __restrict__ ranges,
                                                                 unsigned* __restrict__ keys,
                                                                 unsigned* __restrict__ vals) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles)
        return;
    const uint2 r = ranges[t];
    const unsigned len = r.y > r.x ? r.y - r.x : 0u;
    keys[t] = 0xffffu - (len < 0xffffu ? len : 0xffffu);
    vals[t] = t;
}

// --------------------------------------------------------- stages 7 / 8 --
enum BatchSchedule : int { kSchedStatic = 0, kSchedDynamic = 1, kSchedHeavyFirst = 2 };

struct TileLookup {
    const BatchView* views;
    const unsigned short* tile_view;
    const unsigned* tile_order; // heaviest-first permutation (schedule 2)
};

// Next tile of this CTA (uniform across the CTA), or >= tiles when done.
template <int SCHED>
__device__ __forceinline__ unsigned next_tile(unsigned& k, unsigned tiles, unsigned* queue,
                                              unsigned* s_item, const TileLookup& L) {
    unsigned item;
    if constexpr (SCHED == kSchedStatic) {
        __syncthreads();
        item = blockIdx.x + k * gridDim.x;
        ++k;
    } else {
        if (threadIdx.x == 0)
            *s_item = atomicAdd(queue, 1u);
        __syncthreads();
        item = *s_item;
        __syncthreads();
    }
    if (item >= tiles)
        return item;
    return SCHED == kSchedHeavyFirst ? L.tile_order[item] : item;
}

template <int TW, int TH, int PX, int SCHED>
__global__ void __launch_bounds__(TileGeom<TW, TH, PX>::kThreads) batch_forward_kernel(
    unsigned tiles, const uint2* __restrict__ ranges, const unsigned* __restrict__ order,
    GaussianState st, TileLookup L, unsigned* __restrict__ queue, float3 bg,
    float* __restrict__ color, float* __restrict__ alpha, float* __restrict__ pix_T,
    unsigned* __restrict__ pix_last) {
    using G = TileGeom<TW, TH, PX>;
    __shared__ TileStage<G::kBatch> s;
    __shared__ unsigned char s_vis[G::kBatch];
    __shared__ unsigned s_item;
    for (int k = threadIdx.x; k < G::kBatch; k += G::kThreads)
        s_vis[k] = 0;
    unsigned k = 0;
    for (;;) {
        const unsigned tile = next_tile<SCHED>(k, tiles, queue, &s_item, L);
        if (tile >= tiles)
            break;
        const unsigned v = L.tile_view[tile];
        const BatchView& bv = L.views[v];
        const int gx = bv.K.grid_x;
        const unsigned local = tile - bv.tile_base;
        const size_t pb = bv.pix_base;
        const ViewTarget o{bv.K.width, bv.K.height, bv.K.alpha_clip, bg, color + 3 * pb,
                           alpha + pb, pix_T + pb, pix_last + pb};
        composite_forward_tile<TW, TH, PX>(s, s_vis, int(local % unsigned(gx)),
                                           int(local / unsigned(gx)), ranges[tile], order, st, o,
                                           nullptr);
    }
}

template <int TW, int TH, int PX, int SCHED>
__global__ void __launch_bounds__(TileGeom<TW, TH, PX>::kThreads) batch_backward_kernel(
    unsigned tiles, const uint2* __restrict__ ranges, const unsigned* __restrict__ order,
    GaussianState st, TileLookup L, unsigned* __restrict__ queue, float3 bg,
    const float* __restrict__ pix_T, const unsigned* __restrict__ pix_last,
    const float* __restrict__ dL_color, const float* __restrict__ dL_alpha) {
    using G = TileGeom<TW, TH, PX>;
    __shared__ BackStage<G::kBatch> sb;
    __shared__ unsigned s_wmax[G::kWarps];
    __shared__ unsigned s_item;
    for (int k = threadIdx.x; k < G::kBatch * 12; k += G::kThreads)
        (&sb.acc[0][0])[k] = 0.f;
    unsigned k = 0;
    for (;;) {
        const unsigned tile = next_tile<SCHED>(k, tiles, queue, &s_item, L);
        if (tile >= tiles)
            break;
        const unsigned v = L.tile_view[tile];
        const BatchView& bv = L.views[v];
        const int gx = bv.K.grid_x;
        const unsigned local = tile - bv.tile_base;
        const size_t pb = bv.pix_base;
        const ViewGrads o{bv.K.width,  bv.K.height,
                          bv.K.alpha_clip, bg,
                          pix_T + pb,  pix_last + pb,
                          dL_color + 3 * pb, dL_alpha ? dL_alpha + pb : nullptr,
                          nullptr};
        composite_backward_tile<TW, TH, PX, true, false>(sb, s_wmax, int(local % unsigned(gx)),
                                                         int(local / unsigned(gx)), ranges[tile],
                                                         order, st, o);
    }
}

// ------------------------------------------------------------- stage 9 --
constexpr int kBGBlock = 128;
constexpr int kBShStride = 49;

// One thread per Gaussian; loops over the views that saw it, summing the
// projection and SH adjoints in registers / its shared SH row, then writes
// each gradient once (accumulating into the caller's buffers). Consumes and
// re-zeroes the per-pair gradient slots.
__global__ void __launch_bounds__(kBGBlock) batch_gaussian_backward_kernel(
    int n, int views, const float* __restrict__ means, const float* __restrict__ log_scales,
    const float* __restrict__ quats, const float* __restrict__ logits,
    const float* __restrict__ filter_3d, const float* __restrict__ sh, int sh_degree,
    int sh_bases, const BatchView* __restrict__ bviews, GaussianState st,
    const int* __restrict__ radii, GradOutArgs out) {
    extern __shared__ float smem[];
    Camera* sK = reinterpret_cast<Camera*>(smem);
    float* s_acc = smem + views * int(sizeof(Camera) / 4); // [kBGBlock][kBShStride]
    float* s_tmp = s_acc + kBGBlock * kBShStride;          // [kBGBlock][kBShStride]
    constexpr int kWords = int(sizeof(Camera) / 4);
    for (int k = threadIdx.x; k < views * kWords; k += kBGBlock) {
        const int v = k / kWords, w = k - v * kWords;
        reinterpret_cast<unsigned*>(sK)[k] = reinterpret_cast<const unsigned*>(&bviews[v].K)[w];
    }
    __syncthreads();
    const int i = blockIdx.x * kBGBlock + threadIdx.x;
    if (i >= n)
        return;
    const int stride = sh ? sh_bases * 3 : 0;
    float* acc = s_acc + threadIdx.x * kBShStride;
    float* tmp = s_tmp + threadIdx.x * kBShStride;
    for (int c = 0; c < stride; ++c)
        acc[c] = 0.f;
    const float3 mean = make_float3(means[3 * i], means[3 * i + 1], means[3 * i + 2]);
    const Activated act = activate(log_scales, quats, logits, filter_3d, i);
    ProjGrad sum;
    sum.d_mean = make_float3(0.f, 0.f, 0.f);
    sum.d_scale = make_float3(0.f, 0.f, 0.f);
    sum.d_rot = make_float4(0.f, 0.f, 0.f, 0.f);
    sum.d_opac = 0.f;
    float3 dcol_sum = make_float3(0.f, 0.f, 0.f);
    float refine = 0.f;
    bool any = false;
    for (int v = 0; v < views; ++v) {
        const size_t slot = size_t(v) * size_t(n) + size_t(i);
        if (radii[slot] <= 0)
            continue;
        any = true;
        float4* gslot = st.grad + slot * kGradSlots;
        const float4 g0 = gslot[0], g1 = gslot[1], g2 = gslot[2];
        gslot[0] = make_float4(0.f, 0.f, 0.f, 0.f);
        gslot[1] = make_float4(0.f, 0.f, 0.f, 0.f);
        gslot[2] = make_float4(0.f, 0.f, 0.f, 0.f);
        const Camera& K = sK[v];
        const ProjGrad pg =
            projection_backward(mean, K, act.scale, act.rot, g0, make_float2(g1.x, g1.y));
        sum.d_mean.x += pg.d_mean.x;
        sum.d_mean.y += pg.d_mean.y;
        sum.d_mean.z += pg.d_mean.z;
        sum.d_scale.x += pg.d_scale.x;
        sum.d_scale.y += pg.d_scale.y;
        sum.d_scale.z += pg.d_scale.z;
        sum.d_rot.x += pg.d_rot.x;
        sum.d_rot.y += pg.d_rot.y;
        sum.d_rot.z += pg.d_rot.z;
        sum.d_rot.w += pg.d_rot.w;
        sum.d_opac += pg.d_opac;
        refine += g1.z;
        const float3 dcol = make_float3(g2.x, g2.y, g2.z);
        if (sh) {
            const unsigned clamp_bits = __float_as_uint(st.rgb[slot].w);
            const float3 dm = sh_color_backward(
                reinterpret_cast<const float3*>(sh) + size_t(i) * sh_bases, sh_degree, sh_bases,
                mean, make_float3(K.center[0], K.center[1], K.center[2]), clamp_bits, dcol,
                reinterpret_cast<float3*>(tmp));
            sum.d_mean.x += dm.x;
            sum.d_mean.y += dm.y;
            sum.d_mean.z += dm.z;
            for (int c = 0; c < stride; ++c)
                acc[c] += tmp[c];
        } else {
            dcol_sum.x += dcol.x;
            dcol_sum.y += dcol.y;
            dcol_sum.z += dcol.z;
        }
    }
    if (!any)
        return;
    if (sh && out.sh)
        for (int c = 0; c < stride; ++c)
            out.sh[size_t(i) * stride + c] += acc[c];
    if (!sh && out.colors) {
        out.colors[3 * i + 0] += dcol_sum.x;
        out.colors[3 * i + 1] += dcol_sum.y;
        out.colors[3 * i + 2] += dcol_sum.z;
    }
    if (out.refine_weight)
        out.refine_weight[i] += refine;
    if (out.means) {
        out.means[3 * i + 0] += sum.d_mean.x;
        out.means[3 * i + 1] += sum.d_mean.y;
        out.means[3 * i + 2] += sum.d_mean.z;
    }
    if (out.activated) {
        if (out.scales) {
            out.scales[3 * i + 0] += sum.d_scale.x;
            out.scales[3 * i + 1] += sum.d_scale.y;
            out.scales[3 * i + 2] += sum.d_scale.z;
        }
        if (out.rotations) {
            out.rotations[4 * i + 0] += sum.d_rot.x;
            out.rotations[4 * i + 1] += sum.d_rot.y;
            out.rotations[4 * i + 2] += sum.d_rot.z;
            out.rotations[4 * i + 3] += sum.d_rot.w;
        }
        if (out.opacities)
            out.opacities[i] += sum.d_opac;
    } else {
        const RawGrad rg = chain_to_raw(sum, act, quats, logits, filter_3d, i);
        if (out.scales)
            for (int k = 0; k < 3; ++k) out.scales[3 * i + k] += rg.log_s[k];
        if (out.rotations)
            for (int k = 0; k < 4; ++k) out.rotations[4 * i + k] += rg.quat[k];
        if (out.opacities)
            out.opacities[i] += rg.logit;
    }
}

size_t batch_gaussian_backward_smem(int views) {
    return size_t(views) * sizeof(Camera) + size_t(2) * kBGBlock * kBShStride * sizeof(float);
}

} // namespace gsb

// ------------------------------------------------------------------ host --
namespace {

struct Shape {
    int tw, th, ppt;
};

bool valid_shape(int tw, int th, int ppt) {
    if (tw == 8 && th == 8) return ppt == 1 || ppt == 2;
    if (tw == 16 && th == 16) return ppt == 2 || ppt == 4;
    if (tw == 16 && th == 32) return ppt == 2 || ppt == 4;
    return false;
}

// Dispatch a lambda templated on <TW, TH> / <TW, TH, PX> to the compiled variants.
template <typename F> void with_tile(int tw, int th, F&& f) {
    if (tw == 8 && th == 8) f.template operator()<8, 8>();
    else if (tw == 16 && th == 16) f.template operator()<16, 16>();
    else if (tw == 16 && th == 32) f.template operator()<16, 32>();
    else throw InvalidArg("gsplat_b200: unsupported batch tile shape");
}

template <typename F> void with_shape(int tw, int th, int ppt, F&& f) {
    if (tw == 8 && th == 8 && ppt == 1) f.template operator()<8, 8, 1>();
    else if (tw == 8 && th == 8 && ppt == 2) f.template operator()<8, 8, 2>();
    else if (tw == 16 && th == 16 && ppt == 2) f.template operator()<16, 16, 2>();
    else if (tw == 16 && th == 16 && ppt == 4) f.template operator()<16, 16, 4>();
    else if (tw == 16 && th == 32 && ppt == 2) f.template operator()<16, 32, 2>();
    else if (tw == 16 && th == 32 && ppt == 4) f.template operator()<16, 32, 4>();
    else throw InvalidArg("gsplat_b200: unsupported batch tile shape / pixels per thread");
}

} // namespace

struct gs_batch {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    // plan
    bool planned = false;
    gs_gaussians g{};
    gs_settings s{};
    gs_batch_schedule sched{16, 16, 4, kSchedDynamic, 0};
    int views = 0;
    size_t pairs = 0, capacity = 0, total_pixels = 0;
    unsigned total_tiles = 0;
    int tile_bits = 0, cost_bits = 16;
    int grid_fwd = 0, grid_bwd = 0;
    int depth_result = 0, inst_result = 0, cost_result = 0;
    std::vector<BatchView> host_views;
    // device buffers
    DevBuf views_buf, tile_view_buf, state_buf, grad_buf, radii_buf, dsort_buf, isort_buf,
        ranges_buf, cost_buf, pixel_buf, hist_buf, status_buf, scan_status_buf, tile_ctr_buf,
        counters_buf, groups_buf;
    unsigned* emit_groups = nullptr; // the emit's instance groups, cut by the offset scan
    int group_shift = 9;
    unsigned group_cap = 0;
    BatchView* d_views = nullptr;
    unsigned short* d_tile_view = nullptr;
    GaussianState st{};
    int* radii = nullptr;
    unsigned* dkeys[2] = {nullptr, nullptr};
    unsigned* dvals[2] = {nullptr, nullptr};
    unsigned* ikeys[2] = {nullptr, nullptr};
    unsigned* ivals[2] = {nullptr, nullptr};
    unsigned* ckeys[2] = {nullptr, nullptr};
    unsigned* cvals[2] = {nullptr, nullptr};
    uint2* ranges = nullptr;
    float* pix_T = nullptr;
    unsigned* pix_last = nullptr;
    unsigned* counters = nullptr;
    unsigned* host_counters = nullptr; // pinned
    bool have_forward = false;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
};

namespace {

template <typename F> gs_status bguard(gs_batch* b, F&& f) {
    if (!b)
        return GS_ERR_INVALID;
    try {
        ck(cudaSetDevice(b->device), "cudaSetDevice");
        f();
        b->error.clear();
        return GS_OK;
    } catch (const InvalidArg& e) {
        b->error = e.what();
        return GS_ERR_INVALID;
    } catch (const StateError& e) {
        b->error = e.what();
        return GS_ERR_STATE;
    } catch (const CudaError& e) {
        b->error = e.what();
        return GS_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        b->error = "gsplat_b200: host allocation failed";
        return GS_ERR_CUDA;
    } catch (const std::exception& e) {
        b->error = e.what();
        return GS_ERR_CUDA;
    }
}

void drop_graph(gs_batch* b) {
    if (b->graph_exec)
        cudaGraphExecDestroy(b->graph_exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
}

GaussianState carve_state(char* p, size_t cap) {
    GaussianState st{};
    st.mean2d = reinterpret_cast<float2*>(p);
    p += align_up(cap * 8);
    st.conic = reinterpret_cast<float4*>(p);
    p += align_up(cap * 16);
    st.rgb = reinterpret_cast<float4*>(p);
    p += align_up(cap * 16);
    st.depth = reinterpret_cast<unsigned*>(p);
    p += align_up(cap * 4);
    st.touched = reinterpret_cast<unsigned*>(p);
    p += align_up(cap * 4);
    st.offset = reinterpret_cast<unsigned*>(p);
    p += align_up(cap * 4);
    st.bounds = reinterpret_cast<ushort4*>(p);
    p += align_up(cap * 8);
    st.spans = reinterpret_cast<uint4*>(p);
    return st;
}

size_t state_bytes(size_t cap) {
    return align_up(cap * 8) + align_up(cap * 16) * 2 + align_up(cap * 4) * 3 + align_up(cap * 8) +
           align_up(cap * 16);
}

void launch_preprocess_stage(gs_batch* b) {
    const gs_gaussians& g = b->g;
    const int n = g.count;
    const dim3 grid((n + kBlock - 1) / kBlock, b->views);
    with_tile(b->sched.tile_w, b->sched.tile_h, [&]<int TW, int TH>() {
        batch_preprocess_kernel<TW, TH><<<grid, kBlock, 0, b->stream>>>(
            n, g.means, g.log_scales, g.quaternions, g.opacity_logits, g.filter_3d, g.sh, g.colors,
            g.sh_degree, g.sh_bases, b->d_views, b->st, b->radii, b->dkeys[0], b->dvals[0],
            b->counters);
    });
}

// Counting pass (preprocess only) used by planning to size the instances.
size_t count_instances(gs_batch* b) {
    ck(cudaMemsetAsync(b->counters, 0, kBcWords * sizeof(unsigned), b->stream), "counters");
    launch_preprocess_stage(b);
    ck(cudaGetLastError(), "batch preprocess launch");
    ck(cudaMemcpyAsync(b->host_counters, b->counters, kBcWords * sizeof(unsigned),
                       cudaMemcpyDeviceToHost, b->stream),
       "count readback");
    ck(cudaStreamSynchronize(b->stream), "count sync");
    return *reinterpret_cast<const unsigned long long*>(b->host_counters + kBcInstances64);
}

void enqueue_forward(gs_batch* b, float* color, float* alpha) {
    const int n = b->g.count;
    cudaStream_t s = b->stream;
    ck(cudaMemsetAsync(b->counters, 0, kBcWords * sizeof(unsigned), s), "counters");
    launch_preprocess_stage(b);
    // device-side counts of the sorts: pairs and tiles (static), instances
    batch_counts_kernel<<<1, 1, 0, s>>>(b->counters, unsigned(b->capacity), unsigned(b->pairs),
                                        b->total_tiles);
    unsigned* hist = reinterpret_cast<unsigned*>(b->hist_buf.p);
    unsigned* status = reinterpret_cast<unsigned*>(b->status_buf.p);
    unsigned* tctr = reinterpret_cast<unsigned*>(b->tile_ctr_buf.p);
    b->depth_result = launch_radix_sort<unsigned>(s, b->dkeys, b->dvals, b->pairs,
                                                  b->counters + kBcPairs, 0, 32, hist, status,
                                                  tctr, b->counters + kBcErr);
    const unsigned* order = b->dvals[b->depth_result];
    launch_scan(s, int(b->pairs), b->st.touched, order, b->st.offset,
                reinterpret_cast<unsigned long long*>(b->scan_status_buf.p), tctr + 8,
                b->counters + kBcTotal, b->counters + kBcErr, /*zeroed=*/false, b->emit_groups,
                b->group_shift, b->group_cap);
    const unsigned emit_blocks = (b->group_cap + kBatchEmitBlock / 32 - 1) / (kBatchEmitBlock / 32);
    with_shape(b->sched.tile_w, b->sched.tile_h, b->sched.pixels_per_thread,
               [&]<int TW, int TH, int PX>() {
                   batch_emit_kernel<TW, TH><<<emit_blocks, kBatchEmitBlock, 0, s>>>(
                       n, b->counters, b->emit_groups, b->group_shift, b->group_cap, order, b->st,
                       b->d_views, b->ikeys[0], b->ivals[0], unsigned(b->capacity));
               });
    b->inst_result = launch_radix_sort<unsigned>(s, b->ikeys, b->ivals, b->capacity,
                                                 b->counters + kBcSorted, 0, b->tile_bits, hist,
                                                 status, tctr, b->counters + kBcErr);
    ck(cudaMemsetAsync(b->ranges, 0, size_t(b->total_tiles) * sizeof(uint2), s), "ranges");
    batch_ranges_kernel<<<int((b->capacity + kBlock - 1) / kBlock), kBlock, 0, s>>>(
        b->counters, b->ikeys[b->inst_result], b->ranges, b->total_tiles);
    if (b->sched.schedule == kSchedHeavyFirst) {
        batch_tile_cost_kernel<<<int((b->total_tiles + kBlock - 1) / kBlock), kBlock, 0, s>>>(
            b->total_tiles, b->ranges, b->ckeys[0], b->cvals[0]);
        b->cost_result = launch_radix_sort<unsigned>(s, b->ckeys, b->cvals, b->total_tiles,
                                                     b->counters + kBcTiles, 0, b->cost_bits,
                                                     hist, status, tctr, b->counters + kBcErr);
    }
    const TileLookup L{b->d_views, b->d_tile_view, b->cvals[b->cost_result]};
    const float3 bg = make_float3(b->s.background[0], b->s.background[1], b->s.background[2]);
    with_shape(b->sched.tile_w, b->sched.tile_h, b->sched.pixels_per_thread,
               [&]<int TW, int TH, int PX>() {
                   using G = TileGeom<TW, TH, PX>;
                   auto go = [&](auto kernel) {
                       kernel<<<b->grid_fwd, G::kThreads, 0, s>>>(
                           b->total_tiles, b->ranges, b->ivals[b->inst_result], b->st, L,
                           b->counters + kBcWork, bg, color, alpha, b->pix_T, b->pix_last);
                   };
                   if (b->sched.schedule == kSchedStatic)
                       go(batch_forward_kernel<TW, TH, PX, kSchedStatic>);
                   else if (b->sched.schedule == kSchedDynamic)
                       go(batch_forward_kernel<TW, TH, PX, kSchedDynamic>);
                   else
                       go(batch_forward_kernel<TW, TH, PX, kSchedHeavyFirst>);
               });
    ck(cudaGetLastError(), "batch forward launch");
}

void enqueue_backward(gs_batch* b, const float* dL_color, const float* dL_alpha,
                      const gs_model_grads* grads) {
    cudaStream_t s = b->stream;
    ck(cudaMemsetAsync(b->counters + kBcWorkBack, 0, sizeof(unsigned), s), "queue reset");
    const TileLookup L{b->d_views, b->d_tile_view, b->cvals[b->cost_result]};
    const float3 bg = make_float3(b->s.background[0], b->s.background[1], b->s.background[2]);
    with_shape(b->sched.tile_w, b->sched.tile_h, b->sched.pixels_per_thread,
               [&]<int TW, int TH, int PX>() {
                   using G = TileGeom<TW, TH, PX>;
                   auto go = [&](auto kernel) {
                       kernel<<<b->grid_bwd, G::kThreads, 0, s>>>(
                           b->total_tiles, b->ranges, b->ivals[b->inst_result], b->st, L,
                           b->counters + kBcWorkBack, bg, b->pix_T, b->pix_last, dL_color,
                           dL_alpha);
                   };
                   if (b->sched.schedule == kSchedStatic)
                       go(batch_backward_kernel<TW, TH, PX, kSchedStatic>);
                   else if (b->sched.schedule == kSchedDynamic)
                       go(batch_backward_kernel<TW, TH, PX, kSchedDynamic>);
                   else
                       go(batch_backward_kernel<TW, TH, PX, kSchedHeavyFirst>);
               });
    GradOutArgs out{};
    if (grads) {
        out.means = grads->means;
        out.scales = grads->scales;
        out.rotations = grads->rotations;
        out.opacities = grads->opacities;
        out.sh = grads->sh;
        out.colors = grads->colors;
        out.refine_weight = grads->refine_weight;
        out.activated = grads->activated;
    }
    const gs_gaussians& g = b->g;
    batch_gaussian_backward_kernel<<<(g.count + kBGBlock - 1) / kBGBlock, kBGBlock,
                                     batch_gaussian_backward_smem(b->views), s>>>(
        g.count, b->views, g.means, g.log_scales, g.quaternions, g.opacity_logits, g.filter_3d,
        g.sh, g.sh_degree, g.sh_bases, b->d_views, b->st, b->radii, out);
    ck(cudaGetLastError(), "batch backward launch");
}

} // namespace

namespace {

__global__ void fill_f32_kernel(float* __restrict__ p, size_t n, float v) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
         i += size_t(gridDim.x) * blockDim.x)
        p[i] = v;
}

void validate_gaussians(const gs_gaussians* g) {
    req(g && g->count > 0 && g->means && g->log_scales && g->quaternions && g->opacity_logits,
        "batch needs a non-empty Gaussian set");
    req((g->sh != nullptr) != (g->colors != nullptr), "exactly one of sh / colors");
    req(!g->sh || (g->sh_bases >= 1 && g->sh_bases <= 16 && g->sh_degree >= 0 &&
                   (g->sh_degree + 1) * (g->sh_degree + 1) <= g->sh_bases),
        "invalid SH layout");
}

int occupancy(const void* kernel, int threads, size_t smem) {
    int blocks = 0;
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem),
       "occupancy query");
    return std::max(blocks, 1);
}

void plan(gs_batch* b, const gs_gaussians* g, const gs_camera* cams, int views,
          const gs_settings* s, const gs_batch_schedule* sched, size_t instance_capacity) {
    validate_gaussians(g);
    req(cams && views >= 1 && views <= 4096, "batch needs 1..4096 cameras");
    req(s != nullptr, "settings required");
    gs_batch_schedule sc{16, 16, 4, kSchedDynamic, 0};
    if (sched)
        sc = *sched;
    req(valid_shape(sc.tile_w, sc.tile_h, sc.pixels_per_thread),
        "tile shape must be 8x8 (1|2 px/thread), 16x16 or 16x32 (2|4 px/thread)");
    req(sc.schedule >= 0 && sc.schedule <= 2 && sc.ctas_per_sm >= 0, "invalid schedule");
    const size_t pairs = size_t(views) * size_t(g->count);
    req(pairs < (size_t(1) << 31), "views * N must stay below 2^31");
    drop_graph(b);
    b->planned = false;
    b->have_forward = false;
    b->g = *g;
    b->s = *s;
    b->sched = sc;
    b->views = views;
    b->pairs = pairs;
    cudaStream_t st = b->stream;
    // views, tile table
    b->host_views.assign(size_t(views), BatchView{});
    std::vector<unsigned short> tile_view;
    size_t tiles = 0, pixels = 0;
    for (int v = 0; v < views; ++v) {
        const gs_camera& c = cams[v];
        req(c.width > 0 && c.height > 0 && c.width <= 65535 && c.height <= 65535,
            "camera size out of range");
        BatchView& bv = b->host_views[size_t(v)];
        Camera& K = bv.K;
        std::memcpy(K.view, c.world_to_camera, sizeof(K.view));
        std::memcpy(K.center, c.center, sizeof(K.center));
        K.fx = c.fx;
        K.fy = c.fy;
        K.cx = c.cx;
        K.cy = c.cy;
        K.near_plane = c.near_plane;
        K.alpha_clip = c.alpha_clip;
        K.width = c.width;
        K.height = c.height;
        K.grid_x = (c.width + sc.tile_w - 1) / sc.tile_w;
        K.grid_y = (c.height + sc.tile_h - 1) / sc.tile_h;
        K.compensate_2d = c.compensate_2d;
        K.kernel_size = s->kernel_size;
        K.scale_modifier = s->scale_modifier;
        bv.tile_base = unsigned(tiles);
        bv.pix_base = unsigned(pixels);
        const size_t vt = size_t(K.grid_x) * K.grid_y;
        tile_view.insert(tile_view.end(), vt, static_cast<unsigned short>(v));
        tiles += vt;
        pixels += size_t(c.width) * c.height;
    }
    req(tiles < (size_t(1) << 30) && pixels < (size_t(1) << 32) && views <= 65535,
        "batch too large");
    b->total_tiles = unsigned(tiles);
    b->total_pixels = pixels;
    b->tile_bits = msb_bits(unsigned(tiles));
    b->d_views = reinterpret_cast<BatchView*>(
        b->views_buf.exact(sizeof(BatchView) * size_t(views), st));
    ck(cudaMemcpyAsync(b->d_views, b->host_views.data(), sizeof(BatchView) * size_t(views),
                       cudaMemcpyHostToDevice, st),
       "views upload");
    b->d_tile_view = reinterpret_cast<unsigned short*>(b->tile_view_buf.exact(tiles * 2, st));
    ck(cudaMemcpyAsync(b->d_tile_view, tile_view.data(), tiles * 2, cudaMemcpyHostToDevice, st),
       "tile table upload");
    // per-pair state
    b->st = carve_state(b->state_buf.exact(state_bytes(pairs), st), pairs);
    b->st.grad = reinterpret_cast<float4*>(
        b->grad_buf.exact(pairs * kGradSlots * sizeof(float4), st, /*zero=*/true));
    b->radii = reinterpret_cast<int*>(b->radii_buf.exact(pairs * 4, st));
    char* d = b->dsort_buf.exact(align_up(pairs * 4) * 4, st);
    for (int k = 0; k < 2; ++k) {
        b->dkeys[k] = reinterpret_cast<unsigned*>(d + align_up(pairs * 4) * k);
        b->dvals[k] = reinterpret_cast<unsigned*>(d + align_up(pairs * 4) * (2 + k));
    }
    char* px = b->pixel_buf.exact(align_up(pixels * 4) * 2, st);
    b->pix_T = reinterpret_cast<float*>(px);
    b->pix_last = reinterpret_cast<unsigned*>(px + align_up(pixels * 4));
    b->ranges = reinterpret_cast<uint2*>(b->ranges_buf.exact(tiles * sizeof(uint2), st));
    char* cst = b->cost_buf.exact(align_up(tiles * 4) * 4, st);
    for (int k = 0; k < 2; ++k) {
        b->ckeys[k] = reinterpret_cast<unsigned*>(cst + align_up(tiles * 4) * k);
        b->cvals[k] = reinterpret_cast<unsigned*>(cst + align_up(tiles * 4) * (2 + k));
    }
    b->counters = reinterpret_cast<unsigned*>(b->counters_buf.exact(kBcWords * 4, st, true));
    b->hist_buf.exact(8 * 256 * sizeof(unsigned), st);
    b->tile_ctr_buf.exact(64 * sizeof(unsigned), st);
    b->scan_status_buf.exact(std::max<size_t>(scan_status_bytes(int(pairs)), 256), st);
    // the schedule's kernels: grid sizes and attributes
    const size_t gsmem = batch_gaussian_backward_smem(views);
    req(gsmem <= 227 * 1024, "too many views for the per-Gaussian backward");
    ck(cudaFuncSetAttribute(batch_gaussian_backward_kernel,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(gsmem)),
       "smem attribute");
    with_shape(sc.tile_w, sc.tile_h, sc.pixels_per_thread, [&]<int TW, int TH, int PX>() {
        using G = TileGeom<TW, TH, PX>;
        const void* fk;
        const void* bk;
        if (sc.schedule == kSchedStatic) {
            fk = reinterpret_cast<const void*>(batch_forward_kernel<TW, TH, PX, kSchedStatic>);
            bk = reinterpret_cast<const void*>(batch_backward_kernel<TW, TH, PX, kSchedStatic>);
        } else if (sc.schedule == kSchedDynamic) {
            fk = reinterpret_cast<const void*>(batch_forward_kernel<TW, TH, PX, kSchedDynamic>);
            bk = reinterpret_cast<const void*>(batch_backward_kernel<TW, TH, PX, kSchedDynamic>);
        } else {
            fk = reinterpret_cast<const void*>(batch_forward_kernel<TW, TH, PX, kSchedHeavyFirst>);
            bk = reinterpret_cast<const void*>(
                batch_backward_kernel<TW, TH, PX, kSchedHeavyFirst>);
        }
        const int of = sc.ctas_per_sm > 0 ? sc.ctas_per_sm : occupancy(fk, G::kThreads, 0);
        const int ob = sc.ctas_per_sm > 0 ? sc.ctas_per_sm : occupancy(bk, G::kThreads, 0);
        b->grid_fwd = int(std::min<size_t>(size_t(b->sms) * of, tiles));
        b->grid_bwd = int(std::min<size_t>(size_t(b->sms) * ob, tiles));
    });
    // instance capacity
    size_t cap = instance_capacity;
    if (cap == 0) {
        const size_t want = count_instances(b);
        cap = want + want / 4 + 4096;
    }
    // positions are 32-bit: the capacity stays below 2^32 with room for one
    // sort tile of padding
    req(cap < (size_t(1) << 32) - (size_t(1) << 20), "instance capacity must stay below 2^32");
    b->capacity = cap;
    // emit groups: sized by the capacity (the instance count is known only on
    // the device); instances past the capacity are never written
    b->group_shift = emit_group_shift(unsigned(cap));
    b->group_cap = unsigned((cap >> b->group_shift) + 2);
    b->emit_groups = reinterpret_cast<unsigned*>(
        b->groups_buf.exact(size_t(b->group_cap) * sizeof(unsigned), st));
    char* ik = b->isort_buf.exact(align_up(cap * 4) * 4, st);
    for (int k = 0; k < 2; ++k) {
        b->ikeys[k] = reinterpret_cast<unsigned*>(ik + align_up(cap * 4) * k);
        b->ivals[k] = reinterpret_cast<unsigned*>(ik + align_up(cap * 4) * (2 + k));
    }
    const size_t status = std::max({sort_status_bytes(pairs, 4),
                                    sort_status_bytes(cap, radix_passes(b->tile_bits)),
                                    sort_status_bytes(tiles, radix_passes(b->cost_bits)),
                                    size_t(256)});
    b->status_buf.exact(status, st);
    b->cost_result = 0;
    ck(cudaStreamSynchronize(st), "plan sync");
    b->planned = true;
}

} // namespace

extern "C" {

gs_status gs_batch_create(gs_batch** out, int device, void* stream) {
    if (!out)
        return GS_ERR_INVALID;
    *out = nullptr;
    gs_batch* b = new (std::nothrow) gs_batch();
    if (!b)
        return GS_ERR_CUDA;
    b->device = device;
    b->stream = static_cast<cudaStream_t>(stream);
    const gs_status s = bguard(b, [&] {
        int sms = 0;
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
        b->sms = sms > 0 ? sms : 148;
        ck(cudaMallocHost(&b->host_counters, kBcWords * sizeof(unsigned)), "pinned counters");
    });
    if (s != GS_OK) {
        gs_batch_destroy(b);
        return s;
    }
    *out = b;
    return GS_OK;
}

void gs_batch_destroy(gs_batch* b) {
    if (!b)
        return;
    cudaSetDevice(b->device);
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    else
        cudaDeviceSynchronize();
    drop_graph(b);
    for (DevBuf* d : {&b->views_buf, &b->tile_view_buf, &b->state_buf, &b->grad_buf,
                      &b->radii_buf, &b->dsort_buf, &b->isort_buf, &b->ranges_buf, &b->cost_buf,
                      &b->pixel_buf, &b->hist_buf, &b->status_buf, &b->scan_status_buf,
                      &b->tile_ctr_buf, &b->counters_buf})
        d->release();
    if (b->host_counters)
        cudaFreeHost(b->host_counters);
    delete b;
}

const char* gs_batch_last_error(const gs_batch* b) { return b ? b->error.c_str() : "null batch"; }

gs_status gs_batch_set_stream(gs_batch* b, void* stream) {
    return bguard(b, [&] {
        drop_graph(b);
        b->stream = static_cast<cudaStream_t>(stream);
    });
}

gs_status gs_batch_plan(gs_batch* b, const gs_gaussians* g, const gs_camera* cams, int views,
                        const gs_settings* s, const gs_batch_schedule* sched,
                        size_t instance_capacity) {
    return bguard(b, [&] { plan(b, g, cams, views, s, sched, instance_capacity); });
}

gs_status gs_batch_get_info(gs_batch* b, gs_batch_info* out) {
    return bguard(b, [&] {
        req(out != nullptr, "info output required");
        std::memset(out, 0, sizeof(*out));
        if (!b->planned)
            return;
        ck(cudaMemcpyAsync(b->host_counters, b->counters, kBcWords * sizeof(unsigned),
                           cudaMemcpyDeviceToHost, b->stream),
           "counter readback");
        ck(cudaStreamSynchronize(b->stream), "info sync");
        out->pairs = b->pairs;
        out->instance_capacity = b->capacity;
        out->total_pixels = b->total_pixels;
        out->total_tiles = int(b->total_tiles);
        out->views = b->views;
        out->instances =
            *reinterpret_cast<const long long*>(b->host_counters + kBcInstances64);
        out->visible = int(b->host_counters[kBcVisible]);
        out->device_error = int(b->host_counters[kBcErr]);
        out->overflow = (b->host_counters[kBcErr] & kDevCapacity) ? 1 : 0;
    });
}

gs_status gs_batch_forward(gs_batch* b, float* color, float* alpha, int* radii_out) {
    return bguard(b, [&] {
        if (!b->planned)
            throw StateError("gsplat_b200: batch forward before a plan");
        req(color && alpha, "colour and alpha outputs required");
        enqueue_forward(b, color, alpha);
        if (radii_out)
            ck(cudaMemcpyAsync(radii_out, b->radii, b->pairs * sizeof(int),
                               cudaMemcpyDeviceToDevice, b->stream),
               "radii copy");
        b->have_forward = true;
    });
}

gs_status gs_batch_backward(gs_batch* b, const float* dL_color, const float* dL_alpha,
                            const gs_model_grads* grads) {
    return bguard(b, [&] {
        if (!b->have_forward)
            throw StateError("gsplat_b200: batch backward without a forward");
        req(dL_color != nullptr, "colour gradient required");
        enqueue_backward(b, dL_color, dL_alpha, grads);
    });
}

gs_status gs_batch_capture(gs_batch* b, float* color, float* alpha, int* radii_out,
                           const float* dL_color, const float* dL_alpha,
                           const gs_model_grads* grads) {
    return bguard(b, [&] {
        if (!b->planned)
            throw StateError("gsplat_b200: batch capture before a plan");
        req(color && alpha, "colour and alpha outputs required");
        req(b->stream != nullptr, "graph capture needs a non-default stream");
        drop_graph(b);
        ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            enqueue_forward(b, color, alpha);
            if (radii_out)
                ck(cudaMemcpyAsync(radii_out, b->radii, b->pairs * sizeof(int),
                                   cudaMemcpyDeviceToDevice, b->stream),
                   "radii copy");
            if (dL_color)
                enqueue_backward(b, dL_color, dL_alpha, grads);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(b->stream, &g);
            if (g)
                cudaGraphDestroy(g);
            throw;
        }
        ck(cudaStreamEndCapture(b->stream, &b->graph), "end capture");
        ck(cudaGraphInstantiate(&b->graph_exec, b->graph, 0), "graph instantiate");
        b->have_forward = true;
    });
}

gs_status gs_batch_replay(gs_batch* b) {
    return bguard(b, [&] {
        if (!b->graph_exec)
            throw StateError("gsplat_b200: no captured batch graph");
        ck(cudaGraphLaunch(b->graph_exec, b->stream), "graph launch");
    });
}

gs_status gs_batch_autotune(gs_batch* b, const gs_gaussians* g, const gs_camera* cams, int views,
                            const gs_settings* s, int iterations, gs_batch_schedule* best,
                            float* best_ms, gs_batch_schedule* tried, float* tried_ms,
                            int* n_tried) {
    return bguard(b, [&] {
        validate_gaussians(g);
        req(best != nullptr && iterations >= 1, "autotune needs an output and iterations >= 1");
        const int cap_tried = (tried && tried_ms && n_tried) ? *n_tried : 0;
        if (n_tried)
            *n_tried = 0;
        static const int kShapes[6][3] = {{8, 8, 1},  {8, 8, 2},  {16, 16, 2},
                                          {16, 16, 4}, {16, 32, 2}, {16, 32, 4}};
        // scratch images, loss gradient and parameter gradients
        size_t pixels = 0;
        for (int v = 0; v < views; ++v)
            pixels += size_t(cams[v].width) * cams[v].height;
        const size_t n = size_t(g->count);
        const size_t stride = g->sh ? size_t(g->sh_bases) * 3 : 3;
        DevBuf scratch;
        const size_t img = align_up(pixels * 4);
        const size_t grad_floats = n * (3 + 3 + 4 + 1 + 1 + stride);
        // colour (3 planes), alpha, loss gradient (3 planes), parameter gradients
        char* p = scratch.exact(img * 7 + align_up(grad_floats * 4), b->stream, true);
        float* color = reinterpret_cast<float*>(p);
        float* alpha = reinterpret_cast<float*>(p + 3 * img);
        float* dL_color = reinterpret_cast<float*>(p + 4 * img);
        fill_f32_kernel<<<1024, 256, 0, b->stream>>>(dL_color, pixels * 3, 1e-3f);
        float* gp = reinterpret_cast<float*>(p + 7 * img);
        gs_model_grads mg{};
        mg.means = gp;
        mg.scales = gp + 3 * n;
        mg.rotations = gp + 6 * n;
        mg.opacities = gp + 10 * n;
        mg.refine_weight = gp + 11 * n;
        if (g->sh)
            mg.sh = gp + 12 * n;
        else
            mg.colors = gp + 12 * n;
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        float best_t = 1e30f;
        gs_batch_schedule best_s{};
        int count = 0;
        try {
            for (const auto& sh : kShapes)
                for (int sched = 0; sched < 3; ++sched) {
                    const gs_batch_schedule cand{sh[0], sh[1], sh[2], sched, 0};
                    plan(b, g, cams, views, s, &cand, 0);
                    for (int w = 0; w < 2; ++w) {
                        enqueue_forward(b, color, alpha);
                        enqueue_backward(b, dL_color, nullptr, &mg);
                    }
                    ck(cudaEventRecord(e0, b->stream), "event record");
                    for (int it = 0; it < iterations; ++it) {
                        enqueue_forward(b, color, alpha);
                        enqueue_backward(b, dL_color, nullptr, &mg);
                    }
                    ck(cudaEventRecord(e1, b->stream), "event record");
                    ck(cudaEventSynchronize(e1), "event sync");
                    float ms = 0.f;
                    ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
                    ms /= float(iterations);
                    ck(cudaMemcpy(b->host_counters, b->counters, kBcWords * sizeof(unsigned),
                                  cudaMemcpyDeviceToHost),
                       "counter readback");
                    if (b->host_counters[kBcErr] != 0)
                        ms = 1e30f; // a candidate that overflowed or timed out is not kept
                    if (count < cap_tried) {
                        tried[count] = cand;
                        tried_ms[count] = ms;
                    }
                    ++count;
                    if (ms < best_t) {
                        best_t = ms;
                        best_s = cand;
                    }
                }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            scratch.release();
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        ck(cudaStreamSynchronize(b->stream), "autotune sync");
        scratch.release();
        req(best_t < 1e29f, "no batch schedule ran without error");
        plan(b, g, cams, views, s, &best_s, 0);
        *best = best_s;
        if (best_ms)
            *best_ms = best_t;
        if (n_tried)
            *n_tried = std::min(count, cap_tried);
    });
}

} // extern "C"
