// C ABI and host orchestration of one forward/backward pair.
//
// Mirrors splat_drender::Rasterizer::forward/backward
// (third_party/splat_drender/src/pipeline.cu:457-615, :651-712):
//   forward:  preprocess -> scan of tile counts -> ONE host readback of
//             {instances, visible} (pipeline.cu:208-212) -> duplicate-with-keys
//             -> onesweep sort -> tile ranges -> composite
//   backward: composite adjoint -> per-Gaussian adjoint (+ fused Adam)
// Differences by design: the context owns a grow-only workspace instead of
// caller pool callbacks, every launch goes to the context stream, the camera
// travels by value, and no snapshot/bucket state is kept (the backward
// recomputes transmittance per tile from the stored final T).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/gsplat_b200.h"
#include "common.cuh"
#include "host.h"
#include "kernels.h"

using namespace gsb;

using namespace gsb::host;

// Automatic compositing schedule: one pixel per thread up to this many 16x16
// tiles, two up to kAutoPx2Tiles, four above (measured on B200: 256 tiles,
// 1,200 tiles and 8,160 tiles).
constexpr int kAutoPx1Tiles = 600;
constexpr int kAutoPx2Tiles = 2400;

struct gs_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string error;
    // workspace
    DevBuf gauss, grad, scan_status, counters, inst_keys, inst_vals, sort_hist, sort_status,
        sort_counters, ranges, pixel, depth_sort, loss, probe, geo_grad, rec, emit_groups;
    unsigned* host_counts = nullptr; // pinned [16]: [0, 8) draw counts, [8] error word after the sorts
    size_t gauss_cap = 0, grad_cap = 0, inst_cap = 0, pixel_cap = 0, geo_grad_cap = 0;
    GaussianState st{};
    RecStaging staging{};     // tensor map of st.rec for the compositing kernels' TMA gathers
    float4* plane = nullptr;  // ray planes and normals of the median-depth channel
    float4* normal = nullptr;
    unsigned long long* keys[2] = {nullptr, nullptr};
    unsigned* vals[2] = {nullptr, nullptr};
    unsigned* dkeys[2] = {nullptr, nullptr}; // depth sort keys / Gaussian ids
    unsigned* dvals[2] = {nullptr, nullptr};
    size_t depth_cap = 0;
    // last forward
    bool have_forward = false;
    bool record_backward = false;
    gs_gaussians g{};
    Camera K{};
    float3 bg{};
    int tiles = 0;
    int instances = 0;
    int visible = 0;
    int sorted_buf = 0;
    int sort_bits = 0;
    float* pix_T = nullptr;
    unsigned* pix_last = nullptr;
    float* pix_dtdt = nullptr; // dT/dt at the median depth (geometry training forwards)
    unsigned* tile_order = nullptr; // the last colour training forward's tiles, heaviest first
    bool geometry = false;     // the last forward rendered the median-depth / normal channels
    const float* fwd_depth = nullptr;  // its median-depth and normal outputs (caller memory)
    const float* fwd_normal = nullptr;
    int pixels_per_thread = 0; // compositing schedule (1, 2, 4, 8; 0: by tile count), gs_set_schedule
    // timing: two event sets used alternately per step, so the previous
    // step's intervals are read at the next forward's count readback without
    // an extra host synchronisation.
    bool timing = false;
    cudaEvent_t ev[2][16] = {}; // stage k: begin 2k, end 2k+1
    cudaEvent_t ev_counts = nullptr; // the draw-count read-back of the forward
    cudaEvent_t ev_sorted = nullptr; // the error word read back after the forward's sorts
    int ev_set = 0;
    bool ev_pending = false;
    double acc_ms[8] = {};
    long acc_steps = 0;
};

namespace {

template <typename F> gs_status guarded(gs_context* ctx, F&& f) {
    if (!ctx)
        return GS_ERR_INVALID;
    try {
        ck(cudaSetDevice(ctx->device), "cudaSetDevice");
        f();
        ctx->error.clear();
        return GS_OK;
    } catch (const InvalidArg& e) {
        ctx->error = e.what();
        return GS_ERR_INVALID;
    } catch (const StateError& e) {
        ctx->error = e.what();
        return GS_ERR_STATE;
    } catch (const TimeoutError& e) {
        ctx->error = e.what();
        return GS_ERR_TIMEOUT;
    } catch (const CudaError& e) {
        ctx->error = e.what();
        return GS_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        ctx->error = "gsplat_b200: host allocation failed";
        return GS_ERR_CUDA;
    } catch (const std::exception& e) {
        ctx->error = e.what();
        return GS_ERR_CUDA;
    }
}

// Stage k: 0 preprocess, 1 depth sort + offset scan, 2 emit, 3 tile sort,
// 4 ranges, 5 composite, 6 composite backward, 7 gaussian backward (+Adam).
// Pixels per thread of the compositing kernels. Automatic (0): a frame's
// compositing time is the longest tile's serial walk when there are too few
// tiles to fill the GPU, and fewer pixels per thread shorten that walk (more
// threads share each tile); with many tiles, four pixels per thread amortise
// the staging and the per-Gaussian setup best.
int compositing_px(const gs_context* c, int tiles) {
    if (c->pixels_per_thread > 0)
        return c->pixels_per_thread;
    return tiles <= kAutoPx1Tiles ? 1 : tiles <= kAutoPx2Tiles ? 2 : 4;
}

void mark(gs_context* c, int stage, bool end) {
    if (c->timing)
        ck(cudaEventRecord(c->ev[c->ev_set][2 * stage + (end ? 1 : 0)], c->stream),
           "event record");
}

// Adds the completed intervals of event set `set` to the running totals.
void harvest(gs_context* c, int set) {
    float ms[8];
    for (int k = 0; k < 8; ++k)
        if (cudaEventElapsedTime(&ms[k], c->ev[set][2 * k], c->ev[set][2 * k + 1]) !=
            cudaSuccess) {
            cudaGetLastError();
            return; // incomplete step (e.g. forward without backward): skip it
        }
    for (int k = 0; k < 8; ++k)
        c->acc_ms[k] += ms[k];
    ++c->acc_steps;
}

Camera make_camera(const gs_camera* cam, const gs_settings* s) {
    Camera K;
    std::memcpy(K.view, cam->world_to_camera, sizeof(K.view));
    std::memcpy(K.center, cam->center, sizeof(K.center));
    K.fx = cam->fx;
    K.fy = cam->fy;
    K.cx = cam->cx;
    K.cy = cam->cy;
    K.near_plane = cam->near_plane;
    K.alpha_clip = cam->alpha_clip;
    K.width = cam->width;
    K.height = cam->height;
    K.grid_x = (cam->width + kTileW - 1) / kTileW;
    K.grid_y = (cam->height + kTileH - 1) / kTileH;
    K.compensate_2d = cam->compensate_2d;
    K.kernel_size = s->kernel_size;
    K.scale_modifier = s->scale_modifier;
    return K;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// The device error word is counters[2]: look-back waits that gave up set it.
unsigned* device_error_word(gs_context* c) {
    return reinterpret_cast<unsigned*>(c->counters.p) + 2;
}

// Clears a set error word and reports it; the draw list of the forward it
// came from is dropped (no backward or reuse may run on it).
[[noreturn]] void raise_timeout(gs_context* c, unsigned word, const char* where) {
    ck(cudaMemsetAsync(device_error_word(c), 0, sizeof(unsigned), c->stream), "error reset");
    c->have_forward = false;
    throw TimeoutError(std::string("gsplat_b200: a device-side bounded wait timed out ") +
                       where + " (error word " + std::to_string(word) + ")");
}

// Before anything consumes the last forward's draw list: waits for the error
// word copied back right after the forward's sorts (the host usually reaches
// this while the compositing still runs) and refuses a list whose sort gave up.
void check_forward_sorts(gs_context* c) {
    ck(cudaEventSynchronize(c->ev_sorted), "sort status sync");
    if (c->host_counts[8])
        raise_timeout(c, c->host_counts[8], "in the forward's sorts");
}

// The record array as a [rows][16] float32 tensor with a box of one row (the
// shape tile::gather4 copies), encoded through the driver's
// cuTensorMapEncodeTiled (reached through the runtime, so the library links
// no driver stub). The driver checks the base (16-byte aligned) and the row
// stride (64 bytes).
void encode_record_map(gs_context* c, size_t rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q{};
        ck(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled",
                                            reinterpret_cast<void**>(&encode), 12000,
                                            cudaEnableDefault, &q),
           "driver entry point cuTensorMapEncodeTiled");
        if (q != cudaDriverEntryPointSuccess || !encode)
            throw std::runtime_error("gsplat_b200: cuTensorMapEncodeTiled is not available");
    }
    const cuuint64_t dims[2] = {16, cuuint64_t(rows)};
    const cuuint64_t strides[1] = {sizeof(SplatRec)};
    const cuuint32_t box[2] = {16, 1};
    const cuuint32_t elem[2] = {1, 1};
    const CUresult r = encode(&c->staging.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, c->st.rec,
                              dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        throw std::runtime_error("gsplat_b200: cuTensorMapEncodeTiled failed (" +
                                 std::to_string(int(r)) + ")");
}

const RecStaging& record_staging(gs_context* c) {
    c->staging.err = device_error_word(c);
    return c->staging;
}

void carve_gaussians(gs_context* c, int n) {
    const size_t N = size_t(n);
    if (N > c->gauss_cap) {
        const size_t cap = N + N / 4 + 1024;
        const size_t bytes = align_up(cap * 8) + align_up(cap * 16) * 4 + align_up(cap * 4) * 3 +
                             align_up(cap * 8);
        char* p = c->gauss.ensure(bytes, c->stream);
        c->st.mean2d = reinterpret_cast<float2*>(p);
        p += align_up(cap * 8);
        c->st.conic = reinterpret_cast<float4*>(p);
        p += align_up(cap * 16);
        c->st.rgb = reinterpret_cast<float4*>(p);
        p += align_up(cap * 16);
        c->st.depth = reinterpret_cast<unsigned*>(p);
        p += align_up(cap * 4);
        c->st.touched = reinterpret_cast<unsigned*>(p);
        p += align_up(cap * 4);
        c->st.offset = reinterpret_cast<unsigned*>(p);
        p += align_up(cap * 4);
        c->st.bounds = reinterpret_cast<ushort4*>(p);
        p += align_up(cap * 8);
        c->plane = reinterpret_cast<float4*>(p);
        p += align_up(cap * 16);
        c->normal = reinterpret_cast<float4*>(p);
        c->st.rec = reinterpret_cast<SplatRec*>(c->rec.ensure(cap * sizeof(SplatRec), c->stream));
        encode_record_map(c, cap);
        c->gauss_cap = cap;
    }
    if (N > c->grad_cap) {
        const size_t cap = std::max(N + N / 4 + 1024, c->gauss_cap);
        c->st.grad = reinterpret_cast<float4*>(
            c->grad.ensure(cap * kGradSlots * sizeof(float4), c->stream, /*zero=*/true));
        c->grad_cap = cap;
    }
}

void ensure_instances(gs_context* c, size_t count, int passes) {
    if (count > c->inst_cap) {
        const size_t cap = count + count / 4 + 4096;
        char* k = c->inst_keys.ensure(align_up(cap * 8) * 2, c->stream);
        c->keys[0] = reinterpret_cast<unsigned long long*>(k);
        c->keys[1] = reinterpret_cast<unsigned long long*>(k + align_up(cap * 8));
        char* v = c->inst_vals.ensure(align_up(cap * 4) * 2, c->stream);
        c->vals[0] = reinterpret_cast<unsigned*>(v);
        c->vals[1] = reinterpret_cast<unsigned*>(v + align_up(cap * 4));
        c->inst_cap = cap;
    }
}

void ensure_depth_sort(gs_context* c, size_t n) {
    if (n > c->depth_cap) {
        const size_t cap = n + n / 4 + 1024;
        char* p = c->depth_sort.ensure(align_up(cap * 4) * 4, c->stream);
        for (int k = 0; k < 2; ++k) {
            c->dkeys[k] = reinterpret_cast<unsigned*>(p + align_up(cap * 4) * k);
            c->dvals[k] = reinterpret_cast<unsigned*>(p + align_up(cap * 4) * (2 + k));
        }
        c->depth_cap = cap;
    }
}

} // namespace

extern "C" {

int gs_abi_version(void) { return GS_ABI_VERSION; }

gs_status gs_create(gs_context** out, int device, void* stream) {
    if (!out)
        return GS_ERR_INVALID;
    *out = nullptr;
    gs_context* c = new (std::nothrow) gs_context();
    if (!c)
        return GS_ERR_CUDA;
    c->device = device;
    c->stream = static_cast<cudaStream_t>(stream);
    const gs_status st = guarded(c, [&] {
        ck(cudaMallocHost(&c->host_counts, 16 * sizeof(unsigned)), "pinned counters");
        std::memset(c->host_counts, 0, 16 * sizeof(unsigned));
        c->counters.ensure(64, c->stream, true);
        c->sort_hist.ensure(8 * 256 * sizeof(unsigned), c->stream);
        c->sort_counters.ensure(64, c->stream);
        for (auto& set : c->ev)
            for (auto& e : set)
                ck(cudaEventCreate(&e), "event create");
        ck(cudaEventCreateWithFlags(&c->ev_counts, cudaEventDisableTiming), "event create");
        ck(cudaEventCreateWithFlags(&c->ev_sorted, cudaEventDisableTiming), "event create");
    });
    if (st != GS_OK) {
        gs_destroy(c);
        return st;
    }
    *out = c;
    return GS_OK;
}

void gs_destroy(gs_context* c) {
    if (!c)
        return;
    cudaSetDevice(c->device);
    if (c->stream)
        cudaStreamSynchronize(c->stream);
    else
        cudaDeviceSynchronize();
    for (DevBuf* b : {&c->gauss, &c->grad, &c->scan_status, &c->counters, &c->inst_keys,
                      &c->inst_vals, &c->sort_hist, &c->sort_status, &c->sort_counters,
                      &c->ranges, &c->pixel, &c->depth_sort, &c->loss, &c->probe,
                      &c->geo_grad})
        b->release();
    if (c->host_counts)
        cudaFreeHost(c->host_counts);
    for (auto& set : c->ev)
        for (auto& e : set)
            if (e)
                cudaEventDestroy(e);
    if (c->ev_counts)
        cudaEventDestroy(c->ev_counts);
    if (c->ev_sorted)
        cudaEventDestroy(c->ev_sorted);
    delete c;
}

gs_status gs_set_stream(gs_context* c, void* stream) {
    return guarded(c, [&] { c->stream = static_cast<cudaStream_t>(stream); });
}

const char* gs_last_error(const gs_context* c) { return c ? c->error.c_str() : "null context"; }

size_t gs_workspace_bytes(const gs_context* c) {
    if (!c)
        return 0;
    size_t t = 0;
    for (const DevBuf* b : {&c->gauss, &c->grad, &c->scan_status, &c->counters, &c->inst_keys,
                            &c->inst_vals, &c->sort_hist, &c->sort_status, &c->sort_counters,
                            &c->ranges, &c->pixel, &c->depth_sort, &c->loss, &c->probe,
                            &c->geo_grad})
        t += b->bytes;
    return t;
}

gs_status gs_forward(gs_context* c, const gs_gaussians* g, const gs_camera* cam,
                     const gs_settings* s, const gs_outputs* out, gs_forward_info* info) {
    return guarded(c, [&] {
        req(g && cam && s && out, "null argument");
        req(g->count > 0 && cam->width > 0 && cam->height > 0, "empty inputs");
        req(g->means && g->log_scales && g->quaternions && g->opacity_logits,
            "means, log_scales, quaternions and opacity_logits are required");
        req((g->sh != nullptr) != (g->colors != nullptr), "exactly one color source required");
        req(!g->sh || (g->sh_bases >= 1 && g->sh_bases <= 16 && g->sh_degree >= 0 &&
                       (g->sh_degree + 1) * (g->sh_degree + 1) <= g->sh_bases),
            "invalid SH degree/bases");
        req(out->color && out->alpha && out->radii, "forward outputs required");
        const bool geometry = s->need_depth != 0;
        req(!geometry || (out->median_depth && out->normal),
            "need_depth requires the median_depth and normal outputs");
        req(aligned16(g->quaternions), "quaternions must be 16-byte aligned");
        req(cam->fx > 0.f && cam->fy > 0.f, "focal lengths must be positive");
        req(size_t(cam->width) * cam->height < (size_t(1) << 31), "image too large");
        c->have_forward = false;
        const int n = g->count;
        const Camera K = make_camera(cam, s);
        const int tiles = K.grid_x * K.grid_y;
        const size_t P = size_t(cam->width) * cam->height;
        cudaStream_t st = c->stream;
        carve_gaussians(c, n);
        if (P > c->pixel_cap) {
            const size_t cap = P + P / 4;
            char* p = c->pixel.ensure(align_up(cap * 4) * 3, st);
            c->pix_T = reinterpret_cast<float*>(p);
            c->pix_last = reinterpret_cast<unsigned*>(p + align_up(cap * 4));
            c->pix_dtdt = reinterpret_cast<float*>(p + 2 * align_up(cap * 4));
            c->pixel_cap = cap;
        }
        unsigned* counters = reinterpret_cast<unsigned*>(c->counters.p);
        // counters: [0] instances [1] visible [2] device error [3] scan tile counter
        //           [4] min depth bits [5] max depth bits [6] Gaussian count [7] scan total
        launch_frame_counters_init(st, counters);
        const int prev_set = c->ev_set;
        const bool prev_pending = c->ev_pending && c->timing;
        c->ev_set ^= 1;
        c->ev_pending = false;
        mark(c, 0, false);
        // The geometry channels' ray planes and normals are computed only
        // when they are rendered (a NULL plane array turns them off).
        GaussianState gst = c->st;
        gst.plane = geometry ? c->plane : nullptr;
        gst.normal = geometry ? c->normal : nullptr;
        launch_preprocess(st, n, g->means, g->log_scales, g->quaternions, g->opacity_logits,
                          g->filter_3d, g->sh, g->colors, g->sh_degree, g->sh_bases, K, gst,
                          out->radii, counters);
        ck(cudaGetLastError(), "preprocess launch");
        mark(c, 0, true);
        ck(cudaMemcpyAsync(c->host_counts, counters, 8 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                           st),
           "read draw counts");
        ck(cudaEventRecord(c->ev_counts, st), "count event");
        // While the host waits for the counts, the GPU zeroes this frame's
        // scratch and compacts the visible Gaussians (the compaction reads the
        // depth range on the device). The scratch sized by n and the tile
        // count sits in one buffer, zeroed by one memset: tile ranges first
        // (they stay for the backward), then the digit histograms, the
        // look-back status words and tile counters of the compaction, depth
        // sort (at most 4 passes of n keys) and offset scan.
        ensure_depth_sort(c, size_t(n));
        size_t frame = 0;
        auto carve = [&](size_t bytes) {
            const size_t at = frame;
            frame += align_up(std::max<size_t>(bytes, 1));
            return at;
        };
        const size_t o_hist_d = (carve(size_t(tiles) * sizeof(uint2)), carve(4 * 256 * 4));
        const size_t o_hist_t = carve(4 * 256 * 4);
        const size_t o_compact = carve(scan_status_bytes(n));
        const size_t o_scan = carve(scan_status_bytes(n));
        const size_t o_dsort = carve(sort_status_bytes(size_t(n), 4));
        const size_t o_ctr = carve(16 * sizeof(unsigned));
        // per-tile adjoint work (accumulated by the compositing) and the
        // backward's tile order (heaviest first)
        const size_t o_work = carve(size_t(tiles) * sizeof(unsigned));
        const size_t o_order = carve(size_t(tiles) * sizeof(unsigned));
        char* fb = c->ranges.ensure(frame, st);
        unsigned* tile_work = reinterpret_cast<unsigned*>(fb + o_work);
        unsigned* tile_order = reinterpret_cast<unsigned*>(fb + o_order);
        c->tile_order = nullptr; // set below once the order is computed
        unsigned* fctr = reinterpret_cast<unsigned*>(fb + o_ctr); // [0] compaction [1] scan
                                                                  // [2..6) depth sort passes
        unsigned* hist = reinterpret_cast<unsigned*>(fb + o_hist_d);
        mark(c, 1, false);
        ck(cudaMemsetAsync(fb, 0, frame, st), "frame reset");
        launch_depth_compact(st, n, c->st, counters, c->dkeys[0], c->dvals[0], hist,
                             reinterpret_cast<unsigned long long*>(fb + o_compact), fctr + 0,
                             counters + 2, /*zeroed=*/true);
        ck(cudaEventSynchronize(c->ev_counts), "draw count sync");
        if (prev_pending)
            harvest(c, prev_set);
        const unsigned instances = c->host_counts[0];
        const unsigned visible = c->host_counts[1];
        const unsigned dev_err = c->host_counts[2];
        const unsigned dmin = c->host_counts[4], dmax = c->host_counts[5];
        if (dev_err)
            raise_timeout(c, dev_err, "before this forward's draw counts");
        req(instances < (1u << 30), "instance count exceeds 2^30");
        // enough bits to hold the tile count itself, so an all-ones sentinel
        // key sorts after every tile
        const int tile_bits = msb_bits(unsigned(tiles));
        const int depth_bits = msb_bits(visible ? dmax - dmin + 1u : 1u);
        ensure_instances(c, std::max<size_t>(instances, 1), 2);
        // The tile sort's status and counters, sized by the instance count.
        const int tpasses = radix_passes(tile_bits);
        const size_t tstat = align_up(sort_status_bytes(instances, tpasses));
        char* ts = c->sort_status.ensure(tstat + 256, st);
        ck(cudaMemsetAsync(ts, 0, tstat + 256, st), "tile sort reset");
        int cur = 0;
        if (instances > 0) {
            // 1. visible Gaussians in (depth, index) order
            const int dcur = launch_radix_sort<unsigned>(
                st, c->dkeys, c->dvals, size_t(visible), counters + 1, 0, depth_bits, hist,
                reinterpret_cast<unsigned*>(fb + o_dsort), fctr + 2, counters + 2,
                /*hist_ready=*/true, /*zeroed=*/true);
            const unsigned* order = c->dvals[dcur];
            // the offsets in depth order, cut into the emit's instance groups
            const int gshift = emit_group_shift(instances);
            const unsigned gcap = emit_group_count(instances, gshift) + 1;
            unsigned* egroups = reinterpret_cast<unsigned*>(
                c->emit_groups.ensure(size_t(gcap) * sizeof(unsigned), st));
            launch_scan(st, int(visible), c->st.touched, order, c->st.offset,
                        reinterpret_cast<unsigned long long*>(fb + o_scan), fctr + 1,
                        counters + 7, counters + 2, /*zeroed=*/true, egroups, gshift, gcap);
            ck(cudaGetLastError(), "depth sort launch");
            mark(c, 1, true);
            // 2. duplicate-with-keys in depth order
            mark(c, 2, false);
            unsigned* tkeys[2] = {reinterpret_cast<unsigned*>(c->keys[0]),
                                  reinterpret_cast<unsigned*>(c->keys[1])};
            unsigned* thist = reinterpret_cast<unsigned*>(fb + o_hist_t);
            launch_emit_keys(st, int(visible), instances, egroups, gshift, order, c->st,
                             K.grid_x, K.grid_y, tkeys[0], c->vals[0], unsigned(c->inst_cap),
                             tile_bits, thist);
            ck(cudaGetLastError(), "emit launch");
            mark(c, 2, true);
            // 3. stable sort of the instances on their tile bits
            mark(c, 3, false);
            cur = launch_radix_sort<unsigned>(st, tkeys, c->vals, instances, counters + 0, 0,
                                              tile_bits, thist, reinterpret_cast<unsigned*>(ts),
                                              reinterpret_cast<unsigned*>(ts + tstat), counters + 2,
                                              /*hist_ready=*/true, /*zeroed=*/true);
            ck(cudaGetLastError(), "sort launch");
            mark(c, 3, true);
            mark(c, 4, false);
            launch_tile_ranges(st, int(instances), tkeys[cur],
                               reinterpret_cast<uint2*>(c->ranges.p), tiles);
            ck(cudaGetLastError(), "ranges launch");
            mark(c, 4, true);
            // The error word of the compaction, depth sort, offset scan and
            // tile sort, for check_forward_sorts (4 bytes; the host waits on
            // it only where the draw list is consumed again).
            ck(cudaMemcpyAsync(c->host_counts + 8, counters + 2, sizeof(unsigned),
                               cudaMemcpyDeviceToHost, st),
               "read sort status");
        } else {
            c->host_counts[8] = 0;
            for (int k = 1; k <= 4; ++k) {
                mark(c, k, false);
                mark(c, k, true);
            }
        }
        ck(cudaEventRecord(c->ev_sorted, st), "sort status event");
        const int bits = depth_bits + tile_bits;
        mark(c, 5, false);
        const float3 bg = make_float3(s->background[0], s->background[1], s->background[2]);
        if (geometry)
            launch_composite_geometry(st, tiles, reinterpret_cast<const uint2*>(c->ranges.p),
                                      c->vals[cur], gst, K, bg, out->color, out->alpha,
                                      c->pix_T, c->pix_last,
                                      s->record_backward_state ? c->pix_dtdt : nullptr,
                                      out->visibility, out->median_depth, out->normal);
        else {
            const bool train = s->record_backward_state != 0;
            launch_composite_forward(st, tiles, reinterpret_cast<const uint2*>(c->ranges.p),
                                     c->vals[cur], c->st, K, bg, out->color, out->alpha,
                                     c->pix_T, c->pix_last, out->visibility,
                                     compositing_px(c, tiles), record_staging(c),
                                     train ? tile_work : nullptr);
            if (train) {
                launch_tile_order(st, tile_work, tiles, tile_order);
                c->tile_order = tile_order;
            }
        }
        ck(cudaGetLastError(), "composite launch");
        mark(c, 5, true);
        c->g = *g;
        c->K = K;
        c->bg = make_float3(s->background[0], s->background[1], s->background[2]);
        c->tiles = tiles;
        c->instances = int(instances);
        c->visible = int(visible);
        c->sorted_buf = cur;
        c->sort_bits = bits;
        c->record_backward = s->record_backward_state != 0;
        c->geometry = geometry;
        c->fwd_depth = geometry ? out->median_depth : nullptr;
        c->fwd_normal = geometry ? out->normal : nullptr;
        c->have_forward = true;
        if (info) {
            info->instance_count = int(instances);
            info->visible_count = int(visible);
            info->depth_bits = depth_bits;
            info->tile_bits = tile_bits;
            info->tiles = tiles;
        }
    });
}

gs_status gs_backward(gs_context* c, const float* fwd_alpha, const int* fwd_radii,
                      const gs_loss_grads* dL, const gs_model_grads* grads,
                      const gs_structure_adam* adam, const gs_sh_adam* sh_adam) {
    return guarded(c, [&] {
        if (!c->have_forward)
            throw StateError("gsplat_b200: backward without a forward");
        if (!c->record_backward)
            throw StateError("gsplat_b200: cannot backpropagate an inference-only render");
        req(dL && dL->color, "color gradient required");
        req(fwd_radii, "forward radii required");
        const bool geo_grads = dL->median_depth != nullptr || dL->normal != nullptr;
        if (geo_grads && !c->geometry)
            throw StateError("gsplat_b200: median-depth / normal gradients need a forward that "
                             "rendered those channels (need_depth)");
        check_forward_sorts(c);
        (void)fwd_alpha;
        const gs_gaussians& g = c->g;
        if (sh_adam) {
            req(g.sh != nullptr, "fused SH Adam needs SH colours");
            req(sh_adam->parameter && sh_adam->first && sh_adam->packed && sh_adam->bounds,
                "fused SH Adam state incomplete");
            req(sh_adam->stride == g.sh_bases * 3 && sh_adam->stride <= 48,
                "fused SH Adam stride must equal sh_bases*3 (<= 48)");
        }
        if (adam)
            req(adam->means && adam->log_scales && adam->quaternions && adam->opacity_logits &&
                    adam->means_first && adam->means_second && adam->scales_first &&
                    adam->scales_second && adam->rotations_first && adam->rotations_second &&
                    adam->opacity_first && adam->opacity_second,
                "fused structure Adam state incomplete");
        cudaStream_t st = c->stream;
        if (c->instances <= 0 && !adam && !sh_adam)
            return; // nothing drawn: no gradient (pipeline.cu:657-658)
        GaussianState gst = c->st;
        if (geo_grads) {
            // per-Gaussian ray-plane and normal gradient scratch, zeroed once;
            // the per-Gaussian backward re-zeroes what it consumes
            const size_t n = size_t(c->g.count);
            if (n > c->geo_grad_cap) {
                const size_t cap = std::max(n + n / 4 + 1024, c->gauss_cap);
                c->geo_grad.ensure(cap * kGeoGradSlots * sizeof(float4), st, /*zero=*/true);
                c->geo_grad_cap = cap;
            }
            gst.geo_grad = reinterpret_cast<float4*>(c->geo_grad.p);
            gst.plane = c->plane;
            gst.normal = c->normal;
        }
        mark(c, 6, false);
        if (c->instances > 0 && geo_grads)
            launch_composite_backward_geometry(
                st, c->tiles, reinterpret_cast<const uint2*>(c->ranges.p), c->vals[c->sorted_buf],
                gst, c->K, c->bg, c->pix_T, c->pix_last, c->pix_dtdt, dL->color, dL->alpha,
                dL->densify_map, grads && grads->refine_weight ? 1 : 0, dL->median_depth,
                dL->normal, c->fwd_depth, c->fwd_normal);
        else if (c->instances > 0)
            launch_composite_backward(st, c->tiles, reinterpret_cast<const uint2*>(c->ranges.p),
                                      c->vals[c->sorted_buf], c->st, c->K, c->bg, c->pix_T,
                                      c->pix_last, dL->color, dL->alpha, dL->densify_map,
                                      grads && grads->refine_weight ? 1 : 0,
                                      compositing_px(c, c->tiles), record_staging(c),
                                      c->tile_order);
        ck(cudaGetLastError(), "composite backward launch");
        mark(c, 6, true);
        mark(c, 7, false);
        GradOutArgs out{};
        if (grads) {
            out.means = grads->means;
            out.scales = grads->scales;
            out.rotations = grads->rotations;
            out.opacities = grads->opacities;
            out.sh = grads->sh;
            out.colors = grads->colors;
            out.refine_weight = grads->refine_weight;
            out.densify_weight = grads->densify_weight;
            out.densify_weight_den = grads->densify_weight_den;
            out.activated = grads->activated;
        }
        StructureAdamArgs sa{};
        if (adam) {
            static_assert(sizeof(StructureAdamArgs) == sizeof(gs_structure_adam),
                          "structure Adam layout");
            std::memcpy(&sa, adam, sizeof(sa));
        }
        ShAdamArgs sha{};
        if (sh_adam) {
            sha.parameter = sh_adam->parameter;
            sha.lr = sh_adam->lr;
            sha.rest_lr = sh_adam->rest_lr;
            sha.beta1 = sh_adam->beta1;
            sha.beta2 = sh_adam->beta2;
            sha.correction1 = sh_adam->correction1;
            sha.correction2 = sh_adam->correction2;
            sha.epsilon = sh_adam->epsilon;
            sha.regularization = sh_adam->regularization_factor;
            sha.first = sh_adam->first;
            sha.packed = sh_adam->packed;
            sha.bounds = sh_adam->bounds;
            sha.stride = sh_adam->stride;
        }
        launch_gaussian_backward(st, g.count, g.means, g.log_scales, g.quaternions,
                                 g.opacity_logits, g.filter_3d, g.sh, g.sh_degree, g.sh_bases,
                                 c->K, gst, fwd_radii, out, adam ? &sa : nullptr,
                                 sh_adam ? &sha : nullptr, geo_grads);
        ck(cudaGetLastError(), "gaussian backward launch");
        mark(c, 7, true);
        c->ev_pending = c->timing;
    });
}

gs_status gs_device_status(gs_context* c) {
    return guarded(c, [&] {
        ck(cudaStreamSynchronize(c->stream), "status sync");
        unsigned word = 0;
        ck(cudaMemcpy(&word, device_error_word(c), sizeof(unsigned), cudaMemcpyDeviceToHost),
           "read error word");
        if (word)
            raise_timeout(c, word, "in work enqueued on this context");
    });
}

gs_status gs_debug_lookback_probe(gs_context* c, int which, unsigned spin_limit) {
    return guarded(c, [&] {
        req(which >= 0 && which <= 2,
            "probe: which must be 0 (scan), 1 (onesweep) or 2 (compositing staging)");
        req(spin_limit >= 1 && spin_limit <= (1u << 20), "probe: spin_limit must be in [1, 2^20]");
        char* scratch = c->probe.ensure(lookback_probe_bytes(), c->stream);
        // a word set before the probe belongs to earlier work: report that first
        ck(cudaStreamSynchronize(c->stream), "probe sync");
        unsigned before = 0;
        ck(cudaMemcpy(&before, device_error_word(c), sizeof(unsigned), cudaMemcpyDeviceToHost),
           "read error word");
        if (before)
            raise_timeout(c, before, "in work enqueued before the probe");
        if (which == 2)
            launch_stage_probe(c->stream, spin_limit, device_error_word(c));
        else
            launch_lookback_probe(c->stream, which, spin_limit, scratch, device_error_word(c));
        ck(cudaGetLastError(), "probe launch");
        ck(cudaStreamSynchronize(c->stream), "probe sync");
        unsigned word = 0;
        ck(cudaMemcpy(&word, device_error_word(c), sizeof(unsigned), cudaMemcpyDeviceToHost),
           "read error word");
        if (word)
            raise_timeout(c, word, which == 0   ? "in the scan probe"
                                   : which == 1 ? "in the onesweep probe"
                                                : "in the staging probe");
    });
}

gs_status gs_debug_composite_pairs(gs_context* c, float* color, float* alpha,
                                   unsigned long long* pairs_out) {
    return guarded(c, [&] {
        if (!c->have_forward)
            throw StateError("gsplat_b200: pair count without a forward");
        if (!c->record_backward || c->geometry)
            throw StateError("gsplat_b200: pair count needs a colour training forward");
        req(color && alpha && pairs_out, "invalid pair count arguments");
        check_forward_sorts(c);
        pairs_out[0] = pairs_out[1] = 0;
        if (c->instances <= 0)
            return;
        char* scratch = c->probe.ensure(std::max<size_t>(lookback_probe_bytes(), 256), c->stream);
        auto* dev = reinterpret_cast<unsigned long long*>(scratch);
        ck(cudaMemsetAsync(dev, 0, 2 * sizeof(unsigned long long), c->stream), "pair count reset");
        launch_composite_count_pairs(c->stream, c->tiles,
                                     reinterpret_cast<const uint2*>(c->ranges.p),
                                     c->vals[c->sorted_buf], c->st, c->K, c->bg, color, alpha,
                                     c->pix_T, c->pix_last, compositing_px(c, c->tiles), dev,
                                     record_staging(c));
        ck(cudaGetLastError(), "pair count launch");
        ck(cudaMemcpyAsync(pairs_out, dev, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           c->stream),
           "pair count read-back");
        ck(cudaStreamSynchronize(c->stream), "pair count sync");
    });
}

gs_status gs_set_schedule(gs_context* c, int pixels_per_thread) {
    return guarded(c, [&] {
        req(pixels_per_thread == 0 || pixels_per_thread == 1 || pixels_per_thread == 2 ||
                pixels_per_thread == 4 || pixels_per_thread == 8,
            "pixels_per_thread must be 0 (automatic), 1, 2, 4 or 8");
        c->pixels_per_thread = pixels_per_thread;
    });
}

gs_status gs_debug_draw_list(gs_context* c, unsigned long long* keys_out, unsigned* values_out,
                             unsigned* ranges_out) {
    return guarded(c, [&] {
        if (!c->have_forward)
            throw StateError("gsplat_b200: no forward");
        check_forward_sorts(c);
        const size_t I = size_t(c->instances);
        if (keys_out && I) {
            launch_compose_keys(c->stream, int(I),
                                reinterpret_cast<const unsigned*>(c->keys[c->sorted_buf]),
                                c->vals[c->sorted_buf], c->st.depth, keys_out);
            ck(cudaGetLastError(), "key export");
        }
        if (values_out && I)
            ck(cudaMemcpyAsync(values_out, c->vals[c->sorted_buf], I * 4,
                               cudaMemcpyDeviceToDevice, c->stream),
               "value export");
        if (ranges_out)
            ck(cudaMemcpyAsync(ranges_out, c->ranges.p, size_t(c->tiles) * 8,
                               cudaMemcpyDeviceToDevice, c->stream),
               "range export");
    });
}

gs_status gs_enable_stage_timing(gs_context* c, int enable) {
    return guarded(c, [&] {
        c->timing = enable != 0;
        c->ev_pending = false;
        for (double& v : c->acc_ms)
            v = 0.0;
        c->acc_steps = 0;
    });
}

gs_status gs_stage_times(gs_context* c, float* ms_out, int n) {
    return guarded(c, [&] {
        req(ms_out && n > 0, "null output");
        if (!c->timing)
            throw StateError("gsplat_b200: stage timing disabled");
        ck(cudaStreamSynchronize(c->stream), "timing sync");
        if (c->ev_pending) {
            harvest(c, c->ev_set);
            c->ev_pending = false;
        }
        for (int k = 0; k < n && k < 8; ++k)
            ms_out[k] = c->acc_steps ? float(c->acc_ms[k] / double(c->acc_steps)) : -1.f;
        if (n > 8)
            ms_out[8] = float(c->acc_steps);
    });
}

gs_status gs_exclusive_scan_u32(gs_context* c, const unsigned* in, unsigned* out, int n,
                                unsigned* total_out) {
    return guarded(c, [&] {
        req(n >= 0 && (n == 0 || (in && out)), "invalid scan arguments");
        if (n == 0) {
            if (total_out)
                ck(cudaMemsetAsync(total_out, 0, sizeof(unsigned), c->stream), "scan total");
            return;
        }
        c->scan_status.ensure(scan_status_bytes(n) + 256, c->stream);
        unsigned* counters = reinterpret_cast<unsigned*>(c->counters.p);
        // counters[3]: tile counter, [7]: total when the caller wants none, [2]: error word
        launch_scan(c->stream, n, in, nullptr, out,
                    reinterpret_cast<unsigned long long*>(c->scan_status.p), counters + 3,
                    total_out ? total_out : counters + 7, counters + 2);
        ck(cudaGetLastError(), "scan launch");
    });
}

gs_status gs_sort_pairs_u64(gs_context* c, const unsigned long long* keys_in,
                            const unsigned* vals_in, unsigned long long* keys_out,
                            unsigned* vals_out, size_t count, int begin_bit, int end_bit) {
    return guarded(c, [&] {
        req(count == 0 || (keys_in && vals_in && keys_out && vals_out), "invalid sort arguments");
        req(begin_bit >= 0 && end_bit <= 64 && begin_bit <= end_bit, "invalid sort bit range");
        req(count < (size_t(1) << 30), "sort count exceeds 2^30");
        if (count == 0)
            return;
        cudaStream_t st = c->stream;
        ensure_instances(c, count, 8);
        c->sort_status.ensure(std::max<size_t>(sort_status_bytes(c->inst_cap, 8), 256), st);
        c->have_forward = false; // the instance buffers are reused here
        ck(cudaMemcpyAsync(c->keys[0], keys_in, count * 8, cudaMemcpyDeviceToDevice, st), "sort in");
        ck(cudaMemcpyAsync(c->vals[0], vals_in, count * 4, cudaMemcpyDeviceToDevice, st), "sort in");
        unsigned* counters = reinterpret_cast<unsigned*>(c->counters.p);
        const unsigned n32 = unsigned(count);
        ck(cudaMemcpyAsync(counters + 6, &n32, sizeof(unsigned), cudaMemcpyHostToDevice, st),
           "sort count");
        const int cur = launch_radix_sort<unsigned long long>(
            st, c->keys, c->vals, count, counters + 6, begin_bit, end_bit,
            reinterpret_cast<unsigned*>(c->sort_hist.p),
            reinterpret_cast<unsigned*>(c->sort_status.p),
            reinterpret_cast<unsigned*>(c->sort_counters.p), counters + 2);
        ck(cudaGetLastError(), "sort launch");
        ck(cudaMemcpyAsync(keys_out, c->keys[cur], count * 8, cudaMemcpyDeviceToDevice, st),
           "sort out");
        ck(cudaMemcpyAsync(vals_out, c->vals[cur], count * 4, cudaMemcpyDeviceToDevice, st),
           "sort out");
        ck(cudaStreamSynchronize(st), "sort sync"); // n32 lives on the host stack
    });
}

gs_status gs_fused_l1_ssim(gs_context* c, const float* prediction, const float* target,
                           const float* mask, int width, int height, float ssim_weight,
                           float photometric_weight, float* grad_out, float* loss_out) {
    return guarded(c, [&] {
        req(prediction && target && grad_out, "invalid fused SSIM arguments");
        req(width > 10 && height > 10, "fused SSIM requires width and height > 10");
        float* partial = reinterpret_cast<float*>(
            c->loss.ensure(ssim_partial_floats(width, height) * sizeof(float), c->stream));
        ck(launch_fused_l1_ssim(c->stream, prediction, target, mask, width, height, ssim_weight,
                                photometric_weight, grad_out, loss_out, partial),
           "fused SSIM launch");
    });
}

gs_status gs_ssim_metric(gs_context* c, const float* prediction, const float* target,
                         const float* mask, int width, int height, float* out) {
    return guarded(c, [&] {
        req(prediction && target && out && width > 0 && height > 0, "invalid SSIM arguments");
        if (width <= 10 || height <= 10) {
            ck(cudaMemsetAsync(out, 0, sizeof(float), c->stream), "SSIM metric");
            return;
        }
        float* partial = reinterpret_cast<float*>(
            c->loss.ensure(ssim_partial_floats(width, height) * sizeof(float), c->stream));
        ck(launch_ssim_metric(c->stream, prediction, target, mask, width, height, out, partial),
           "SSIM metric launch");
    });
}

gs_status gs_forward_colors(gs_context* c, const float* colors, const gs_outputs* out) {
    return guarded(c, [&] {
        if (!c->have_forward)
            throw StateError("gsplat_b200: colour reuse without a forward");
        if (!c->record_backward)
            throw StateError("gsplat_b200: color reuse requires a training forward");
        if (!c->g.colors || c->g.sh)
            throw StateError("gsplat_b200: color reuse requires precomputed colors");
        req(colors && out && out->color && out->alpha, "invalid colour reuse arguments");
        check_forward_sorts(c);
        const int n = c->g.count;
        ck(launch_set_colors(c->stream, n, colors, c->st.rgb, c->st.rec), "colour slots");
        c->g.colors = colors;
        // empty tiles (ranges zeroed by the forward) composite the background
        launch_composite_forward(c->stream, c->tiles, reinterpret_cast<const uint2*>(c->ranges.p),
                                 c->vals[c->sorted_buf], c->st, c->K, c->bg, out->color,
                                 out->alpha, c->pix_T, c->pix_last, out->visibility,
                                 compositing_px(c, c->tiles), record_staging(c));
        ck(cudaGetLastError(), "colour reuse composite launch");
    });
}

gs_status gs_pruning_scores(gs_context* c, const float* image, int gaussian_pop,
                            float* scores) {
    return guarded(c, [&] {
        if (!c->have_forward)
            throw StateError("gsplat_b200: pruning scores without a forward");
        if (!c->record_backward)
            throw StateError("gsplat_b200: pruning scores need a forward that recorded its "
                             "per-pixel state (record_backward_state)");
        req(image && scores, "invalid pruning score arguments");
        check_forward_sorts(c);
        if (c->instances <= 0)
            return; // nothing drawn: no score
        ck(launch_pruning_scores(c->stream, c->tiles, reinterpret_cast<const uint2*>(c->ranges.p),
                                 c->vals[c->sorted_buf], c->st, c->K, c->pix_last, image,
                                 gaussian_pop ? 1 : 0, scores),
           "pruning score launch");
    });
}

gs_status gs_split_gaussians_mode(gs_context* c, const gs_split_args* a) {
    return guarded(c, [&] {
        req(a && a->count >= 0 && a->mode >= 0 && a->mode <= 3, "invalid split arguments");
        if (a->count == 0)
            return;
        req(a->parent_means && a->parent_log_scales && a->parent_opacity_logits &&
                a->parent_quaternions && a->child_means && a->child_log_scales &&
                a->child_opacity_logits && a->parents,
            "split needs the parent and child arrays and the parent indices");
        req(!(a->mode == 1 || a->mode == 2) || a->random_samples,
            "dense_tangent and igs_random splits need random samples");
        const SplitModeArgs k{a->parent_means, a->parent_log_scales, a->parent_opacity_logits,
                              a->parent_quaternions, a->child_means, a->child_log_scales,
                              a->child_opacity_logits, a->parents, a->random_samples,
                              a->screen_sizes, a->count, a->mode,
                              std::clamp(a->minimum_opacity, 1e-8f, 0.49f),
                              std::max(a->split_at_screen_size, 0.f),
                              std::clamp(a->split_opacity_k, 1e-4f, 1.f - 1e-4f)};
        ck(launch_split_mode(c->stream, k), "split launch");
    });
}

gs_status gs_adc_decay(gs_context* c, size_t count, float* log_scales, float* opacity_logits,
                       float opacity_decay, float scale_decay) {
    return guarded(c, [&] {
        req(count == 0 || (log_scales && opacity_logits), "invalid ADC decay arguments");
        const float scale_factor = std::max(1.f - scale_decay, 1e-6f);
        ck(launch_adc_decay(c->stream, log_scales, opacity_logits, count,
                            std::max(opacity_decay, 0.f), std::log(scale_factor)),
           "ADC decay launch");
    });
}

gs_status gs_select_rows(gs_context* c, int n, const unsigned char* keep, int* indices_out,
                         int* count_out) {
    return guarded(c, [&] {
        req(n >= 0 && count_out && (n == 0 || (keep && indices_out)),
            "invalid row selection arguments");
        unsigned* scratch = reinterpret_cast<unsigned*>(
            c->loss.ensure(select_rows_scratch_words(n) * sizeof(unsigned), c->stream));
        ck(launch_select_rows(c->stream, keep, n, indices_out, count_out, scratch),
           "row selection launch");
    });
}

gs_status gs_gather_rows(gs_context* c, int count, const int* indices, int arrays,
                         const void* const* src, void* const* dst, const size_t* row_bytes) {
    return guarded(c, [&] {
        req(count >= 0 && arrays >= 0 && arrays <= kMaxGatherArrays,
            "gather takes 0..32 arrays and count >= 0");
        if (count == 0 || arrays == 0)
            return;
        req(indices && src && dst && row_bytes, "invalid gather arguments");
        GatherRowsArgs g{};
        g.indices = indices;
        g.count = count;
        g.arrays = arrays;
        for (int a = 0; a < arrays; ++a) {
            req(src[a] && dst[a] && src[a] != dst[a], "gather arrays must be distinct and set");
            req(row_bytes[a] > 0 && row_bytes[a] % 4 == 0 && row_bytes[a] / 4 < (1u << 30),
                "gather row sizes must be positive multiples of 4 bytes");
            const int words = int(row_bytes[a] / 4);
            const bool vec4 = words % 4 == 0 &&
                              reinterpret_cast<uintptr_t>(src[a]) % 16 == 0 &&
                              reinterpret_cast<uintptr_t>(dst[a]) % 16 == 0;
            g.array[a] = GatherArray{src[a], dst[a], words, vec4 ? 1 : 0};
        }
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        ck(launch_gather_rows(c->stream, g, sms), "gather launch");
    });
}

gs_status gs_training_loss(gs_context* c, const gs_loss_images* im, const gs_loss_options* o,
                           const gs_loss_outputs* out) {
    return guarded(c, [&] {
        req(im && o && out, "invalid training loss arguments");
        req(im->width > 0 && im->height > 0, "training loss needs a non-empty image");
        req(im->color && im->target_color && out->grad_color && out->grad_alpha,
            "training loss needs colour, target colour and both gradient images");
        req(!o->mask_enabled || im->mask, "mask_enabled without a mask");
        req(!(o->mask_enabled && o->alpha_mode == 1 && o->match_alpha_weight > 0.f) || im->alpha,
            "transparent alpha mode needs the rendered alpha");
        req(!(o->depth_weight > 0.f) || (im->median_depth && im->target_depth),
            "the depth term needs median_depth and target_depth");
        req(!(o->normal_weight > 0.f) || (im->normal && im->target_normal),
            "the normal term needs normal and target_normal");
        const bool consistency = o->depth_normal_weight > 0.f && out->grad_depth && out->grad_normal;
        req(!consistency || (im->median_depth && im->normal && im->fx != 0.f && im->fy != 0.f),
            "depth-normal consistency needs median_depth, normal and the intrinsics");
        const bool fused = im->width > 10 && im->height > 10;
        const size_t loss_floats = image_loss_partial_floats(im->width, im->height);
        const size_t ssim_floats = fused ? ssim_partial_floats(im->width, im->height) : 0;
        float* scratch = reinterpret_cast<float*>(
            c->loss.ensure((loss_floats + ssim_floats) * sizeof(float), c->stream));
        const ImageLossImages kim{im->color, im->alpha, im->median_depth, im->normal,
                                  im->target_color, im->target_depth, im->target_normal,
                                  im->mask, im->width, im->height, im->fx, im->fy, im->cx,
                                  im->cy};
        const ImageLossOptions ko{o->depth_weight, o->normal_weight, o->depth_normal_weight,
                                  o->match_alpha_weight, o->geometry_epsilon, o->mask_enabled,
                                  o->alpha_mode, o->ai_prior};
        const ImageLossOutputs ko_out{out->grad_color, out->grad_alpha, out->grad_depth,
                                      out->grad_normal, out->terms};
        ck(launch_image_loss(c->stream, kim, ko, ko_out, fused ? 0.f : o->photometric_weight,
                             scratch),
           "training loss launch");
        if (fused) {
            const float ssim_weight = std::clamp(o->ssim_weight, 0.f, 1.f);
            ck(launch_fused_l1_ssim(c->stream, im->color, im->target_color,
                                    o->mask_enabled ? im->mask : nullptr, im->width, im->height,
                                    ssim_weight, o->photometric_weight, out->grad_color,
                                    out->terms, scratch + loss_floats),
               "fused SSIM launch");
        }
    });
}

gs_status gs_l1_loss(gs_context* c, const float* image, const float* target, int pixels,
                     float weight, float* grad_out, float* loss_out) {
    return guarded(c, [&] {
        req(image && target && grad_out && pixels > 0, "invalid L1 arguments");
        const size_t n = size_t(pixels) * 3;
        launch_l1(c->stream, image, target, n, weight / float(n), grad_out, loss_out);
        ck(cudaGetLastError(), "l1 launch");
    });
}

gs_status gs_adam(gs_context* c, float* param, const float* grad, float* first, float* second,
                  size_t n, float lr, float beta1, float beta2, float correction1,
                  float correction2, float epsilon, float clamp_min, float clamp_max) {
    return guarded(c, [&] {
        req(param && grad && first && second, "invalid Adam arguments");
        launch_adam(c->stream, param, grad, first, second, n, lr, beta1, beta2, correction1,
                    correction2, epsilon, clamp_min, clamp_max);
        ck(cudaGetLastError(), "adam launch");
    });
}

static DensifyStatsArgs stats_args(const gs_densify_stats* s) {
    req(s && s->grad_acc && s->count && s->max_screen && s->depth_acc && s->age,
        "densify statistics required");
    return {s->grad_acc, s->count, s->max_screen, s->err_num, s->err_den, s->depth_acc, s->age};
}

gs_status gs_densify_accumulate(gs_context* c, int n, const float* refine_weight,
                                const int* radii, const float* densify_weight,
                                const float* densify_weight_den, float inv_resolution,
                                const float* means, const float* depth_row_host,
                                const gs_densify_stats* stats) {
    return guarded(c, [&] {
        req(n >= 0 && radii && means && depth_row_host, "invalid densify accumulate arguments");
        const DensifyStatsArgs s = stats_args(stats);
        req(!densify_weight || (s.err_num && s.err_den), "error statistics arrays required");
        launch_densify_accumulate(c->stream, n, refine_weight, radii, densify_weight,
                                  densify_weight_den, inv_resolution, means, depth_row_host, s);
        ck(cudaGetLastError(), "densify accumulate launch");
    });
}

gs_status gs_accumulate_densification(gs_context* c, const gs_densify_accum* a) {
    return guarded(c, [&] {
        req(a && a->count_rows >= 0, "invalid densification accumulate arguments");
        if (a->count_rows == 0)
            return;
        req(a->refine_weight && a->radii && a->gradient && a->count && a->max_screen_radius &&
                a->priority,
            "densification accumulate needs the refine weight, radii and the four statistics");
        req(!a->require_visibility || a->visibility, "require_visibility needs the visibility");
        req(!a->geometry_gradient || a->max_geometry_gradient,
            "a geometry score needs its running-max array");
        req(a->view_index < 0 || (a->first_view && a->view_support),
            "view tracking needs first_view and view_support");
        req(!a->image_error || a->accumulated_error, "an image error needs its accumulator");
        static_assert(sizeof(DensifyAccumArgs) == sizeof(gs_densify_accum), "accumulate layout");
        DensifyAccumArgs k;
        std::memcpy(&k, a, sizeof(k));
        ck(launch_accumulate_densification(c->stream, k), "densification accumulate launch");
    });
}

gs_status gs_densify_features(gs_context* c, int n, const float* means, const float* log_scales,
                              const float* opacity_logits, const float* sh, int sh_stride,
                              const gs_densify_stats* stats, const float* center3_host,
                              float extent, const float* norm, float* features_out) {
    return guarded(c, [&] {
        req(n >= 0 && means && log_scales && opacity_logits && sh && center3_host &&
                features_out && extent > 0.f,
            "invalid densify feature arguments");
        launch_densify_features(c->stream, n, means, log_scales, opacity_logits, sh, sh_stride,
                                stats_args(stats), center3_host, extent, norm, features_out);
        ck(cudaGetLastError(), "densify features launch");
    });
}

gs_status gs_adc_decide(gs_context* c, int n, const float* log_scales, const float* opacity_logits,
                        const gs_densify_stats* stats, const gs_adc_params* p, int* action_out) {
    return guarded(c, [&] {
        req(n >= 0 && log_scales && opacity_logits && p && action_out, "invalid ADC arguments");
        AdcArgs a{p->grad_threshold, p->percent_dense, p->extent, p->prune_opacity,
                  p->prune_world_scale, p->prune_screen, p->densify};
        launch_adc_decide(c->stream, n, log_scales, opacity_logits, stats_args(stats), a,
                          action_out);
        ck(cudaGetLastError(), "adc decide launch");
    });
}

gs_status gs_proposal_policy(gs_context* c, int n, const float* logits, const int* fallback,
                             const gs_densify_stats* stats, float min_confidence,
                             int* action_out) {
    return guarded(c, [&] {
        req(n >= 0 && logits && fallback && action_out, "invalid policy arguments");
        launch_proposal_policy(c->stream, n, logits, fallback, stats_args(stats), min_confidence,
                               action_out);
        ck(cudaGetLastError(), "policy launch");
    });
}

gs_status gs_split_gaussians(gs_context* c, int count, const int* parents, int child0,
                             float* means, float* log_scales, const float* quaternions,
                             float* opacity_logits) {
    return guarded(c, [&] {
        req(count >= 0 && child0 >= 0 && (count == 0 || (parents && means && log_scales &&
                                                          quaternions && opacity_logits)),
            "invalid split arguments");
        launch_split(c->stream, count, parents, child0, means, log_scales, quaternions,
                     opacity_logits);
        ck(cudaGetLastError(), "split launch");
    });
}

int gs_mlp_param_count(void) { return mlp_param_count(); }

gs_status gs_mlp_forward(gs_context* c, int n, const float* features, const void* weights_bf16,
                         float* logits_out) {
    return guarded(c, [&] {
        req(n >= 0 && (n == 0 || (features && weights_bf16 && logits_out)),
            "invalid MLP forward arguments");
        launch_mlp_forward(c->stream, n, features, weights_bf16, logits_out);
        ck(cudaGetLastError(), "mlp forward launch");
    });
}

gs_status gs_mlp_train_step(gs_context* c, int n, const float* features, const int* labels,
                            const float* row_weights, const void* weights_bf16, float weight_sum,
                            float* grad_out, float* loss_out) {
    return guarded(c, [&] {
        req(n >= 0 && weight_sum > 0.f &&
                (n == 0 || (features && labels && row_weights && weights_bf16 && grad_out &&
                            loss_out)),
            "invalid MLP training arguments");
        launch_mlp_train(c->stream, n, features, labels, row_weights, weights_bf16,
                         1.f / weight_sum, grad_out, loss_out);
        ck(cudaGetLastError(), "mlp train launch");
    });
}

gs_status gs_mlp_adam(gs_context* c, float* master, void* weights_bf16, const float* grad,
                      float* first, float* second, float lr, float beta1, float beta2,
                      float correction1, float correction2, float epsilon) {
    return guarded(c, [&] {
        req(master && weights_bf16 && grad && first && second, "invalid MLP Adam arguments");
        launch_mlp_adam(c->stream, master, weights_bf16, grad, first, second, lr, beta1, beta2,
                        correction1, correction2, epsilon);
        ck(cudaGetLastError(), "mlp adam launch");
    });
}

} // extern "C"
