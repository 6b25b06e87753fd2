// Per-Gaussian preprocess, duplicate-with-keys and tile-range kernels.
//
// Reference behaviour followed:
//   preprocess_gaussians  third_party/splat_drender/src/render_forward.cu:30-139
//   emit_instances        third_party/splat_drender/src/render_forward.cu:144-194
//   extract_packed_ranges third_party/splat_drender/src/render_forward.cu:196-212
// The draw order is (tile, depth bits, Gaussian index), the order both of the
// reference's sort paths produce (pipeline.cu:231-311). It is built in two
// stable radix sorts: visible Gaussians by depth bits (rebased on the frame's
// minimum so only the varying low bits are sorted; culled Gaussians get a
// sentinel that sorts last), then instances emitted in that depth order with
// their tile id as a 32-bit key and sorted on the tile bits only. Because the
// second sort is stable and its input is already in (depth, index) order, the
// result equals a full sort of the reference's 64-bit (tile << 32 | depth)
// keys with index tie-break; those keys are recomposed only for export.
#include <algorithm>

#include "emit.cuh"
#include "kernels.h"
#include "preprocess.cuh"

namespace gsb {

// One thread per Gaussian. Writes the forward state of visible Gaussians and
// zero tiles/radius for culled ones. Frame totals are reduced per warp, then
// per block in shared memory, with one set of global atomics per block.
template <bool kGeometry>
__global__ void __launch_bounds__(kBlock) preprocess_kernel(
    int n, const float* __restrict__ means, const float* __restrict__ log_scales,
    const float* __restrict__ quats, const float* __restrict__ logits,
    const float* __restrict__ filter_3d, const float* __restrict__ sh,
    const float* __restrict__ colors, int sh_degree, int sh_bases, const Camera K,
    GaussianState st, int* __restrict__ radii, unsigned* __restrict__ counters) {
    __shared__ unsigned s_tot[4]; // instances, visible, min / max depth bits
    if (threadIdx.x < 4)
        s_tot[threadIdx.x] = threadIdx.x == 2 ? 0xffffffffu : 0u;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned touched = 0, depth_bits = 0;
    if (i < n) {
        const PreResult r = preprocess_one<kTileW, kTileH, kGeometry>(
            i, size_t(i), means, log_scales, quats, logits, filter_3d, sh, colors, sh_degree,
            sh_bases, K, st);
        touched = r.touched;
        depth_bits = r.depth_bits;
        st.touched[i] = touched;
        radii[i] = r.radius;
    }
    const unsigned full = 0xffffffffu;
    const unsigned w_inst = __reduce_add_sync(full, touched);
    const unsigned w_vis = __popc(__ballot_sync(full, touched > 0));
    const unsigned w_min = __reduce_min_sync(full, touched > 0 ? depth_bits : 0xffffffffu);
    const unsigned w_max = __reduce_max_sync(full, depth_bits);
    if (lane_id() == 0 && w_vis) {
        atomicAdd(&s_tot[0], w_inst);
        atomicAdd(&s_tot[1], w_vis);
        atomicMin(&s_tot[2], w_min);
        atomicMax(&s_tot[3], w_max);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_tot[1]) {
        atomicAdd(&counters[0], s_tot[0]);
        atomicAdd(&counters[1], s_tot[1]);
        atomicMin(&counters[4], s_tot[2]);
        atomicMax(&counters[5], s_tot[3]);
    }
    if (i == 0)
        counters[6] = unsigned(n);
}

// The radix sort's digit histograms of the keys a kernel writes, counted as
// they are written (8-bit digits over key bits [0, bits), up to 4 passes):
// the sort then skips its own read of the keys. Per-block shared histograms,
// flushed with one global atomic per non-empty bin.
struct DigitCounter {
    unsigned (*h)[256];
    __device__ __forceinline__ void zero() {
        for (int k = threadIdx.x; k < 4 * 256; k += blockDim.x)
            (&h[0][0])[k] = 0;
    }
    __device__ __forceinline__ void count(unsigned key, int bits) {
        for (int p = 0, shift = 0; shift < bits; ++p, shift += 8) {
            const int b = min(8, bits - shift);
            atomicAdd(&h[p][(key >> shift) & ((1u << b) - 1u)], 1u);
        }
    }
    __device__ __forceinline__ void flush(unsigned* __restrict__ hist, int bits) {
        const int passes = (bits + 7) / 8;
        for (int k = threadIdx.x; k < passes * 256; k += blockDim.x) {
            const unsigned v = (&h[0][0])[k];
            if (v)
                atomicAdd(&hist[k], v);
        }
    }
};

// Depth sort input, compacted: the visible Gaussians (touched > 0) in index
// order, keyed by their depth bits rebased on the frame minimum, with their
// indices as values; the sort then orders only them. The compaction is an
// exclusive scan of the visibility flags with decoupled look-back (tiles of
// 2,048 Gaussians, eight consecutive per thread). The kernel also counts the
// sort's digit histograms of key bits [0, bits) into hist (zeroed by the
// caller), so the sort reads its keys once less. status: one u64 per tile,
// zeroed; tile_counter zeroed.
constexpr int kCompactItems = 8;
constexpr int kCompactTile = kBlock * kCompactItems;

__global__ void __launch_bounds__(kBlock) depth_compact_kernel(
    int n, GaussianState st, const unsigned* __restrict__ counters, unsigned* __restrict__ keys,
    unsigned* __restrict__ values, unsigned* __restrict__ hist,
    unsigned long long* __restrict__ status, unsigned* __restrict__ tile_counter,
    unsigned* __restrict__ err) {
    // The frame's depth range comes from the preprocess counters on the
    // device ([4] min, [5] max depth bits), so the kernel can run while the
    // host is still reading the draw counts back.
    const unsigned dmin = counters[4];
    const int bits = 32 - __clz(int(counters[5] - dmin + 1u));
    __shared__ unsigned s_hist[4][256];
    __shared__ unsigned s_warp[8];
    __shared__ unsigned s_tile, s_prefix;
    DigitCounter dc{s_hist};
    dc.zero();
    if (threadIdx.x == 0)
        s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const unsigned tile = s_tile;
    const int base = int(tile) * kCompactTile + int(threadIdx.x) * kCompactItems;
    unsigned vis = 0, cnt = 0;
#pragma unroll
    for (int k = 0; k < kCompactItems; ++k) {
        const int i = base + k;
        if (i < n && st.touched[i] > 0) {
            vis |= 1u << k;
            ++cnt;
        }
    }
    unsigned tile_sum;
    const unsigned excl = block_excl_scan256(cnt, s_warp, tile_sum);
    if (threadIdx.x < 32) {
        const unsigned long long prefix =
            warp_lookback(status, tile, tile_sum, err, kDevLookbackTimeout);
        if (threadIdx.x == 0)
            s_prefix = unsigned(prefix);
    }
    __syncthreads();
    unsigned out = s_prefix + excl;
#pragma unroll
    for (int k = 0; k < kCompactItems; ++k) {
        if ((vis >> k) & 1u) {
            const unsigned key = st.depth[base + k] - dmin;
            keys[out] = key;
            values[out] = unsigned(base + k);
            dc.count(key, bits);
            ++out;
        }
    }
    __syncthreads();
    dc.flush(hist, bits);
}

// Duplicate-with-keys. Warps take the visible Gaussians in depth order in
// groups of about S = 2^group_shift instances (a group is the Gaussians whose
// first instance falls in [g S, (g + 1) S), cut by the offset scan), so
// heavy and light stretches of the depth order cost the same, and expand
// their span records (emit_warp_range). Keys are tile ids; the following
// radix sort's digit histograms are counted here.
// Threads per emit CTA.
constexpr int kEmitBlock = 256;

__global__ void __launch_bounds__(kEmitBlock) emit_keys_kernel(
    int visible, unsigned group_count, const unsigned* __restrict__ groups,
    const unsigned* __restrict__ order, GaussianState st, int grid_x, int grid_y,
    unsigned* __restrict__ keys, unsigned* __restrict__ values, unsigned capacity, int bits,
    unsigned* __restrict__ hist) {
    // column: (first instance in the 32 Gaussians' range, first tile, tile step, Gaussian)
    __shared__ uint4 s_col[kEmitBlock / 32][32 * kSpanCols];
    __shared__ unsigned s_hist[4][256];
    DigitCounter dc{s_hist};
    dc.zero();
    __syncthreads();
    const int warp = int(threadIdx.x >> 5);
    const unsigned g = blockIdx.x * (kEmitBlock / 32) + unsigned(warp);
    const int r_begin = g < group_count ? int(groups[g]) : visible;
    const int r_end = g + 1 < group_count ? int(groups[g + 1]) : visible;
    emit_warp_range<kTileW, kTileH>(
        r_begin, r_end, order, st, [&](unsigned i) { return __ldg(&st.rec[i].spans); },
        [&](unsigned) { return EmitView{grid_x, grid_y, 0u}; }, keys, values, capacity,
        s_col[warp], [&](unsigned key) { dc.count(key, bits); });
    __syncthreads();
    dc.flush(hist, bits);
}

// Per-tile [start, end) from the sorted keys. ranges[] is zeroed beforehand.
__global__ void __launch_bounds__(kBlock) tile_ranges_kernel(
    int count, const unsigned* __restrict__ keys, uint2* __restrict__ ranges, unsigned tiles) {
    // Four consecutive keys per thread (one 16-byte load when whole) and the
    // key before them; a boundary between positions i-1 and i ends the range
    // of the key at i-1 and starts the range of the key at i.
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = 4 * t;
    if (i0 >= count)
        return;
    unsigned k[4];
    if (i0 + 4 <= count) {
        const uint4 v = reinterpret_cast<const uint4*>(keys)[t];
        k[0] = v.x;
        k[1] = v.y;
        k[2] = v.z;
        k[3] = v.w;
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            k[j] = i0 + j < count ? keys[i0 + j] : 0u;
    }
    unsigned prev = i0 > 0 ? keys[i0 - 1] : 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = i0 + j;
        if (i >= count)
            break;
        const unsigned tile = k[j];
        if (i == 0) {
            if (tile < tiles)
                ranges[tile].x = 0;
        } else if (tile != prev) {
            if (prev < tiles)
                ranges[prev].y = unsigned(i);
            if (tile < tiles)
                ranges[tile].x = unsigned(i);
        }
        if (i == count - 1 && tile < tiles)
            ranges[tile].y = unsigned(count);
        prev = tile;
    }
}

// Frame counters before the preprocess: instances, visible, min / max depth
// bits (the error word [2] is left for the host to read and clear).
__global__ void frame_counters_init_kernel(unsigned* __restrict__ counters) {
    if (threadIdx.x == 0) {
        counters[0] = 0;
        counters[1] = 0;
        counters[4] = 0xffffffffu;
        counters[5] = 0;
    }
}

void launch_frame_counters_init(cudaStream_t s, unsigned* counters) {
    frame_counters_init_kernel<<<1, 32, 0, s>>>(counters);
}

void launch_preprocess(cudaStream_t s, int n, const float* means, const float* log_scales,
                       const float* quats, const float* logits, const float* filter_3d,
                       const float* sh, const float* colors, int sh_degree, int sh_bases,
                       const Camera& K, const GaussianState& st, int* radii, unsigned* counters) {
    const int blocks = (n + kBlock - 1) / kBlock;
    // st.plane != NULL: the median-depth channel's ray planes and normals too
    if (st.plane)
        preprocess_kernel<true><<<blocks, kBlock, 0, s>>>(n, means, log_scales, quats, logits,
                                                          filter_3d, sh, colors, sh_degree,
                                                          sh_bases, K, st, radii, counters);
    else
        preprocess_kernel<false><<<blocks, kBlock, 0, s>>>(n, means, log_scales, quats, logits,
                                                           filter_3d, sh, colors, sh_degree,
                                                           sh_bases, K, st, radii, counters);
}

void launch_depth_compact(cudaStream_t s, int n, const GaussianState& st,
                          const unsigned* counters, unsigned* keys, unsigned* values,
                          unsigned* hist, unsigned long long* status, unsigned* tile_counter,
                          unsigned* err, bool zeroed) {
    if (n <= 0)
        return;
    const int tiles = (n + kCompactTile - 1) / kCompactTile;
    if (!zeroed) {
        cudaMemsetAsync(status, 0, size_t(tiles) * sizeof(unsigned long long), s);
        cudaMemsetAsync(tile_counter, 0, sizeof(unsigned), s);
    }
    depth_compact_kernel<<<tiles, kBlock, 0, s>>>(n, st, counters, keys, values, hist, status,
                                                  tile_counter, err);
}

// The reference's 64-bit (tile << 32 | depth bits) keys of the sorted list.
__global__ void __launch_bounds__(kBlock) compose_keys_kernel(
    int count, const unsigned* __restrict__ tiles, const unsigned* __restrict__ values,
    const unsigned* __restrict__ depth, unsigned long long* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count)
        out[i] = (static_cast<unsigned long long>(tiles[i]) << 32) | depth[values[i]];
}

void launch_compose_keys(cudaStream_t s, int count, const unsigned* tiles,
                         const unsigned* values, const unsigned* depth,
                         unsigned long long* out) {
    if (count > 0)
        compose_keys_kernel<<<(count + kBlock - 1) / kBlock, kBlock, 0, s>>>(count, tiles, values,
                                                                             depth, out);
}

void launch_emit_keys(cudaStream_t s, int visible, unsigned instances, const unsigned* groups,
                      int group_shift, const unsigned* order, const GaussianState& st,
                      int grid_x, int grid_y, unsigned* keys, unsigned* values,
                      unsigned capacity, int bits, unsigned* hist) {
    if (visible <= 0 || instances == 0)
        return;
    const unsigned group_count = emit_group_count(instances, group_shift);
    const unsigned warps = kEmitBlock / 32;
    const unsigned blocks = (group_count + warps - 1) / warps;
    emit_keys_kernel<<<blocks, kEmitBlock, 0, s>>>(visible, group_count, groups, order, st, grid_x,
                                                   grid_y, keys, values, capacity, bits, hist);
}

void launch_tile_ranges(cudaStream_t s, int count, const unsigned* keys, uint2* ranges,
                        int tiles) {
    if (count <= 0)
        return;
    // keys must be 16-byte aligned (the sort's buffers are)
    const int threads = (count + 3) / 4;
    tile_ranges_kernel<<<(threads + kBlock - 1) / kBlock, kBlock, 0, s>>>(count, keys, ranges,
                                                                          unsigned(tiles));
}

} // namespace gsb
