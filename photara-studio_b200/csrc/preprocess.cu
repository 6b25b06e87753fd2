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
// heavy and light stretches of the depth order cost the same; a
// warp's Gaussians fill one contiguous output range. The warp takes them 32 at
// a time: their span records (the preprocess's walk, kept in the splat
// records) become a list of columns in shared memory, each a run of instances
// with tile ids start, start + step, ... (step 1 or the tile grid width), and
// the warp writes the range 32 consecutive instances at a time, coalesced: a
// lane finds its column from one ballot over the columns that start inside
// the window. A Gaussian whose walk does not fit a span record is one skipped
// column, walked again by the whole warp afterwards (a column per lane). Keys
// are tile ids; the following radix sort's digit histograms are counted here.
// Threads per emit CTA.
constexpr int kEmitBlock = 256;
constexpr unsigned kColSkip = 0xffffffffu; // column step of a Gaussian walked again

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
    const unsigned full = 0xffffffffu;
    const unsigned lane = lane_id();
    const int warp = int(threadIdx.x >> 5);
    uint4* cols = s_col[warp];
    const unsigned g = blockIdx.x * (kEmitBlock / 32) + unsigned(warp);
    const int r_begin = g < group_count ? int(groups[g]) : visible;
    const int r_end = g + 1 < group_count ? int(groups[g + 1]) : visible;
    for (int wr0 = r_begin; wr0 < r_end; wr0 += 32) { // warp-uniform
        const int r = wr0 + int(lane);
        unsigned i = 0, cnt = 0;
        uint4 sp = make_uint4(0u, 0u, 0u, 0u);
        if (r < r_end) {
            i = order[r];
            cnt = st.touched[i];
            sp = __ldg(&st.rec[i].spans);
        }
        const unsigned incl = warp_incl_scan(cnt);
        const unsigned e = incl - cnt; // lane's first instance in the 32 Gaussians' range
        const unsigned total = __shfl_sync(full, incl, 31);
        const unsigned gbase = st.offset[wr0];
        const bool walk = cnt > 0 && (sp.x & kSpanWalk);
        unsigned ncol = walk ? 1u : 0u;
        if (cnt > 0 && !walk) {
#pragma unroll
            for (int c = 0; c < kSpanCols; ++c) {
                const unsigned word = c < 2 ? sp.y : (c < 4 ? sp.z : sp.w);
                ncol += ((word >> (16 * (c & 1) + 8)) & 0xffu) ? 1u : 0u;
            }
        }
        const unsigned cincl = warp_incl_scan(ncol);
        unsigned cb = cincl - ncol;
        const unsigned ncols = __shfl_sync(full, cincl, 31);
        __syncwarp(); // the previous 32 Gaussians' windows are done with the list
        if (walk) {
            cols[cb] = make_uint4(e, 0u, kColSkip, i);
        } else if (cnt > 0) {
            const unsigned u_min = sp.x & 0xfffu;
            const unsigned v_base = (sp.x >> 12) & 0xfffu;
            const bool along_x = (sp.x >> 27) & 1u;
            const unsigned step = along_x ? unsigned(grid_x) : 1u;
            unsigned first = e;
#pragma unroll
            for (int c = 0; c < kSpanCols; ++c) {
                const unsigned word = c < 2 ? sp.y : (c < 4 ? sp.z : sp.w);
                const unsigned f = (word >> (16 * (c & 1))) & 0xffffu;
                if (f >> 8) {
                    const unsigned tu = u_min + unsigned(c);
                    const unsigned tv = v_base + (f & 0xffu);
                    const unsigned tile0 = along_x ? tv * unsigned(grid_x) + tu
                                                   : tu * unsigned(grid_x) + tv;
                    cols[cb++] = make_uint4(first, tile0, step, i);
                    first += f >> 8;
                }
            }
        }
        __syncwarp();
        // c0: the column holding instance w0 (the last one starting at or before it)
        unsigned c0 = 0;
        for (unsigned w0 = 0; w0 < total; w0 += 32) {
            const unsigned cand = c0 + 1 + lane; // columns starting in (w0, w0 + 32]
            unsigned bit = 0;
            if (cand < ncols) {
                const unsigned s0 = cols[cand].x;
                if (s0 <= w0 + 32)
                    bit = 1u << (s0 - w0 - 1);
            }
            const unsigned starts = __reduce_or_sync(full, bit);
            const unsigned own = c0 + __popc(starts & ((1u << lane) - 1u));
            c0 += __popc(starts);
            const unsigned q = w0 + lane;
            if (q < total) {
                const uint4 col = cols[own];
                const unsigned pos = gbase + q;
                if (col.z != kColSkip && pos < capacity) {
                    const unsigned tile = col.y + (q - col.x) * col.z;
                    keys[pos] = tile;
                    values[pos] = col.w;
                    dc.count(tile, bits);
                }
            }
        }
        // Gaussians whose walk did not fit a span record: the lanes take 32
        // columns at a time, and the chunk's instances are written 32 at a
        // time, each lane finding its column by a binary search over the
        // lanes' inclusive column ends.
        unsigned pending = __ballot_sync(full, walk);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            const unsigned gi = __shfl_sync(full, i, src);
            const unsigned gcnt = __shfl_sync(full, cnt, src);
            const unsigned ge = gbase + __shfl_sync(full, e, src);
            TileWalk w;
            unsigned k0 = 0;
            if (walk_setup(st.mean2d[gi], st.conic[gi], grid_x, grid_y, w)) {
                for (int u0 = w.u_min; u0 < w.u_max && k0 < gcnt; u0 += 32) {
                    const int tu = u0 + int(lane);
                    int v_min = 0, v_max = 0;
                    if (tu < w.u_max)
                        walk_column(w, tu, v_min, v_max);
                    const unsigned len = v_max > v_min ? unsigned(v_max - v_min) : 0u;
                    const unsigned lincl = warp_incl_scan(len);
                    const unsigned chunk = __shfl_sync(full, lincl, 31);
                    for (unsigned p0 = 0; p0 < chunk; p0 += 32) {
                        const unsigned p = p0 + lane;
                        // c: the number of columns ending at or before p
                        unsigned c = 0;
#pragma unroll
                        for (unsigned step = 16; step; step >>= 1)
                            if (__shfl_sync(full, lincl, int(c + step - 1)) <= p)
                                c += step;
                        const unsigned c_end = __shfl_sync(full, lincl, int(c));
                        const unsigned c_len = __shfl_sync(full, len, int(c));
                        const int c_vmin = __shfl_sync(full, v_min, int(c));
                        const unsigned k = k0 + p;
                        if (p < chunk && k < gcnt && ge + k < capacity) {
                            const unsigned tile = walk_tile_id(
                                w, u0 + int(c), c_vmin + int(p - (c_end - c_len)));
                            keys[ge + k] = tile;
                            values[ge + k] = gi;
                            dc.count(tile, bits);
                        }
                    }
                    k0 += chunk;
                }
            }
            // The walk re-runs the counting walk on the stored state and must
            // agree; should it ever come up short, the unused slots get a
            // sentinel key whose sorted bits exceed every tile id (the sort
            // covers enough bits to hold the tile count) and which the range
            // pass ignores.
            for (unsigned k = k0 + lane; k < gcnt; k += 32)
                if (ge + k < capacity) {
                    keys[ge + k] = 0xffffffffu;
                    values[ge + k] = gi;
                    dc.count(0xffffffffu, bits);
                }
        }
    }
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
