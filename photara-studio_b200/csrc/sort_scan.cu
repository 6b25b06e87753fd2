// Hand-written device-wide scan and onesweep LSD radix sort (sm_100a).
//
// The reference calls CUB DeviceScan::InclusiveSum and
// DeviceRadixSort::SortPairs (third_party/splat_drender/src/pipeline.cu:231-311).
// Both are replaced here:
//  * scan: single-pass chained scan with decoupled look-back;
//  * sort: one histogram pass computing every digit histogram at once, then one
//    kernel per 8-bit digit that ranks its tile stably (warp ballot
//    multisplit), resolves its global digit offsets by decoupled look-back over
//    preceding tiles, stages the tile in shared memory in digit order and
//    writes coalesced digit runs (Adinets & Merrill, "Onesweep", 2022).
// Every look-back spin is bounded by kSpinLimit; on timeout the kernel sets
// the device error word and proceeds, so a broken invariant reports an error
// instead of hanging the GPU.
#include "common.cuh"
#include "kernels.h"

namespace gsb {

// ------------------------------------------------------------------ scan --
static_assert(kScanTile == kBlock * kScanItems, "scan tile = block x items per thread");

// Exclusive scan of u32 `in` (read through `index` when given: in[index[k]])
// into `out`; total written to *total. status: one u64 per tile, zeroed;
// tile_counter zeroed. With `groups`, the running sum is also cut into groups
// of 2^group_shift: groups[b] = the first element whose exclusive sum is at
// least b << group_shift, for every b <= total >> group_shift below
// group_cap (elements of value 0 never start a group after the first).
__global__ void __launch_bounds__(kBlock) scan_kernel(int n, const unsigned* __restrict__ in,
                                                      const unsigned* __restrict__ index,
                                                      unsigned* __restrict__ out,
                                                      unsigned long long* __restrict__ status,
                                                      unsigned* __restrict__ tile_counter,
                                                      unsigned* __restrict__ total,
                                                      unsigned* __restrict__ err,
                                                      unsigned spin_limit,
                                                      unsigned* __restrict__ groups,
                                                      int group_shift, unsigned group_cap) {
    __shared__ unsigned s_tile;
    __shared__ unsigned s_warp[8];
    __shared__ unsigned long long s_prefix;
    if (threadIdx.x == 0)
        s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const unsigned tile = s_tile;
    const size_t base = size_t(tile) * kScanTile + size_t(threadIdx.x) * kScanItems;
    unsigned v[kScanItems];
    unsigned sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const size_t idx = base + k;
        v[k] = idx < size_t(n) ? in[index ? index[idx] : idx] : 0u;
        sum += v[k];
    }
    unsigned tile_sum;
    const unsigned excl = block_excl_scan256(sum, s_warp, tile_sum);
    if (threadIdx.x < 32) {
        const unsigned long long prefix =
            warp_lookback(status, tile, tile_sum, err, kDevLookbackTimeout, spin_limit);
        if (threadIdx.x == 0) {
            s_prefix = prefix;
            if (size_t(tile + 1) * kScanTile >= size_t(n))
                *total = unsigned(prefix + tile_sum);
        }
    }
    __syncthreads();
    unsigned run = unsigned(s_prefix) + excl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const size_t idx = base + k;
        if (idx < size_t(n)) {
            out[idx] = run;
            if (groups) {
                // element idx + 1 starts every group whose first sum lies in
                // (run, run + v]
                if (idx == 0)
                    groups[0] = 0;
                const unsigned b_end = min((run + v[k]) >> group_shift, group_cap - 1u);
                for (unsigned b = (run >> group_shift) + 1; b <= b_end; ++b)
                    groups[b] = unsigned(idx + 1);
            }
        }
        run += v[k];
    }
}

// ------------------------------------------------------------------ sort --
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortItems = 12;
constexpr int kSortTile = kBlock * kSortItems; // 3072 keys per tile
constexpr int kWarpItems = 32 * kSortItems;    // 384 keys per warp
constexpr unsigned kStFlagAgg = 1u << 30;
constexpr unsigned kStFlagPre = 2u << 30;
constexpr unsigned kStMask = (1u << 30) - 1;

// Digit of `bits` (<= 8) bits starting at `shift`; bits above the sorted
// range never take part.
template <typename Key>
__device__ __forceinline__ unsigned digit_of(Key key, int shift, int bits = kRadixBits) {
    return unsigned(key >> shift) & ((1u << bits) - 1u);
}

// All digit histograms in one read of the keys. hist: [passes][256], zeroed.
// Per-block shared-memory histograms with one shared atomic per key and pass
// (a block's keys spread over the 256 bins, so conflicts are rare), flushed
// with one global atomic per non-empty bin. This replaced a ballot-per-bit
// warp aggregation that cost 8 ballots per key and pass (85 against 33 us for
// the 8.3M tile keys of a 1080p frame).
template <typename Key>
__global__ void __launch_bounds__(kBlock) radix_histogram_kernel(
    const Key* __restrict__ keys, const unsigned* __restrict__ count_ptr,
    int begin_bit, int end_bit, int passes, unsigned* __restrict__ hist) {
    __shared__ unsigned s_hist[8][kRadix];
    for (int k = threadIdx.x; k < 8 * kRadix; k += kBlock)
        (&s_hist[0][0])[k] = 0;
    __syncthreads();
    const size_t n = *count_ptr;
    const size_t stride = size_t(gridDim.x) * kBlock;
#pragma unroll 4
    for (size_t i = size_t(blockIdx.x) * kBlock + threadIdx.x; i < n; i += stride) {
        const Key key = keys[i];
        for (int p = 0; p < passes; ++p) {
            const int shift = begin_bit + p * kRadixBits;
            atomicAdd(&s_hist[p][digit_of(key, shift, min(kRadixBits, end_bit - shift))], 1u);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < passes * kRadix; k += kBlock) {
        const unsigned v = (&s_hist[0][0])[k];
        if (v)
            atomicAdd(&hist[k], v);
    }
}

// hist[p][d] -> exclusive offsets in place, one warp per pass.
__global__ void radix_offsets_kernel(unsigned* __restrict__ hist, int passes) {
    const int p = threadIdx.x >> 5;
    if (p >= passes)
        return;
    unsigned* h = hist + p * kRadix;
    unsigned carry = 0;
    for (int c = 0; c < kRadix; c += 32) {
        const unsigned v = h[c + lane_id()];
        const unsigned incl = warp_incl_scan(v);
        h[c + lane_id()] = carry + incl - v;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// One stable digit pass of kBits (<= 8) bits. status: [tiles][256] zeroed;
// tile_counter zeroed.
template <typename Key, int kBits>
__global__ void __launch_bounds__(kBlock, 4) onesweep_kernel(
    const Key* __restrict__ keys_in, const unsigned* __restrict__ vals_in,
    Key* __restrict__ keys_out, unsigned* __restrict__ vals_out,
    const unsigned* __restrict__ count_ptr, int shift,
    const unsigned* __restrict__ bin_offset,
    unsigned* __restrict__ status, unsigned* __restrict__ tile_counter,
    unsigned* __restrict__ err, unsigned spin_limit) {
    __shared__ unsigned s_tile;
    __shared__ unsigned s_whist[8][kRadix]; // per-warp digit counts, then warp prefix
    __shared__ unsigned s_tprefix[kRadix];  // tile-local digit start
    __shared__ unsigned s_gbase[kRadix];    // global start of the digit run - its tile start
    __shared__ unsigned s_warp[8];
    __shared__ Key s_keys[kSortTile];
    __shared__ unsigned s_vals[kSortTile];

    const unsigned n = *count_ptr;
    const unsigned tiles = (n + kSortTile - 1) / kSortTile;
    if (threadIdx.x == 0)
        s_tile = atomicAdd(tile_counter, 1u);
    for (int k = threadIdx.x; k < 8 * kRadix; k += kBlock)
        (&s_whist[0][0])[k] = 0;
    __syncthreads();
    const unsigned tile = s_tile;
    if (tile >= tiles)
        return;
    const int warp = threadIdx.x >> 5;
    const unsigned lane = lane_id();
    const size_t wbase = size_t(tile) * kSortTile + size_t(warp) * kWarpItems;

    // Only the last tile is partial; full tiles skip the bounds tests.
    const bool full = size_t(tile + 1) * kSortTile <= n;
    Key key[kSortItems];
    unsigned val[kSortItems];
    unsigned rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + size_t(k) * 32 + lane;
        const bool valid = full || idx < n;
        key[k] = valid ? keys_in[idx] : Key(~Key(0));
        val[k] = valid ? vals_in[idx] : 0u;
    }
    // Warp multisplit in index order (k-major, lane-minor == global order):
    // the lanes holding the same digit are found with one ballot per digit bit
    // (all items' ballots first, independent of the counters), then each
    // item's rank from the warp's running digit counts: the group's first
    // lane bumps the counter and every lane reads the old count from its
    // group's leader in one full-warp shuffle (a shuffle under each group's
    // own mask runs once per group).
    unsigned peers[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + size_t(k) * 32 + lane;
        const bool valid = full || idx < n;
        const unsigned d = digit_of(key[k], shift, kBits);
        unsigned p = full ? 0xffffffffu : __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < kBits; ++b) {
            const bool bit = (d >> b) & 1u;
            const unsigned vote = __ballot_sync(0xffffffffu, bit);
            p &= bit ? vote : ~vote;
        }
        peers[k] = p;
    }
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + size_t(k) * 32 + lane;
        const bool valid = full || idx < n;
        const unsigned d = digit_of(key[k], shift, kBits);
        const unsigned leader = peers[k] ? unsigned(__ffs(peers[k]) - 1) : lane;
        unsigned prior = 0;
        if (valid && lane == leader) {
            prior = s_whist[warp][d];
            s_whist[warp][d] = prior + __popc(peers[k]);
        }
        prior = __shfl_sync(0xffffffffu, prior, int(leader));
        rank[k] = valid ? prior + __popc(peers[k] & lanemask_lt()) : 0u;
        __syncwarp();
    }
    __syncthreads();
    // Thread d owns digit d: warp prefix, tile count, look-back.
    const unsigned d = threadIdx.x;
    unsigned cnt = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const unsigned c = s_whist[w][d];
        s_whist[w][d] = cnt;
        cnt += c;
    }
    unsigned* st = status + size_t(tile) * kRadix + d;
    unsigned excl = 0;
    if (tile == 0) {
        st_relaxed(st, kStFlagPre | cnt);
    } else {
        st_relaxed(st, kStFlagAgg | cnt);
        int pred = int(tile) - 1;
        unsigned spins = 0;
        while (pred >= 0) {
            const unsigned s = ld_relaxed(status + size_t(pred) * kRadix + d);
            const unsigned flag = s >> 30;
            if (flag == 0) {
                if (++spins > spin_limit) {
                    atomicOr(err, kDevLookbackTimeout);
                    break;
                }
                continue;
            }
            excl += s & kStMask;
            if (flag == 2)
                break;
            --pred;
        }
        st_relaxed(st, kStFlagPre | (excl + cnt));
    }
    unsigned tile_total;
    const unsigned tp = block_excl_scan256(cnt, s_warp, tile_total);
    s_tprefix[d] = tp;
    s_gbase[d] = bin_offset[d] + excl - tp;
    __syncthreads();
    // Stage the tile in digit order.
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const size_t idx = wbase + size_t(k) * 32 + lane;
        if (full || idx < n) {
            const unsigned dk = digit_of(key[k], shift, kBits);
            const unsigned pos = s_tprefix[dk] + s_whist[warp][dk] + rank[k];
            s_keys[pos] = key[k];
            s_vals[pos] = val[k];
        }
    }
    __syncthreads();
    for (unsigned pos = threadIdx.x; pos < tile_total; pos += kBlock) {
        const Key kk = s_keys[pos];
        const unsigned out = s_gbase[digit_of(kk, shift, kBits)] + pos;
        if (out < n) { // always true unless a look-back gave up (error word set)
            keys_out[out] = kk;
            vals_out[out] = s_vals[pos];
        }
    }
}

size_t scan_status_bytes(int n) {
    const size_t tiles = (size_t(n) + kScanTile - 1) / kScanTile;
    return tiles * sizeof(unsigned long long);
}

void launch_scan(cudaStream_t s, int n, const unsigned* in, const unsigned* index, unsigned* out,
                 unsigned long long* status, unsigned* tile_counter, unsigned* total,
                 unsigned* err, bool zeroed, unsigned* groups, int group_shift,
                 unsigned group_cap) {
    if (n <= 0)
        return;
    const int tiles = (n + kScanTile - 1) / kScanTile;
    if (!zeroed) {
        cudaMemsetAsync(status, 0, size_t(tiles) * sizeof(unsigned long long), s);
        cudaMemsetAsync(tile_counter, 0, sizeof(unsigned), s);
    }
    scan_kernel<<<tiles, kBlock, 0, s>>>(n, in, index, out, status, tile_counter, total, err,
                                         kSpinLimit, groups, group_shift, group_cap);
}

int radix_passes(int bits) { return (bits + kRadixBits - 1) / kRadixBits; }

size_t sort_status_bytes(size_t count, int passes) {
    const size_t tiles = (count + kSortTile - 1) / kSortTile;
    return size_t(passes) * tiles * kRadix * sizeof(unsigned);
}

int sort_tile_count(size_t count) { return int((count + kSortTile - 1) / kSortTile); }

// Sorts (keys, vals) of `count` elements (count also on device at count_dev)
// on bits [begin_bit, end_bit). Ping-pongs between the two buffers; returns
// the index (0 or 1) of the buffer holding the result.
template <typename Key>
int launch_radix_sort(cudaStream_t s, Key* keys[2], unsigned* vals[2], size_t count,
                      const unsigned* count_dev, int begin_bit, int end_bit, unsigned* hist,
                      unsigned* status, unsigned* tile_counters, unsigned* err,
                      bool hist_ready, bool zeroed) {
    const int passes = radix_passes(end_bit - begin_bit);
    if (count <= 1 || passes <= 0)
        return 0;
    const int tiles = sort_tile_count(count);
    if (!zeroed) {
        cudaMemsetAsync(status, 0, sort_status_bytes(count, passes), s);
        cudaMemsetAsync(tile_counters, 0, size_t(passes) * sizeof(unsigned), s);
    }
    if (!hist_ready) {
        if (!zeroed)
            cudaMemsetAsync(hist, 0, size_t(passes) * kRadix * sizeof(unsigned), s);
        const int hist_blocks = min(tiles, 148 * 4);
        radix_histogram_kernel<Key>
            <<<hist_blocks, kBlock, 0, s>>>(keys[0], count_dev, begin_bit, end_bit, passes, hist);
    }
    radix_offsets_kernel<<<1, 32 * passes, 0, s>>>(hist, passes);
    int cur = 0;
    for (int p = 0; p < passes; ++p) {
        const int shift = begin_bit + p * kRadixBits;
        const int bits = min(kRadixBits, end_bit - shift);
        auto pass = [&](auto kernel) {
            kernel<<<tiles, kBlock, 0, s>>>(keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1],
                                            count_dev, shift, hist + p * kRadix,
                                            status + size_t(p) * tiles * kRadix,
                                            tile_counters + p, err, kSpinLimit);
        };
        switch (bits) {
        case 1: pass(onesweep_kernel<Key, 1>); break;
        case 2: pass(onesweep_kernel<Key, 2>); break;
        case 3: pass(onesweep_kernel<Key, 3>); break;
        case 4: pass(onesweep_kernel<Key, 4>); break;
        case 5: pass(onesweep_kernel<Key, 5>); break;
        case 6: pass(onesweep_kernel<Key, 6>); break;
        case 7: pass(onesweep_kernel<Key, 7>); break;
        default: pass(onesweep_kernel<Key, 8>); break;
        }
        cur ^= 1;
    }
    return cur;
}

namespace {
constexpr size_t align16(size_t v) { return (v + 15) / 16 * 16; }
} // namespace

size_t lookback_probe_bytes() {
    // counters, then the larger of the two probes' buffers: the scan's input,
    // output and two status words, or the sort's keys and values in and out,
    // two tiles of status words and the digit offsets
    const size_t scan = align16(2 * kScanTile * 4) * 2 + align16(2 * 8);
    const size_t sort = align16(2 * kSortTile * 4) * 4 + align16(2 * kRadix * 4) + align16(kRadix * 4);
    return align16(16) + (scan > sort ? scan : sort);
}

// One block of the scan kernel (which == 0) or of an 8-bit onesweep pass
// (which == 1) over two tiles of zeros, with its tile counter starting at 1:
// the block takes tile 1, and tile 0 is never published, so its look-back
// waits for a predecessor that nothing sets until `spin_limit` re-reads have
// passed and then sets kDevLookbackTimeout in *err. Every access stays inside
// `scratch` (lookback_probe_bytes(), zeroed here): the input and output of
// both tiles and the status words of tiles 0 and 1.
void launch_lookback_probe(cudaStream_t s, int which, unsigned spin_limit, char* scratch,
                           unsigned* err) {
    cudaMemsetAsync(scratch, 0, lookback_probe_bytes(), s);
    char* p = scratch;
    auto take = [&](size_t bytes) {
        char* q = p;
        p += align16(bytes);
        return q;
    };
    unsigned* counter = reinterpret_cast<unsigned*>(take(16)); // [0] tile counter [1] count
    unsigned* count = counter + 1;                              // [2] scan total
    unsigned* total = counter + 2;
    // pageable host source: the copy is staged before cudaMemcpyAsync returns
    const unsigned init[2] = {1u, 2u * kSortTile};
    cudaMemcpyAsync(counter, init, sizeof(init), cudaMemcpyHostToDevice, s);
    if (which == 0) {
        unsigned* in = reinterpret_cast<unsigned*>(take(2 * kScanTile * 4));
        unsigned* out = reinterpret_cast<unsigned*>(take(2 * kScanTile * 4));
        auto* status = reinterpret_cast<unsigned long long*>(take(2 * 8));
        scan_kernel<<<1, kBlock, 0, s>>>(2 * kScanTile, in, nullptr, out, status, counter, total,
                                         err, spin_limit, nullptr, 0, 0u);
    } else {
        unsigned* keys_in = reinterpret_cast<unsigned*>(take(2 * kSortTile * 4));
        unsigned* vals_in = reinterpret_cast<unsigned*>(take(2 * kSortTile * 4));
        unsigned* keys_out = reinterpret_cast<unsigned*>(take(2 * kSortTile * 4));
        unsigned* vals_out = reinterpret_cast<unsigned*>(take(2 * kSortTile * 4));
        unsigned* status = reinterpret_cast<unsigned*>(take(2 * kRadix * 4));
        unsigned* offsets = reinterpret_cast<unsigned*>(take(kRadix * 4));
        // every key is 0: the block's 3,072 keys go to output positions below
        // its tile's prefix (0 once the wait gives up), all inside [0, 6144)
        onesweep_kernel<unsigned, 8><<<1, kBlock, 0, s>>>(keys_in, vals_in, keys_out, vals_out,
                                                          count, 0, offsets, status, counter,
                                                          err, spin_limit);
    }
}

template int launch_radix_sort<unsigned>(cudaStream_t, unsigned* [2], unsigned* [2], size_t,
                                         const unsigned*, int, int, unsigned*, unsigned*,
                                         unsigned*, unsigned*, bool, bool);
template int launch_radix_sort<unsigned long long>(cudaStream_t, unsigned long long* [2],
                                                   unsigned* [2], size_t, const unsigned*, int,
                                                   int, unsigned*, unsigned*, unsigned*,
                                                   unsigned*, bool, bool);

} // namespace gsb
