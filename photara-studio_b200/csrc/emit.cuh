// Duplicate-with-keys for one warp: the shared body of the single-view and
// the batched emit kernels.
//
// Reference behaviour followed:
//   emit_instances  third_party/splat_drender/src/render_forward.cu:144-194
// (the same tiles in the same walk order per Gaussian; keys here are tile ids
// only, the depth order coming from the order the Gaussians are taken in).
#pragma once

#include "common.cuh"

namespace gsb {

constexpr unsigned kColSkip = 0xffffffffu; // column step of a Gaussian walked again

// A Gaussian slot's tile grid and the global id of its view's first tile.
struct EmitView {
    int grid_x, grid_y;
    unsigned tile_base;
};

// Writes the instances of the Gaussians order[r], r in [r_begin, r_end),
// which are consecutive in depth order, so their instances fill one
// contiguous output range starting at st.offset[r_begin]. The warp takes
// them 32 at a time: their span records (span_of(slot), the preprocess's
// walk) become a list of columns in `cols` (32 * kSpanCols entries of this
// warp's shared memory), each a run of instances with tile ids start,
// start + step, ... (step 1 or the tile grid width), and the warp writes the
// range 32 consecutive instances at a time, coalesced: a lane finds its
// column from one ballot over the columns that start inside the window. A
// Gaussian whose walk does not fit a span record is one skipped column,
// walked again by the whole warp afterwards (a column per lane). Keys are
// view_of(slot).tile_base + tile id; count(key) sees every key written.
// Called by whole warps with warp-uniform r_begin / r_end.
template <int TW, int TH, typename SpanOf, typename ViewOf, typename Count>
__device__ __forceinline__ void emit_warp_range(int r_begin, int r_end,
                                                const unsigned* __restrict__ order,
                                                const GaussianState& st, SpanOf span_of,
                                                ViewOf view_of, unsigned* __restrict__ keys,
                                                unsigned* __restrict__ values,
                                                unsigned capacity, uint4* cols, Count count) {
    const unsigned full = 0xffffffffu;
    const unsigned lane = lane_id();
    for (int wr0 = r_begin; wr0 < r_end; wr0 += 32) { // warp-uniform
        const int r = wr0 + int(lane);
        unsigned i = 0, cnt = 0;
        uint4 sp = make_uint4(0u, 0u, 0u, 0u);
        if (r < r_end) {
            i = order[r];
            cnt = st.touched[i];
            sp = span_of(i);
        }
        const unsigned incl = warp_incl_scan(cnt);
        const unsigned e = incl - cnt; // lane's first instance in the 32 Gaussians' range
        const unsigned total = __shfl_sync(full, incl, 31);
        const unsigned gbase = st.offset[wr0];
        if (gbase >= capacity) // nothing further fits (the caller flags the overflow)
            break;
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
            const EmitView vw = view_of(i);
            const unsigned gx = unsigned(vw.grid_x);
            const unsigned u_min = sp.x & 0xfffu;
            const unsigned v_base = (sp.x >> 12) & 0xfffu;
            const bool along_x = (sp.x >> 27) & 1u;
            const unsigned step = along_x ? gx : 1u;
            unsigned first = e;
#pragma unroll
            for (int c = 0; c < kSpanCols; ++c) {
                const unsigned word = c < 2 ? sp.y : (c < 4 ? sp.z : sp.w);
                const unsigned f = (word >> (16 * (c & 1))) & 0xffffu;
                if (f >> 8) {
                    const unsigned tu = u_min + unsigned(c);
                    const unsigned tv = v_base + (f & 0xffu);
                    const unsigned tile0 =
                        vw.tile_base + (along_x ? tv * gx + tu : tu * gx + tv);
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
                    count(tile);
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
            const EmitView gv = view_of(gi);
            TileWalk w;
            unsigned k0 = 0;
            if (walk_setup<TW, TH>(st.mean2d[gi], st.conic[gi], gv.grid_x, gv.grid_y, w)) {
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
                            const unsigned tile =
                                gv.tile_base +
                                walk_tile_id(w, u0 + int(c), c_vmin + int(p - (c_end - c_len)));
                            keys[ge + k] = tile;
                            values[ge + k] = gi;
                            count(tile);
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
                    count(0xffffffffu);
                }
        }
    }
}

} // namespace gsb
