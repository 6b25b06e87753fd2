// Shared device helpers and the per-context device state layout.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "splat_math.cuh"

namespace gsb {

constexpr int kBlock = 256;

// Device-side error word set by bounded waits and capacity guards; the host
// reads it after a step and turns it into a status.
enum DeviceError : unsigned {
    kDevOk = 0,
    kDevLookbackTimeout = 1u,
    kDevCapacity = 2u,
    kDevStageTimeout = 4u, // a compositing CTA's wait for its staged Gaussians gave up
};

// The compositing inputs of one Gaussian in one 64-byte record (four per
// TMA gather): conic and opacity, colour and clamp bits, centre, alpha box.
// Written by the preprocess next to the per-field arrays; the single-view
// compositing kernels stage it into shared memory with tile::gather4 copies.
// The last 16 bytes, which the compositing kernels do not read, hold the
// preprocess's tile walk in compact form (TileSpans) for the instance emit.
struct __align__(16) SplatRec {
    float4 co;      // conic (xx, xy, yy), opacity * coefficient
    float4 rgb;     // colour; w holds the clamp bits
    float2 xy;      // pixel-space centre
    ushort4 bounds; // [x0, x1) [y0, y1) pixel box of the alpha >= 1/255 ellipse
    uint4 spans;    // TileSpans encoding of the tile walk
};
static_assert(sizeof(SplatRec) == 64, "one TMA row per record");

// Per-Gaussian forward state (structure of arrays, one slot per Gaussian).
struct GaussianState {
    float2* mean2d;     // pixel-space centre
    float4* conic;      // inverse screen covariance (xx, xy, yy), opacity * coef
    float4* rgb;        // SH colour; w holds the clamp bits as an int
    unsigned* depth;    // radial depth as ordered float bits
    unsigned* touched;  // tiles overlapped
    unsigned* offset;   // exclusive scan of touched
    ushort4* bounds;    // [x0,x1) [y0,y1) pixel box of the alpha >= 1/255 ellipse
    float4* grad;       // 3 float4 per Gaussian, see GradSlot
    float4* plane;      // ray plane (depth over screen offset, peak distance, 1/sigma);
                        // NULL unless the median-depth channel is rendered
    float4* normal;     // camera-space footprint normal (w unused); with plane
    float4* geo_grad;   // 2 float4 per Gaussian, see kGeoGradSlots; NULL unless the
                        // median-depth / normal channels are differentiated
    SplatRec* rec;      // packed compositing inputs (NULL: not written)
    uint4* spans;       // the tile walk's span records where no SplatRec holds them
                        // (NULL: not written)
};

// Geometry-channel backward scratch per Gaussian, 2 x float4 (32 B), zeroed
// once and re-zeroed by the per-Gaussian backward that consumes it:
//  [0] dL/d ray plane (x, y: screen slopes, z: peak distance, w: 1/sigma)
//  [1] dL/d footprint normal (x, y, z), w unused
constexpr int kGeoGradSlots = 2;

// Backward scratch per Gaussian, 3 x float4 (48 B):
//  [0] dL/dconic.x, dL/dconic.y (half of off-diagonal), dL/dconic.z, dL/dopacity*coef
//  [1] dL/dmean2d.x, dL/dmean2d.y, refine magnitude, densify numerator
//  [2] dL/dcolor r, g, b, densify denominator
constexpr int kGradSlots = 3;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive warp scan of u32.
__device__ __forceinline__ unsigned warp_incl_scan(unsigned v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned n = __shfl_up_sync(0xffffffffu, v, o);
        if (int(lane_id()) >= o)
            v += n;
    }
    return v;
}

// Exclusive block scan of one u32 per thread for a 256-thread block.
// `warp_tot` must hold 8 u32 of shared memory. Returns the exclusive prefix;
// `total` receives the block sum.
__device__ __forceinline__ unsigned block_excl_scan256(unsigned v, unsigned* warp_tot,
                                                       unsigned& total) {
    const unsigned incl = warp_incl_scan(v);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 31)
        warp_tot[w] = incl;
    __syncthreads();
    unsigned base = 0, sum = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const unsigned t = warp_tot[k];
        base += (k < w) ? t : 0u;
        sum += t;
    }
    total = sum;
    __syncthreads();
    return base + incl - v;
}

// Relaxed device-scope load / store used by the decoupled look-back scans.
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned* p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Iteration limit of every spin in this library; a wait that reaches it sets
// the device error word and gives up instead of hanging the GPU.
constexpr unsigned kSpinLimit = 1u << 22;

// Decoupled look-back status words of the single-pass scans: flag in the top
// two bits (0 not ready, 1 tile aggregate, 2 inclusive prefix), value below.
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPre = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

// Exclusive prefix of tile `tile` (sum of the values of tiles 0 .. tile-1),
// called by all 32 lanes of one warp; publishes the tile's aggregate first
// and its inclusive prefix last. The look-back reads windows of 32
// predecessors (lane l reads tile end - l): the window's nearest inclusive
// prefix ends the walk, and it and the aggregates after it are added in one
// warp sum; tiles before tile 0 read as an inclusive prefix of 0. A window
// with a tile not yet ready is re-read, at most `spin_limit` times, after which
// err gets `timeout_bit` and the prefix found so far is returned.
__device__ __forceinline__ unsigned long long warp_lookback(unsigned long long* status,
                                                            unsigned tile,
                                                            unsigned long long tile_sum,
                                                            unsigned* err, unsigned timeout_bit,
                                                            unsigned spin_limit = kSpinLimit) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long prefix = 0;
    if (tile == 0) {
        if (lane == 0)
            st_relaxed64(&status[0], kFlagPre | tile_sum);
        return 0;
    }
    if (lane == 0)
        st_relaxed64(&status[tile], kFlagAgg | tile_sum);
    int end = int(tile) - 1;
    unsigned spins = 0;
    while (true) {
        const int pred = end - int(lane);
        const unsigned long long sv = pred >= 0 ? ld_relaxed64(&status[pred]) : kFlagPre;
        const unsigned flag = unsigned(sv >> 62);
        if (__any_sync(0xffffffffu, flag == 0)) {
            if (++spins > spin_limit) {
                if (lane == 0)
                    atomicOr(err, timeout_bit);
                break;
            }
            continue;
        }
        const unsigned pre = __ballot_sync(0xffffffffu, flag == 2);
        const unsigned first = pre ? unsigned(__ffs(pre) - 1) : 31u;
        unsigned long long v = lane <= first ? (sv & kValMask) : 0ull;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, off);
        prefix += v;
        if (pre)
            break;
        end -= 32;
    }
    if (lane == 0) {
        __threadfence();
        st_relaxed64(&status[tile], kFlagPre | (prefix + tile_sum));
    }
    return prefix;
}

} // namespace gsb
