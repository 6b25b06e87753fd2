// Densification apply kernels: the four split operators of
// split_gaussians_kernel (photara/src/splat/cuda_ops.cu:1720-1845;
// SplitMode, ops.hpp:282), the ADC decay (adc_decay_kernel,
// cuda_ops.cu:1847-1861, with apply_adc_decay's host clamps at :3388-3400),
// and the row selection that prunes a model together with its optimizer
// state (select_training_rows_gpu, densification_adc_plus.cpp:68-77: every
// parameter, both Adam moments and the quantized SH-Adam rows re-indexed by
// the kept rows).
//
// The split and decay follow the reference's per-Gaussian expressions (the
// children must land on the same floats). The row selection is organised
// for the GPU: a stable stream compaction of the keep mask (per-block counts,
// one scan, per-warp ballots), then one launch that gathers every array of
// the model and its optimizer state in 16-byte words where the rows allow it,
// instead of one index_select per tensor.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace gsb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float sigmoid_ref(float v) { return 1.f / (1.f + expf(-v)); }

// Rotation of a local offset by the normalised quaternion (w, x, y, z):
// v + w t + q x t with t = 2 q x v.
__device__ __forceinline__ void rotate_by_quaternion(const float* raw, float x, float y, float z,
                                                     float& ox, float& oy, float& oz) {
    const float inverse_norm = rsqrtf(
        fmaxf(raw[0] * raw[0] + raw[1] * raw[1] + raw[2] * raw[2] + raw[3] * raw[3], 1e-20f));
    const float w = raw[0] * inverse_norm;
    const float qx = raw[1] * inverse_norm;
    const float qy = raw[2] * inverse_norm;
    const float qz = raw[3] * inverse_norm;
    const float tx = 2.f * (qy * z - qz * y);
    const float ty = 2.f * (qz * x - qx * z);
    const float tz = 2.f * (qx * y - qy * x);
    ox = x + w * tx + (qy * tz - qz * ty);
    oy = y + w * ty + (qz * tx - qx * tz);
    oz = z + w * tz + (qx * ty - qy * tx);
}

__global__ void __launch_bounds__(kThreads) split_mode_kernel(SplitModeArgs a) {
    const int child = blockIdx.x * kThreads + threadIdx.x;
    if (child >= a.count)
        return;
    const size_t parent = size_t(a.parents[child]);
    const float* ls = a.parent_log_scales + 3 * parent;
    float local[3] = {0.f, 0.f, 0.f};
    float delta[3] = {0.f, 0.f, 0.f};
    if (a.mode == 1) { // dense_tangent: split in the local tangent plane
        constexpr float tangent_offset = 0.5f;
        constexpr float tangent_scale = 0.7071067811865475f;
        local[0] = expf(ls[0]) * a.random_samples[3 * child] * tangent_offset;
        local[1] = expf(ls[1]) * a.random_samples[3 * child + 1] * tangent_offset;
        delta[0] = logf(tangent_scale);
        delta[1] = logf(tangent_scale);
    } else if (a.mode == 0) { // adc_covariance: rank-one offset along the major axis
        float maximum_scale_squared = 0.f;
        float scale_squared[3];
        int major = 0;
        for (int axis = 0; axis < 3; ++axis) {
            const float scale = expf(ls[axis]);
            scale_squared[axis] = scale * scale;
            if (scale_squared[axis] > maximum_scale_squared) {
                maximum_scale_squared = scale_squared[axis];
                major = axis;
            }
        }
        const float standard_k = rsqrtf(2.f);
        const float screen = a.screen_sizes ? fmaxf(a.screen_sizes[child], 1e-6f) : 1e-6f;
        const float maximum_k = a.split_at_screen_size > 0.f
                                    ? fminf(standard_k, a.split_at_screen_size / screen)
                                    : standard_k;
        for (int axis = 0; axis < 3; ++axis) {
            const float k = axis == major ? maximum_k : 1.f;
            local[axis] = sqrtf(fmaxf(1.f - k * k, 0.f)) * sqrtf(scale_squared[axis]);
            delta[axis] = logf(fmaxf(k, 1e-12f));
        }
    } else if (a.mode == 2) { // igs_random: one shared scalar along every axis
        int largest = 0;
        if (ls[1] > ls[largest])
            largest = 1;
        if (ls[2] > ls[largest])
            largest = 2;
        for (int axis = 0; axis < 3; ++axis) {
            local[axis] = expf(ls[axis]) * a.random_samples[3 * child];
            delta[axis] = axis == largest ? logf(0.5f) : 0.f;
        }
    } else { // long_axis: half the major scale along that axis
        int largest = 0;
        for (int axis = 1; axis < 3; ++axis)
            if (ls[axis] > ls[largest])
                largest = axis;
        const float offset = 0.5f * expf(ls[largest]);
        for (int axis = 0; axis < 3; ++axis) {
            local[axis] = axis == largest ? offset : 0.f;
            delta[axis] = axis == largest ? logf(0.5f) : logf(0.85f);
        }
    }
    float off[3];
    rotate_by_quaternion(a.parent_quaternions + 4 * parent, local[0], local[1], local[2], off[0],
                         off[1], off[2]);
    for (int axis = 0; axis < 3; ++axis) {
        const float center = a.parent_means[3 * parent + axis];
        a.parent_means[3 * parent + axis] = center - off[axis];
        a.child_means[3 * size_t(child) + axis] = center + off[axis];
        a.parent_log_scales[3 * parent + axis] += delta[axis];
        a.child_log_scales[3 * size_t(child) + axis] += delta[axis];
    }
    float logit;
    if (a.mode == 3) {
        const float denominator = 1.f + expf(-a.parent_opacity_logits[parent]) - a.split_opacity_k;
        const float mapped = denominator > 1e-6f
                                 ? fminf(fmaxf(a.split_opacity_k / denominator, 1e-6f), 1.f - 1e-6f)
                                 : 1.f - 1e-6f;
        logit = logf(mapped / (1.f - mapped));
    } else {
        const float opacity = sigmoid_ref(a.parent_opacity_logits[parent]);
        const float power = a.mode == 0 ? rsqrtf(2.f) : 0.5f;
        const float revised = fminf(
            fmaxf(1.f - powf(fmaxf(1.f - opacity, 0.f), power), a.minimum_opacity),
            1.f - a.minimum_opacity);
        logit = logf(revised / (1.f - revised));
    }
    a.parent_opacity_logits[parent] = logit;
    a.child_opacity_logits[child] = logit;
}

__global__ void __launch_bounds__(kThreads) adc_decay_kernel(float* __restrict__ log_scales,
                                                            float* __restrict__ opacity_logits,
                                                            size_t count, float opacity_decay,
                                                            float log_scale_decay) {
    const size_t i = size_t(blockIdx.x) * kThreads + threadIdx.x;
    if (i >= count)
        return;
    const float opacity =
        fminf(fmaxf(sigmoid_ref(opacity_logits[i]) - opacity_decay, 1e-12f), 1.f - 1e-12f);
    opacity_logits[i] = logf(opacity / (1.f - opacity));
    for (int axis = 0; axis < 3; ++axis)
        log_scales[3 * i + axis] += log_scale_decay;
}

// Stable compaction of a keep mask into row indices: per-block counts, an
// exclusive scan of the counts in one block, per-warp ballots for the ranks.
constexpr int kSelectRows = 1024; // rows per block (4 per thread)

__global__ void __launch_bounds__(kThreads) select_count_kernel(const unsigned char* __restrict__ keep,
                                                               int n, unsigned* __restrict__ counts) {
    const int base = blockIdx.x * kSelectRows;
    int c = 0;
    for (int r = threadIdx.x; r < kSelectRows; r += kThreads)
        c += (base + r < n && keep[base + r]) ? 1 : 0;
    __shared__ int s[kThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0)
        s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kThreads / 32; ++w)
            t += s[w];
        counts[blockIdx.x] = unsigned(t);
    }
}

// One block: counts[b] <- exclusive prefix; counts[blocks] <- total.
__global__ void __launch_bounds__(1024) select_scan_kernel(unsigned* __restrict__ counts,
                                                           int blocks, int* __restrict__ total_out) {
    __shared__ unsigned s_warp[32];
    __shared__ unsigned s_carry;
    if (threadIdx.x == 0)
        s_carry = 0;
    __syncthreads();
    for (int base = 0; base < blocks; base += 1024) {
        const int i = base + threadIdx.x;
        const unsigned v = i < blocks ? counts[i] : 0u;
        unsigned x = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, off);
            if ((threadIdx.x & 31) >= off)
                x += y;
        }
        if ((threadIdx.x & 31) == 31)
            s_warp[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            unsigned w = s_warp[threadIdx.x];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, w, off);
                if (threadIdx.x >= off)
                    w += y;
            }
            s_warp[threadIdx.x] = w;
        }
        __syncthreads();
        const unsigned warp_prefix = (threadIdx.x >= 32) ? s_warp[(threadIdx.x >> 5) - 1] : 0u;
        const unsigned carry = s_carry;
        if (i < blocks)
            counts[i] = carry + warp_prefix + x - v;
        __syncthreads();
        if (threadIdx.x == 1023)
            s_carry = carry + warp_prefix + x;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *total_out = int(s_carry);
}

__global__ void __launch_bounds__(kThreads) select_write_kernel(const unsigned char* __restrict__ keep,
                                                               int n,
                                                               const unsigned* __restrict__ offsets,
                                                               int* __restrict__ indices) {
    __shared__ unsigned s_warp[kThreads / 32];
    __shared__ unsigned s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0)
        s_base = offsets[blockIdx.x];
    __syncthreads();
    // rows in four rounds of kThreads; each round keeps row order
    for (int round = 0; round < kSelectRows / kThreads; ++round) {
        const int r = blockIdx.x * kSelectRows + round * kThreads + threadIdx.x;
        const bool k = r < n && keep[r];
        const unsigned ballot = __ballot_sync(0xffffffffu, k);
        if (lane == 0)
            s_warp[warp] = __popc(ballot);
        __syncthreads();
        unsigned before = 0, round_total = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            before += w < warp ? s_warp[w] : 0u;
            round_total += s_warp[w];
        }
        const unsigned base = s_base;
        if (k)
            indices[base + before + __popc(ballot & ((1u << lane) - 1u))] = r;
        __syncthreads();
        if (threadIdx.x == 0)
            s_base = base + round_total;
        __syncthreads();
    }
}

// dst_a[i] = src_a[indices[i]] for every array a, rows of row_words 4-byte
// words (4-word vectors when every row and base allows it).
__global__ void __launch_bounds__(kThreads) gather_rows_kernel(GatherRowsArgs g) {
    const size_t stride = size_t(gridDim.x) * kThreads;
    const size_t t0 = size_t(blockIdx.x) * kThreads + threadIdx.x;
    for (int a = 0; a < g.arrays; ++a) {
        const GatherArray& arr = g.array[a];
        if (arr.vec4) {
            const size_t q = size_t(arr.row_words / 4);
            const size_t total = size_t(g.count) * q;
            const uint4* src = reinterpret_cast<const uint4*>(arr.src);
            uint4* dst = reinterpret_cast<uint4*>(arr.dst);
            for (size_t w = t0; w < total; w += stride) {
                const size_t row = w / q, col = w - row * q;
                dst[w] = src[size_t(g.indices[row]) * q + col];
            }
        } else {
            const size_t q = size_t(arr.row_words);
            const size_t total = size_t(g.count) * q;
            const unsigned* src = reinterpret_cast<const unsigned*>(arr.src);
            unsigned* dst = reinterpret_cast<unsigned*>(arr.dst);
            for (size_t w = t0; w < total; w += stride) {
                const size_t row = w / q, col = w - row * q;
                dst[w] = src[size_t(g.indices[row]) * q + col];
            }
        }
    }
}

} // namespace

cudaError_t launch_split_mode(cudaStream_t s, const SplitModeArgs& a) {
    if (a.count > 0)
        split_mode_kernel<<<(a.count + kThreads - 1) / kThreads, kThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adc_decay(cudaStream_t s, float* log_scales, float* opacity_logits,
                             size_t count, float opacity_decay, float log_scale_decay) {
    if (count > 0)
        adc_decay_kernel<<<unsigned((count + kThreads - 1) / kThreads), kThreads, 0, s>>>(
            log_scales, opacity_logits, count, opacity_decay, log_scale_decay);
    return cudaGetLastError();
}

size_t select_rows_scratch_words(int n) { return size_t((n + kSelectRows - 1) / kSelectRows) + 1; }

cudaError_t launch_select_rows(cudaStream_t s, const unsigned char* keep, int n, int* indices,
                               int* count_out, unsigned* scratch) {
    const int blocks = (n + kSelectRows - 1) / kSelectRows;
    if (blocks == 0)
        return cudaMemsetAsync(count_out, 0, sizeof(int), s);
    select_count_kernel<<<blocks, kThreads, 0, s>>>(keep, n, scratch);
    select_scan_kernel<<<1, 1024, 0, s>>>(scratch, blocks, count_out);
    select_write_kernel<<<blocks, kThreads, 0, s>>>(keep, n, scratch, indices);
    return cudaGetLastError();
}

cudaError_t launch_gather_rows(cudaStream_t s, const GatherRowsArgs& g, int sm_count) {
    if (g.count <= 0 || g.arrays <= 0)
        return cudaSuccess;
    size_t words = 0;
    for (int a = 0; a < g.arrays; ++a)
        words += size_t(g.count) * g.array[a].row_words;
    const size_t want = (words + kThreads - 1) / kThreads;
    const unsigned blocks = unsigned(want < size_t(sm_count) * 8 ? (want ? want : 1)
                                                                  : size_t(sm_count) * 8);
    gather_rows_kernel<<<blocks, kThreads, 0, s>>>(g);
    return cudaGetLastError();
}

} // namespace gsb
