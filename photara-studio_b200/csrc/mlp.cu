// Densification proposal MLP: 8 -> 64 -> 64 -> 4 (ReLU), BF16 weights,
// FP32 accumulation; hand-written inference and training kernels.
//
// Parameter block (FP32 master copy and its BF16 image share this layout,
// kMlpParams values):
//   W1[8][64]  b1[64]  W2[64][64]  b2[64]  W3[64][4]  b3[4]
// Inference stages the BF16 weights in shared memory as FP32 (every thread
// reads the same weight at the same time: broadcast, no bank conflicts) and
// runs one row per thread. Training runs one row per thread for the forward
// and the activation gradients, then forms the weight gradients as small
// GEMMs over the CTA's rows out of shared memory (dW = H^T dZ) and adds one
// CTA partial per weight to the FP32 gradient with atomics; Adam updates the
// FP32 master weights and refreshes the BF16 image.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"

namespace gsb {

constexpr int kIn = 8, kHid = 64, kOut = 4;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kIn * kHid, kOffW2 = kOffB1 + kHid,
              kOffB2 = kOffW2 + kHid * kHid, kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kOut,
              kMlpParams = kOffB3 + kOut; // 4996
constexpr int kMlpRows = 128;             // rows per CTA

__device__ __forceinline__ void load_weights(float* s_w, const __nv_bfloat16* __restrict__ w) {
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x)
        s_w[k] = __bfloat162float(w[k]);
}

// Forward of one row from shared weights. h1/h2 receive the post-ReLU
// activations, z the output logits.
__device__ __forceinline__ void mlp_row_forward(const float* __restrict__ s_w, const float (&x)[kIn],
                                                float (&h1)[kHid], float (&h2)[kHid],
                                                float (&z)[kOut]) {
#pragma unroll
    for (int j = 0; j < kHid; ++j) {
        float a = s_w[kOffB1 + j];
#pragma unroll
        for (int i = 0; i < kIn; ++i)
            a = fmaf(x[i], s_w[kOffW1 + i * kHid + j], a);
        h1[j] = fmaxf(a, 0.f);
    }
#pragma unroll
    for (int j = 0; j < kHid; ++j)
        h2[j] = s_w[kOffB2 + j];
#pragma unroll 4
    for (int i = 0; i < kHid; ++i) {
        const float hi = h1[i];
#pragma unroll
        for (int j = 0; j < kHid; ++j)
            h2[j] = fmaf(hi, s_w[kOffW2 + i * kHid + j], h2[j]);
    }
#pragma unroll
    for (int j = 0; j < kHid; ++j)
        h2[j] = fmaxf(h2[j], 0.f);
#pragma unroll
    for (int o = 0; o < kOut; ++o) {
        float a = s_w[kOffB3 + o];
#pragma unroll
        for (int i = 0; i < kHid; ++i)
            a = fmaf(h2[i], s_w[kOffW3 + i * kOut + o], a);
        z[o] = a;
    }
}

// features: [n][8] (already normalised); logits: [n][4].
__global__ void __launch_bounds__(kMlpRows) mlp_forward_kernel(int n, const float* __restrict__ feats,
                                                               const __nv_bfloat16* __restrict__ w,
                                                               float* __restrict__ logits) {
    __shared__ float s_w[kMlpParams];
    load_weights(s_w, w);
    __syncthreads();
    const int r = blockIdx.x * kMlpRows + threadIdx.x;
    if (r >= n)
        return;
    float x[kIn], h1[kHid], h2[kHid], z[kOut];
#pragma unroll
    for (int i = 0; i < kIn; ++i)
        x[i] = feats[size_t(r) * kIn + i];
    mlp_row_forward(s_w, x, h1, h2, z);
#pragma unroll
    for (int o = 0; o < kOut; ++o)
        logits[size_t(r) * kOut + o] = z[o];
}

// One training pass over `n` rows: softmax cross-entropy against `labels`
// (0..3) weighted by `weights`, mean over the weight sum `wsum` (device
// scalar). Accumulates dL/dparams into grad (FP32, zeroed by the caller) and
// the loss into *loss.
__global__ void __launch_bounds__(kMlpRows) mlp_train_kernel(
    int n, const float* __restrict__ feats, const int* __restrict__ labels,
    const float* __restrict__ weights, const __nv_bfloat16* __restrict__ w, float inv_wsum,
    float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ float smem[];
    float* s_w = smem;                          // [kMlpParams]
    float* s_x = s_w + kMlpParams;              // [rows][kIn]
    float* s_h1 = s_x + kMlpRows * kIn;         // [rows][kHid + 1]
    float* s_d2 = s_h1 + kMlpRows * (kHid + 1); // [rows][kHid + 1]  dL/d(pre-ReLU layer 2)
    float* s_d1 = s_d2 + kMlpRows * (kHid + 1); // [rows][kHid + 1]  dL/d(pre-ReLU layer 1)
    float* s_h2 = s_d1 + kMlpRows * (kHid + 1); // [rows][kHid + 1]
    float* s_dz = s_h2 + kMlpRows * (kHid + 1); // [rows][kOut]
    constexpr int H = kHid + 1;
    load_weights(s_w, w);
    __syncthreads();
    const int t = threadIdx.x;
    const int r = blockIdx.x * kMlpRows + t;
    const bool valid = r < n;
    float x[kIn], h1[kHid], h2[kHid], z[kOut];
#pragma unroll
    for (int i = 0; i < kIn; ++i)
        x[i] = valid ? feats[size_t(r) * kIn + i] : 0.f;
    mlp_row_forward(s_w, x, h1, h2, z);
    const float wr = valid ? weights[r] * inv_wsum : 0.f;
    const int lab = valid ? labels[r] : 0;
    float zmax = z[0];
#pragma unroll
    for (int o = 1; o < kOut; ++o)
        zmax = fmaxf(zmax, z[o]);
    float e[kOut], se = 0.f;
#pragma unroll
    for (int o = 0; o < kOut; ++o) {
        e[o] = expf(z[o] - zmax);
        se += e[o];
    }
    float dz[kOut];
    float zl = z[0];
#pragma unroll
    for (int o = 0; o < kOut; ++o) {
        if (o == lab) zl = z[o];
        dz[o] = wr * (e[o] / se - (o == lab ? 1.f : 0.f));
    }
    float row_loss = wr * (logf(se) + zmax - zl);
    // dL/dh2 (post-ReLU) -> pre-ReLU
    float d2[kHid];
#pragma unroll
    for (int i = 0; i < kHid; ++i) {
        float a = 0.f;
#pragma unroll
        for (int o = 0; o < kOut; ++o)
            a = fmaf(dz[o], s_w[kOffW3 + i * kOut + o], a);
        d2[i] = h2[i] > 0.f ? a : 0.f;
    }
    // dL/dh1 (post-ReLU) -> pre-ReLU
#pragma unroll
    for (int i = 0; i < kHid; ++i) {
        float a = 0.f;
#pragma unroll 8
        for (int j = 0; j < kHid; ++j)
            a = fmaf(d2[j], s_w[kOffW2 + i * kHid + j], a);
        s_d1[t * H + i] = h1[i] > 0.f ? a : 0.f;
    }
#pragma unroll
    for (int i = 0; i < kIn; ++i)
        s_x[t * kIn + i] = x[i];
#pragma unroll
    for (int i = 0; i < kHid; ++i) {
        s_h1[t * H + i] = h1[i];
        s_h2[t * H + i] = h2[i];
        s_d2[t * H + i] = d2[i];
    }
#pragma unroll
    for (int o = 0; o < kOut; ++o)
        s_dz[t * kOut + o] = dz[o];
    // loss: warp reduce then one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        row_loss += __shfl_xor_sync(0xffffffffu, row_loss, o);
    if ((t & 31) == 0)
        atomicAdd(loss, row_loss);
    __syncthreads();
    // Weight gradients as GEMMs over the CTA's rows; each thread owns outputs
    // p = t, t + kMlpRows, ... of the parameter block.
    const int rows = kMlpRows;
    for (int p = t; p < kMlpParams; p += kMlpRows) {
        float g = 0.f;
        if (p < kOffB1) { // W1[i][j] = sum_r x[r][i] d1[r][j]
            const int i = p / kHid, j = p % kHid;
            for (int q = 0; q < rows; ++q) g = fmaf(s_x[q * kIn + i], s_d1[q * H + j], g);
        } else if (p < kOffW2) { // b1[j]
            const int j = p - kOffB1;
            for (int q = 0; q < rows; ++q) g += s_d1[q * H + j];
        } else if (p < kOffB2) { // W2[i][j] = sum_r h1[r][i] d2[r][j]
            const int i = (p - kOffW2) / kHid, j = (p - kOffW2) % kHid;
            for (int q = 0; q < rows; ++q) g = fmaf(s_h1[q * H + i], s_d2[q * H + j], g);
        } else if (p < kOffW3) { // b2[j]
            const int j = p - kOffB2;
            for (int q = 0; q < rows; ++q) g += s_d2[q * H + j];
        } else if (p < kOffB3) { // W3[i][o] = sum_r h2[r][i] dz[r][o]
            const int i = (p - kOffW3) / kOut, o = (p - kOffW3) % kOut;
            for (int q = 0; q < rows; ++q) g = fmaf(s_h2[q * H + i], s_dz[q * kOut + o], g);
        } else { // b3[o]
            const int o = p - kOffB3;
            for (int q = 0; q < rows; ++q) g += s_dz[q * kOut + o];
        }
        if (g != 0.f)
            atomicAdd(&grad[p], g);
    }
}

// Adam on the FP32 master parameters; refreshes the BF16 image.
__global__ void mlp_adam_kernel(float* __restrict__ master, __nv_bfloat16* __restrict__ w,
                                const float* __restrict__ grad, float* __restrict__ m,
                                float* __restrict__ v, float lr, float b1, float b2, float c1,
                                float c2, float eps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams)
        return;
    const float g = grad[p];
    const float mm = b1 * m[p] + (1.f - b1) * g;
    const float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float val = master[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    master[p] = val;
    w[p] = __float2bfloat16_rn(val);
}

int mlp_param_count() { return kMlpParams; }

size_t mlp_train_smem() {
    return size_t(kMlpParams + kMlpRows * kIn + 4 * kMlpRows * (kHid + 1) + kMlpRows * kOut) *
           sizeof(float);
}

void launch_mlp_forward(cudaStream_t s, int n, const float* feats, const void* w_bf16,
                        float* logits) {
    if (n <= 0)
        return;
    mlp_forward_kernel<<<(n + kMlpRows - 1) / kMlpRows, kMlpRows, 0, s>>>(
        n, feats, static_cast<const __nv_bfloat16*>(w_bf16), logits);
}

void launch_mlp_train(cudaStream_t s, int n, const float* feats, const int* labels,
                      const float* weights, const void* w_bf16, float inv_wsum, float* grad,
                      float* loss) {
    if (n <= 0)
        return;
    const size_t smem = mlp_train_smem();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem));
        attr = true;
    }
    mlp_train_kernel<<<(n + kMlpRows - 1) / kMlpRows, kMlpRows, smem, s>>>(
        n, feats, labels, weights, static_cast<const __nv_bfloat16*>(w_bf16), inv_wsum, grad,
        loss);
}

void launch_mlp_adam(cudaStream_t s, float* master, void* w_bf16, const float* grad, float* m,
                     float* v, float lr, float b1, float b2, float c1, float c2, float eps) {
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, s>>>(
        master, static_cast<__nv_bfloat16*>(w_bf16), grad, m, v, lr, b1, b2, c1, c2, eps);
}

} // namespace gsb
