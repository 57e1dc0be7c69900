// mlp.cuh - the refinement proposer's multilayer perceptron: forward, backward and Adam kernels.
//
// Network: x[F] -> tanh(W1 x + b1)[H] -> tanh(W2 h + b2)[H] -> tanh(W3 h + b3)[H] -> w4.h + b4.
// Master parameters are FP32; the forward and backward products read a BF16 copy of the weight
// matrices (biases stay FP32) and accumulate in FP32.  Loss: mean squared error.
//
// Parallel layout: one CTA of H threads per tile of MLP_TILE samples; thread j owns output
// neuron j of every layer (its weight row lives in registers), the tile's activations live in
// shared memory and are read as broadcasts.  Weight gradients of a CTA are written to its own
// slot of a partial buffer and reduced in CTA order, so training is deterministic.
#pragma once
#include <cuda_bf16.h>
#include "common.cuh"

#define MLP_H 64
#define MLP_F 8
#define MLP_TILE 32

// Parameter offsets (floats): W1[H][F] b1[H] W2[H][H] b2[H] W3[H][H] b3[H] w4[H] b4[1]
struct MlpLayout {
    static constexpr int W1 = 0;
    static constexpr int B1 = W1 + MLP_H * MLP_F;
    static constexpr int W2 = B1 + MLP_H;
    static constexpr int B2 = W2 + MLP_H * MLP_H;
    static constexpr int W3 = B2 + MLP_H;
    static constexpr int B3 = W3 + MLP_H * MLP_H;
    static constexpr int W4 = B3 + MLP_H;
    static constexpr int B4 = W4 + MLP_H;
    static constexpr int COUNT = B4 + 1;
};

// Round the master weights to the BF16 compute copy.
__global__ void mlp_to_bf16_kernel(const float *__restrict__ master, __nv_bfloat16 *__restrict__ w, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        w[i] = __float2bfloat16_rn(master[i]);
}

WNLQG_D float mlp_w(const __nv_bfloat16 *w, int i) { return __bfloat162float(w[i]); }

// Forward over a tile; keeps the three hidden activations in shared memory (h[l][s][j]).
// Returns the output of sample s in out_s (valid for threadIdx.x == 0 .. tile).
WNLQG_D void mlp_tile_forward(const __nv_bfloat16 *__restrict__ wb, const float *__restrict__ master,
                              const float *__restrict__ x, int64_t n, int64_t s0, float (*xs)[MLP_F],
                              float (*h)[MLP_TILE][MLP_H], float *y) {
    const int j = threadIdx.x;
    for (int e = threadIdx.x; e < MLP_TILE * MLP_F; e += blockDim.x) {
        const int s = e / MLP_F, f = e % MLP_F;
        xs[s][f] = (s0 + s < n) ? x[(s0 + s) * MLP_F + f] : 0.0f;
    }
    __syncthreads();
    {
        float wr[MLP_F];
#pragma unroll
        for (int f = 0; f < MLP_F; ++f) wr[f] = mlp_w(wb, MlpLayout::W1 + j * MLP_F + f);
        const float bj = master[MlpLayout::B1 + j];
        for (int s = 0; s < MLP_TILE; ++s) {
            float z = bj;
#pragma unroll
            for (int f = 0; f < MLP_F; ++f) z = fmaf(wr[f], xs[s][f], z);
            h[0][s][j] = tanhf(z);
        }
    }
    __syncthreads();
    for (int l = 1; l < 3; ++l) {
        const int WO = l == 1 ? MlpLayout::W2 : MlpLayout::W3;
        const int BO = l == 1 ? MlpLayout::B2 : MlpLayout::B3;
        float wr[MLP_H];
#pragma unroll
        for (int i = 0; i < MLP_H; ++i) wr[i] = mlp_w(wb, WO + j * MLP_H + i);
        const float bj = master[BO + j];
        for (int s = 0; s < MLP_TILE; ++s) {
            float z = bj;
#pragma unroll
            for (int i = 0; i < MLP_H; ++i) z = fmaf(wr[i], h[l - 1][s][i], z);
            h[l][s][j] = tanhf(z);
        }
        __syncthreads();
    }
    if (j < MLP_TILE) {
        float z = master[MlpLayout::B4];
        for (int i = 0; i < MLP_H; ++i) z = fmaf(mlp_w(wb, MlpLayout::W4 + i), h[2][j][i], z);
        y[j] = z;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(MLP_H) mlp_forward_kernel(const __nv_bfloat16 *__restrict__ wb,
                                                            const float *__restrict__ master,
                                                            const float *__restrict__ x, int64_t n,
                                                            float *__restrict__ out) {
    __shared__ float xs[MLP_TILE][MLP_F];
    __shared__ float h[3][MLP_TILE][MLP_H];
    __shared__ float y[MLP_TILE];
    for (int64_t s0 = (int64_t)blockIdx.x * MLP_TILE; s0 < n; s0 += (int64_t)gridDim.x * MLP_TILE) {
        mlp_tile_forward(wb, master, x, n, s0, xs, h, y);
        if (threadIdx.x < MLP_TILE && s0 + threadIdx.x < n) out[s0 + threadIdx.x] = y[threadIdx.x];
        __syncthreads();
    }
}

// Loss and gradient of the mean squared error over n samples.  partial[cta][COUNT + 1]
// receives this CTA's gradient and loss sum (slot COUNT).
__global__ void __launch_bounds__(MLP_H) mlp_backward_kernel(const __nv_bfloat16 *__restrict__ wb,
                                                             const float *__restrict__ master,
                                                             const float *__restrict__ x,
                                                             const float *__restrict__ target, int64_t n,
                                                             float *__restrict__ partial) {
    __shared__ float xs[MLP_TILE][MLP_F];
    __shared__ float h[3][MLP_TILE][MLP_H];
    __shared__ float y[MLP_TILE];
    __shared__ float g[MLP_TILE];
    __shared__ float dz[2][MLP_TILE][MLP_H];
    const int j = threadIdx.x;
    float gw1[MLP_F], gw2[MLP_H], gw3[MLP_H];
    float gb1 = 0.f, gb2 = 0.f, gb3 = 0.f, gw4 = 0.f, gb4 = 0.f, loss = 0.f;
#pragma unroll
    for (int f = 0; f < MLP_F; ++f) gw1[f] = 0.f;
#pragma unroll
    for (int i = 0; i < MLP_H; ++i) { gw2[i] = 0.f; gw3[i] = 0.f; }
    const float inv_n = 1.0f / (float)n;
    for (int64_t s0 = (int64_t)blockIdx.x * MLP_TILE; s0 < n; s0 += (int64_t)gridDim.x * MLP_TILE) {
        mlp_tile_forward(wb, master, x, n, s0, xs, h, y);
        if (j < MLP_TILE) {
            const bool ok = s0 + j < n;
            const float d = ok ? y[j] - target[s0 + j] : 0.0f;
            g[j] = 2.0f * d * inv_n;
            if (j == 0) {
                float ls = 0.f;
                for (int s = 0; s < MLP_TILE; ++s)
                    if (s0 + s < n) { const float e = y[s] - target[s0 + s]; ls += e * e; }
                loss += ls * inv_n;
            }
        }
        __syncthreads();
        // Output layer and dz of layer 3: dz3[s][j] = g_s w4_j (1 - h3^2).
        const float w4j = mlp_w(wb, MlpLayout::W4 + j);
        for (int s = 0; s < MLP_TILE; ++s) {
            gw4 = fmaf(g[s], h[2][s][j], gw4);
            const float hv = h[2][s][j];
            dz[0][s][j] = g[s] * w4j * (1.0f - hv * hv);
        }
        if (j == 0)
            for (int s = 0; s < MLP_TILE; ++s) gb4 += g[s];
        __syncthreads();
        // Layer 3: gradW3 row j, dh2 = W3^T dz3 -> dz2 (thread j owns input neuron j for dh).
        for (int s = 0; s < MLP_TILE; ++s) {
            const float d = dz[0][s][j];
            gb3 += d;
#pragma unroll
            for (int i = 0; i < MLP_H; ++i) gw3[i] = fmaf(d, h[1][s][i], gw3[i]);
        }
        {
            float wc[MLP_H];
#pragma unroll
            for (int o = 0; o < MLP_H; ++o) wc[o] = mlp_w(wb, MlpLayout::W3 + o * MLP_H + j);
            for (int s = 0; s < MLP_TILE; ++s) {
                float acc = 0.f;
#pragma unroll
                for (int o = 0; o < MLP_H; ++o) acc = fmaf(wc[o], dz[0][s][o], acc);
                const float hv = h[1][s][j];
                dz[1][s][j] = acc * (1.0f - hv * hv);
            }
        }
        __syncthreads();
        // Layer 2: gradW2 row j, dh1 = W2^T dz2 -> dz1 (stored in dz[0]).
        for (int s = 0; s < MLP_TILE; ++s) {
            const float d = dz[1][s][j];
            gb2 += d;
#pragma unroll
            for (int i = 0; i < MLP_H; ++i) gw2[i] = fmaf(d, h[0][s][i], gw2[i]);
        }
        {
            float wc[MLP_H];
#pragma unroll
            for (int o = 0; o < MLP_H; ++o) wc[o] = mlp_w(wb, MlpLayout::W2 + o * MLP_H + j);
            for (int s = 0; s < MLP_TILE; ++s) {
                float acc = 0.f;
#pragma unroll
                for (int o = 0; o < MLP_H; ++o) acc = fmaf(wc[o], dz[1][s][o], acc);
                const float hv = h[0][s][j];
                dz[0][s][j] = acc * (1.0f - hv * hv);
            }
        }
        __syncthreads();
        // Layer 1.
        for (int s = 0; s < MLP_TILE; ++s) {
            const float d = dz[0][s][j];
            gb1 += d;
#pragma unroll
            for (int f = 0; f < MLP_F; ++f) gw1[f] = fmaf(d, xs[s][f], gw1[f]);
        }
        __syncthreads();
    }
    float *p = partial + (int64_t)blockIdx.x * (MlpLayout::COUNT + 1);
#pragma unroll
    for (int f = 0; f < MLP_F; ++f) p[MlpLayout::W1 + j * MLP_F + f] = gw1[f];
    p[MlpLayout::B1 + j] = gb1;
#pragma unroll
    for (int i = 0; i < MLP_H; ++i) p[MlpLayout::W2 + j * MLP_H + i] = gw2[i];
    p[MlpLayout::B2 + j] = gb2;
#pragma unroll
    for (int i = 0; i < MLP_H; ++i) p[MlpLayout::W3 + j * MLP_H + i] = gw3[i];
    p[MlpLayout::B3 + j] = gb3;
    p[MlpLayout::W4 + j] = gw4;
    if (j == 0) {
        p[MlpLayout::B4] = gb4;
        p[MlpLayout::COUNT] = loss;
    }
}

// grad[i] = sum over CTAs (in order) of partial[c][i]; slot COUNT is the loss.
__global__ void mlp_reduce_kernel(const float *__restrict__ partial, int nslots, float *__restrict__ grad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= MlpLayout::COUNT; i += gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int c = 0; c < nslots; ++c) acc += partial[(int64_t)c * (MlpLayout::COUNT + 1) + i];
        grad[i] = acc;
    }
}

// Adam update of the FP32 master parameters (Kingma & Ba 2015), then the BF16 copy.
__global__ void mlp_adam_kernel(float *__restrict__ master, const float *__restrict__ grad, float *__restrict__ m,
                                float *__restrict__ v, __nv_bfloat16 *__restrict__ wb, float lr, float beta1,
                                float beta2, float eps, float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MlpLayout::COUNT; i += gridDim.x * blockDim.x) {
        const float gi = grad[i];
        const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
        const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float p = master[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        master[i] = p;
        wb[i] = __float2bfloat16_rn(p);
    }
}
