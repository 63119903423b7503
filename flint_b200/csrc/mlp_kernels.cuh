// Cost model of the learned schedule: a fully connected network
//     x (n_in) -> 64 ReLU -> 64 ReLU -> 64 ReLU -> 1,   fp32,
// predicting the log of a product's device time from request features and a
// candidate configuration.  Hand-written forward, backward and Adam kernels;
// training minimises the mean squared error over a batch.
//
// Parameter vector layout (floats): W1[n_in][64], b1[64], W2[64][64], b2[64],
// W3[64][64], b3[64], W4[64], b4 -- W[i][j] connects input i to unit j.
//
// Execution: a block of 64 threads (thread j = hidden unit j) takes a tile of
// MLP_TILE samples; activations of the tile live in shared memory, a unit's
// incoming weights in registers.  The backward pass writes each block's
// gradient contribution to its own row of a partial-gradient buffer, and a
// second kernel sums the rows in a fixed order, so gradients are
// deterministic (no floating-point atomics).
#pragma once
#include <stdint.h>

namespace fb {

constexpr int MLP_H = 64;
constexpr int MLP_MAX_IN = 32;
constexpr int MLP_TILE = 32;

__host__ __device__ constexpr int mlp_nparams(int n_in)
{
    return n_in * MLP_H + MLP_H + 2 * (MLP_H * MLP_H + MLP_H) + MLP_H + 1;
}

struct MlpOffsets {
    int W1, b1, W2, b2, W3, b3, W4, b4, total;
};

__host__ __device__ inline MlpOffsets mlp_offsets(int n_in)
{
    MlpOffsets o;
    o.W1 = 0;
    o.b1 = o.W1 + n_in * MLP_H;
    o.W2 = o.b1 + MLP_H;
    o.b2 = o.W2 + MLP_H * MLP_H;
    o.W3 = o.b2 + MLP_H;
    o.b3 = o.W3 + MLP_H * MLP_H;
    o.W4 = o.b3 + MLP_H;
    o.b4 = o.W4 + MLP_H;
    o.total = o.b4 + 1;
    return o;
}

// sum over the 64 threads of the block (two warps) into every thread
__device__ __forceinline__ float block64_sum(float v, float* red)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const float s = red[0] + red[1];
    __syncthreads();
    return s;
}

// One dense layer for a tile: out[s][j] = relu(b[j] + sum_i in[s][i] W[i][j])
template <int NIN>
__device__ __forceinline__ void mlp_layer(const float* __restrict__ W, const float* __restrict__ b,
                                          int nin, const float (*in)[MLP_H + 1], float (*out)[MLP_H + 1],
                                          int ns)
{
    const int j = threadIdx.x;
    float w[NIN];
#pragma unroll
    for (int i = 0; i < NIN; i++) w[i] = i < nin ? W[i * MLP_H + j] : 0.0f;
    const float bj = b[j];
    for (int s = 0; s < ns; s++) {
        float acc = bj;
#pragma unroll
        for (int i = 0; i < NIN; i++) acc = fmaf(in[s][i], w[i], acc);
        out[s][j] = fmaxf(acc, 0.0f);
    }
}

// Forward pass.  grid = ceil(n / MLP_TILE), block = 64.  y[s] = prediction;
// with acts != NULL the three hidden layers' outputs are stored as
// acts[(l n + s) 64 + j] for the backward pass.
__global__ void __launch_bounds__(MLP_H)
k_mlp_forward(const float* __restrict__ P, int n_in, const float* __restrict__ X, int n,
              float* __restrict__ y, float* __restrict__ acts)
{
    __shared__ float hx[MLP_TILE][MLP_H + 1];
    __shared__ float ha[MLP_TILE][MLP_H + 1];
    __shared__ float hb[MLP_TILE][MLP_H + 1];
    __shared__ float red[2];
    const MlpOffsets o = mlp_offsets(n_in);
    const int s0 = blockIdx.x * MLP_TILE;
    const int ns = min(MLP_TILE, n - s0);
    const int j = threadIdx.x;
    for (int f = j; f < MLP_TILE * MLP_MAX_IN; f += MLP_H) {
        const int s = f / MLP_MAX_IN, i = f % MLP_MAX_IN;
        hx[s][i] = (s < ns && i < n_in) ? X[(size_t)(s0 + s) * n_in + i] : 0.0f;
    }
    __syncthreads();
    mlp_layer<MLP_MAX_IN>(P + o.W1, P + o.b1, n_in, hx, ha, ns);
    __syncthreads();
    if (acts)
        for (int s = 0; s < ns; s++) acts[((size_t)0 * n + s0 + s) * MLP_H + j] = ha[s][j];
    mlp_layer<MLP_H>(P + o.W2, P + o.b2, MLP_H, ha, hb, ns);
    __syncthreads();
    if (acts)
        for (int s = 0; s < ns; s++) acts[((size_t)1 * n + s0 + s) * MLP_H + j] = hb[s][j];
    mlp_layer<MLP_H>(P + o.W3, P + o.b3, MLP_H, hb, ha, ns);
    __syncthreads();
    if (acts)
        for (int s = 0; s < ns; s++) acts[((size_t)2 * n + s0 + s) * MLP_H + j] = ha[s][j];
    const float w4 = P[o.W4 + j], b4 = P[o.b4];
    for (int s = 0; s < ns; s++) {
        const float t = block64_sum(ha[s][j] * w4, red);
        if (j == 0) y[s0 + s] = t + b4;
    }
}

// Backward pass of the mean squared error L = (1/n) sum_s (y_s - t_s)^2 for
// one tile; needs the forward pass's y and acts.  Writes the tile's gradient
// contribution to part + blockIdx.x * nparams and its loss share to
// lpart[blockIdx.x].  grid = ceil(n / MLP_TILE), block = 64.
__global__ void __launch_bounds__(MLP_H)
k_mlp_backward(const float* __restrict__ P, int n_in, const float* __restrict__ X, int n,
               const float* __restrict__ y, const float* __restrict__ t,
               const float* __restrict__ acts, float* __restrict__ part, float* __restrict__ lpart)
{
    __shared__ float hx[MLP_TILE][MLP_H + 1];
    __shared__ float h1[MLP_TILE][MLP_H + 1];
    __shared__ float h2[MLP_TILE][MLP_H + 1];
    __shared__ float h3[MLP_TILE][MLP_H + 1];   // reused for the deltas once read
    __shared__ float da[MLP_TILE][MLP_H + 1];
    float (*db)[MLP_H + 1] = h3;
    __shared__ float dy[MLP_TILE];
    __shared__ float red[2];
    const MlpOffsets o = mlp_offsets(n_in);
    const int s0 = blockIdx.x * MLP_TILE;
    const int ns = min(MLP_TILE, n - s0);
    const int j = threadIdx.x;
    float* __restrict__ G = part + (size_t)blockIdx.x * o.total;
    for (int f = j; f < MLP_TILE * MLP_MAX_IN; f += MLP_H) {
        const int s = f / MLP_MAX_IN, i = f % MLP_MAX_IN;
        hx[s][i] = (s < ns && i < n_in) ? X[(size_t)(s0 + s) * n_in + i] : 0.0f;
    }
    for (int s = 0; s < MLP_TILE; s++) {
        const bool v = s < ns;
        h1[s][j] = v ? acts[((size_t)0 * n + s0 + s) * MLP_H + j] : 0.0f;
        h2[s][j] = v ? acts[((size_t)1 * n + s0 + s) * MLP_H + j] : 0.0f;
        h3[s][j] = v ? acts[((size_t)2 * n + s0 + s) * MLP_H + j] : 0.0f;
    }
    if (j < MLP_TILE) {
        const float e = j < ns ? y[s0 + j] - t[s0 + j] : 0.0f;
        dy[j] = 2.0f * e / (float)n;
    }
    __syncthreads();
    // loss share
    {
        float l = 0.0f;
        if (j < ns) {
            const float e = y[s0 + j] - t[s0 + j];
            l = e * e / (float)n;
        }
        l = block64_sum(l, red);
        if (j == 0) lpart[blockIdx.x] = l;
    }
    // output layer: dW4[j] = sum_s dy h3, db4 = sum_s dy; delta3 = dy W4 relu'
    {
        const float w4 = P[o.W4 + j];
        float g = 0.0f;
        for (int s = 0; s < MLP_TILE; s++) {
            g = fmaf(dy[s], h3[s][j], g);
            da[s][j] = h3[s][j] > 0.0f ? dy[s] * w4 : 0.0f;
        }
        G[o.W4 + j] = g;
        if (j == 0) {
            float gb = 0.0f;
            for (int s = 0; s < MLP_TILE; s++) gb += dy[s];
            G[o.b4] = gb;
        }
    }
    __syncthreads();   // h3 is free from here on (db aliases it)
    // hidden layers, from the top: delta (da) of layer l, inputs hin
    auto dense_back = [&](int oW, int ob, float (*hin)[MLP_H + 1], int nin, float (*dout)[MLP_H + 1],
                          bool relu_in) {
        // dW[i][j] = sum_s hin[s][i] delta[s][j]; db[j] = sum_s delta[s][j]
        float gb = 0.0f;
        for (int s = 0; s < MLP_TILE; s++) gb += da[s][j];
        G[ob + j] = gb;
        for (int i = 0; i < nin; i++) {
            float g = 0.0f;
            for (int s = 0; s < MLP_TILE; s++) g = fmaf(hin[s][i], da[s][j], g);
            G[oW + i * MLP_H + j] = g;
        }
        if (dout) {
            // thread j now stands for input unit i = j: dout[s][i] = relu'(hin) sum_k delta[s][k] W[i][k]
            const int i = j;
            float w[MLP_H];
#pragma unroll
            for (int k = 0; k < MLP_H; k++) w[k] = P[oW + i * MLP_H + k];
            for (int s = 0; s < MLP_TILE; s++) {
                float acc = 0.0f;
#pragma unroll
                for (int k = 0; k < MLP_H; k++) acc = fmaf(da[s][k], w[k], acc);
                dout[s][i] = (!relu_in || hin[s][i] > 0.0f) ? acc : 0.0f;
            }
        }
        __syncthreads();
    };
    dense_back(o.W3, o.b3, h2, MLP_H, db, true);
    for (int s = 0; s < MLP_TILE; s++) da[s][j] = db[s][j];
    __syncthreads();
    dense_back(o.W2, o.b2, h1, MLP_H, db, true);
    for (int s = 0; s < MLP_TILE; s++) da[s][j] = db[s][j];
    __syncthreads();
    dense_back(o.W1, o.b1, hx, n_in, nullptr, false);
}

// g[k] = sum over blocks b of part[b * np + k] (fixed order); loss likewise
__global__ void k_mlp_reduce(const float* __restrict__ part, int nblocks, int np, float* __restrict__ g,
                             const float* __restrict__ lpart, float* __restrict__ loss)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < np) {
        float s = 0.0f;
        for (int b = 0; b < nblocks; b++) s += part[(size_t)b * np + k];
        g[k] = s;
    }
    if (k == 0 && loss) {
        float s = 0.0f;
        for (int b = 0; b < nblocks; b++) s += lpart[b];
        *loss = s;
    }
}

// Adam (Kingma and Ba, 2015) with bias correction; step t >= 1
__global__ void k_mlp_adam(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, int np, float lr, float b1, float b2, float eps,
                           float c1, float c2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.0f - b1) * gk;
    const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    P[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

}  // namespace fb
