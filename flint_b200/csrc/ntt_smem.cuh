// Block-cooperative number-theoretic transforms on vectors held in shared
// memory.
//
// A forward transform of length L = 2^k is a Gentleman-Sande (decimation in
// frequency) network: natural-order input, bit-reversed output.  Level with
// half-size h pairs positions (j, j + h) inside blocks of 2h and computes
//     (a, b) -> (a + b, (a - b) * w2h^jj),   jj = j mod h, w2h a 2h-th root.
// The inverse is the transposed Cooley-Tukey (decimation in time) network
// with inverse twiddles: bit-reversed input, natural output, scaled by L.
//
// Both are executed as passes of Q levels: each thread loads E = 2^Q
// elements that are closed under those levels into registers, runs the
// butterflies there and writes them back, so shared memory is touched once
// per Q levels instead of once per level.
//
// Twiddles come from per-prime tables tw[h + jj] = (w2h^jj, Shoup companion)
// for h a power of two; one table serves every transform length because the
// entry for a given (h, jj) does not depend on L.
//
// The reference computes the same transforms with radix-4 double-precision
// butterflies over 256-point blocks (src/fft_small/sd_fft.c:1230-1274,
// src/fft_small/sd_ifft.c:1503-1533); the output order here differs, which
// is harmless because only pointwise products are formed in transform space.
#pragma once
#include "modarith.cuh"

namespace fb {

// Bank-conflict-avoiding permutation of shared-memory word addresses: the low
// five bits (the bank) are XORed with a fold of the higher bits, so that
// power-of-two strides up to 2^15 words spread over all banks.  It is a
// bijection that keeps every address inside its aligned 32-word row.
__device__ __forceinline__ int swz(int a)
{
    return a ^ (((a >> 5) ^ (a >> 10)) & 31);
}

struct VecLayout {
    int nvec;      // number of independent vectors
    int logL;      // log2 of the vector length
    int vstride;   // word distance between vectors
    int estride;   // word distance between consecutive elements of a vector
    bool vec_fast; // consecutive threads take consecutive vectors
};

__device__ __forceinline__ int vl_addr(const VecLayout& V, int v, int j)
{
    return swz(v * V.vstride + j * V.estride);
}

// One Gentleman-Sande pass: levels with half-sizes h, h/2, ..., h/2^(Q-1).
template <int Q>
__device__ __forceinline__ void gs_pass(uint32_t* sm, const VecLayout& V, int h,
                                        const uint2* __restrict__ tw, uint32_t p)
{
    constexpr int E = 1 << Q;
    const int logS = __ffs(h) - 1 - (Q - 1);   // S = h >> (Q-1)
    const int S = 1 << logS;
    const int lognsub = V.logL - Q;
    const int total = V.nvec << lognsub;
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
        int v, s;
        if (V.vec_fast) { v = f % V.nvec; s = f / V.nvec; }
        else            { s = f & ((1 << lognsub) - 1); v = f >> lognsub; }
        const int jj0 = s & (S - 1);
        const int base = ((s >> logS) << (logS + Q)) + jj0;   // blk * 2h + jj0
        uint32_t x[E];
#pragma unroll
        for (int m = 0; m < E; m++) x[m] = sm[vl_addr(V, v, base + m * S)];
#pragma unroll
        for (int t = 0; t < Q; t++) {
            const int hm = E >> (t + 1);
            const int ht = h >> t;
#pragma unroll
            for (int m = 0; m < E; m++) {
                if ((m & hm) == 0) {
                    const int jj = jj0 + (m & (hm - 1)) * S;
                    const uint2 w = tw[ht + jj];
                    const uint32_t a = x[m], b = x[m + hm];
                    x[m] = add_mod(a, b, p);
                    x[m + hm] = mul_shoup(a - b + p, w.x, w.y, p);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < E; m++) sm[vl_addr(V, v, base + m * S)] = x[m];
    }
}

// One Cooley-Tukey pass: levels with half-sizes h, 2h, ..., 2^(Q-1) h.
template <int Q>
__device__ __forceinline__ void ct_pass(uint32_t* sm, const VecLayout& V, int h,
                                        const uint2* __restrict__ twi, uint32_t p)
{
    constexpr int E = 1 << Q;
    const int logh = __ffs(h) - 1;
    const int lognsub = V.logL - Q;
    const int total = V.nvec << lognsub;
    for (int f = threadIdx.x; f < total; f += blockDim.x) {
        int v, s;
        if (V.vec_fast) { v = f % V.nvec; s = f / V.nvec; }
        else            { s = f & ((1 << lognsub) - 1); v = f >> lognsub; }
        const int jj0 = s & (h - 1);
        const int base = ((s >> logh) << (logh + Q)) + jj0;
        uint32_t x[E];
#pragma unroll
        for (int m = 0; m < E; m++) x[m] = sm[vl_addr(V, v, base + m * h)];
#pragma unroll
        for (int t = 0; t < Q; t++) {
            const int hm = 1 << t;
            const int ht = h << t;
#pragma unroll
            for (int m = 0; m < E; m++) {
                if ((m & hm) == 0) {
                    const int jj = jj0 + (m & (hm - 1)) * h;
                    const uint2 w = twi[ht + jj];
                    const uint32_t a = x[m];
                    const uint32_t b = mul_shoup(x[m + hm], w.x, w.y, p);
                    x[m] = add_mod(a, b, p);
                    x[m + hm] = sub_mod(a, b, p);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < E; m++) sm[vl_addr(V, v, base + m * h)] = x[m];
    }
}

// Full forward transform of every vector (caller synchronises before).
__device__ __forceinline__ void ntt_forward(uint32_t* sm, const VecLayout& V,
                                            const uint2* __restrict__ tw, uint32_t p)
{
    int rem = V.logL;
    int h = (1 << V.logL) >> 1;
    while (rem > 0) {
        if (rem >= 4)      { gs_pass<4>(sm, V, h, tw, p); h >>= 4; rem -= 4; }
        else if (rem == 3) { gs_pass<3>(sm, V, h, tw, p); h >>= 3; rem -= 3; }
        else if (rem == 2) { gs_pass<2>(sm, V, h, tw, p); h >>= 2; rem -= 2; }
        else               { gs_pass<1>(sm, V, h, tw, p); h >>= 1; rem -= 1; }
        __syncthreads();
    }
}

// Full inverse transform (times L) of every vector.
__device__ __forceinline__ void ntt_inverse(uint32_t* sm, const VecLayout& V,
                                            const uint2* __restrict__ twi, uint32_t p)
{
    int rem = V.logL;
    int h = 1;
    while (rem > 0) {
        if (rem >= 4)      { ct_pass<4>(sm, V, h, twi, p); h <<= 4; rem -= 4; }
        else if (rem == 3) { ct_pass<3>(sm, V, h, twi, p); h <<= 3; rem -= 3; }
        else if (rem == 2) { ct_pass<2>(sm, V, h, twi, p); h <<= 2; rem -= 2; }
        else               { ct_pass<1>(sm, V, h, twi, p); h <<= 1; rem -= 1; }
        __syncthreads();
    }
}

}  // namespace fb
