// nmod polynomial products: CRT of the exact coefficient followed by a
// reduction modulo the user's word-size modulus n.
//
// Reference: the per-prime reduction of the inputs and the CRT back to Z/nZ
// in src/fft_small/nmod_poly_mul.c:33-232 (_mod, _mod_red) and 239-659
// (_crt_1/_crt_2/_crt_3, CRT_DEFINE).  Here the inputs go through the same
// split kernel as the integer path (a coefficient < n < 2^64 is one limb),
// and the exact coefficient from the CRT is reduced mod n with division by
// an invariant integer (N. Moller and T. Granlund, "Improved division by
// invariant integers", IEEE Trans. Computers 60 (2011), Algorithm 4).
#pragma once
#include "mpn_kernels.cuh"

namespace fb {

struct NmodConst {
    uint64_t n;     // modulus
    uint64_t dn;    // n << shift (normalised)
    uint64_t v;     // floor((2^128 - 1) / dn) - 2^64
    int shift;      // leading zeros of n
};

// (u1 2^64 + u0) mod d for normalised d, u1 < d
__device__ __forceinline__ uint64_t divrem21(uint64_t u1, uint64_t u0, uint64_t d, uint64_t v)
{
    uint64_t q0 = v * u1;
    uint64_t q1 = __umul64hi(v, u1);
    const uint64_t s = q0 + u0;
    q1 += u1 + 1 + (s < q0);
    q0 = s;
    uint64_t r = u0 - q1 * d;
    if (r > q0) r += d;
    if (r >= d) r -= d;
    return r;
}

__device__ __forceinline__ uint64_t reduce192(uint64_t c0, uint64_t c1, uint64_t c2, const NmodConst& N)
{
    const int s = N.shift;
    uint64_t w3 = 0, w2 = c2, w1 = c1, w0 = c0;
    if (s) {
        w3 = c2 >> (64 - s);
        w2 = (c2 << s) | (c1 >> (64 - s));
        w1 = (c1 << s) | (c0 >> (64 - s));
        w0 = c0 << s;
    }
    uint64_t r = divrem21(w3, w2, N.dn, N.v);
    r = divrem21(r, w1, N.dn, N.v);
    r = divrem21(r, w0, N.dn, N.v);
    return r >> s;
}

// z[k - zl] = h_k mod n for k in [zl, zh); requires zh <= number of
// coefficients with exact values in the cyclic result.
template <int NP>
__global__ void __launch_bounds__(256)
k_crt_nmod(const uint32_t* __restrict__ res, int logM, uint64_t zl, uint64_t zh,
           uint64_t* __restrict__ z, CrtConst K, NmodConst N)
{
    const uint64_t k = zl + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= zh) return;
    uint64_t c0, c1, c2;
    const uint64_t pos = k & (((uint64_t)1 << logM) - 1);
    crt_coeff<NP>(res, logM, pos, K, c0, c1, c2);
    z[k - zl] = reduce192(c0, c1, c2, N);
}

}  // namespace fb

namespace fb {

// Elementwise helpers of the nmod division (values in [0, n), n < 2^64).
__device__ __forceinline__ uint64_t nmod_add64(uint64_t x, uint64_t y, uint64_t n)
{
    const uint64_t s = x + y;
    return (s < x || s >= n) ? s - n : s;
}

__device__ __forceinline__ uint64_t nmod_sub64(uint64_t x, uint64_t y, uint64_t n)
{
    return x >= y ? x - y : x - y + n;
}

// dst[i] = src[len - 1 - i]
__global__ void k_nmod_reverse(uint64_t* __restrict__ dst, const uint64_t* __restrict__ src, uint64_t len)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
         i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[len - 1 - i];
}

// dst[i] = -src[i] mod n
__global__ void k_nmod_neg(uint64_t* __restrict__ dst, const uint64_t* __restrict__ src, uint64_t len,
                           uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
         i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[i] ? n - src[i] : 0;
}

// dst[i] = sum_{k = i mod N, k < an} a[k] mod n, for i < N (a mod x^N - 1)
__global__ void k_nmod_fold(uint64_t* __restrict__ dst, const uint64_t* __restrict__ a, uint64_t an,
                            uint64_t N, uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = 0;
        for (uint64_t k = i; k < an; k += N) s = nmod_add64(s, a[k], n);
        dst[i] = s;
    }
}

// r[i] = (sum_{k = i mod N, k < an} a[k]) - c[i] mod n, for i < cnt
// (the reference's _nmod_poly_sub_mod_xpNm1, nmod_poly_mul.c:1196-1212)
__global__ void k_nmod_fold_sub(uint64_t* __restrict__ r, const uint64_t* __restrict__ a, uint64_t an,
                                uint64_t N, const uint64_t* __restrict__ c, uint64_t cnt, uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = nmod_sub64(a[i], c[i], n);
        for (uint64_t k = i + N; k < an; k += N) s = nmod_add64(s, a[k], n);
        r[i] = s;
    }
}

}  // namespace fb
