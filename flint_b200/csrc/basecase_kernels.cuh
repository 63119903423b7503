// Basecase (schoolbook) product for small or very unbalanced operands.
//
// For a short operand y (yn <= BASECASE_MAX limbs) the column sums
//     s_k = sum_j x[k - j] y[j],   0 <= k < xn + yn - 1,
// are below yn 2^128 < 2^138 and are accumulated exactly as 192-bit values;
// they are written as three planes of 64-bit words and the carry kernel's
// direct mode (k_crt_carry<0>) turns them into limbs.  The number-theoretic
// transform path has a fixed cost of four launches and 2 np M residues, which
// this path avoids; it wins when yn is small, whatever xn is.
//
// The reference routes such operands to GMP's basecase and Karatsuba code
// through flint_mpn_mul's size thresholds (src/mpn_extras/mul.c:52-75).
#pragma once
#include <stdint.h>

namespace fb {

constexpr int BASECASE_MAX = 1024;
constexpr int BASECASE_THREADS = 256;

__device__ __forceinline__ void mac192(uint64_t& a0, uint64_t& a1, uint64_t& a2, uint64_t x, uint64_t y)
{
    const uint64_t lo = x * y, hi = __umul64hi(x, y);
    asm("add.cc.u64  %0, %0, %3;\n\t"
        "addc.cc.u64 %1, %1, %4;\n\t"
        "addc.u64    %2, %2, 0;"
        : "+l"(a0), "+l"(a1), "+l"(a2)
        : "l"(lo), "l"(hi));
}

// grid = ceil((xn + yn - 1) / THREADS); thread k0 + t computes s_(k0+t).
// planes: s[k], s[P + k], s[2 P + k] with plane stride P >= xn + yn - 1.
__global__ void __launch_bounds__(BASECASE_THREADS)
k_basecase_sums(const uint64_t* __restrict__ x, uint64_t xn, const uint64_t* __restrict__ y,
                uint32_t yn, uint64_t* __restrict__ s, uint64_t P)
{
    __shared__ uint64_t sy[BASECASE_MAX];
    __shared__ uint64_t sx[BASECASE_THREADS + BASECASE_MAX];
    const uint64_t k0 = (uint64_t)blockIdx.x * BASECASE_THREADS;
    for (uint32_t i = threadIdx.x; i < yn; i += BASECASE_THREADS) sy[i] = y[i];
    // x window k0 - (yn - 1) .. k0 + THREADS - 1, zero outside [0, xn)
    const int64_t xb = (int64_t)k0 - (int64_t)(yn - 1);
    for (uint32_t i = threadIdx.x; i < BASECASE_THREADS + yn - 1; i += BASECASE_THREADS) {
        const int64_t xi = xb + (int64_t)i;
        sx[i] = (xi >= 0 && (uint64_t)xi < xn) ? x[xi] : 0ull;
    }
    __syncthreads();
    const uint64_t k = k0 + threadIdx.x;
    const uint64_t L = xn + yn - 1;
    uint64_t a0 = 0, a1 = 0, a2 = 0;
    const uint64_t* px = sx + threadIdx.x + (yn - 1);   // px[-j] = x[k - j]
#pragma unroll 4
    for (uint32_t j = 0; j < yn; j++) mac192(a0, a1, a2, px[-(int)j], sy[j]);
    if (k < L) {
        s[k] = a0;
        s[P + k] = a1;
        s[2 * P + k] = a2;
    }
}

}  // namespace fb
