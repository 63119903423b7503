// Integer-polynomial products: signed CRT and per-coefficient recombination.
//
// The operands' coefficients were split into 64-bit chunks and laid out as
// polynomials in y with slot stride S (FzShape), so output coefficient j is
//     c_j = sum_{t < S} C_{jS+t} 2^(64 t),
// where C_n is the coefficient of y^n in the chunk product.  |C_n| is below
// min(an, bn) min(wa, wb) 2^128 < P/2, so the CRT's symmetric residue is C_n
// itself, signed: crt_values returns X = sum y_j (P/p_j) - round(sum y_j/p_j) P,
// which for a signed C_n is its two's complement over the CRT words.
//
// The reference reaches the same products through _fmpz_poly_mul_mid_mpn_ctx
// (src/fft_small/fmpz_poly_mul.c:309-401, multimodular with its CRT helpers)
// and, for large coefficients, Kronecker substitution into flint_mpn_mul
// (src/fmpz_poly/mul.c:100-186).  The chunk layout here covers both ranges
// with one transform length rule.
#pragma once
#include "mpn_kernels.cuh"

namespace fb {

// One thread per output coefficient j in [zl, zh): zw limbs of c_j in two's
// complement at z + (j - zl) zw (truncated to zw limbs, sign-extended above
// the S + 2 limbs a coefficient can occupy).
template <int NP>
__global__ void __launch_bounds__(256)
k_fmpz_crt(const uint32_t* __restrict__ res, int logM, uint64_t Ly, uint32_t S, uint64_t zl,
           uint64_t zh, uint32_t zw, uint64_t* __restrict__ z, CrtConst K)
{
    const uint64_t j = zl + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= zh) return;
    uint64_t* __restrict__ out = z + (j - zl) * zw;
    const uint64_t n0 = j * S;
    // limb u of c_j: lo(C_u) + mid(C_{u-1}) + hi(C_{u-2}) + carry, hi signed
    uint64_t mid1 = 0, hi1 = 0, hi2 = 0;   // mid(C_{u-1}), hi(C_{u-1}), hi(C_{u-2})
    __int128 carry = 0;
    const uint32_t top = S + 2;
    for (uint32_t u = 0; u < zw; u++) {
        uint64_t c0 = 0, c1 = 0, c2 = 0;
        const uint64_t n = n0 + u;
        if (u < S && n < Ly) {
            uint32_t y[NP];
#pragma unroll
            for (int jp = 0; jp < NP; jp++) y[jp] = res[((size_t)jp << logM) + n];
            crt_values<NP>(y, K, c0, c1, c2);
            if (NP == 5) c2 = (uint64_t)(int64_t)(int32_t)(uint32_t)c2;   // 160-bit sign
        }
        if (u < top) {
            const __int128 acc = carry + (__int128)c0 + (__int128)mid1 + (__int128)(int64_t)hi2;
            out[u] = (uint64_t)acc;
            carry = acc >> 64;
        } else {
            out[u] = (uint64_t)(int64_t)carry;   // sign extension: carry is 0 or -1
        }
        hi2 = hi1;
        hi1 = c2;
        mid1 = c1;
    }
}

// The same coefficients, J = max(1, min(256, FZ_CRT_POS / S)) per block
// (slot strides S <= FZ_CRT_POS): the block first recombines every chunk
// position of its J coefficients by CRT -- one thread per position, so the
// residue loads are coalesced and all positions are in flight at once -- into
// shared memory, then one thread per coefficient runs k_fmpz_crt's limb loop
// on those values.  k_fmpz_crt ran one thread per coefficient over all its
// positions (a wide coefficient is a long chain of dependent loads, and a
// product has few coefficients per SM).
constexpr uint32_t FZ_CRT_POS = 2048;

template <int NP>
__global__ void __launch_bounds__(256)
k_fmpz_crt_tiled(const uint32_t* __restrict__ res, int logM, uint64_t Ly, uint32_t S, uint32_t J,
                 uint64_t zl, uint64_t zh, uint32_t zw, uint64_t* __restrict__ z, CrtConst K)
{
    __shared__ uint64_t sc0[FZ_CRT_POS], sc1[FZ_CRT_POS], sc2[FZ_CRT_POS];
    const uint64_t j0 = zl + (uint64_t)blockIdx.x * J;
    if (j0 >= zh) return;
    const uint32_t nj = (uint32_t)(zh - j0 < J ? zh - j0 : J);
    const uint64_t p0 = j0 * S;
    const uint32_t npos = nj * S;
    for (uint32_t t = threadIdx.x; t < npos; t += blockDim.x) {
        const uint64_t n = p0 + t;
        uint64_t c0 = 0, c1 = 0, c2 = 0;
        if (n < Ly) {
            uint32_t y[NP];
#pragma unroll
            for (int jp = 0; jp < NP; jp++) y[jp] = res[((size_t)jp << logM) + n];
            crt_values<NP>(y, K, c0, c1, c2);
            if (NP == 5) c2 = (uint64_t)(int64_t)(int32_t)(uint32_t)c2;   // 160-bit sign
        }
        sc0[t] = c0;
        sc1[t] = c1;
        sc2[t] = c2;
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < nj; q += blockDim.x) {
        uint64_t* __restrict__ out = z + (j0 + q - zl) * zw;
        const uint32_t base = q * S;
        uint64_t mid1 = 0, hi1 = 0, hi2 = 0;
        __int128 carry = 0;
        const uint32_t top = S + 2;
        for (uint32_t u = 0; u < zw; u++) {
            uint64_t c0 = 0, c1 = 0, c2 = 0;
            if (u < S) {
                c0 = sc0[base + u];
                c1 = sc1[base + u];
                c2 = sc2[base + u];
            }
            if (u < top) {
                const __int128 acc = carry + (__int128)c0 + (__int128)mid1 + (__int128)(int64_t)hi2;
                out[u] = (uint64_t)acc;
                carry = acc >> 64;
            } else {
                out[u] = (uint64_t)(int64_t)carry;
            }
            hi2 = hi1;
            hi1 = c2;
            mid1 = c1;
        }
    }
}

}  // namespace fb
