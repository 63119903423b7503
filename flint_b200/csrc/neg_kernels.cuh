// Negacyclic products z = x y mod 2^N + 1, batched: the pointwise stage of
// Schoenhage-Strassen convolutions.
//
// Operands have n + 1 limbs (N = 64 n): n low limbs and a top limb that is 0
// or 1 (2^N itself, or an unreduced value below 2^(N+1)).  With N = m b, an
// operand is the polynomial X(t) = sum_(i<m) x_i t^i in b-bit digits at
// t = 2^b, and x y mod 2^N + 1 is [X Y mod (t^m + 1)](2^b) mod 2^N + 1.  The
// negacyclic product X Y mod t^m + 1 is a cyclic one after the twist
// t -> omega t, omega^m = -1 (omega of order 2m):
//
//   k_neg_split     digit i -> residue, times omega^i        [per prime]
//   k_rows          length-m forward transforms of x and y, pointwise product
//                   with 2^128 / m, inverse transform (the mpn row kernel, one
//                   row per product)
//   k_neg_finish    per product: untwist omega^-i with the CRT cofactor
//                   inverse, add a bias B = 2^(2b + log m) so every coefficient
//                   is non-negative, CRT, recompose sum V_i 2^(b i) with the
//                   carries, add (-biaspoly mod 2^N + 1), fold mod 2^N + 1.
//
// The staged variant (a cached transform of y) runs k_rows_fwd on x,
// k_neg_pointwise against the cached spectrum and k_rows_inv instead of k_rows.
//
// Reference counterpart: src/fft_small/negacyclic.c (digits, twist w^i and
// untwist w^-i m^-1, bias polynomial, CRT recomposition and fold,
// negacyclic.c:65-175, 291-489); residues here are modulo 31-bit primes
// instead of the reference's 50-bit primes in doubles.
#pragma once
#include "mpn_kernels.cuh"

namespace fb {

struct NegShape {
    uint32_t n;        // limbs below 2^N; operands and results have n + 1 limbs
    uint32_t b;        // digit bits, N = m b, b <= 127
    int logm;          // m = 2^logm digits, 5 <= logm <= 14
    int logR;          // prime stride of the residue buffers: 2^(logR + logm) words
    uint64_t stride;   // limbs between consecutive operands / results of a batch
};

struct NegConst {
    uint32_t biasres[MAX_NP];   // B (P/p_k)^-1 mod p_k
    uint32_t vb;                // bits of the biased coefficients V_i = c_i + B
    uint32_t hl;                // limbs of the recomposed value above 2^N
    uint32_t tl;                // limbs per recomposition tile
};

// Residues of the digits of `count` operands, twisted by omega^i (tw holds
// omega^i 2^32 mod p_k, so one Montgomery product applies it).  Residues keep
// the mpn path's convention (value 2^-32 mod p).  Element (k, prod, i) goes to
// buf[k 2^(logR + logm) + prod m + i].
__global__ void k_neg_split(DevTables T, const uint64_t* __restrict__ x, uint32_t count, NegShape sh,
                            int np, const uint32_t* __restrict__ tw, uint32_t* __restrict__ buf)
{
    const uint32_t m = 1u << sh.logm;
    const uint64_t total = (uint64_t)count << sh.logm;
    const uint32_t b = sh.b;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t prod = (uint32_t)(e >> sh.logm), i = (uint32_t)e & (m - 1);
        const uint64_t* __restrict__ xp = x + (size_t)prod * sh.stride;
        // digit i = bits [b i, b i + b) of the n low limbs (b i + b <= 64 n)
        const uint64_t bit = (uint64_t)b * i;
        const uint32_t l = (uint32_t)(bit >> 6), o = (uint32_t)(bit & 63);
        const uint64_t w0 = xp[l];
        const uint64_t w1 = l + 1 < sh.n ? xp[l + 1] : 0ull;
        const uint64_t w2 = (b > 64 && l + 2 < sh.n) ? xp[l + 2] : 0ull;
        uint64_t d0 = o ? (w0 >> o) | (w1 << (64 - o)) : w0;
        uint64_t d1 = o ? (w1 >> o) | (w2 << (64 - o)) : w1;
        if (b < 64) { d0 &= (1ull << b) - 1; d1 = 0; }
        else if (b == 64) d1 = 0;
        else d1 &= (1ull << (b - 64)) - 1;
        // a top limb 1 stands for 2^N = -1: digit 0 loses one
        const bool top = i == 0 && xp[sh.n] != 0;
        for (int k = 0; k < np; k++) {
            const PrimeInfo P = T.pi[k];
            uint32_t r = limb_redc(d0, P.p, P.pneg_inv, P.c32);              // d0 2^-32
            if (d1) r = add_mod(r, mul_mont((uint32_t)d1, P.r2, P.p, P.pneg_inv), P.p);   // + d1 2^32
            if (top) r = sub_mod(r, limb_redc(1ull, P.p, P.pneg_inv, P.c32), P.p);
            buf[((size_t)k << (sh.logR + sh.logm)) + e] =
                mul_mont(r, tw[((size_t)k << sh.logm) + i], P.p, P.pneg_inv);
        }
    }
}

// X <- X F scale_k 2^-64 (the fused row pass's pointwise normalisation) on
// rows 0 .. count-1 of every prime; X and F share the layout of k_neg_split.
__global__ void k_neg_pointwise(DevTables T, uint32_t* __restrict__ X, const uint32_t* __restrict__ F,
                                uint32_t count, int logm, int logR, int np,
                                const uint32_t* __restrict__ scale)
{
    const uint64_t per = (uint64_t)count << logm;
    const uint64_t total = per * np;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const int k = (int)(e / per);
        const size_t idx = ((size_t)k << (logR + logm)) + (e - (uint64_t)k * per);
        const PrimeInfo& P = T.pi[k];
        X[idx] = mul_mont(mul_mont(X[idx], F[idx], P.p, P.pneg_inv), scale[k], P.p, P.pneg_inv);
    }
}

// bits [s, s + 64) of the 192-bit value (v0, v1, v2), s in (-64, 192)
__device__ __forceinline__ uint64_t bits64(uint64_t v0, uint64_t v1, uint64_t v2, int s)
{
    if (s < 0) return v0 << (-s);
    const int w = s >> 6, o = s & 63;
    const uint64_t lo = w == 0 ? v0 : (w == 1 ? v1 : v2);
    const uint64_t hi = w == 0 ? v1 : (w == 1 ? v2 : 0ull);
    return o ? (lo >> o) | (hi << (64 - o)) : lo;
}

#ifndef FB_NEG_THREADS
#define FB_NEG_THREADS 512
#endif
constexpr int NEG_THREADS = FB_NEG_THREADS;   // one output limb per thread per tile
constexpr int NEG_CMAX = 2560;   // biased coefficients held per recomposition tile

// Carry-lookahead over one tile (one limb per thread): (g, p) -> carry into
// this thread's limb from the positions below it in the block.
__device__ __forceinline__ bool neg_block_carry_in(bool g, bool p, uint32_t* s_warp)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int NW = NEG_THREADS / 32;
    // inclusive warp scan of (g, p): (g2, p2) o (g1, p1) = (g2 | p2 g1, p2 p1)
    bool G = g, Pp = p;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const bool g1 = __shfl_up_sync(0xffffffffu, G, d);
        const bool p1 = __shfl_up_sync(0xffffffffu, Pp, d);
        if (lane >= d) { G = G || (Pp && g1); Pp = Pp && p1; }
    }
    if (lane == 31) s_warp[wid] = (G ? 1u : 0u) | (Pp ? 2u : 0u);
    __syncthreads();
    if (wid == 0) {
        const uint32_t v = lane < NW ? s_warp[lane] : 0u;
        bool WG = v & 1u, WP = (v & 2u) != 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const bool g1 = __shfl_up_sync(0xffffffffu, WG, d);
            const bool p1 = __shfl_up_sync(0xffffffffu, WP, d);
            if (lane >= d) { WG = WG || (WP && g1); WP = WP && p1; }
        }
        // exclusive: carry out of the warps below lane
        const bool ex = __shfl_up_sync(0xffffffffu, WG, 1);
        if (lane < NW) s_warp[NW + lane] = (lane > 0 && ex) ? 1u : 0u;
    }
    __syncthreads();
    const bool cw = s_warp[NW + wid] != 0;              // carry into this warp
    // exclusive within the warp, then the warp's carry through the lanes below
    const bool gx = __shfl_up_sync(0xffffffffu, G, 1);
    const bool px = __shfl_up_sync(0xffffffffu, Pp, 1);
    bool c;
    if (lane == 0) c = cw;
    else c = gx || (px && cw);
    __syncthreads();   // s_warp is reused by the next tile
    return c;
}

// One CTA per product: untwist, bias, CRT, recomposition, fold.
// buf: residues after the inverse transforms (natural order, layout of
// k_neg_split); itw holds omega^-i (P/p_k)^-1 2^32 mod p_k; beta holds
// (-sum_i B 2^(b i)) mod 2^N + 1 in n + 1 limbs.  Dynamic shared memory:
// 3 NEG_CMAX 64-bit words.
template <int NP>
__global__ void __launch_bounds__(NEG_THREADS)
k_neg_finish(DevTables T, const uint32_t* __restrict__ buf, const uint32_t* __restrict__ itw,
             CrtConst K, NegConst Q, NegShape sh, const uint64_t* __restrict__ beta,
             uint64_t* __restrict__ z)
{
    extern __shared__ uint64_t sv[];               // [3][NEG_CMAX] coefficient words
    __shared__ uint32_t s_warp[2 * NEG_THREADS / 32];
    __shared__ uint64_t s_top[4];                  // limbs n .. n + hl - 1
    __shared__ uint64_t s_cin;                     // carry into the next tile
    __shared__ int s_first;
    const int t = threadIdx.x;
    const uint32_t prod = blockIdx.x;
    const uint32_t m = 1u << sh.logm, b = sh.b, n = sh.n;
    const int64_t vb = Q.vb;
    const uint32_t whi = n + Q.hl;
    uint64_t* __restrict__ zp = z + (size_t)prod * sh.stride;
    const size_t pstride = (size_t)1 << (sh.logR + sh.logm);
    const uint32_t* __restrict__ rp = buf + ((size_t)prod << sh.logm);
    if (t == 0) s_cin = 0;
    __syncthreads();

    for (uint32_t J = 0; J < whi; J += Q.tl) {
        const uint32_t jend = min(whi, J + Q.tl);
        // coefficients overlapping limbs [J, jend): b i + vb > 64 J, b i < 64 jend
        const int64_t lo_bits = 64 * (int64_t)J - vb;
        const uint32_t i_lo = lo_bits < 0 ? 0u : (uint32_t)(lo_bits / b) + 1;
        const uint32_t i_hi = min(m - 1, (uint32_t)((64 * (uint64_t)jend - 1) / b));
        const int nco = i_hi >= i_lo ? (int)(i_hi - i_lo + 1) : 0;
        for (int c = t; c < nco; c += NEG_THREADS) {
            const uint32_t i = i_lo + c;
            uint32_t y[NP];
#pragma unroll
            for (int k = 0; k < NP; k++) {
                const PrimeInfo& P = T.pi[k];
                const uint32_t r = mul_mont(rp[k * pstride + i], itw[((size_t)k << sh.logm) + i], P.p,
                                            P.pneg_inv);
                y[k] = add_mod(r, Q.biasres[k], P.p);
            }
            uint64_t c0, c1, c2;
            crt_values<NP>(y, K, c0, c1, c2);
            sv[c] = c0;
            sv[NEG_CMAX + c] = c1;
            sv[2 * NEG_CMAX + c] = c2;
        }
        __syncthreads();
        // limb j = J + t: sum of the overlapping 64-bit pieces (+ beta_j)
        const uint32_t j = J + t;
        const bool live = j < jend;
        uint64_t lo = 0, hi = 0;
        if (live) {
            if (j <= n) lo = beta[j];
            const int64_t jb = 64 * (int64_t)j;
            const uint32_t ia = jb - vb < 0 ? 0u : (uint32_t)((jb - vb) / b) + 1;
            const uint32_t ib = min(m - 1, (uint32_t)((jb + 63) / b));
            for (uint32_t i = max(ia, i_lo); i <= ib; i++) {
                const int c = (int)(i - i_lo);
                const uint64_t piece = bits64(sv[c], sv[NEG_CMAX + c], sv[2 * NEG_CMAX + c],
                                              (int)(jb - (int64_t)b * i));
                lo += piece;
                hi += lo < piece;
            }
        }
        // s_j = lo_j + hi_(j-1) (the tile's carry-in for its first limb)
        uint64_t hprev = __shfl_up_sync(0xffffffffu, hi, 1);
        if ((t & 31) == 0) hprev = 0;
        __syncthreads();                        // every thread has read sv; s_warp is free
        if ((t & 31) == 31) s_warp[t >> 5] = (uint32_t)hi;   // hi < 2^32 (few pieces)
        __syncthreads();
        if ((t & 31) == 0) hprev = t == 0 ? s_cin : (uint64_t)s_warp[(t >> 5) - 1];
        __syncthreads();
        const uint64_t s = lo + hprev;
        const bool g = live && s < lo;
        const bool p = live && s == ~0ull;
        const bool cin = neg_block_carry_in(g, p, s_warp);
        if (live) {
            const uint64_t v = s + (cin ? 1ull : 0ull);
            if (j < n) zp[j] = v;
            else s_top[j - n] = v;
            if (j == jend - 1) s_cin = hi + ((g || (p && cin)) ? 1ull : 0ull);
        }
        __syncthreads();
    }

    // fold: z = W_lo - W_hi mod 2^N + 1, W_hi = s_top[0 .. hl)
    const uint32_t hl = Q.hl;
    const uint32_t hs = min(hl, n);            // low limbs the subtraction touches directly
    __shared__ uint64_t s_d[4];
    __shared__ int s_borrow;
    if (t == 0) {
        uint64_t br = 0;
        for (uint32_t k = 0; k < hs; k++) {
            const uint64_t a = zp[k], h = s_top[k];
            const uint64_t d = a - h - br;
            br = (a < h) || (a - h < br) ? 1ull : 0ull;
            s_d[k] = d;
        }
        // W_hi limbs beyond n (only when n < hl) count 2^N each: -2^N = +1
        // mod 2^N + 1; such tiny rings are excluded on the host (n >= hl)
        s_borrow = (int)br;
        s_first = (int)n;
    }
    __syncthreads();
    const bool borrow = s_borrow != 0;
    __syncthreads();                           // s_borrow is rewritten below
    if (borrow) {
        // the borrow runs up to the first non-zero limb at or above hs
        for (uint32_t base = hs; base < n; base += NEG_THREADS) {
            const uint32_t k = base + t;
            const bool nz = k < n && zp[k] != 0;
            if (nz) atomicMin(&s_first, (int)k);
            if (__syncthreads_or(nz)) break;
        }
        const uint32_t f = (uint32_t)s_first;
        if (f < n) {
            // D = W_lo - W_hi >= 0: limbs [hs, f) become all ones, limb f drops by one
            for (uint32_t k = hs + t; k < f; k += NEG_THREADS) zp[k] = ~0ull;
            if (t == 0) {
                zp[f] = zp[f] - 1;
                for (uint32_t k = 0; k < hs; k++) zp[k] = s_d[k];
                zp[n] = 0;
            }
        } else {
            // W_lo < W_hi: D = W_lo - W_hi + 2^N has ones in [hs, n); z = D + 1
            if (t == 0) {
                uint64_t cy = 1;
                for (uint32_t k = 0; k < hs; k++) {
                    s_d[k] += cy;
                    cy = (cy && s_d[k] == 0) ? 1ull : 0ull;
                }
                s_borrow = (int)cy + 1;           // 2: the increment ran through all limbs
            }
            __syncthreads();
            const bool wrap = s_borrow == 2;     // D + 1 = 2^N
            for (uint32_t k = hs + t; k < n; k += NEG_THREADS) zp[k] = wrap ? 0ull : ~0ull;
            if (t == 0) {
                for (uint32_t k = 0; k < hs; k++) zp[k] = wrap ? 0ull : s_d[k];
                zp[n] = wrap ? 1ull : 0ull;
            }
        }
    } else if (t == 0) {
        for (uint32_t k = 0; k < hs; k++) zp[k] = s_d[k];
        zp[n] = 0;
    }
}

}  // namespace fb
