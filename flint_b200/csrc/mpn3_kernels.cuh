// Column passes of transforms of M = 3 2^k points (the truncated lengths
// between powers of two).
//
// The reference truncates its transforms to multiples of its 256-point
// blocks (sd_fft_trunc, src/fft_small/sd_fft.c:1230-1274; sd_ifft_trunc,
// src/fft_small/sd_ifft.c:1503-1533), so its cost follows an + bn smoothly.
// Here a product whose length L satisfies 2^(k+1) < L <= 3 2^k runs a
// 3 2^k-point cyclic transform instead of a 2^(k+2)-point one: 3/4 of the
// work.  The four-step split keeps rows of C = 2^13 points (the row pass is
// unchanged) and makes the columns R = 3 R' long, R' = 2^r:
//
//   forward column  radix-3 stage over (u, u + R', u + 2R') with twiddles
//                   omega_R^(u v2), then three length-R' Gentleman-Sande
//                   transforms (the power-of-two column code on each third),
//                   twist w_M^(i v) with v = 3 bitrev_r(u') + v2;
//   inverse column  untwist, three length-R' Cooley-Tukey transforms,
//                   inverse radix-3 stage.
//
// All primes used here (the first NP3) have roots of order 3 2^25: w3, with
// w3^3 = w the root of order 2^25 behind the power-of-two tables, so the
// mixed transform evaluates the input at every M-th root of unity and each
// stage is undone by its inverse.  Residue planes keep a power-of-two
// stride (2^(k+2) words), so the row pass and the CRT/carry kernel read
// them unchanged.
//
// Radix-3 butterfly (w of order 3, c = w - w^2): with a = x1 + x2 and
// b = x1 - x2, t0 = x0 + a and 2 t1 = 2 x0 - a + c b, 2 t2 = 2 x0 - a - c b;
// the halving is folded into the stage twiddles (tables hold omega^e / 2), so
// a triple costs three Shoup products.  The inverse uses
// c' = w^-1 - w^-2 and x0 = t0 + 2 h, x1 = t0 - h + c' g, x2 = t0 - h - c' g
// with h = (t1 + t2) / 2 and g = (t1 - t2) / 2 (the 1/3 is part of the 1/M
// of the pointwise scale).
#pragma once
#include "mpn_kernels.cuh"

namespace fb {

// columns per tile: 3 2^r rows x G columns of at most 3 2^13 words, G >= 8
__host__ __device__ constexpr int cols_per_tile3(int logR) { return logR >= 10 ? 8 : (1 << (13 - logR)); }

__device__ __forceinline__ uint32_t table_power3(uint32_t e, const uint2* __restrict__ th3,
                                                 const uint2* __restrict__ tl3, uint32_t p)
{
    const uint2 w1 = th3[e >> 13];
    const uint2 w2 = tl3[e & 8191];
    return mul_shoup(w1.x, w2.x, w2.y, p);
}

// Twist of the 32 consecutive positions u' = 32 s + m of third t of a column:
// position gets w_M^(col v), v = 3 bitrev_r(u') + t, w_M = w3^(2^(25 - k)).
// As in twist32: factors alpha beta^bitrev5(m) from a Shoup chain, applied
// with Montgomery products; fsc != 0 folds a pointwise scale in.
template <int LOGR>
__device__ __forceinline__ void twist32_3(uint32_t (&x)[32], uint32_t col, int s, int t, int k,
                                          const uint2* __restrict__ th3, const uint2* __restrict__ tl3,
                                          const PrimeInfo& P, uint32_t fsc)
{
    const uint32_t p = P.p;
    const int sh = LOG_MAXM - k;
    // col v < M = 3 2^k, so exponents stay below 3 2^25
    const uint32_t e0 = (col * (uint32_t)(t + 3 * (int)bitrev_bits((uint32_t)s, LOGR - 5))) << sh;
    const uint32_t e1 = (col * (3u << (LOGR - 5))) << sh;
    const uint32_t alpha = table_power3(e0, th3, tl3, p);
    const uint32_t beta = table_power3(e1, th3, tl3, p);
    const uint32_t bq = shoup_companion_dev(beta, p);
    uint32_t F = mul_mont(alpha, P.r2, p, P.pneg_inv);
    if (fsc) F = mul_mont(F, fsc, p, P.pneg_inv);
#pragma unroll
    for (int kk = 0; kk < 32; kk++) {
        const int m = (int)(__brev((unsigned)kk) >> 27);
        x[m] = mul_mont(x[m], F, p, P.pneg_inv);
        if (kk < 31) F = mul_shoup(F, beta, bq, p);
    }
}

// The strided passes of the three thirds of a column tile (three independent
// transforms of 2^LOGL points down G columns, `third` words apart): each pass
// runs on all three before one barrier, instead of three pass sequences with
// a barrier after every pass.
template <int LOGL, int G, int QMAX, int H, int REM>
__device__ __forceinline__ void gs_passes3(uint32_t* sm, int third, const uint2* __restrict__ tw, uint32_t p)
{
    if constexpr (REM > 0) {
        constexpr int Q = balanced_pass<REM, QMAX>();
#pragma unroll 1
        for (int t = 0; t < 3; t++) gs_pass_smem<LOGL, Q, H, G>(sm + t * third, 1, tw, p);
        __syncthreads();
        gs_passes3<LOGL, G, QMAX, (H >> Q), REM - Q>(sm, third, tw, p);
    }
}
template <int LOGL, int G, int QMAX, int H, int REM>
__device__ __forceinline__ void ct_passes3(uint32_t* sm, int third, const uint2* __restrict__ twi, uint32_t p)
{
    if constexpr (REM > 0) {
        constexpr int Q = balanced_pass<REM, QMAX>();
#pragma unroll 1
        for (int t = 0; t < 3; t++) ct_pass_smem<LOGL, Q, H, G>(sm + t * third, 1, twi, p);
        __syncthreads();
        ct_passes3<LOGL, G, QMAX, (H << Q), REM - Q>(sm, third, twi, p);
    }
}
// as gs_strided_all / ct_strided_all with their column-layout defaults (QMAX
// 4, the five lowest levels left to the register pass)
template <int LOGL, int G>
__device__ __forceinline__ void gs_strided_all3(uint32_t* sm, int third, const uint2* __restrict__ tw, uint32_t p)
{
    if constexpr (LOGL > 5) gs_passes3<LOGL, G, 4, (1 << (LOGL - 1)), LOGL - 5>(sm, third, tw, p);
}
template <int LOGL, int G>
__device__ __forceinline__ void ct_strided_all3(uint32_t* sm, int third, const uint2* __restrict__ twi, uint32_t p)
{
    if constexpr (LOGL > 5) ct_passes3<LOGL, G, 4, (1 << 5), LOGL - 5>(sm, third, twi, p);
}

// Forward column pass of a 3 2^k-point transform: limbs -> residues, radix-3
// stage, three length-2^LOGR transforms, twist.  grid = (np, C / G, operands);
// block 512; smem = padw(3 2^LOGR G) + 32 words.  logMs: log2 of the residue
// plane stride; rows of C = 2^LOGC3 points.  fscale / fmask as in k_fwd_cols;
// FZ: integer-polynomial operands (an, bn coefficients, chunk layout fz) as in
// k_fwd_cols.
constexpr int LOGC3 = 13;
template <int LOGR, int G, bool FZ = false>
__global__ void __launch_bounds__(512)
k_fwd_cols3(DevTables T, const uint64_t* __restrict__ a, uint64_t an, const uint64_t* __restrict__ b,
            uint64_t bn, uint32_t* __restrict__ ra, uint32_t* __restrict__ rb, int logMs, int k,
            const uint32_t* __restrict__ fscale, int fmask, FzShape fz)
{
    extern __shared__ uint32_t sm[];
    constexpr int RP = 1 << LOGR;           // R' (power-of-two part of the column)
    constexpr int C = 1 << LOGC3;
    const int j = blockIdx.x;
    const int i0 = blockIdx.y * G;
    const bool opb = (blockIdx.z & 1) != 0;
    const uint64_t* __restrict__ x = opb ? b : a;
    const uint64_t xn = opb ? bn : an;
    uint32_t* __restrict__ out = (opb ? rb : ra) + ((size_t)j << logMs);
    const PrimeInfo P = T.pi[j];
    const uint32_t p = P.p;

    // limbs of rows 0 .. 3R' - 1 (element n = u C + i; zero beyond the operand).
    // blockDim == 512: thread t loads rows u_t + k 512/G of its column, so its
    // shared offsets are compile-time constants and its global address a
    // pointer bump; the in-range loads are counted once (a shift)
    {
        constexpr int K = 3 * RP * G / 512;
        constexpr int ROWS_PER = 512 / G;
        const int t = threadIdx.x;
        const int u_t = t / G, c = t & (G - 1);
        const uint64_t n0 = (uint64_t)u_t * C + i0 + c;
        static_assert(RP * G == 8192, "tiles of 3 2^13 words");
        uint32_t* d = sm + padw(u_t * G) + c;
        if constexpr (!FZ) {
            constexpr int lstep = LOGR - 4 + LOGC3;   // log2(ROWS_PER C): ROWS_PER = 2^(LOGR - 4)
            int kin = 0;
            if (n0 < xn) {
                const uint64_t q = ((xn - n0 - 1) >> lstep) + 1;
                kin = q < (uint64_t)K ? (int)q : K;
            }
            const uint64_t* px = x + n0;
#pragma unroll 8
            for (int k = 0; k < K; k++, px += (size_t)ROWS_PER * C)
                d[k * (ROWS_PER * G + ROWS_PER * G / 32)] = k < kin ? limb_redc(*px, p, P.pneg_inv, P.c32) : 0u;
        } else {
            // chunk (n mod S) of coefficient n / S, with the slot, the chunk
            // and the limb offset advanced incrementally (as in k_fwd_cols)
            const uint32_t S = fz.S, xw = opb ? fz.wb : fz.wa;
            const uint32_t step = (uint32_t)ROWS_PER * C;
            uint32_t ci = (uint32_t)n0 / S, ck = (uint32_t)n0 - ci * S;
            const uint32_t sq = step / S, sr = step - sq * S;
            size_t off = (size_t)ci * xw + ck;
            const size_t doff = (size_t)sq * xw + sr;
#pragma unroll 8
            for (int k = 0; k < K; k++) {
                uint32_t r = 0;
                if (ck < xw && ci < xn) {
                    const uint64_t v = x[off];
                    r = limb_redc(v, p, P.pneg_inv, P.c32);
                    // a negative top limb stands for v - 2^64
                    if (ck == xw - 1 && (int64_t)v < 0) r = sub_mod(r, P.c32, p);
                }
                d[k * (ROWS_PER * G + ROWS_PER * G / 32)] = r;
                ci += sq;
                ck += sr;
                off += doff;
                if (ck >= S) {
                    ck -= S;
                    ci++;
                    off -= (size_t)(S - xw);   // S >= xw
                }
            }
        }
    }
    __syncthreads();
    // radix-3 stage: (u1, u1 + R', u1 + 2R') -> t0, t1 omega^u1, t2 omega^(2 u1)
    {
        const uint2 cw = T.w3c[(size_t)j * 2];
        const uint2* __restrict__ tw3 = T.tw3f + (size_t)j * TW3_SZ;
        for (int f = threadIdx.x; f < RP * G; f += blockDim.x) {
            const int u1 = f / G, c = f & (G - 1);
            const int o0 = padw(u1 * G) + c, o1 = padw((u1 + RP) * G) + c, o2 = padw((u1 + 2 * RP) * G) + c;
            const uint32_t x0 = sm[o0], x1 = sm[o1], x2 = sm[o2];
            const uint32_t s = add_mod(x1, x2, p), d = sub_mod(x1, x2, p);
            const uint32_t cd = mul_shoup(d, cw.x, cw.y, p);
            const uint32_t h = sub_mod(add_mod(x0, x0, p), s, p);  // 2 x0 - a
            const int e = u1 << (LOG_R3 - LOGR);
            const uint2 w1 = tw3[e], w2 = tw3[2 * e];
            sm[o0] = add_mod(x0, s, p);
            sm[o1] = mul_shoup(h + cd, w1.x, w1.y, p);             // h + cd < 2p: any 32-bit input
            sm[o2] = mul_shoup(h - cd + p, w2.x, w2.y, p);
        }
    }
    __syncthreads();
    const uint2* __restrict__ twf = T.twf + (size_t)j * TW_SZ;
    gs_strided_all3<LOGR, G>(sm, padw(RP * G), twf, p);
    const uint32_t fsc = (fmask >> (opb ? 1 : 0)) & 1 ? fscale[j] : 0u;
    const uint2* __restrict__ th3 = T.th3 + (size_t)j * TH3_SZ;
    const uint2* __restrict__ tl3 = T.tl3 + (size_t)j * TL_SZ;
    constexpr int NS = RP / 32;
    for (int f = threadIdx.x; f < 3 * G * NS; f += blockDim.x) {
        const int t = f / (G * NS), rem = f - t * (G * NS);
        const int v = rem & (G - 1), s = rem / G;
        const int pb = padw(t * RP * G) + 33 * G * s + v;
        uint32_t xr[32];
#pragma unroll
        for (int m = 0; m < 32; m++) xr[m] = sm[pb + padw(m * G)];
        gs_contig<5, COL_FMA_ADDS>(xr, c_w32[j], p);
        const uint32_t col = (uint32_t)(i0 + v);
        twist32_3<LOGR>(xr, col, s, t, k, th3, tl3, P, fsc);
        uint32_t* o = out + ((size_t)(t * RP + 32 * s) << LOGC3) + col;
#pragma unroll
        for (int m = 0; m < 32; m++) o[m * C] = xr[m];
    }
}

// Inverse column pass of a 3 2^k-point transform, in place: untwist, three
// length-2^LOGR inverse transforms, inverse radix-3 stage.
// grid = (C / G, np); block 512; smem as k_fwd_cols3.
template <int LOGR, int G>
__global__ void __launch_bounds__(512)
k_inv_cols3(DevTables T, uint32_t* __restrict__ ra, int logMs, int k)
{
    extern __shared__ uint32_t sm[];
    constexpr int RP = 1 << LOGR;
    constexpr int C = 1 << LOGC3;
    const int j = blockIdx.y;
    const int i0 = blockIdx.x * G;
    uint32_t* __restrict__ buf = ra + ((size_t)j << logMs);
    const PrimeInfo P = T.pi[j];
    const uint32_t p = P.p;
    const uint2* __restrict__ th3 = T.th3i + (size_t)j * TH3_SZ;
    const uint2* __restrict__ tl3 = T.tl3i + (size_t)j * TL_SZ;
    constexpr int NS = RP / 32;
    for (int f = threadIdx.x; f < 3 * G * NS; f += blockDim.x) {
        const int t = f / (G * NS), rem = f - t * (G * NS);
        const int v = rem & (G - 1), s = rem / G;
        const uint32_t col = (uint32_t)(i0 + v);
        const uint32_t* src = buf + ((size_t)(t * RP + 32 * s) << LOGC3) + col;
        uint32_t xr[32];
#pragma unroll
        for (int m = 0; m < 32; m++) xr[m] = src[m * C];
        twist32_3<LOGR>(xr, col, s, t, k, th3, tl3, P, 0u);
        ct_contig<5, COL_CT_FMA_ADDS>(xr, c_w32[j], p);
        const int pb = padw(t * RP * G) + 33 * G * s + v;
#pragma unroll
        for (int m = 0; m < 32; m++) sm[pb + padw(m * G)] = xr[m];
    }
    __syncthreads();
    const uint2* __restrict__ twi = T.twi + (size_t)j * TW_SZ;
    ct_strided_all3<LOGR, G>(sm, padw(RP * G), twi, p);
    __syncthreads();
    const uint2 cw = T.w3c[(size_t)j * 2 + 1];
    const uint2* __restrict__ tw3 = T.tw3i + (size_t)j * TW3_SZ;
    for (int f = threadIdx.x; f < RP * G; f += blockDim.x) {
        const int u1 = f / G, c = f & (G - 1);
        const uint32_t z0 = sm[padw(u1 * G) + c], z1 = sm[padw((u1 + RP) * G) + c];
        const uint32_t z2 = sm[padw((u1 + 2 * RP) * G) + c];
        const int e = u1 << (LOG_R3 - LOGR);
        const uint2 w1 = tw3[e], w2 = tw3[2 * e];
        const uint32_t t1h = mul_shoup(z1, w1.x, w1.y, p), t2h = mul_shoup(z2, w2.x, w2.y, p);
        const uint32_t h = add_mod(t1h, t2h, p), g = sub_mod(t1h, t2h, p);
        const uint32_t cg = mul_shoup(g, cw.x, cw.y, p);
        const uint32_t m0 = sub_mod(z0, h, p);
        uint32_t* o = buf + (size_t)u1 * C + i0 + c;
        o[0] = add_mod(add_mod(z0, h, p), h, p);
        o[(size_t)RP * C] = add_mod(m0, cg, p);
        o[(size_t)2 * RP * C] = sub_mod(m0, cg, p);
    }
}

}  // namespace fb
