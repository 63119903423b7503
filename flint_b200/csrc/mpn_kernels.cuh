// Kernels of the integer multiplication path z = a * b (mpn limbs, 64-bit).
//
// Coefficients are single limbs (64-bit chunks); the cyclic convolution of
// length M = 2^m = R * C is computed modulo np word-size primes with a
// four-step transform (C = 2^14 once M > 2^14, R = M / C <= 2^11):
//
//   k_fwd_cols   limbs -> residues (split fused into the load), length-R
//                forward transforms down G columns at a time, four-step twist
//                w_M^(i*k1) applied in registers, write.  [one pass over HBM]
//   k_rows       per row: forward transform of b (kept in registers), forward
//                transform of a, pointwise product with the CRT/normalisation
//                scale, inverse transform.               [one pass over HBM]
//   k_inv_cols   untwist in registers, length-R inverse transforms down the
//                columns.                                 [one pass over HBM]
//   k_crt_carry  np residues -> exact coefficient (CRT), coefficients ->
//                limbs with the carry chain resolved by a decoupled
//                look-back scan across tiles.             [one pass over HBM]
//
// Reference counterparts: limb splitting mpn_to_ffts_* (src/fft_small/
// mpn_mul.c:422-696), the per-prime transform/pointwise/inverse worker
// (mpn_mul.c:1505-1527), and CRT + carry recomposition _mpn_from_ffts_NP
// with the serial overhang stitch (mpn_mul.c:802-993, 1934-1973).
#pragma once
#include "ntt_smem.cuh"

namespace fb {

constexpr int LOG_MAXM = 25;              // largest cyclic length 2^25
constexpr int LOG_MAXC = 14;              // longest row transform
constexpr int TW_SZ = 1 << LOG_MAXC;      // local twiddle table entries per prime
constexpr int TH_SZ = 1 << (LOG_MAXM - 13);   // twist table: w^(t 2^13), t < 2^12
constexpr int TL_SZ = 1 << 13;            // twist table: w^t, t < 2^13

// Transforms of 3 2^k points (the first NP3 primes have roots of order
// 3 2^25): twist powers of w3 (order 3 2^25) and radix-3 stage twiddles
constexpr int NP3 = 5;
constexpr int TH3_SZ = 3 << (LOG_MAXM - 13);   // w3^(t 2^13), t < 3 2^12
constexpr int LOG_R3 = 11;                      // radix-3 stage tables serve columns up to 3 2^11
constexpr int TW3_SZ = 2 << LOG_R3;             // (omega^e / 2), e < 2^12, omega of order 3 2^11

struct DevTables {
    const PrimeInfo* pi;   // [MAX_NP]
    const uint2* twf;      // [MAX_NP][TW_SZ] forward local twiddles
    const uint2* twi;      // [MAX_NP][TW_SZ] inverse local twiddles
    const uint2* th;       // [MAX_NP][TH_SZ] w_{2^25}^(t 2^13)
    const uint2* tl;       // [MAX_NP][TL_SZ] w_{2^25}^t
    const uint2* thi;      // inverses of the above
    const uint2* tli;
    const uint2* th3;      // [NP3][TH3_SZ] w3^(t 2^13)
    const uint2* tl3;      // [NP3][TL_SZ] w3^t
    const uint2* th3i;     // inverses of the above
    const uint2* tl3i;
    const uint2* tw3f;     // [NP3][TW3_SZ] omega^e / 2, omega = w3^(2^14) of order 3 2^11
    const uint2* tw3i;     // [NP3][TW3_SZ] omega^-e / 2
    const uint2* w3c;      // [NP3][2] (w - w^2, w^-1 - w^-2), w = w3^(2^25) of order 3
};

// w_M^e * x for e in units of the largest transform (e < 2^25)
__device__ __forceinline__ uint32_t twist_mul(uint32_t x, uint32_t e, const uint2* __restrict__ th,
                                              const uint2* __restrict__ tl, uint32_t p)
{
    const uint2 w1 = th[e >> 13];
    const uint2 w2 = tl[e & 8191];
    x = mul_shoup(x, w1.x, w1.y, p);
    return mul_shoup(x, w2.x, w2.y, p);
}

__device__ __forceinline__ uint32_t bitrev_bits(uint32_t u, int bits)
{
    return bits == 0 ? 0u : (__brev(u) >> (32 - bits));
}

struct MulShape {
    int logR, logC;        // M = 2^(logR + logC)
    int G;                 // columns per column-pass tile
};

// columns per tile for a column length 2^logR: 64 KB tiles, at least 8
// columns (32-byte row segments)
__host__ __device__ constexpr int cols_per_tile(int logR)
{
    return logR >= 11 ? 8 : (1 << (14 - logR));
}

// w^e for e in units of the largest transform, from the two-level tables
__device__ __forceinline__ uint32_t table_power(uint32_t e, const uint2* __restrict__ th,
                                                const uint2* __restrict__ tl, uint32_t p)
{
    const uint2 w1 = th[e >> 13];
    const uint2 w2 = tl[e & 8191];
    return mul_shoup(w1.x, w2.x, w2.y, p);
}

// Shoup companion floor(w 2^32 / p) on the device: a double-precision
// estimate (error well below 1) corrected by one exact remainder test.
__device__ __forceinline__ uint32_t shoup_companion_dev(uint32_t w, uint32_t p)
{
    const double est = (double)w * (4294967296.0 / (double)p);
    uint32_t q = (uint32_t)est;
    const int64_t r = (int64_t)((uint64_t)w << 32) - (int64_t)((uint64_t)q * p);
    if (r >= (int64_t)p) q++;
    else if (r < 0) q--;
    return q;
}

// Four-step twist of the 32 consecutive column positions u = 32 s + m held by
// one thread: position u gets w_M^(col * bitrev_r(u)).  Since
// bitrev_r(32 s + m) = bitrev_(r-5)(s) + 2^(r-5) bitrev_5(m), the factors are
// alpha * beta^k, k = bitrev_5(m), with alpha = w^(col bitrev_(r-5)(s)) and
// beta = w^(col 2^(r-5)).  They are generated by a Shoup chain in Montgomery
// form (F_(k+1) = F_k beta) and applied with one Montgomery product each,
// so no table is read per element.
// fsc != 0 multiplies every factor by fsc (a pointwise scale folded into
// this operand's transform; one extra product per thread).
template <int LOGR>
__device__ __forceinline__ void twist32(uint32_t (&x)[32], uint32_t col, int s, int logM,
                                        const uint2* __restrict__ th, const uint2* __restrict__ tl,
                                        const PrimeInfo& P, uint32_t fsc = 0)
{
    const uint32_t p = P.p;
    const uint32_t mmask = (1u << logM) - 1;
    const int sh = LOG_MAXM - logM;
    const uint32_t e0 = ((col * bitrev_bits((uint32_t)s, LOGR - 5)) & mmask) << sh;
    const uint32_t e1 = ((col << (LOGR - 5)) & mmask) << sh;
    const uint32_t alpha = table_power(e0, th, tl, p);
    const uint32_t beta = table_power(e1, th, tl, p);
    const uint32_t bq = shoup_companion_dev(beta, p);
    uint32_t F = mul_mont(alpha, P.r2, p, P.pneg_inv);   // alpha in Montgomery form
    if (fsc) F = mul_mont(F, fsc, p, P.pneg_inv);         // alpha fsc, Montgomery form
#pragma unroll
    for (int k = 0; k < 32; k++) {
        const int m = (int)(__brev((unsigned)k) >> 27);
        x[m] = mul_mont(x[m], F, p, P.pneg_inv);
        if (k < 31) F = mul_shoup(F, beta, bq, p);
    }
}

// One product of a batch: operands, result, its residue scratch (a's np
// transforms at ra, b's at ra + np M) and its first CRT tile within the launch.
struct InstDesc {
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* z;
    uint32_t* ra;
    uint64_t an, bn;
    uint32_t tile0, ntiles;
};

// Integer-polynomial operands: coefficient i of an operand is w 64-bit limbs
// in two's complement (the top limb signed), chunk k of it is placed at
// position i S + k of a polynomial in y (S = wa + wb - 1, so the chunk
// products of different output coefficients never share a position).
struct FzShape {
    uint32_t S;       // slot stride in y
    uint32_t wa, wb;  // limbs per coefficient of a and of b
};

// Residue (times 2^-32) of chunk k of coefficient i of an xn-coefficient
// polynomial with w limbs per coefficient (zero beyond the coefficient's
// limbs or the polynomial).
__device__ __forceinline__ uint32_t load_chunk(const uint64_t* __restrict__ x, uint32_t i, uint32_t k,
                                               uint64_t xn, uint32_t w, const PrimeInfo& P)
{
    if (k >= w || i >= xn) return 0u;
    const uint64_t v = x[(size_t)i * w + k];
    uint32_t r = limb_redc(v, P.p, P.pneg_inv, P.c32);
    // a negative top limb stands for v - 2^64, and 2^64 2^-32 = 2^32
    if (k == w - 1 && (int64_t)v < 0) r = sub_mod(r, P.c32, P.p);
    return r;
}

// Residue (times 2^-32) of operand element n.  Limb source: limb n of an
// xn-limb integer.  Coefficient source: chunk (n mod S) of coefficient n / S
// of an xn-coefficient polynomial with w limbs per coefficient.
template <bool FZ>
__device__ __forceinline__ uint32_t load_residue(const uint64_t* __restrict__ x, uint64_t n, uint64_t xn,
                                                 uint32_t S, uint32_t w, const PrimeInfo& P)
{
    if constexpr (!FZ) {
        return n < xn ? limb_redc(x[n], P.p, P.pneg_inv, P.c32) : 0u;
    } else {
        const uint32_t nn = (uint32_t)n;      // y-lengths stay below 2^32
        const uint32_t i = nn / S, k = nn - i * S;
        return load_chunk(x, i, k, xn, w, P);
    }
}

// ---------------------------------------------------------------------------
// Column pass, forward: split + length-R transforms + twist.
// grid = (np, C / G, operands) -- the prime index varies fastest so that the
// np tiles that read the same limbs run together and share them through L2;
// with a batch descriptor, grid.z = 2 * instance + operand.  FZ selects the
// integer-polynomial source (an, bn count coefficients, shape in fz).
// smem = padw(R * G) words.
// LC != 0: the row length 2^LC is a compile-time constant (logC == LC), so
// the strided stores take immediate offsets instead of address arithmetic.
template <int LOGR, int G, bool FZ, int LC>
__device__ __forceinline__ void
fwd_cols_body(DevTables T, const uint64_t* __restrict__ a, uint64_t an,
              const uint64_t* __restrict__ b, uint64_t bn,
              uint32_t* __restrict__ ra, uint32_t* __restrict__ rb, int logC, int gcols,
              const InstDesc* __restrict__ desc, int np, FzShape fz, const uint32_t* __restrict__ fscale,
              int fmask)
{
    extern __shared__ uint32_t sm[];
    constexpr int R = 1 << LOGR;
    if constexpr (LC != 0) logC = LC;
    const int C = 1 << logC;
    const int logM = LOGR + logC;
    const int GR = G ? G : gcols;          // runtime tile width for short columns
    const int j = blockIdx.x;
    const int i0 = blockIdx.y * GR;
    const bool opb = (blockIdx.z & 1) != 0;
    if (desc) {
        const InstDesc& D = desc[blockIdx.z >> 1];
        a = D.a; b = D.b; an = D.an; bn = D.bn;
        ra = D.ra;
        rb = D.ra + ((size_t)np << logM);
    }
    const uint64_t* __restrict__ x = opb ? b : a;
    const uint64_t xn = opb ? bn : an;
    const uint32_t xw = opb ? fz.wb : fz.wa;
    uint32_t* __restrict__ out = (opb ? rb : ra) + ((size_t)j << logM);
    const PrimeInfo P = T.pi[j];
    const uint32_t p = P.p;
    const uint64_t M = (uint64_t)1 << logM;
    const int tot = R * GR;
    // threads of a tile with columns of 2^5 points or more: one per 32-point
    // column segment (512 for the 2^14-word tiles, fewer for narrow ones)
    constexpr int NT = G ? (G * R / 32 < 512 ? G * R / 32 : 512) : 512;
    constexpr int PNT = NT + NT / 32;     // padw(NT)

    if (LOGR >= 5 && (FZ || xn <= M)) {
        // blockDim == G R / 32 == NT: thread t loads elements t + NT k, i.e.
        // rows u_t + k NT/G of its fixed column; shared offsets are constants
        const int t = threadIdx.x;
        const int GG = G ? G : 1;
        const int u_t = t / GG, c = t & (GG - 1);
        const uint64_t step = (uint64_t)(NT / GG) * C;
        uint64_t n = (uint64_t)u_t * C + i0 + c;
        uint32_t* d = sm + padw(u_t * GG) + c;
        if constexpr (!FZ && LOGR >= 5) {
            // step is a power of two: the number of loads inside the operand
            // is a shift, and a pointer bump per row keeps the 64-bit address
            // arithmetic off the FMA pipe (measured 1.267 -> 1.249 ms for the
            // two operands of a 2^24 x 2^24 product)
            constexpr int K = R * GG / NT;
            const int lstep = (31 - __clz(NT / GG)) + logC;
            int kin = 0;
            if (n < xn) {
                const uint64_t q = ((xn - n - 1) >> lstep) + 1;
                kin = q < (uint64_t)K ? (int)q : K;
            }
            const uint64_t* px = x + n;
#pragma unroll 8
            for (int k = 0; k < K; k++, px += step)
                d[k * PNT] = k < kin ? limb_redc(*px, p, P.pneg_inv, P.c32) : 0u;
        } else if constexpr (FZ) {
            // integer-polynomial source: n advances by `step`, so its slot
            // n / S and chunk n mod S advance by fixed amounts (one division
            // per thread instead of one per element)
            const uint32_t S = fz.S;
            uint32_t ci = (uint32_t)n / S, ck = (uint32_t)n - ci * S;
            const uint32_t sq = (uint32_t)step / S, sr = (uint32_t)step - sq * S;
            // the limb offset ci w + ck advances the same way
            size_t off = (size_t)ci * xw + ck;
            const size_t doff = (size_t)sq * xw + sr;
#pragma unroll 8
            for (int k = 0; k < R * GG / NT; k++) {
                uint32_t r = 0;
                if (ck < xw && ci < xn) {
                    const uint64_t v = x[off];
                    r = limb_redc(v, p, P.pneg_inv, P.c32);
                    // a negative top limb stands for v - 2^64
                    if (ck == xw - 1 && (int64_t)v < 0) r = sub_mod(r, P.c32, p);
                }
                d[k * PNT] = r;
                ci += sq;
                ck += sr;
                off += doff;
                if (ck >= S) {
                    ck -= S;
                    ci++;
                    off -= (size_t)(S - xw);   // S >= xw: one slot on, minus the chunks it carries
                }
            }
        } else {
#pragma unroll 8
            for (int k = 0; k < R * GG / NT; k++, n += step)
                d[k * PNT] = load_residue<FZ>(x, n, xn, fz.S, xw, P);
        }
    } else if (FZ || xn <= M) {
        // four loads in flight per thread (small transforms are bound by
        // their latency)
        for (int f0 = threadIdx.x; f0 < tot; f0 += 4 * blockDim.x) {
            uint32_t v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int f = f0 + q * (int)blockDim.x;
                const int u = f / GR, c = f - u * GR;
                v[q] = f < tot ? load_residue<FZ>(x, (uint64_t)u * C + i0 + c, xn, fz.S, xw, P) : 0u;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int f = f0 + q * (int)blockDim.x;
                const int u = f / GR, c = f - u * GR;
                if (f < tot) sm[padw(u * GR) + c] = v[q];
            }
        }
    } else {
        // cyclic fold: an operand longer than M wraps around (x mod X^M - 1)
        for (int f = threadIdx.x; f < tot; f += blockDim.x) {
            const int u = f / GR, c = f - u * GR;
            uint32_t r = 0;
            for (uint64_t n = (uint64_t)u * C + i0 + c; n < xn; n += M)
                r = add_mod(r, limb_redc(x[n], p, P.pneg_inv, P.c32), p);
            sm[padw(u * GR) + c] = r;
        }
    }
    __syncthreads();
    const uint2* __restrict__ th = T.th + (size_t)j * TH_SZ;
    const uint2* __restrict__ tl = T.tl + (size_t)j * TL_SZ;
    const int sh = LOG_MAXM - logM;
    const uint32_t mmask = (uint32_t)(M - 1);
    if constexpr (LOGR >= 5) {
        // pointwise scale folded into this operand's twist (fmask bit 0: the
        // first operand, bit 1: the second)
        const uint32_t fsc = (fmask >> (opb ? 1 : 0)) & 1 ? fscale[j] : 0u;
        gs_strided_all<LOGR, G>(sm, 1, T.twf + (size_t)j * TW_SZ, p);
        constexpr int NS = R / 32;
        for (int f = threadIdx.x; f < G * NS; f += blockDim.x) {
            const int v = f & (G - 1), s = f / G;
            const int pb = 33 * G * s + v;
            uint32_t xr[32];
#pragma unroll
            for (int m = 0; m < 32; m++) xr[m] = sm[pb + padw(m * G)];
            gs_contig<5, COL_FMA_ADDS>(xr, c_w32[j], p);
            const uint32_t col = (uint32_t)(i0 + v);
            twist32<LOGR>(xr, col, s, logM, th, tl, P, fsc);
            // rows 32 s .. 32 s + 31 of column col: a pointer bump per row keeps
            // the address arithmetic on the ALU pipe (the FMA pipe is this
            // kernel's busiest unit)
            uint32_t* o = out + ((size_t)(32 * s) << logC) + col;
            if constexpr (LC != 0) {
#pragma unroll
                for (int m = 0; m < 32; m++) o[m * (1 << LC)] = xr[m];
            } else {
#pragma unroll
                for (int m = 0; m < 32; m++, o += C) *o = xr[m];
            }
        }
    } else {
        // short columns: one thread owns a whole column
        for (int v = threadIdx.x; v < GR; v += blockDim.x) {
            uint32_t xr[R];
#pragma unroll
            for (int m = 0; m < R; m++) xr[m] = sm[padw(m * GR) + v];
            if constexpr (LOGR > 0) gs_contig<LOGR, COL_FMA_ADDS>(xr, c_w32[j], p);
            const uint32_t col = (uint32_t)(i0 + v);
#pragma unroll
            for (int m = 0; m < R; m++) {
                uint32_t val = xr[m];
                if constexpr (LOGR > 0) {
                    const uint32_t e = ((col * bitrev_bits(m, LOGR)) & mmask) << sh;
                    val = twist_mul(val, e, th, tl, p);
                }
                out[(size_t)m * C + col] = val;
            }
        }
    }
}

// Kernel instances: LC = 0 takes the row length at run time; LC = 14 serves
// 2^14-point rows under 2^11-point columns (2^25 points) and LC = 13 2^13-point
// rows under 2^9- to 2^11-point columns, with constant strides (measured on
// the 2^25-point forward pass: 1.28 -> 1.13 ms).  An LC instance also holds
// the run-time body behind a branch that never takes it for its shape: with
// that second body the compiler schedules the constant-stride one better
// (1.21 ms alone, 1.13 ms with it; three bodies in one kernel: 1.24 ms).
template <int LOGR, int G, bool FZ, int LC = 0>
__global__ void __launch_bounds__(512)
k_fwd_cols(DevTables T, const uint64_t* __restrict__ a, uint64_t an,
           const uint64_t* __restrict__ b, uint64_t bn,
           uint32_t* __restrict__ ra, uint32_t* __restrict__ rb, int logC, int gcols,
           const InstDesc* __restrict__ desc, int np, FzShape fz, const uint32_t* __restrict__ fscale,
           int fmask)
{
    if (LC != 0 && logC == LC)
        fwd_cols_body<LOGR, G, FZ, LC>(T, a, an, b, bn, ra, rb, logC, gcols, desc, np, fz, fscale, fmask);
    else
        fwd_cols_body<LOGR, G, FZ, 0>(T, a, an, b, bn, ra, rb, logC, gcols, desc, np, fz, fscale, fmask);
}

// ---------------------------------------------------------------------------
// Row pass, persistent: each CTA walks over items of nv rows (one prime per
// item).  For every item: forward transforms of a and b as one interleaved
// network (shared twiddle loads, twice the independent work per thread; b's
// spectrum ends in registers), pointwise product times scale[j], inverse
// transform; the result overwrites the a rows.  Three shared buffers: b, and
// a ping-pong pair for a, so the next item's a rows stream in (cp.async)
// during the whole current item and its b rows as soon as b's spectrum is in
// registers.  grid = min(items, resident CTAs); block = nv * C / 32;
// smem = 3 * nv * padw(C) words.  `squaring`: 0 a b, 1 a a (b unused), 2 a
// times a b whose rows already hold its spectrum in this kernel's order
// (k_rows_fwd output; the chunks of a split product share one).
__device__ __forceinline__ void cp_async4(uint32_t* dst, const uint32_t* src, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? 4 : 0;   // a zero source size fills the word with zeros
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void cp_async4_full(uint32_t* dst, const uint32_t* src)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src));
}

// 16 bytes, both addresses 16-byte aligned; bypasses L1 (.cg)
__device__ __forceinline__ void cp_async16(uint32_t* dst, const uint32_t* src)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src));
}

// LOGE: log2 of the elements each thread owns in the row kernel's
// contiguous pass (blockDim = nv C / 2^LOGE).  UNP: a single row (nv = 1,
// rows of at least 2^10 words) lands unpadded, as 16-byte copies that bypass
// L1 -- 4x fewer copy instructions than the padded layout's 4-byte ones and
// no L1 allocation; the first forward pass pads it (gs_pass_first_unpadded).
// The row base and dst must be 16-byte aligned (residue planes and rows are
// multiples of 2^10 words; dst is a row buffer at a multiple of padw(C)).
template <int LOGC, int LOGE = 5>
__device__ __forceinline__ constexpr bool rows_unpadded(int nv)
{
    return LOGE == 5 && LOGC >= 10 && nv == 1;
}

template <int LOGC, int LOGE = 5, bool UNP = false>
__device__ __forceinline__ void rows_prefetch(uint32_t* dst, const uint32_t* __restrict__ base,
                                              int u0, int nv, int R)
{
    constexpr int C = 1 << LOGC;
    constexpr int PC = padw(C);
    constexpr int NSUB = C >> LOGE;
    if (UNP && rows_unpadded<LOGC, LOGE>(nv)) {
        // blockDim == NSUB == C / 32: 16-byte chunk c = t + k NSUB, k < 8
        const uint32_t* src = base + (size_t)u0 * C;
#pragma unroll
        for (int k = 0; k < (1 << LOGE) / 4; k++) {
            const int c = threadIdx.x + k * NSUB;
            cp_async16(dst + 4 * c, src + 4 * c);
        }
    } else if (nv == 1 && NSUB % 32 == 0) {
        // one row, blockDim == NSUB: element t + k NSUB, compile-time offsets
        const int t = threadIdx.x;
        const uint32_t* src = base + (size_t)u0 * C + t;
        uint32_t* d = dst + padw(t);
#pragma unroll
        for (int k = 0; k < (1 << LOGE); k++) cp_async4_full(d + k * (NSUB / 32 * 33), src + k * NSUB);
    } else {
        for (int f = threadIdx.x; f < nv * C; f += blockDim.x) {
            const int v = f >> LOGC, i = f & (C - 1);
            const int u = u0 + v;
            cp_async4(&dst[v * PC + padw(i)], base + (size_t)min(u, R - 1) * C + i, u < R);
        }
    }
    cp_async_commit();
}

template <int LOGC, int LOGE = 5>
__global__ void __launch_bounds__(LOGE == 4 ? 1024 : 512, 1)
k_rows(DevTables T, uint32_t* __restrict__ ra, const uint32_t* __restrict__ rb,
       int logR, int nv, int np, const uint32_t* __restrict__ scale, int squaring,
       const InstDesc* __restrict__ desc, int ninst, int rows)
{
    extern __shared__ __align__(16) uint32_t sm[];   // 16-byte copies land in the row buffers
    constexpr int C = 1 << LOGC;
    constexpr int PC = padw(C);
    constexpr int E = 1 << LOGE;          // elements per thread in the contiguous pass
    constexpr int NSUB = C / E;
    constexpr int QMAX = LOGE;            // strided passes: at least one sub-transform per thread
    const int R = rows;                    // rows per prime (<= 2^logR, the prime stride's rows)
    const int logM = logR + LOGC;
    const int groups = (R + nv - 1) / nv;
    const int per = groups * np;           // items of one product
    const int total = per * ninst;
    uint32_t* sb = sm;
    // a ping-pong pair at sm + nv PC and sm + 2 nv PC (pointer arithmetic, not
    // an indexed array, so nothing goes to local memory)
    auto sa_buf = [&](int c) { return sm + (1 + c) * nv * PC; };
    const int t = threadIdx.x;
    const int pb = (t / NSUB) * PC + padw(E * (t & (NSUB - 1)));
    // item -> (prime, first row, residue base of a, of b)
    auto decode = [&](int gg, int& jj, int& uu, uint32_t*& A, const uint32_t*& B) {
        const int inst = gg / per;
        const int r = gg - inst * per;
        jj = r / groups;
        uu = (r - jj * groups) * nv;
        if (desc) { A = desc[inst].ra; B = A + ((size_t)np << logM); }
        else { A = ra; B = rb; }
    };

    int g = blockIdx.x;
    if (g >= total) return;
    {
        int j, u0;
        uint32_t* A;
        const uint32_t* B;
        decode(g, j, u0, A, B);
        rows_prefetch<LOGC, LOGE, true>(sa_buf(0), A + ((size_t)j << logM), u0, nv, R);
        if (squaring == 0) rows_prefetch<LOGC, LOGE, true>(sb, B + ((size_t)j << logM), u0, nv, R);
        else if (squaring == 2) rows_prefetch<LOGC, LOGE, false>(sb, B + ((size_t)j << logM), u0, nv, R);
        else cp_async_commit();
    }
    int cur = 0;
    for (; g < total; g += gridDim.x) {
        int j, u0, j2 = 0, u2 = 0;
        uint32_t *A, *A2 = nullptr;
        const uint32_t *B, *B2 = nullptr;
        decode(g, j, u0, A, B);
        const int g2 = g + gridDim.x;
        if (g2 < total) decode(g2, j2, u2, A2, B2);
        const PrimeInfo P = T.pi[j];
        const uint32_t p = P.p;
        const uint2* __restrict__ twf = T.twf + (size_t)j * TW_SZ;
        const uint2* __restrict__ twi = T.twi + (size_t)j * TW_SZ;
        uint32_t* sa = sa_buf(cur);

        // this item's a and b rows have landed; the other a buffer is free
        // (its last item stored from it before the barrier)
        cp_async_wait<0>();
        __syncthreads();
        if (g2 < total) rows_prefetch<LOGC, LOGE, true>(sa_buf(cur ^ 1), A2 + ((size_t)j2 << logM), u2, nv, R);
        else cp_async_commit();

        uint32_t xr[E];
        uint32_t breg[E];
        if (squaring == 0) {
            if constexpr (LOGE == 5) {
                if (rows_unpadded<LOGC, LOGE>(nv)) gs_strided_all2<LOGC, QMAX, LOGE, true>(sa, sb, nv, twf, p);
                else gs_strided_all2<LOGC, QMAX, LOGE>(sa, sb, nv, twf, p);
            } else {
                gs_strided_all2<LOGC, QMAX, LOGE>(sa, sb, nv, twf, p);
            }
#pragma unroll
            for (int m = 0; m < E; m++) {
                xr[m] = sa[pb + m];
                breg[m] = sb[pb + m];
            }
            gs_contig2<LOGE, ROW_GS_FMA_ADDS>(xr, breg, c_w32[j], p);
            __syncthreads();   // b fully read: refill it for the next item
            if (g2 < total) rows_prefetch<LOGC, LOGE, true>(sb, B2 + ((size_t)j2 << logM), u2, nv, R);
            else cp_async_commit();
        } else {
            // a squaring, or b's rows already hold its spectrum in this
            // kernel's order (squaring == 2: k_rows_fwd output, landed padded)
            if constexpr (LOGE == 5) {
                if (rows_unpadded<LOGC, LOGE>(nv)) gs_strided_all<LOGC, 0, QMAX, LOGE, true>(sa, nv, twf, p);
                else gs_strided_all<LOGC, 0, QMAX, LOGE>(sa, nv, twf, p);
            } else {
                gs_strided_all<LOGC, 0, QMAX, LOGE>(sa, nv, twf, p);
            }
#pragma unroll
            for (int m = 0; m < E; m++) xr[m] = sa[pb + m];
            gs_contig<LOGE, ROW_GS_FMA_ADDS>(xr, c_w32[j], p);
            if (squaring == 2) {
#pragma unroll
                for (int m = 0; m < E; m++) breg[m] = sb[pb + m];
                __syncthreads();   // b fully read: refill it for the next item
                if (g2 < total) rows_prefetch<LOGC, LOGE, false>(sb, B2 + ((size_t)j2 << logM), u2, nv, R);
                else cp_async_commit();
            } else {
                cp_async_commit();
            }
        }
        if (scale) {
            const uint32_t sc = scale[j];
#pragma unroll
            for (int m = 0; m < E; m++) {
                const uint32_t y = squaring == 1 ? xr[m] : breg[m];
                xr[m] = mul_mont(mul_mont(xr[m], y, p, P.pneg_inv), sc, p, P.pneg_inv);
            }
        } else {
            // the scale was folded into b's forward transform (k_fwd_cols)
#pragma unroll
            for (int m = 0; m < E; m++) xr[m] = mul_mont(xr[m], breg[m], p, P.pneg_inv);
        }
        ct_contig<LOGE, ROW_CT_FMA_ADDS>(xr, c_w32[j], p);
#pragma unroll
        for (int m = 0; m < E; m++) sa[pb + m] = xr[m];
        __syncthreads();
        uint32_t* __restrict__ abase = A + ((size_t)j << logM);
        if constexpr (LOGC > LOGE) {
            if (nv == 1) {
                // one row: the last inverse pass writes it to HBM directly
                ct_strided_all_out<LOGC, QMAX, LOGE>(sa, twi, p, abase + (size_t)u0 * C);
                cur ^= 1;
                continue;
            }
        }
        ct_strided_all<LOGC, 0, QMAX, LOGE>(sa, nv, twi, p);
        if (nv == 1 && NSUB % 32 == 0) {
            uint32_t* dst = abase + (size_t)u0 * C + t;
            const uint32_t* s_ = sa + padw(t);
#pragma unroll
            for (int k = 0; k < E; k++) dst[k * NSUB] = s_[k * (NSUB / 32 * 33)];
        } else {
            for (int f = t; f < nv * C; f += blockDim.x) {
                const int v = f >> LOGC, i = f & (C - 1);
                const int u = u0 + v;
                if (u < R) abase[(size_t)u * C + i] = sa[v * PC + padw(i)];
            }
        }
        cur ^= 1;
    }
    cp_async_wait<0>();
}

// Destination of one chunk of a split product (a long operand cut into
// chunks, each multiplied by the short one): the inverse column pass writes
// the chunk's residues into acc (prime stride 2^logMf) at offset shift
// instead of back in place, adds them mod p below `overlap` (where the
// previous chunk's product ends), and skips positions at or beyond nvalid
// (past the chunk's product).  acc == nullptr: in place.
struct ChunkOut {
    uint32_t* acc;
    int logMf;
    uint64_t shift, overlap, nvalid;
};

// ---------------------------------------------------------------------------
// Column pass, inverse: untwist in registers + length-R inverse transforms,
// in place (or into a split product's residues, ChunkOut).  grid = (C / G, np, instances); smem = padw(R * G) words.
template <int LOGR, int G, int LC>
__device__ __forceinline__ void
inv_cols_body(DevTables T, uint32_t* __restrict__ ra, int logC, int gcols,
              const InstDesc* __restrict__ desc, ChunkOut co)
{
    extern __shared__ uint32_t sm[];
    constexpr int R = 1 << LOGR;
    if constexpr (LC != 0) logC = LC;
    const int C = 1 << logC;
    const int logM = LOGR + logC;
    const int GR = G ? G : gcols;
    const int j = blockIdx.y;
    const int i0 = blockIdx.x * GR;
    if (desc) ra = desc[blockIdx.z].ra;
    uint32_t* __restrict__ buf = ra + ((size_t)j << logM);
    const PrimeInfo P = T.pi[j];
    const uint32_t p = P.p;
    const uint2* __restrict__ th = T.thi + (size_t)j * TH_SZ;
    const uint2* __restrict__ tl = T.tli + (size_t)j * TL_SZ;
    const int sh = LOG_MAXM - logM;
    const uint32_t mmask = (uint32_t)(((uint64_t)1 << logM) - 1);

    if constexpr (LOGR >= 5) {
        constexpr int NS = R / 32;
        for (int f = threadIdx.x; f < G * NS; f += blockDim.x) {
            const int v = f & (G - 1), s = f / G;
            const uint32_t col = (uint32_t)(i0 + v);
            uint32_t xr[32];
            const uint32_t* src = buf + ((size_t)(32 * s) << logC) + col;
#pragma unroll
            for (int m = 0; m < 32; m++) xr[m] = src[(size_t)m * C];
            twist32<LOGR>(xr, col, s, logM, th, tl, P);
            ct_contig<5, COL_CT_FMA_ADDS>(xr, c_w32[j], p);
            const int pb = 33 * G * s + v;
#pragma unroll
            for (int m = 0; m < 32; m++) sm[pb + padw(m * G)] = xr[m];
        }
        __syncthreads();
        ct_strided_all<LOGR, G>(sm, 1, T.twi + (size_t)j * TW_SZ, p);
        // blockDim == G R / 32 == NT: thread t stores rows u_t + k NT/G of
        // its column (the inverse of the forward pass's load mapping)
        constexpr int NT = G * R / 32 < 512 ? G * R / 32 : 512;
        constexpr int PNT = NT + NT / 32;     // padw(NT)
        const int t = threadIdx.x;
        const int u_t = t / G, c = t & (G - 1);
        const size_t step = (size_t)(NT / G) * C;
        const uint32_t* s_ = sm + padw(u_t * G) + c;
        if (!co.acc) {
            uint32_t* dst = buf + (size_t)u_t * C + i0 + c;
#pragma unroll 8
            for (int k = 0; k < R * G / NT; k++) dst[k * step] = s_[k * PNT];
        } else {
            uint32_t* __restrict__ out = co.acc + ((size_t)j << co.logMf) + co.shift;
            const uint64_t n0 = (uint64_t)u_t * C + i0 + c;
#pragma unroll 8
            for (int k = 0; k < R * G / NT; k++) {
                const uint64_t n = n0 + (uint64_t)k * step;
                if (n < co.nvalid) {
                    const uint32_t v = s_[k * PNT];
                    out[n] = n < co.overlap ? add_mod(out[n], v, p) : v;
                }
            }
        }
    } else if constexpr (LOGR > 0) {
        for (int v = threadIdx.x; v < GR; v += blockDim.x) {
            const uint32_t col = (uint32_t)(i0 + v);
            uint32_t xr[R];
#pragma unroll
            for (int m = 0; m < R; m++) {
                const uint32_t e = ((col * bitrev_bits(m, LOGR)) & mmask) << sh;
                xr[m] = twist_mul(buf[(size_t)m * C + col], e, th, tl, p);
            }
            ct_contig<LOGR, COL_CT_FMA_ADDS>(xr, c_w32[j], p);
#pragma unroll
            for (int m = 0; m < R; m++) buf[(size_t)m * C + col] = xr[m];
        }
    }
}

template <int LOGR, int G, int LC = 0>
__global__ void __launch_bounds__(512)
k_inv_cols(DevTables T, uint32_t* __restrict__ ra, int logC, int gcols,
           const InstDesc* __restrict__ desc, ChunkOut co)
{
    inv_cols_body<LOGR, G, LC>(T, ra, logC, gcols, desc, co);
}

// ---------------------------------------------------------------------------
// CRT + carry.
//
// The inverse transforms leave y_j = (h mod p_j) * (P/p_j)^-1 mod p_j for each
// coefficient h of the product (the factor was folded into the pointwise
// scale).  Then h = sum_j y_j (P/p_j) - k P with k = round(sum_j y_j / p_j):
// the coefficient bound guarantees h < P/2, so the fractional part of
// sum_j y_j / p_j is h / P < 1/2 and the float estimate rounds to k exactly.
struct CrtConst {
    int np;
    uint32_t P[MAX_NP];               // product of the primes, 32-bit words
    uint32_t cof[MAX_NP][MAX_NP];     // P / p_j, 32-bit words
    float finv[MAX_NP];
};

template <int NP>
__device__ __forceinline__ void crt_values(const uint32_t (&y)[NP], const CrtConst& K, uint64_t& c0,
                                           uint64_t& c1, uint64_t& c2);

template <int NP>
__device__ __forceinline__ void crt_coeff(const uint32_t* __restrict__ res, int logM, uint64_t n,
                                          const CrtConst& K, uint64_t& c0, uint64_t& c1, uint64_t& c2)
{
    if constexpr (NP == 0) {
        // direct values: three word planes of L words each (L = 2^logM here)
        const uint64_t* v = reinterpret_cast<const uint64_t*>(res);
        const size_t L = (size_t)1 << logM;
        c0 = v[n]; c1 = v[L + n]; c2 = v[2 * L + n];
    } else {
        uint32_t y[NP];
#pragma unroll
        for (int jp = 0; jp < NP; jp++) y[jp] = res[((size_t)jp << logM) + n];
        crt_values<NP>(y, K, c0, c1, c2);
    }
}

// A[0..5] += y * (c0, c1, c2, c3): one PTX carry chain per partial-product row
__device__ __forceinline__ void mac4(uint32_t (&A)[7], uint32_t y, const uint32_t* c)
{
    asm("mad.lo.cc.u32  %0, %7, %8, %0;\n\t"
        "madc.lo.cc.u32 %1, %7, %9, %1;\n\t"
        "madc.lo.cc.u32 %2, %7, %10, %2;\n\t"
        "madc.lo.cc.u32 %3, %7, %11, %3;\n\t"
        "addc.cc.u32    %4, %4, 0;\n\t"
        "addc.u32       %5, %5, 0;\n\t"
        "mad.hi.cc.u32  %1, %7, %8, %1;\n\t"
        "madc.hi.cc.u32 %2, %7, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %7, %10, %3;\n\t"
        "madc.hi.cc.u32 %4, %7, %11, %4;\n\t"
        "addc.u32       %5, %5, 0;"
        : "+r"(A[0]), "+r"(A[1]), "+r"(A[2]), "+r"(A[3]), "+r"(A[4]), "+r"(A[5]), "+r"(A[6])
        : "r"(y), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]));
}

// A[0..6] += y * (c0 .. c4)
__device__ __forceinline__ void mac5(uint32_t (&A)[7], uint32_t y, const uint32_t* c)
{
    asm("mad.lo.cc.u32  %0, %7, %8, %0;\n\t"
        "madc.lo.cc.u32 %1, %7, %9, %1;\n\t"
        "madc.lo.cc.u32 %2, %7, %10, %2;\n\t"
        "madc.lo.cc.u32 %3, %7, %11, %3;\n\t"
        "madc.lo.cc.u32 %4, %7, %12, %4;\n\t"
        "addc.cc.u32    %5, %5, 0;\n\t"
        "addc.u32       %6, %6, 0;\n\t"
        "mad.hi.cc.u32  %1, %7, %8, %1;\n\t"
        "madc.hi.cc.u32 %2, %7, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %7, %10, %3;\n\t"
        "madc.hi.cc.u32 %4, %7, %11, %4;\n\t"
        "madc.hi.cc.u32 %5, %7, %12, %5;\n\t"
        "addc.u32       %6, %6, 0;"
        : "+r"(A[0]), "+r"(A[1]), "+r"(A[2]), "+r"(A[3]), "+r"(A[4]), "+r"(A[5]), "+r"(A[6])
        : "r"(y), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]));
}

// A[0..5] -= k * (P0 .. P4)   (k < 8; the result is non-negative)
__device__ __forceinline__ void msub5(uint32_t (&A)[7], uint32_t k, const uint32_t* P)
{
    asm("{\n\t.reg .u32 t0, t1, t2, t3, t4, t5;\n\t"
        "mul.lo.u32     t0, %6, %7;\n\t"
        "mul.lo.u32     t1, %6, %8;\n\t"
        "mul.lo.u32     t2, %6, %9;\n\t"
        "mul.lo.u32     t3, %6, %10;\n\t"
        "mul.lo.u32     t4, %6, %11;\n\t"
        "mad.hi.cc.u32  t1, %6, %7, t1;\n\t"
        "madc.hi.cc.u32 t2, %6, %8, t2;\n\t"
        "madc.hi.cc.u32 t3, %6, %9, t3;\n\t"
        "madc.hi.cc.u32 t4, %6, %10, t4;\n\t"
        "madc.hi.u32    t5, %6, %11, 0;\n\t"
        "sub.cc.u32     %0, %0, t0;\n\t"
        "subc.cc.u32    %1, %1, t1;\n\t"
        "subc.cc.u32    %2, %2, t2;\n\t"
        "subc.cc.u32    %3, %3, t3;\n\t"
        "subc.cc.u32    %4, %4, t4;\n\t"
        "subc.u32       %5, %5, t5;\n\t}"
        : "+r"(A[0]), "+r"(A[1]), "+r"(A[2]), "+r"(A[3]), "+r"(A[4]), "+r"(A[5])
        : "r"(k), "r"(P[0]), "r"(P[1]), "r"(P[2]), "r"(P[3]), "r"(P[4]));
}

// A[0..6] -= k * (P0 .. P5)
__device__ __forceinline__ void msub6(uint32_t (&A)[7], uint32_t k, const uint32_t* P)
{
    asm("{\n\t.reg .u32 t0, t1, t2, t3, t4, t5, t6;\n\t"
        "mul.lo.u32     t0, %7, %8;\n\t"
        "mul.lo.u32     t1, %7, %9;\n\t"
        "mul.lo.u32     t2, %7, %10;\n\t"
        "mul.lo.u32     t3, %7, %11;\n\t"
        "mul.lo.u32     t4, %7, %12;\n\t"
        "mul.lo.u32     t5, %7, %13;\n\t"
        "mad.hi.cc.u32  t1, %7, %8, t1;\n\t"
        "madc.hi.cc.u32 t2, %7, %9, t2;\n\t"
        "madc.hi.cc.u32 t3, %7, %10, t3;\n\t"
        "madc.hi.cc.u32 t4, %7, %11, t4;\n\t"
        "madc.hi.cc.u32 t5, %7, %12, t5;\n\t"
        "madc.hi.u32    t6, %7, %13, 0;\n\t"
        "sub.cc.u32     %0, %0, t0;\n\t"
        "subc.cc.u32    %1, %1, t1;\n\t"
        "subc.cc.u32    %2, %2, t2;\n\t"
        "subc.cc.u32    %3, %3, t3;\n\t"
        "subc.cc.u32    %4, %4, t4;\n\t"
        "subc.cc.u32    %5, %5, t5;\n\t"
        "subc.u32       %6, %6, t6;\n\t}"
        : "+r"(A[0]), "+r"(A[1]), "+r"(A[2]), "+r"(A[3]), "+r"(A[4]), "+r"(A[5]), "+r"(A[6])
        : "r"(k), "r"(P[0]), "r"(P[1]), "r"(P[2]), "r"(P[3]), "r"(P[4]), "r"(P[5]));
}

template <int NP>
__device__ __forceinline__ void crt_values(const uint32_t (&y)[NP], const CrtConst& K, uint64_t& c0,
                                           uint64_t& c1, uint64_t& c2)
{
    if constexpr (NP == 5 || NP == 6) {
        // carry-chain form: X = sum_j y_j (P/p_j) - k P in 32-bit words
        float fk = 0.0f;
#pragma unroll
        for (int jp = 0; jp < NP; jp++) fk = fmaf((float)y[jp], K.finv[jp], fk);
        uint32_t A[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int jp = 0; jp < NP; jp++) {
            if constexpr (NP == 5) mac4(A, y[jp], K.cof[jp]);
            else mac5(A, y[jp], K.cof[jp]);
        }
        const uint32_t k = (uint32_t)rintf(fk);
        if constexpr (NP == 5) msub5(A, k, K.P);
        else msub6(A, k, K.P);
        c0 = (uint64_t)A[0] | ((uint64_t)A[1] << 32);
        c1 = (uint64_t)A[2] | ((uint64_t)A[3] << 32);
        c2 = (uint64_t)A[4] | (NP == 6 ? ((uint64_t)A[5] << 32) : 0ull);
        return;
    }
    float fk = 0.0f;
#pragma unroll
    for (int jp = 0; jp < NP; jp++) {
        fk = fmaf((float)y[jp], K.finv[jp], fk);
    }
    // P/p_j has NP-1 words (one when NP == 1); the sum has NP words.
    constexpr int CW = NP > 1 ? NP - 1 : 1;
    uint64_t acc[NP + 1];
#pragma unroll
    for (int w = 0; w <= NP; w++) acc[w] = 0;
#pragma unroll
    for (int jp = 0; jp < NP; jp++) {
#pragma unroll
        for (int w = 0; w < CW; w++) {
            const uint64_t pr = (uint64_t)y[jp] * K.cof[jp][w];
            acc[w] += (uint32_t)pr;
            acc[w + 1] += pr >> 32;
        }
    }
    const uint32_t k = (uint32_t)rintf(fk);
    uint32_t X[NP];
    uint64_t carry = 0;
#pragma unroll
    for (int w = 0; w < NP; w++) {
        const uint64_t t = acc[w] + carry;
        X[w] = (uint32_t)t;
        carry = t >> 32;
    }
    int64_t borrow = 0;
#pragma unroll
    for (int w = 0; w < NP; w++) {
        const int64_t t = (int64_t)X[w] - (int64_t)((uint64_t)k * K.P[w]) - borrow;
        X[w] = (uint32_t)t;
        borrow = -(t >> 32);
    }
    uint32_t W[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int w = 0; w < NP && w < 6; w++) W[w] = X[w];
    c0 = (uint64_t)W[0] | ((uint64_t)W[1] << 32);
    c1 = (uint64_t)W[2] | ((uint64_t)W[3] << 32);
    c2 = (uint64_t)W[4] | ((uint64_t)W[5] << 32);
}

// Look-back status word: [31:4] epoch, [3:2] state (1 aggregate, 2 inclusive),
// [1] generate / carry-out, [0] propagate.
constexpr uint32_t ST_AGG = 1u << 2, ST_INC = 2u << 2;
constexpr long LOOKBACK_SPIN_LIMIT = 1L << 22;
// Residue CRT/carry tiles: CRT_THREADS threads of 4 coefficients.  Measured
// on the B200 (2^24 x 2^24 product): 128-thread tiles 0.330 ms, 256 0.337,
// 512 0.377 -- smaller tiles keep more of them resident per SM while one
// waits on its ticket or look-back.
constexpr int CRT_THREADS = 128;
constexpr int CRT_TILE = 4 * CRT_THREADS;

// NP == 0 is the direct mode: the coefficient values are precomputed (the
// basecase kernel's column sums) instead of recombined from residues.
template <int NP, int THREADS>
__global__ void __launch_bounds__(THREADS)
k_crt_carry(const uint32_t* __restrict__ res, int logM, uint64_t L, uint64_t zn,
            uint64_t* __restrict__ z, CrtConst K, uint32_t* __restrict__ status,
            unsigned long long* __restrict__ ticket, unsigned long long ticket_base,
            uint32_t epoch, int* __restrict__ err,
            const InstDesc* __restrict__ desc, const uint32_t* __restrict__ tile_inst,
            uint64_t base)
{
    constexpr int PER = 4;
    constexpr int TILE = PER * THREADS;
    constexpr int NW = THREADS / 32;
    // last three coefficients of each warp (slot w + 1; slot 0 = the tile's
    // halo, coefficients n0 - 3 .. n0 - 1): c0, c1, c2 of the last, c1, c2 of
    // the one before, c2 of the one before that
    __shared__ uint64_t wlast[NW + 1][6];
    __shared__ uint32_t sh_tile;
    __shared__ uint32_t wg[NW], wp[NW];
    __shared__ uint32_t sh_carry_in;

    if (threadIdx.x == 0) sh_tile = (uint32_t)(atomicAdd(ticket, 1ull) - ticket_base);
    __syncthreads();
    // `gtile` numbers tiles across the launch (status words, look-back order);
    // `tile` is the tile inside its product: a batch launch runs the tiles of
    // all its products back to back, and each product's first tile starts a
    // fresh carry chain, so look-backs never cross into the previous product.
    const uint32_t gtile = sh_tile;
    uint32_t tile = gtile;
    if (desc) {
        const InstDesc& D = desc[tile_inst[gtile]];
        tile = gtile - D.tile0;
        res = D.ra;
        L = D.an + D.bn - 1;
        zn = D.an + D.bn;
        z = D.z;
    }
    // coefficient / limb index of the tile's first position: a window product
    // starts at limb `base` (z[0] is limb base; limbs below it are not
    // produced and their carry into the window is not added -- the lower
    // approximation of a windowed product)
    const int64_t n0 = (int64_t)base + (int64_t)tile * TILE;
    // limbs below zn need coefficients below zn only; a window's transform
    // length covers min(L, zn) coefficients, not necessarily L
    L = L < zn ? L : zn;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // this thread's coefficients n0 + 4t .. n0 + 4t + 3, kept in registers;
    // a thread's four residues per prime are one 16-byte load when they lie
    // inside the array
    uint64_t c0[PER], c1[PER], c2[PER];
    {
        const uint64_t nb = (uint64_t)(n0 + threadIdx.x * PER);
        if constexpr (NP == 0) {
            // direct mode: values given as three planes of 2^logM 64-bit words
#pragma unroll
            for (int q = 0; q < PER; q++) {
                c0[q] = c1[q] = c2[q] = 0;
                if (nb + q < L) crt_coeff<0>(res, logM, nb + q, K, c0[q], c1[q], c2[q]);
            }
        } else {
            uint32_t y[PER][NP];
            // 16-byte loads need nb % 4 == 0 (always true for whole products; a
            // window may start at any limb) and the four residues inside the array
            if ((nb & 3) == 0 && nb + PER <= ((uint64_t)1 << logM)) {
#pragma unroll
                for (int jp = 0; jp < NP; jp++) {
                    const uint4 v = *reinterpret_cast<const uint4*>(res + ((size_t)jp << logM) + nb);
                    y[0][jp] = v.x; y[1][jp] = v.y; y[2][jp] = v.z; y[3][jp] = v.w;
                }
            } else {
#pragma unroll
                for (int q = 0; q < PER; q++)
#pragma unroll
                    for (int jp = 0; jp < NP; jp++)
                        y[q][jp] = (nb + q < L) ? res[((size_t)jp << logM) + nb + q] : 0u;
            }
#pragma unroll
            for (int q = 0; q < PER; q++) {
                c0[q] = c1[q] = c2[q] = 0;
                if (nb + q < L) crt_values<NP>(y[q], K, c0[q], c1[q], c2[q]);
            }
        }
    }
    if (lane == 31) {
        uint64_t* w = wlast[warp + 1];
        w[0] = c0[3]; w[1] = c1[3]; w[2] = c2[3]; w[3] = c1[2]; w[4] = c2[2]; w[5] = c2[1];
    }
    if (threadIdx.x < 3) {
        // halo: coefficients n0 - 1, n0 - 2, n0 - 3 (zero before the product),
        // one per lane of warp 0 so the three CRTs run side by side
        const int d = threadIdx.x + 1;
        const int64_t n = n0 - d;
        uint64_t h0 = 0, h1 = 0, h2 = 0;
        if (n >= 0 && (uint64_t)n < L) crt_coeff<NP>(res, logM, (uint64_t)n, K, h0, h1, h2);
        uint64_t* w = wlast[0];
        if (d == 1) { w[0] = h0; w[1] = h1; w[2] = h2; }
        else if (d == 2) { w[3] = h1; w[4] = h2; }
        else { w[5] = h2; }
    }
    __syncthreads();
    // the previous thread's last three coefficients (shuffle, or the slot of
    // the previous warp / the halo for lane 0)
    uint64_t p0 = __shfl_up_sync(0xffffffffu, c0[3], 1);
    uint64_t p1 = __shfl_up_sync(0xffffffffu, c1[3], 1);
    uint64_t p2 = __shfl_up_sync(0xffffffffu, c2[3], 1);
    uint64_t q1 = __shfl_up_sync(0xffffffffu, c1[2], 1);
    uint64_t q2 = __shfl_up_sync(0xffffffffu, c2[2], 1);
    uint64_t r2 = __shfl_up_sync(0xffffffffu, c2[1], 1);
    if (lane == 0) {
        const uint64_t* w = wlast[warp];
        p0 = w[0]; p1 = w[1]; p2 = w[2]; q1 = w[3]; q2 = w[4]; r2 = w[5];
    }

    // limb n receives s_n = X0[n] + X1[n-1] + X2[n-2] = lo_n + 2^64 cr_n (cr_n <= 2),
    // and then t_n = lo_n + cr_(n-1): a single-bit carry chain remains.
    auto s3 = [](uint64_t a, uint64_t b, uint64_t c, uint64_t& lo) -> uint32_t {
        uint64_t s = a;
        uint32_t cr = 0;
        uint64_t t = s + b; cr += t < s; s = t;
        t = s + c; cr += t < s; s = t;
        lo = s;
        return cr;
    };
    // X0, X1, X2 of coefficients 4t - 3 .. 4t + 3 relative to the thread
    const uint64_t x0[5] = {p0, c0[0], c0[1], c0[2], c0[3]};               // coefficients 4t-1 .. 4t+3
    const uint64_t x1[6] = {q1, p1, c1[0], c1[1], c1[2], c1[3]};           // 4t-2 .. 4t+3
    const uint64_t x2[7] = {r2, q2, p2, c2[0], c2[1], c2[2], c2[3]};       // 4t-3 .. 4t+3
    uint64_t tv[PER];
    uint32_t gbits = 0, pbits = 0;
    {
        uint64_t lo_prev;
        // s at limb 4t - 1: X0[4t-1] + X1[4t-2] + X2[4t-3]
        uint32_t cr_prev = (n0 + threadIdx.x * PER >= 1) ? s3(x0[0], x1[0], x2[0], lo_prev) : 0;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            uint64_t lo;
            const uint32_t cr = s3(x0[q + 1], x1[q + 1], x2[q + 1], lo);
            const uint64_t t = lo + cr_prev;
            const uint32_t g = t < lo;
            tv[q] = t;
            gbits |= g << q;
            pbits |= (uint32_t)(t == ~0ull) << q;
            cr_prev = cr;
        }
    }
    // thread aggregate (G, P) over its PER limbs, low to high
    uint32_t Gt = 0, Pt = 1;
    for (int q = 0; q < PER; q++) {
        const uint32_t g = (gbits >> q) & 1, pq = (pbits >> q) & 1;
        Gt = g | (pq & Gt);
        Pt = Pt & pq;
    }
    // inclusive warp scan of (G, P)
    uint32_t Gi = Gt, Pi = Pt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t Go = __shfl_up_sync(0xffffffffu, Gi, d);
        const uint32_t Po = __shfl_up_sync(0xffffffffu, Pi, d);
        if (lane >= d) { Gi = Gi | (Pi & Go); Pi = Pi & Po; }
    }
    if (lane == 31) { wg[warp] = Gi; wp[warp] = Pi; }
    __syncthreads();
    // exclusive prefix over warps (small, done redundantly per thread)
    uint32_t Gw = 0, Pw = 1;
    for (int w = 0; w < warp; w++) { Gw = wg[w] | (wp[w] & Gw); Pw = Pw & wp[w]; }
    // exclusive prefix for this thread within the tile
    uint32_t Ge = __shfl_up_sync(0xffffffffu, Gi, 1), Pe = __shfl_up_sync(0xffffffffu, Pi, 1);
    if (lane == 0) { Ge = 0; Pe = 1; }
    Ge = Ge | (Pe & Gw);
    Pe = Pe & Pw;

    if (threadIdx.x == THREADS - 1) {
        // tile aggregate = inclusive prefix of the last thread
        const uint32_t Gtile = Gi | (Pi & Gw);
        const uint32_t Ptile = Pi & Pw;
        uint32_t cin = 0;
        if (tile == 0) {
            __threadfence();
            atomicExch(&status[gtile], (epoch << 4) | ST_INC | (Gtile << 1));
        } else {
            atomicExch(&status[gtile], (epoch << 4) | ST_AGG | (Gtile << 1) | Ptile);
            uint32_t Gr = 0, Pr = 1;
            int64_t k = (int64_t)gtile - 1;
            long spins = 0;
            while (true) {
                const uint32_t st = *(volatile uint32_t*)&status[k];
                if ((st >> 4) != epoch || (st & (3u << 2)) == 0) {
                    if (++spins > LOOKBACK_SPIN_LIMIT) { atomicExch(err, 1); cin = 0; break; }
                    __nanosleep(64);
                    continue;
                }
                const uint32_t bg = (st >> 1) & 1, bp = st & 1;
                if ((st & (3u << 2)) == ST_INC) { cin = Gr | (Pr & bg); break; }
                Gr = Gr | (Pr & bg);
                Pr = Pr & bp;
                if (!Pr) { cin = Gr; break; }
                --k;
                if (k < 0) { cin = Gr; break; }
            }
            const uint32_t cout = Gtile | (Ptile & cin);
            atomicExch(&status[gtile], (epoch << 4) | ST_INC | (cout << 1));
        }
        sh_carry_in = cin;
    }
    __syncthreads();
    uint32_t c = Ge | (Pe & sh_carry_in);
    uint64_t v[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        v[q] = tv[q] + c;
        c = ((gbits >> q) & 1) | (((pbits >> q) & 1) & c);
    }
    const uint64_t nb = (uint64_t)(n0 + threadIdx.x * PER);
    uint64_t* dst = z + (nb - base);
    if (nb + PER <= zn && ((uintptr_t)dst & 15) == 0) {
        reinterpret_cast<ulonglong2*>(dst)[0] = make_ulonglong2(v[0], v[1]);
        reinterpret_cast<ulonglong2*>(dst)[1] = make_ulonglong2(v[2], v[3]);
    } else {
#pragma unroll
        for (int q = 0; q < PER; q++)
            if (nb + q < zn) dst[q] = v[q];
    }
}

// ---------------------------------------------------------------------------
// Calibration: the transforms' Gentleman-Sande butterfly (same form and pipe
// mix as the row passes) in a register-only loop, 16 values per thread, four
// levels per iteration -- the integer-pipe peak the product kernels are
// measured against.  Every value is stored at the end (out holds gridDim.x *
// blockDim.x * 16 words).
constexpr int CAL_ITERS = 256;

__global__ void __launch_bounds__(256)
k_bfly_rate(uint32_t* __restrict__ out, const uint2* __restrict__ tw, uint32_t p, uint32_t seed)
{
    constexpr int NV = 16;
    uint32_t x[NV];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int i = 0; i < NV; i++) x[i] = (seed * (t + 1) * (uint32_t)(2 * i + 7)) % p;
    uint32_t w[4], wq[4];
#pragma unroll
    for (int l = 0; l < 4; l++) { w[l] = tw[1 + l].x; wq[l] = tw[1 + l].y; }
    for (int it = 0; it < CAL_ITERS; it++) {
#pragma unroll
        for (int l = 0; l < 4; l++) {
            const int h = 1 << l;
#pragma unroll
            for (int i = 0; i < NV; i++)
                if (!(i & h)) bfly_gs<ROW_GS_FMA_ADDS>(x[i], x[i + h], w[l], wq[l], p);
        }
    }
    uint32_t* o = out + (size_t)t * NV;
#pragma unroll
    for (int i = 0; i < NV; i++) o[i] = x[i];
}

}  // namespace fb
