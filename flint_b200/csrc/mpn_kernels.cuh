// Kernels of the integer multiplication path z = a * b (mpn limbs, 64-bit).
//
// Coefficients are single limbs (64-bit chunks); the cyclic convolution of
// length M = 2^m = R * C is computed modulo np word-size primes with a
// four-step transform:
//
//   k_fwd_cols   limbs -> residues (split fused into the load), length-R
//                forward transforms down every column, four-step twist
//                w_M^(i*k1), write.                     [one pass over HBM]
//   k_rows       per row: forward transforms of a and b, pointwise product
//                with the CRT/normalisation scale, inverse transform.
//                                                        [one pass over HBM]
//   k_inv_cols   untwist, length-R inverse transforms down every column.
//                                                        [one pass over HBM]
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

constexpr int LOG_MAXM = 25;          // largest cyclic length 2^25
constexpr int TW_SZ = 8192;           // local twiddle table entries per prime
constexpr int TH_SZ = 4096;           // twist table: w^(t * 2^13), t < 2^12
constexpr int TL_SZ = 8192;           // twist table: w^t, t < 2^13
constexpr int MAX_NP = 7;

struct DevTables {
    const PrimeInfo* pi;   // [MAX_NP]
    const uint2* twf;      // [MAX_NP][TW_SZ] forward local twiddles
    const uint2* twi;      // [MAX_NP][TW_SZ] inverse local twiddles
    const uint2* th;       // [MAX_NP][TH_SZ] w_{2^25}^(t 2^13)
    const uint2* tl;       // [MAX_NP][TL_SZ] w_{2^25}^t
    const uint2* thi;      // inverses of the above
    const uint2* tli;
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

// ---------------------------------------------------------------------------
// Column pass, forward: split + length-R transforms + twist.
// grid = (C / G, np, 2 operands); smem = R * G words.
__global__ void __launch_bounds__(512)
k_fwd_cols(DevTables T, const uint64_t* __restrict__ a, uint64_t an,
           const uint64_t* __restrict__ b, uint64_t bn,
           uint32_t* __restrict__ ra, uint32_t* __restrict__ rb, MulShape S)
{
    extern __shared__ uint32_t sm[];
    const int G = S.G;
    const int logR = S.logR, logC = S.logC;
    const int R = 1 << logR, C = 1 << logC;
    const int logM = logR + logC;
    const int j = blockIdx.y;
    const int i0 = blockIdx.x * G;
    const bool opb = blockIdx.z != 0;
    const uint64_t* __restrict__ x = opb ? b : a;
    const uint64_t xn = opb ? bn : an;
    uint32_t* __restrict__ out = (opb ? rb : ra) + ((size_t)j << logM);
    const PrimeInfo P = T.pi[j];
    const int tot = R * G;

    const uint64_t M = (uint64_t)1 << logM;
    for (int f = threadIdx.x; f < tot; f += blockDim.x) {
        const int u = f / G, c = f - u * G;
        uint64_t n = (uint64_t)u * C + i0 + c;
        uint32_t r = 0;
        // cyclic fold: an operand longer than M wraps around (x mod X^M - 1)
        for (; n < xn; n += M) r = add_mod(r, limb_redc(x[n], P.p, P.pneg_inv, P.c32), P.p);
        sm[swz(u * G + c)] = r;
    }
    __syncthreads();
    if (logR > 0) {
        VecLayout V{G, logR, 1, G, true};
        ntt_forward(sm, V, T.twf + (size_t)j * TW_SZ, P.p);
    }
    const uint2* __restrict__ th = T.th + (size_t)j * TH_SZ;
    const uint2* __restrict__ tl = T.tl + (size_t)j * TL_SZ;
    const int sh = LOG_MAXM - logM;
    for (int f = threadIdx.x; f < tot; f += blockDim.x) {
        const int u = f / G, c = f - u * G;
        const uint32_t k1 = bitrev_bits(u, logR);
        const uint32_t e = (((uint32_t)(i0 + c) * k1) & ((1u << logM) - 1)) << sh;
        const uint32_t v = twist_mul(sm[swz(u * G + c)], e, th, tl, P.p);
        out[(size_t)u * C + i0 + c] = v;
    }
}

// ---------------------------------------------------------------------------
// Row pass: forward transforms of a and b rows, pointwise product times
// scale[j], inverse transform; result overwrites the a row.
// grid = (R, np); smem = 2 * C words.
__global__ void __launch_bounds__(512)
k_rows(DevTables T, uint32_t* __restrict__ ra, const uint32_t* __restrict__ rb,
       MulShape S, const uint32_t* __restrict__ scale, int squaring)
{
    extern __shared__ uint32_t sm[];
    const int logC = S.logC;
    const int C = 1 << logC;
    const int logM = S.logR + logC;
    const int u = blockIdx.x;
    const int j = blockIdx.y;
    const PrimeInfo P = T.pi[j];
    uint32_t* __restrict__ arow = ra + ((size_t)j << logM) + (size_t)u * C;
    const uint32_t* __restrict__ brow = rb + ((size_t)j << logM) + (size_t)u * C;
    const int nv = squaring ? 1 : 2;

    for (int i = threadIdx.x; i < C; i += blockDim.x) {
        sm[swz(i)] = arow[i];
        if (!squaring) sm[swz(C + i)] = brow[i];
    }
    __syncthreads();
    {
        VecLayout V{nv, logC, C, 1, false};
        ntt_forward(sm, V, T.twf + (size_t)j * TW_SZ, P.p);
    }
    const uint32_t sc = scale[j];
    for (int i = threadIdx.x; i < C; i += blockDim.x) {
        const uint32_t x = sm[swz(i)];
        const uint32_t y = squaring ? x : sm[swz(C + i)];
        sm[swz(i)] = mul_mont(mul_mont(x, y, P.p, P.pneg_inv), sc, P.p, P.pneg_inv);
    }
    __syncthreads();
    {
        VecLayout V{1, logC, C, 1, false};
        ntt_inverse(sm, V, T.twi + (size_t)j * TW_SZ, P.p);
    }
    for (int i = threadIdx.x; i < C; i += blockDim.x) arow[i] = sm[swz(i)];
}

// ---------------------------------------------------------------------------
// Column pass, inverse: untwist + length-R inverse transforms, in place.
// grid = (C / G, np); smem = R * G words.
__global__ void __launch_bounds__(512)
k_inv_cols(DevTables T, uint32_t* __restrict__ ra, MulShape S)
{
    extern __shared__ uint32_t sm[];
    const int G = S.G;
    const int logR = S.logR, logC = S.logC;
    const int R = 1 << logR, C = 1 << logC;
    const int logM = logR + logC;
    const int j = blockIdx.y;
    const int i0 = blockIdx.x * G;
    uint32_t* __restrict__ buf = ra + ((size_t)j << logM);
    const PrimeInfo P = T.pi[j];
    const uint2* __restrict__ th = T.thi + (size_t)j * TH_SZ;
    const uint2* __restrict__ tl = T.tli + (size_t)j * TL_SZ;
    const int sh = LOG_MAXM - logM;
    const int tot = R * G;

    for (int f = threadIdx.x; f < tot; f += blockDim.x) {
        const int u = f / G, c = f - u * G;
        const uint32_t k1 = bitrev_bits(u, logR);
        const uint32_t e = (((uint32_t)(i0 + c) * k1) & ((1u << logM) - 1)) << sh;
        sm[swz(u * G + c)] = twist_mul(buf[(size_t)u * C + i0 + c], e, th, tl, P.p);
    }
    __syncthreads();
    if (logR > 0) {
        VecLayout V{G, logR, 1, G, true};
        ntt_inverse(sm, V, T.twi + (size_t)j * TW_SZ, P.p);
    }
    for (int f = threadIdx.x; f < tot; f += blockDim.x) {
        const int u = f / G, c = f - u * G;
        buf[(size_t)u * C + i0 + c] = sm[swz(u * G + c)];
    }
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
__device__ __forceinline__ void crt_coeff(const uint32_t* __restrict__ res, int logM, uint64_t n,
                                          const CrtConst& K, uint64_t& c0, uint64_t& c1, uint64_t& c2)
{
    uint32_t y[NP];
    float fk = 0.0f;
#pragma unroll
    for (int jp = 0; jp < NP; jp++) {
        y[jp] = res[((size_t)jp << logM) + n];
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

template <int NP, int THREADS>
__global__ void __launch_bounds__(THREADS)
k_crt_carry(const uint32_t* __restrict__ res, int logM, uint64_t L, uint64_t zn,
            uint64_t* __restrict__ z, CrtConst K, uint32_t* __restrict__ status,
            unsigned long long* __restrict__ ticket, unsigned long long ticket_base,
            uint32_t epoch, int* __restrict__ err)
{
    constexpr int PER = 4;
    constexpr int TILE = PER * THREADS;
    __shared__ uint64_t X0[TILE + 3], X1[TILE + 3], X2[TILE + 3];
    __shared__ uint32_t sh_tile;
    __shared__ uint32_t wg[THREADS / 32], wp[THREADS / 32];
    __shared__ uint32_t sh_carry_in;

    if (threadIdx.x == 0) sh_tile = (uint32_t)(atomicAdd(ticket, 1ull) - ticket_base);
    __syncthreads();
    const uint32_t tile = sh_tile;
    const int64_t n0 = (int64_t)tile * TILE;

    // coefficients n0-3 .. n0+TILE-1 into shared memory
    for (int q = 0; q < PER; q++) {
        const int idx = threadIdx.x * PER + q;
        const uint64_t n = (uint64_t)(n0 + idx);
        uint64_t c0 = 0, c1 = 0, c2 = 0;
        if (n < L) crt_coeff<NP>(res, logM, n, K, c0, c1, c2);
        X0[idx + 3] = c0; X1[idx + 3] = c1; X2[idx + 3] = c2;
    }
    if (threadIdx.x < 3) {
        const int64_t n = n0 - 3 + threadIdx.x;
        uint64_t c0 = 0, c1 = 0, c2 = 0;
        if (n >= 0 && (uint64_t)n < L) crt_coeff<NP>(res, logM, (uint64_t)n, K, c0, c1, c2);
        X0[threadIdx.x] = c0; X1[threadIdx.x] = c1; X2[threadIdx.x] = c2;
    }
    __syncthreads();

    // limb n receives s_n = X0[n] + X1[n-1] + X2[n-2] = lo_n + 2^64 cr_n (cr_n <= 2),
    // and then t_n = lo_n + cr_(n-1): a single-bit carry chain remains.
    auto s_at = [&](int idx, uint64_t& lo) -> uint32_t {   // idx = n - n0 + 3
        uint64_t s = X0[idx];
        uint32_t cr = 0;
        uint64_t t = s + X1[idx - 1]; cr += t < s; s = t;
        t = s + X2[idx - 2]; cr += t < s; s = t;
        lo = s;
        return cr;
    };
    uint64_t tv[PER];
    uint32_t gbits = 0, pbits = 0;
    {
        const int idx0 = threadIdx.x * PER + 3;
        uint64_t lo_prev;
        uint32_t cr_prev = (n0 + threadIdx.x * PER >= 1) ? s_at(idx0 - 1, lo_prev) : 0;
        for (int q = 0; q < PER; q++) {
            uint64_t lo;
            const uint32_t cr = s_at(idx0 + q, lo);
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
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
            atomicExch(&status[0], (epoch << 4) | ST_INC | (Gtile << 1));
        } else {
            atomicExch(&status[tile], (epoch << 4) | ST_AGG | (Gtile << 1) | Ptile);
            uint32_t Gr = 0, Pr = 1;
            int64_t k = (int64_t)tile - 1;
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
            atomicExch(&status[tile], (epoch << 4) | ST_INC | (cout << 1));
        }
        sh_carry_in = cin;
    }
    __syncthreads();
    uint32_t c = Ge | (Pe & sh_carry_in);
    for (int q = 0; q < PER; q++) {
        const uint64_t n = (uint64_t)(n0 + threadIdx.x * PER + q);
        const uint64_t v = tv[q] + c;
        c = ((gbits >> q) & 1) | (((pbits >> q) & 1) & c);
        if (n < zn) z[n] = v;
    }
}

}  // namespace fb
