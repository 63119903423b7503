// Transformed operands: the product pipeline cut at its pointwise stage.
//
// A transformed operand is the forward transform of one operand modulo each
// of np primes, kept in HBM as np vectors of M words: k_fwd_cols (split,
// column transforms, twist) followed by k_rows_fwd (row transforms), whose
// output order is the row kernel's own (bit-reversed within each row) and
// the same for every operand of a plan, so pointwise operations need no
// reordering.  Products are formed elementwise (k_op_pointwise, with the
// normalisation folded into the multiplication exactly as the fused row
// pass does), then k_rows_inv and k_inv_cols transform back and a CRT kernel
// exports the result.  The reference's counterpart is the op API of
// src/fft_small/op.c:18-471 over plans of src/fft_small/plan.c.
#pragma once
#include "mpn_kernels.cuh"

namespace fb {

// forward row transforms of one operand, in place: grid = items
// (row groups x primes), block = nv C / 32, smem = nv padw(C) words; rows of
// prime j start at buf + j 2^(logR + LOGC), of which the first `rows` are used
template <int LOGC>
__global__ void __launch_bounds__(512)
k_rows_fwd(DevTables T, uint32_t* __restrict__ buf, int logR, int nv, int np, int rows)
{
    extern __shared__ uint32_t sm[];
    constexpr int C = 1 << LOGC;
    constexpr int PC = padw(C);
    constexpr int NSUB = C / 32;
    const int R = rows;                    // rows per prime (<= 2^logR)
    const int logM = logR + LOGC;
    const int groups = (R + nv - 1) / nv;
    const int j = blockIdx.x / groups;
    const int u0 = (blockIdx.x - j * groups) * nv;
    if (j >= np) return;
    const int t = threadIdx.x;
    const int pb = (t / NSUB) * PC + 33 * (t & (NSUB - 1));
    uint32_t* __restrict__ base = buf + ((size_t)j << logM);
    rows_prefetch<LOGC>(sm, base, u0, nv, R);
    cp_async_wait<0>();
    __syncthreads();
    const uint32_t p = T.pi[j].p;
    gs_strided_all<LOGC, 0>(sm, nv, T.twf + (size_t)j * TW_SZ, p);
    uint32_t xr[32];
#pragma unroll
    for (int m = 0; m < 32; m++) xr[m] = sm[pb + m];
    gs_contig<5>(xr, c_w32[j], p);
#pragma unroll
    for (int m = 0; m < 32; m++) sm[pb + m] = xr[m];
    __syncthreads();
    for (int f = t; f < nv * C; f += blockDim.x) {
        const int v = f >> LOGC, i = f & (C - 1);
        const int u = u0 + v;
        if (u < R) base[(size_t)u * C + i] = sm[v * PC + padw(i)];
    }
}

// inverse row transforms, in place (the normalisation was applied by the
// pointwise stage); launch shape as k_rows_fwd
template <int LOGC>
__global__ void __launch_bounds__(512)
k_rows_inv(DevTables T, uint32_t* __restrict__ buf, int logR, int nv, int np, int rows)
{
    extern __shared__ uint32_t sm[];
    constexpr int C = 1 << LOGC;
    constexpr int PC = padw(C);
    constexpr int NSUB = C / 32;
    const int R = rows;                    // rows per prime (<= 2^logR)
    const int logM = logR + LOGC;
    const int groups = (R + nv - 1) / nv;
    const int j = blockIdx.x / groups;
    const int u0 = (blockIdx.x - j * groups) * nv;
    if (j >= np) return;
    const int t = threadIdx.x;
    const int pb = (t / NSUB) * PC + 33 * (t & (NSUB - 1));
    uint32_t* __restrict__ base = buf + ((size_t)j << logM);
    rows_prefetch<LOGC>(sm, base, u0, nv, R);
    cp_async_wait<0>();
    __syncthreads();
    const uint32_t p = T.pi[j].p;
    uint32_t xr[32];
#pragma unroll
    for (int m = 0; m < 32; m++) xr[m] = sm[pb + m];
    ct_contig<5, 3>(xr, c_w32[j], p);
#pragma unroll
    for (int m = 0; m < 32; m++) sm[pb + m] = xr[m];
    __syncthreads();
    ct_strided_all<LOGC, 0>(sm, nv, T.twi + (size_t)j * TW_SZ, p);
    for (int f = t; f < nv * C; f += blockDim.x) {
        const int v = f >> LOGC, i = f & (C - 1);
        const int u = u0 + v;
        if (u < R) base[(size_t)u * C + i] = sm[v * PC + padw(i)];
    }
}

// Elementwise operations on np vectors of M words (words of prime j at j M).
// The products carry the plan's normalisation: a b scale_j 2^-64 (two
// Montgomery reductions), as in the fused row pass.
enum OpKind { OP_MUL = 0, OP_SQR = 1, OP_ADDMUL = 2, OP_SUBMUL = 3, OP_ADD = 4, OP_SUB = 5, OP_NEG = 6 };

__global__ void k_op_pointwise(DevTables T, int op, uint32_t* __restrict__ Z, const uint32_t* __restrict__ A,
                               const uint32_t* __restrict__ B, int logM, int np,
                               const uint32_t* __restrict__ scale)
{
    const size_t M = (size_t)1 << logM;
    const size_t total = M * np;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e >> logM);
        const PrimeInfo& P = T.pi[j];
        const uint32_t p = P.p;
        const uint32_t a = A[e];
        uint32_t r;
        switch (op) {
        case OP_MUL:
            r = mul_mont(mul_mont(a, B[e], p, P.pneg_inv), scale[j], p, P.pneg_inv);
            break;
        case OP_SQR:
            r = mul_mont(mul_mont(a, a, p, P.pneg_inv), scale[j], p, P.pneg_inv);
            break;
        case OP_ADDMUL:
            r = add_mod(Z[e], mul_mont(mul_mont(a, B[e], p, P.pneg_inv), scale[j], p, P.pneg_inv), p);
            break;
        case OP_SUBMUL:
            r = sub_mod(Z[e], mul_mont(mul_mont(a, B[e], p, P.pneg_inv), scale[j], p, P.pneg_inv), p);
            break;
        case OP_ADD:
            r = add_mod(a, B[e], p);
            break;
        case OP_SUB:
            r = sub_mod(a, B[e], p);
            break;
        default:
            r = a ? p - a : 0u;
            break;
        }
        Z[e] = r;
    }
}

// ---------------------------------------------------------------------------
// Signed export (the reference's fft_small_export_mpn_signed[_trunc],
// src/fft_small/export_signed.c): V = sum_(j < L) c_j 2^(64 j) with every
// coefficient lifted to the centered range (-P/2, P/2], written as the two's
// complement of V mod 2^(64 zw) and then as sign and magnitude.
//
// Limb u sums lo(c_u) + mid(c_(u-1)) + top(c_(u-2)), the top word signed
// (c_j as 192-bit two's complement), so with a carry-in in {-1, 0, 1, 2} its
// carry-out stays in {-1, 0, 1, 2}.  A carry map holds the carry-out for each
// of the four carry-ins (2 bits each, value + 1); maps compose, which gives a
// block scan inside each tile, one scan across tiles, and a fix-up that adds
// each tile's carry-in to its limbs.

constexpr int SIG_TILE = 512;             // limbs per tile, one per thread
constexpr uint32_t SIG_IDENTITY = 0xE4u;  // carry-in c -> carry-out c

// (g after f): carry-in -> f -> g
__device__ __forceinline__ uint32_t sig_compose(uint32_t g, uint32_t f)
{
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const uint32_t fc = (f >> (2 * c)) & 3u;
        r |= ((g >> (2 * fc)) & 3u) << (2 * c);
    }
    return r;
}

// centered coefficient j (0 beyond L) as 192-bit two's complement.  The
// CRT's quotient estimate rounds to nearest, so crt_values already returns
// the representative in (-P/2, P/2) (two's complement over 32 NP bits); five
// primes leave the top word 32 bits wide, sign-extended here as the integer
// polynomial export does.
template <int NP>
__device__ __forceinline__ void sig_coeff(const uint32_t* __restrict__ res, int logM, int64_t j, uint64_t L,
                                          const CrtConst& K, uint64_t& c0, uint64_t& c1, uint64_t& c2)
{
    c0 = c1 = c2 = 0;
    if (j < 0 || (uint64_t)j >= L) return;
    crt_coeff<NP>(res, logM, (uint64_t)j, K, c0, c1, c2);
    if (NP == 5) c2 = (uint64_t)(int64_t)(int32_t)(uint32_t)c2;
}

// per tile: limbs with a zero carry-in into z[0, zw), the tile's carry map
template <int NP>
__global__ void __launch_bounds__(SIG_TILE)
k_sig_tiles(const uint32_t* __restrict__ res, int logM, uint64_t L, uint64_t zw, uint64_t* __restrict__ z,
            CrtConst K, uint8_t* __restrict__ maps)
{
    __shared__ uint64_t s0[SIG_TILE], s1[SIG_TILE + 1], s2[SIG_TILE + 2];
    __shared__ uint32_t s_w[SIG_TILE / 32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int64_t u = (int64_t)blockIdx.x * SIG_TILE + t;
    uint64_t c0, c1, c2;
    sig_coeff<NP>(res, logM, u, L, K, c0, c1, c2);
    s0[t] = c0;
    s1[t + 1] = c1;
    s2[t + 2] = c2;
    if (t < 2) {   // the two coefficients below the tile
        uint64_t h0, h1, h2;
        sig_coeff<NP>(res, logM, (int64_t)blockIdx.x * SIG_TILE - 2 + t, L, K, h0, h1, h2);
        if (t == 1) s1[0] = h1;
        s2[t] = h2;
    }
    __syncthreads();
    // s = lo(c_u) + mid(c_(u-1)) + top(c_(u-2)), top signed: a 128-bit signed sum
    const uint64_t a = s0[t], b = s1[t], h = s2[t];
    uint64_t lo = a + b;
    int64_t hi = (int64_t)(lo < a);
    const uint64_t l2 = lo + h;
    hi += (int64_t)(l2 < lo) - (int64_t)(h >> 63);
    lo = l2;
    // carry map of this limb and the limb value for carry-ins -1 .. 2
    uint32_t f = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int64_t cin = c - 1;
        const uint64_t v = lo + (uint64_t)cin;
        int64_t cout = hi;
        if (cin > 0 && v < lo) cout += 1;
        if (cin < 0 && lo == 0) cout -= 1;
        f |= (uint32_t)(cout + 1) << (2 * c);
    }
    if ((uint64_t)u >= zw) f = SIG_IDENTITY;
    // inclusive scan of maps over the block (lower limbs applied first)
    uint32_t incl = f;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl = sig_compose(incl, o);
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < SIG_TILE / 32 ? s_w[lane] : SIG_IDENTITY;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w = sig_compose(w, o);
        }
        if (lane < SIG_TILE / 32) s_w[lane] = w;
    }
    __syncthreads();
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = SIG_IDENTITY;
    if (wid > 0) excl = sig_compose(excl, s_w[wid - 1]);
    // carry into this limb with a zero carry-in to the tile
    const int64_t cin = (int64_t)((excl >> 2) & 3u) - 1;
    if ((uint64_t)u < zw) z[u] = lo + (uint64_t)cin;
    if (t == SIG_TILE - 1) maps[blockIdx.x] = (uint8_t)s_w[SIG_TILE / 32 - 1];
}

// carry-in of every tile (one block): exclusive scan of the tile maps
__global__ void __launch_bounds__(1024)
k_sig_scan(const uint8_t* __restrict__ maps, uint64_t ntiles, int8_t* __restrict__ cin)
{
    __shared__ uint32_t s_w[32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const uint64_t per = (ntiles + 1023) / 1024;
    const uint64_t b0 = t * per, b1 = min(ntiles, b0 + per);
    uint32_t m = SIG_IDENTITY;
    for (uint64_t k = b0; k < b1; k++) m = sig_compose(maps[k], m);
    uint32_t incl = m;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl = sig_compose(incl, o);
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = s_w[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w = sig_compose(w, o);
        }
        s_w[lane] = w;
    }
    __syncthreads();
    uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = SIG_IDENTITY;
    if (wid > 0) excl = sig_compose(excl, s_w[wid - 1]);
    for (uint64_t k = b0; k < b1; k++) {
        cin[k] = (int8_t)((int)((excl >> 2) & 3u) - 1);
        excl = sig_compose(maps[k], excl);
    }
}

// adds each tile's carry-in (-1 .. 2) to its limbs; the ripple stays inside
// the tile (what leaves it is the next tile's carry-in)
__global__ void __launch_bounds__(SIG_TILE)
k_sig_fix(uint64_t* __restrict__ z, uint64_t zw, const int8_t* __restrict__ cin)
{
    __shared__ int s_first;
    const int c = cin[blockIdx.x];
    if (c == 0) return;
    const uint64_t base = (uint64_t)blockIdx.x * SIG_TILE;
    const uint64_t end = min(zw, base + SIG_TILE);
    const int t = threadIdx.x;
    if (t == 0) s_first = SIG_TILE;
    __syncthreads();
    const uint64_t v0 = z[base];
    // does the first limb pass the carry (borrow) on?
    const bool pass = c > 0 ? (v0 + (uint64_t)c < v0) : (v0 == 0);
    const uint64_t u = base + t;
    if (pass && t >= 1 && u < end) {
        const uint64_t v = z[u];
        if (c > 0 ? v != ~0ull : v != 0ull) atomicMin(&s_first, t);
    }
    __syncthreads();
    const int k = s_first;                      // first limb that stops the ripple
    if (t == 0) z[base] = v0 + (uint64_t)(int64_t)c;
    if (pass && t >= 1 && u < end) {
        if (t < k) z[u] = c > 0 ? 0ull : ~0ull;
        else if (t == k) z[u] = c > 0 ? z[u] + 1 : z[u] - 1;
    }
}

// first non-zero limb of z[0, zw) (atomicMin into *first, set to zw before)
__global__ void k_sig_first_nonzero(const uint64_t* __restrict__ z, uint64_t zw, unsigned long long* first)
{
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < zw; u += (uint64_t)gridDim.x * blockDim.x)
        if (z[u] != 0) { atomicMin(first, (unsigned long long)u); break; }
}

// magnitude: if the top bit of z[zw - 1] is set, z = -z mod 2^(64 zw); the
// window [lo, lo + zn) goes to out, flags[0] = negative, flags[1] = window
// non-zero (out may alias z when lo == 0)
__global__ void k_sig_magnitude(uint64_t* __restrict__ z, uint64_t zw, const unsigned long long* first,
                                uint64_t lo, uint64_t zn, uint64_t* out, int* flags)
{
    const bool neg = (z[zw - 1] >> 63) != 0;
    const uint64_t k = *first;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < zn; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t u = lo + i;
        uint64_t v = z[u];
        if (neg) v = u < k ? 0ull : (u == k ? 0ull - v : ~v);
        out[i] = v;
        if (v) flags[1] = 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) flags[0] = neg ? 1 : 0;
}

}  // namespace fb
