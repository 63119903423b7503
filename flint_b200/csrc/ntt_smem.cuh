// Block-cooperative number-theoretic transforms on vectors held in shared
// memory (and, for the last forward / first inverse levels, in registers).
//
// A forward transform of length L = 2^k is a Gentleman-Sande (decimation in
// frequency) network: natural-order input, bit-reversed output.  The level
// with half-size h pairs positions (j, j + h) inside blocks of 2h:
//     (a, b) -> (a + b, (a - b) * w_2h^(j mod h)).
// The inverse is the transposed Cooley-Tukey (decimation in time) network
// with inverse twiddles: bit-reversed input, natural output, scaled by L.
//
// Execution is split into passes; each thread loads the 2^Q elements of one
// radix-2^Q sub-transform, runs Q levels in registers and writes back:
//   * strided passes (levels with half-size >= 32): element stride S >= 32,
//     consecutive threads take consecutive sub-transforms, per-thread
//     twiddles w_2h^(jj0 + k S) are read from a table, each distinct one once;
//   * the contiguous pass (the five levels h = 16..1): each thread owns 32
//     consecutive positions; its twiddles are powers of w_32, the same for
//     every thread, and come from constant memory.
// How many additions per butterfly go to the FMA pipe is set per pass kind
// (ROW_GS_FMA_ADDS, ROW_CT_FMA_ADDS, COL_FMA_ADDS; see bfly_gs).
// Shared memory holds one pad word per 32 (physical = a + a/32), which makes
// both kinds of pass conflict-free and lets every address be a per-thread
// base plus a compile-time offset.
//
// Table layout: tw[h + jj] = (w_2h^jj, Shoup companion) for h a power of two;
// the entry for (h, jj) does not depend on L, so one table serves all lengths.
//
// The reference computes the same transforms with radix-4 double-precision
// butterflies over 256-point blocks (src/fft_small/sd_fft.c:1230-1274,
// src/fft_small/sd_ifft.c:1503-1533); the output order differs, which is
// harmless because only pointwise products are formed in transform space.
#pragma once
#include "modarith.cuh"

namespace fb {

constexpr int MAX_NP = 7;
// Butterfly form per pass kind (bfly_gs's F): column passes, row forward
// (Gentleman-Sande) passes, row inverse (Cooley-Tukey) passes.  Measured on
// the B200 (2^24 x 2^24 product): the row pass is fastest with the fused
// add-and-minimum form (F = -1: 1.500 -> 1.474 ms with the twiddle-1
// butterflies off the FMA pipe); the column passes, whose kernels run at 64
// registers, are fastest with separate adds and minima (F = 0; the fused
// form took the forward column pass from 1.28 to 1.56 ms); FMA-pipe
// additions (F >= 1) were slower everywhere (row pass 1.98 ms with 2/3 of
// them, 1.74 ms with none).
#ifndef FB_COL_FMA_ADDS
#define FB_COL_FMA_ADDS 0
#endif
// inverse column passes: fused reductions with FMA-pipe twiddle-1 butterflies
// (F = -2: 0.561 -> 0.539 ms against F = 0)
#ifndef FB_COL_CT_FMA_ADDS
#define FB_COL_CT_FMA_ADDS (-2)
#endif
#ifndef FB_ROW_GS_FMA_ADDS
#define FB_ROW_GS_FMA_ADDS (-1)
#endif
#ifndef FB_ROW_CT_FMA_ADDS
#define FB_ROW_CT_FMA_ADDS (-1)
#endif
constexpr int COL_FMA_ADDS = FB_COL_FMA_ADDS;
constexpr int COL_CT_FMA_ADDS = FB_COL_CT_FMA_ADDS;
// unroll factor of the strided passes' sub-transform loops
#ifndef FB_PASS_UNROLL
#define FB_PASS_UNROLL 1
#endif
constexpr int PASS_UNROLL = FB_PASS_UNROLL;
constexpr int ROW_GS_FMA_ADDS = FB_ROW_GS_FMA_ADDS;
constexpr int ROW_CT_FMA_ADDS = FB_ROW_CT_FMA_ADDS;

__host__ __device__ constexpr int padw(int a) { return a + (a >> 5); }

// w_32^k and w_32^-k (k < 16) with Shoup companions, per prime
struct W32Table {
    uint2 f[16];
    uint2 i[16];
};
__constant__ W32Table c_w32[MAX_NP];

// ---------------------------------------------------------------------------
// butterflies on registers

// Q Gentleman-Sande levels on 2^Q consecutive positions (half-sizes 2^(Q-1)..1)
template <int Q, int F = 2>
__device__ __forceinline__ void gs_contig(uint32_t (&x)[1 << Q], const W32Table& W, uint32_t p)
{
    constexpr int E = 1 << Q;
#pragma unroll
    for (int t = 0; t < Q; t++) {
        const int hm = E >> (t + 1);
#pragma unroll
        for (int m = 0; m < E; m++) {
            if ((m & hm) == 0) {
                const int k = m & (hm - 1);
                if (k == 0) {
                    bfly_gs1<F>(x[m], x[m + hm], p);
                } else {
                    const uint2 w = W.f[k * (16 / hm)];
                    bfly_gs<F>(x[m], x[m + hm], w.x, w.y, p);
                }
            }
        }
    }
}

// gs_contig on two independent vectors with the same twiddles (twice the
// independent work per thread for the scheduler)
template <int Q, int F = 2>
__device__ __forceinline__ void gs_contig2(uint32_t (&x)[1 << Q], uint32_t (&y)[1 << Q], const W32Table& W,
                                           uint32_t p)
{
    constexpr int E = 1 << Q;
#pragma unroll
    for (int t = 0; t < Q; t++) {
        const int hm = E >> (t + 1);
#pragma unroll
        for (int m = 0; m < E; m++) {
            if ((m & hm) == 0) {
                const int k = m & (hm - 1);
                if (k == 0) {
                    bfly_gs1<F>(x[m], x[m + hm], p);
                    bfly_gs1<F>(y[m], y[m + hm], p);
                } else {
                    const uint2 w = W.f[k * (16 / hm)];
                    bfly_gs<F>(x[m], x[m + hm], w.x, w.y, p);
                    bfly_gs<F>(y[m], y[m + hm], w.x, w.y, p);
                }
            }
        }
    }
}

// Q Cooley-Tukey levels on 2^Q consecutive positions (half-sizes 1..2^(Q-1))
template <int Q, int F = 2>
__device__ __forceinline__ void ct_contig(uint32_t (&x)[1 << Q], const W32Table& W, uint32_t p)
{
    constexpr int E = 1 << Q;
#pragma unroll
    for (int t = 0; t < Q; t++) {
        const int hm = 1 << t;
#pragma unroll
        for (int m = 0; m < E; m++) {
            if ((m & hm) == 0) {
                const int k = m & (hm - 1);
                if (k == 0) {
                    bfly_ct1<F>(x[m], x[m + hm], p);
                } else {
                    const uint2 w = W.i[k * (16 / hm)];
                    bfly_ct<F>(x[m], x[m + hm], w.x, w.y, p);
                }
            }
        }
    }
}

// Q Gentleman-Sande levels, half-sizes H..H/2^(Q-1), element stride S = H/2^(Q-1).
// Level t is a separate instantiation so every register index is a constant.
template <int Q, int H, int t, int F>
__device__ __forceinline__ void gs_strided_level(uint32_t (&x)[1 << Q], const uint2* __restrict__ tw,
                                                 int jj0, uint32_t p)
{
    constexpr int E = 1 << Q;
    constexpr int S = H >> (Q - 1);
    constexpr int hm = E >> (t + 1);
    constexpr int ht = H >> t;
    uint2 w[hm];
#pragma unroll
    for (int k = 0; k < hm; k++) w[k] = tw[ht + jj0 + k * S];
#pragma unroll
    for (int m = 0; m < E; m++)
        if ((m & hm) == 0) bfly_gs<F>(x[m], x[m + hm], w[m & (hm - 1)].x, w[m & (hm - 1)].y, p);
    if constexpr (t + 1 < Q) gs_strided_level<Q, H, t + 1, F>(x, tw, jj0, p);
}

template <int Q, int H, int F>
__device__ __forceinline__ void gs_strided(uint32_t (&x)[1 << Q], const uint2* __restrict__ tw,
                                           int jj0, uint32_t p)
{
    gs_strided_level<Q, H, 0, F>(x, tw, jj0, p);
}

// gs_strided on two vectors sharing the twiddle loads
template <int Q, int H, int t, int F>
__device__ __forceinline__ void gs_strided_level2(uint32_t (&x)[1 << Q], uint32_t (&y)[1 << Q],
                                                  const uint2* __restrict__ tw, int jj0, uint32_t p)
{
    constexpr int E = 1 << Q;
    constexpr int S = H >> (Q - 1);
    constexpr int hm = E >> (t + 1);
    constexpr int ht = H >> t;
    uint2 w[hm];
#pragma unroll
    for (int k = 0; k < hm; k++) w[k] = tw[ht + jj0 + k * S];
#pragma unroll
    for (int m = 0; m < E; m++)
        if ((m & hm) == 0) {
            bfly_gs<F>(x[m], x[m + hm], w[m & (hm - 1)].x, w[m & (hm - 1)].y, p);
            bfly_gs<F>(y[m], y[m + hm], w[m & (hm - 1)].x, w[m & (hm - 1)].y, p);
        }
    if constexpr (t + 1 < Q) gs_strided_level2<Q, H, t + 1, F>(x, y, tw, jj0, p);
}

// Q Cooley-Tukey levels, half-sizes H..2^(Q-1) H, element stride S = H
template <int Q, int H, int t, int F>
__device__ __forceinline__ void ct_strided_level(uint32_t (&x)[1 << Q], const uint2* __restrict__ twi,
                                                 int jj0, uint32_t p)
{
    constexpr int E = 1 << Q;
    constexpr int hm = 1 << t;
    constexpr int ht = H << t;
    uint2 w[hm];
#pragma unroll
    for (int k = 0; k < hm; k++) w[k] = twi[ht + jj0 + k * H];
#pragma unroll
    for (int m = 0; m < E; m++)
        if ((m & hm) == 0) bfly_ct<F>(x[m], x[m + hm], w[m & (hm - 1)].x, w[m & (hm - 1)].y, p);
    if constexpr (t + 1 < Q) ct_strided_level<Q, H, t + 1, F>(x, twi, jj0, p);
}

template <int Q, int H, int F>
__device__ __forceinline__ void ct_strided(uint32_t (&x)[1 << Q], const uint2* __restrict__ twi,
                                           int jj0, uint32_t p)
{
    ct_strided_level<Q, H, 0, F>(x, twi, jj0, p);
}

// ---------------------------------------------------------------------------
// Shared-memory layouts.
//   Rows:    NV vectors of length 2^LOGL, vector v at v * padw(L), element j
//            at padw(j) inside it.
//   Columns: G interleaved columns of length 2^LOGL, element j of column v at
//            padw(j * G) + v (valid because G divides 32 and v < G).

template <int LOGL, int G>
struct ColLayout {
    static constexpr int L = 1 << LOGL;
    __device__ static int addr(int v, int j) { return padw(j * G) + v; }
};

// One strided GS pass over every sub-transform of the tile.
// Rows layout (G == 0): NV vectors; columns layout: G columns.
template <int LOGL, int Q, int H, int G>
__device__ __forceinline__ void gs_pass_smem(uint32_t* sm, int nv, const uint2* __restrict__ tw, uint32_t p)
{
    constexpr int L = 1 << LOGL;
    constexpr int E = 1 << Q;
    constexpr int S = H >> (Q - 1);
    constexpr int NSUB = L / E;
    const int TOT = (G ? G : nv) * NSUB;
    // element m of a sub-transform sits at pb + padw(m S G'): a compile-time
    // offset when S G' is a multiple of 32, and also for S = 16 in the rows
    // layout (the base then lies in the low half of a 32-word bank row)
    static_assert(S * (G ? G : 1) % 32 == 0 || (G == 0 && S == 16), "unsupported pass stride");
    constexpr int SG = S * (G ? G : 1);
#pragma unroll PASS_UNROLL
    for (int f = threadIdx.x; f < TOT; f += blockDim.x) {
        int v, s;
        if (G) { v = f & (G - 1); s = f / (G ? G : 1); }
        else   { s = f & (NSUB - 1); v = f / NSUB; }
        const int jj0 = s & (S - 1);
        const int base = (s / S) * (2 * H) + jj0;
        const int pb = G ? padw(base * G) + v : v * padw(L) + padw(base);
        uint32_t x[E];
#pragma unroll
        for (int m = 0; m < E; m++) x[m] = sm[pb + padw(m * SG)];
        gs_strided<Q, H, (G == 0 ? ROW_GS_FMA_ADDS : COL_FMA_ADDS)>(x, tw, jj0, p);
#pragma unroll
        for (int m = 0; m < E; m++) sm[pb + padw(m * SG)] = x[m];
    }
}

// gs_pass_smem over two row buffers (rows layout) with one set of twiddles
template <int LOGL, int Q, int H>
__device__ __forceinline__ void gs_pass_smem2(uint32_t* sx, uint32_t* sy, int nv,
                                              const uint2* __restrict__ tw, uint32_t p)
{
    constexpr int L = 1 << LOGL;
    constexpr int E = 1 << Q;
    constexpr int S = H >> (Q - 1);
    constexpr int NSUB = L / E;
    const int TOT = nv * NSUB;
    static_assert(S % 32 == 0 || S == 16, "unsupported pass stride");
#pragma unroll PASS_UNROLL
    for (int f = threadIdx.x; f < TOT; f += blockDim.x) {
        const int s = f & (NSUB - 1), v = f / NSUB;
        const int jj0 = s & (S - 1);
        const int base = (s / S) * (2 * H) + jj0;
        const int pb = v * padw(L) + padw(base);
        uint32_t x[E], y[E];
#pragma unroll
        for (int m = 0; m < E; m++) {
            x[m] = sx[pb + padw(m * S)];
            y[m] = sy[pb + padw(m * S)];
        }
        gs_strided_level2<Q, H, 0, ROW_GS_FMA_ADDS>(x, y, tw, jj0, p);
#pragma unroll
        for (int m = 0; m < E; m++) {
            sx[pb + padw(m * S)] = x[m];
            sy[pb + padw(m * S)] = y[m];
        }
    }
}

template <int LOGL, int Q, int H, int G>
__device__ __forceinline__ void ct_pass_smem(uint32_t* sm, int nv, const uint2* __restrict__ twi, uint32_t p)
{
    constexpr int L = 1 << LOGL;
    constexpr int E = 1 << Q;
    constexpr int S = H;
    constexpr int NSUB = L / E;
    const int TOT = (G ? G : nv) * NSUB;
    static_assert(S * (G ? G : 1) % 32 == 0 || (G == 0 && S == 16), "unsupported pass stride");
    constexpr int SG = S * (G ? G : 1);
#pragma unroll PASS_UNROLL
    for (int f = threadIdx.x; f < TOT; f += blockDim.x) {
        int v, s;
        if (G) { v = f & (G - 1); s = f / (G ? G : 1); }
        else   { s = f & (NSUB - 1); v = f / NSUB; }
        const int jj0 = s & (S - 1);
        const int base = (s / S) * (S * E) + jj0;
        const int pb = G ? padw(base * G) + v : v * padw(L) + padw(base);
        uint32_t x[E];
#pragma unroll
        for (int m = 0; m < E; m++) x[m] = sm[pb + padw(m * SG)];
        ct_strided<Q, H, (G == 0 ? ROW_CT_FMA_ADDS : COL_CT_FMA_ADDS)>(x, twi, jj0, p);
#pragma unroll
        for (int m = 0; m < E; m++) sm[pb + padw(m * SG)] = x[m];
    }
}

// Strided part of the forward transform: all levels with half-size >= 32,
// i.e. LOGL - 5 levels, split into as few passes as QMAX allows with their
// sizes balanced (a one-level pass costs a full shared-memory round trip).
template <int REM, int QMAX>
constexpr int balanced_pass()
{
    return (REM + (REM + QMAX - 1) / QMAX - 1) / ((REM + QMAX - 1) / QMAX);
}

// First forward pass of rows that landed unpadded (rows layout, one row per
// block, blockDim = L / 32; the row kernel fills them with 16-byte copies,
// which the padded layout's 33-word lines cannot take).  The first pass has
// H = L / 2 and stride S = L / E, so sub-transform s covers s + m S: every
// thread reads its 32 / E sub-transforms of each vector into registers, and
// only after a barrier -- the padded positions overlap unpadded ones other
// threads have yet to read -- runs the levels and stores them padded.
template <int LOGL, int Q, int NVEC>
__device__ __forceinline__ void gs_pass_first_unpadded(uint32_t* sx, uint32_t* sy, const uint2* __restrict__ tw,
                                                       uint32_t p)
{
    constexpr int L = 1 << LOGL;
    constexpr int E = 1 << Q;
    constexpr int H = L / 2;
    constexpr int S = H >> (Q - 1);
    constexpr int IT = 32 / E;
    static_assert(S == L / E && IT >= 1 && L % 32 == 0, "unsupported first pass");
    uint32_t x[IT][E], y[NVEC == 2 ? IT : 1][NVEC == 2 ? E : 1];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int s = threadIdx.x + it * (L / 32);
#pragma unroll
        for (int m = 0; m < E; m++) {
            x[it][m] = sx[s + m * S];
            if constexpr (NVEC == 2) y[it][m] = sy[s + m * S];
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int s = threadIdx.x + it * (L / 32);
        if constexpr (NVEC == 2) gs_strided_level2<Q, H, 0, ROW_GS_FMA_ADDS>(x[it], y[it], tw, s, p);
        else gs_strided<Q, H, ROW_GS_FMA_ADDS>(x[it], tw, s, p);
        const int pb = padw(s);
#pragma unroll
        for (int m = 0; m < E; m++) {
            sx[pb + padw(m * S)] = x[it][m];
            if constexpr (NVEC == 2) sy[pb + padw(m * S)] = y[it][m];
        }
    }
}

// UNP: the data landed unpadded (gs_pass_first_unpadded; rows layout, nv = 1)
template <int LOGL, int G, int QMAX, int H, int REM, bool UNP = false>
__device__ __forceinline__ void gs_passes(uint32_t* sm, int nv, const uint2* __restrict__ tw, uint32_t p)
{
    if constexpr (REM > 0) {
        constexpr int Q = balanced_pass<REM, QMAX>();
        if constexpr (UNP) gs_pass_first_unpadded<LOGL, Q, 1>(sm, sm, tw, p);
        else gs_pass_smem<LOGL, Q, H, G>(sm, nv, tw, p);
        __syncthreads();
        gs_passes<LOGL, G, QMAX, (H >> Q), REM - Q>(sm, nv, tw, p);
    }
}

// LOGE: levels of the contiguous (register) pass that follows, 5 or 4
template <int LOGL, int G, int QMAX = (G ? 4 : 5), int LOGE = 5, bool UNP = false>
__device__ __forceinline__ void gs_strided_all(uint32_t* sm, int nv, const uint2* __restrict__ tw, uint32_t p)
{
    static_assert(!UNP || (G == 0 && LOGE == 5), "unpadded landing: rows layout, 32 per thread");
    if constexpr (LOGL > LOGE) gs_passes<LOGL, G, QMAX, (1 << (LOGL - 1)), LOGL - LOGE, UNP>(sm, nv, tw, p);
}

template <int LOGL, int QMAX, int H, int REM, bool UNP = false>
__device__ __forceinline__ void gs_passes2(uint32_t* sx, uint32_t* sy, int nv, const uint2* __restrict__ tw,
                                           uint32_t p)
{
    if constexpr (REM > 0) {
        constexpr int Q = balanced_pass<REM, QMAX>();
        if constexpr (UNP) gs_pass_first_unpadded<LOGL, Q, 2>(sx, sy, tw, p);
        else gs_pass_smem2<LOGL, Q, H>(sx, sy, nv, tw, p);
        __syncthreads();
        gs_passes2<LOGL, QMAX, (H >> Q), REM - Q>(sx, sy, nv, tw, p);
    }
}

// gs_strided_all for two row buffers at once (rows layout)
template <int LOGL, int QMAX = 5, int LOGE = 5, bool UNP = false>
__device__ __forceinline__ void gs_strided_all2(uint32_t* sx, uint32_t* sy, int nv, const uint2* __restrict__ tw,
                                                uint32_t p)
{
    static_assert(!UNP || LOGE == 5, "unpadded landing: 32 per thread");
    if constexpr (LOGL > LOGE) gs_passes2<LOGL, QMAX, (1 << (LOGL - 1)), LOGL - LOGE, UNP>(sx, sy, nv, tw, p);
}

// Strided part of the inverse transform (half-sizes 32 .. L/2), after the
// contiguous first pass; the mirror image of the forward schedule.
template <int LOGL, int G, int QMAX, int H, int REM>
__device__ __forceinline__ void ct_passes(uint32_t* sm, int nv, const uint2* __restrict__ twi, uint32_t p)
{
    if constexpr (REM > 0) {
        constexpr int Q = balanced_pass<REM, QMAX>();
        ct_pass_smem<LOGL, Q, H, G>(sm, nv, twi, p);
        __syncthreads();
        ct_passes<LOGL, G, QMAX, (H << Q), REM - Q>(sm, nv, twi, p);
    }
}

template <int LOGL, int G, int QMAX = (G ? 4 : 5), int LOGE = 5>
__device__ __forceinline__ void ct_strided_all(uint32_t* sm, int nv, const uint2* __restrict__ twi, uint32_t p)
{
    if constexpr (LOGL > LOGE) ct_passes<LOGL, G, QMAX, (1 << LOGE), LOGL - LOGE>(sm, nv, twi, p);
}

// The last inverse pass of one row (rows layout, one vector) with its output
// written straight to `out` (natural order) instead of back to shared
// memory: sub-transform s holds positions base + m H, consecutive threads
// take consecutive s, so each warp stores 32 consecutive words per m.
template <int LOGL, int Q, int H>
__device__ __forceinline__ void ct_pass_smem_out(const uint32_t* sm, const uint2* __restrict__ twi, uint32_t p,
                                                 uint32_t* __restrict__ out)
{
    constexpr int L = 1 << LOGL;
    constexpr int E = 1 << Q;
    constexpr int S = H;
    constexpr int NSUB = L / E;
    static_assert(S % 32 == 0, "unsupported pass stride");
#pragma unroll PASS_UNROLL
    for (int s = threadIdx.x; s < NSUB; s += blockDim.x) {
        const int jj0 = s & (S - 1);
        const int base = (s / S) * (S * E) + jj0;
        const int pb = padw(base);
        uint32_t x[E];
#pragma unroll
        for (int m = 0; m < E; m++) x[m] = sm[pb + padw(m * S)];
        ct_strided<Q, H, ROW_CT_FMA_ADDS>(x, twi, jj0, p);
#pragma unroll
        for (int m = 0; m < E; m++) out[base + m * S] = x[m];
    }
}

template <int LOGL, int QMAX, int H, int REM>
__device__ __forceinline__ void ct_passes_out(uint32_t* sm, const uint2* __restrict__ twi, uint32_t p,
                                              uint32_t* __restrict__ out)
{
    constexpr int Q = balanced_pass<REM, QMAX>();
    if constexpr (REM > Q) {
        ct_pass_smem<LOGL, Q, H, 0>(sm, 1, twi, p);
        __syncthreads();
        ct_passes_out<LOGL, QMAX, (H << Q), REM - Q>(sm, twi, p, out);
    } else {
        ct_pass_smem_out<LOGL, Q, H>(sm, twi, p, out);
    }
}

// ct_strided_all for one row (rows layout, nv = 1) whose final pass stores
// the row to global memory at `out`; needs LOGL > LOGE.  The shared buffer
// is read, not written, by the final pass.
template <int LOGL, int QMAX = 5, int LOGE = 5>
__device__ __forceinline__ void ct_strided_all_out(uint32_t* sm, const uint2* __restrict__ twi, uint32_t p,
                                                   uint32_t* __restrict__ out)
{
    static_assert(LOGL > LOGE, "row shorter than the contiguous pass");
    ct_passes_out<LOGL, QMAX, (1 << LOGE), LOGL - LOGE>(sm, twi, p, out);
}

}  // namespace fb
