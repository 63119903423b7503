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
#include "mpn_kernels.cuh"

namespace fb {

constexpr int BASECASE_MAX = 4096;          // short operand of a single product
constexpr int BASECASE_BATCH_MAX = 1024;    // short operand of a planned batch's product
constexpr int BASECASE_THREADS = 256;
constexpr int BASECASE_PER = 4;                                  // positions per thread
constexpr int BASECASE_TILE = BASECASE_THREADS * BASECASE_PER;   // = the carry kernel's tile

__device__ __forceinline__ void mac192(uint64_t& a0, uint64_t& a1, uint64_t& a2, uint64_t x, uint64_t y)
{
    const uint64_t lo = x * y, hi = __umul64hi(x, y);
    asm("add.cc.u64  %0, %0, %3;\n\t"
        "addc.cc.u64 %1, %1, %4;\n\t"
        "addc.u64    %2, %2, 0;"
        : "+l"(a0), "+l"(a1), "+l"(a2)
        : "l"(lo), "l"(hi));
}

// One tile of 1024 positions per block; thread t computes positions
// k0 + 4t .. k0 + 4t + 3 with a sliding window of four x values (one shared
// load and four multiply-accumulates per y limb).  Planes: s[k], s[P + k],
// s[2P + k] with P = 2^logM.  With a batch descriptor the block's instance
// comes from tile_inst (the same tile map as the carry kernel) and x, y, s
// from the instance (s = its residue scratch).
__global__ void __launch_bounds__(BASECASE_THREADS)
k_basecase_sums(const uint64_t* __restrict__ x, uint64_t xn, const uint64_t* __restrict__ y,
                uint64_t yn, uint64_t* __restrict__ s, int logM,
                const InstDesc* __restrict__ desc, const uint32_t* __restrict__ tile_inst)
{
    __shared__ uint64_t sy[BASECASE_BATCH_MAX];
    __shared__ uint64_t sx[BASECASE_TILE + BASECASE_BATCH_MAX];
    uint32_t tile = blockIdx.x;
    if (desc) {
        const InstDesc& D = desc[tile_inst[blockIdx.x]];
        tile = blockIdx.x - D.tile0;
        x = D.a; xn = D.an; y = D.b; yn = D.bn;
        if (yn > xn) {
            const uint64_t* t = x; x = y; y = t;
            const uint64_t tn = xn; xn = yn; yn = tn;
        }
        s = reinterpret_cast<uint64_t*>(D.ra);
    }
    const uint64_t L = xn + yn - 1;
    const uint64_t k0 = (uint64_t)tile * BASECASE_TILE;
    for (uint32_t i = threadIdx.x; i < yn; i += BASECASE_THREADS) sy[i] = y[i];
    // x window k0 - (yn - 1) .. k0 + TILE - 1, zero outside [0, xn)
    const int64_t xb = (int64_t)k0 - (int64_t)(yn - 1);
    for (uint32_t i = threadIdx.x; i < BASECASE_TILE + yn - 1; i += BASECASE_THREADS) {
        const int64_t xi = xb + (int64_t)i;
        sx[i] = (xi >= 0 && (uint64_t)xi < xn) ? x[xi] : 0ull;
    }
    __syncthreads();
    // position k0 + 4t + q reads x[k0 + 4t + q - j] = sx[4t + q + yn - 1 - j]
    const uint64_t* px = sx + BASECASE_PER * threadIdx.x + (yn - 1);
    uint64_t w0 = px[0], w1 = px[1], w2 = px[2], w3 = px[3];
    uint64_t a[BASECASE_PER][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (uint32_t j = 0; j < yn; j++) {
        const uint64_t yj = sy[j];
        mac192(a[0][0], a[0][1], a[0][2], w0, yj);
        mac192(a[1][0], a[1][1], a[1][2], w1, yj);
        mac192(a[2][0], a[2][1], a[2][2], w2, yj);
        mac192(a[3][0], a[3][1], a[3][2], w3, yj);
        // slide: the next j needs x one position lower for every q
        w3 = w2; w2 = w1; w1 = w0;
        w0 = (j + 1 < yn) ? px[-(int64_t)(j + 1)] : 0ull;
    }
    const size_t P = (size_t)1 << logM;
#pragma unroll
    for (int q = 0; q < BASECASE_PER; q++) {
        const uint64_t k = k0 + BASECASE_PER * threadIdx.x + q;
        if (k < L) {
            s[k] = a[q][0];
            s[P + k] = a[q][1];
            s[2 * P + k] = a[q][2];
        }
    }
}

// Single products: the column sums split over both dimensions, so that a
// small product spreads over many blocks instead of one block per 1024
// positions.  Block (t, c) adds the partial sums of positions k0 .. k0 +
// BC_POS - 1 (k0 = t BC_POS) over y limbs j0 .. j0 + BC_JCH - 1 (j0 = c
// BC_JCH) into the planes by 64-bit atomic additions: the planes start at
// zero and the thread that adds word w of a partial also adds the carry out
// of that addition into word w + 1, so once every block has finished the
// planes hold the exact 192-bit sums (in any order of the additions).
// Inside a block, thread (p, r) takes positions k0 + 4p .. k0 + 4p + 3 over
// the r-th BC_JCH / BC_SPLIT limbs of the chunk; the BC_SPLIT partials of a
// position are summed in shared memory before the atomics.
constexpr int BC_POS = 128;                           // positions per block
constexpr int BC_SPLIT = 8;                           // sub-ranges of a chunk
constexpr int BC_JCH = 256;                           // y limbs per block
constexpr int BC_THREADS = (BC_POS / 4) * BC_SPLIT;   // 256

__device__ __forceinline__ void add192(uint64_t& a0, uint64_t& a1, uint64_t& a2, uint64_t b0, uint64_t b1,
                                       uint64_t b2)
{
    asm("add.cc.u64  %0, %0, %3;\n\t"
        "addc.cc.u64 %1, %1, %4;\n\t"
        "addc.u64    %2, %2, %5;"
        : "+l"(a0), "+l"(a1), "+l"(a2)
        : "l"(b0), "l"(b1), "l"(b2));
}

__global__ void __launch_bounds__(BC_THREADS)
k_basecase_split(const uint64_t* __restrict__ x, uint64_t xn, const uint64_t* __restrict__ y, uint64_t yn,
                 unsigned long long* __restrict__ s, int logM)
{
    __shared__ uint64_t sy[BC_JCH];
    __shared__ uint64_t sx[BC_POS + BC_JCH];
    __shared__ uint64_t part[BC_SPLIT][3][BC_POS];
    const int64_t k0 = (int64_t)blockIdx.x * BC_POS;
    const int64_t j0 = (int64_t)blockIdx.y * BC_JCH;
    // x indices k - j of the block: k0 - j0 - (BC_JCH - 1) .. k0 - j0 + BC_POS - 1;
    // a block entirely outside [0, xn) adds nothing (the test is the same for
    // every thread of the block)
    if (k0 - j0 + BC_POS - 1 < 0 || k0 - j0 - (BC_JCH - 1) >= (int64_t)xn) return;
    const int jn = (int)((int64_t)yn - j0 < BC_JCH ? (int64_t)yn - j0 : BC_JCH);
    for (int i = threadIdx.x; i < BC_JCH; i += BC_THREADS) sy[i] = i < jn ? y[j0 + i] : 0ull;
    const int64_t xb = k0 - j0 - (BC_JCH - 1);
    for (int i = threadIdx.x; i < BC_POS + BC_JCH - 1; i += BC_THREADS) {
        const int64_t xi = xb + i;
        sx[i] = (xi >= 0 && xi < (int64_t)xn) ? x[xi] : 0ull;
    }
    __syncthreads();
    constexpr int SUB = BC_JCH / BC_SPLIT;
    const int p = threadIdx.x % (BC_POS / 4), r = threadIdx.x / (BC_POS / 4);
    // position k0 + 4p + q times limb j0 + r SUB + i reads
    // x[k - j] = sx[4p + q - r SUB - i + BC_JCH - 1]
    const uint64_t* px = sx + 4 * p + (BC_JCH - 1) - r * SUB;
    uint64_t a[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    const int cnt = jn - r * SUB < SUB ? jn - r * SUB : SUB;   // <= 0: this sub-range is past y
    if (cnt > 0) {
        uint64_t w0 = px[0], w1 = px[1], w2 = px[2], w3 = px[3];
        for (int i = 0; i < cnt; i++) {
            const uint64_t yj = sy[r * SUB + i];
            mac192(a[0][0], a[0][1], a[0][2], w0, yj);
            mac192(a[1][0], a[1][1], a[1][2], w1, yj);
            mac192(a[2][0], a[2][1], a[2][2], w2, yj);
            mac192(a[3][0], a[3][1], a[3][2], w3, yj);
            w3 = w2; w2 = w1; w1 = w0;
            w0 = i + 1 < SUB ? px[-(i + 1)] : 0ull;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int w = 0; w < 3; w++) part[r][w][4 * p + q] = a[q][w];
    __syncthreads();
    if (threadIdx.x < BC_POS) {
        const int k = threadIdx.x;
        uint64_t s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
        for (int rr = 0; rr < BC_SPLIT; rr++) add192(s0, s1, s2, part[rr][0][k], part[rr][1][k], part[rr][2][k]);
        const uint64_t kk = (uint64_t)k0 + k;
        if (kk < xn + yn - 1 && (s0 | s1 | s2)) {
            const size_t P = (size_t)1 << logM;
            const uint64_t o0 = atomicAdd(&s[kk], (unsigned long long)s0);
            const uint64_t c0 = o0 + s0 < o0;
            const uint64_t t1 = s1 + c0;
            const uint64_t c1a = t1 < s1;
            const uint64_t o1 = atomicAdd(&s[P + kk], (unsigned long long)t1);
            const uint64_t c1b = o1 + t1 < o1;
            atomicAdd(&s[2 * P + kk], (unsigned long long)(s2 + c1a + c1b));
        }
    }
}

}  // namespace fb
