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

}  // namespace fb
