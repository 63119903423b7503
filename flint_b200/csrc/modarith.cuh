// 32-bit modular arithmetic for the small-prime NTT (device and host).
//
// Primes p satisfy 2^30 < p < 2^31 and 2^24 | p - 1.  Residues are kept
// fully reduced in [0, p) between butterflies: with p above 2^31/2 there is
// only one spare bit in a 32-bit word, so a sum of two residues fits but a
// sum of two lazily reduced values in [0, 2p) would not.
//
// Two multiplication forms are used:
//   * Shoup's precomputed-quotient multiplication (V. Shoup, NTL; see also
//     D. Harvey, "Faster arithmetic for number-theoretic transforms", 2014)
//     for multiplication by a constant w with companion w' = floor(w 2^32/p):
//     q = hi32(a w'), r = a w - q p lies in [0, 2p) for every 32-bit a.
//   * Montgomery multiplication (P. Montgomery, 1985) with R = 2^32 for
//     products of two variables: REDC(a b) = a b R^-1 mod p.
//
// The reference does the same job with 50-bit primes held in doubles and
// fused multiply-add (src/machine_vectors.h:680-700, src/fft_small.h:206-222);
// this file replaces that arithmetic, it does not restate it.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define FB_HD __host__ __device__ __forceinline__
#else
#define FB_HD static inline
#endif

// Per-prime constants used by the kernels.
struct PrimeInfo {
    uint32_t p;        // the prime
    uint32_t pneg_inv; // -p^-1 mod 2^32 (Montgomery)
    uint32_t r2;       // 2^64 mod p (converts into Montgomery form)
    uint32_t c32;      // 2^32 mod p
    float    finv;     // 1/p rounded to float (CRT quotient estimate)
    uint32_t pad[3];
};

FB_HD uint32_t mulhi32(uint32_t a, uint32_t b)
{
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// r -> r mod p for r in [0, 2p)
FB_HD uint32_t red1(uint32_t r, uint32_t p)
{
    uint32_t t = r - p;
    return t < r ? t : r;   // unsigned min(r, r - p)
}

FB_HD uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p)
{
    return red1(a + b, p);
}

FB_HD uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p)
{
    return red1(a - b + p, p);
}

// Shoup companion floor(w 2^32 / p) for w < p
FB_HD uint32_t shoup_companion(uint32_t w, uint32_t p)
{
    return (uint32_t)(((uint64_t)w << 32) / p);
}

// a * w mod p in [0, 2p), any 32-bit a
FB_HD uint32_t mul_shoup_lazy(uint32_t a, uint32_t w, uint32_t wq, uint32_t p)
{
    uint32_t q = mulhi32(a, wq);
    return a * w - q * p;
}

FB_HD uint32_t mul_shoup(uint32_t a, uint32_t w, uint32_t wq, uint32_t p)
{
    return red1(mul_shoup_lazy(a, w, wq, p), p);
}

// Montgomery reduction of t < p 2^32: returns t 2^-32 mod p in [0, p)
FB_HD uint32_t redc64(uint64_t t, uint32_t p, uint32_t pneg_inv)
{
    uint32_t m = (uint32_t)t * pneg_inv;
    uint64_t u = t + (uint64_t)m * p;   // < 2 p 2^32 < 2^64
    return red1((uint32_t)(u >> 32), p);
}

// a b 2^-32 mod p for a, b < p
FB_HD uint32_t mul_mont(uint32_t a, uint32_t b, uint32_t p, uint32_t pneg_inv)
{
    return redc64((uint64_t)a * b, p, pneg_inv);
}

// Residue of a 64-bit limb times 2^-32: (hi 2^32 + lo) 2^-32 mod p.
// hi * c32 + lo <= (2^32-1)(p-1) + 2^32-1 < p 2^32, so one REDC suffices.
FB_HD uint32_t limb_redc(uint64_t x, uint32_t p, uint32_t pneg_inv, uint32_t c32)
{
    uint64_t t = (uint64_t)(uint32_t)(x >> 32) * c32 + (uint32_t)x;
    return redc64(t, p, pneg_inv);
}

#ifdef __CUDACC__
// Pipe balancing.  Integer adds, compares and min/max issue to the ALU pipe;
// IMAD issues to the FMA pipe.  Both run at half the issue rate, so an
// addition can be moved to the FMA pipe by writing it as x * one + y with
// `one` an opaque constant-memory 1 that the compiler cannot fold.  The
// butterflies take the number of such additions as a template parameter;
// the kernels' choices are measured (ntt_smem.cuh).
__constant__ uint32_t c_one;        // 1
__constant__ uint32_t c_minus_one;  // 0xffffffff

__device__ __forceinline__ uint32_t fadd(uint32_t x, uint32_t y) { return x * c_one + y; }
__device__ __forceinline__ uint32_t fsub(uint32_t x, uint32_t y) { return y * c_minus_one + x; }

// min(x + y, x + y - p) style reductions use the fused add-and-minimum
// (VIADDMNMX on sm_100, one ALU instruction for the add and the unsigned
// minimum): viaddmin(x, y, z) = min(x + y, z).
__device__ __forceinline__ uint32_t viaddmin(uint32_t x, uint32_t y, uint32_t z) { return __viaddmin_u32(x, y, z); }

// Butterfly forms.  F selects how the additions and reductions issue:
//   F = -1  fused add-and-minimum (VIADDMNMX) for every reduction, twiddle-1
//           butterflies on the ALU only: the fewest instructions;
//   F = -2  fused reductions, twiddle-1 butterflies as for F = 0;
//   F =  0  separate add and minimum, twiddle-1 butterflies with their add
//           and subtract on the FMA pipe (fadd / fsub);
//   F >= 1  as 0 with F of the additions on the FMA pipe.
// On sm_100 the three multiplications of Shoup's product hold the FMA pipe
// for 8 cycles per warp (the high-half multiply takes 4).  Which form runs
// fastest depends on the kernel around it (register budget and what else
// competes for the pipes); the choices are measured per pass kind
// (ntt_smem.cuh).

// Gentleman-Sande butterfly, inputs and outputs in [0, p):
// (a, b) -> (a + b, (a - b) w).
template <int F = 0>
__device__ __forceinline__ void bfly_gs(uint32_t& a, uint32_t& b, uint32_t w, uint32_t wq, uint32_t p)
{
    const uint32_t d = a - b + p;           // ALU, in [1, 2p)
    const uint32_t q = __umulhi(d, wq);
    const uint32_t r = d * w - q * p;       // [0, 2p)
    if constexpr (F < 0) {
        a = viaddmin(a, b, a + b - p);      // min(a + b, a + b - p)
        b = viaddmin(r, 0u - p, r);         // min(r - p, r)
    } else {
        const uint32_t s = F >= 1 ? fadd(a, b) : a + b;
        const uint32_t s1 = a + b - p;
        const uint32_t r1 = F >= 2 ? fadd(r, 0u - p) : r - p;
        a = min(s, s1);
        b = min(r, r1);
    }
}

// Gentleman-Sande butterfly with twiddle 1
template <int F = 0>
__device__ __forceinline__ void bfly_gs1(uint32_t& a, uint32_t& b, uint32_t p)
{
    if constexpr (F == -1) {
        const uint32_t s1 = a + b - p;
        const uint32_t d = a - b;
        a = viaddmin(a, b, s1);             // min(a + b, a + b - p)
        b = viaddmin(d, p, d);              // min(a - b + p, a - b)
    } else {
        const uint32_t s = fadd(a, b);
        const uint32_t s1 = a + b - p;
        const uint32_t d = a - b + p;
        const uint32_t d1 = fsub(a, b);
        a = min(s, s1);
        b = min(d, d1);
    }
}

// Cooley-Tukey butterfly, inputs and outputs in [0, p):
// (x, y) -> (x + y w, x - y w)
template <int F = 0>
__device__ __forceinline__ void bfly_ct(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wq, uint32_t p)
{
    const uint32_t q = __umulhi(y, wq);
    uint32_t t = y * w - q * p;             // [0, 2p)
    if constexpr (F < 0) {
        t = viaddmin(t, 0u - p, t);         // [0, p)
        const uint32_t s1 = x + t - p;
        const uint32_t d = x - t;
        x = viaddmin(x, t, s1);
        y = viaddmin(d, p, d);
    } else {
        t = min(t, F >= 3 ? fadd(t, 0u - p) : t - p);
        const uint32_t s = F >= 1 ? fadd(x, t) : x + t;
        const uint32_t s1 = x + t - p;
        const uint32_t d = x - t + p;
        const uint32_t d1 = F >= 2 ? fsub(x, t) : x - t;
        x = min(s, s1);
        y = min(d, d1);
    }
}

// Cooley-Tukey butterfly with twiddle 1 (the same arithmetic as bfly_gs1)
template <int F = 0>
__device__ __forceinline__ void bfly_ct1(uint32_t& x, uint32_t& y, uint32_t p)
{
    bfly_gs1<F>(x, y, p);
}
#endif

// host-side helpers ---------------------------------------------------------
static inline uint32_t h_mulmod(uint32_t a, uint32_t b, uint32_t p)
{
    return (uint32_t)(((uint64_t)a * b) % p);
}

static inline uint32_t h_powmod(uint32_t a, uint64_t e, uint32_t p)
{
    uint64_t r = 1, x = a % p;
    while (e) {
        if (e & 1) r = r * x % p;
        x = x * x % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

static inline uint32_t h_invmod(uint32_t a, uint32_t p)
{
    return h_powmod(a, p - 2, p);
}
