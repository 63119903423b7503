/*
    gpu_fft_small.h -- C ABI of the B200 small-prime NTT multiplication path.

    A drop-in, at function level, for the mpn_ctx route of FLINT's fft_small
    module.  Each entry point has the shape of the reference function it
    replaces (named beside it, file:line in the reference tree); the context
    type is opaque because the reference's mpn_ctx_struct holds CPU twiddle
    tables (src/fft_small.h:382-413) that have no meaning here.

    Conventions (same as the reference, src/fft_small.h and
    doc/source/fft_small.rst):
      * limbs are 64-bit, little-endian; the caller owns every array;
      * z must not overlap a or b; z receives an + bn limbs (mpn products)
        or zh - zl coefficients (polynomial windows);
      * a == b with an == bn is a squaring;
      * a context is not reentrant: calls on one context must not overlap
        (the reference's context shares one scratch buffer the same way,
        src/fft_small/mpn_mul.c:1342-1362).

    Errors: the void functions report failures through the throw handler
    (default: print and abort(), like flint_throw in
    src/generic_files/exception.c); the *_status variants and the
    device-pointer variants return 0 on success or a GPU_FFT_SMALL_E* code.
    There is no CPU fallback: without a usable GPU every call fails.
*/
#ifndef GPU_FFT_SMALL_H
#define GPU_FFT_SMALL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GPU_FFT_SMALL_API __attribute__((visibility("default")))
#else
#define GPU_FFT_SMALL_API
#endif

typedef unsigned long gpu_ulong;   /* FLINT ulong / mp_limb_t on LP64 */
typedef long gpu_slong;

/* status codes */
#define GPU_FFT_SMALL_OK          0
#define GPU_FFT_SMALL_EINVAL      1   /* bad argument (sizes, aliasing, modulus) */
#define GPU_FFT_SMALL_ETOOBIG     2   /* beyond the supported transform length */
#define GPU_FFT_SMALL_ECUDA       3   /* CUDA runtime error (no GPU, OOM, ...) */
#define GPU_FFT_SMALL_ETIMEOUT    4   /* a bounded device wait gave up */
#define GPU_FFT_SMALL_ENOPRIMES   5   /* coefficient bound exceeds the primes */

/* Opaque context, used exactly like mpn_ctx_t: declare, init, use, clear. */
typedef struct {
    void *impl;
} gpu_mpn_ctx_struct;
typedef gpu_mpn_ctx_struct gpu_mpn_ctx_t[1];

/* nmod_t of the reference (src/flint.h.in:440-447): n, its preinverse, and
   the normalisation shift; only n is read. */
typedef struct {
    gpu_ulong n;
    gpu_ulong ninv;
    gpu_ulong norm;
} gpu_nmod_t;

/* --- context (replaces mpn_ctx_init / mpn_ctx_clear, src/fft_small.h:422-423) */

/* p plays the role of the reference's starting prime (DEFAULT_PRIME,
   src/fft_small/default_ctx.c:17); the GPU path uses its own fixed set of
   31-bit primes and records p only for identification.  Binds the context to
   the current CUDA device. */
GPU_FFT_SMALL_API void gpu_mpn_ctx_init(gpu_mpn_ctx_t R, gpu_ulong p);
GPU_FFT_SMALL_API int gpu_mpn_ctx_init_status(gpu_mpn_ctx_t R, gpu_ulong p);
GPU_FFT_SMALL_API void gpu_mpn_ctx_clear(gpu_mpn_ctx_t R);

/* --- integer products ---------------------------------------------------- */

/* z[0, an+bn) = a * b.  Replaces mpn_ctx_mpn_mul (src/fft_small.h:433,
   src/fft_small/mpn_mul.c:1980-1983).  Requires an, bn >= 1.  Products of
   up to 2^25 + 1 limbs in all; beyond, an unbalanced product whose short
   operand leaves room for chunks of at most 2^25 points runs split (up to
   2^30 limbs), anything else is GPU_FFT_SMALL_ETOOBIG
   (gpu_mpn_mul_split_plan tells which). */
GPU_FFT_SMALL_API void gpu_mpn_ctx_mpn_mul(gpu_mpn_ctx_t R, gpu_ulong *z,
                         const gpu_ulong *a, gpu_ulong an,
                         const gpu_ulong *b, gpu_ulong bn);
GPU_FFT_SMALL_API int gpu_mpn_ctx_mpn_mul_status(gpu_mpn_ctx_t R, gpu_ulong *z,
                               const gpu_ulong *a, gpu_ulong an,
                               const gpu_ulong *b, gpu_ulong bn);

/* Pipelines of host-pointer products (no counterpart in the reference, whose
   calls return with the product done).  A pipeline holds `depth` contexts
   (slots, 1..GPU_MPN_PIPE_MAX_DEPTH) that take submitted products in turn,
   so one product's download, the next one's upload and another one's kernels
   overlap; from pinned host memory the copies run asynchronously, from
   pageable memory a submission waits for its uploads.
   gpu_mpn_pipe_submit queues z[0, an+bn) = a * b (an, bn >= 1) and returns
   a ticket; a, b and z must stay valid and unchanged until the ticket has
   been waited for.  A submission to a busy slot first completes the product
   that slot holds.  gpu_mpn_pipe_wait returns the product's status once z
   holds it; every ticket is waited for once (a second wait, or an unknown
   ticket, is EINVAL), and the statuses of completed products are kept
   until then.
   gpu_mpn_pipe_clear completes every product in flight and frees the
   pipeline.  Not reentrant, like a context. */
#define GPU_MPN_PIPE_MAX_DEPTH 4
typedef struct {
    void *impl;
} gpu_mpn_pipe_struct;
typedef gpu_mpn_pipe_struct gpu_mpn_pipe_t[1];
GPU_FFT_SMALL_API int gpu_mpn_pipe_init(gpu_mpn_pipe_t P, int depth);
GPU_FFT_SMALL_API int gpu_mpn_pipe_submit(gpu_mpn_pipe_t P, gpu_ulong *z,
                        const gpu_ulong *a, gpu_ulong an,
                        const gpu_ulong *b, gpu_ulong bn, long long *ticket);
GPU_FFT_SMALL_API int gpu_mpn_pipe_wait(gpu_mpn_pipe_t P, long long ticket);
GPU_FFT_SMALL_API void gpu_mpn_pipe_clear(gpu_mpn_pipe_t P);

/* Limbs [lo, hi) of a * b into z[0, hi-lo), zero beyond an + bn.  Replaces
   _mpn_ctx_mpn_mul_range (src/fft_small.h:462, src/fft_small/mpn_mul.c:
   1617-1978) with its contract (src/fft_small/test/t-mpn_mulmid.c): exact for
   lo = 0; for lo > 0 a lower approximation of floor(a b / 2^(64 lo)) that
   depends on a, b and lo only (not on hi), here short by at most 2 units --
   the carry rippling up from the limbs below lo is not added, and is zero
   unless limb lo - 1 of the exact product is within 2 of 2^64 - 1.  A window
   well below the top of the product runs a shorter cyclic transform. */
GPU_FFT_SMALL_API void _gpu_mpn_ctx_mpn_mul_range(gpu_mpn_ctx_t R, gpu_ulong *z,
                                gpu_ulong lo, gpu_ulong hi,
                                const gpu_ulong *a, gpu_ulong an,
                                const gpu_ulong *b, gpu_ulong bn);

/* Device-pointer twin of _gpu_mpn_ctx_mpn_mul_range: limbs [lo, hi) of a * b
   into z_dev[0, min(hi, an+bn) - lo) on `stream` (no zero fill; hi is
   clamped to an + bn). */
GPU_FFT_SMALL_API int gpu_mpn_mul_range_device(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong lo, gpu_ulong hi,
                                               const uint64_t *a_dev, gpu_ulong an,
                                               const uint64_t *b_dev, gpu_ulong bn, void *stream);
/* Same signature as flint_mpn_mulmid_fft_small (src/mpn_extras.h:686,
   src/mpn_extras/mulmid_fft_small.c:26-31): the window [zlo, zhi) on the
   calling thread's default context. */
GPU_FFT_SMALL_API void gpu_mpn_mulmid_default_mpn_ctx(gpu_ulong *z, const gpu_ulong *a, gpu_slong an,
                                                      const gpu_ulong *b, gpu_slong bn, gpu_slong zlo,
                                                      gpu_slong zhi);

/* Device-pointer twin of gpu_mpn_ctx_mpn_mul: a, b, z are device addresses,
   the work is queued on `stream` (a cudaStream_t; NULL is CUDA's default
   stream) and the call returns without synchronising when it succeeds. */
GPU_FFT_SMALL_API int gpu_mpn_mul_device(gpu_mpn_ctx_t R, uint64_t *z_dev,
                       const uint64_t *a_dev, gpu_ulong an,
                       const uint64_t *b_dev, gpu_ulong bn, void *stream);

/* Allocation-free product on device pointers (no counterpart in the
   reference).  For callers that cannot call cudaMalloc: a framework that owns
   all device memory through its own pool and forbids outside allocations, or
   a latency-critical pipeline that cannot take cudaMalloc's implicit
   device-wide synchronisation.  The caller passes device buffers for a, b and
   z; every other byte used lives in arrays that are part of the library's
   device image (about 10 MB of scratch plus 2 MB of tables, held on every GPU
   that loads the library until the process exits).  The call allocates
   nothing and does not synchronise; the work goes on `stream` (NULL is CUDA's
   default stream).
     * Limit: an + bn <= 2^18 + 1 limbs; larger products return
       GPU_FFT_SMALL_ETOOBIG.  Empty operands return GPU_FFT_SMALL_EINVAL.
     * The first call on a device does a one-time set-up there (table
       generation, a device synchronisation); make that first call before
       any stream capture.
     * All calls share the scratch, which keeps the last call's contents:
       calls whose work overlaps on the GPU (other streams, other host
       threads) race, so the caller must serialise them.
     * The return code covers argument checks, the set-up and the launches
       only.  The carry pass's bounded wait (which valid inputs never
       exhaust) flags a timeout in the library's scratch, which a call that
       does not synchronise cannot read back, so such a device-side error is
       not reported here. */
GPU_FFT_SMALL_API int gpu_mpn_mul_device_noalloc(uint64_t *z_dev, const uint64_t *a_dev,
                                                 gpu_ulong an, const uint64_t *b_dev,
                                                 gpu_ulong bn, void *stream);

/* --- nmod polynomials ---------------------------------------------------- */

/* z[0, zh-zl) = coefficients [zl, zh) of a * b mod n, inputs reduced mod n.
   Replaces _nmod_poly_mul_mid_mpn_ctx (src/fft_small.h:769-774,
   src/fft_small/nmod_poly_mul.c:904-972). */
GPU_FFT_SMALL_API void _gpu_nmod_poly_mul_mid_mpn_ctx(gpu_ulong *z, gpu_ulong zl, gpu_ulong zh,
                                    const gpu_ulong *a, gpu_ulong an,
                                    const gpu_ulong *b, gpu_ulong bn,
                                    gpu_nmod_t mod, gpu_mpn_ctx_t R);
GPU_FFT_SMALL_API int _gpu_nmod_poly_mul_mid_status(gpu_ulong *z, gpu_ulong zl, gpu_ulong zh,
                                  const gpu_ulong *a, gpu_ulong an,
                                  const gpu_ulong *b, gpu_ulong bn,
                                  gpu_nmod_t mod, gpu_mpn_ctx_t R);

/* Device-pointer twin of _gpu_nmod_poly_mul_mid_mpn_ctx: coefficients
   [zl, zh) of a * b mod n into z_dev[0, zh - zl) (zero where the product has
   no coefficient), a and b reduced mod n, all device addresses; queued on
   `stream` (a cudaStream_t), returns without synchronising. */
GPU_FFT_SMALL_API int gpu_nmod_poly_mul_mid_device(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong zl, gpu_ulong zh,
                                                   const uint64_t *a_dev, gpu_ulong an,
                                                   const uint64_t *b_dev, gpu_ulong bn,
                                                   gpu_nmod_t mod, void *stream);

/* q[0, an-bn+1) and r[0, bn-1): quotient and remainder of a by b mod n
   (an >= bn > 1, b's leading coefficient a unit mod n, inputs reduced mod n).
   Replaces _nmod_poly_divrem_mpn_ctx (src/fft_small.h:776-782,
   src/fft_small/nmod_poly_mul.c:1248-1277): the power-series inverse of the
   reversed divisor by Newton iteration, the quotient from one middle product,
   the remainder from a cyclic product mod x^N - 1, all on the device. */
GPU_FFT_SMALL_API void _gpu_nmod_poly_divrem_mpn_ctx(gpu_ulong *q, gpu_ulong *r,
                                                     const gpu_ulong *a, gpu_ulong an,
                                                     const gpu_ulong *b, gpu_ulong bn,
                                                     gpu_nmod_t mod, gpu_mpn_ctx_t R);
GPU_FFT_SMALL_API int _gpu_nmod_poly_divrem_status(gpu_ulong *q, gpu_ulong *r,
                                                   const gpu_ulong *a, gpu_ulong an,
                                                   const gpu_ulong *b, gpu_ulong bn,
                                                   gpu_nmod_t mod, gpu_mpn_ctx_t R);

/* --- default context (replaces src/fft_small/default_ctx.c:29-51) ---------- */

/* One context per host thread, created on first use with the reference's
   default starting prime. */
GPU_FFT_SMALL_API gpu_mpn_ctx_struct *gpu_get_default_mpn_ctx(void);

/* Releases the calling thread's default context (its device buffers and
   streams), as mpn_ctx_cleanup does when flint_cleanup runs
   (src/fft_small/default_ctx.c:19-27); the next default-context call makes
   a new one.  No-op when the thread has none. */
GPU_FFT_SMALL_API void gpu_default_mpn_ctx_cleanup(void);

/* Same signature and argument meaning as mpn_mul_default_mpn_ctx
   (src/fft_small.h:852): r1 = i1 * i2, n1 >= n2 >= 1. */
GPU_FFT_SMALL_API void gpu_mpn_mul_default_mpn_ctx(gpu_ulong *r1, const gpu_ulong *i1, gpu_slong n1,
                                 const gpu_ulong *i2, gpu_slong n2);

/* Same signature as _nmod_poly_mul_mid_default_mpn_ctx (src/fft_small.h:853). */
GPU_FFT_SMALL_API void _gpu_nmod_poly_mul_mid_default_mpn_ctx(gpu_ulong *res, gpu_slong zl, gpu_slong zh,
                                            const gpu_ulong *a, gpu_slong an,
                                            const gpu_ulong *b, gpu_slong bn,
                                            gpu_nmod_t mod);

/* --- precomputed transforms for nmod products and division (replaces
       mul_precomp_struct, _mul_precomp_init/_clear, _nmod_poly_mul_mid_precomp
       and the nmod_poly_divrem_precomp_* family, src/fft_small.h:796-848,
       src/fft_small/nmod_poly_mul.c:1054-1320) --------------------------- */

/* b's forward transforms of length 2^depth (at least 32) for one modulus,
   kept in device memory; bn and btrunc are recorded as in the reference
   (the GPU transforms at full length).  Operands longer than the transform
   are folded mod x^M - 1 and mod n, so every cyclic coefficient sums at most
   M products: the prime count is chosen for M (n - 1)^2 once. */
typedef struct {
    void *impl;
    gpu_ulong bn;
    gpu_ulong btrunc;
    gpu_ulong depth;   /* log2 of the transform length actually used */
} gpu_mul_precomp_struct;

/* As _mul_precomp_init (src/fft_small.h:803-808): b on the host, reduced mod
   n; depth <= 25.  Returns 0, GPU_FFT_SMALL_EINVAL, _ETOOBIG, _ENOPRIMES or
   _ECUDA; the void form raises through the error handler. */
GPU_FFT_SMALL_API int gpu_mul_precomp_init_status(gpu_mul_precomp_struct *M, const gpu_ulong *b, gpu_ulong bn,
                                                  gpu_ulong btrunc, gpu_ulong depth, gpu_nmod_t mod,
                                                  gpu_mpn_ctx_t R);
GPU_FFT_SMALL_API void _gpu_mul_precomp_init(gpu_mul_precomp_struct *M, const gpu_ulong *b, gpu_ulong bn,
                                             gpu_ulong btrunc, gpu_ulong depth, gpu_nmod_t mod, gpu_mpn_ctx_t R);
/* As _mul_precomp_clear (src/fft_small.h:810-814). */
GPU_FFT_SMALL_API void _gpu_mul_precomp_clear(gpu_mul_precomp_struct *M);
/* As _nmod_poly_mul_mid_precomp (src/fft_small.h:816-822): z = coefficients
   [zl, zh) of a b mod n (zero beyond an + bn - 1), host pointers; returns 1,
   or 0 when the window does not fit the transform without wrap-around
   (zh > 2^depth or an + bn - 1 - zl > 2^depth), as the reference's
   _fft_small_plan_fit_window refusal; other errors raise. */
GPU_FFT_SMALL_API int _gpu_nmod_poly_mul_mid_precomp(gpu_ulong *z, gpu_ulong zl, gpu_ulong zh,
                                                     const gpu_ulong *a, gpu_ulong an, gpu_mul_precomp_struct *M,
                                                     gpu_nmod_t mod, gpu_mpn_ctx_t R);
/* Device-pointer form queued on `stream`: 0, or GPU_FFT_SMALL_ETOOBIG when
   the window does not fit. */
GPU_FFT_SMALL_API int gpu_nmod_poly_mul_mid_precomp_device(uint64_t *z, gpu_ulong zl, gpu_ulong zh,
                                                           const uint64_t *a, gpu_ulong an,
                                                           gpu_mul_precomp_struct *M, void *stream);

typedef struct {
    gpu_mul_precomp_struct quo_maker[1];   /* rev(rev(b)^-1 mod x^Bn), 2^depth >= 2 Bn - 1 */
    gpu_mul_precomp_struct rem_maker[1];   /* b, 2^depth = N >= bn - 1 */
} gpu_nmod_poly_divrem_precomp_struct;

/* As _nmod_poly_divrem_precomp_init (src/fft_small.h:834-840): the inverse
   series of the reversed divisor to precision Bn (device Newton iteration)
   and both transforms.  b's leading coefficient must be a unit mod n. */
GPU_FFT_SMALL_API int _gpu_nmod_poly_divrem_precomp_init_status(gpu_nmod_poly_divrem_precomp_struct *M,
                                                                const gpu_ulong *b, gpu_ulong bn, gpu_ulong Bn,
                                                                gpu_nmod_t mod, gpu_mpn_ctx_t R);
GPU_FFT_SMALL_API void _gpu_nmod_poly_divrem_precomp_init(gpu_nmod_poly_divrem_precomp_struct *M,
                                                          const gpu_ulong *b, gpu_ulong bn, gpu_ulong Bn,
                                                          gpu_nmod_t mod, gpu_mpn_ctx_t R);
/* As _nmod_poly_divrem_precomp (src/fft_small.h:842-848): a = q b + r with
   q of an - bn + 1 and r of bn - 1 coefficients, host pointers; returns 1, or
   0 when the quotient is longer than the precision Bn. */
GPU_FFT_SMALL_API int _gpu_nmod_poly_divrem_precomp(gpu_ulong *q, gpu_ulong *r, const gpu_ulong *a, gpu_ulong an,
                                                    gpu_nmod_poly_divrem_precomp_struct *M, gpu_nmod_t mod,
                                                    gpu_mpn_ctx_t R);
/* Device-pointer form queued on `stream`: 0, or GPU_FFT_SMALL_ETOOBIG when
   the quotient is longer than Bn. */
GPU_FFT_SMALL_API int gpu_nmod_poly_divrem_precomp_device(uint64_t *q, uint64_t *r, const uint64_t *a,
                                                          gpu_ulong an, gpu_nmod_poly_divrem_precomp_struct *M,
                                                          void *stream);
/* As _nmod_poly_divrem_precomp_clear (src/fft_small.h:828-832). */
GPU_FFT_SMALL_API void _gpu_nmod_poly_divrem_precomp_clear(gpu_nmod_poly_divrem_precomp_struct *M);

/* --- negacyclic products mod 2^N + 1 (replaces src/fft_small/negacyclic.c,
       the pointwise engine of Schoenhage-Strassen convolutions) ------------ */

/* Operands and results are n + 1 limbs, N = 64 n: the n low limbs and a top
   limb that is 0 or 1 (inputs may be unreduced below 2^(N+1), as in the
   reference, negacyclic.c:288-290); results are the unique representative in
   [0, 2^N], top limb 1 only for 2^N itself.  A context fixes N and the digit
   split N = m b; it uses (and must not outlive) an mpn context. */
typedef struct { void *impl; } gpu_mulmod_2expp1_ctx_struct;
typedef gpu_mulmod_2expp1_ctx_struct gpu_mulmod_2expp1_ctx_t[1];

/* As sd_fft_mpn_mulmod_2expp1_ctx_init (src/fft_small.h:908, negacyclic.c:
   65-175): N a positive multiple of 64, m a power of two >= 16 dividing N,
   or 0 to let the context choose.  The digit count actually used is a power
   of two in [32, 2^14]: a request outside that range is moved into it by
   doubling or halving the digit size, and a request whose digits are too
   wide for six 31-bit primes takes more, narrower digits.  The product does
   not depend on the split.
   Returns 0, GPU_FFT_SMALL_EINVAL or GPU_FFT_SMALL_ENOPRIMES (no split fits
   six 31-bit primes: 2 b + log2 m + 2 must stay below their ~183 bits). */
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_ctx_init_status(gpu_mulmod_2expp1_ctx_struct *C, gpu_mpn_ctx_t R,
                                                         gpu_slong N, gpu_slong m);
/* Same, raising errors through the error handler (the reference throws). */
GPU_FFT_SMALL_API void gpu_mulmod_2expp1_ctx_init(gpu_mulmod_2expp1_ctx_struct *C, gpu_mpn_ctx_t R,
                                                  gpu_slong N, gpu_slong m);
/* As sd_fft_mpn_mulmod_2expp1_ctx_clear (src/fft_small.h:910). */
GPU_FFT_SMALL_API void gpu_mulmod_2expp1_ctx_clear(gpu_mulmod_2expp1_ctx_struct *C);
/* The context's N, digit count m, digit bits b and prime count (the fields
   C->N, C->m, C->b, C->np of the reference's context struct). */
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_ctx_info(const gpu_mulmod_2expp1_ctx_struct *C, gpu_slong *N,
                                                 gpu_slong *m, gpu_slong *b, gpu_slong *np);
/* As sd_fft_mpn_mulmod_2expp1_choose_np (src/fft_small.h:907) over this
   library's primes: the fewest that hold the biased coefficient bound
   2^(2 b + depth + 1) with one bit to spare; -1 when six do not. */
GPU_FFT_SMALL_API gpu_slong gpu_mulmod_2expp1_choose_np(gpu_slong b, gpu_slong depth);
/* As sd_fft_mpn_mulmod_2expp1 (src/fft_small.h:911): z = x y mod 2^N + 1,
   host pointers.  The reference's scratch argument has no counterpart (the
   context owns its device buffers; a context is not reentrant). */
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_status(const gpu_mulmod_2expp1_ctx_struct *C, gpu_ulong *z,
                                               const gpu_ulong *x, const gpu_ulong *y);
GPU_FFT_SMALL_API void gpu_mulmod_2expp1(const gpu_mulmod_2expp1_ctx_struct *C, gpu_ulong *z,
                                         const gpu_ulong *x, const gpu_ulong *y);
/* Batched device form (the pointwise stage of one convolution in one call):
   z_i = x_i y_i mod 2^N + 1 for i < count, operand i at x + i stride (stride
   >= n + 1 limbs), all device pointers, queued on `stream`.  x == y squares. */
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_batch_device(const gpu_mulmod_2expp1_ctx_struct *C, uint64_t *z,
                                                     const uint64_t *x, const uint64_t *y,
                                                     gpu_ulong count, gpu_ulong stride, void *stream);
/* Staged form (sd_fft_mpn_mulmod_2expp1_transformed_size / _transform /
   _mul_cached, src/fft_small.h:916-923): the transforms of `count` operands
   take gpu_mulmod_2expp1_transformed_size(C, count) 32-bit words of device
   memory; mul_cached multiplies operand i of x by cached transform i and
   must be given the same count as the transform call that filled F (the
   layout depends on it). */
GPU_FFT_SMALL_API gpu_slong gpu_mulmod_2expp1_transformed_size(const gpu_mulmod_2expp1_ctx_struct *C,
                                                               gpu_ulong count);
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_transform_device(const gpu_mulmod_2expp1_ctx_struct *C, uint32_t *F,
                                                         const uint64_t *y, gpu_ulong count,
                                                         gpu_ulong stride, void *stream);
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_mul_cached_device(const gpu_mulmod_2expp1_ctx_struct *C, uint64_t *z,
                                                          const uint64_t *x, const uint32_t *F,
                                                          gpu_ulong count, gpu_ulong stride, void *stream);
/* One-operand host forms of the staged pair; F is device memory of
   gpu_mulmod_2expp1_transformed_size(C, 1) words. */
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_transform(const gpu_mulmod_2expp1_ctx_struct *C, uint32_t *F,
                                                  const gpu_ulong *y);
GPU_FFT_SMALL_API int gpu_mulmod_2expp1_mul_cached(const gpu_mulmod_2expp1_ctx_struct *C, gpu_ulong *z,
                                                   const gpu_ulong *x, const uint32_t *F);

/* --- explicit schedules (no counterpart in the reference; its counterpart
       is the profile choice of mpn_ctx_best_profile, src/fft_small/mpn_mul.c:
       1248-1340, which is internal) --------------------------------------- */

#define GPU_MUL_ROUTE_NTT       0   /* number-theoretic transform */
#define GPU_MUL_ROUTE_BASECASE  1   /* schoolbook; shorter operand <= 4096 limbs
                                       (<= 1024 in a planned batch) */

/* How one product is computed.  Zero fields take the default: the fewest
   primes that hold the coefficient bound, the shortest transform that holds
   the product, rows of 2^logM points up to 2^13, 32-point columns from 2^14
   to 2^17 points, 64-point columns at 2^18, 2^13-point rows from 2^19 to
   2^24 points, 2^14 at 2^25.  Any valid choice gives the same (exact)
   product; only the time differs. */
typedef struct {
    int route;   /* GPU_MUL_ROUTE_* */
    int np;      /* primes, minimal .. 6 */
    int logM;    /* transform length 2^logM, minimal .. 2^25 */
    int logC;    /* four-step row length 2^logC, max(5, logM - 11) .. min(logM, 14); below
                    2^14 points at most 16 columns (logC >= logM - 4) */
    int flags;   /* GPU_MUL_FLAG_*: 0 = one transform of 2^logM points */
} gpu_mul_config;
/* flags of a transform configuration (whole products on device pointers,
   gpu_mpn_mul_device_config and the per-instance list; planned batches take
   flags = 0):
   THREE: run a transform of 3 2^(logM - 2) points (valid when the product
     fits it, five primes, 2^18 <= 3 2^(logM - 2) / 3 <= 2^23; rows of 2^13);
     also the one flag integer-polynomial products take (their chunk product
     must fit it), and both kinds take that length by default, without a
     configuration, where it fits;
   SPLIT: run the product as chunks of the long operand against one
     transform of the short one, chunk length by the default rule (valid when
     that rule splits the product);
   ROWS16 / ROWS32: the row pass with 16 / 32 points per thread (ROWS16
     needs rows of 2^9 points or more, and neither THREE nor SPLIT).
     Without either the launch takes 16 where 32 would leave it fewer than
     16 warps per SM. */
#define GPU_MUL_FLAG_THREE 1
#define GPU_MUL_FLAG_SPLIT 2
#define GPU_MUL_FLAG_ROWS16 4
#define GPU_MUL_FLAG_ROWS32 8

/* Fills the zero fields of cfg with the defaults for an an x bn product and
   checks the rest; returns 0 or GPU_FFT_SMALL_EINVAL naming the bad field. */
GPU_FFT_SMALL_API int gpu_mpn_mul_config_resolve(gpu_ulong an, gpu_ulong bn, gpu_mul_config *cfg);
/* gpu_mpn_mul_device under an explicit configuration (NULL = default). */
GPU_FFT_SMALL_API int gpu_mpn_mul_device_config(gpu_mpn_ctx_t R, uint64_t *z_dev, const uint64_t *a_dev,
                                                gpu_ulong an, const uint64_t *b_dev, gpu_ulong bn,
                                                const gpu_mul_config *cfg, void *stream);

/* The configuration the reference's own profile choice would make
   (mpn_ctx_best_profile, src/fft_small/mpn_mul.c:1248-1340, ported to this
   configuration space): among single transforms with the longest rows --
   the fewest primes or one more, the shortest power-of-two length or the
   3 2^k length where the product fits it -- the least score
   (1 - ratio / 4) np depth L_t (L_t the transform's points,
   depth = ceil(log2 L_t), ratio = L_t / 2^depth).  kind 0: an x bn limbs
   (aw, bw ignored); kind 1: integer polynomials of aw- and bw-limb
   coefficients.  The autotuner's "method without the model" baseline. */
GPU_FFT_SMALL_API int gpu_mul_reference_rule(int kind, gpu_ulong an, gpu_ulong aw, gpu_ulong bn,
                                             gpu_ulong bw, gpu_mul_config *cfg);

/* Integer-polynomial counterparts (raw coefficient rows, transform route;
   the window must lie inside the product). */
GPU_FFT_SMALL_API int gpu_fmpz_poly_mul_config_resolve(gpu_ulong an, gpu_ulong aw, gpu_ulong bn,
                                                       gpu_ulong bw, gpu_mul_config *cfg);
GPU_FFT_SMALL_API int gpu_fmpz_poly_mul_mid_device_config(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong zw,
                                                          gpu_ulong zl, gpu_ulong zh,
                                                          const uint64_t *a_dev, gpu_ulong aw,
                                                          gpu_ulong an, const uint64_t *b_dev,
                                                          gpu_ulong bw, gpu_ulong bn,
                                                          const gpu_mul_config *cfg, void *stream);

/* A list of integer-polynomial products queued by one call (no counterpart
   in the reference, whose callers multiply one polynomial pair per
   _fmpz_poly_mul call, src/fmpz_poly/mul.c:100-186): coefficients [zl, zh)
   of a * b into z (zh - zl rows of zw limbs), raw two's complement rows as
   for gpu_fmpz_poly_mul_mid_device_config, all device pointers.  Every
   request is planned first (any invalid one fails the call before anything
   is queued; the message names its index), the context's scratch is sized
   once for the largest, and the products are queued in order on `stream`
   without a host synchronisation.  cfgs: NULL or one configuration per
   request.  Requests run one after another on the stream, so they may share
   operands but must not write overlapping z. */
typedef struct {
    uint64_t *z;
    gpu_ulong zw, zl, zh;
    const uint64_t *a;
    gpu_ulong aw, an;
    const uint64_t *b;
    gpu_ulong bw, bn;
} gpu_fmpz_mul_req;
GPU_FFT_SMALL_API int gpu_fmpz_poly_mul_mid_device_list(gpu_mpn_ctx_t R, const gpu_fmpz_mul_req *reqs,
                                                        size_t n, const gpu_mul_config *cfgs,
                                                        void *stream);

/* Test hooks for the failure paths of the bounded device waits, which valid
   inputs do not reach (no counterpart in the reference).
   gpu_test_crt_lookback_timeout runs one CRT/carry tile whose carry
   look-back waits for a predecessor that never publishes its status, so the
   wait runs out (a few seconds) and the kernel sets the context's error
   flag and finishes; returns the status the host reads back
   (GPU_FFT_SMALL_ETIMEOUT) and leaves the context usable.
   gpu_test_set_device_error sets the error flag as such a kernel would: the
   next host-pointer product on the context returns GPU_FFT_SMALL_ETIMEOUT
   and clears it.  gpu_test_pipe_slot_ctx returns the context behind slot
   `slot` of a pipeline (the impl of a gpu_mpn_ctx_t), or NULL. */
GPU_FFT_SMALL_API int gpu_test_crt_lookback_timeout(gpu_mpn_ctx_t R);
GPU_FFT_SMALL_API int gpu_test_set_device_error(gpu_mpn_ctx_t R);
GPU_FFT_SMALL_API void *gpu_test_pipe_slot_ctx(gpu_mpn_pipe_t P, int slot);

/* Integer-pipe calibration (no counterpart in the reference): the rate, in
   butterflies per second, of the transforms' 31-bit modular butterfly run
   from registers only on every SM (median of five timed launches of about a
   millisecond on the context's stream).  The product kernels' compute
   roofline: a product of transform length M with np primes and two forward
   and one inverse transform performs 3 log2(M) M/2 np butterflies. */
GPU_FFT_SMALL_API int gpu_butterfly_rate(gpu_mpn_ctx_t R, double *per_s);

/* Autotuner measurement: median device time (CUDA events on the context's
   stream, after one warm-up call) of `reps` products under cfg, on operands
   filled on the device from a fixed seed.  kind 0: an x bn-limb mpn product
   (aw, bw ignored); kind 1: integer polynomials of an and bn coefficients of
   aw and bw limbs (full product).  Returns 0 and *ms, or an error code. */
GPU_FFT_SMALL_API int gpu_mul_time_config(gpu_mpn_ctx_t R, int kind, gpu_ulong an, gpu_ulong aw,
                                          gpu_ulong bn, gpu_ulong bw, const gpu_mul_config *cfg,
                                          int reps, double *ms);

/* The same for products inside a batch: `copies` an x bn products of one
   configuration run as one planned batch (gpu_mpn_batch_*, graph replay);
   *ms_per_product = median batch time / copies, the marginal cost of a
   product in batched execution. */
GPU_FFT_SMALL_API int gpu_mpn_mul_time_batched(gpu_mpn_ctx_t R, gpu_ulong an, gpu_ulong bn,
                                               const gpu_mul_config *cfg, int copies, int reps,
                                               double *ms_per_product);

/* --- cost model of the learned schedule (no counterpart in the reference) --

   A fully connected network n_in -> 64 -> 64 -> 64 -> 1 (ReLU, fp32) that
   predicts log device time from request features and a candidate
   gpu_mul_config; trained and evaluated by the library's own CUDA kernels on
   the current device.  Host-pointer arguments unless named _dev.  The
   parameter vector is W1[n_in][64], b1[64], W2[64][64], b2[64], W3[64][64],
   b3[64], W4[64], b4. */
typedef struct gpu_mlp_struct *gpu_mlp_t;

/* He-uniform weights from a splitmix64 stream seeded with `seed`, zero
   biases; 1 <= n_in <= 32. */
GPU_FFT_SMALL_API int gpu_mlp_init(gpu_mlp_t *M, int n_in, unsigned long long seed);
GPU_FFT_SMALL_API int gpu_mlp_nparams(gpu_mlp_t M);
GPU_FFT_SMALL_API int gpu_mlp_get_params(gpu_mlp_t M, float *params, size_t n);
/* Replaces the parameters and resets the optimiser state. */
GPU_FFT_SMALL_API int gpu_mlp_set_params(gpu_mlp_t M, const float *params, size_t n);
/* y[s] = network(X[s][0 .. n_in)) for s < n. */
GPU_FFT_SMALL_API int gpu_mlp_predict(gpu_mlp_t M, const float *X, int n, float *y);
GPU_FFT_SMALL_API int gpu_mlp_predict_device(gpu_mlp_t M, const float *X_dev, int n, float *y_dev,
                                             void *stream);
/* Gradient of the mean squared error (1/n) sum (y_s - t_s)^2 with respect to
   the parameters (deterministic summation order), and the loss. */
GPU_FFT_SMALL_API int gpu_mlp_gradient(gpu_mlp_t M, const float *X, const float *t, int n,
                                       float *grad, float *loss);
/* Adam (lr, 0.9, 0.999, 1e-8) on minibatches of `batch` samples, reshuffled
   every epoch from a splitmix64 stream seeded with `seed`; final_loss (may be
   NULL) receives the full-batch loss after training. */
GPU_FFT_SMALL_API int gpu_mlp_train(gpu_mlp_t M, const float *X, const float *t, int n, int epochs,
                                    int batch, float lr, unsigned long long seed, float *final_loss);
GPU_FFT_SMALL_API void gpu_mlp_clear(gpu_mlp_t M);

/* --- integer polynomials ---------------------------------------------------

   Coefficients [zl, zh) of the product of integer polynomials a (an
   coefficients) and b (bn).  Beyond an + bn - 1 the window is zero-filled.
   Any coefficient size is handled (chunked Kronecker layout on 64-bit limbs);
   the limits are a chunk-product length (an + bn - 1)(wa + wb - 1) <= 2^25 and
   min(an,bn) min(wa,wb) < 2^53. */

/* Same signature as _fmpz_poly_mul_mid_mpn_ctx (src/fft_small.h:856-860).
   fmpz is FLINT's tagged word (src/flint.h.in:467-477); inputs may hold
   inline values or mpz pointers.  Output coefficients are written through
   the setter registered with gpu_fmpz_set_signed_hook (FLINT's
   fmpz_set_signed_ui_array, src/fmpz.h:239, is the intended one); without a
   setter only inline results into inline entries are possible and anything
   else is an error.  Returns 1 on success and 0 when the product is beyond
   the prime set or the transform length (the caller falls back, as
   _fmpz_poly_mul does in src/fmpz_poly/mul.c:122-126); other failures go to
   the throw handler. */
GPU_FFT_SMALL_API int _gpu_fmpz_poly_mul_mid_mpn_ctx(gpu_slong *z, gpu_ulong zl, gpu_ulong zh,
                                                     const gpu_slong *a, gpu_ulong an,
                                                     const gpu_slong *b, gpu_ulong bn,
                                                     gpu_mpn_ctx_t R);
/* Same signature as _fmpz_poly_mul_mid_default_mpn_ctx (src/fft_small.h:862-865). */
GPU_FFT_SMALL_API int _gpu_fmpz_poly_mul_mid_default_mpn_ctx(gpu_slong *z, gpu_slong zl, gpu_slong zh,
                                                             const gpu_slong *a, gpu_slong an,
                                                             const gpu_slong *b, gpu_slong bn);
/* Output setter for the fmpz entry points: set *f to the n-limb two's
   complement value at limbs (NULL unregisters). */
GPU_FFT_SMALL_API void gpu_fmpz_set_signed_hook(void (*set_signed)(gpu_slong *f, const gpu_ulong *limbs,
                                                                   gpu_slong n));

/* Raw form (no counterpart in the reference; the fmpz entry points run on
   it): each coefficient is a fixed number of 64-bit limbs in two's
   complement -- aw for a, bw for b, zw for the result (zw must hold every
   result coefficient: zw >= (bits(a) + bits(b) + ceil(log2 min(an,bn)) + 1)
   / 64 rounded up; wider is sign-extended).  Host pointers; returns 0 or a
   GPU_FFT_SMALL_E* code (ENOPRIMES / ETOOBIG beyond the limits above). */
GPU_FFT_SMALL_API int _gpu_fmpz_poly_mul_mid_raw(gpu_ulong *z, gpu_ulong zw, gpu_ulong zl, gpu_ulong zh,
                                                 const gpu_ulong *a, gpu_ulong aw, gpu_ulong an,
                                                 const gpu_ulong *b, gpu_ulong bw, gpu_ulong bn,
                                                 gpu_mpn_ctx_t R);
/* Device-pointer twin of the raw form, queued on `stream`. */
GPU_FFT_SMALL_API int gpu_fmpz_poly_mul_mid_device(gpu_mpn_ctx_t R, uint64_t *z_dev, gpu_ulong zw,
                                                   gpu_ulong zl, gpu_ulong zh,
                                                   const uint64_t *a_dev, gpu_ulong aw, gpu_ulong an,
                                                   const uint64_t *b_dev, gpu_ulong bw, gpu_ulong bn,
                                                   void *stream);

/* --- plans and transformed operands ------------------------------------------

   The reference's plan / op API (src/fft_small.h:466-700, src/fft_small/op.c):
   a plan fixes the primes, the transform length and the output window; an
   op holds one operand's forward transforms, resident in device memory
   (np vectors of 2^logM words), so an operand transformed once can be
   combined with many others.  Forward transforms are in the PRIMAL domain;
   mul / sqr / addmul / submul produce the PRODUCT domain (normalisation
   folded in once); add / sub need both operands in the same domain.  All
   data pointers are device pointers and every call is queued on `stream`
   (NULL = CUDA's default stream); gpu_fft_op_check synchronises and
   reports a kernel error. */
typedef struct gpu_fft_plan_struct *gpu_fft_plan_t;
typedef struct gpu_fft_op_struct *gpu_fft_op_t;

#define GPU_FFT_OP_MUL     0   /* Z = A B         */
#define GPU_FFT_OP_SQR     1   /* Z = A^2         */
#define GPU_FFT_OP_ADDMUL  2   /* Z = Z + A B     */
#define GPU_FFT_OP_SUBMUL  3   /* Z = Z - A B     */
#define GPU_FFT_OP_ADD     4   /* Z = A + B       */
#define GPU_FFT_OP_SUB     5   /* Z = A - B       */
#define GPU_FFT_OP_NEG     6   /* Z = -A          */

/* fft_small_plan_init_mpn (src/fft_small.h:577-579): integer operands of at
   most an_max and bn_max limbs, at most len_bound elementary products
   accumulated per coefficient; is_signed adds the reference's spare factor
   two.  Returns 0, GPU_FFT_SMALL_ENOPRIMES or GPU_FFT_SMALL_ETOOBIG. */
GPU_FFT_SMALL_API int gpu_fft_plan_init_mpn(gpu_fft_plan_t *P, gpu_mpn_ctx_t R, gpu_ulong an_max,
                                            gpu_ulong bn_max, gpu_ulong len_bound, int is_signed);
/* fft_small_plan_init_nmod (src/fft_small.h:559-561): the window [zl, zh) of
   a length-zn convolution over Z/nZ, len_bound products of absolute value
   below 2^prod_bits per output coefficient. */
GPU_FFT_SMALL_API int gpu_fft_plan_init_nmod(gpu_fft_plan_t *P, gpu_mpn_ctx_t R, gpu_ulong zl, gpu_ulong zh,
                                             gpu_ulong zn, gpu_ulong len_bound, gpu_ulong prod_bits,
                                             gpu_nmod_t mod);
/* fft_small_plan_init_mpn_np (src/fft_small.h:587-589): as
   gpu_fft_plan_init_mpn with the prime count forced (np = 0: the automatic
   choice; otherwise np primes if they hold the bound, else
   GPU_FFT_SMALL_ENOPRIMES; the reference's two-prime geometry does not exist
   here, 64-bit coefficients need five primes). */
GPU_FFT_SMALL_API int gpu_fft_plan_init_mpn_np(gpu_fft_plan_t *P, gpu_mpn_ctx_t R, gpu_ulong an_max,
                                               gpu_ulong bn_max, gpu_ulong len_bound, int is_signed, int np);
/* fft_small_plan_init_nmod_cyclic (src/fft_small.h:591-593): convolutions
   mod x^N - 1, N = 2^depth (5 <= depth <= 25), output coefficients [0, zh).
   Operands longer than N are folded mod x^N - 1 and mod n by the forward
   transform. */
GPU_FFT_SMALL_API int gpu_fft_plan_init_nmod_cyclic(gpu_fft_plan_t *P, gpu_mpn_ctx_t R, gpu_ulong depth,
                                                    gpu_ulong zh, gpu_ulong len_bound, gpu_ulong prod_bits,
                                                    gpu_nmod_t mod);
/* fft_small_plan_init_mpn_cyclic (src/fft_small.h:600-601): products of
   integers of at most *nn limbs mod 2^(64 *nn) - 1, *nn rounded up to a
   power of two (at least 32) and written back.  gpu_fft_export_mpn gives
   the non-negative sum of the coefficients (below len_bound 2^(64 nn + 128 +
   log2 nn)); export at least nn + 3 limbs and fold the top limbs back. */
GPU_FFT_SMALL_API int gpu_fft_plan_init_mpn_cyclic(gpu_fft_plan_t *P, gpu_mpn_ctx_t R, gpu_ulong *nn,
                                                   gpu_ulong len_bound);
GPU_FFT_SMALL_API int gpu_fft_plan_info(gpu_fft_plan_t P, int *np, int *logM);
GPU_FFT_SMALL_API void gpu_fft_plan_clear(gpu_fft_plan_t P);
/* fft_small_op_init / fft_small_op_clear */
GPU_FFT_SMALL_API int gpu_fft_op_init(gpu_fft_op_t *X, gpu_fft_plan_t P);
GPU_FFT_SMALL_API void gpu_fft_op_clear(gpu_fft_op_t X);
/* fft_small_op_sizeof_data / fft_small_op_init_borrowed (src/fft_small.h:
   636-638): an operand in caller-provided device memory of
   gpu_fft_op_sizeof_data(P) bytes (16-byte aligned, outliving the operand;
   gpu_fft_op_clear does not free it). */
GPU_FFT_SMALL_API gpu_ulong gpu_fft_op_sizeof_data(gpu_fft_plan_t P);
GPU_FFT_SMALL_API int gpu_fft_op_init_borrowed(gpu_fft_op_t *X, gpu_fft_plan_t P, void *data_dev);
/* fft_small_fft_mpn / fft_small_fft_nmod: forward transforms of a (an limbs
   or coefficients; nmod coefficients reduced mod n) into X */
GPU_FFT_SMALL_API int gpu_fft_fft_mpn(gpu_fft_op_t X, const uint64_t *a_dev, gpu_ulong an,
                                      gpu_fft_plan_t P, void *stream);
GPU_FFT_SMALL_API int gpu_fft_fft_nmod(gpu_fft_op_t X, const uint64_t *a_dev, gpu_ulong an,
                                       gpu_fft_plan_t P, void *stream);
/* fft_small_op_mul / _sqr / _addmul / _submul / _add / _sub / _neg
   (op = GPU_FFT_OP_*; B is ignored by SQR and NEG; Z may alias A or B) */
GPU_FFT_SMALL_API int gpu_fft_op_pointwise(int op, gpu_fft_op_t Z, gpu_fft_op_t A, gpu_fft_op_t B,
                                           gpu_fft_plan_t P, void *stream);
/* fft_small_ifft: inverse transform in place */
GPU_FFT_SMALL_API int gpu_fft_ifft(gpu_fft_op_t X, gpu_fft_plan_t P, void *stream);
/* fft_small_export_mpn: the low zn limbs of the accumulated integer
   (reduced mod 2^(64 zn) if it does not fit) */
GPU_FFT_SMALL_API int gpu_fft_export_mpn(uint64_t *z_dev, gpu_ulong zn, gpu_fft_op_t X, gpu_fft_plan_t P,
                                         void *stream);
/* fft_small_export_nmod_range: coefficients [zl, zh) mod n (inside the plan's
   window) */
GPU_FFT_SMALL_API int gpu_fft_export_nmod(uint64_t *z_dev, gpu_ulong zl, gpu_ulong zh, gpu_fft_op_t X,
                                          gpu_nmod_t mod, gpu_fft_plan_t P, void *stream);
/* fft_small_export_mpn_signed / _signed_trunc (src/fft_small.h:681-686):
   the value sum_(j < nslots) c_j 2^(64 j) with every coefficient c_j in the
   centered range (-P/2, P/2] (plans made with is_signed keep true values in
   it); z receives limbs [lo_limbs, lo_limbs + zn) of its absolute value and
   *sign its sign (0 when those limbs are zero).  lo_limbs + zn must be at
   least nslots + 3 so that the sign is inside.  The window is exact (the
   reference's truncated form may drop carries from below it).  Synchronises
   `stream` to return the sign. */
GPU_FFT_SMALL_API int gpu_fft_export_mpn_signed(uint64_t *z_dev, gpu_ulong zn, int *sign, gpu_fft_op_t X,
                                                gpu_ulong nslots, gpu_fft_plan_t P, void *stream);
GPU_FFT_SMALL_API int gpu_fft_export_mpn_signed_trunc(uint64_t *z_dev, gpu_ulong zn, int *sign, gpu_fft_op_t X,
                                                      gpu_ulong nslots, gpu_ulong lo_limbs, gpu_fft_plan_t P,
                                                      void *stream);
/* Synchronises `stream`; GPU_FFT_SMALL_ETIMEOUT if a carry wait gave up. */
GPU_FFT_SMALL_API int gpu_fft_op_check(gpu_fft_plan_t P, void *stream);

/* --- batches of uneven products (no counterpart in the reference, which
       multiplies one product per mpn_ctx_mpn_mul call, src/fft_small.h:433) */

/* One product of a batch: z[0 .. an+bn) = a * b, all device pointers.  The
   same rules as gpu_mpn_mul_device hold per product (no aliasing of z with
   a or b; distinct products write disjoint z). */
typedef struct {
    gpu_ulong *z;
    const gpu_ulong *a;
    gpu_ulong an;
    const gpu_ulong *b;
    gpu_ulong bn;
} gpu_mpn_mul_req;

/* A list of products queued by one call (no counterpart in the reference):
   each request runs as gpu_mpn_mul_device would run it (its own launches,
   under cfgs[i] when cfgs is not NULL), one after another on `stream`,
   without a host synchronisation; every request is planned and the context's
   scratch sized for the largest before anything is queued (an invalid
   request fails the call, naming its index).  The per-product counterpart
   of a planned batch, without its class merging or graph. */
GPU_FFT_SMALL_API int gpu_mpn_mul_device_list(gpu_mpn_ctx_t R, const gpu_mpn_mul_req *reqs, size_t n,
                                              const gpu_mul_config *cfgs, void *stream);

/* Schedule of a batch.  promote_small: products whose (primes, transform
   length) class holds fewer than this many products are run at the next
   longer length together with that class (0 = off).  max_streams: classes run
   concurrently on up to this many streams (0 = 4).  use_graph: record the
   first run as a CUDA graph and replay it afterwards. */
typedef struct {
    int promote_small;
    int max_streams;
    int use_graph;
} gpu_mpn_batch_options;

typedef struct gpu_mpn_batch_struct *gpu_mpn_batch_t;

/* Plans a batch of n products over the context's device: groups them into
   classes, allocates their residue scratch and descriptors.  opt == NULL
   selects {0, 4, 1}.  The requests' pointers are captured; the operands may
   change between runs, the pointers may not.  Returns 0 on success. */
GPU_FFT_SMALL_API int gpu_mpn_batch_init(gpu_mpn_batch_t *B, gpu_mpn_ctx_t R,
                                         const gpu_mpn_mul_req *reqs, size_t n,
                                         const gpu_mpn_batch_options *opt);
/* gpu_mpn_batch_init with a configuration per request (cfgs[i] for reqs[i],
   see gpu_mul_config; NULL = defaults): products sharing a configuration run
   in the same launches. */
GPU_FFT_SMALL_API int gpu_mpn_batch_init_config(gpu_mpn_batch_t *B, gpu_mpn_ctx_t R,
                                                const gpu_mpn_mul_req *reqs, const gpu_mul_config *cfgs,
                                                size_t n, const gpu_mpn_batch_options *opt);
/* Queues every product of the batch on `stream` (NULL = CUDA's default
   stream) and returns without synchronising.  Runs of one batch must not
   overlap.  Kernel errors (a carry look-back that gave up) are reported by
   gpu_mpn_batch_check. */
GPU_FFT_SMALL_API int gpu_mpn_batch_run(gpu_mpn_batch_t B, void *stream);
/* Waits for `stream` and returns GPU_FFT_SMALL_ETIMEOUT if any kernel of the
   context recorded an error since the last check, else 0. */
GPU_FFT_SMALL_API int gpu_mpn_batch_check(gpu_mpn_batch_t B, void *stream);
/* Kernel launches of one run, and the number of (primes, length) classes. */
GPU_FFT_SMALL_API int gpu_mpn_batch_launches(gpu_mpn_batch_t B);
GPU_FFT_SMALL_API int gpu_mpn_batch_classes(gpu_mpn_batch_t B);
/* Waits for pending runs and frees the batch. */
GPU_FFT_SMALL_API void gpu_mpn_batch_clear(gpu_mpn_batch_t B);

/* --- error handling ------------------------------------------------------ */

/* Handler called by the void entry points on failure (the analogue of
   flint_set_throw); NULL restores the default print-and-abort. */
GPU_FFT_SMALL_API void gpu_fft_small_set_throw(void (*handler)(int code, const char *msg));
/* Message of the most recent failure on this host thread. */
GPU_FFT_SMALL_API const char *gpu_fft_small_last_error(void);

/* --- introspection (for tests and benchmarks) ----------------------------- */

/* Number of primes the GPU path would use and the transform length 2^logM
   for an an x bn product; returns 0 on success. */
GPU_FFT_SMALL_API int gpu_mpn_mul_plan(gpu_ulong an, gpu_ulong bn, int *np, int *logM);
/* For a whole non-squaring an x bn product under the default plan: the
   log2 transform length of the chunks it is split into (chunks of the long
   operand against one transform of the short one), or 0 when it runs as a
   single transform; returns 0 on success. */
GPU_FFT_SMALL_API int gpu_mpn_mul_split_plan(gpu_ulong an, gpu_ulong bn, int *chunk_logM);
/* Points of the cyclic transform a whole an x bn product (squaring when
   square != 0) runs under the default plan: 2^logM, or 3 2^(logM - 2) when
   the product fits that truncated length (the counterpart of the
   reference's transform truncation, src/fft_small/sd_fft.c:1230-1274), or
   the chunk transform of a split product; 0 for the basecase route.
   Returns 0 on success. */
GPU_FFT_SMALL_API int gpu_mpn_mul_transform_points(gpu_ulong an, gpu_ulong bn, int square,
                                                   gpu_ulong *points);
/* The i-th prime of the GPU prime set (0 if out of range). */
GPU_FFT_SMALL_API gpu_ulong gpu_fft_small_prime(int i);
/* Kernel launches issued by the most recent call on this context. */
GPU_FFT_SMALL_API int gpu_mpn_ctx_last_launches(gpu_mpn_ctx_t R);
/* Per-kernel device timing with CUDA events on the launching stream, off by
   default.  set_timing resets the totals; kernel_times returns the number of
   kernel slots filled (split+column pass, row pass, inverse column pass,
   CRT+carry) with total milliseconds and launch counts for each. */
GPU_FFT_SMALL_API int gpu_mpn_ctx_set_timing(gpu_mpn_ctx_t R, int on);
GPU_FFT_SMALL_API int gpu_mpn_ctx_kernel_times(gpu_mpn_ctx_t R, double *ms, long *count,
                                               int max);

#ifdef __cplusplus
}
#endif

#endif
