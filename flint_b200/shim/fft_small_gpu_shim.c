/* FLINT-side binding of the GPU small-prime NTT multiplication.
 *
 * Compiled against FLINT's headers (flint.h, fmpz.h, fft_small.h) and
 * include/gpu_fft_small.h, linked with libflint_b200.so.  Each function has
 * the signature of the fft_small entry point it replaces and forwards to the
 * GPU library's C ABI:
 *
 *   gpu_shim_mpn_ctx_mpn_mul               mpn_ctx_mpn_mul (src/fft_small.h:433)
 *   gpu_shim__mpn_ctx_mpn_mul_range        _mpn_ctx_mpn_mul_range (src/fft_small.h:462)
 *   gpu_shim__nmod_poly_mul_mid_mpn_ctx    _nmod_poly_mul_mid_mpn_ctx (src/fft_small.h:769-774)
 *   gpu_shim__fmpz_poly_mul_mid_mpn_ctx    _fmpz_poly_mul_mid_mpn_ctx (src/fft_small.h:856-860)
 *   gpu_shim__nmod_poly_divrem_mpn_ctx     _nmod_poly_divrem_mpn_ctx (src/fft_small.h:776-781)
 *
 * A FLINT build can select them with the preprocessor (for example
 * -Dmpn_ctx_mpn_mul=gpu_shim_mpn_ctx_mpn_mul for the translation units that
 * call the path), which is how the reference's own tests are run against the
 * GPU (oracle/build_ref_tests.py).  The FLINT context argument is accepted and
 * not used: the GPU path keeps one context of its own per host thread.
 * gpu_shim_init registers FLINT's exception handler and FLINT's fmpz setter
 * with the library; the wrappers call it on first use.
 */
#include "flint.h"
#include "fmpz.h"
#include "fft_small.h"
#include "gpu_fft_small.h"

static FLINT_TLS_PREFIX gpu_mpn_ctx_struct shim_ctx_store;
static FLINT_TLS_PREFIX int shim_ctx_ready = 0;
static int shim_hooks_ready = 0;

/* errors of the GPU path become FLINT exceptions */
static void shim_throw(int code, const char * msg)
{
    flint_throw(FLINT_ERROR, "gpu_fft_small (%d): %s\n", code, msg);
}

/* coefficients of integer-polynomial products are set by FLINT, which owns
   the allocation of any mpz they need */
static void shim_set_fmpz(gpu_slong * f, const gpu_ulong * limbs, gpu_slong n)
{
    fmpz_set_signed_ui_array((fmpz *) f, (const ulong *) limbs, n);
}

void gpu_shim_init(void)
{
    if (!shim_hooks_ready)
    {
        gpu_fft_small_set_throw(shim_throw);
        gpu_fmpz_set_signed_hook(shim_set_fmpz);
        shim_hooks_ready = 1;
    }
}

static gpu_mpn_ctx_struct * shim_ctx(void)
{
    if (!shim_ctx_ready)
    {
        gpu_shim_init();
        gpu_mpn_ctx_init(&shim_ctx_store, UWORD(0x0003f00000000001));
        shim_ctx_ready = 1;
    }
    return &shim_ctx_store;
}

void gpu_shim_mpn_ctx_mpn_mul(mpn_ctx_t R, ulong * z, const ulong * a, ulong an,
                              const ulong * b, ulong bn)
{
    (void) R;
    gpu_mpn_ctx_mpn_mul(shim_ctx(), z, a, an, b, bn);
}

void gpu_shim__mpn_ctx_mpn_mul_range(mpn_ctx_t R, ulong * z, ulong lo, ulong hi,
                                     const ulong * a, ulong an, const ulong * b, ulong bn)
{
    (void) R;
    _gpu_mpn_ctx_mpn_mul_range(shim_ctx(), z, lo, hi, a, an, b, bn);
}

void gpu_shim__nmod_poly_mul_mid_mpn_ctx(ulong * z, ulong zl, ulong zh, const ulong * a, ulong an,
                                         const ulong * b, ulong bn, nmod_t mod, mpn_ctx_t R)
{
    gpu_nmod_t gm;
    (void) R;
    gm.n = mod.n;
    gm.ninv = mod.ninv;
    gm.norm = mod.norm;
    _gpu_nmod_poly_mul_mid_mpn_ctx(z, zl, zh, a, an, b, bn, gm, shim_ctx());
}

int gpu_shim__fmpz_poly_mul_mid_mpn_ctx(fmpz * z, ulong zl, ulong zh, const fmpz * a, ulong an,
                                        const fmpz * b, ulong bn, mpn_ctx_t R)
{
    (void) R;
    return _gpu_fmpz_poly_mul_mid_mpn_ctx((gpu_slong *) z, zl, zh, (const gpu_slong *) a, an,
                                          (const gpu_slong *) b, bn, shim_ctx());
}

void gpu_shim__nmod_poly_divrem_mpn_ctx(ulong * q, ulong * r, const ulong * a, ulong an,
                                        const ulong * b, ulong bn, nmod_t mod, mpn_ctx_t R)
{
    gpu_nmod_t gm;
    (void) R;
    gm.n = mod.n;
    gm.ninv = mod.ninv;
    gm.norm = mod.norm;
    _gpu_nmod_poly_divrem_mpn_ctx(q, r, a, an, b, bn, gm, shim_ctx());
}
