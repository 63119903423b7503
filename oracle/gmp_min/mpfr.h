/*
    Minimal MPFR declarations for the oracle build of the reference (test
    infrastructure).  The reference memory manager calls mpfr_free_cache(),
    and fmpz/get.c defines a conversion to mpfr_t that nothing on the
    multiplication path calls; the type layout below is the one the MPFR
    manual documents ("Nomenclature and Types").  The recipe links the
    system libmpfr.so.6.
*/
#ifndef __MPFR_H
#define __MPFR_H
#include <gmp.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef long mpfr_prec_t;
typedef int mpfr_sign_t;
typedef long mpfr_exp_t;
typedef struct {
    mpfr_prec_t _mpfr_prec;
    mpfr_sign_t _mpfr_sign;
    mpfr_exp_t _mpfr_exp;
    mp_limb_t *_mpfr_d;
} __mpfr_struct;
typedef __mpfr_struct mpfr_t[1];
typedef __mpfr_struct *mpfr_ptr;
typedef const __mpfr_struct *mpfr_srcptr;
typedef enum { MPFR_RNDN = 0, MPFR_RNDZ, MPFR_RNDU, MPFR_RNDD, MPFR_RNDA } mpfr_rnd_t;
void mpfr_free_cache(void);
int mpfr_set_si_2exp(mpfr_ptr, long, mpfr_exp_t, mpfr_rnd_t);
#define mpfr_set_si(x, v, r) mpfr_set_si_2exp((x), (v), 0, (r))
int mpfr_set_z(mpfr_ptr, mpz_srcptr, mpfr_rnd_t);
#ifdef __cplusplus
}
#endif
#endif
