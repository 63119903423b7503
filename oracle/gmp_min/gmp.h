/*
    Minimal GMP declarations for building the reference FLINT closure that the
    oracle links against.  Written for this project from the public GMP manual
    ("GNU MP: The GNU Multiple Precision Arithmetic Library", chapters
    "Integer Functions", "Low-level Functions" and "Random Number Functions"):
    types, the documented structure layouts, and prototypes of the functions
    the compiled closure calls.  Linkage names follow the exported symbols of
    the system libgmp.so.10 (the public mpz_/mpn_ names are aliases of
    __gmpz_/__gmpn_ symbols there).

    This header is test infrastructure: it exists only so that the oracle build
    recipe (oracle/build_ref.py) can compile the reference sources without a
    libgmp-dev package.  Nothing in the product includes it.
*/
#ifndef __GMP_H__
#define __GMP_H__

#include <stddef.h>
#include <stdio.h>
#include <limits.h>

#ifdef __cplusplus
extern "C" {
#endif

#define __GNU_MP__ 6
#define __GNU_MP_VERSION 6
#define __GNU_MP_VERSION_MINOR 3
#define __GNU_MP_VERSION_PATCHLEVEL 0
#define __GNU_MP_RELEASE 60300

#define GMP_LIMB_BITS 64
#define GMP_NAIL_BITS 0
#define GMP_NUMB_BITS 64
#define GMP_NUMB_MASK (~(mp_limb_t) 0)
#define GMP_NUMB_MAX GMP_NUMB_MASK
#define GMP_NAIL_MASK 0

typedef unsigned long int mp_limb_t;
typedef long int mp_limb_signed_t;
typedef unsigned long int mp_bitcnt_t;
typedef long int mp_size_t;
typedef long int mp_exp_t;
typedef mp_limb_t *mp_ptr;
typedef const mp_limb_t *mp_srcptr;

/* documented layout: alloc, signed size (sign = sign of the integer), limbs */
typedef struct
{
    int _mp_alloc;
    int _mp_size;
    mp_limb_t *_mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;
typedef __mpz_struct MP_INT;

typedef struct
{
    __mpz_struct _mp_num;
    __mpz_struct _mp_den;
} __mpq_struct;

typedef __mpq_struct mpq_t[1];
typedef __mpq_struct *mpq_ptr;
typedef const __mpq_struct *mpq_srcptr;

typedef struct
{
    int _mp_prec;
    int _mp_size;
    mp_exp_t _mp_exp;
    mp_limb_t *_mp_d;
} __mpf_struct;

typedef __mpf_struct mpf_t[1];
typedef __mpf_struct *mpf_ptr;
typedef const __mpf_struct *mpf_srcptr;

typedef enum
{
    GMP_RAND_ALG_DEFAULT = 0,
    GMP_RAND_ALG_LC = GMP_RAND_ALG_DEFAULT
} gmp_randalg_t;

typedef struct
{
    mpz_t _mp_seed;
    gmp_randalg_t _mp_alg;
    union { void *_mp_lc; } _mp_algdata;
} __gmp_randstate_struct;

typedef __gmp_randstate_struct gmp_randstate_t[1];

extern const char * const __gmp_version;
#define gmp_version __gmp_version

/* ---- memory ---------------------------------------------------------- */
#define mp_set_memory_functions __gmp_set_memory_functions
void mp_set_memory_functions(void *(*)(size_t),
                             void *(*)(void *, size_t, size_t),
                             void (*)(void *, size_t));
#define mp_get_memory_functions __gmp_get_memory_functions
void mp_get_memory_functions(void *(**)(size_t),
                             void *(**)(void *, size_t, size_t),
                             void (**)(void *, size_t));

/* ---- random state ---------------------------------------------------- */
#define gmp_randinit_default __gmp_randinit_default
void gmp_randinit_default(gmp_randstate_t);
#define gmp_randseed_ui __gmp_randseed_ui
void gmp_randseed_ui(gmp_randstate_t, unsigned long int);
#define gmp_randclear __gmp_randclear
void gmp_randclear(gmp_randstate_t);

#define gmp_printf __gmp_printf
int gmp_printf(const char *, ...);
#define gmp_sprintf __gmp_sprintf
int gmp_sprintf(char *, const char *, ...);

/* ---- integers (mpz) -------------------------------------------------- */
#define mpz_init __gmpz_init
void mpz_init(mpz_ptr);
#define mpz_init2 __gmpz_init2
void mpz_init2(mpz_ptr, mp_bitcnt_t);
#define mpz_clear __gmpz_clear
void mpz_clear(mpz_ptr);
#define mpz_realloc __gmpz_realloc
void *mpz_realloc(mpz_ptr, mp_size_t);
#define _mpz_realloc __gmpz_realloc
#define mpz_realloc2 __gmpz_realloc2
void mpz_realloc2(mpz_ptr, mp_bitcnt_t);
#define mpz_set __gmpz_set
void mpz_set(mpz_ptr, mpz_srcptr);
#define mpz_set_ui __gmpz_set_ui
void mpz_set_ui(mpz_ptr, unsigned long int);
#define mpz_set_si __gmpz_set_si
void mpz_set_si(mpz_ptr, signed long int);
#define mpz_set_d __gmpz_set_d
void mpz_set_d(mpz_ptr, double);
#define mpz_set_q __gmpz_set_q
void mpz_set_q(mpz_ptr, mpq_srcptr);
#define mpz_set_f __gmpz_set_f
void mpz_set_f(mpz_ptr, mpf_srcptr);
#define mpz_set_str __gmpz_set_str
int mpz_set_str(mpz_ptr, const char *, int);
#define mpz_swap __gmpz_swap
void mpz_swap(mpz_ptr, mpz_ptr);
#define mpz_init_set_ui __gmpz_init_set_ui
void mpz_init_set_ui(mpz_ptr, unsigned long int);
#define mpz_init_set_si __gmpz_init_set_si
void mpz_init_set_si(mpz_ptr, signed long int);
#define mpz_init_set __gmpz_init_set
void mpz_init_set(mpz_ptr, mpz_srcptr);
#define mpz_get_ui __gmpz_get_ui
unsigned long int mpz_get_ui(mpz_srcptr);
#define mpz_get_si __gmpz_get_si
signed long int mpz_get_si(mpz_srcptr);
#define mpz_get_d __gmpz_get_d
double mpz_get_d(mpz_srcptr);
#define mpz_get_d_2exp __gmpz_get_d_2exp
double mpz_get_d_2exp(signed long int *, mpz_srcptr);
#define mpz_get_str __gmpz_get_str
char *mpz_get_str(char *, int, mpz_srcptr);
#define mpz_getlimbn __gmpz_getlimbn
mp_limb_t mpz_getlimbn(mpz_srcptr, mp_size_t);
#define mpz_size __gmpz_size
size_t mpz_size(mpz_srcptr);
#define mpz_sizeinbase __gmpz_sizeinbase
size_t mpz_sizeinbase(mpz_srcptr, int);
#define mpz_limbs_read __gmpz_limbs_read
mp_srcptr mpz_limbs_read(mpz_srcptr);
#define mpz_limbs_write __gmpz_limbs_write
mp_ptr mpz_limbs_write(mpz_ptr, mp_size_t);
#define mpz_limbs_modify __gmpz_limbs_modify
mp_ptr mpz_limbs_modify(mpz_ptr, mp_size_t);
#define mpz_limbs_finish __gmpz_limbs_finish
void mpz_limbs_finish(mpz_ptr, mp_size_t);
#define mpz_roinit_n __gmpz_roinit_n
mpz_srcptr mpz_roinit_n(mpz_ptr, mp_srcptr, mp_size_t);

#define mpz_add __gmpz_add
void mpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_add_ui __gmpz_add_ui
void mpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_sub __gmpz_sub
void mpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_sub_ui __gmpz_sub_ui
void mpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_ui_sub __gmpz_ui_sub
void mpz_ui_sub(mpz_ptr, unsigned long int, mpz_srcptr);
#define mpz_mul __gmpz_mul
void mpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_mul_si __gmpz_mul_si
void mpz_mul_si(mpz_ptr, mpz_srcptr, long int);
#define mpz_mul_ui __gmpz_mul_ui
void mpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_addmul __gmpz_addmul
void mpz_addmul(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_addmul_ui __gmpz_addmul_ui
void mpz_addmul_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_submul __gmpz_submul
void mpz_submul(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_submul_ui __gmpz_submul_ui
void mpz_submul_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_mul_2exp __gmpz_mul_2exp
void mpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_neg __gmpz_neg
void mpz_neg(mpz_ptr, mpz_srcptr);
#define mpz_abs __gmpz_abs
void mpz_abs(mpz_ptr, mpz_srcptr);

#define mpz_cdiv_q __gmpz_cdiv_q
void mpz_cdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_cdiv_r __gmpz_cdiv_r
void mpz_cdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_cdiv_qr __gmpz_cdiv_qr
void mpz_cdiv_qr(mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_cdiv_q_ui __gmpz_cdiv_q_ui
unsigned long int mpz_cdiv_q_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_cdiv_r_ui __gmpz_cdiv_r_ui
unsigned long int mpz_cdiv_r_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_cdiv_qr_ui __gmpz_cdiv_qr_ui
unsigned long int mpz_cdiv_qr_ui(mpz_ptr, mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_cdiv_ui __gmpz_cdiv_ui
unsigned long int mpz_cdiv_ui(mpz_srcptr, unsigned long int);
#define mpz_cdiv_q_2exp __gmpz_cdiv_q_2exp
void mpz_cdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_cdiv_r_2exp __gmpz_cdiv_r_2exp
void mpz_cdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_fdiv_q __gmpz_fdiv_q
void mpz_fdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_fdiv_r __gmpz_fdiv_r
void mpz_fdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_fdiv_qr __gmpz_fdiv_qr
void mpz_fdiv_qr(mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_fdiv_q_ui __gmpz_fdiv_q_ui
unsigned long int mpz_fdiv_q_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_fdiv_r_ui __gmpz_fdiv_r_ui
unsigned long int mpz_fdiv_r_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_fdiv_qr_ui __gmpz_fdiv_qr_ui
unsigned long int mpz_fdiv_qr_ui(mpz_ptr, mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_fdiv_ui __gmpz_fdiv_ui
unsigned long int mpz_fdiv_ui(mpz_srcptr, unsigned long int);
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
void mpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_fdiv_r_2exp __gmpz_fdiv_r_2exp
void mpz_fdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_tdiv_q __gmpz_tdiv_q
void mpz_tdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_tdiv_r __gmpz_tdiv_r
void mpz_tdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_tdiv_qr __gmpz_tdiv_qr
void mpz_tdiv_qr(mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_tdiv_q_ui __gmpz_tdiv_q_ui
unsigned long int mpz_tdiv_q_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_tdiv_r_ui __gmpz_tdiv_r_ui
unsigned long int mpz_tdiv_r_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_tdiv_qr_ui __gmpz_tdiv_qr_ui
unsigned long int mpz_tdiv_qr_ui(mpz_ptr, mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_tdiv_ui __gmpz_tdiv_ui
unsigned long int mpz_tdiv_ui(mpz_srcptr, unsigned long int);
#define mpz_tdiv_q_2exp __gmpz_tdiv_q_2exp
void mpz_tdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_tdiv_r_2exp __gmpz_tdiv_r_2exp
void mpz_tdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
#define mpz_div_2exp __gmpz_fdiv_q_2exp
#define mpz_mod __gmpz_mod
void mpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_mod_ui __gmpz_fdiv_r_ui
#define mpz_divexact __gmpz_divexact
void mpz_divexact(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_divexact_ui __gmpz_divexact_ui
void mpz_divexact_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_divisible_p __gmpz_divisible_p
int mpz_divisible_p(mpz_srcptr, mpz_srcptr);
#define mpz_divisible_ui_p __gmpz_divisible_ui_p
int mpz_divisible_ui_p(mpz_srcptr, unsigned long int);
#define mpz_congruent_p __gmpz_congruent_p
int mpz_congruent_p(mpz_srcptr, mpz_srcptr, mpz_srcptr);
#define mpz_congruent_ui_p __gmpz_congruent_ui_p
int mpz_congruent_ui_p(mpz_srcptr, unsigned long, unsigned long);

#define mpz_powm __gmpz_powm
void mpz_powm(mpz_ptr, mpz_srcptr, mpz_srcptr, mpz_srcptr);
#define mpz_powm_ui __gmpz_powm_ui
void mpz_powm_ui(mpz_ptr, mpz_srcptr, unsigned long int, mpz_srcptr);
#define mpz_pow_ui __gmpz_pow_ui
void mpz_pow_ui(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
void mpz_ui_pow_ui(mpz_ptr, unsigned long int, unsigned long int);
#define mpz_root __gmpz_root
int mpz_root(mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_rootrem __gmpz_rootrem
void mpz_rootrem(mpz_ptr, mpz_ptr, mpz_srcptr, unsigned long int);
#define mpz_sqrt __gmpz_sqrt
void mpz_sqrt(mpz_ptr, mpz_srcptr);
#define mpz_sqrtrem __gmpz_sqrtrem
void mpz_sqrtrem(mpz_ptr, mpz_ptr, mpz_srcptr);
#define mpz_perfect_power_p __gmpz_perfect_power_p
int mpz_perfect_power_p(mpz_srcptr);
#define mpz_perfect_square_p __gmpz_perfect_square_p
int mpz_perfect_square_p(mpz_srcptr);

#define mpz_probab_prime_p __gmpz_probab_prime_p
int mpz_probab_prime_p(mpz_srcptr, int);
#define mpz_nextprime __gmpz_nextprime
void mpz_nextprime(mpz_ptr, mpz_srcptr);
#define mpz_gcd __gmpz_gcd
void mpz_gcd(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_gcdext __gmpz_gcdext
void mpz_gcdext(mpz_ptr, mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_lcm __gmpz_lcm
void mpz_lcm(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_invert __gmpz_invert
int mpz_invert(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_jacobi __gmpz_jacobi
int mpz_jacobi(mpz_srcptr, mpz_srcptr);
#define mpz_kronecker __gmpz_jacobi
#define mpz_remove __gmpz_remove
mp_bitcnt_t mpz_remove(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_fac_ui __gmpz_fac_ui
void mpz_fac_ui(mpz_ptr, unsigned long int);
#define mpz_bin_uiui __gmpz_bin_uiui
void mpz_bin_uiui(mpz_ptr, unsigned long int, unsigned long int);
#define mpz_fib_ui __gmpz_fib_ui
void mpz_fib_ui(mpz_ptr, unsigned long int);

#define mpz_cmp __gmpz_cmp
int mpz_cmp(mpz_srcptr, mpz_srcptr);
#define mpz_cmp_ui __gmpz_cmp_ui
int mpz_cmp_ui(mpz_srcptr, unsigned long int);
#define mpz_cmp_si __gmpz_cmp_si
int mpz_cmp_si(mpz_srcptr, signed long int);
#define mpz_cmpabs __gmpz_cmpabs
int mpz_cmpabs(mpz_srcptr, mpz_srcptr);
#define mpz_cmpabs_ui __gmpz_cmpabs_ui
int mpz_cmpabs_ui(mpz_srcptr, unsigned long int);
/* documented as macros: sign and parity read the structure directly */
#define mpz_sgn(z) ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)
#define mpz_odd_p(z) (((z)->_mp_size != 0) & (int) (z)->_mp_d[0])
#define mpz_even_p(z) (!mpz_odd_p(z))

#define mpz_and __gmpz_and
void mpz_and(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_ior __gmpz_ior
void mpz_ior(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_xor __gmpz_xor
void mpz_xor(mpz_ptr, mpz_srcptr, mpz_srcptr);
#define mpz_com __gmpz_com
void mpz_com(mpz_ptr, mpz_srcptr);
#define mpz_popcount __gmpz_popcount
mp_bitcnt_t mpz_popcount(mpz_srcptr);
#define mpz_scan1 __gmpz_scan1
mp_bitcnt_t mpz_scan1(mpz_srcptr, mp_bitcnt_t);
#define mpz_setbit __gmpz_setbit
void mpz_setbit(mpz_ptr, mp_bitcnt_t);
#define mpz_clrbit __gmpz_clrbit
void mpz_clrbit(mpz_ptr, mp_bitcnt_t);
#define mpz_combit __gmpz_combit
void mpz_combit(mpz_ptr, mp_bitcnt_t);
#define mpz_tstbit __gmpz_tstbit
int mpz_tstbit(mpz_srcptr, mp_bitcnt_t);

#define mpz_fits_slong_p __gmpz_fits_slong_p
int mpz_fits_slong_p(mpz_srcptr);
#define mpz_import __gmpz_import
void mpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
#define mpz_export __gmpz_export
void *mpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);
#define mpz_urandomb __gmpz_urandomb
void mpz_urandomb(mpz_ptr, gmp_randstate_t, mp_bitcnt_t);
#define mpz_urandomm __gmpz_urandomm
void mpz_urandomm(mpz_ptr, gmp_randstate_t, mpz_srcptr);
#define mpz_rrandomb __gmpz_rrandomb
void mpz_rrandomb(mpz_ptr, gmp_randstate_t, mp_bitcnt_t);
#define mpz_out_str __gmpz_out_str
size_t mpz_out_str(FILE *, int, mpz_srcptr);
#define mpz_inp_str __gmpz_inp_str
size_t mpz_inp_str(mpz_ptr, FILE *, int);
#define mpz_out_raw __gmpz_out_raw
size_t mpz_out_raw(FILE *, mpz_srcptr);
#define mpz_inp_raw __gmpz_inp_raw
size_t mpz_inp_raw(mpz_ptr, FILE *);

/* ---- rationals and floats (only what headers reference) ---------------- */
#define mpq_init __gmpq_init
void mpq_init(mpq_ptr);
#define mpq_clear __gmpq_clear
void mpq_clear(mpq_ptr);
#define mpq_numref(q) (&((q)->_mp_num))
#define mpq_denref(q) (&((q)->_mp_den))
#define mpf_init __gmpf_init
void mpf_init(mpf_ptr);
#define mpf_clear __gmpf_clear
void mpf_clear(mpf_ptr);
#define mpf_get_d __gmpf_get_d
double mpf_get_d(mpf_srcptr);

/* ---- natural numbers (mpn) ------------------------------------------- */
#define mpn_add_n __gmpn_add_n
mp_limb_t mpn_add_n(mp_ptr, mp_srcptr, mp_srcptr, mp_size_t);
#define mpn_add_1 __gmpn_add_1
mp_limb_t mpn_add_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_add __gmpn_add
mp_limb_t mpn_add(mp_ptr, mp_srcptr, mp_size_t, mp_srcptr, mp_size_t);
#define mpn_sub_n __gmpn_sub_n
mp_limb_t mpn_sub_n(mp_ptr, mp_srcptr, mp_srcptr, mp_size_t);
#define mpn_sub_1 __gmpn_sub_1
mp_limb_t mpn_sub_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_sub __gmpn_sub
mp_limb_t mpn_sub(mp_ptr, mp_srcptr, mp_size_t, mp_srcptr, mp_size_t);
#define mpn_neg __gmpn_neg
mp_limb_t mpn_neg(mp_ptr, mp_srcptr, mp_size_t);
#define mpn_mul __gmpn_mul
mp_limb_t mpn_mul(mp_ptr, mp_srcptr, mp_size_t, mp_srcptr, mp_size_t);
#define mpn_mul_n __gmpn_mul_n
void mpn_mul_n(mp_ptr, mp_srcptr, mp_srcptr, mp_size_t);
#define mpn_sqr __gmpn_sqr
void mpn_sqr(mp_ptr, mp_srcptr, mp_size_t);
#define mpn_mul_1 __gmpn_mul_1
mp_limb_t mpn_mul_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_addmul_1 __gmpn_addmul_1
mp_limb_t mpn_addmul_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_submul_1 __gmpn_submul_1
mp_limb_t mpn_submul_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_tdiv_qr __gmpn_tdiv_qr
void mpn_tdiv_qr(mp_ptr, mp_ptr, mp_size_t, mp_srcptr, mp_size_t, mp_srcptr, mp_size_t);
#define mpn_divrem_1 __gmpn_divrem_1
mp_limb_t mpn_divrem_1(mp_ptr, mp_size_t, mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_divmod_1(qp, np, nn, d) mpn_divrem_1(qp, 0, np, nn, d)
#define mpn_divexact_1 __gmpn_divexact_1
void mpn_divexact_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_mod_1 __gmpn_mod_1
mp_limb_t mpn_mod_1(mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_lshift __gmpn_lshift
mp_limb_t mpn_lshift(mp_ptr, mp_srcptr, mp_size_t, unsigned int);
#define mpn_rshift __gmpn_rshift
mp_limb_t mpn_rshift(mp_ptr, mp_srcptr, mp_size_t, unsigned int);
#define mpn_cmp __gmpn_cmp
int mpn_cmp(mp_srcptr, mp_srcptr, mp_size_t);
#define mpn_zero_p __gmpn_zero_p
int mpn_zero_p(mp_srcptr, mp_size_t);
#define mpn_gcd __gmpn_gcd
mp_size_t mpn_gcd(mp_ptr, mp_ptr, mp_size_t, mp_ptr, mp_size_t);
#define mpn_gcd_1 __gmpn_gcd_1
mp_limb_t mpn_gcd_1(mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_gcdext __gmpn_gcdext
mp_size_t mpn_gcdext(mp_ptr, mp_ptr, mp_size_t *, mp_ptr, mp_size_t, mp_ptr, mp_size_t);
#define mpn_sqrtrem __gmpn_sqrtrem
mp_size_t mpn_sqrtrem(mp_ptr, mp_ptr, mp_srcptr, mp_size_t);
#define mpn_get_str __gmpn_get_str
size_t mpn_get_str(unsigned char *, int, mp_ptr, mp_size_t);
#define mpn_set_str __gmpn_set_str
mp_size_t mpn_set_str(mp_ptr, const unsigned char *, size_t, int);
#define mpn_scan1 __gmpn_scan1
mp_bitcnt_t mpn_scan1(mp_srcptr, mp_bitcnt_t);
#define mpn_popcount __gmpn_popcount
mp_bitcnt_t mpn_popcount(mp_srcptr, mp_size_t);
#define mpn_random __gmpn_random
void mpn_random(mp_ptr, mp_size_t);
#define mpn_random2 __gmpn_random2
void mpn_random2(mp_ptr, mp_size_t);
#define mpn_com __gmpn_com
void mpn_com(mp_ptr, mp_srcptr, mp_size_t);
#define mpn_copyi __gmpn_copyi
void mpn_copyi(mp_ptr, mp_srcptr, mp_size_t);
#define mpn_zero __gmpn_zero
void mpn_zero(mp_ptr, mp_size_t);

/* exported by libgmp.so.10 although not in the manual; the closure calls
   them only behind FLINT_HAVE_NATIVE_* switches that the recipe leaves off,
   or as documented-equivalent helpers */
#define mpn_modexact_1_odd __gmpn_modexact_1_odd
mp_limb_t mpn_modexact_1_odd(mp_srcptr, mp_size_t, mp_limb_t);
#define mpn_gcdext_1 __gmpn_gcdext_1
mp_limb_t mpn_gcdext_1(mp_limb_signed_t *, mp_limb_signed_t *, mp_limb_t, mp_limb_t);
#define mpn_invert_limb __gmpn_invert_limb
mp_limb_t mpn_invert_limb(mp_limb_t);

#ifdef __cplusplus
}
#endif

#endif
