/*
 * Minimal, project-owned declarations for the MPFR 4.x and GMP 6.x runtime
 * libraries (libmpfr.so.6, libgmp.so.10).
 *
 * The image ships the MPFR/GMP shared objects but no development headers.
 * This file declares only what this project (and the reference code it
 * compiles as a test oracle) calls.  The types follow the public ABI that the
 * MPFR manual documents (section "Nomenclature and Types": mpfr_t is a
 * one-element array of a struct holding precision, sign, exponent and a
 * pointer to 64-bit limbs) and the names follow the libraries' exported
 * symbols (`nm -D`).  GMP exports its documented API under a `__g` prefix
 * (gmp_randinit_mt -> __gmp_randinit_mt), and MPFR exports its stdio-based
 * printf family under `__gmpfr_`; the macros below map the documented names
 * onto those symbols.
 *
 * Test infrastructure and host-side pack/unpack only: nothing here runs on
 * the GPU.
 */
#ifndef MPFFT_MPFR_DECLS_H
#define MPFFT_MPFR_DECLS_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GMP types (x86-64 LP64: mp_limb_t is a 64-bit unsigned long) ---- */
typedef unsigned long mp_limb_t;
typedef long mp_exp_t;
typedef unsigned long mp_bitcnt_t;

typedef struct {
  int _mp_alloc;   /* limbs allocated */
  int _mp_size;    /* |size| = limbs used, sign = sign of the integer */
  mp_limb_t *_mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

typedef struct {
  __mpz_struct _mp_seed[1];
  int _mp_alg;
  union { void *_mp_lc; } _mp_algdata;
} __gmp_randstate_struct;
typedef __gmp_randstate_struct gmp_randstate_t[1];

void __gmp_randinit_mt(gmp_randstate_t);
void __gmp_randseed_ui(gmp_randstate_t, unsigned long);
void __gmp_randclear(gmp_randstate_t);
#define gmp_randinit_mt __gmp_randinit_mt
#define gmp_randseed_ui __gmp_randseed_ui
#define gmp_randclear __gmp_randclear

void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
char *__gmpz_get_str(char *, int, mpz_srcptr);
int __gmpz_set_str(mpz_ptr, const char *, int);
#define mpz_init __gmpz_init
#define mpz_clear __gmpz_clear
#define mpz_get_str __gmpz_get_str
#define mpz_set_str __gmpz_set_str

/* ---- MPFR types ---- */
typedef long mpfr_prec_t;
typedef int mpfr_sign_t;
typedef long mpfr_exp_t;

typedef enum {
  MPFR_RNDN = 0, /* round to nearest, ties to even */
  MPFR_RNDZ,     /* toward zero */
  MPFR_RNDU,     /* toward +infinity */
  MPFR_RNDD,     /* toward -infinity */
  MPFR_RNDA,     /* away from zero */
  MPFR_RNDF,     /* faithful */
  MPFR_RNDNA = -1
} mpfr_rnd_t;

typedef struct {
  mpfr_prec_t _mpfr_prec; /* precision in bits */
  mpfr_sign_t _mpfr_sign; /* +1 / -1 */
  mpfr_exp_t _mpfr_exp;   /* value = sign * 0.d[...] * 2^exp; special values use reserved exps */
  mp_limb_t *_mpfr_d;     /* ceil(prec/64) limbs, most significant limb last, MSB set */
} __mpfr_struct;
typedef __mpfr_struct mpfr_t[1];
typedef __mpfr_struct *mpfr_ptr;
typedef const __mpfr_struct *mpfr_srcptr;

/* initialisation and assignment */
void mpfr_init2(mpfr_ptr, mpfr_prec_t);
void mpfr_inits2(mpfr_prec_t, mpfr_ptr, ...);
void mpfr_clear(mpfr_ptr);
void mpfr_clears(mpfr_ptr, ...);
void mpfr_set_prec(mpfr_ptr, mpfr_prec_t);
mpfr_prec_t mpfr_get_prec(mpfr_srcptr);
int mpfr_prec_round(mpfr_ptr, mpfr_prec_t, mpfr_rnd_t);
int mpfr_set(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_set_ui(mpfr_ptr, unsigned long, mpfr_rnd_t);
int mpfr_set_si(mpfr_ptr, long, mpfr_rnd_t);
int mpfr_set_d(mpfr_ptr, double, mpfr_rnd_t);
int mpfr_set_ui_2exp(mpfr_ptr, unsigned long, mpfr_exp_t, mpfr_rnd_t);
int mpfr_set_z_2exp(mpfr_ptr, mpz_srcptr, mpfr_exp_t, mpfr_rnd_t);
mpfr_exp_t mpfr_get_z_2exp(mpz_ptr, mpfr_srcptr);
int mpfr_set_str(mpfr_ptr, const char *, int, mpfr_rnd_t);
void mpfr_set_zero(mpfr_ptr, int);
void mpfr_set_nan(mpfr_ptr);
void mpfr_set_inf(mpfr_ptr, int);
double mpfr_get_d(mpfr_srcptr, mpfr_rnd_t);
int mpfr_sub_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
int mpfr_add_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
double mpfr_get_d_2exp(long *, mpfr_srcptr, mpfr_rnd_t);
mpfr_exp_t mpfr_get_exp(mpfr_srcptr);
char *mpfr_get_str(char *, mpfr_exp_t *, int, size_t, mpfr_srcptr, mpfr_rnd_t);
size_t mpfr_get_str_ndigits(int, mpfr_prec_t);
void mpfr_free_str(char *);

/* arithmetic */
int mpfr_add(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sub(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_mul(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_div(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sqrt(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_neg(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_abs(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_add_ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_sub_ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_mul_ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_div_ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_ui_div(mpfr_ptr, unsigned long, mpfr_srcptr, mpfr_rnd_t);
int mpfr_mul_2si(mpfr_ptr, mpfr_srcptr, long, mpfr_rnd_t);
int mpfr_div_2si(mpfr_ptr, mpfr_srcptr, long, mpfr_rnd_t);
int mpfr_mul_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
int mpfr_mul_2ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_div_2ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_log2(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);

/* special functions and constants */
int mpfr_const_pi(mpfr_ptr, mpfr_rnd_t);
int mpfr_cos(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sin(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sin_cos(mpfr_ptr, mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
void mpfr_free_cache(void);

/* comparison and predicates */
int mpfr_cmp(mpfr_srcptr, mpfr_srcptr);
int mpfr_cmpabs(mpfr_srcptr, mpfr_srcptr);
int mpfr_sgn(mpfr_srcptr);
int mpfr_zero_p(mpfr_srcptr);
int mpfr_nan_p(mpfr_srcptr);
int mpfr_inf_p(mpfr_srcptr);
int mpfr_number_p(mpfr_srcptr);
int mpfr_regular_p(mpfr_srcptr);

/* random numbers */
int mpfr_urandom(mpfr_ptr, gmp_randstate_t, mpfr_rnd_t);

/* formatted output */
int mpfr_printf(const char *, ...);
int mpfr_asprintf(char **, const char *, ...);
int __gmpfr_fprintf(FILE *, const char *, ...);
#define mpfr_fprintf __gmpfr_fprintf

const char *mpfr_get_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MPFFT_MPFR_DECLS_H */
