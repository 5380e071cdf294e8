// The subset of the MPFR 4.x / GMP 6.x runtime ABI that libmpfft_b200 uses
// for host-side conversion between mpfr_t arrays and device limb planes and
// for building twiddle tables.  The image carries libmpfr.so.6/libgmp.so.10
// but no development headers, so the public types are declared here from the
// MPFR manual ("Nomenclature and Types") and the libraries' exported names.
// A user who compiles against the real <mpfr.h> gets the identical layout.
#pragma once

#include <cstddef>

extern "C" {

typedef unsigned long mp_limb_t;

typedef struct {
  int _mp_alloc;
  int _mp_size;  // sign = sign of the integer, |size| = limbs in use
  mp_limb_t *_mp_d;
} __mpz_struct;
typedef const __mpz_struct *mpz_srcptr;
typedef __mpz_struct *mpz_ptr;

typedef long mpfr_prec_t;
typedef int mpfr_sign_t;
typedef long mpfr_exp_t;

typedef enum { MPFR_RNDN = 0, MPFR_RNDZ, MPFR_RNDU, MPFR_RNDD, MPFR_RNDA, MPFR_RNDF } mpfr_rnd_t;

typedef struct {
  mpfr_prec_t _mpfr_prec;
  mpfr_sign_t _mpfr_sign;
  mpfr_exp_t _mpfr_exp;  // value = sign * 0.d * 2^exp for regular numbers
  mp_limb_t *_mpfr_d;    // ceil(prec/64) limbs, least significant first, MSB set
} __mpfr_struct;
typedef __mpfr_struct mpfr_t[1];
typedef __mpfr_struct *mpfr_ptr;
typedef const __mpfr_struct *mpfr_srcptr;

void mpfr_init2(mpfr_ptr, mpfr_prec_t);
void mpfr_clear(mpfr_ptr);
mpfr_prec_t mpfr_get_prec(mpfr_srcptr);
int mpfr_set(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_set_ui(mpfr_ptr, unsigned long, mpfr_rnd_t);
int mpfr_set_z_2exp(mpfr_ptr, mpz_srcptr, mpfr_exp_t, mpfr_rnd_t);
mpfr_exp_t mpfr_get_z_2exp(mpz_ptr, mpfr_srcptr);
void mpfr_set_zero(mpfr_ptr, int);
void mpfr_set_nan(mpfr_ptr);
int mpfr_zero_p(mpfr_srcptr);
int mpfr_nan_p(mpfr_srcptr);
int mpfr_inf_p(mpfr_srcptr);
int mpfr_number_p(mpfr_srcptr);
int mpfr_const_pi(mpfr_ptr, mpfr_rnd_t);
int mpfr_mul_ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_div_ui(mpfr_ptr, mpfr_srcptr, unsigned long, mpfr_rnd_t);
int mpfr_mul_2si(mpfr_ptr, mpfr_srcptr, long, mpfr_rnd_t);
int mpfr_add(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sub(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sub_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
int mpfr_add_d(mpfr_ptr, mpfr_srcptr, double, mpfr_rnd_t);
void mpfr_set_prec(mpfr_ptr, mpfr_prec_t);
double mpfr_get_d(mpfr_srcptr, mpfr_rnd_t);
int mpfr_abs(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_rint(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_sgn(mpfr_srcptr);
int mpfr_sin_cos(mpfr_ptr, mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
void mpfr_free_cache(void);
mpfr_exp_t mpfr_get_emin(void);
mpfr_exp_t mpfr_get_emax(void);
}
