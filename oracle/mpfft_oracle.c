/*
 * mpFFT CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's hot path, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product library (mpfft_b200/) never links or calls this file.
 *
 * Contents
 *  - orc_mp_*: the multiprecision conjugate-pair split-radix 2/4 DIT FFT,
 *    restating lab/parallel/mp/parallel_mp_fft2.c:121-328 (serial twin
 *    lab/serial/mp/serial_mp_fft3.c:121-253).  Every MPFR operation is the
 *    same correctly-rounded operation on the same operands at the same
 *    precision as in the reference, so results are bit-identical to it
 *    (pinned by tests against the compiled reference and golden vectors).
 *  - orc_d_*: the FP64 conjugate-pair split-radix FFT with hard-coded n=8
 *    and n=16 base cases, restating lab/serial/double/serial_d_fft6.c:93-429.
 *    Same IEEE operations in the same association; bit-identical.
 *  - orc_mp_dft: the direct O(N^2) DFT in MPFR at a chosen (typically 2P)
 *    precision -- algorithm-independent accuracy oracle.
 *  - input generators (seeded MT uniform[-1,1) at full precision, the
 *    reference's IN 2 closed form), error metrics, hex (de)serialisation.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mpfr_decls.h"

#define OAPI __attribute__((visibility("default")))
#define RN MPFR_RNDN

/* ------------------------------------------------------------------------ */
/* array helpers                                                            */
/* ------------------------------------------------------------------------ */

OAPI mpfr_t *orc_mp_alloc(unsigned long n, long prec) {
  mpfr_t *a = (mpfr_t *)calloc(n ? n : 1, sizeof(mpfr_t));
  for (unsigned long k = 0; k < n; k++) {
    mpfr_init2(a[k], prec);
    mpfr_set_ui(a[k], 0, RN);
  }
  return a;
}

OAPI void orc_mp_free(mpfr_t *a, unsigned long n) {
  if (!a) return;
  for (unsigned long k = 0; k < n; k++) mpfr_clear(a[k]);
  free(a);
}

/* a[0] = the number written in s (any MPFR string syntax, e.g. the "%Ra"
 * hexadecimal form "0x1.8p+3"), rounded to a's precision; 0 on success */
OAPI int orc_mp_set_str(mpfr_t *a, const char *s) { return mpfr_set_str(a[0], s, 0, RN); }

/* element pointer (lets Python address a[k] of an mpfr_t array) */
OAPI mpfr_ptr orc_mp_at(mpfr_t *a, unsigned long k) { return a[k]; }

OAPI void orc_mp_copy(mpfr_t *dst, mpfr_t *src, unsigned long n) {
  for (unsigned long k = 0; k < n; k++) mpfr_set(dst[k], src[k], RN);
}

/* strided copy dst[k] = src[k*stride] */
OAPI void orc_mp_gather(mpfr_t *dst, mpfr_t *src, unsigned long n, unsigned long stride) {
  for (unsigned long k = 0; k < n; k++) mpfr_set(dst[k], src[k * stride], RN);
}

OAPI void orc_mp_set_prec_all(mpfr_t *a, unsigned long n, long prec) {
  for (unsigned long k = 0; k < n; k++) mpfr_set_prec(a[k], prec);
}

OAPI void orc_mp_set_d(mpfr_t *a, const double *v, unsigned long n) {
  for (unsigned long k = 0; k < n; k++) mpfr_set_d(a[k], v[k], RN);
}

OAPI void orc_mp_get_d(mpfr_t *a, double *v, unsigned long n) {
  for (unsigned long k = 0; k < n; k++) v[k] = mpfr_get_d(a[k], RN);
}

OAPI void orc_mp_set_ui(mpfr_t *a, unsigned long n, unsigned long v) {
  for (unsigned long k = 0; k < n; k++) mpfr_set_ui(a[k], v, RN);
}

/* a[k] *= 2^e for k in [0,n) (exact) */
OAPI void orc_mp_scale2(mpfr_t *a, unsigned long n, long e) {
  for (unsigned long k = 0; k < n; k++) mpfr_mul_2si(a[k], a[k], e, RN);
}

/* Full spectrum of a real signal of n >= 2 points from its half spectrum
 * h[0..n/2]: f[k] = h[k] for k <= n/2 and f[n-k] = conj h[k] for 0 < k < n/2;
 * the imaginary parts of f[0] and f[n/2] are set to zero (a real signal's
 * spectrum has none there).  Used to state the inverse real transform as a
 * complex DFT. */
OAPI void orc_mp_hermitian_extend(unsigned long n, mpfr_t *hr, mpfr_t *hi, mpfr_t *fr, mpfr_t *fi) {
  const unsigned long m = n / 2;
  for (unsigned long k = 0; k <= m; k++) {
    mpfr_set(fr[k], hr[k], RN);
    if (k == 0 || k == m) mpfr_set_ui(fi[k], 0, RN);
    else mpfr_set(fi[k], hi[k], RN);
  }
  for (unsigned long k = 1; k < m; k++) {
    mpfr_set(fr[n - k], hr[k], RN);
    mpfr_neg(fi[n - k], hi[k], RN);
  }
}

/* double-double views: hi[k] = a[k] rounded to double, lo[k] = (a[k] - hi[k])
 * rounded; set: a[k] = hi[k] + lo[k] (rounded to a's precision) */
OAPI void orc_mp_get_dd(mpfr_t *a, double *hi, double *lo, unsigned long n) {
  mpfr_t r;
  mpfr_init2(r, mpfr_get_prec(a[0]) + 64);
  for (unsigned long k = 0; k < n; k++) {
    hi[k] = mpfr_get_d(a[k], RN);
    mpfr_sub_d(r, a[k], hi[k], RN);
    lo[k] = mpfr_get_d(r, RN);
  }
  mpfr_clear(r);
}

OAPI void orc_mp_set_dd(mpfr_t *a, const double *hi, const double *lo, unsigned long n) {
  for (unsigned long k = 0; k < n; k++) {
    mpfr_set_d(a[k], hi[k], RN);
    mpfr_add_d(a[k], a[k], lo[k], RN);
  }
}

OAPI void orc_mp_set_nan(mpfr_t *a, unsigned long k) { mpfr_set_nan(a[k]); }
OAPI void orc_mp_set_inf(mpfr_t *a, unsigned long k, int sign) { mpfr_set_inf(a[k], sign); }

/* number of k where a[k] and b[k] differ as values (NaN == NaN) */
OAPI unsigned long orc_mp_count_diff(mpfr_t *a, mpfr_t *b, unsigned long n) {
  unsigned long bad = 0;
  for (unsigned long k = 0; k < n; k++) {
    if (mpfr_nan_p(a[k]) || mpfr_nan_p(b[k])) {
      bad += !(mpfr_nan_p(a[k]) && mpfr_nan_p(b[k]));
      continue;
    }
    if (mpfr_cmp(a[k], b[k]) != 0) bad++;
    else if (mpfr_zero_p(a[k]) && mpfr_sgn(a[k]) == 0 && a[k]->_mpfr_sign != b[k]->_mpfr_sign) bad++;
  }
  return bad;
}

/* Exact text form "[-]0x<hex integer>p<binary exponent>", or "0", "nan",
 * "inf", "-inf".  Returns the number of bytes needed (incl. NUL). */
OAPI int orc_mp_to_hex(mpfr_ptr x, char *buf, int buflen) {
  char tmp[64];
  const char *s = NULL;
  if (mpfr_nan_p(x)) s = "nan";
  else if (mpfr_inf_p(x)) s = mpfr_sgn(x) > 0 ? "inf" : "-inf";
  else if (mpfr_zero_p(x)) s = x->_mpfr_sign < 0 ? "-0" : "0";
  if (s) {
    int need = (int)strlen(s) + 1;
    if (buf && buflen >= need) memcpy(buf, s, need);
    return need;
  }
  mpz_t z;
  mpz_init(z);
  mpfr_exp_t e = mpfr_get_z_2exp(z, x);
  char *digits = mpz_get_str(NULL, 16, z); /* "-abc" or "abc" */
  int neg = digits[0] == '-';
  snprintf(tmp, sizeof tmp, "p%ld", (long)e);
  int need = (int)(strlen(digits) + 2 + strlen(tmp) + 1);
  if (buf && buflen >= need) {
    snprintf(buf, buflen, "%s0x%s%s", neg ? "-" : "", digits + neg, tmp);
  }
  free(digits);
  mpz_clear(z);
  return need;
}

OAPI int orc_mp_from_hex(mpfr_ptr x, const char *s) {
  if (!strcmp(s, "nan")) { mpfr_set_nan(x); return 0; }
  if (!strcmp(s, "inf")) { mpfr_set_inf(x, 1); return 0; }
  if (!strcmp(s, "-inf")) { mpfr_set_inf(x, -1); return 0; }
  if (!strcmp(s, "0")) { mpfr_set_zero(x, 1); return 0; }
  if (!strcmp(s, "-0")) { mpfr_set_zero(x, -1); return 0; }
  return mpfr_set_str(x, s, 16, RN);
}

/* ------------------------------------------------------------------------ */
/* inputs                                                                   */
/* ------------------------------------------------------------------------ */

/* re/im i.i.d. uniform [-1,1) at the arrays' full precision: one Mersenne-
 * twister stream (gmp_randinit_mt + gmp_randseed_ui), draws interleaved re,im
 * per k as in the reference's IN 1 (lab/parallel/mp/parallel_mp_fft2.c:92-100),
 * then mapped u -> 2u-1. */
OAPI void orc_mp_fill_uniform(mpfr_t *re, mpfr_t *im, unsigned long n, unsigned long seed) {
  gmp_randstate_t st;
  gmp_randinit_mt(st);
  gmp_randseed_ui(st, seed);
  for (unsigned long k = 0; k < n; k++) {
    mpfr_urandom(re[k], st, RN);
    mpfr_urandom(im[k], st, RN);
    mpfr_mul_2ui(re[k], re[k], 1, RN);
    mpfr_sub_ui(re[k], re[k], 1, RN);
    mpfr_mul_2ui(im[k], im[k], 1, RN);
    mpfr_sub_ui(im[k], im[k], 1, RN);
  }
  gmp_randclear(st);
}

/* The reference's IN 1 exactly: uniform [0,1) (parallel_mp_fft2.c:92-100). */
OAPI void orc_mp_fill_urandom01(mpfr_t *re, mpfr_t *im, unsigned long n, unsigned long seed) {
  gmp_randstate_t st;
  gmp_randinit_mt(st);
  gmp_randseed_ui(st, seed);
  for (unsigned long k = 0; k < n; k++) {
    mpfr_urandom(re[k], st, RN);
    mpfr_urandom(im[k], st, RN);
  }
  gmp_randclear(st);
}

/* The reference's IN 2: re = 1/(1+k^2), im = 1/(1+k^4), with the same MPFR
 * operation sequence as parallel_mp_fft2.c:104-114 (aux at the arrays'
 * precision). */
OAPI void orc_mp_fill_in2(mpfr_t *re, mpfr_t *im, unsigned long n) {
  mpfr_t aux;
  mpfr_init2(aux, mpfr_get_prec(re[0]));
  for (unsigned long k = 0; k < n; k++) {
    mpfr_set_ui(aux, k * k, RN);
    mpfr_add_ui(re[k], aux, 1, RN);
    mpfr_ui_div(re[k], 1, re[k], RN);
    mpfr_mul(aux, aux, aux, RN);
    mpfr_add_ui(im[k], aux, 1, RN);
    mpfr_ui_div(im[k], 1, im[k], RN);
  }
  mpfr_clear(aux);
}

/* ------------------------------------------------------------------------ */
/* multiprecision conjugate-pair split-radix FFT                            */
/* ------------------------------------------------------------------------ */

typedef struct {
  unsigned long N;
  long P;
  mpfr_t *wr, *wi, *ws, *wd; /* cos, sin, cos+sin, cos-sin of 2*pi*k/N, k < N/4 */
  mpfr_t t[9];               /* butterfly temporaries at precision P */
  unsigned long cnt[4];      /* mults, adds, calls, recursion breaks */
  int count;
} orc_mp_ctx;

/* Twiddle table as in the reference's lut() (parallel_mp_fft2.c:71-82):
 * a = pi/N, then for each k: cos(2k*a), sin(2k*a), their sum and difference,
 * every step rounded to nearest at precision P. */
OAPI orc_mp_ctx *orc_mp_new(unsigned long N, long P) {
  orc_mp_ctx *c = (orc_mp_ctx *)calloc(1, sizeof *c);
  c->N = N;
  c->P = P;
  unsigned long q = N / 4;
  c->wr = orc_mp_alloc(q, P);
  c->wi = orc_mp_alloc(q, P);
  c->ws = orc_mp_alloc(q, P);
  c->wd = orc_mp_alloc(q, P);
  for (int i = 0; i < 9; i++) mpfr_init2(c->t[i], P);
  mpfr_t a, x;
  mpfr_inits2(P, a, x, (mpfr_ptr)0);
  mpfr_const_pi(a, RN);
  mpfr_div_ui(a, a, N, RN);
  for (unsigned long k = 0; k < q; k++) {
    mpfr_mul_ui(x, a, 2 * k, RN);
    mpfr_cos(c->wr[k], x, RN);
    mpfr_sin(c->wi[k], x, RN);
    mpfr_add(c->ws[k], c->wr[k], c->wi[k], RN);
    mpfr_sub(c->wd[k], c->wr[k], c->wi[k], RN);
  }
  mpfr_clears(a, x, (mpfr_ptr)0);
  return c;
}

OAPI void orc_mp_delete(orc_mp_ctx *c) {
  if (!c) return;
  unsigned long q = c->N / 4;
  orc_mp_free(c->wr, q);
  orc_mp_free(c->wi, q);
  orc_mp_free(c->ws, q);
  orc_mp_free(c->wd, q);
  for (int i = 0; i < 9; i++) mpfr_clear(c->t[i]);
  free(c);
}

OAPI void orc_mp_counts(orc_mp_ctx *c, unsigned long *out4, int reset, int enable) {
  if (out4) memcpy(out4, c->cnt, sizeof c->cnt);
  if (reset) memset(c->cnt, 0, sizeof c->cnt);
  c->count = enable;
}

#define CNT(c, m, a, f, r)                                                   \
  do {                                                                       \
    if ((c)->count) {                                                        \
      (c)->cnt[0] += (m); (c)->cnt[1] += (a); (c)->cnt[2] += (f); (c)->cnt[3] += (r); \
    }                                                                        \
  } while (0)

/* Radix-2 or radix-4 leaf; x(j) is element j of the strided subsequence, with
 * the j=0 element wrapped to index N when sn<0 (reference :128,:139,:152). */
static void mp_leaf(orc_mp_ctx *c, unsigned long n, unsigned long s, long sn,
                    mpfr_t *xr, mpfr_t *xi, mpfr_t *yr, mpfr_t *yi) {
  unsigned long j0 = sn < 0 ? c->N : 0;
  if (n == 1) {
    mpfr_set(yr[0], xr[j0], RN);
    mpfr_set(yi[0], xi[j0], RN);
    CNT(c, 0, 0, 0, 1);
    return;
  }
  if (n == 2) {
    mpfr_add(yr[0], xr[j0], xr[s], RN);
    mpfr_sub(yr[1], xr[j0], xr[s], RN);
    mpfr_add(yi[0], xi[j0], xi[s], RN);
    mpfr_sub(yi[1], xi[j0], xi[s], RN);
    CNT(c, 0, 4, 0, 1);
    return;
  }
  /* n == 4: even pair (x0,x2) into y[0..1], odd pair (x1,x3) into sum/diff,
   * then the radix-2 combine with the -i rotation of the odd difference. */
  mpfr_ptr sr = c->t[5], si = c->t[6], dr = c->t[7], di = c->t[8];
  unsigned long j1 = s, j2 = 2 * s, j3 = 3 * s;
  mpfr_add(yr[0], xr[j0], xr[j2], RN);
  mpfr_sub(yr[1], xr[j0], xr[j2], RN);
  mpfr_add(yi[0], xi[j0], xi[j2], RN);
  mpfr_sub(yi[1], xi[j0], xi[j2], RN);
  mpfr_add(sr, xr[j1], xr[j3], RN);
  mpfr_sub(dr, xr[j1], xr[j3], RN);
  mpfr_add(si, xi[j1], xi[j3], RN);
  mpfr_sub(di, xi[j1], xi[j3], RN);
  mpfr_sub(yr[2], yr[0], sr, RN);
  mpfr_add(yr[0], yr[0], sr, RN);
  mpfr_sub(yr[3], yr[1], di, RN);
  mpfr_add(yr[1], yr[1], di, RN);
  mpfr_sub(yi[2], yi[0], si, RN);
  mpfr_add(yi[0], yi[0], si, RN);
  mpfr_add(yi[3], yi[1], dr, RN);
  mpfr_sub(yi[1], yi[1], dr, RN);
  CNT(c, 0, 16, 0, 1);
}

/* The L-shaped combine of one butterfly index k (reference :238-252):
 * (mr_p, mi_p) = Z+ * w^k, (mr_m, mi_m) = Z- * w^-k, already formed. */
static void mp_combine(orc_mp_ctx *c, mpfr_t *yr, mpfr_t *yi, unsigned long k, unsigned long q,
                       mpfr_ptr mr_p, mpfr_ptr mi_p, mpfr_ptr mr_m, mpfr_ptr mi_m) {
  mpfr_ptr sr = c->t[5], si = c->t[6], dr = c->t[7], di = c->t[8];
  mpfr_add(sr, mr_p, mr_m, RN);
  mpfr_sub(dr, mr_p, mr_m, RN);
  mpfr_add(si, mi_p, mi_m, RN);
  mpfr_sub(di, mi_p, mi_m, RN);
  mpfr_sub(yr[k + 2 * q], yr[k], sr, RN);
  mpfr_add(yr[k], yr[k], sr, RN);
  mpfr_sub(yr[k + 3 * q], yr[k + q], di, RN);
  mpfr_add(yr[k + q], yr[k + q], di, RN);
  mpfr_sub(yi[k + 2 * q], yi[k], si, RN);
  mpfr_add(yi[k], yi[k], si, RN);
  mpfr_add(yi[k + 3 * q], yi[k + q], dr, RN);
  mpfr_sub(yi[k + q], yi[k + q], dr, RN);
  CNT(c, 0, 12, 0, 0);
}

/* X[k] = sum_j x[(sn + j*s) mod N] w_n^{jk}, k < n, written to y[0..n). */
OAPI void orc_mp_fft(orc_mp_ctx *c, unsigned long n, unsigned long s, long sn,
                     mpfr_t *xr, mpfr_t *xi, mpfr_t *yr, mpfr_t *yi) {
  CNT(c, 0, 0, 1, 0);
  if (n <= 4) {
    mp_leaf(c, n, s, sn, xr, xi, yr, yi);
    return;
  }
  unsigned long q = n / 4;
  /* even half, then the two conjugate-pair quarters (reference :180-182) */
  orc_mp_fft(c, n / 2, 2 * s, sn, xr, xi, yr, yi);
  orc_mp_fft(c, q, 4 * s, sn + (long)s, xr + s, xi + s, yr + 2 * q, yi + 2 * q);
  orc_mp_fft(c, q, 4 * s, sn - (long)s, xr - s, xi - s, yr + 3 * q, yi + 3 * q);

  mpfr_ptr tmp = c->t[0], pr = c->t[1], pi = c->t[2], mr = c->t[3], mi = c->t[4];
  /* k = 0: twiddle 1 (reference :184-201) */
  mp_combine(c, yr, yi, 0, q, yr[2 * q], yi[2 * q], yr[3 * q], yi[3 * q]);

  unsigned long stride = c->N / n;
  for (unsigned long k = 1; k < q; k++) {
    unsigned long kn = k * stride;
    mpfr_ptr zpr = yr[k + 2 * q], zpi = yi[k + 2 * q], zmr = yr[k + 3 * q], zmi = yi[k + 3 * q];
    if (2 * k == q) {
      /* w^k = (1-i)/sqrt2: four products by cos(pi/4) (reference :213-221) */
      mpfr_add(pr, zpr, zpi, RN); mpfr_mul(pr, pr, c->wr[kn], RN);
      mpfr_sub(pi, zpi, zpr, RN); mpfr_mul(pi, pi, c->wr[kn], RN);
      mpfr_sub(mr, zmr, zmi, RN); mpfr_mul(mr, mr, c->wr[kn], RN);
      mpfr_add(mi, zmr, zmi, RN); mpfr_mul(mi, mi, c->wr[kn], RN);
      CNT(c, 4, 4, 0, 0);
    } else {
      /* 3 mults + 3 adds per complex product, using cos+sin and cos-sin
       * (reference :222-236) */
      mpfr_mul(pr, c->wd[kn], zpi, RN);
      mpfr_mul(mr, c->wd[kn], zmi, RN);
      mpfr_mul(pi, c->ws[kn], zpr, RN);
      mpfr_mul(mi, c->ws[kn], zmr, RN);
      mpfr_add(tmp, zpr, zpi, RN); mpfr_mul(tmp, tmp, c->wr[kn], RN);
      mpfr_sub(pr, tmp, pr, RN); mpfr_sub(pi, tmp, pi, RN);
      mpfr_sub(tmp, zmr, zmi, RN); mpfr_mul(tmp, tmp, c->wr[kn], RN);
      mpfr_add(mr, tmp, mr, RN); mpfr_sub(mi, mi, tmp, RN);
      CNT(c, 6, 6, 0, 0);
    }
    mp_combine(c, yr, yi, k, q, pr, pi, mr, mi);
  }
}

/* Top-level convenience: full forward transform of n = N contiguous points. */
OAPI void orc_mp_fft_top(orc_mp_ctx *c, mpfr_t *xr, mpfr_t *xi, mpfr_t *yr, mpfr_t *yi) {
  orc_mp_fft(c, c->N, 1, 0, xr, xi, yr, yi);
}

/* ------------------------------------------------------------------------ */
/* the weighted power loss of the adjoint configuration                     */
/* ------------------------------------------------------------------------ */

/* Multiword views (the compensated tiers' formats): out[h*stride + k] = word
 * h of a[k], h < K -- the nearest double (or float, is_float) to a[k], then
 * the nearest to what is left, ...  set: a[k] = the words' exact sum rounded
 * to a's precision. */
OAPI void orc_mp_get_words(mpfr_t *a, unsigned long n, int K, int is_float, void *out, unsigned long stride) {
  mpfr_t t;
  mpfr_init2(t, 64);
  for (unsigned long k = 0; k < n; k++) {
    if (mpfr_get_prec(t) < mpfr_get_prec(a[k])) mpfr_set_prec(t, mpfr_get_prec(a[k]));
    mpfr_set(t, a[k], RN);
    for (int h = 0; h < K; h++) {
      double w = mpfr_get_d(t, RN);
      if (is_float) w = (double)(float)w;
      mpfr_sub_d(t, t, w, RN);
      if (is_float) ((float *)out)[h * stride + k] = (float)w;
      else ((double *)out)[h * stride + k] = w;
    }
  }
  mpfr_clear(t);
}

OAPI void orc_mp_set_words(mpfr_t *a, unsigned long n, int K, int is_float, const void *in, unsigned long stride) {
  mpfr_t acc;
  mpfr_init2(acc, 2200);
  for (unsigned long k = 0; k < n; k++) {
    mpfr_set_ui(acc, 0, RN);
    for (int h = 0; h < K; h++)
      mpfr_add_d(acc, acc, is_float ? (double)((const float *)in)[h * stride + k] : ((const double *)in)[h * stride + k],
                 RN);
    mpfr_set(a[k], acc, RN);
  }
  mpfr_clear(acc);
}

/* a[0] -= b[0] (rounded to a's precision) */
OAPI void orc_mp_sub_into(mpfr_t *a, mpfr_t *b) { mpfr_sub(a[0], a[0], b[0], RN); }

/* a[k] *= w[k] (rounded to a's precision) */
OAPI void orc_mp_mul_d(mpfr_t *a, const double *w, unsigned long n) {
  for (unsigned long k = 0; k < n; k++) mpfr_mul_d(a[k], a[k], w[k], RN);
}

/* out[0] = L(x) = sum_k w_k |X_k|^2 with X = the reference transform of x at
 * the context's precision (summed at out's precision) */
OAPI void orc_mp_power_loss(orc_mp_ctx *c, const double *w, mpfr_t *xr, mpfr_t *xi, mpfr_t *out) {
  const unsigned long n = c->N;
  mpfr_t *yr = orc_mp_alloc(n, c->P), *yi = orc_mp_alloc(n, c->P);
  orc_mp_fft(c, n, 1, 0, xr, xi, yr, yi);
  mpfr_t t, u;
  mpfr_inits2(mpfr_get_prec(out[0]), t, u, (mpfr_ptr)0);
  mpfr_set_ui(out[0], 0, RN);
  for (unsigned long k = 0; k < n; k++) {
    mpfr_mul(t, yr[k], yr[k], RN);
    mpfr_mul(u, yi[k], yi[k], RN);
    mpfr_add(t, t, u, RN);
    mpfr_mul_d(t, t, w[k], RN);
    mpfr_add(out[0], out[0], t, RN);
  }
  mpfr_clears(t, u, (mpfr_ptr)0);
  orc_mp_free(yr, n);
  orc_mp_free(yi, n);
}

/* Central difference of the loss above in component j (part 0 real, 1
 * imaginary) with step h = 2^h_exp:  out[0] = (L(x + h e) - L(x - h e)) / 2h.
 * L is quadratic in x, so the central difference has no truncation error:
 * out equals dL/dx_j up to the rounding of the two losses.  x is restored. */
OAPI void orc_mp_power_loss_fd(orc_mp_ctx *c, const double *w, mpfr_t *xr, mpfr_t *xi, unsigned long j, int part,
                               long h_exp, mpfr_t *out) {
  mpfr_ptr xj = part ? xi[j] : xr[j];
  const long pw = mpfr_get_prec(out[0]);
  mpfr_t save, lp, lm;
  mpfr_init2(save, mpfr_get_prec(xj));
  mpfr_inits2(pw, lp, lm, (mpfr_ptr)0);
  mpfr_set(save, xj, RN);
  mpfr_t h;
  mpfr_init2(h, 2);
  mpfr_set_ui_2exp(h, 1, h_exp, RN);
  mpfr_add(xj, save, h, RN);
  orc_mp_power_loss(c, w, xr, xi, &lp);
  mpfr_sub(xj, save, h, RN);
  orc_mp_power_loss(c, w, xr, xi, &lm);
  mpfr_set(xj, save, RN);
  mpfr_sub(out[0], lp, lm, RN);
  mpfr_div_2si(out[0], out[0], h_exp + 1, RN);
  mpfr_clears(save, lp, lm, h, (mpfr_ptr)0);
}

/* ------------------------------------------------------------------------ */
/* direct DFT at a chosen precision                                         */
/* ------------------------------------------------------------------------ */

/* y[k] = sum_j x[j] exp(-2 pi i jk/N), accumulated at prec+64+log2(N) bits
 * with twiddles cos/sin(2 pi m/N) at prec+64 bits, rounded once into y
 * (whose precision the caller chooses, typically 2P). */
OAPI void orc_mp_dft(unsigned long N, long prec, mpfr_t *xr, mpfr_t *xi, mpfr_t *yr, mpfr_t *yi) {
  long lg = 0;
  while ((1UL << lg) < N) lg++;
  long pw = prec + 64, pa = prec + 64 + lg + 2;
  mpfr_t *cw = orc_mp_alloc(N, pw), *sw = orc_mp_alloc(N, pw);
  {
    mpfr_t a, x;
    mpfr_inits2(pw + 16, a, x, (mpfr_ptr)0);
    mpfr_const_pi(a, RN);
    mpfr_mul_2ui(a, a, 1, RN);
    mpfr_div_ui(a, a, N, RN);
    for (unsigned long m = 0; m < N; m++) {
      mpfr_mul_ui(x, a, m, RN);
      mpfr_sin_cos(sw[m], cw[m], x, RN);
    }
    mpfr_clears(a, x, (mpfr_ptr)0);
  }
#pragma omp parallel
  {
    mpfr_t ar, ai, t;
    mpfr_inits2(pa, ar, ai, t, (mpfr_ptr)0);
#pragma omp for schedule(dynamic, 8)
    for (long k = 0; k < (long)N; k++) {
      mpfr_set_ui(ar, 0, RN);
      mpfr_set_ui(ai, 0, RN);
      for (unsigned long j = 0; j < N; j++) {
        unsigned long m = (j * (unsigned long)k) % N;
        /* (xr + i xi)(c - i s) = (xr c + xi s) + i (xi c - xr s) */
        mpfr_mul(t, xr[j], cw[m], RN); mpfr_add(ar, ar, t, RN);
        mpfr_mul(t, xi[j], sw[m], RN); mpfr_add(ar, ar, t, RN);
        mpfr_mul(t, xi[j], cw[m], RN); mpfr_add(ai, ai, t, RN);
        mpfr_mul(t, xr[j], sw[m], RN); mpfr_sub(ai, ai, t, RN);
      }
      mpfr_set(yr[k], ar, RN);
      mpfr_set(yi[k], ai, RN);
    }
    mpfr_clears(ar, ai, t, (mpfr_ptr)0);
    mpfr_free_cache();
  }
  orc_mp_free(cw, N);
  orc_mp_free(sw, N);
}

/* Multi-dimensional DFT of rank dimensions dims[0] x ... (row-major, last
 * index fastest) at precision prec: the direct DFT above along every axis in
 * turn, each line rounded into prec-bit intermediates. */
OAPI void orc_mp_dft_nd(int rank, const unsigned long *dims, long prec, mpfr_t *xr, mpfr_t *xi, mpfr_t *yr,
                        mpfr_t *yi) {
  unsigned long n = 1;
  for (int a = 0; a < rank; a++) n *= dims[a];
  for (unsigned long k = 0; k < n; k++) {
    mpfr_set(yr[k], xr[k], RN);
    mpfr_set(yi[k], xi[k], RN);
  }
  unsigned long stride = n;
  for (int a = 0; a < rank; a++) {
    const unsigned long d = dims[a];
    stride /= d;  /* distance between consecutive points of axis a */
    const unsigned long outer = n / (d * stride);
    mpfr_t *lr = orc_mp_alloc(d, prec), *li = orc_mp_alloc(d, prec);
    mpfr_t *tr = orc_mp_alloc(d, prec), *ti = orc_mp_alloc(d, prec);
    for (unsigned long o = 0; o < outer; o++)
      for (unsigned long q = 0; q < stride; q++) {
        const unsigned long base = o * d * stride + q;
        for (unsigned long j = 0; j < d; j++) {
          mpfr_set(lr[j], yr[base + j * stride], RN);
          mpfr_set(li[j], yi[base + j * stride], RN);
        }
        orc_mp_dft(d, prec, lr, li, tr, ti);
        for (unsigned long j = 0; j < d; j++) {
          mpfr_set(yr[base + j * stride], tr[j], RN);
          mpfr_set(yi[base + j * stride], ti[j], RN);
        }
      }
    orc_mp_free(lr, d);
    orc_mp_free(li, d);
    orc_mp_free(tr, d);
    orc_mp_free(ti, d);
  }
}

/* ------------------------------------------------------------------------ */
/* error metrics                                                            */
/* ------------------------------------------------------------------------ */

static double log2_of(mpfr_srcptr x) {
  if (mpfr_zero_p(x)) return -INFINITY;
  if (!mpfr_number_p(x)) return INFINITY;
  long e;
  double d = mpfr_get_d_2exp(&e, x, RN);
  return (double)e + log2(fabs(d));
}

/* out[0] = log2( max_k max(|dRe|,|dIm|) / max_k max(|refRe|,|refIm|) )
 *          (normwise relative error of (yr,yi) against the reference)
 * out[1], out[2] = log2 rRMSE of the real / imaginary parts
 *          (the reference's test() measure, parallel_mp_fft2.c:466-473)
 * out[3] = log2 max abs error, out[4] = log2 max |ref|.
 * Computed at a working precision wide enough to be exact for differences. */
OAPI void orc_mp_errors(unsigned long n, mpfr_t *yr, mpfr_t *yi, mpfr_t *rr, mpfr_t *ri, double *out) {
  long pw = 64;
  for (unsigned long k = 0; k < n; k++) {
    long p1 = mpfr_get_prec(yr[k]), p2 = mpfr_get_prec(rr[k]);
    if (p1 + 64 > pw) pw = p1 + 64;
    if (p2 + 64 > pw) pw = p2 + 64;
  }
  pw += 64;
  mpfr_t d, a, maxd, maxr, sdr, sdi, srr, sri, t;
  mpfr_inits2(pw, d, a, maxd, maxr, sdr, sdi, srr, sri, t, (mpfr_ptr)0);
  mpfr_set_ui(maxd, 0, RN); mpfr_set_ui(maxr, 0, RN);
  mpfr_set_ui(sdr, 0, RN); mpfr_set_ui(sdi, 0, RN);
  mpfr_set_ui(srr, 0, RN); mpfr_set_ui(sri, 0, RN);
  int bad = 0;
  for (unsigned long k = 0; k < n; k++) {
    for (int part = 0; part < 2; part++) {
      mpfr_ptr y = part ? yi[k] : yr[k], r = part ? ri[k] : rr[k];
      if (!mpfr_number_p(y) || !mpfr_number_p(r)) { bad = 1; continue; }
      mpfr_sub(d, y, r, RN);
      mpfr_abs(a, d, RN);
      if (mpfr_cmp(a, maxd) > 0) mpfr_set(maxd, a, RN);
      mpfr_abs(a, r, RN);
      if (mpfr_cmp(a, maxr) > 0) mpfr_set(maxr, a, RN);
      mpfr_mul(t, d, d, RN);
      mpfr_add(part ? sdi : sdr, part ? sdi : sdr, t, RN);
      mpfr_mul(t, r, r, RN);
      mpfr_add(part ? sri : srr, part ? sri : srr, t, RN);
    }
  }
  double lmd = log2_of(maxd), lmr = log2_of(maxr);
  out[0] = bad ? INFINITY : lmd - lmr;
  out[1] = bad ? INFINITY : 0.5 * (log2_of(sdr) - log2_of(srr));
  out[2] = bad ? INFINITY : 0.5 * (log2_of(sdi) - log2_of(sri));
  out[3] = bad ? INFINITY : lmd;
  out[4] = lmr;
  mpfr_clears(d, a, maxd, maxr, sdr, sdi, srr, sri, t, (mpfr_ptr)0);
}

/* ------------------------------------------------------------------------ */
/* FP64 conjugate-pair split-radix FFT (4m2a, n=8/16 base cases)            */
/* ------------------------------------------------------------------------ */

typedef struct {
  unsigned long N;
  double *wr, *wi;
  double c8, c16a, c16b, c16c, c16d; /* cos(pi/4), cos(pi/8), cos(pi/8)-cos(3pi/8), cos(3pi/8), cos(pi/8)+cos(3pi/8) */
  unsigned long cnt[4];
  int count;
} orc_d_ctx;

/* Twiddles exactly as the reference lut() (serial_d_fft6.c:52-62). */
OAPI orc_d_ctx *orc_d_new(unsigned long N) {
  orc_d_ctx *c = (orc_d_ctx *)calloc(1, sizeof *c);
  c->N = N;
  unsigned long q = N / 4;
  c->wr = (double *)malloc((q ? q : 1) * sizeof(double));
  c->wi = (double *)malloc((q ? q : 1) * sizeof(double));
  for (unsigned long k = 0; k < q; k++) {
    c->wr[k] = cos(2. * M_PI * k / N);
    c->wi[k] = sin(2. * M_PI * k / N);
  }
  c->c8 = cos(2. * M_PI * 1 / 8);
  c->c16a = cos(2. * M_PI * 1 / 16);
  c->c16b = cos(2. * M_PI * 1 / 16) - cos(2. * M_PI * 3 / 16);
  c->c16c = cos(2. * M_PI * 3 / 16);
  c->c16d = cos(2. * M_PI * 1 / 16) + cos(2. * M_PI * 3 / 16);
  return c;
}

OAPI void orc_d_delete(orc_d_ctx *c) {
  if (!c) return;
  free(c->wr);
  free(c->wi);
  free(c);
}

OAPI void orc_d_counts(orc_d_ctx *c, unsigned long *out4, int reset, int enable) {
  if (out4) memcpy(out4, c->cnt, sizeof c->cnt);
  if (reset) memset(c->cnt, 0, sizeof c->cnt);
  c->count = enable;
}

OAPI void orc_d_twiddles(orc_d_ctx *c, double *out5) {
  out5[0] = c->c8; out5[1] = c->c16a; out5[2] = c->c16b; out5[3] = c->c16c; out5[4] = c->c16d;
}

/* 8-point kernel on one part (re or im) of the inputs: returns the
 * intermediate values b1..b8 of serial_d_fft6.c:153-191 in v[0..7]. */
static void d8_part(const orc_d_ctx *c, const double *x /* 8 */, double *v) {
  double s04 = x[0] + x[4], d04 = x[0] - x[4];
  double s26 = x[2] + x[6], d26 = x[2] - x[6];
  double s17 = x[1] + x[7], d17 = x[1] - x[7];
  double s35 = x[3] + x[5], d35 = x[3] - x[5];
  double p = c->c8 * (d17 + d35);
  double q = c->c8 * (s17 - s35);
  v[0] = s17 + s35; /* b1 */
  v[1] = s04 + s26; /* b2 */
  v[2] = s04 - s26; /* b3 */
  v[3] = d17 - d35; /* b4 */
  v[4] = d04 + q;   /* b5 */
  v[5] = d04 - q;   /* b6 */
  v[6] = d26 + p;   /* b7 */
  v[7] = d26 - p;   /* b8 */
}

static void d_leaf8(const orc_d_ctx *c, const double *xr, const double *xi, double *yr, double *yi) {
  double R[8], I[8];
  d8_part(c, xr, R);
  d8_part(c, xi, I);
  /* outputs (serial_d_fft6.c:193-209) */
  yr[0] = R[1] + R[0]; yr[4] = R[1] - R[0];
  yi[0] = I[1] + I[0]; yi[4] = I[1] - I[0];
  yr[1] = R[4] + I[6]; yr[7] = R[4] - I[6];
  yi[1] = I[4] - R[6]; yi[7] = I[4] + R[6];
  yr[2] = R[2] + I[3]; yr[6] = R[2] - I[3];
  yi[2] = I[2] - R[3]; yi[6] = I[2] + R[3];
  yr[3] = R[5] - I[7]; yr[5] = R[5] + I[7];
  yi[3] = I[5] + R[7]; yi[5] = I[5] - R[7];
}

/* 16-point kernel on one part: the reference's n=16 base case
 * (serial_d_fft6.c:218-348).  `im` selects the imaginary-part variant, whose
 * a10, b3, b12 and m2, m4, m5, m7 enter with opposite signs.  Returns the
 * quantities the output stage needs: b5 b6 b11 b12 c1..c4 c9..c12 c17..c20. */
typedef struct { double b5, b6, b11, b12, c1, c2, c3, c4, c9, c10, c11, c12, c17, c18, c19, c20; } d16v;

static void d16_part(const orc_d_ctx *c, const double *x /* 16 */, int im, d16v *o) {
  double s[8], d[8];
  for (int j = 0; j < 8; j++) { s[j] = x[j] + x[j + 8]; d[j] = x[j] - x[j + 8]; }
  /* the imaginary variant uses a10 = x12 - x4 */
  double a10 = im ? (-x[4] + x[12]) : d[4];
  double b1 = s[0] - s[4], b2 = s[0] + s[4];
  double b3 = im ? (-s[2] + s[6]) : (s[2] - s[6]);
  double b4 = s[2] + s[6];
  double b7 = s[1] - s[5], b8 = s[1] + s[5];
  double b9 = s[3] - s[7], b10 = s[3] + s[7];
  double b13 = d[1] + d[7], b14 = d[1] - d[7];
  double b15 = d[3] + d[5], b16 = d[5] - d[3];
  o->b5 = b2 + b4;
  o->b6 = b2 - b4;
  o->b11 = b8 + b10;
  o->b12 = im ? (-b8 + b10) : (b8 - b10);
  double m1 = c->c8 * (d[2] - d[6]);
  double m2 = (im ? -c->c8 : c->c8) * (d[2] + d[6]);
  double m3 = c->c8 * (b7 - b9);
  double m4 = (im ? -c->c8 : c->c8) * (b7 + b9);
  double m5 = (im ? -c->c16a : c->c16a) * (b13 + b15);
  double m6 = (im ? c->c16b : -c->c16b) * b13;
  double m7 = (im ? -c->c16d : c->c16d) * b15;
  double m8 = c->c16c * (b14 + b16);
  double m9 = c->c16d * b14;
  double m10 = -c->c16b * b16;
  o->c1 = b1 + m3;
  o->c2 = b1 - m3;
  o->c3 = b3 + m4;
  o->c4 = m4 - b3;
  double c5 = d[0] + m1, c6 = d[0] - m1;
  double c7 = m9 - m8, c8 = m10 - m8;
  o->c9 = c5 + c7;
  o->c10 = c5 - c7;
  o->c11 = c6 + c8;
  o->c12 = c6 - c8;
  double c13 = a10 + m2, c14 = a10 - m2;
  double c15 = m5 + m6, c16 = m5 - m7;
  o->c17 = c13 + c15;
  o->c18 = c13 - c15;
  o->c19 = c14 + c16;
  o->c20 = c14 - c16;
}

static void d_leaf16(const orc_d_ctx *c, const double *xr, const double *xi, double *yr, double *yi) {
  d16v R, I;
  d16_part(c, xr, 0, &R);
  d16_part(c, xi, 1, &I);
  /* output stage (serial_d_fft6.c:350-382) */
  yr[0] = R.b5 + R.b11;   yr[8] = R.b5 - R.b11;
  yi[0] = I.b5 + I.b11;   yi[8] = I.b5 - I.b11;
  yr[4] = R.b6 - I.b12;   yr[12] = R.b6 + I.b12;
  yi[4] = I.b6 - R.b12;   yi[12] = I.b6 + R.b12;
  yr[1] = R.c9 - I.c17;   yr[15] = R.c9 + I.c17;
  yi[1] = I.c9 - R.c17;   yi[15] = I.c9 + R.c17;
  yr[2] = R.c1 - I.c3;    yr[14] = R.c1 + I.c3;
  yi[2] = I.c1 - R.c3;    yi[14] = I.c1 + R.c3;
  yr[3] = R.c12 + I.c20;  yr[13] = R.c12 - I.c20;
  yi[3] = I.c12 + R.c20;  yi[13] = I.c12 - R.c20;
  yr[5] = R.c11 - I.c19;  yr[11] = R.c11 + I.c19;
  yi[5] = I.c11 - R.c19;  yi[11] = I.c11 + R.c19;
  yr[6] = R.c2 - I.c4;    yr[10] = R.c2 + I.c4;
  yi[6] = I.c2 - R.c4;    yi[10] = I.c2 + R.c4;
  yr[7] = R.c10 + I.c18;  yr[9] = R.c10 - I.c18;
  yi[7] = I.c10 + R.c18;  yi[9] = I.c10 - R.c18;
}

OAPI void orc_d_fft(orc_d_ctx *c, unsigned long n, unsigned long s, long sn,
                    const double *xr, const double *xi, double *yr, double *yi) {
  CNT(c, 0, 0, 1, 0);
  unsigned long j0 = sn < 0 ? c->N : 0;
  if (n <= 16) {
    /* gather the strided subsequence (element 0 wrapped when sn<0) */
    double gr[16], gi[16];
    gr[0] = xr[j0]; gi[0] = xi[j0];
    for (unsigned long j = 1; j < n; j++) { gr[j] = xr[j * s]; gi[j] = xi[j * s]; }
    if (n == 1) {
      yr[0] = gr[0]; yi[0] = gi[0];
      CNT(c, 0, 0, 0, 1);
    } else if (n == 2) {
      yr[0] = gr[0] + gr[1]; yr[1] = gr[0] - gr[1];
      yi[0] = gi[0] + gi[1]; yi[1] = gi[0] - gi[1];
      CNT(c, 0, 4, 0, 1);
    } else if (n == 4) {
      double er = gr[0] + gr[2], fr = gr[0] - gr[2], gr2 = gr[1] + gr[3], hr = gr[1] - gr[3];
      double ei = gi[0] + gi[2], fi = gi[0] - gi[2], gi2 = gi[1] + gi[3], hi = gi[1] - gi[3];
      yr[0] = er + gr2; yr[1] = fr + hi; yr[2] = er - gr2; yr[3] = fr - hi;
      yi[0] = ei + gi2; yi[1] = fi - hr; yi[2] = ei - gi2; yi[3] = fi + hr;
      CNT(c, 0, 16, 0, 1);
    } else if (n == 8) {
      d_leaf8(c, gr, gi, yr, yi);
      CNT(c, 4, 52, 0, 1);
    } else {
      d_leaf16(c, gr, gi, yr, yi);
      CNT(c, 20, 148, 0, 1);
    }
    return;
  }
  unsigned long q = n / 4;
  orc_d_fft(c, n / 2, 2 * s, sn, xr, xi, yr, yi);
  orc_d_fft(c, q, 4 * s, sn + (long)s, xr + s, xi + s, yr + 2 * q, yi + 2 * q);
  orc_d_fft(c, q, 4 * s, sn - (long)s, xr - s, xi - s, yr + 3 * q, yi + 3 * q);
  unsigned long stride = c->N / n;
  /* one 4m2a butterfly for every k, twiddle (1,0) included
   * (serial_d_fft6.c:392-427) */
  for (unsigned long k = 0; k < q; k++) {
    double w_r = c->wr[k * stride], w_i = c->wi[k * stride];
    double u0r = yr[k], u1r = yr[k + q], zpr = yr[k + 2 * q], zmr = yr[k + 3 * q];
    double u0i = yi[k], u1i = yi[k + q], zpi = yi[k + 2 * q], zmi = yi[k + 3 * q];
    double pr = w_r * zpr + w_i * zpi, pi = w_r * zpi - w_i * zpr;
    double mr = w_r * zmr - w_i * zmi, mi = w_r * zmi + w_i * zmr;
    double sr = pr + mr, si = pi + mi, dr = pr - mr, di = pi - mi;
    yr[k] = u0r + sr; yr[k + 2 * q] = u0r - sr;
    yr[k + q] = u1r + di; yr[k + 3 * q] = u1r - di;
    yi[k] = u0i + si; yi[k + 2 * q] = u0i - si;
    yi[k + q] = u1i - dr; yi[k + 3 * q] = u1i + dr;
    CNT(c, 8, 16, 0, 0);
  }
}

OAPI void orc_d_fft_top(orc_d_ctx *c, const double *xr, const double *xi, double *yr, double *yi) {
  orc_d_fft(c, c->N, 1, 0, xr, xi, yr, yi);
}

/* seeded uniform [-1,1) doubles: splitmix64 stream, 53-bit mantissas */
OAPI void orc_d_fill_uniform(double *re, double *im, unsigned long n, unsigned long seed) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ULL + 1;
  for (unsigned long k = 0; k < 2 * n; k++) {
    z += 0x9E3779B97F4A7C15ULL;
    uint64_t x = z;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    x ^= x >> 31;
    double u = (double)(x >> 11) * (1.0 / 9007199254740992.0);
    double v = 2.0 * u - 1.0;
    if (k & 1) im[k >> 1] = v; else re[k >> 1] = v;
  }
}

/* ------------------------------------------------------------------------ */
/* misc                                                                     */
/* ------------------------------------------------------------------------ */

OAPI const char *orc_mpfr_version(void) { return mpfr_get_version(); }

OAPI unsigned long long orc_now_ns(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (unsigned long long)t.tv_sec * 1000000000ULL + (unsigned long long)t.tv_nsec;
}

/* ------------------------------------------------------------------------ */
/* raw significand fields (for tests of device-resident significand APIs)   */
/* ------------------------------------------------------------------------ */

/* Component order (c, p, b) -> index (c*n + p)*batch + b, where re = a_re and
 * im = a_im hold `batch` signals of n points (signal b at [b*n, (b+1)*n)).
 * mant: nl 64-bit limbs per component; ex: exponent or INT64_MIN for zero;
 * sg: 1 for negative.  Returns 0, or -1 if an element is NaN/Inf or has
 * more than nl limbs. */
OAPI int orc_mp_export_raw(mpfr_t *a_re, mpfr_t *a_im, unsigned long n, unsigned long batch, int nl,
                           uint64_t *mant, int64_t *ex, uint8_t *sg) {
  for (unsigned long b = 0; b < batch; b++)
    for (int c = 0; c < 2; c++)
      for (unsigned long p = 0; p < n; p++) {
        mpfr_ptr x = (c ? a_im : a_re)[b * n + p];
        size_t t = ((size_t)c * n + p) * batch + b;
        int xl = (int)((mpfr_get_prec(x) + 63) / 64);
        if (!mpfr_number_p(x) || xl > nl) return -1;
        memset(mant + t * nl, 0, (size_t)nl * 8);
        if (mpfr_zero_p(x)) {
          ex[t] = INT64_MIN;
          sg[t] = 0;
        } else {
          /* left-align the significand in nl limbs */
          memcpy(mant + t * nl + (nl - xl), x->_mpfr_d, (size_t)xl * 8);
          ex[t] = x->_mpfr_exp;
          sg[t] = x->_mpfr_sign < 0;
        }
      }
  return 0;
}

/* inverse of orc_mp_export_raw: value = sign * 0.mant * 2^ex, rounded into
 * each destination element at its own precision */
OAPI void orc_mp_import_raw(mpfr_t *a_re, mpfr_t *a_im, unsigned long n, unsigned long batch, int nl,
                            const uint64_t *mant, const int64_t *ex, const uint8_t *sg) {
  for (unsigned long b = 0; b < batch; b++)
    for (int c = 0; c < 2; c++)
      for (unsigned long p = 0; p < n; p++) {
        mpfr_ptr y = (c ? a_im : a_re)[b * n + p];
        size_t t = ((size_t)c * n + p) * batch + b;
        if (ex[t] == INT64_MIN) {
          mpfr_set_zero(y, 1);
          continue;
        }
        __mpz_struct z;
        z._mp_alloc = nl;
        z._mp_size = sg[t] ? -nl : nl;
        z._mp_d = (mp_limb_t *)(mant + t * nl);
        mpfr_set_z_2exp(y, &z, (mpfr_exp_t)(ex[t] - 64L * nl), RN);
      }
}
