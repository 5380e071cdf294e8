/*
 * A plain C program that calls libmpfft_b200 through include/mpfft_b200.h,
 * the way the reference's production driver calls its transform (mpFFT.c:47-91):
 *
 *   - four arrays of N mpfr_t initialised with mpfr_inits2 at precision P
 *     (create_memory, lab/parallel/mp/parallel_mp_fft2.c:55-67);
 *   - the reference's deterministic input IN 2, re = 1/(1+k^2),
 *     im = 1/(1+k^4) (ic(), lab/parallel/mp/parallel_mp_fft2.c:104-114);
 *   - one call  mp_sr24_cp_fft(N, 1, 0, inr, ini, outr, outi)  (the FFT macro,
 *     mpFFT.c:47), then the double transform d_sr24_cp_fft on the same input
 *     rounded to double (mpFFT.h:25).
 *
 * Prints "mp <k> <re> <im>" (MPFR "%Ra" hexadecimal, exact) for every mp
 * output and "d <k> <re> <im>" (C99 "%a") for every double output, so that a
 * test can compare them with the oracle.  Exit status 0 on success, 2 when the
 * library reports an error (message on stderr).
 *
 * Usage: mpfft_caller N P
 */
#include <stdio.h>
#include <stdlib.h>

#include "mpfft_b200.h"

int main(int argc, char **argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s N P\n", argv[0]);
    return 1;
  }
  const unsigned long N = strtoul(argv[1], NULL, 10);
  const long P = strtol(argv[2], NULL, 10);
  mpfr_t *inr = malloc(N * sizeof(mpfr_t)), *ini = malloc(N * sizeof(mpfr_t));
  mpfr_t *outr = malloc(N * sizeof(mpfr_t)), *outi = malloc(N * sizeof(mpfr_t));
  double *dr = malloc(N * sizeof(double)), *di = malloc(N * sizeof(double));
  double *er = malloc(N * sizeof(double)), *ei = malloc(N * sizeof(double));
  if (!inr || !ini || !outr || !outi || !dr || !di || !er || !ei) return 1;
  for (unsigned long k = 0; k < N; k++) mpfr_inits2(P, inr[k], ini[k], outr[k], outi[k], (mpfr_ptr)0);
  mpfr_t aux;
  mpfr_init2(aux, P);
  for (unsigned long k = 0; k < N; k++) {
    mpfr_set_ui(aux, k * k, MPFR_RNDN);
    mpfr_add_ui(inr[k], aux, 1, MPFR_RNDN);
    mpfr_ui_div(inr[k], 1, inr[k], MPFR_RNDN);
    mpfr_mul(aux, aux, aux, MPFR_RNDN);
    mpfr_add_ui(ini[k], aux, 1, MPFR_RNDN);
    mpfr_ui_div(ini[k], 1, ini[k], MPFR_RNDN);
    dr[k] = mpfr_get_d(inr[k], MPFR_RNDN);
    di[k] = mpfr_get_d(ini[k], MPFR_RNDN);
  }
  mpfr_clear(aux);

  mp_sr24_cp_fft(N, 1, 0, inr, ini, outr, outi);
  if (mpfft_last_error() != MPFFT_OK) {
    fprintf(stderr, "mp_sr24_cp_fft: %d %s\n", mpfft_last_error(), mpfft_last_error_string());
    return 2;
  }
  d_sr24_cp_fft(N, 1, 0, dr, di, er, ei);
  if (mpfft_last_error() != MPFFT_OK) {
    fprintf(stderr, "d_sr24_cp_fft: %d %s\n", mpfft_last_error(), mpfft_last_error_string());
    return 2;
  }
  for (unsigned long k = 0; k < N; k++) mpfr_printf("mp %lu %Ra %Ra\n", k, outr[k], outi[k]);
  for (unsigned long k = 0; k < N; k++) printf("d %lu %a %a\n", k, er[k], ei[k]);
  for (unsigned long k = 0; k < N; k++) mpfr_clears(inr[k], ini[k], outr[k], outi[k], (mpfr_ptr)0);
  free(inr), free(ini), free(outr), free(outi), free(dr), free(di), free(er), free(ei);
  return 0;
}
