/*
 * Test-oracle shim: compiles ONE unmodified reference FFT code file of mpFFT
 * (selected by -DREF_SOURCE="<path>") into a shared library with a small C
 * API, so tests and the CPU baseline can run the reference's own
 * implementation on chosen inputs.
 *
 * The reference configures N, P, IN, CC, ... as compile-time macros
 * (mpFFT.c:11-41, lab/serial/mp/serial_mp_main.c:9-42).  Here they expand
 * to file-level variables so one build serves every (N, P).  The reference's
 * globals (LUT*, in*, out*, temporaries, counters) stay in this translation
 * unit with hidden visibility; only the ref_* entry points below are exported.
 *
 * Build flags: -DREF_MP (multiprecision file) or not (double file),
 * -DREF_V2 for the *_v2 (pass-by-shift twiddle index) variants.
 *
 * Test infrastructure only.  Never linked into the product library.
 */
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>
#include <gmp.h>  /* our stand-in headers (oracle/include) */
#include <mpfr.h>

/* Everything the reference defines or declares gets hidden visibility; the
 * library and system headers above keep their default visibility. */
#pragma GCC visibility push(hidden)

#include "mpFFT.h" /* reference header (-I<reference root>) */

static unsigned long ref_N = 1;
static unsigned long ref_P = 64;
static int ref_IN = 1;
static int ref_CC = 0;

#define N ref_N
#define P ref_P
#define M 1
#define IN ref_IN
#define R MPFR_RNDN
#define CC ref_CC
#define CH 0
#define Q 150
#define PRA 0
#define PRB 0
#define PRC 0

#if defined(REF_MP)
#if defined(REF_V2)
#define FFT mp_sr24_cp_fft_v2(N, 0, 1, 0, inr, ini, outr, outi);
#else
#define FFT mp_sr24_cp_fft(N, 1, 0, inr, ini, outr, outi);
#endif
#else
#if defined(REF_V2)
#define FFT d_sr24_cp_fft_v2(N, 0, 1, 0, inr, ini, outr, outi);
#else
#define FFT d_sr24_cp_fft(N, 1, 0, inr, ini, outr, outi);
#endif
#endif

#include REF_SOURCE

#pragma GCC visibility pop

#define REF_API __attribute__((visibility("default")))

static int ref_ready = 0;

/* Allocate the reference's arrays and build its twiddle LUT for (n, prec).
 * prec is ignored by the double files. */
REF_API int ref_init(unsigned long n, unsigned long prec) {
  if (ref_ready) return -1;
  ref_N = n;
  ref_P = prec;
  create_memory();
  lut();
  ref_ready = 1;
  return 0;
}

/* Fill the inputs with the reference's own initial condition ic():
 * IN 1 = seeded uniform [0,1), IN 2 = 1/(1+k^2), 1/(1+k^4). */
REF_API void ref_ic(int in, unsigned long s) {
  ref_IN = in;
  seed = (time_t)s;
  ic();
}

/* 0..3 -> inr, ini, outr, outi (mpfr_t* or double*). */
REF_API void *ref_array(int which) {
  switch (which) {
    case 0: return (void *)inr;
    case 1: return (void *)ini;
    case 2: return (void *)outr;
    default: return (void *)outi;
  }
}

REF_API void ref_set_cc(int on) {
  ref_CC = on;
  cmul = cadd = cfc = crb = 0;
}

REF_API void ref_counts(unsigned long *out4) {
  out4[0] = cmul;
  out4[1] = cadd;
  out4[2] = cfc;
  out4[3] = crb;
}

/* Run the reference transform m times on the current inputs; returns ns. */
REF_API unsigned long long ref_run(unsigned long m) {
  unsigned long long t0 = get_time_int();
  for (unsigned long i = 0; i < m; i++) { FFT }
  return get_time_int() - t0;
}

REF_API void ref_free(void) {
  if (!ref_ready) return;
  clear_memory();
  ref_ready = 0;
}
