/*
 * libmpfft_b200 -- B200 (sm_100a) implementation of mpFFT's conjugate-pair
 * split-radix 2/4 DIT complex FFT, behind mpFFT's own C API.
 *
 * Two groups of entry points:
 *
 * 1. Drop-in replacements for the reference prototypes in mpFFT.h.  Same
 *    names, argument meaning and out-of-place semantics; they return void as
 *    the reference does and record a status readable with mpfft_last_error().
 *    Only the top-level form is meaningful to an external caller (the
 *    reference's own callers use (N,1,0,...), mpFFT.c:47,50): any power-of-two
 *    n >= 1, any input stride s >= 1, sn >= 0 (element j read at in[j*s]).
 *    A negative sn is the reference's internal wrap to its global N and is
 *    rejected with MPFFT_EINVAL.  On any error the outputs are set to NaN.
 *
 * 2. An explicit plan/execute API with int status returns, batched execution
 *    over many signals, device-resident limb planes (no mpfr_t conversion),
 *    and scaled (1/N) output.
 *
 * Multiprecision numbers: the working precision P of a drop-in call is the
 * largest precision among inr[0], ini[0], outr[0], outi[0]; each output
 * element is rounded to nearest at its own precision (as MPFR rounds to the
 * destination).  The device keeps one exponent per signal and fixed-point
 * 32-bit limbs with P + log2(N) + 4 or more fraction bits; additions are
 * exact and each twiddle product is rounded once, so the normwise error is
 * below the reference's own at the same P.
 *
 * Thread safety: every entry point may be called from any host thread and,
 * for the asynchronous device-layout entries, on any stream.  Host-side work
 * of calls on the same plan is serialised.  Where a plan keeps internal device
 * scratch (multi-dimensional plans, large limb counts, real FP64 plans), the
 * device work of its calls is also ordered: a call's stream first waits on the
 * GPU for the previous call that used the scratch, so calls on different
 * streams give the same results as calls made one after another.
 */
#ifndef MPFFT_B200_H
#define MPFFT_B200_H

#include <stdint.h>

#ifndef MPFFT_MPFR_TYPES_PROVIDED
#include <mpfr.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define MPFFT_OK 0
#define MPFFT_EINVAL 1       /* bad argument (n not a power of two, s == 0, sn < 0, NULL, ...) */
#define MPFFT_EUNSUPPORTED 2 /* valid but not supported by this build (e.g. precision too large for n) */
#define MPFFT_ENONFINITE 3   /* NaN or infinity among the inputs */
#define MPFFT_ECUDA 4        /* CUDA runtime error (no device, launch failure, ...) */
#define MPFFT_ENOMEM 5       /* host or device allocation failed */

/* flags */
#define MPFFT_SCALED 1u         /* execute: multiply the result by 1/n (exact) */
#define MPFFT_INVERSE 8u        /* execute (host arrays, FP64 device planes): backward transform,
                                   exp(+2 pi i jk/n); unscaled it is the adjoint (conjugate transpose) */
#define MPFFT_PLAN_HOST_ONLY 2u /* plan creation: conversion (pack/unpack) only, no device state */
#define MPFFT_PLAN_HOST_CONVERSION 4u /* plan creation: convert mpfr_t <-> limbs on the host, not the GPU */
#define MPFFT_PLAN_NO_TENSOR 16u /* plan creation: keep large-precision twiddle products on the integer
                                     pipes (by default 35..260 limbs use int8 tensor-core GEMMs) */
#define MPFFT_PLAN_TENSOR 32u    /* plan creation: tensor-core twiddle products from 8 limbs up */
#define MPFFT_PLAN_FLOAT_TIERS 64u /* plan creation: run host-array transforms of precisions up to 200 bits on a
                                       compensated floating-point tier (see mpfft_mp_plan_form) */
#define MPFFT_PLAN_NATIVE_TIERS 128u /* plan creation: precisions up to 212 bits on the smallest floating word format
                                         holding P bits (float-float 48, FP64 53, double-double 106,
                                         quad-double 212), with that tier's own error */

/* the form an mp plan's host-array transforms run in (mpfft_mp_plan_form) */
#define MPFFT_FORM_LIMBS 0         /* fixed-point 32-bit limbs, integer pipes */
#define MPFFT_FORM_TENSOR 1        /* fixed-point limbs, twiddle products as int8 tensor-core GEMMs */
#define MPFFT_FORM_FLOAT_FLOAT 2   /* float pairs, additions on the FP32 pipe, products in FP64 (P <= 40) */
#define MPFFT_FORM_DOUBLE 3        /* the reference's double transform (40 < P <= 48) */
#define MPFFT_FORM_DOUBLE_DOUBLE 4 /* double-double (48 < P <= 98) */
#define MPFFT_FORM_QUAD_DOUBLE 5   /* quad-double (98 < P <= 200) */

/* ------------------------------------------------------------------------ */
/* 1. drop-in replacements for mpFFT.h                                      */
/* ------------------------------------------------------------------------ */

/* Replaces mp_sr24_cp_fft, mpFFT.h:38,66 (implemented by
 * lab/parallel/mp/parallel_mp_fft2.c:121-328 and
 * lab/serial/mp/serial_mp_fft3.c:121-253). */
void mp_sr24_cp_fft(unsigned long n, unsigned long s, long int sn, mpfr_t *inr, mpfr_t *ini, mpfr_t *outr,
                    mpfr_t *outi);

/* Replaces mp_sr24_cp_fft_v2, mpFFT.h:39 (lab/serial/mp/serial_mp_fft4.c:121-122):
 * the pass-by-shift twiddle-index variant; log2n must be 0 at the top level. */
void mp_sr24_cp_fft_v2(unsigned long n, unsigned long log2n, unsigned long s, long int sn, mpfr_t *inr,
                       mpfr_t *ini, mpfr_t *outr, mpfr_t *outi);

/* Scaled variant planned by the reference (README.md "unscaled and scaled"):
 * out = FFT(in) / n.  The reference normalises with mpfr_div_ui(out,out,N)
 * (lab/parallel/mp/parallel_mp_fft2.c:455); here the 1/n is an exact exponent
 * shift applied before the single rounding into each output. */
void mp_sr24_cp_fft_scaled(unsigned long n, unsigned long s, long int sn, mpfr_t *inr, mpfr_t *ini,
                           mpfr_t *outr, mpfr_t *outi);

/* Inverse transform, normalised: out = (1/n) sum_k in[k] exp(+2 pi i jk/n).  The
 * reference computes its inverse in test() as swap(re,im), forward transform,
 * swap back, divide by N (lab/parallel/mp/parallel_mp_fft2.c:441-455); this is
 * that procedure with the re/im swap done by addressing (no copies) and the
 * 1/n applied exactly before the single rounding into each output. */
void mp_sr24_cp_ifft(unsigned long n, unsigned long s, long int sn, mpfr_t *inr, mpfr_t *ini, mpfr_t *outr,
                     mpfr_t *outi);

/* Replaces d_sr24_cp_fft, mpFFT.h:25,53 (lab/serial/double/serial_d_fft6.c:93-429).
 * Results are bit-identical to the reference's double transform. */
void d_sr24_cp_fft(unsigned long n, unsigned long s, long int sn, double *inr, double *ini, double *outr,
                   double *outi);

/* Replaces d_sr24_cp_fft_v2, mpFFT.h:26 (lab/serial/double/serial_d_fft7.c:93-94). */
void d_sr24_cp_fft_v2(unsigned long n, unsigned long log2n, unsigned long s, long int sn, double *inr,
                      double *ini, double *outr, double *outi);

/* FP64 inverse, normalised; bit-identical to the reference's swap / forward /
 * swap / divide-by-N procedure (lab/serial/double/serial_d_fft6.c:511-524). */
void d_sr24_cp_ifft(unsigned long n, unsigned long s, long int sn, double *inr, double *ini, double *outr,
                    double *outi);

/* FP64 scaled variant: out = FFT(in) * (1/n), exact power-of-two scaling. */
void d_sr24_cp_fft_scaled(unsigned long n, unsigned long s, long int sn, double *inr, double *ini,
                          double *outr, double *outi);

/* Status of the last call made on this host thread (MPFFT_OK or an error
 * code) and a human-readable message.  The reference has no error reporting
 * (void returns, unchecked malloc); these are the drop-in's side channel. */
int mpfft_last_error(void);
const char *mpfft_last_error_string(void);

/* ------------------------------------------------------------------------ */
/* 2. explicit plan / execute API (no counterpart in the reference, which    */
/*    has compile-time N and P and file-static twiddle tables, lut() in      */
/*    lab/parallel/mp/parallel_mp_fft2.c:71-82)                              */
/* ------------------------------------------------------------------------ */

typedef struct mpfft_mp_plan mpfft_mp_plan;
typedef struct mpfft_d_plan mpfft_d_plan;

/* Plan a multiprecision transform of n points at working precision prec
 * bits.  Builds the twiddle tables with MPFR and uploads them once. */
int mpfft_mp_plan_create(mpfft_mp_plan **plan, unsigned long n, long prec);
/* same, with flags (MPFFT_PLAN_HOST_ONLY: pack/unpack only, needs no GPU) */
int mpfft_mp_plan_create_flags(mpfft_mp_plan **plan, unsigned long n, long prec, unsigned flags);
/* Multi-dimensional transform (iterated one-dimensional transforms; the
 * reference's README plans it but never built it): rank 1..3 dimensions
 * dims[0] x ... x dims[rank-1], each a power of two, N = their product (at most
 * 2^26).  A signal is N points in row-major order (last index fastest) in
 * every layout this header describes: host arrays, device limb planes (point
 * p = row-major index).  The limb format is that of an N-point plan; the
 * error bound is that of an N-point transform.  Per axis the device first
 * rotates that axis to the front (one transposition pass) and then runs the
 * one-dimensional kernels over all lines; a device buffer the size of the
 * signals is allocated on first use and kept.  flags as
 * mpfft_mp_plan_create_flags. */
int mpfft_mp_plan_create_nd(mpfft_mp_plan **plan, int rank, const unsigned long *dims, long prec, unsigned flags);
int mpfft_mp_plan_destroy(mpfft_mp_plan *plan);
/* device format of a plan: limbs per real component, fraction bits */
int mpfft_mp_plan_limbs(const mpfft_mp_plan *plan);
/* MPFFT_FORM_* of the plan's host-array transforms.  A plan created with
 * MPFFT_PLAN_FLOAT_TIERS whose precision a compensated floating-point tier
 * covers (normwise error within 8 log2(n) 2^-P, measured against the 2P-bit
 * oracle) converts mpfr_t values to that tier's words on the host and runs the
 * tier's kernels; calls whose inputs lie outside the tier's exponent window
 * run on the limbs instead.  The device-layout entry points always take limb
 * planes.  No counterpart in the reference. */
int mpfft_mp_plan_form(const mpfft_mp_plan *plan);
long mpfft_mp_plan_frac_bits(const mpfft_mp_plan *plan);

/* Transform `batch` signals held in host mpfr_t arrays: signal b occupies
 * elements [b*n, (b+1)*n) of each array.  Synchronous.  When every input has
 * the same number of significand limbs and every output the same precision,
 * the conversion to and from limb planes runs on the GPU (the host only copies
 * significand limbs); otherwise on the host.  Both give identical results. */
int mpfft_mp_execute(mpfft_mp_plan *plan, unsigned long batch, mpfr_t *inr, mpfr_t *ini, mpfr_t *outr,
                     mpfr_t *outi, unsigned flags);

/* Transform `batch` signals held on the device as limb planes: word
 * (c, i, p, b) at base[((c*L + i)*n + p)*batch + b], c = 0 real / 1 imaginary,
 * limb i < L (least significant first), two's complement.  in and out must
 * not overlap.  Asynchronous on `stream` (a cudaStream_t, NULL = default). */
int mpfft_mp_execute_device(mpfft_mp_plan *plan, unsigned long batch, const uint32_t *d_in, uint32_t *d_out,
                            void *stream);

/* Uneven batch (no counterpart in the reference): `count` signals of
 * different lengths n[i] (powers of two) and precisions; signal i occupies
 * inr[i][0..n[i]) etc., working precision the largest of its four arrays'
 * first elements.  Signals with the same length and limb count run as one
 * batched execution of a cached plan (GPU conversion pipeline included), so
 * each result is identical to a single call of the drop-in.  flags:
 * MPFFT_SCALED, MPFFT_INVERSE.  On error the failing groups' outputs are
 * NaN. */
int mpfft_mp_execute_mixed(unsigned long count, const unsigned long *n, mpfr_t *const *inr, mpfr_t *const *ini,
                           mpfr_t *const *outr, mpfr_t *const *outi, unsigned flags);

/* Real transforms (no counterpart in the reference, whose README lists
 * "only complex input"; a real signal there is a complex one with zero
 * imaginary parts).  A real plan for n real points (n a power of two, n >= 2)
 * runs one n/2-point complex transform plus one split step, about half the
 * work of the complex transform of the zero-padded signal.  The limb format
 * (mpfft_mp_plan_limbs/frac_bits) is that of an n-point complex plan, with up
 * to 34 limbs.  MPFFT_PLAN_HOST_CONVERSION is accepted; real plans have no
 * device-layout, pack/unpack or static-scratch entry points. */
int mpfft_mp_plan_create_real(mpfft_mp_plan **plan, unsigned long n, long prec, unsigned flags);
/* X_k = sum_j x_j exp(-2 pi i jk/n) for k = 0..n/2 of `batch` real signals:
 * signal b at in[b*n .. b*n+n-1], outputs at outr/outi[b*(n/2+1) + k]
 * (X_0 and X_(n/2) have zero imaginary parts).  MPFFT_SCALED: times 1/n.
 * Error bound and rounding as mpfft_mp_execute. */
int mpfft_mp_execute_r2c(mpfft_mp_plan *plan, unsigned long batch, mpfr_t *in, mpfr_t *outr, mpfr_t *outi,
                         unsigned flags);
/* Inverse: x_j = sum_(k<n) X_k exp(+2 pi i jk/n) with X_(n-k) = conj(X_k), from
 * the half spectrum inr/ini[b*(n/2+1) + k], k = 0..n/2, into out[b*n + j]
 * (MPFFT_SCALED: times 1/n, the exact inverse of mpfft_mp_execute_r2c).  The
 * imaginary parts of X_0 and X_(n/2) are ignored. */
int mpfft_mp_execute_c2r(mpfft_mp_plan *plan, unsigned long batch, mpfr_t *inr, mpfr_t *ini, mpfr_t *out,
                         unsigned flags);

/* Host-side conversion between mpfr_t arrays and the limb-plane layout
 * above.  exps[b] receives (pack) / supplies (unpack) the block exponent of
 * signal b: a component with fixed-point integer A has value
 * A * 2^(exps[b] - frac_bits).  unpack rounds to each output's precision. */
int mpfft_mp_pack(const mpfft_mp_plan *plan, unsigned long batch, mpfr_t *inr, mpfr_t *ini, uint32_t *planes,
                  long *exps);
int mpfft_mp_unpack(const mpfft_mp_plan *plan, unsigned long batch, const uint32_t *planes, const long *exps,
                    mpfr_t *outr, mpfr_t *outi, unsigned flags);

/* FP64 plans.  Host arrays: signal b at [b*n, (b+1)*n) of each array. */
int mpfft_d_plan_create(mpfft_d_plan **plan, unsigned long n);
/* Double-double tier (about 106 bits; no counterpart in the reference): the
 * same conjugate-pair split-radix transform with every value an unevaluated
 * sum hi + lo of two doubles and every operation a compensated double-double
 * one (error-free TwoSum / Fast2Sum / FMA TwoProd), twiddles rounded to
 * double-double.  Normwise error against an exact DFT about log2(n) * 2^-104
 * (tests bound it by 8 * log2(n) * 2^-104 against a 212-bit MPFR DFT).
 * Host arrays: signal b at [b*n, (b+1)*n) of each of the eight arrays;
 * flags MPFFT_SCALED (times 1/n, exact) and MPFFT_INVERSE.  Device layout:
 * word (c, h, b, p) at base[((c*2 + h)*batch + b)*n + p], c = 0 real / 1
 * imaginary, h = 0 high / 1 low part. */
int mpfft_dd_plan_create(mpfft_d_plan **plan, unsigned long n);
int mpfft_dd_execute(mpfft_d_plan *plan, unsigned long batch, const double *xr_hi, const double *xr_lo,
                     const double *xi_hi, const double *xi_lo, double *yr_hi, double *yr_lo, double *yi_hi,
                     double *yi_lo, unsigned flags);
int mpfft_dd_execute_device(mpfft_d_plan *plan, unsigned long batch, const double *d_in, double *d_out,
                            unsigned flags, void *stream);

/* Quad-double tier (about 212 bits; no counterpart in the reference): values
 * x0 + x1 + x2 + x3 of four doubles, each at most half an ulp of the one above;
 * additions and products summed order by order with error-free
 * transformations and renormalised (Hida, Li and Bailey's quad-double
 * algorithms).  Normwise error about log2(n) 2^-209.  Float-float tier (about
 * 48 bits): values hi + lo of two floats; additions on the FP32 pipe, every
 * twiddle product formed and renormalised in FP64.  Both take the layout of
 * the multiword entries below. */
int mpfft_qd_plan_create(mpfft_d_plan **plan, unsigned long n);
int mpfft_ff_plan_create(mpfft_d_plan **plan, unsigned long n);
/* Words per real component (K: 2 double-double, 4 quad-double, 2 float-float)
 * and bytes per word (8, or 4 for float-float) of a multiword plan. */
int mpfft_multiword_format(const mpfft_d_plan *plan, int *words, int *word_bytes);
/* Multiword plans (double-double, quad-double, float-float): word h of the
 * real (c = 0) or imaginary (c = 1) part of point p of signal b at index
 * ((c*K + h)*batch + b)*n + p of x / y (host arrays; the same layout on the
 * device).  flags: MPFFT_SCALED, MPFFT_INVERSE.  The host entry is
 * synchronous; the device entry is asynchronous on `stream`. */
int mpfft_multiword_execute(mpfft_d_plan *plan, unsigned long batch, const void *x, void *y, unsigned flags);
int mpfft_multiword_execute_device(mpfft_d_plan *plan, unsigned long batch, const void *d_in, void *d_out,
                                   unsigned flags, void *stream);

/* FP64 real transforms of n real points (n a power of two >= 2; no
 * counterpart in the reference): the n/2-point complex transform (the
 * reference's, bit-identical) plus one split step in double.  r2c: in[b*n + j]
 * -> X_k at outr/outi[b*(n/2+1) + k], k = 0..n/2; c2r: the inverse (sum over
 * the Hermitian extension, imaginary parts of X_0 and X_(n/2) ignored) into
 * out[b*n + j].  MPFFT_SCALED: times 1/n.  Rounding as a double FFT: the
 * split step adds three roundings per bin. */
int mpfft_d_plan_create_real(mpfft_d_plan **plan, unsigned long n);
int mpfft_d_execute_r2c(mpfft_d_plan *plan, unsigned long batch, const double *in, double *outr, double *outi,
                        unsigned flags);
int mpfft_d_execute_c2r(mpfft_d_plan *plan, unsigned long batch, const double *inr, const double *ini, double *out,
                        unsigned flags);
/* FP64 multi-dimensional plan (rank 1..3, row-major, at most 2^28 points): the
 * reference's double transform along each axis in turn, last axis first,
 * each bit-identical to d_sr24_cp_fft; layout [c][b][p] with p the row-major
 * index.  MPFFT_SCALED multiplies by 1/N (exactly, one axis at a time). */
int mpfft_d_plan_create_nd(mpfft_d_plan **plan, int rank, const unsigned long *dims);
int mpfft_d_plan_destroy(mpfft_d_plan *plan);
int mpfft_d_execute(mpfft_d_plan *plan, unsigned long batch, const double *inr, const double *ini, double *outr,
                    double *outi, unsigned flags);
/* Device layout: word (c, b, p) at base[(c*batch + b)*n + p], i.e. all real
 * parts (signal after signal), then all imaginary parts. */
int mpfft_d_execute_device(mpfft_d_plan *plan, unsigned long batch, const double *d_in, double *d_out,
                           unsigned flags, void *stream);

/* ------------------------------------------------------------------------ */
/* uneven batches in one graph launch (no counterpart in the reference,      */
/* which transforms one signal per call and parallelises one butterfly loop  */
/* with an OpenMP team per node, lab/parallel/mp/parallel_mp_fft2.c:259-326) */
/* ------------------------------------------------------------------------ */

/* A batch plan for `count` signals of lengths n[i] (powers of two, up to 2^22)
 * and precisions prec[i] bits.  Each signal gets a form: fixed-point limbs
 * (up to 34 limbs), or with MPFFT_PLAN_FLOAT_TIERS / MPFFT_PLAN_NATIVE_TIERS the
 * floating tier mpfft_mp_plan_form names for that precision.  Signals are grouped into
 * one queue per form (per limb count for limbs); each queue is a persistent
 * kernel whose CTAs take whole signals, largest first, from a device counter
 * and transform them end to end.  Limb signals of 4096 points and more form
 * groups of equal length and limb count instead, each group one launch per
 * stage of the transform over all its signals.  The whole batch is captured
 * as one CUDA graph (created here, replayed by every execute).  Every output is
 * bit-identical to a single call of the same signal through
 * mpfft_mp_plan_create_flags with the same flags.  The plan owns an input and
 * an output arena in device memory holding every signal in its form's layout
 * (mpfft_batch_signal_format).  Choices made by mpfft_batch_autotune for the
 * same kind of batch on the same device are read back from the tune file. */
typedef struct mpfft_batch_plan mpfft_batch_plan;
int mpfft_batch_plan_create(mpfft_batch_plan **plan, unsigned long count, const unsigned long *n, const long *prec,
                            unsigned flags);
int mpfft_batch_plan_destroy(mpfft_batch_plan *plan);
/* Form of signal i (MPFFT_FORM_*), its words per real component (the limb
 * count for MPFFT_FORM_LIMBS: limb planes [c][i][p] of 32-bit words, else the
 * tier's K: words [c][h][p], doubles or, for float-float, floats), and its byte
 * offset and size in the arenas. */
int mpfft_batch_signal_format(const mpfft_batch_plan *plan, unsigned long i, int *form, int *words, size_t *offset,
                              size_t *bytes);
/* device addresses and size of the input and output arenas */
int mpfft_batch_arenas(const mpfft_batch_plan *plan, void **d_in, void **d_out, size_t *bytes);
/* One graph launch on `stream`: every signal of the input arena into the
 * output arena (forward, unscaled).  Asynchronous; executions of one plan
 * share its arenas, so executions that overlap on the GPU race. */
int mpfft_batch_execute_device(mpfft_batch_plan *plan, void *stream);
/* Host mpfr_t arrays, signal i at inr[i][0..n[i]) etc.: converted into the
 * arena on the host (limb signals with one block exponent each, floating
 * signals split into words), one copy each way, one graph launch.  flags:
 * MPFFT_SCALED, MPFFT_INVERSE.  A floating signal with exponents outside its
 * tier's window is rejected with MPFFT_EUNSUPPORTED.  Synchronous. */
int mpfft_batch_execute(mpfft_batch_plan *plan, mpfr_t *const *inr, mpfr_t *const *ini, mpfr_t *const *outr,
                        mpfr_t *const *outi, unsigned flags);
/* The autotuner: per queue, times every candidate launch shape -- CTA size
 * and, for floating forms, the largest shared-memory sub-transform -- on the
 * plan's own signals (the input arena as it is), keeps the fastest, re-captures
 * the graph and, when save != 0, records the choices in the tune file
 * (MPFFT_AUTOTUNE_FILE, else $XDG_CACHE_HOME/mpfft_b200/autotune.json, else
 * ~/.cache/mpfft_b200/autotune.json).  No choice changes any result. */
int mpfft_batch_autotune(mpfft_batch_plan *plan, int save);
/* Queue q of the plan: family (0 limbs, 1 FP64, 2 double-double,
 * 3 quad-double, 4 float-float), limb count, CTA size, largest sub-transform,
 * signal count.  The groups of long limb signals follow the queues: family 0,
 * their limb count, CTA size 0, sub = their length.  q < 0: returns the
 * number of queues and groups. */
int mpfft_batch_queue_info(const mpfft_batch_plan *plan, int q, int *family, int *limbs, int *threads, int *sub,
                           int *signals);

/* Transform `batch` signals whose MPFR fields are already in device memory,
 * WITHOUT allocating anything: no cudaMalloc, cudaFree or other allocating
 * call.  No counterpart in the reference.  For callers that cannot allocate
 * device memory when they call -- services that reserve their whole device
 * memory budget at start-up, and code paths that must not pay the implicit
 * device-wide synchronisation of cudaMalloc/cudaFree.  The plan must be
 * created beforehand (plan creation does allocate).
 *
 * Inputs/outputs, component (c, p, b) at index (c*n + p)*batch + b, c = 0 real
 * / 1 imaginary: significand limbs (nl_in resp. ceil(prec_out/64) 64-bit limbs
 * per component, least significant first, normalised as in an mpfr_t),
 * exponents (value = sign * 0.significand * 2^exp; INT64_MIN marks zero) and
 * signs (1 = negative).  Outputs are rounded to nearest-even at prec_out bits,
 * as mpfr_set_z_2exp would.  Inputs must be finite.  flags: MPFFT_SCALED (any
 * other flag is rejected with MPFFT_EINVAL).  The current device must be the
 * one the plan was created on (else MPFFT_EINVAL).
 *
 * Working storage is one static device array of mpfft_static_scratch_bytes()
 * (64 MiB) that every GPU loading this library holds until the process exits:
 * a batch needs 16*L*n*batch + 8*batch bytes (L = mpfft_mp_plan_limbs), and
 * larger batches are rejected with MPFFT_EUNSUPPORTED.  The first call on each
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current; make that first call before any stream capture.  All calls
 * share the array and it keeps the last call's contents (every word a call
 * reads it has written first): calls that overlap on the GPU race, so issue
 * them on one stream or serialise them.  Asynchronous on `stream`. */
int mpfft_mp_execute_significands_static(const mpfft_mp_plan *plan, unsigned long batch, const uint64_t *d_mant_in,
                                         const int64_t *d_exp_in, const uint8_t *d_sign_in, int nl_in,
                                         uint64_t *d_mant_out, int64_t *d_exp_out, uint8_t *d_sign_out,
                                         long prec_out, unsigned flags, void *stream);
/* size in bytes of the static device array used by the entry point above */
size_t mpfft_static_scratch_bytes(void);

/* ------------------------------------------------------------------------ */
/* 3. diagnostics for benchmarks (no counterpart in the reference)          */
/* ------------------------------------------------------------------------ */

/* Breadth-first schedule of a plan: node size and node count of each
 * butterfly launch (after the one leaf launch).  Returns the level count. */
int mpfft_mp_plan_schedule(const mpfft_mp_plan *plan, int *level_n, int *level_nodes, int max_levels);
/* mpfft_mp_execute_device with every launch bracketed by CUDA events on
 * `stream`; launch_ms[0] = leaf launch, launch_ms[1+i] = level i.  A level
 * that ran in one launch with level i-1 (large batches: two levels per
 * launch) reads 0 and the launch's time is in level i-1's entry.  Synchronous. */
int mpfft_mp_execute_device_timed(mpfft_mp_plan *plan, unsigned long batch, const uint32_t *d_in,
                                  uint32_t *d_out, void *stream, float *launch_ms);
/* Measured integer multiply-add rate of the current GPU (ops/s): wide = 0 for
 * 32-bit multiply-add, 1 for 32x32+64 -> 64-bit multiply-add. */
int mpfft_diag_imad_rate(int wide, double *ops_per_s);
/* Measured int8 tensor-core rate of the current GPU: unsigned-byte
 * multiply-adds per second of back-to-back tcgen05.mma kind::i8 (M=128,
 * N=256, K=32) from shared memory into tensor memory, two CTAs per SM. */
int mpfft_diag_tc_int8_rate(double *macs_per_s);
/* The tensor-core twiddle product on its own: out = sign(x) * r for `batch`
 * operands x (device limb planes x[i*batch + b], two's complement, L limbs,
 * |x| < 2^(32L-2)) and one unsigned twiddle w[0..L-1], with
 * r = floor((S + 2^(32L-2)) / 2^(32L-1)), S = the part of |x|*w in byte
 * columns >= 4L-8 rounded down to a multiple of 16.  35 <= L <= 260.
 * Asynchronous on `stream`. */
int mpfft_diag_tc_mul(int limbs, unsigned long batch, const uint32_t *d_x, const uint32_t *d_w, uint32_t *d_out,
                      void *stream);
/* MPFFT_OK, or MPFFT_ECUDA if a bounded wait of a tensor-core kernel expired
 * since the last call (the synchronous host-array calls check this themselves). */
int mpfft_diag_tc_error(void);
/* Limit, in nanoseconds, of each wait of the tensor-core kernels on their own
 * MMAs (default 2e9).  For tests of the expiry path: with 0 every wait gives
 * up at once, the kernel drains its MMAs and returns, and the call reports
 * MPFFT_ECUDA; restore the default afterwards. */
int mpfft_diag_tc_set_wait_limit(unsigned long long ns);
/* Fault injection for tests of the MPFFT_ENOMEM paths: the after-th device or
 * pinned-host allocation of execution buffers from now on (0 = the next one)
 * and every later one fail as cudaMalloc would; after < 0 switches this off. */
int mpfft_diag_fail_allocations(long after);
/* Real multiplications and additions of one transform, counted from the
 * plan's own schedule (its leaves and levels) with the per-butterfly counts of
 * the kernels: the reference's op counters (fft_complexity,
 * lab/parallel/mp/parallel_mp_fft2.c:332-354) give 7172 and 27652 at n = 1024
 * (lab/serial/mp/OPTIONS.md:42).  One-dimensional complex plans. */
int mpfft_mp_plan_counts(const mpfft_mp_plan *plan, unsigned long *mults, unsigned long *adds);

#ifdef __cplusplus
}
#endif

#endif /* MPFFT_B200_H */
