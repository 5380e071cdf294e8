// Real-input (R2C) and real-output (C2R) multiprecision transforms.
//
// The reference notes that a real-input transform halves the work through
// Hermitian symmetry (README "only complex input").  Here a real signal x of
// N = 2M points is transformed as the complex signal z_m = x_(2m) + i x_(2m+1)
// of M points (the host gathers even samples into the real planes and odd
// samples into the imaginary planes), followed by one split step:
//
//   Z = FFT_M(z),  A = Z_k,  B = Z_(M-k),  S = A + conj B,  D = A - conj B,
//   T = w^k D  (w = exp(-2 pi i/N), one 3m3a product, cos from the N-table)
//   2 X_k     = (Sr + Ti,  Si - Tr)
//   2 X_(M-k) = (Sr - Ti, -(Si + Tr))            k = 0 .. M/2
//
// The factor 2 is carried in the block exponent, so the split step is exact
// apart from its three twiddle products.  C2R is the inverse split step,
//   S' = X_k + conj X_(M-k),  D' = X_k - conj X_(M-k),  T' = w^-k D',
//   2 Z_k = (S'r - T'i, S'i + T'r),  2 Z_(M-k) = (S'r + T'i, T'r - S'i),
// written with real and imaginary planes exchanged so that the forward
// complex transform that follows computes the inverse (the swap identity of
// the reference's test()); the host then de-interleaves the result.
//
// Layout as in mp_kernels.cu, with P points per plane set (M for z, M+1 for
// the half spectrum): word (c, i, p, b) at ((c*L + i)*P + p)*B + b.
#include <cstdint>

#include "mp_limbs.cuh"
#include "mpfft_internal.h"

namespace mpfft {

// 64 threads per block keep the three shared product planes (3 * L * 64 words)
// inside the 48 KB static limit for every L up to 34.
constexpr int kRealThreads = 64;

// Streaming signed sums on limb planes: out[j] = sum_t coef[j][t] * in[t],
// input t read at limb stride xs[t], outputs at stride ys, small integer
// coefficients.  Exact: int64 carries with the top limb sign-extended
// (two's-complement values; the format's headroom rules out overflow).
template <int L, int NI, int NO>
__device__ __forceinline__ void ssum(uint32_t *const (&out)[NO], size_t ys, const uint32_t *const (&in)[NI],
                                     const size_t (&xs)[NI], const int (&coef)[NO][NI]) {
  int64_t c[NO];
#pragma unroll
  for (int j = 0; j < NO; ++j) c[j] = 0;
#pragma unroll 1
  for (int i = 0; i < L; ++i) {
    int64_t v[NI];
#pragma unroll
    for (int t = 0; t < NI; ++t) {
      const uint32_t w = in[t][(size_t)i * xs[t]];
      v[t] = (i == L - 1) ? (int64_t)(int32_t)w : (int64_t)w;
    }
#pragma unroll
    for (int j = 0; j < NO; ++j) {
      int64_t acc = c[j];
#pragma unroll
      for (int t = 0; t < NI; ++t) acc += coef[j][t] * v[t];
      out[j][(size_t)i * ys] = (uint32_t)acc;
      c[j] = acc >> 32;
    }
  }
}

// Products of the split step, shared by both directions (side = 0: T = w^k D
// as in the level kernel's Z+ side; side = 1: T = w^-k D as its Z- side):
//   side 0: t1 = c (Dr + Di), Tr = t1 - d Di, Ti = t1 - s Dr
//   side 1: t1 = c (Dr - Di), Tr = t1 + d Di, Ti = s Dr - t1
// D is given by four inputs (Ar, Br, Ai, Bi) and signs: Dr = Ar + sb*Br,
// Di = Ai + sbi*Bi.  Writes Tr, Ti (limb stride ps).
template <int L>
__device__ __forceinline__ void split_products(int side, const uint32_t *Ar, const uint32_t *Br, const uint32_t *Ai,
                                               const uint32_t *Bi, size_t xs, int sbr, int sbi,
                                               const uint32_t *wr, const uint32_t *ws, const uint32_t *wd,
                                               size_t tplane, bool dn, uint32_t *P, uint32_t *Tr, uint32_t *Ti,
                                               size_t ps) {
  uint32_t X[L];
  {
    uint32_t *const o[1] = {P};
    const uint32_t *const in[4] = {Ar, Br, Ai, Bi};
    const size_t st4[4] = {xs, xs, xs, xs};
    const int sd = side ? -1 : 1;
    const int cf[1][4] = {{1, sbr, sd, sd * sbi}};
    ssum<L, 4, 1>(o, ps, in, st4, cf);
  }
  ld<L>(X, P, ps);
  mul_tw<L>(X, wr, tplane);
  st<L>(P, ps, X);
  ld_addsub<L>(X, Ai, Bi, xs, sbi < 0);  // Di
  mul_tw<L>(X, wd, tplane);
  combine_p<L>(X, P, ps, side ? dn : !dn, 1);
  st<L>(Tr, ps, X);
  ld_addsub<L>(X, Ar, Br, xs, sbr < 0);  // Dr
  mul_tw<L>(X, ws, tplane);
  combine_p<L>(X, P, ps, side == 0, side ? -1 : 1);
  st<L>(Ti, ps, X);
}

template <int L>
__global__ void __launch_bounds__(kRealThreads, 8) mp_r2c_post(const uint32_t *__restrict__ z, uint32_t *__restrict__ y, int M,
                                                       int B, const uint32_t *__restrict__ tw,
                                                       const uint8_t *__restrict__ dneg) {
  __shared__ uint32_t Ps[L * kRealThreads], Ts[L * kRealThreads], Us[L * kRealThreads];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)(M / 2 + 1) * B) return;
  const int b = (int)(t % B);
  const int k = (int)(t / B);
  const size_t zp = (size_t)M * B, yp = (size_t)(M + 1) * B;  // limb-plane strides
  const size_t zc = (size_t)L * zp, yc = (size_t)L * yp;      // real -> imaginary
  const uint32_t *Ar = z + (size_t)k * B + b, *Ai = Ar + zc;
  const uint32_t *Br = z + (size_t)((M - k) % M) * B + b, *Bi = Br + zc;
  uint32_t *Ykr = y + (size_t)k * B + b, *Yki = Ykr + yc;
  uint32_t *Ymr = y + (size_t)(M - k) * B + b, *Ymi = Ymr + yc;
  const size_t zs2[2] = {zp, zp};
  if (k == 0) {  // 2X_0 = (2Zr + 2Zi, 0), 2X_M = (2Zr - 2Zi, 0)
    uint32_t *const o[4] = {Ykr, Yki, Ymr, Ymi};
    const uint32_t *const in[2] = {Ar, Ai};
    const int cf[4][2] = {{2, 2}, {0, 0}, {2, -2}, {0, 0}};
    ssum<L, 2, 4>(o, yp, in, zs2, cf);
    return;
  }
  if (2 * k == M) {  // 2X_(M/2) = (2Zr, -2Zi)
    uint32_t *const o[2] = {Ykr, Yki};
    const uint32_t *const in[2] = {Ar, Ai};
    const int cf[2][2] = {{2, 0}, {0, -2}};
    ssum<L, 2, 2>(o, yp, in, zs2, cf);
    return;
  }
  const size_t tplane = (size_t)M / 2;  // N/4 entries: the table is built for N = 2M points
  const uint32_t *wr = tw + k, *ws = tw + (size_t)L * tplane + k, *wd = tw + (size_t)2 * L * tplane + k;
  uint32_t *P = Ps + threadIdx.x, *Tr = Ts + threadIdx.x, *Ti = Us + threadIdx.x;
  const size_t ps = blockDim.x;
  // D = A - conj B = (Ar - Br, Ai + Bi);  T = w^k D
  split_products<L>(0, Ar, Br, Ai, Bi, zp, -1, 1, wr, ws, wd, tplane, dneg[k] != 0, P, Tr, Ti, ps);
  // 2X_k = (Ar + Br + Ti, Ai - Bi - Tr),  2X_(M-k) = (Ar + Br - Ti, Bi - Ai - Tr)
  uint32_t *const o[4] = {Ykr, Ymr, Yki, Ymi};
  const uint32_t *const in[6] = {Ar, Br, Ti, Ai, Bi, Tr};
  const size_t xs6[6] = {zp, zp, ps, zp, zp, ps};
  const int cf[4][6] = {{1, 1, 1, 0, 0, 0}, {1, 1, -1, 0, 0, 0}, {0, 0, 0, 1, -1, -1}, {0, 0, 0, -1, 1, -1}};
  ssum<L, 6, 4>(o, yp, in, xs6, cf);
}

template <int L>
__global__ void __launch_bounds__(kRealThreads, 8) mp_c2r_pre(const uint32_t *__restrict__ x, uint32_t *__restrict__ z, int M,
                                                      int B, const uint32_t *__restrict__ tw,
                                                      const uint8_t *__restrict__ dneg) {
  __shared__ uint32_t Ps[L * kRealThreads], Ts[L * kRealThreads], Us[L * kRealThreads];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)(M / 2 + 1) * B) return;
  const int b = (int)(t % B);
  const int k = (int)(t / B);
  const size_t xp = (size_t)(M + 1) * B, zp = (size_t)M * B;
  const size_t xc = (size_t)L * xp, zc = (size_t)L * zp;
  const uint32_t *Ar = x + (size_t)k * B + b, *Ai = Ar + xc;
  const uint32_t *Br = x + (size_t)(M - k) * B + b, *Bi = Br + xc;
  // 2Z written with real and imaginary planes exchanged (inverse by the swap identity)
  uint32_t *Wkr = z + zc + (size_t)k * B + b, *Wki = z + (size_t)k * B + b;
  uint32_t *Wmr = z + zc + (size_t)((M - k) % M) * B + b, *Wmi = z + (size_t)((M - k) % M) * B + b;
  if (k == 0) {  // 2Z_0 = (X_0 + X_M, X_0 - X_M); imaginary parts of X_0, X_M ignored
    uint32_t *const o[2] = {Wkr, Wki};
    const uint32_t *const in[2] = {Ar, Br};
    const size_t xs2[2] = {xp, xp};
    const int cf[2][2] = {{1, 1}, {1, -1}};
    ssum<L, 2, 2>(o, zp, in, xs2, cf);
    return;
  }
  if (2 * k == M) {  // 2Z_(M/2) = (2 Ar, -2 Ai)
    uint32_t *const o[2] = {Wkr, Wki};
    const uint32_t *const in[2] = {Ar, Ai};
    const size_t xs2[2] = {xp, xp};
    const int cf[2][2] = {{2, 0}, {0, -2}};
    ssum<L, 2, 2>(o, zp, in, xs2, cf);
    return;
  }
  const size_t tplane = (size_t)M / 2;
  const uint32_t *wr = tw + k, *ws = tw + (size_t)L * tplane + k, *wd = tw + (size_t)2 * L * tplane + k;
  uint32_t *P = Ps + threadIdx.x, *Tr = Ts + threadIdx.x, *Ti = Us + threadIdx.x;
  const size_t ps = blockDim.x;
  // D' = X_k - conj X_(M-k) = (Ar - Br, Ai + Bi);  T' = w^-k D'
  split_products<L>(1, Ar, Br, Ai, Bi, xp, -1, 1, wr, ws, wd, tplane, dneg[k] != 0, P, Tr, Ti, ps);
  // 2Z_k = (Ar + Br - T'i, Ai - Bi + T'r),  2Z_(M-k) = (Ar + Br + T'i, T'r - Ai + Bi)
  uint32_t *const o[4] = {Wkr, Wmr, Wki, Wmi};
  const uint32_t *const in[6] = {Ar, Br, Ti, Ai, Bi, Tr};
  const size_t xs6[6] = {xp, xp, ps, xp, xp, ps};
  const int cf[4][6] = {{1, 1, -1, 0, 0, 0}, {1, 1, 1, 0, 0, 0}, {0, 0, 0, 1, -1, 1}, {0, 0, 0, -1, 1, 1}};
  ssum<L, 6, 4>(o, zp, in, xs6, cf);
}

#define MPFFT_REAL_CASE(LL)                                                                       \
  case LL:                                                                                        \
    if (forward) mp_r2c_post<LL><<<blocks, kRealThreads, 0, s>>>(in, out, M, B, tw, dneg);                 \
    else mp_c2r_pre<LL><<<blocks, kRealThreads, 0, s>>>(in, out, M, B, tw, dneg);                           \
    return cudaGetLastError();

// forward: Z (M points) -> 2X (M+1 points); else 2X-form half spectrum (M+1) ->
// swapped 2Z (M points).  tw/dneg: the twiddle table of a 2M-point plan.
cudaError_t mp_real_split(bool forward, int L, const uint32_t *in, uint32_t *out, int M, int B, const uint32_t *tw,
                          const uint8_t *dneg, cudaStream_t s) {
  const long long total = (long long)(M / 2 + 1) * B;
  const int blocks = (int)((total + kRealThreads - 1) / kRealThreads);
  switch (L) {
    MPFFT_REAL_CASE(2) MPFFT_REAL_CASE(3) MPFFT_REAL_CASE(4) MPFFT_REAL_CASE(5) MPFFT_REAL_CASE(6)
    MPFFT_REAL_CASE(7) MPFFT_REAL_CASE(8) MPFFT_REAL_CASE(9) MPFFT_REAL_CASE(10) MPFFT_REAL_CASE(11)
    MPFFT_REAL_CASE(12) MPFFT_REAL_CASE(13) MPFFT_REAL_CASE(14) MPFFT_REAL_CASE(15) MPFFT_REAL_CASE(16)
    MPFFT_REAL_CASE(17) MPFFT_REAL_CASE(18) MPFFT_REAL_CASE(19) MPFFT_REAL_CASE(20) MPFFT_REAL_CASE(21)
    MPFFT_REAL_CASE(22) MPFFT_REAL_CASE(23) MPFFT_REAL_CASE(24) MPFFT_REAL_CASE(25) MPFFT_REAL_CASE(26)
    MPFFT_REAL_CASE(27) MPFFT_REAL_CASE(28) MPFFT_REAL_CASE(29) MPFFT_REAL_CASE(30) MPFFT_REAL_CASE(31)
    MPFFT_REAL_CASE(32) MPFFT_REAL_CASE(33) MPFFT_REAL_CASE(34)
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace mpfft
