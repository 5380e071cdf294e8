// Conversion between MPFR significands and the device limb-plane format.
//
// The host only gathers/scatters the raw fields of each mpfr_t (its 64-bit
// significand limbs, exponent and sign); all O(N*P) bit manipulation happens
// here:
//   import: per signal, the block exponent e_s = max exponent of its nonzero
//           components; per component, A = round(|x| * 2^(F - e_s)) (nearest,
//           half-way away from zero) as an L-limb two's-complement integer.
//   export: per component, A * 2^e2 rounded to nearest-even at the output
//           precision, as normalised significand limbs + exponent + sign, i.e.
//           exactly what mpfr_set_z_2exp(y, A, e2, MPFR_RNDN) stores.
//
// MPFR significands: nl 64-bit limbs, least significant first, value =
// 0.d * 2^exp with the top bit of the top limb set (mpfr_t, MPFR manual
// "Nomenclature and Types").
#include <cstdint>

#include "mpfft_internal.h"

namespace mpfft {

constexpr int64_t kZeroExp = INT64_MIN;  // marks a zero component

// 32 bits of the non-negative integer held in 64-bit limbs m[0..nl), starting
// at bit position pos (may be negative or beyond the top: zeros shifted in).
__device__ __forceinline__ uint32_t bits32_64(const uint64_t *m, int nl, long pos) {
  const long w = pos >= 0 ? pos / 64 : -((-pos + 63) / 64);
  const int off = (int)(pos - w * 64);
  const uint64_t lo = (w >= 0 && w < nl) ? m[w] : 0;
  const uint64_t hi = (w + 1 >= 0 && w + 1 < nl) ? m[w + 1] : 0;
  const uint64_t v = off == 0 ? lo : ((lo >> off) | (hi << (64 - off)));
  return (uint32_t)v;
}

__global__ void mp_import_exp_init(int64_t *es, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < B) es[b] = kZeroExp;
}

// Index of component (c, p, b) in the mant/ex/sg arrays: (c*N + p)*B + b
// (batch innermost), or with sig_major (b*2 + c)*N + p (each signal's
// components contiguous, the order a host walks mpfr_t arrays in).
__device__ __forceinline__ size_t comp_index(bool sig_major, long long t, int b, int c, int p, int N) {
  return sig_major ? ((size_t)b * 2 + c) * N + p : (size_t)t;
}

// block exponents: es[b] = max exp over signal b's nonzero components
// (t runs over the storage index)
// (t runs over the storage index).  Lanes of a warp that share a signal (all of
// them in the signal-major layout) first reduce among themselves, so each
// signal takes one atomic per warp.
__global__ void mp_import_exp(const int64_t *__restrict__ ex, int N, int B, bool sig_major,
                              int64_t *__restrict__ es) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t < 2LL * N * B;
  long long v = in ? (long long)ex[t] : (long long)kZeroExp;  // kZeroExp is the identity of max
  const int b = in ? (sig_major ? (int)(t / (2LL * N)) : (int)(t % B)) : -1;
  const int lane = threadIdx.x & 31;
  for (int off = 1; off < 32; off <<= 1) {  // segmented max over the contiguous lanes of one signal
    const long long ov = __shfl_down_sync(0xffffffffu, v, off);
    const int ob = __shfl_down_sync(0xffffffffu, b, off);
    if (lane + off < 32 && ob == b && ov > v) v = ov;
  }
  const int pb = __shfl_up_sync(0xffffffffu, b, 1);
  const bool head = lane == 0 || pb != b;
  if (in && head && v != (long long)kZeroExp) atomicMax((long long *)&es[b], v);
}

// mant: [component][nl] 64-bit limbs; planes: word (c, i, p, b) at ((c*L + i)*N + p)*B + b
__global__ void mp_import(const uint64_t *__restrict__ mant, const int64_t *__restrict__ ex,
                          const uint8_t *__restrict__ sg, int nl, int N, int B, int L, long F, bool sig_major,
                          const int64_t *__restrict__ es, uint32_t *__restrict__ planes) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2LL * N * B) return;
  const int b = (int)(t % B);
  const long long cp = t / B;  // c*N + p
  const int c = (int)(cp / N);
  const int p = (int)(cp - (long long)c * N);
  const size_t plane = (size_t)N * B;
  uint32_t *dst = planes + ((size_t)c * L * N + p) * B + b;
  const size_t ci = comp_index(sig_major, t, b, c, p, N);
  const int64_t e = ex[ci];
  if (e == kZeroExp) {
    for (int i = 0; i < L; ++i) dst[(size_t)i * plane] = 0;
    return;
  }
  const uint64_t *m = mant + ci * nl;
  // value = M * 2^(e - 64 nl);  A = M * 2^sh
  const long sh = (long)(e - 64L * nl + F - es[b]);
  uint32_t round = 0;
  if (sh < 0) {
    const long rb = -sh - 1;
    round = rb < 64L * nl ? (bits32_64(m, nl, rb) & 1u) : 0u;
  }
  const bool neg = sg[ci] != 0;
  uint32_t cr = round;           // rounding carry (magnitude)
  uint32_t cn = neg ? 1u : 0u;   // negation carry (two's complement)
  const uint32_t mk = neg ? 0xffffffffu : 0u;
  for (int i = 0; i < L; ++i) {
    uint64_t v = (uint64_t)bits32_64(m, nl, 32L * i - sh) + cr;
    cr = (uint32_t)(v >> 32);
    uint64_t u = (uint64_t)((uint32_t)v ^ mk) + cn;
    cn = (uint32_t)(u >> 32);
    dst[(size_t)i * plane] = (uint32_t)u;
  }
}

// out: [component][nlo] 64-bit limbs, oex (kZeroExp for zero), osg
__global__ void mp_export(const uint32_t *__restrict__ planes, int N, int B, int L, const int64_t *__restrict__ es,
                          long F_plus_shift, long prec, int nlo, bool sig_major, uint64_t *__restrict__ out,
                          int64_t *__restrict__ oex, uint8_t *__restrict__ osg) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2LL * N * B) return;
  const int b = (int)(t % B);
  const long long cp = t / B;
  const int c = (int)(cp / N);
  const int p = (int)(cp - (long long)c * N);
  const size_t plane = (size_t)N * B;
  const uint32_t *src = planes + ((size_t)c * L * N + p) * B + b;
  const size_t ci = comp_index(sig_major, t, b, c, p, N);
  uint64_t a[(kMaxLimbsBig + 2) / 2 + 1];  // magnitude in 64-bit limbs
  const int na = (L + 1) / 2;
  const bool neg = (src[(size_t)(L - 1) * plane] >> 31) != 0;
  {
    uint32_t cn = neg ? 1u : 0u;
    const uint32_t mk = neg ? 0xffffffffu : 0u;
    for (int i = 0; i < na; ++i) a[i] = 0;
    for (int i = 0; i < L; ++i) {
      uint64_t u = (uint64_t)(src[(size_t)i * plane] ^ mk) + cn;
      cn = (uint32_t)(u >> 32);
      a[i >> 1] |= (uint64_t)(uint32_t)u << (32 * (i & 1));
    }
  }
  int top = -1;  // index of the highest set bit
  for (int i = na - 1; i >= 0; --i)
    if (a[i]) {
      top = 64 * i + 63 - __clzll((long long)a[i]);
      break;
    }
  uint64_t *o = out + ci * nlo;
  if (top < 0) {
    oex[ci] = kZeroExp;
    osg[ci] = 0;
    for (int k = 0; k < nlo; ++k) o[k] = 0;
    return;
  }
  // keep the top `prec` bits: kept = a >> d (d may be negative), round to nearest even
  const long d = top + 1 - prec;  // bits of a below the kept ones
  bool up = false;
  if (d > 0) {
    const uint32_t rbit = bits32_64(a, na, d - 1) & 1u;
    bool sticky = false;
    for (long pos = 0; pos < d - 1 && !sticky; pos += 32) {
      uint32_t v = bits32_64(a, na, pos);
      const long nb = d - 1 - pos;
      if (nb < 32) v &= (1u << nb) - 1u;
      sticky = v != 0;
    }
    const uint32_t lsb = bits32_64(a, na, d) & 1u;
    up = rbit && (sticky || lsb);
  }
  // Output significand O (nlo limbs, top `prec` bits used): bit j of O is bit
  // (j + shift) of a for j >= base, zero below base; the rounding increment is
  // added at bit `base` and carried upward.
  const long base = 64L * nlo - prec;
  const long shift = d - base;
  uint32_t cr = 0;
  for (int k = 0; k < nlo; ++k) {
    uint64_t w = 0;
    for (int h = 0; h < 2; ++h) {
      const long opos = 64L * k + 32 * h;
      uint32_t v = 0;
      if (opos + 32 > base) {
        v = bits32_64(a, na, opos + shift);
        if (opos < base) v &= ~((1u << (base - opos)) - 1u);
      }
      uint64_t add = cr;
      if (up && opos <= base && base < opos + 32) add += (uint64_t)1 << (base - opos);
      const uint64_t sum = (uint64_t)v + add;
      cr = (uint32_t)(sum >> 32);
      w |= (uint64_t)(uint32_t)sum << (32 * h);
    }
    o[k] = w;
  }
  const bool ovf = cr != 0;  // rounding carried out of the top: significand became 2^prec
  long e = top + 1;
  if (ovf) {
    o[nlo - 1] = 0x8000000000000000ull;  // 0.1000... at one higher exponent
    for (int k = 0; k < nlo - 1; ++k) o[k] = 0;
    e += 1;
  }
  oex[ci] = (int64_t)(e + (long)es[b] - F_plus_shift);
  osg[ci] = neg ? 1 : 0;
}

cudaError_t mp_import_launch(const uint64_t *mant, const int64_t *ex, const uint8_t *sg, int nl, int N, int B,
                             int L, long F, int64_t *es, uint32_t *planes, cudaStream_t s, bool sig_major) {
  mp_import_exp_init<<<(B + 255) / 256, 256, 0, s>>>(es, B);
  const long long total = 2LL * N * B;
  const int blocks = (int)((total + 255) / 256);
  mp_import_exp<<<blocks, 256, 0, s>>>(ex, N, B, sig_major, es);
  mp_import<<<blocks, 256, 0, s>>>(mant, ex, sg, nl, N, B, L, F, sig_major, es, planes);
  return cudaGetLastError();
}

cudaError_t mp_export_launch(const uint32_t *planes, int N, int B, int L, const int64_t *es, long F_plus_shift,
                             long prec, int nlo, uint64_t *out, int64_t *oex, uint8_t *osg, cudaStream_t s,
                             bool sig_major) {
  const long long total = 2LL * N * B;
  const int blocks = (int)((total + 255) / 256);
  mp_export<<<blocks, 256, 0, s>>>(planes, N, B, L, es, F_plus_shift, prec, nlo, sig_major, out, oex, osg);
  return cudaGetLastError();
}

}  // namespace mpfft
