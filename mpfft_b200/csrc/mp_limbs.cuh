// Fixed-point multi-limb arithmetic for the multiprecision FFT kernels.
//
// Number format (device): a signal is stored in block floating point -- one
// exponent per signal, kept on the host -- and each real component is an
// L-limb two's-complement integer A (32-bit limbs, least significant first)
// with F = 32L-1-H fraction bits, H = log2(N)+2 headroom bits.  Because the
// format is fixed point, additions and subtractions are exact carry chains;
// the only rounding in the whole transform is the one in each twiddle product.
//
// Twiddles are unsigned L-limb magnitudes with 32L-1 fraction bits (|w| <= sqrt 2
// for cos+sin), plus a sign that the caller supplies.
//
// Layout: limb i of a component lives at `ptr[i * plane]` -- limb planes, so
// that consecutive threads (consecutive signals or butterfly indices) touch
// consecutive words and every load/store is coalesced.
#pragma once

#include <cstdint>

namespace mpfft {

// ---------------------------------------------------------------------------
// register-array load / store / add / sub
// ---------------------------------------------------------------------------

template <int L>
__device__ __forceinline__ void ld(uint32_t (&x)[L], const uint32_t *p, size_t plane) {
#pragma unroll
  for (int i = 0; i < L; ++i, p += plane) x[i] = *p;
}

template <int L>
__device__ __forceinline__ void st(uint32_t *p, size_t plane, const uint32_t (&x)[L]) {
#pragma unroll
  for (int i = 0; i < L; ++i, p += plane) *p = x[i];
}

// x = a + b (mod 2^(32L))
template <int L>
__device__ __forceinline__ void add(uint32_t (&x)[L], const uint32_t (&a)[L], const uint32_t (&b)[L]) {
  uint32_t c = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    uint64_t t = (uint64_t)a[i] + b[i] + c;
    x[i] = (uint32_t)t;
    c = (uint32_t)(t >> 32);
  }
}

// x = a - b (mod 2^(32L))
template <int L>
__device__ __forceinline__ void sub(uint32_t (&x)[L], const uint32_t (&a)[L], const uint32_t (&b)[L]) {
  uint32_t c = 1;  // a + ~b + 1
#pragma unroll
  for (int i = 0; i < L; ++i) {
    uint64_t t = (uint64_t)a[i] + (uint32_t)~b[i] + c;
    x[i] = (uint32_t)t;
    c = (uint32_t)(t >> 32);
  }
}

// x = pa + pb  or  pa - pb, streamed from memory
template <int L>
__device__ __forceinline__ void ld_addsub(uint32_t (&x)[L], const uint32_t *pa, const uint32_t *pb,
                                          size_t plane, bool subtract) {
  const uint32_t m = subtract ? 0xffffffffu : 0u;
  uint32_t c = subtract ? 1u : 0u;
#pragma unroll
  for (int i = 0; i < L; ++i, pa += plane, pb += plane) {
    uint64_t t = (uint64_t)*pa + (*pb ^ m) + c;
    x[i] = (uint32_t)t;
    c = (uint32_t)(t >> 32);
  }
}

// x = neg ? -x : x  (two's complement), branch free
template <int L>
__device__ __forceinline__ void cond_neg(uint32_t (&x)[L], uint32_t neg) {
  const uint32_t m = 0u - neg;
  uint32_t c = neg;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    uint64_t t = (uint64_t)(x[i] ^ m) + c;
    x[i] = (uint32_t)t;
    c = (uint32_t)(t >> 32);
  }
}

// ---------------------------------------------------------------------------
// truncated, rounded fixed-point product  x <- round(x * w / 2^(32L-1))
// ---------------------------------------------------------------------------
//
// In place: x holds the operand on entry and the product on return.
// x: two's complement, |x| < 2^(32L-2).  w: unsigned magnitude (L limbs at
// stride tplane), sign `wneg` (0/1).  Only partial products x_i*w_j with
// i+j >= L-2 are formed (about L^2/2 + 3L/2 of them); the dropped lower part
// is below L*2^-31 units of the result's last place.  Rounding is to nearest
// (half-way cases away from zero, symmetric in sign).
//
// The product is formed row by row (operand scanning): for each twiddle limb
// w_j, the low halves of x_i*w_j are added with one carry chain and the high
// halves with a second chain one column up.  Each partial product costs two
// multiply-add instructions with carry.
template <int L>
__device__ __forceinline__ void mul_tw(uint32_t (&x)[L], const uint32_t *w, size_t tplane, uint32_t wneg) {
  static_assert(L >= 2, "fixed-point product needs at least two limbs");
  const uint32_t xneg = x[L - 1] >> 31;
  cond_neg<L>(x, xneg);

  // acc[a] holds column (L-2+a), a = 0 .. L+1
  uint32_t acc[L + 2];
#pragma unroll
  for (int a = 0; a < L + 2; ++a) acc[a] = 0;
  acc[1] = 1u << 30;  // + 2^(32L-2): round to nearest on the final >> (32L-1)

#pragma unroll
  for (int j = 0; j < L; ++j, w += tplane) {
    const uint32_t t = *w;
    const int i0 = (L - 2 - j) > 0 ? (L - 2 - j) : 0;
    // low halves: columns i0+j .. L-1+j  ->  acc[i0+j-(L-2)] .. acc[j+1], carry into acc[j+2]
    asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(acc[i0 + j - (L - 2)]) : "r"(x[i0]), "r"(t));
#pragma unroll
    for (int i = i0 + 1; i < L; ++i)
      asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(acc[i + j - (L - 2)]) : "r"(x[i]), "r"(t));
    asm volatile("addc.u32 %0, %0, 0;" : "+r"(acc[j + 2]));
    // high halves: columns i0+j+1 .. L+j  ->  acc[i0+j+1-(L-2)] .. acc[j+2], carry into acc[j+3]
    asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(acc[i0 + j + 1 - (L - 2)]) : "r"(x[i0]), "r"(t));
#pragma unroll
    for (int i = i0 + 1; i < L; ++i)
      asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(acc[i + j + 1 - (L - 2)]) : "r"(x[i]), "r"(t));
    if (j + 3 <= L + 1)  // the last row's high chain cannot carry out (product < 2^(64L))
      asm volatile("addc.u32 %0, %0, 0;" : "+r"(acc[(j + 3 <= L + 1) ? j + 3 : L + 1]));
  }
  // r = (columns L-1 .. 2L-1) >> 31
#pragma unroll
  for (int i = 0; i < L; ++i) x[i] = __funnelshift_r(acc[i + 1], acc[i + 2], 31);
  cond_neg<L>(x, xneg ^ wneg);
}

}  // namespace mpfft
