// Fixed-point multi-limb arithmetic for the multiprecision FFT kernels.
//
// Number format (device): a signal is stored in block floating point -- one
// exponent per signal, kept on the host -- and each real component is an
// L-limb two's-complement integer A (32-bit limbs, least significant first)
// with F = 32L-1-H fraction bits, H = log2(N)+2 headroom bits.  Because the
// format is fixed point, additions and subtractions are exact carry chains
// (modular, so signs need no special handling); the only rounding in the whole
// transform is the one in each twiddle product.
//
// Twiddles are unsigned L-limb magnitudes with 32L-1 fraction bits (|w| <= sqrt 2
// for cos+sin); their signs are applied by the caller when it combines products.
//
// Layout: limb i of a component lives at `ptr[i * plane]` -- limb planes, so
// that consecutive threads (consecutive signals or butterfly indices) touch
// consecutive words and every load/store is coalesced.
#pragma once

#include <cstdint>

namespace mpfft {

// L2 eviction priorities for global accesses (cache-policy operands of
// ld/st ... .L2::cache_hint): evict_last keeps a line that will be read again
// soon, evict_first marks a line that will not be read before it leaves L2.
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_normal() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st_hint(uint32_t *a, uint32_t v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(a), "r"(v), "l"(pol) : "memory");
}
// (asm volatile: the compiler keeps these loads in program order, which also
// stops it from hoisting them far ahead of their use)
__device__ __forceinline__ uint32_t ld_hint(const uint32_t *a, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol) : "memory");
  return v;
}

// one step of a carry chain: returns a + b + c (mod 2^32), c <- carry out
__device__ __forceinline__ uint32_t addc(uint32_t a, uint32_t b, uint32_t &c) {
  const uint64_t t = (uint64_t)a + b + c;
  c = (uint32_t)(t >> 32);
  return (uint32_t)t;
}

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

// x = pa + pb  or  pa - pb, streamed from memory (pb may be null: x = pa)
template <int L>
__device__ __forceinline__ void ld_addsub(uint32_t (&x)[L], const uint32_t *pa, const uint32_t *pb,
                                          size_t plane, bool subtract) {
  if (!pb) {
    ld<L>(x, pa, plane);
    return;
  }
  const uint32_t m = subtract ? 0xffffffffu : 0u;
  uint32_t c = subtract ? 1u : 0u;
#pragma unroll
  for (int i = 0; i < L; ++i, pa += plane, pb += plane) x[i] = addc(*pa, *pb ^ m, c);
}

// x = sx*x + sp*p with sx in {+1,-1}, sp in {+1,-1,0}; p streamed from memory.
// At most one operand is negated: a two's complement negation is ~v + 1.
template <int L>
__device__ __forceinline__ void combine_p(uint32_t (&x)[L], const uint32_t *p, size_t stride, bool negx,
                                          int sp) {
  const uint32_t mx = negx ? 0xffffffffu : 0u;
  const uint32_t mp = sp < 0 ? 0xffffffffu : 0u;
  const uint32_t keep = sp != 0 ? 0xffffffffu : 0u;
  uint32_t c = (negx ? 1u : 0u) + (sp < 0 ? 1u : 0u);
#pragma unroll
  for (int i = 0; i < L; ++i, p += stride) x[i] = addc(x[i] ^ mx, (*p & keep) ^ mp, c);
}

// ---------------------------------------------------------------------------
// truncated, rounded signed fixed-point product  x <- round(x * w / 2^(32L-1))
// ---------------------------------------------------------------------------
//
// In place: x (two's complement, |x| < 2^(32L-2)) holds the operand on entry
// and the product on return.  w: unsigned magnitude, L limbs at stride tplane.
//
// The limbs of x are multiplied as an unsigned integer x_u = x + s*2^(32L)
// (s = sign bit); the signed product is x_u*w - s*w*2^(32L), so for negative
// x the twiddle is subtracted once from the columns at and above 32L.  Only
// partial products x_i*w_j with i+j >= L-2 are formed (about L^2/2 + 3L/2 of
// them); the dropped lower part is below L*2^-31 units of the result's last
// place.  Adding 2^(32L-2) before the final shift rounds to nearest.
//
// The product is formed row by row (operand scanning): for each twiddle limb
// w_j, one multiply-add-carry chain adds x_i*w_j into columns i+j.  Each step
// is a 32x32+32+32 -> 64-bit multiply-add (it cannot overflow), written in
// plain C so the compiler can schedule the two halves freely; on sm_100a this
// issues faster than PTX mad.lo.cc/madc.hi.cc chains (measured).
//
// kPacked: w holds the L limbs contiguously in shared memory, 16-byte aligned
// (tplane unused); they are read four at a time with 128-bit loads.
template <int L, bool kPacked = false>
__device__ __forceinline__ void mul_tw(uint32_t (&x)[L], const uint32_t *w, size_t tplane) {
  static_assert(L >= 2, "fixed-point product needs at least two limbs");
  // limb j of the twiddle: p points at it (strided planes) or at limb 0 (packed)
  uint4 v4;  // packed: limbs 4*(j/4) .. 4*(j/4)+3
  auto limb = [&](const uint32_t *p, int j) -> uint32_t {
    if (!kPacked) return *p;
    if ((j & 3) == 0) v4 = *reinterpret_cast<const uint4 *>(p + j);
    return (j & 3) == 0 ? v4.x : (j & 3) == 1 ? v4.y : (j & 3) == 2 ? v4.z : v4.w;
  };
  const uint32_t smask = 0u - (x[L - 1] >> 31);

  // acc[a] holds column (L-2+a), a = 0 .. L+1
  uint32_t acc[L + 2];
#pragma unroll
  for (int a = 0; a < L + 2; ++a) acc[a] = 0;
  acc[1] = 1u << 30;  // + 2^(32L-2): round to nearest on the final >> (32L-1)

  const uint32_t *w0 = w;
#pragma unroll
  for (int j = 0; j < L; ++j, w += kPacked ? 0 : tplane) {
    const uint32_t t = limb(w, j);
    const int i0 = (L - 2 - j) > 0 ? (L - 2 - j) : 0;
    uint32_t c = 0;
#pragma unroll
    for (int i = i0; i < L; ++i) {
      const uint64_t pr = (uint64_t)x[i] * t + acc[i + j - (L - 2)] + c;
      acc[i + j - (L - 2)] = (uint32_t)pr;
      c = (uint32_t)(pr >> 32);
    }
    acc[j + 2] = c;  // column L+j is still empty: rows < j reach column L+j-1
  }
  // signed correction: acc -= s * w * 2^(32L)  (columns L .. 2L-1 = acc[2 .. L+1])
  {
    uint32_t c = 1;
#pragma unroll
    for (int j = 0; j < L; ++j, w0 += kPacked ? 0 : tplane) acc[j + 2] = addc(acc[j + 2], ~(limb(w0, j) & smask), c);
  }
  // x = (columns L-1 .. 2L-1) >> 31
#pragma unroll
  for (int i = 0; i < L; ++i) x[i] = __funnelshift_r(acc[i + 1], acc[i + 2], 31);
}

}  // namespace mpfft
