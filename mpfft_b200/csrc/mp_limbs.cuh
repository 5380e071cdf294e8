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

namespace mpfft {

// ---------------------------------------------------------------------------
// the same product, column by column (product scanning)
// ---------------------------------------------------------------------------
//
// mul_tw keeps all L+2 accumulator words of the product in registers next to
// the L operand limbs.  Here the columns are formed one after another:
// column c = L-2+a sums x_i * w_(c-i) into a running total whose low word is
// final (word a) and whose upper two words carry into column c+1.  The
// integer is the same -- every partial product with i + j >= L-2, 2^30 added
// in word 1, the twiddle subtracted from word 2 on when x is negative, all
// modulo 2^(32(L+2)) -- so the rounded result limbs are bit-identical to
// mul_tw's, with only x and a few words live (about half the registers).
//
// The twiddle comes from shared memory reversed (wr[t] = w_(L-1-t)), so that
// the limbs a column needs are consecutive, in four copies shifted by 0..3
// words (copy s, word u = wr[u - s], zero outside 0 <= u-s < L) so that every
// column reads them in aligned 128-bit loads.  Result limb r_i is passed to
// sink(i, r_i) as soon as words i+1 and i+2 are final, in increasing i.
template <int L>
__host__ __device__ constexpr int cols_stride() {
  return (L + 6 + 3) & ~3;  // words per copy, covering the over-read of the last quad
}

template <int L, class Sink>
__device__ __forceinline__ void mul_tw_cols(const uint32_t (&x)[L], const uint32_t *wq, Sink &&sink) {
  constexpr int Lq = cols_stride<L>();
  const uint32_t smask = 0u - (x[L - 1] >> 31);
  uint32_t c0 = 0, c1 = 0;  // carry of the previous column (two words)
  uint32_t prev = 0;        // word a-1
#pragma unroll
  for (int a = 0; a < L + 2; ++a) {
    const int c = a + L - 2;
    const int i_lo = c - (L - 1) > 0 ? c - (L - 1) : 0;
    const int i_hi = c < L - 1 ? c : L - 1;
    uint32_t t0, t1, t2 = 0;
    {
      const uint64_t init = (uint64_t)c0 + (a == 1 ? (1u << 30) : 0u);  // + 2^(32L-2): round to nearest
      t0 = (uint32_t)init;
      const uint64_t h = (uint64_t)c1 + (init >> 32);
      t1 = (uint32_t)h;
      t2 = (uint32_t)(h >> 32);
    }
    if (i_lo <= i_hi) {
      const int tt = L - 1 - c + i_lo;  // wr index of the column's first limb
      const int s = (4 - (tt & 3)) & 3;
      const uint32_t *base = wq + s * Lq + tt + s;  // 16-byte aligned
#pragma unroll
      for (int i = i_lo; i <= i_hi; i += 4) {
        const uint4 v = *reinterpret_cast<const uint4 *>(base + (i - i_lo));
        const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (i + e <= i_hi) {
            const uint64_t pr = (uint64_t)x[i + e] * wv[e] + t0;
            t0 = (uint32_t)pr;
            const uint64_t h = (uint64_t)t1 + (pr >> 32);
            t1 = (uint32_t)h;
            t2 += (uint32_t)(h >> 32);
          }
        }
      }
    }
    if (a >= 2) {  // signed correction: + ~(w_(a-2) & s) (+1 at a = 2), i.e. - s*w*2^(32L)
      const uint32_t wj = wq[L + 1 - a];  // copy 0: wr[L+1-a] = w_(a-2)
      const uint64_t pr = (uint64_t)t0 + (uint32_t)~(wj & smask) + (a == 2 ? 1u : 0u);
      t0 = (uint32_t)pr;
      const uint64_t h = (uint64_t)t1 + (pr >> 32);
      t1 = (uint32_t)h;
      t2 += (uint32_t)(h >> 32);
      sink(a - 2, __funnelshift_r(prev, t0, 31));
    }
    prev = t0;
    c0 = t1;
    c1 = t2;
  }
}

}  // namespace mpfft
