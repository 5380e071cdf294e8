// Warp-parallel multi-limb arithmetic: one number's limbs across the lanes of
// a warp, carries resolved by shuffles and a ballot carry-lookahead.
//
// The per-thread arithmetic of mp_limbs.cuh runs an L-limb addition as an
// L-step carry chain and an L x L product as ~L^2/2 dependent multiply-adds,
// which is efficient when 32 lanes hold 32 different numbers (batches) but
// leaves a launch of a few hundred butterflies (one signal) bound by one
// thread's chain.  Here a warp holds ONE number: element e (a limb, or a
// column of a product) lives in lane e, register `a`, or lane e-32, register
// `b` (when the vector is longer than 32).  An addition is one add per lane
// plus a carry-lookahead over the warp; a product is L multiply-adds per lane
// (its columns side by side) plus a carry resolution.  Every operation
// computes exactly the same integer as its per-thread counterpart, so the
// kernels built on either are bit-identical.
#pragma once

#include <cstdint>

namespace mpfft {

__device__ __forceinline__ unsigned lane_index() { return threadIdx.x & 31u; }

// s <- s + (carry into this element), where element e's own addition left the
// 32-bit sum s and the carry-out g (0 or 1), and the carry into element e is
// the carry-out of element e-1 after its own carry-in (generate g, propagate
// s == 2^32-1).  With G and P the warp's generate/propagate masks, the carry
// into every element at once is ((G|P) + G) ^ (G|P) ^ G: the binary addition
// ripples exactly through runs of propagating elements.
template <bool kTwo>
__device__ __forceinline__ void lanes_resolve(uint32_t &sa, uint32_t ga, uint32_t &sb, uint32_t gb) {
  const unsigned lane = lane_index();
  uint64_t G = __ballot_sync(~0u, ga != 0), P = __ballot_sync(~0u, sa == ~0u);
  if (kTwo) {
    G |= (uint64_t)__ballot_sync(~0u, gb != 0) << 32;
    P |= (uint64_t)__ballot_sync(~0u, sb == ~0u) << 32;
  }
  const uint64_t GP = G | P;
  const uint64_t C = (GP + G) ^ GP ^ G;  // bit e: carry into element e
  sa += (uint32_t)(C >> lane) & 1u;
  if (kTwo) sb += (uint32_t)(C >> (lane + 32)) & 1u;
}

// (ra, rb) <- element e-d of (a, b); zero below element 0
template <bool kTwo>
__device__ __forceinline__ void lanes_up(uint32_t a, uint32_t b, unsigned d, uint32_t &ra, uint32_t &rb) {
  const unsigned lane = lane_index();
  const uint32_t xa = __shfl_sync(~0u, a, (lane - d) & 31u);
  ra = lane >= d ? xa : 0u;
  if (kTwo) {
    const uint32_t xb = __shfl_sync(~0u, b, (lane - d) & 31u);
    rb = lane >= d ? xb : xa;
  }
}

// (ra, rb) <- element e+d of (a, b); zero past element 31 (one register) or
// unspecified past element 63
template <bool kTwo>
__device__ __forceinline__ void lanes_down(uint32_t a, uint32_t b, unsigned d, uint32_t &ra, uint32_t &rb) {
  const unsigned lane = lane_index();
  const uint32_t xa = __shfl_sync(~0u, a, (lane + d) & 31u);
  if (kTwo) {
    const uint32_t xb = __shfl_sync(~0u, b, (lane + d) & 31u);
    ra = lane + d < 32 ? xa : xb;
    rb = xb;
  } else {
    ra = lane + d < 32 ? xa : 0u;
  }
}

// x <- x + y + c0 (c0 in {0, 1}, added at element 0), modulo 2^(32 * elements)
template <bool kTwo>
__device__ __forceinline__ void lanes_add(uint32_t &xa, uint32_t &xb, uint32_t ya, uint32_t yb, uint32_t c0) {
  const uint64_t ta = (uint64_t)xa + ya + (lane_index() == 0 ? c0 : 0u);
  const uint64_t tb = kTwo ? (uint64_t)xb + yb : 0;
  xa = (uint32_t)ta;
  xb = (uint32_t)tb;
  lanes_resolve<kTwo>(xa, (uint32_t)(ta >> 32), xb, (uint32_t)(tb >> 32));
}

// limbs 0..L-1 of a limb-plane number (limb i at p[i * plane]); zero elsewhere
template <int L, bool kTwo>
__device__ __forceinline__ void lanes_ld(uint32_t &a, uint32_t &b, const uint32_t *p, size_t plane) {
  const unsigned lane = lane_index();
  a = lane < L ? p[lane * plane] : 0u;
  b = (kTwo && lane + 32 < L) ? p[(lane + 32) * plane] : 0u;
}

template <int L, bool kTwo>
__device__ __forceinline__ void lanes_st(uint32_t *p, size_t plane, uint32_t a, uint32_t b) {
  const unsigned lane = lane_index();
  if (lane < L) p[lane * plane] = a;
  if (kTwo && lane + 32 < L) p[(lane + 32) * plane] = b;
}

// Length of a warp's zero-padded twiddle row (lanes_mul_tw): L-1 zeros, the L
// limbs, then zeros up to the last index a lane reads.
template <int L>
__host__ __device__ constexpr int lanes_tw_len() {
  return 2 * L + 64;
}

// x <- round(x * w / 2^(32L-1)): the product of mul_tw (mp_limbs.cuh) -- the
// same partial products x_i w_j (i + j >= L-2), the same rounding constant
// 2^(32L-2), the same signed correction -s w 2^(32L) -- on the warp.
//
// Element e holds column L-2+e of the product, e = 0 .. L+1 (two registers
// when L+2 > 32): the lane adds x_i w_(e+L-2-i) over i as a 96-bit sum (a
// 32-bit low word with a carry-free 64-bit high part), reading x_i from Xs
// (this warp's copy of x, L words, 16-byte aligned: one broadcast 128-bit load
// per four steps) and w_j from Wp[j + L-1] (the row zero-padded so that the
// terms with j outside 0..L-1 add zero and the loop is the same on every
// lane).  The column sums are then three 32-bit digits at elements e, e+1,
// e+2; two shuffled additions and one carry-lookahead give the columns of the
// exact sum mod 2^(32(L+2)), the integer mul_tw forms in its accumulator, and
// result limb i = (column i+1 >> 31) | (column i+2 << 1).
template <int L>
__device__ __forceinline__ void lanes_mul_tw(uint32_t &xa, uint32_t &xb, const uint32_t *__restrict__ Xs,
                                             const uint32_t *__restrict__ Wp) {
  static_assert(L >= 2 && L <= 62, "columns must fit two registers per lane");
  constexpr bool kTwo = L + 2 > 32;
  const unsigned lane = lane_index();
  const uint32_t *wa = Wp + lane + 2 * L - 3;  // element e, step i: Wp[e + 2L-3 - i]
  uint32_t lo_a = 0, lo_b = 0;
  uint64_t hi_a = 0, hi_b = 0;
#pragma unroll
  for (int i0 = 0; i0 < L; i0 += 4) {
    const uint4 x4 = *reinterpret_cast<const uint4 *>(Xs + i0);
    const uint32_t xs[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u;
      if (i < L) {
        const uint64_t pa = (uint64_t)xs[u] * wa[-i] + lo_a;
        lo_a = (uint32_t)pa;
        hi_a += pa >> 32;
        // columns 32 .. L+1 have terms only for i >= 31 (w_j = 0 for j >= L)
        if (kTwo && i >= 31) {
          const uint64_t pb = (uint64_t)xs[u] * wa[32 - i] + lo_b;
          lo_b = (uint32_t)pb;
          hi_b += pb >> 32;
        }
      }
    }
  }
  // rounding constant at column L-1 (element 1); signed correction
  // -s w 2^(32L) = (~(w & smask) + 1) at columns L .. 2L-1 (elements 2 .. L+1)
  const uint32_t smask = 0u - (Xs[L - 1] >> 31);
  auto addk = [&](uint32_t &lo, uint64_t &hi, int e) {
    const bool corr = e >= 2 && e <= L + 1;
    const uint32_t w = Wp[corr ? e + L - 3 : L - 1];
    const uint64_t k = corr ? (uint64_t)(~(w & smask)) + (e == 2 ? 1u : 0u) : (e == 1 ? (1u << 30) : 0u);
    const uint64_t t = (uint64_t)lo + k;
    lo = (uint32_t)t;
    hi += t >> 32;
  };
  addk(lo_a, hi_a, (int)lane);
  if (kTwo) addk(lo_b, hi_b, (int)lane + 32);
  // digits: lo at e, (uint32)hi at e+1, hi >> 32 at e+2 (hi < L 2^32 + 2^32)
  uint32_t p1a, p1b = 0, p2a, p2b = 0;
  lanes_up<kTwo>((uint32_t)hi_a, (uint32_t)hi_b, 1, p1a, p1b);
  lanes_up<kTwo>((uint32_t)(hi_a >> 32), (uint32_t)(hi_b >> 32), 2, p2a, p2b);
  const uint64_t ta = (uint64_t)lo_a + p1a + p2a;              // < 3 2^32
  const uint64_t tb = kTwo ? (uint64_t)lo_b + p1b + p2b : 0;
  uint32_t ca, cb = 0;
  lanes_up<kTwo>((uint32_t)(ta >> 32), (uint32_t)(tb >> 32), 1, ca, cb);  // carries 0..2
  const uint64_t ua = (uint64_t)(uint32_t)ta + ca, ub = kTwo ? (uint64_t)(uint32_t)tb + cb : 0;
  uint32_t sa = (uint32_t)ua, sb = (uint32_t)ub;
  lanes_resolve<kTwo>(sa, (uint32_t)(ua >> 32), sb, (uint32_t)(ub >> 32));
  uint32_t n1a, n1b = 0, n2a, n2b = 0;
  lanes_down<kTwo>(sa, sb, 1, n1a, n1b);
  lanes_down<kTwo>(sa, sb, 2, n2a, n2b);
  xa = lane < L ? __funnelshift_r(n1a, n2a, 31) : 0u;
  xb = (kTwo && lane + 32 < L) ? __funnelshift_r(n1b, n2b, 31) : 0u;
}

}  // namespace mpfft
