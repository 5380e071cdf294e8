// Device functions of the multiprecision split-radix kernels: one leaf and one
// L-shaped butterfly of one signal, on limb planes (word (c, i, p, b) at
// base[((c*L + i)*N + p)*B + b]).  Shared by the per-level kernels
// (mp_kernels.cu) and the persistent work-queue kernels (queue_kernels.cu),
// so both compute bit-identical results.
#pragma once

#include <cstdint>

#include "mp_limbs.cuh"
#include "mpfft_internal.h"

namespace mpfft {

// ---------------------------------------------------------------------------
// leaves: size-1, size-2 and size-4 DFTs of strided input subsequences
// (reference base cases, lab/parallel/mp/parallel_mp_fft2.c:125-177).  Exact
// in fixed point.
// ---------------------------------------------------------------------------
// One leaf of one signal b of a batch of B (the body of mp_leaf_kernel).
template <int L>
__device__ __forceinline__ void mp_leaf_one(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, int N,
                                            int B, int b, const MpLeaf lf) {
  const size_t plane = (size_t)N * B;   // distance between limb planes
  const size_t cim = (size_t)L * plane; // real -> imaginary component
  // element j of the leaf's subsequence: index (sn + j*s), j=0 wrapped to sn+N
  int idx[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) idx[j] = (j == 0 && lf.sn < 0) ? lf.sn + N : lf.sn + j * lf.s;
  const uint32_t *x[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) x[j] = in + (size_t)(j < lf.n ? idx[j] : 0) * B + b;
  uint32_t *y = out + (size_t)lf.out * B + b;
  const size_t yB = B;

  if (lf.n == 4) {
    // X0 = x0+x2 + (x1+x3)      X2 = x0+x2 - (x1+x3)
    // X1 = x0-x2 - i(x1-x3)     X3 = x0-x2 + i(x1-x3)
    int64_t c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < L; ++i) {
      const size_t o = i * plane;
      int64_t r[4], m[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t vr = x[j][o], vi = x[j][o + cim];
        r[j] = (i == L - 1) ? (int64_t)(int32_t)vr : (int64_t)vr;
        m[j] = (i == L - 1) ? (int64_t)(int32_t)vi : (int64_t)vi;
      }
      const int64_t er = r[0] + r[2], fr = r[0] - r[2], gr = r[1] + r[3], hr = r[1] - r[3];
      const int64_t ei = m[0] + m[2], fi = m[0] - m[2], gi = m[1] + m[3], hi = m[1] - m[3];
      const int64_t v[8] = {c[0] + er + gr, c[1] + fr + hi, c[2] + er - gr, c[3] + fr - hi,
                            c[4] + ei + gi, c[5] + fi - hr, c[6] + ei - gi, c[7] + fi + hr};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        y[o + q * yB] = (uint32_t)v[q];
        y[o + cim + q * yB] = (uint32_t)v[4 + q];
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) c[q] = v[q] >> 32;
    }
  } else if (lf.n == 2) {
    int64_t c[4] = {0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < L; ++i) {
      const size_t o = i * plane;
      int64_t r0 = x[0][o], r1 = x[1][o], i0 = x[0][o + cim], i1 = x[1][o + cim];
      if (i == L - 1) {
        r0 = (int32_t)r0; r1 = (int32_t)r1; i0 = (int32_t)i0; i1 = (int32_t)i1;
      }
      const int64_t v[4] = {c[0] + r0 + r1, c[1] + r0 - r1, c[2] + i0 + i1, c[3] + i0 - i1};
      y[o] = (uint32_t)v[0];
      y[o + yB] = (uint32_t)v[1];
      y[o + cim] = (uint32_t)v[2];
      y[o + cim + yB] = (uint32_t)v[3];
#pragma unroll
      for (int q = 0; q < 4; ++q) c[q] = v[q] >> 32;
    }
  } else {
#pragma unroll
    for (int i = 0; i < L; ++i) {
      const size_t o = i * plane;
      y[o] = x[0][o];
      y[o + cim] = x[0][o + cim];
    }
  }
}

// CTAs of 128 threads per SM the register allocation of a one-thread-per-
// butterfly kernel must allow: more warps hide more latency while the product
// still fits without spills (measured at N=1024, batch 2048: 13 limbs +15 %
// with 6 instead of 4, 17 limbs +8.5 % with 5; from 20 limbs up the smaller
// allocation spills).
template <int L>
constexpr int level_min_blocks() {
  return L <= 14 ? 6 : (L <= 19 ? 5 : 4);
}

// ---------------------------------------------------------------------------
// L-shaped combine of one butterfly (reference :238-252), streamed limb by
// limb: a1 = m1 + m2, a2 = m1 - m2, then U0 +/- a1 and U1 -/+ i a2, twelve
// independent modular carry chains.  m1 = Z+ w^k and m2 = Z- w^-k sit in the
// Z+ / Z- slots; when `swapped`, each slot holds (imag, real) instead of
// (real, imag) -- the twiddle stage writes them that way to stay in place.
// ---------------------------------------------------------------------------
template <int L>
__device__ __forceinline__ void combine(uint32_t *u0, uint32_t *u1, uint32_t *zp, uint32_t *zm, size_t plane,
                                        size_t cim, bool swapped) {
  const size_t sre = swapped ? cim : 0, sim = swapped ? 0 : cim;
  // carry-in of each chain: 0 for additions, 1 for subtractions (a - b = a + ~b + 1)
  uint32_t ca1r = 0, ca1i = 0, ca2r = 1, ca2i = 1;
  uint32_t c0r = 0, c2r = 1, c1r = 0, c3r = 1, c0i = 0, c2i = 1, c1i = 1, c3i = 0;
#pragma unroll
  for (int i = 0; i < L; ++i, u0 += plane, u1 += plane, zp += plane, zm += plane) {
    const uint32_t U0r = u0[0], U0i = u0[cim], U1r = u1[0], U1i = u1[cim];
    const uint32_t m1r = zp[sre], m1i = zp[sim], m2r = zm[sre], m2i = zm[sim];
    const uint32_t a1r = addc(m1r, m2r, ca1r), a1i = addc(m1i, m2i, ca1i);
    const uint32_t a2r = addc(m1r, ~m2r, ca2r), a2i = addc(m1i, ~m2i, ca2i);
    u0[0] = addc(U0r, a1r, c0r);
    zp[0] = addc(U0r, ~a1r, c2r);
    u1[0] = addc(U1r, a2i, c1r);
    zm[0] = addc(U1r, ~a2i, c3r);
    u0[cim] = addc(U0i, a1i, c0i);
    zp[cim] = addc(U0i, ~a1i, c2i);
    u1[cim] = addc(U1i, ~a2r, c1i);
    zm[cim] = addc(U1i, a2r, c3i);
  }
}

// ---------------------------------------------------------------------------
// the L-shaped butterfly with its twiddle products
// ---------------------------------------------------------------------------
//
// Butterfly k of a node (q = n/4 at output offset `off`):
//   U0 = y[off+k], U1 = y[off+k+q], Z+ = y[off+k+2q], Z- = y[off+k+3q]
//   k = 0     : no twiddle (reference :184-201)
//   k = q/2   : w^k = (1-i)/sqrt 2, products by cos(pi/4) (:213-221)
//   otherwise : 3 products per complex multiply with cos, cos+sin, cos-sin
//               (3m3a, :222-236); twiddle index kn = k*(N/n) into the N/4 table.
// Both twiddled cases run as six steps of one rolled loop around a single
// inlined product (one copy of its ~L^2 instructions keeps the instruction
// cache warm).  Per side (Z+ then Z-), the step's operand, twiddle and the
// rule that merges the product with P (the first product of the side, kept in
// shared memory) are:
//            step 0           step 1                      step 2
//   general  P=(Zr+-Zi)c      m.r = P -+ d Zi -> im slot   m.i = +-(P - s Zr) -> re slot
//   k = q/2  P=(Zr+-Zi)c      m.i = (Zi-Zr)c | (Zr+Zi)c    m.r = P -> im slot
//                                   -> re slot
// so m.r ends in the imaginary slot and m.i in the real slot ("swapped").
//
// The six twiddle steps of butterfly k != 0 of one signal, without the
// combine: the products of the Z+ slots (zp) and Z- slots (zm) by w^k and
// w^-k, merged and stored back into the slots swapped (m.r in the imaginary
// slot, m.i in the real one).  n: the node size (q = n/4); P: this thread's
// slot for the side's first product (words ps apart); Twp: the CTA's packed
// twiddles (kPackedTw only).  The merged products are stored with L2 priority
// evict_last (a fused thread of mp_level_pair_kernel reads them back only
// after two more butterflies).  mp_bfly_one below spells out the same steps
// inline (its register allocation at 33 limbs spills less that way); the
// kernels built on each are checked to be bit-identical.
template <int L, bool kPackedTw>
__device__ __forceinline__ void mp_bfly_steps(uint32_t *zp, uint32_t *zm, size_t plane, size_t cim, int N, int n,
                                              int k, const uint32_t *__restrict__ tw,
                                              const uint8_t *__restrict__ dneg, int tws, uint32_t *P, size_t ps,
                                              const uint32_t *Twp) {
  const int q = n >> 2;
  const size_t tplane = (size_t)(N >> 2) * tws;  // twiddle limb-plane stride
  const int kn = k * (N / n) * tws;
  const uint32_t *wr = tw + kn;                           // cos
  const uint32_t *ws = tw + (size_t)L * tplane + kn;      // cos + sin
  const uint32_t *wd = tw + (size_t)2 * L * tplane + kn;  // |cos - sin|
  const bool special = (2 * k == q);
  const bool dn = special ? false : (dneg[kn] != 0);
  constexpr int Lp = (L + 3) & ~3;  // packed twiddle stride: 16-byte aligned rows
  uint32_t X[L];
#pragma unroll 1
  for (int st_ = 0; st_ < 6; ++st_) {
    const int side = st_ >= 3;
    const int step = st_ - 3 * side;
    uint32_t *zr = side ? zm : zp;
    uint32_t *zi = zr + cim;
    const uint32_t *pa = zr, *pb = nullptr, *w = wr;
    int wsel = 0;  // packed twiddle row: 0 cos, 1 cos+sin, 2 |cos-sin|
    bool sub = false, negx = false, mul = true;
    int sp = 0;
    uint32_t *dst = nullptr;  // null: the product becomes P
    if (step == 0) {
      pb = zi;
      sub = side;
    } else if (!special) {
      if (step == 1) {
        pa = zi;
        w = wd;
        wsel = 2;
        negx = dn ^ (side == 0);
        sp = 1;
        dst = zi;
      } else {
        w = ws;
        wsel = 1;
        negx = (side == 0);
        sp = side ? -1 : 1;
        dst = zr;
      }
    } else {
      if (step == 1) {
        pa = side ? zr : zi;
        pb = side ? zi : zr;
        sub = !side;
        dst = zr;
      } else {
        mul = false;
        sp = 1;
        dst = zi;
      }
    }
    if (mul) {
      ld_addsub<L>(X, pa, pb, plane, sub);
      if (kPackedTw) mul_tw<L, true>(X, Twp + wsel * Lp, 0);
      else mul_tw<L>(X, w, tplane);
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) X[i] = 0;
    }
    if (!dst) {
      st<L>(P, ps, X);
    } else {
      combine_p<L>(X, P, ps, negx, sp);
      // the merged product is read again by the combine: keep it in L2
      const uint64_t keep = l2_policy_evict_last();
#pragma unroll
      for (int i = 0; i < L; ++i) st_hint(dst + (size_t)i * plane, X[i], keep);
    }
  }
}

// One butterfly k of one signal b (the body of mp_level_kernel): the node of
// size n at output offset off.  P: this thread's slot for the side's first
// product (words ps apart); Twp: the CTA's packed twiddles (kPackedTw only).
template <int L, bool kPackedTw>
__device__ __forceinline__ void mp_bfly_one(uint32_t *__restrict__ y, int N, int B, int b, int n, int off, int k,
                                            const uint32_t *__restrict__ tw, const uint8_t *__restrict__ dneg,
                                            int tws, uint32_t *P, size_t ps, const uint32_t *Twp) {
  const int q = n >> 2;
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  uint32_t *u0 = y + (size_t)(off + k) * B + b;
  uint32_t *u1 = u0 + (size_t)q * B;
  uint32_t *zp = u0 + (size_t)2 * q * B;
  uint32_t *zm = u0 + (size_t)3 * q * B;

  if (k == 0) {
    combine<L>(u0, u1, zp, zm, plane, cim, false);
    return;
  }
  const size_t tplane = (size_t)(N >> 2) * tws;  // twiddle limb-plane stride
  const int kn = k * (N / n) * tws;
  const uint32_t *wr = tw + kn;                           // cos
  const uint32_t *ws = tw + (size_t)L * tplane + kn;      // cos + sin
  const uint32_t *wd = tw + (size_t)2 * L * tplane + kn;  // |cos - sin|
  const bool special = (2 * k == q);
  const bool dn = special ? false : (dneg[kn] != 0);
  constexpr int Lp = (L + 3) & ~3;  // packed twiddle stride: 16-byte aligned rows
  uint32_t X[L];
#pragma unroll 1
  for (int st_ = 0; st_ < 6; ++st_) {
    const int side = st_ >= 3;
    const int step = st_ - 3 * side;
    uint32_t *zr = side ? zm : zp;
    uint32_t *zi = zr + cim;
    const uint32_t *pa = zr, *pb = nullptr, *w = wr;
    int wsel = 0;  // packed twiddle row: 0 cos, 1 cos+sin, 2 |cos-sin|
    bool sub = false, negx = false, mul = true;
    int sp = 0;
    uint32_t *dst = nullptr;  // null: the product becomes P
    if (step == 0) {
      pb = zi;
      sub = side;
    } else if (!special) {
      if (step == 1) {
        pa = zi;
        w = wd;
        wsel = 2;
        negx = dn ^ (side == 0);
        sp = 1;
        dst = zi;
      } else {
        w = ws;
        wsel = 1;
        negx = (side == 0);
        sp = side ? -1 : 1;
        dst = zr;
      }
    } else {
      if (step == 1) {
        pa = side ? zr : zi;
        pb = side ? zi : zr;
        sub = !side;
        dst = zr;
      } else {
        mul = false;
        sp = 1;
        dst = zi;
      }
    }
    if (mul) {
      ld_addsub<L>(X, pa, pb, plane, sub);
      if (kPackedTw) mul_tw<L, true>(X, Twp + wsel * Lp, 0);
      else mul_tw<L>(X, w, tplane);
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) X[i] = 0;
    }
    if (!dst) {
      st<L>(P, ps, X);
    } else {
      combine_p<L>(X, P, ps, negx, sp);
      st<L>(dst, plane, X);
    }
  }
  combine<L>(u0, u1, zp, zm, plane, cim, true);
}

}  // namespace mpfft
