// Streamed limb arithmetic shared by the large-limb kernels (mp_big_kernels.cu,
// mp_tc_kernels.cu): every operand stays in memory (limb planes at a stride)
// and is processed limb by limb with carries.
#pragma once
#include <cstdint>

namespace mpfft {

__device__ __forceinline__ uint32_t add_c(uint32_t a, uint32_t b, uint32_t &c) {
  const uint64_t t = (uint64_t)a + b + c;
  c = (uint32_t)(t >> 32);
  return (uint32_t)t;
}

// dst = pa +/- pb (or pa when pb is null), streamed; returns the sign bit of dst
__device__ inline uint32_t big_addsub(uint32_t *dst, size_t ds, const uint32_t *pa, const uint32_t *pb, size_t ps, int L,
                                      bool sub) {
  const uint32_t m = sub ? 0xffffffffu : 0u;
  uint32_t c = sub ? 1u : 0u, v = 0;
  for (int i = 0; i < L; ++i) {
    v = pb ? add_c(pa[(size_t)i * ps], pb[(size_t)i * ps] ^ m, c) : pa[(size_t)i * ps];
    dst[(size_t)i * ds] = v;
  }
  return v >> 31;
}

// x = -x in place when neg (two's complement)
__device__ inline void big_cond_neg(uint32_t *x, size_t xs, int L, uint32_t neg) {
  if (!neg) return;
  uint32_t c = 1;
  for (int i = 0; i < L; ++i) x[(size_t)i * xs] = add_c(~x[(size_t)i * xs], 0, c);
}

// The L-combine, streamed (see mp_kernels.cu combine()).
__device__ inline void big_combine(uint32_t *u0, uint32_t *u1, uint32_t *zp, uint32_t *zm, size_t plane, size_t cim, int L,
                            bool swapped) {
  const size_t sre = swapped ? cim : 0, sim = swapped ? 0 : cim;
  uint32_t ca1r = 0, ca1i = 0, ca2r = 1, ca2i = 1;
  uint32_t c0r = 0, c2r = 1, c1r = 0, c3r = 1, c0i = 0, c2i = 1, c1i = 1, c3i = 0;
  for (int i = 0; i < L; ++i) {
    const size_t o = (size_t)i * plane;
    const uint32_t U0r = u0[o], U0i = u0[o + cim], U1r = u1[o], U1i = u1[o + cim];
    const uint32_t m1r = zp[o + sre], m1i = zp[o + sim], m2r = zm[o + sre], m2i = zm[o + sim];
    const uint32_t a1r = add_c(m1r, m2r, ca1r), a1i = add_c(m1i, m2i, ca1i);
    const uint32_t a2r = add_c(m1r, ~m2r, ca2r), a2i = add_c(m1i, ~m2i, ca2i);
    u0[o] = add_c(U0r, a1r, c0r);
    zp[o] = add_c(U0r, ~a1r, c2r);
    u1[o] = add_c(U1r, a2i, c1r);
    zm[o] = add_c(U1r, ~a2i, c3r);
    u0[o + cim] = add_c(U0i, a1i, c0i);
    zp[o + cim] = add_c(U0i, ~a1i, c2i);
    u1[o + cim] = add_c(U1i, ~a2r, c1i);
    zm[o + cim] = add_c(U1i, a2r, c3i);
  }
}

}  // namespace mpfft
