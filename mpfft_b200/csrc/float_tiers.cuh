// Compensated floating-point tiers of the conjugate-pair split-radix FFT
// (device code shared by float_tier_kernels.cu and queue_kernels.cu):
// double-double (about 106 bits), quad-double (about 212 bits) and
// float-float (about 48 bits).
//
// A tier value is an unevaluated sum of K machine numbers (the "words") of
// decreasing magnitude, each at most half an ulp of the one above:
//   double-double  K = 2 doubles    hi + lo
//   quad-double    K = 4 doubles    x0 + x1 + x2 + x3
//   float-float    K = 2 floats     hi + lo
// The arithmetic is built from the published error-free transformations --
// Knuth's TwoSum, Dekker's Fast2Sum, the FMA form of TwoProd -- combined as in
// Hida, Li and Bailey's double-double / quad-double algorithms ("Algorithms
// for quad-double precision floating point arithmetic", ARITH 15, 2001):
// terms are summed order by order (order k = magnitude about 2^(-53k) of the
// leading word), the rounding errors of each order carried into the next,
// and the result renormalised with Fast2Sum / TwoSum chains.  Float-float
// keeps its additions on the FP32 pipe but forms every twiddle product, and
// rounds it back to a float pair, in FP64 (a float pair is exact in a
// double), which keeps the products at 2^-52 before the final 2^-48 rounding.
//
// Same tree and schedule as the FP64 kernels (d_kernels.cu): maximal nodes of
// up to T points run in shared memory (DIT-order gather, base cases of at
// most 4 points, every level up to the node), the levels above in global
// memory.  T is the largest sub-transform whose planes fit 64 KB: 2048 points
// for double-double, 1024 for quad-double, 4096 for float-float.  Every level
// is the 4m2a butterfly with twiddles cos and sin of 2 pi k/N rounded to the
// tier by MPFR (float-float: to double).  Layout: word (c, h, b, p) at
// base[((c*K + h)*B + b)*N + p] -- c real/imaginary, h the word, each signal
// contiguous.
#pragma once

#include <cstdint>

#include "mpfft_internal.h"

namespace mpfft {

// ---------------------------------------------------------------------------
// error-free transformations
// ---------------------------------------------------------------------------

struct dd {
  double h, l;
};

__device__ __forceinline__ dd two_sum(double a, double b) {  // Knuth: s + e = a + b exactly
  const double s = a + b;
  const double bb = s - a;
  return dd{s, (a - (s - bb)) + (b - bb)};
}

__device__ __forceinline__ dd fast_two_sum(double a, double b) {  // Dekker, |a| >= |b|
  const double s = a + b;
  return dd{s, b - (s - a)};
}

__device__ __forceinline__ dd two_prod(double a, double b) {  // p + e = a * b exactly (FMA)
  const double p = a * b;
  return dd{p, fma(a, b, -p)};
}

struct ff {
  float h, l;
};

__device__ __forceinline__ ff two_sum_f(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  return ff{s, __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb))};
}

__device__ __forceinline__ ff fast_two_sum_f(float a, float b) {
  const float s = __fadd_rn(a, b);
  return ff{s, __fsub_rn(b, __fsub_rn(s, a))};
}

// ---------------------------------------------------------------------------
// double-double
// ---------------------------------------------------------------------------

struct DDT {
  using W = double;  // storage word
  using V = dd;      // value
  using TW = dd;     // twiddle
  static constexpr int K = 2;
  static constexpr int kSubMax = kDDSubMax;

  // accurate addition (two TwoSums, two renormalisations)
  static __device__ __forceinline__ V add(V x, V y) {
    dd s = two_sum(x.h, y.h);
    const dd t = two_sum(x.l, y.l);
    s.l += t.h;
    s = fast_two_sum(s.h, s.l);
    s.l += t.l;
    return fast_two_sum(s.h, s.l);
  }
  static __device__ __forceinline__ V neg(V x) { return V{-x.h, -x.l}; }
  static __device__ __forceinline__ V sub(V x, V y) { return add(x, neg(y)); }
  static __device__ __forceinline__ V mul(V x, V y) {
    const double p = x.h * y.h;
    double e = fma(x.h, y.h, -p);  // TwoProd: p + e = x.h * y.h exactly
    e = fma(x.h, y.l, e);
    e = fma(x.l, y.h, e);
    return fast_two_sum(p, e);
  }
  static __device__ __forceinline__ V scale(V x, double s) { return V{x.h * s, x.l * s}; }
  static __device__ __forceinline__ V load(const W *p, size_t stride) { return V{p[0], p[stride]}; }
  static __device__ __forceinline__ void store(W *p, size_t stride, V v) {
    p[0] = v.h;
    p[stride] = v.l;
  }
  static __device__ __forceinline__ TW twiddle(const double *const *t, size_t k) {
    return TW{__ldg(t[0] + k), __ldg(t[1] + k)};
  }
};

// ---------------------------------------------------------------------------
// quad-double
// ---------------------------------------------------------------------------

struct qd {
  double x0, x1, x2, x3;
};

// Five terms of decreasing order -> four non-overlapping words: a Fast2Sum
// chain from the bottom compresses the terms, a TwoSum chain from the top
// (exact whatever the magnitudes) pushes what overlaps down again.
__device__ __forceinline__ qd qd_renorm(double c0, double c1, double c2, double c3, double c4) {
  dd t = fast_two_sum(c3, c4);
  c3 = t.h, c4 = t.l;
  t = fast_two_sum(c2, c3);
  c2 = t.h, c3 = t.l;
  t = fast_two_sum(c1, c2);
  c1 = t.h, c2 = t.l;
  t = fast_two_sum(c0, c1);
  c0 = t.h, c1 = t.l;
  t = two_sum(c1, c2);
  c1 = t.h, c2 = t.l;
  t = two_sum(c2, c3);
  c2 = t.h, c3 = t.l + c4;
  return qd{c0, c1, c2, c3};
}

struct QDT {
  using W = double;
  using V = qd;
  using TW = qd;
  static constexpr int K = 4;
  static constexpr int kSubMax = kQDSubMax;

  // Sum order by order: word i of x and of y are order i; the error of an
  // order-i TwoSum is order i+1; order 3 is summed plainly (its errors are
  // below 2^-212 relative).
  static __device__ __forceinline__ V add(const V &a, const V &b) {
    const dd s0 = two_sum(a.x0, b.x0);
    const dd s1 = two_sum(a.x1, b.x1);
    const dd s2 = two_sum(a.x2, b.x2);
    const double s3 = a.x3 + b.x3;
    const dd t1 = two_sum(s1.h, s0.l);   // order 1
    const dd u = two_sum(s2.h, s1.l);    // order 2 ...
    const dd t2 = two_sum(u.h, t1.l);
    const double t3 = s3 + s2.l + u.l + t2.l;  // order 3
    return qd_renorm(s0.h, t1.h, t2.h, t3, 0.0);
  }
  static __device__ __forceinline__ V neg(const V &x) { return V{-x.x0, -x.x1, -x.x2, -x.x3}; }
  static __device__ __forceinline__ V sub(const V &x, const V &y) { return add(x, neg(y)); }
  // Products of order 0..2 exactly (TwoProd), order 3 plainly, order >= 4
  // dropped (below 2^-210 relative); each order summed with TwoSums whose
  // errors go to the next order.
  static __device__ __forceinline__ V mul(const V &a, const V &b) {
    const dd p00 = two_prod(a.x0, b.x0);
    const dd p01 = two_prod(a.x0, b.x1), p10 = two_prod(a.x1, b.x0);
    const dd p02 = two_prod(a.x0, b.x2), p11 = two_prod(a.x1, b.x1), p20 = two_prod(a.x2, b.x0);
    const double o3 = fma(a.x0, b.x3, fma(a.x1, b.x2, fma(a.x2, b.x1, a.x3 * b.x0)));
    const dd t = two_sum(p01.h, p10.h);  // order 1
    const dd t1 = two_sum(t.h, p00.l);
    const dd u = two_sum(p02.h, p11.h);  // order 2
    const dd v = two_sum(u.h, p20.h);
    const dd w = two_sum(v.h, p01.l);
    const dd x = two_sum(w.h, p10.l);
    const dd y = two_sum(x.h, t.l);
    const dd t2 = two_sum(y.h, t1.l);
    const double t3 = o3 + (p02.l + p11.l + p20.l) + (u.l + v.l + w.l) + (x.l + y.l + t2.l);  // order 3
    return qd_renorm(p00.h, t1.h, t2.h, t3, 0.0);
  }
  static __device__ __forceinline__ V scale(const V &x, double s) { return V{x.x0 * s, x.x1 * s, x.x2 * s, x.x3 * s}; }
  static __device__ __forceinline__ V load(const W *p, size_t stride) {
    return V{p[0], p[stride], p[2 * stride], p[3 * stride]};
  }
  static __device__ __forceinline__ void store(W *p, size_t stride, const V &v) {
    p[0] = v.x0;
    p[stride] = v.x1;
    p[2 * stride] = v.x2;
    p[3 * stride] = v.x3;
  }
  static __device__ __forceinline__ TW twiddle(const double *const *t, size_t k) {
    return TW{__ldg(t[0] + k), __ldg(t[1] + k), __ldg(t[2] + k), __ldg(t[3] + k)};
  }
};

// ---------------------------------------------------------------------------
// float-float (additions on the FP32 pipe, twiddle products in FP64)
// ---------------------------------------------------------------------------

struct FFT_ {
  using W = float;
  using V = ff;
  using TW = double;
  static constexpr int K = 2;
  static constexpr int kSubMax = kFFSubMax;

  static __device__ __forceinline__ V add(V a, V b) {
    const ff s = two_sum_f(a.h, b.h);
    return fast_two_sum_f(s.h, __fadd_rn(s.l, __fadd_rn(a.l, b.l)));
  }
  static __device__ __forceinline__ V neg(V x) { return V{-x.h, -x.l}; }
  static __device__ __forceinline__ V sub(V x, V y) { return add(x, neg(y)); }
  static __device__ __forceinline__ V scale(V x, double s) { return V{x.h * (float)s, x.l * (float)s}; }
  static __device__ __forceinline__ double to_d(V a) { return (double)a.h + (double)a.l; }
  // renormalisation in FP64: the nearest float, then the nearest float to the rest
  static __device__ __forceinline__ V from_d(double v) {
    const float h = __double2float_rn(v);
    return V{h, __double2float_rn(v - (double)h)};
  }
  static __device__ __forceinline__ V load(const W *p, size_t stride) { return V{p[0], p[stride]}; }
  static __device__ __forceinline__ void store(W *p, size_t stride, V v) {
    p[0] = v.h;
    p[stride] = v.l;
  }
  static __device__ __forceinline__ TW twiddle(const double *const *t, size_t k) { return __ldg(t[0] + k); }
};

// ---------------------------------------------------------------------------
// the butterflies
// ---------------------------------------------------------------------------

// P = Z+ (c - i s) and M = Z- (c + i s), the twiddle products of the 4m2a
// butterfly (reference butterfly: lab/serial/double/serial_d_fft6.c:392-427)
template <class NT>
struct TwProducts {
  static __device__ __forceinline__ void run(typename NT::V zpr, typename NT::V zpi, typename NT::V zmr,
                                             typename NT::V zmi, typename NT::TW c, typename NT::TW s,
                                             typename NT::V &pr, typename NT::V &pi, typename NT::V &mr,
                                             typename NT::V &mi) {
    pr = NT::add(NT::mul(c, zpr), NT::mul(s, zpi));
    pi = NT::sub(NT::mul(c, zpi), NT::mul(s, zpr));
    mr = NT::sub(NT::mul(c, zmr), NT::mul(s, zmi));
    mi = NT::add(NT::mul(c, zmi), NT::mul(s, zmr));
  }
};

template <>
struct TwProducts<FFT_> {  // each complex product formed in FP64, rounded once to a float pair
  static __device__ __forceinline__ void run(ff zpr, ff zpi, ff zmr, ff zmi, double c, double s, ff &pr, ff &pi,
                                             ff &mr, ff &mi) {
    const double a = FFT_::to_d(zpr), b = FFT_::to_d(zpi), u = FFT_::to_d(zmr), v = FFT_::to_d(zmi);
    pr = FFT_::from_d(fma(c, a, s * b));
    pi = FFT_::from_d(fma(c, b, -(s * a)));
    mr = FFT_::from_d(fma(c, u, -(s * v)));
    mi = FFT_::from_d(fma(c, v, s * u));
  }
};

template <class NT>
__device__ __forceinline__ void bfly(typename NT::V &u0r, typename NT::V &u0i, typename NT::V &u1r,
                                     typename NT::V &u1i, typename NT::V &zpr, typename NT::V &zpi,
                                     typename NT::V &zmr, typename NT::V &zmi, typename NT::TW c, typename NT::TW s) {
  using V = typename NT::V;
  V pr, pi, mr, mi;
  TwProducts<NT>::run(zpr, zpi, zmr, zmi, c, s, pr, pi, mr, mi);
  const V sr = NT::add(pr, mr), si = NT::add(pi, mi), dr = NT::sub(pr, mr), di = NT::sub(pi, mi);
  const V a0r = NT::add(u0r, sr), a0i = NT::add(u0i, si), a2r = NT::sub(u0r, sr), a2i = NT::sub(u0i, si);
  const V a1r = NT::add(u1r, di), a1i = NT::sub(u1i, dr), a3r = NT::sub(u1r, di), a3i = NT::add(u1i, dr);
  u0r = a0r, u0i = a0i, u1r = a1r, u1i = a1i, zpr = a2r, zpi = a2i, zmr = a3r, zmi = a3i;
}

// shared-memory index: low 4 bits XOR-ed with bits 4-7 ^ 8-11, a permutation
// inside each 16-aligned block (for double-double 17 % fewer wavefronts than
// padding on this schedule, counted by simulating its accesses)
__device__ __forceinline__ int swz(int m) { return m ^ (((m >> 4) ^ (m >> 8)) & 15); }

// one shared-memory instance: 2K planes of pl words, [c][h][m]
template <class NT>
struct SPlanes {
  typename NT::W *base;
  int pl;
  __device__ typename NT::V re(int m) const { return NT::load(base + swz(m), pl); }
  __device__ typename NT::V im(int m) const { return NT::load(base + (size_t)NT::K * pl + swz(m), pl); }
  __device__ void set(int m, typename NT::V r, typename NT::V i) const {
    NT::store(base + swz(m), pl, r);
    NT::store(base + (size_t)NT::K * pl + swz(m), pl, i);
  }
};

// base cases on positions [o, o+n), in place (n = 4, 2, 1)
template <class NT>
__device__ void leaf(const SPlanes<NT> &P, int o, int n) {
  using V = typename NT::V;
  if (n == 4) {
    const V x0r = P.re(o), x1r = P.re(o + 1), x2r = P.re(o + 2), x3r = P.re(o + 3);
    const V x0i = P.im(o), x1i = P.im(o + 1), x2i = P.im(o + 2), x3i = P.im(o + 3);
    const V er = NT::add(x0r, x2r), fr = NT::sub(x0r, x2r), gr = NT::add(x1r, x3r), hr = NT::sub(x1r, x3r);
    const V ei = NT::add(x0i, x2i), fi = NT::sub(x0i, x2i), gi = NT::add(x1i, x3i), hi = NT::sub(x1i, x3i);
    P.set(o, NT::add(er, gr), NT::add(ei, gi));
    P.set(o + 1, NT::add(fr, hi), NT::sub(fi, hr));
    P.set(o + 2, NT::sub(er, gr), NT::sub(ei, gi));
    P.set(o + 3, NT::sub(fr, hi), NT::add(fi, hr));
  } else if (n == 2) {
    const V x0r = P.re(o), x1r = P.re(o + 1), x0i = P.im(o), x1i = P.im(o + 1);
    P.set(o, NT::add(x0r, x1r), NT::add(x0i, x1i));
    P.set(o + 1, NT::sub(x0r, x1r), NT::sub(x0i, x1i));
  }
}

struct TierTw {
  const double *c[4], *s[4];  // words of cos and sin of 2 pi k/N, k < N/4
};

// One CTA = G instances (sub-transform root x signal) in shared memory; see
// d_sub_kernel (d_kernels.cu) for the schedule.  swap_in / swap_out: read the
// input's / write the output's real and imaginary planes exchanged.
template <class NT, bool SINGLE>
__device__ __forceinline__ void tier_sub_instances(const typename NT::W *__restrict__ in,
                                                   typename NT::W *__restrict__ out, int N, int B, int b0, int G_here,
                                                   SubRoot rt, const SubSchedule &big, const SubSchedule &small,
                                                   const TierTw &tw, double scale, int swap_in, int swap_out,
                                                   typename NT::W *sm) {
  using W = typename NT::W;
  using V = typename NT::V;
  constexpr int K = NT::K;
  const int Tmax = big.size;
  const int lgT = 31 - __clz(Tmax);
  const int pl = Tmax;  // plane length
  const int tws = N / Tmax;
  const bool is_big = SINGLE || rt.size == Tmax;
  const int T = rt.size;
  const int *perm = is_big ? big.perm : small.perm;
  const Leaf *leaves = is_big ? big.leaves : small.leaves;
  const int nleaves = is_big ? big.nleaves : small.nleaves;
  const int nlevels = is_big ? big.nlevels : small.nlevels;
  auto inst = [&](int g) { return SPlanes<NT>{sm + (size_t)g * 2 * K * pl, pl}; };
  const size_t hplane = (size_t)B * N;          // word h -> word h+1
  const size_t cplane = (size_t)K * hplane;     // real -> imaginary component
  const size_t in_re = swap_in ? cplane : 0, in_im = swap_in ? 0 : cplane;
  const size_t out_re = swap_out ? cplane : 0, out_im = swap_out ? 0 : cplane;
  // gather: element j of instance g to DIT position perm[j], 4 elements per thread in flight
  const int total = G_here << lgT;
  for (int e0 = 0; e0 < total; e0 += 4 * (int)blockDim.x) {
    V vr[4], vi[4];
    int dst[4], gg[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * (int)blockDim.x + (int)threadIdx.x;
      const int g = e >> lgT, j = e & (Tmax - 1);
      dst[u] = -1;
      gg[u] = g;
      if (e < total && (SINGLE || j < T)) {
        int idx = rt.sn + j * rt.s;
        if (idx < 0) idx += N;
        const size_t o = (size_t)(b0 + g) * N + idx;
        vr[u] = NT::load(in + in_re + o, hplane);
        vi[u] = NT::load(in + in_im + o, hplane);
        dst[u] = perm[j];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (dst[u] >= 0) inst(gg[u]).set(dst[u], vr[u], vi[u]);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < G_here * nleaves; e += blockDim.x) {
    const int g = SINGLE ? e / nleaves : 0, l = SINGLE ? e - g * nleaves : e;
    const Leaf lf = leaves[l];
    leaf<NT>(inst(g), lf.out, lf.n);
  }
  for (int lv = 0; lv < nlevels; ++lv) {
    __syncthreads();
    const int n = big.level_n[lv], q = n >> 2, lgq = 29 - __clz(n);
    const int cnt = is_big ? big.level_count[lv] : small.level_count[lv];
    const int *nodes = (is_big ? big.node_off : small.node_off) + (is_big ? big.level_start[lv] : small.level_start[lv]);
    const int per = cnt * q;
    for (int e = threadIdx.x; e < G_here * per; e += blockDim.x) {
      const int g = SINGLE ? e / per : 0, t = SINGLE ? e - g * per : e;
      const int node = t >> lgq, k = t & (q - 1);
      const size_t km = (size_t)(k << (lgT - (lgq + 2))) * tws;  // k * (N/n)
      const SPlanes<NT> P = inst(g);
      const int off = nodes[node];
      V u0r = P.re(off + k), u0i = P.im(off + k), u1r = P.re(off + k + q), u1i = P.im(off + k + q);
      V zpr = P.re(off + k + 2 * q), zpi = P.im(off + k + 2 * q), zmr = P.re(off + k + 3 * q),
        zmi = P.im(off + k + 3 * q);
      bfly<NT>(u0r, u0i, u1r, u1i, zpr, zpi, zmr, zmi, NT::twiddle(tw.c, km), NT::twiddle(tw.s, km));
      P.set(off + k, u0r, u0i);
      P.set(off + k + q, u1r, u1i);
      P.set(off + k + 2 * q, zpr, zpi);
      P.set(off + k + 3 * q, zmr, zmi);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int g = e >> lgT, m = e & (Tmax - 1);
    if (!SINGLE && m >= T) continue;
    const SPlanes<NT> P = inst(g);
    const size_t o = (size_t)(b0 + g) * N + rt.out + m;
    NT::store(out + out_re + o, hplane, NT::scale(P.re(m), scale));
    NT::store(out + out_im + o, hplane, NT::scale(P.im(m), scale));
  }
}

// butterfly k of the node at offset off (size n) of signal b, above the
// shared-memory sub-transforms (in place in global memory)
template <class NT>
__device__ __forceinline__ void tier_level_one(typename NT::W *__restrict__ y, int N, int B, int n, int off, int k,
                                               int b, const TierTw &tw, double scale, int swap_out) {
  using W = typename NT::W;
  using V = typename NT::V;
  const int q = n >> 2;
  off += k;
  const size_t hplane = (size_t)B * N, cplane = (size_t)NT::K * hplane;
  W *re = y + (size_t)b * N, *im = y + cplane + (size_t)b * N;
  V u0r = NT::load(re + off, hplane), u0i = NT::load(im + off, hplane);
  V u1r = NT::load(re + off + q, hplane), u1i = NT::load(im + off + q, hplane);
  V zpr = NT::load(re + off + 2 * q, hplane), zpi = NT::load(im + off + 2 * q, hplane);
  V zmr = NT::load(re + off + 3 * q, hplane), zmi = NT::load(im + off + 3 * q, hplane);
  const size_t km = (size_t)k * (N / n);
  bfly<NT>(u0r, u0i, u1r, u1i, zpr, zpi, zmr, zmi, NT::twiddle(tw.c, km), NT::twiddle(tw.s, km));
  W *ore = swap_out ? im : re, *oim = swap_out ? re : im;
  NT::store(ore + off, hplane, NT::scale(u0r, scale));
  NT::store(oim + off, hplane, NT::scale(u0i, scale));
  NT::store(ore + off + q, hplane, NT::scale(u1r, scale));
  NT::store(oim + off + q, hplane, NT::scale(u1i, scale));
  NT::store(ore + off + 2 * q, hplane, NT::scale(zpr, scale));
  NT::store(oim + off + 2 * q, hplane, NT::scale(zpi, scale));
  NT::store(ore + off + 3 * q, hplane, NT::scale(zmr, scale));
  NT::store(oim + off + 3 * q, hplane, NT::scale(zmi, scale));
}

}  // namespace mpfft
