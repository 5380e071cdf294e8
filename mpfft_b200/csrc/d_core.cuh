// Device functions of the FP64 conjugate-pair split-radix kernels: the
// reference's n=8 and n=16 base cases, the 4m2a butterfly and one CTA's
// shared-memory sub-transform instances.  Shared by the per-launch kernels
// (d_kernels.cu) and the persistent work-queue kernels (queue_kernels.cu);
// every file that includes it is compiled with --fmad=false so that no
// multiply-add is contracted and results stay bit-identical to the reference.
#pragma once

#include <cstdint>

#include "mpfft_internal.h"

namespace mpfft {

struct DConst {
  double c8, c16a, c16b, c16c, c16d;
};

// 8-point base case on one part (reference :153-191); v = b1..b8
__device__ __forceinline__ void d8_part(const DConst &K, const double *x, double *v) {
  const double s04 = x[0] + x[4], d04 = x[0] - x[4];
  const double s26 = x[2] + x[6], d26 = x[2] - x[6];
  const double s17 = x[1] + x[7], d17 = x[1] - x[7];
  const double s35 = x[3] + x[5], d35 = x[3] - x[5];
  const double p = K.c8 * (d17 + d35);
  const double q = K.c8 * (s17 - s35);
  v[0] = s17 + s35;
  v[1] = s04 + s26;
  v[2] = s04 - s26;
  v[3] = d17 - d35;
  v[4] = d04 + q;
  v[5] = d04 - q;
  v[6] = d26 + p;
  v[7] = d26 - p;
}

struct D16 {
  double b5, b6, b11, b12, c1, c2, c3, c4, c9, c10, c11, c12, c17, c18, c19, c20;
};

// 16-point base case on one part (reference :218-348); the imaginary-part
// variant has a10, b3, b12 and the products m2, m4, m5, m6, m7 with the
// opposite sign convention, exactly as the reference writes them.
__device__ __forceinline__ void d16_part(const DConst &K, const double *x, bool im, D16 &o) {
  double s[8], d[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    s[j] = x[j] + x[j + 8];
    d[j] = x[j] - x[j + 8];
  }
  const double a10 = im ? (-x[4] + x[12]) : d[4];
  const double b1 = s[0] - s[4], b2 = s[0] + s[4];
  const double b3 = im ? (-s[2] + s[6]) : (s[2] - s[6]);
  const double b4 = s[2] + s[6];
  const double b7 = s[1] - s[5], b8 = s[1] + s[5];
  const double b9 = s[3] - s[7], b10 = s[3] + s[7];
  const double b13 = d[1] + d[7], b14 = d[1] - d[7];
  const double b15 = d[3] + d[5], b16 = d[5] - d[3];
  o.b5 = b2 + b4;
  o.b6 = b2 - b4;
  o.b11 = b8 + b10;
  o.b12 = im ? (-b8 + b10) : (b8 - b10);
  const double m1 = K.c8 * (d[2] - d[6]);
  const double m2 = (im ? -K.c8 : K.c8) * (d[2] + d[6]);
  const double m3 = K.c8 * (b7 - b9);
  const double m4 = (im ? -K.c8 : K.c8) * (b7 + b9);
  const double m5 = (im ? -K.c16a : K.c16a) * (b13 + b15);
  const double m6 = (im ? K.c16b : -K.c16b) * b13;
  const double m7 = (im ? -K.c16d : K.c16d) * b15;
  const double m8 = K.c16c * (b14 + b16);
  const double m9 = K.c16d * b14;
  const double m10 = -K.c16b * b16;
  o.c1 = b1 + m3;
  o.c2 = b1 - m3;
  o.c3 = b3 + m4;
  o.c4 = m4 - b3;
  const double c5 = d[0] + m1, c6 = d[0] - m1;
  const double c7 = m9 - m8, c8 = m10 - m8;
  o.c9 = c5 + c7;
  o.c10 = c5 - c7;
  o.c11 = c6 + c8;
  o.c12 = c6 - c8;
  const double c13 = a10 + m2, c14 = a10 - m2;
  const double c15 = m5 + m6, c16 = m5 - m7;
  o.c17 = c13 + c15;
  o.c18 = c13 - c15;
  o.c19 = c14 + c16;
  o.c20 = c14 - c16;
}

// Shared-memory index: the low 4 bits of m XOR-ed with bits 4-7 ^ 8-11 (a
// permutation inside every 16-aligned block, so a plane needs no padding).
// Leaves work on 16 (or 8) consecutive elements per thread, levels on
// consecutive k, the DIT gather on scattered positions; over the whole
// 4096-point schedule this needs 29 % fewer shared-memory wavefronts than one
// pad slot per 16 elements (counted by simulating every access of the
// schedule per half-warp and bank).
__device__ __forceinline__ int pidx(int m) { return m ^ (((m >> 4) ^ (m >> 8)) & 15); }

// Leaf of size 16 at positions [o, o+16) (reference :213-385), in place.
__device__ __forceinline__ void d_leaf16(const DConst &K, double *yr, double *yi, int o) {
  double xr[16], xi[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    xr[j] = yr[pidx(o + j)];
    xi[j] = yi[pidx(o + j)];
  }
  D16 R, I;
  d16_part(K, xr, false, R);
  d16_part(K, xi, true, I);
  // output stage (reference :350-382)
  double *r = yr, *i = yi;
#define P(j) pidx(o + (j))
  r[P(0)] = R.b5 + R.b11;  r[P(8)] = R.b5 - R.b11;
  i[P(0)] = I.b5 + I.b11;  i[P(8)] = I.b5 - I.b11;
  r[P(4)] = R.b6 - I.b12;  r[P(12)] = R.b6 + I.b12;
  i[P(4)] = I.b6 - R.b12;  i[P(12)] = I.b6 + R.b12;
  r[P(1)] = R.c9 - I.c17;  r[P(15)] = R.c9 + I.c17;
  i[P(1)] = I.c9 - R.c17;  i[P(15)] = I.c9 + R.c17;
  r[P(2)] = R.c1 - I.c3;   r[P(14)] = R.c1 + I.c3;
  i[P(2)] = I.c1 - R.c3;   i[P(14)] = I.c1 + R.c3;
  r[P(3)] = R.c12 + I.c20; r[P(13)] = R.c12 - I.c20;
  i[P(3)] = I.c12 + R.c20; i[P(13)] = I.c12 - R.c20;
  r[P(5)] = R.c11 - I.c19; r[P(11)] = R.c11 + I.c19;
  i[P(5)] = I.c11 - R.c19; i[P(11)] = I.c11 + R.c19;
  r[P(6)] = R.c2 - I.c4;   r[P(10)] = R.c2 + I.c4;
  i[P(6)] = I.c2 - R.c4;   i[P(10)] = I.c2 + R.c4;
  r[P(7)] = R.c10 + I.c18; r[P(9)] = R.c10 - I.c18;
  i[P(7)] = I.c10 + R.c18; i[P(9)] = I.c10 - R.c18;
#undef P
}

// Leaf of size 8 at positions [o, o+8) (reference :148-212), in place.
__device__ __forceinline__ void d_leaf8(const DConst &K, double *yr, double *yi, int o) {
  double xr[8], xi[8], R[8], I[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    xr[j] = yr[pidx(o + j)];
    xi[j] = yi[pidx(o + j)];
  }
  d8_part(K, xr, R);
  d8_part(K, xi, I);
  // output stage (reference :193-209)
#define P(j) pidx(o + (j))
  yr[P(0)] = R[1] + R[0]; yr[P(4)] = R[1] - R[0];
  yi[P(0)] = I[1] + I[0]; yi[P(4)] = I[1] - I[0];
  yr[P(1)] = R[4] + I[6]; yr[P(7)] = R[4] - I[6];
  yi[P(1)] = I[4] - R[6]; yi[P(7)] = I[4] + R[6];
  yr[P(2)] = R[2] + I[3]; yr[P(6)] = R[2] - I[3];
  yi[P(2)] = I[2] - R[3]; yi[P(6)] = I[2] + R[3];
  yr[P(3)] = R[5] - I[7]; yr[P(5)] = R[5] + I[7];
  yi[P(3)] = I[5] + R[7]; yi[P(5)] = I[5] - R[7];
#undef P
}

// Leaves of size 4, 2, 1 (only when the whole transform has N <= 4).
__device__ __forceinline__ void d_leaf_small(double *yr, double *yi, int o, int n) {
  double xr[4], xi[4];
  for (int j = 0; j < n; ++j) {
    xr[j] = yr[pidx(o + j)];
    xi[j] = yi[pidx(o + j)];
  }
  if (n == 4) {  // reference :121-147
    const double er = xr[0] + xr[2], fr = xr[0] - xr[2], gr = xr[1] + xr[3], hr = xr[1] - xr[3];
    const double ei = xi[0] + xi[2], fi = xi[0] - xi[2], gi = xi[1] + xi[3], hi = xi[1] - xi[3];
    yr[pidx(o + 0)] = er + gr; yr[pidx(o + 1)] = fr + hi; yr[pidx(o + 2)] = er - gr; yr[pidx(o + 3)] = fr - hi;
    yi[pidx(o + 0)] = ei + gi; yi[pidx(o + 1)] = fi - hr; yi[pidx(o + 2)] = ei - gi; yi[pidx(o + 3)] = fi + hr;
  } else if (n == 2) {  // reference :108-120
    yr[pidx(o)] = xr[0] + xr[1]; yr[pidx(o + 1)] = xr[0] - xr[1];
    yi[pidx(o)] = xi[0] + xi[1]; yi[pidx(o + 1)] = xi[0] - xi[1];
  }
}

// 4m2a butterfly k of a node of size n at y[off..) (reference :392-427)
// (outputs to the planes exchanged when swap_out: the last launch of an inverse)
__device__ __forceinline__ void d_butterfly(double *yr, double *yi, size_t stride, int off, int k, int q,
                                            double w_r, double w_i, double scale, bool swap_out = false) {
  double *r0 = yr + (size_t)(off + k) * stride, *i0 = yi + (size_t)(off + k) * stride;
  const size_t qs = (size_t)q * stride;
  const double u0r = r0[0], u1r = r0[qs], zpr = r0[2 * qs], zmr = r0[3 * qs];
  const double u0i = i0[0], u1i = i0[qs], zpi = i0[2 * qs], zmi = i0[3 * qs];
  const double pr = w_r * zpr + w_i * zpi, pi = w_r * zpi - w_i * zpr;
  const double mr = w_r * zmr - w_i * zmi, mi = w_r * zmi + w_i * zmr;
  const double sr = pr + mr, si = pi + mi, dr = pr - mr, di = pi - mi;
  if (swap_out) {
    double *t = r0;
    r0 = i0;
    i0 = t;
  }
  r0[0] = (u0r + sr) * scale;
  r0[2 * qs] = (u0r - sr) * scale;
  r0[qs] = (u1r + di) * scale;
  r0[3 * qs] = (u1r - di) * scale;
  i0[0] = (u0i + si) * scale;
  i0[2 * qs] = (u0i - si) * scale;
  i0[qs] = (u1i - dr) * scale;
  i0[3 * qs] = (u1i + dr) * scale;
}

// 4m2a butterfly on values in registers: (U0, U1, Z+, Z-) -> the outputs that
// go to the same four positions (the operations of d_butterfly)
struct DCplx {
  double r, i;
};
__device__ __forceinline__ void d_bfly_vals(DCplx &u0, DCplx &u1, DCplx &zp, DCplx &zm, double w_r, double w_i,
                                            double scale) {
  const double pr = w_r * zp.r + w_i * zp.i, pi = w_r * zp.i - w_i * zp.r;
  const double mr = w_r * zm.r - w_i * zm.i, mi = w_r * zm.i + w_i * zm.r;
  const double sr = pr + mr, si = pi + mi, dr = pr - mr, di = pi - mi;
  const DCplx a = u0, b = u1;
  u0 = DCplx{(a.r + sr) * scale, (a.i + si) * scale};
  zp = DCplx{(a.r - sr) * scale, (a.i - si) * scale};
  u1 = DCplx{(b.r + di) * scale, (b.i - dr) * scale};
  zm = DCplx{(b.r - di) * scale, (b.i + dr) * scale};
}

// 4m2a butterfly in shared memory (padded indices)
__device__ __forceinline__ void d_butterfly_smem(double *yr, double *yi, int off, int k, int q, double w_r,
                                                 double w_i, double scale) {
  const int a[4] = {pidx(off + k), pidx(off + k + q), pidx(off + k + 2 * q), pidx(off + k + 3 * q)};
  DCplx v[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) v[j] = DCplx{yr[a[j]], yi[a[j]]};
  d_bfly_vals(v[0], v[1], v[2], v[3], w_r, w_i, scale);
#pragma unroll
  for (int j = 0; j < 4; ++j) yr[a[j]] = v[j].r, yi[a[j]] = v[j].i;
}

// Two levels of one node in shared memory: butterfly k of the first child X
// (size n, q = n/4, at the node's offset) and butterflies k and k+q of the node
// Y (size 2n), whose U inputs are exactly X's four outputs -- they stay in
// registers between the two levels.  wx: X's twiddle; wy0, wy1: Y's for k and
// k+q; scale applies to Y's outputs.
__device__ __forceinline__ void d_bfly_pair_smem(double *yr, double *yi, int off, int k, int q, double wx_r,
                                                 double wx_i, double wy0_r, double wy0_i, double wy1_r,
                                                 double wy1_i, double scale) {
  int a[8];
  DCplx v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    a[j] = pidx(off + k + j * q);
    v[j] = DCplx{yr[a[j]], yi[a[j]]};
  }
  d_bfly_vals(v[0], v[1], v[2], v[3], wx_r, wx_i, 1.0);
  d_bfly_vals(v[0], v[2], v[4], v[6], wy0_r, wy0_i, scale);
  d_bfly_vals(v[1], v[3], v[5], v[7], wy1_r, wy1_i, scale);
#pragma unroll
  for (int j = 0; j < 8; ++j) yr[a[j]] = v[j].r, yi[a[j]] = v[j].i;
}

// One CTA = G instances (sub-transform root x signal) entirely in shared
// memory.  SINGLE: N < 4096, one root per signal, G signals per CTA, all with
// the big schedule.  Otherwise G = 1 and the CTA's root may be of size T or
// T/2.  Per instance: gather the root's input sequence in input order
// (coalesced reads) into DIT positions, leaves, levels, then write the outputs
// once.  The twiddles the levels need, LUT[m*(N/T)] for m < T/4, are read
// through L1 (a few KB, shared by all CTAs).
// The instances of one CTA: G_here signals b0.. of root rt (SINGLE: the whole
// transform, several signals per CTA; otherwise one signal, and the root may
// be of size T or T/2), sm the CTA's shared memory.
template <bool SINGLE>
__device__ __forceinline__ void d_sub_instances(const double *__restrict__ in, double *__restrict__ out, int N, int B,
                                                int b0, int G_here, SubRoot rt, const SubSchedule &big,
                                                const SubSchedule &small, const double *__restrict__ wr,
                                                const double *__restrict__ wi, const DConst &K, double scale,
                                                int swap_in, int swap_out, double *sm) {
  const int Tmax = big.size;
  const int lgT = 31 - __clz(Tmax);
  const int istride = 2 * Tmax;  // doubles per instance: real plane, imaginary plane
  const int tws = N / Tmax;                  // twiddle table stride of this sub-transform
  const bool is_big = SINGLE || rt.size == Tmax;
  const int T = rt.size;
  const int *perm = is_big ? big.perm : small.perm;
  const Leaf *leaves = is_big ? big.leaves : small.leaves;
  const int nleaves = is_big ? big.nleaves : small.nleaves;
  const int n16 = is_big ? big.nleaf16 : small.nleaf16, n8 = is_big ? big.nleaf8 : small.nleaf8;
  const int nlevels = is_big ? big.nlevels : small.nlevels;
  // gather: element j of instance g to DIT position perm[j]; 8 elements per
  // thread are loaded before any is stored, so their latencies overlap
  const int total = G_here << lgT;
  for (int e0 = 0; e0 < total; e0 += 8 * (int)blockDim.x) {
    double vr[8], vi[8];
    int dst[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * (int)blockDim.x + (int)threadIdx.x;
      const int g = e >> lgT, j = e & (Tmax - 1);
      dst[u] = -1;
      if (e < total && (SINGLE || j < T)) {
        int idx = rt.sn + j * rt.s;
        if (idx < 0) idx += N;
        const size_t b = (size_t)(b0 + g);
        vr[u] = in[(swap_in ? (size_t)B + b : b) * N + idx];
        vi[u] = in[(swap_in ? b : (size_t)B + b) * N + idx];
        dst[u] = g * istride + pidx(perm[j]);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (dst[u] >= 0) {
        sm[dst[u]] = vr[u];
        sm[dst[u] + Tmax] = vi[u];
      }
  }
  __syncthreads();
  // leaves, grouped by size: 16-point, then 8-point, then (N <= 4 only) smaller
  for (int e = threadIdx.x; e < G_here * nleaves; e += blockDim.x) {
    const int g = SINGLE ? e / nleaves : 0, l = SINGLE ? e - g * nleaves : e;
    double *yr = sm + (size_t)g * istride, *yi = yr + Tmax;
    const Leaf lf = leaves[l];
    if (l < n16) d_leaf16(K, yr, yi, lf.out);
    else if (l < n16 + n8) d_leaf8(K, yr, yi, lf.out);
    else d_leaf_small(yr, yi, lf.out, lf.n);
  }
  if (nlevels == 0 && scale != 1.0) {
    __syncthreads();
    for (int e = threadIdx.x; e < (G_here << lgT); e += blockDim.x) {
      const int g = e >> lgT, m = e & (Tmax - 1);
      double *yr = sm + (size_t)g * istride, *yi = yr + Tmax;
      yr[pidx(m)] *= scale;
      yi[pidx(m)] *= scale;
    }
  }
  // levels (the small schedule's levels are the big one's minus the last),
  // two per pass: each node of the upper level with its first child, then the
  // lower level's other nodes; an odd top level runs alone
  const SubSchedule &S = is_big ? big : small;
  for (int lv = 0; lv < nlevels; ++lv) {
    __syncthreads();
    const int n = big.level_n[lv], q = n >> 2, lgq = 29 - __clz(n);
    if (lv + 1 < nlevels) {
      const int cy = S.level_count[lv + 1], cu = S.pair_count[lv];
      const int *ynodes = S.node_off + S.level_start[lv + 1], *unodes = S.pair_nodes + S.pair_start[lv];
      const int per = (cy + cu) * q;
      const double sc = lv + 1 == nlevels - 1 ? scale : 1.0;
      for (int e = threadIdx.x; e < G_here * per; e += blockDim.x) {
        const int g = SINGLE ? e / per : 0, t = SINGLE ? e - g * per : e;
        const int node = t >> lgq, k = t & (q - 1);
        const int km = k << (lgT - (lgq + 2));  // k * (T/n)
        double *yr = sm + (size_t)g * istride, *yi = yr + Tmax;
        if (node < cy) {
          const int ky0 = k << (lgT - (lgq + 3)), ky1 = (k + q) << (lgT - (lgq + 3));  // k * (T/2n), (k+q) * (T/2n)
          d_bfly_pair_smem(yr, yi, ynodes[node], k, q, __ldg(wr + (size_t)km * tws), __ldg(wi + (size_t)km * tws),
                           __ldg(wr + (size_t)ky0 * tws), __ldg(wi + (size_t)ky0 * tws),
                           __ldg(wr + (size_t)ky1 * tws), __ldg(wi + (size_t)ky1 * tws), sc);
        } else {
          d_butterfly_smem(yr, yi, unodes[node - cy], k, q, __ldg(wr + (size_t)km * tws),
                           __ldg(wi + (size_t)km * tws), 1.0);
        }
      }
      ++lv;
      continue;
    }
    const int cnt = is_big ? big.level_count[lv] : small.level_count[lv];
    const int *nodes = (is_big ? big.node_off : small.node_off) + (is_big ? big.level_start[lv] : small.level_start[lv]);
    const int per = cnt * q;
    const double sc = lv == nlevels - 1 ? scale : 1.0;
    for (int e = threadIdx.x; e < G_here * per; e += blockDim.x) {
      const int g = SINGLE ? e / per : 0, t = SINGLE ? e - g * per : e;
      const int node = t >> lgq, k = t & (q - 1);
      const int km = k << (lgT - (lgq + 2));  // k * (T/n)
      double *yr = sm + (size_t)g * istride, *yi = yr + Tmax;
      d_butterfly_smem(yr, yi, nodes[node], k, q, __ldg(wr + (size_t)km * tws), __ldg(wi + (size_t)km * tws), sc);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < (G_here << lgT); e += blockDim.x) {
    const int g = e >> lgT, m = e & (Tmax - 1);
    if (!SINGLE && m >= T) continue;
    const int b = b0 + g;
    const double *yr = sm + (size_t)g * istride, *yi = yr + Tmax;
    out[(swap_out ? (size_t)B + b : (size_t)b) * N + rt.out + m] = yr[pidx(m)];
    out[(swap_out ? (size_t)b : (size_t)B + b) * N + rt.out + m] = yi[pidx(m)];
  }
}

}  // namespace mpfft
