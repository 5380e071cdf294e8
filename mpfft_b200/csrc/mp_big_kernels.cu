// Multiprecision kernels for large limb counts (L > 34, i.e. P above ~1040
// bits; up to kMaxLimbsBig limbs), where an operand no longer fits in
// registers.
//
// Same schedule, number format and arithmetic as mp_kernels.cu (one leaf
// launch, one launch per node size, 3m3a butterflies, L-combine), but every
// operand stays in memory and is streamed limb by limb:
//   * adds, subtracts and the L-combine are single passes with carries;
//   * a twiddle product is formed column block by column block (product
//     scanning): each block of 8 result columns accumulates its partial
//     products x_i * w_(c-i) as 96-bit column sums while a window of twiddle
//     limbs slides along, then the columns are carried out in order, shifted
//     by 31 bits and streamed into their destination;
//   * per thread, the magnitude of the current operand and the first product
//     of the current side live in a global scratch buffer (plan-owned, limb
//     planes indexed by thread), read back through L1/L2.
// As in the register kernels, partial products below column L-2 are dropped
// (error < L*2^-31 ulp) and the product is rounded to nearest.
#include <cstdint>

#include "mp_stream.cuh"
#include "mpfft_internal.h"

namespace mpfft {

constexpr int kCB = 8;  // result columns per block

// Signed product streamed into its use:
//   r = sign * round(|x| * w / 2^(32L-1))       (|x| in ax, sign = xneg)
//   dst = sx*r + sp*P                           (sx = -1 when negx; sp in {-1,0,1})
// w: twiddle magnitude limbs at stride tw_s.  Column sums of columns L-2 ..
// 2L-1 are built in blocks of kCB; limbs are carried out in order and every
// finished result limb is negated / merged / stored immediately.
__device__ void big_mul_merge(const uint32_t *ax, size_t as, const uint32_t *w, size_t tw_s, int L, uint32_t xneg,
                              bool negx, const uint32_t *P, size_t ps, int sp, uint32_t *dst, size_t ds) {
  const int ncol = L + 2;  // columns L-2 .. 2L-1 -> a = 0 .. L+1
  // carry state between blocks (column value carried upward: < 2^41)
  uint64_t carry = 0;
  uint32_t prev = 0;        // limb a-1 (for the >> 31 funnel shift)
  int emitted = 0;          // result limbs written so far
  // output chains: result sign (r = -r when xneg), merge sign and P
  const bool rneg = (xneg != 0) != negx;  // sx * sign
  const uint32_t rm = rneg ? 0xffffffffu : 0u;
  uint32_t cr = rneg ? 1u : 0u;
  const uint32_t pm = sp < 0 ? 0xffffffffu : 0u;
  const uint32_t keep = sp != 0 ? 0xffffffffu : 0u;
  uint32_t cm = sp < 0 ? 1u : 0u;
  for (int a0 = 0; a0 < ncol; a0 += kCB) {
    uint64_t lo[kCB];
    uint32_t hi[kCB];
#pragma unroll
    for (int u = 0; u < kCB; ++u) {
      lo[u] = 0;
      hi[u] = 0;
    }
    if (a0 <= 1 && 1 < a0 + kCB) lo[1 - a0] = 1ull << 30;  // rounding: + 2^(32L-2)
    const int c0 = L - 2 + a0;                            // first column of the block
    const int c1 = min(L - 2 + a0 + kCB - 1, 2 * L - 1);  // last column
    // i ranges over x limbs contributing to any column of the block
    const int ilo = max(0, c0 - (L - 1)), ihi = min(L - 1, c1);
    // window: wv[u] = w[c0 + u - i]
    uint32_t wv[kCB];
#pragma unroll
    for (int u = 0; u < kCB; ++u) {
      const int j = c0 + u - ilo;
      wv[u] = (j >= 0 && j < L) ? w[(size_t)j * tw_s] : 0u;
    }
    for (int i = ilo; i <= ihi; ++i) {
      const uint32_t xi = ax[(size_t)i * as];
#pragma unroll
      for (int u = 0; u < kCB; ++u) {
        const uint64_t p = (uint64_t)xi * wv[u];
        const uint64_t s = lo[u] + p;
        hi[u] += s < p;
        lo[u] = s;
      }
      // slide: next i needs w[c0 + u - i - 1]
#pragma unroll
      for (int u = kCB - 1; u > 0; --u) wv[u] = wv[u - 1];
      const int j = c0 - i - 1;
      wv[0] = (j >= 0 && j < L) ? w[(size_t)j * tw_s] : 0u;
    }
    // carry out the block's columns in order and stream the result limbs
    for (int u = 0; u < kCB && a0 + u < ncol; ++u) {
      const int a = a0 + u;
      // column value + carry (carry < 2^41, column < 2^73): split into limb and carry
      const uint64_t s = lo[u] + carry;
      const uint64_t hc = (uint64_t)hi[u] + (s < lo[u] ? 1u : 0u);
      const uint32_t limb = (uint32_t)s;
      carry = (s >> 32) | (hc << 32);
      if (a >= 2) {  // result limb a-2 = (limb a-1 >> 31) | (limb a << 1)
        const uint32_t r = __funnelshift_r(prev, limb, 31);
        const uint32_t rv = add_c(r ^ rm, 0, cr);
        const uint32_t pv = P ? ((P[(size_t)emitted * ps] & keep) ^ pm) : 0u;
        dst[(size_t)emitted * ds] = add_c(rv, pv, cm);
        ++emitted;
      }
      prev = limb;
    }
  }
}

// leaves (n = 4, 2, 1), streamed; see mp_leaf_kernel
__global__ void __launch_bounds__(256) mp_big_leaf_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                           int N, int B, int L, const Leaf *__restrict__ leaves,
                                                           int nleaves) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nleaves * B) return;
  const int b = (int)(t % B);
  const Leaf lf = leaves[t / B];
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  int idx[4];
  for (int j = 0; j < 4; ++j) idx[j] = (j == 0 && lf.sn < 0) ? lf.sn + N : lf.sn + j * lf.s;
  const uint32_t *x[4];
  for (int j = 0; j < 4; ++j) x[j] = in + (size_t)(j < lf.n ? idx[j] : 0) * B + b;
  uint32_t *y = out + (size_t)lf.out * B + b;
  const size_t yB = B;
  int64_t c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < L; ++i) {
    const size_t o = (size_t)i * plane;
    const bool top = i == L - 1;
    auto s64 = [top](uint32_t v) -> int64_t { return top ? (int64_t)(int32_t)v : (int64_t)v; };
    if (lf.n == 4) {
      int64_t r[4], m[4];
      for (int j = 0; j < 4; ++j) {
        r[j] = s64(x[j][o]);
        m[j] = s64(x[j][o + cim]);
      }
      const int64_t er = r[0] + r[2], fr = r[0] - r[2], gr = r[1] + r[3], hr = r[1] - r[3];
      const int64_t ei = m[0] + m[2], fi = m[0] - m[2], gi = m[1] + m[3], hi = m[1] - m[3];
      const int64_t v[8] = {c[0] + er + gr, c[1] + fr + hi, c[2] + er - gr, c[3] + fr - hi,
                            c[4] + ei + gi, c[5] + fi - hr, c[6] + ei - gi, c[7] + fi + hr};
      for (int q = 0; q < 4; ++q) {
        y[o + q * yB] = (uint32_t)v[q];
        y[o + cim + q * yB] = (uint32_t)v[4 + q];
      }
      for (int q = 0; q < 8; ++q) c[q] = v[q] >> 32;
    } else if (lf.n == 2) {
      const int64_t r0 = s64(x[0][o]), r1 = s64(x[1][o]), i0 = s64(x[0][o + cim]), i1 = s64(x[1][o + cim]);
      const int64_t v[4] = {c[0] + r0 + r1, c[1] + r0 - r1, c[2] + i0 + i1, c[3] + i0 - i1};
      y[o] = (uint32_t)v[0];
      y[o + yB] = (uint32_t)v[1];
      y[o + cim] = (uint32_t)v[2];
      y[o + cim + yB] = (uint32_t)v[3];
      for (int q = 0; q < 4; ++q) c[q] = v[q] >> 32;
    } else {
      y[o] = x[0][o];
      y[o + cim] = x[0][o + cim];
    }
  }
}

// every butterfly of every node of size n; scratch: [2][L][nthreads] words
// (|operand| and P of each thread)
__global__ void __launch_bounds__(128) mp_big_level_kernel(uint32_t *__restrict__ y, int N, int B, int L, int n,
                                                            const int *__restrict__ node_off, int nnodes,
                                                            const uint32_t *__restrict__ tw,
                                                            const uint8_t *__restrict__ dneg, int tws,
                                                            uint32_t *__restrict__ scratch) {
  const int q = n >> 2;
  const long long total = (long long)nnodes * q * B;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int b = (int)(t % B);
  const long long r = t / B;
  const int k = (int)(r % q);
  const int off = node_off[r / q];
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  uint32_t *u0 = y + (size_t)(off + k) * B + b;
  uint32_t *u1 = u0 + (size_t)q * B;
  uint32_t *zp = u0 + (size_t)2 * q * B;
  uint32_t *zm = u0 + (size_t)3 * q * B;
  if (k == 0) {
    big_combine(u0, u1, zp, zm, plane, cim, L, false);
    return;
  }
  const size_t ss = (size_t)total;                   // scratch limb-plane stride
  uint32_t *AX = scratch + t;                        // |operand|
  uint32_t *P = scratch + (size_t)L * ss + t;        // first product of the side
  const size_t tplane = (size_t)(N >> 2) * tws;
  const int kn = k * (N / n) * tws;
  const uint32_t *wr = tw + kn, *ws = tw + (size_t)L * tplane + kn, *wd = tw + (size_t)2 * L * tplane + kn;
  const bool special = 2 * k == q;
  const bool dn = special ? false : (dneg[kn] != 0);
  for (int st_ = 0; st_ < 6; ++st_) {  // same step table as mp_level_kernel
    const int side = st_ >= 3;
    const int step = st_ - 3 * side;
    uint32_t *zr = side ? zm : zp;
    uint32_t *zi = zr + cim;
    const uint32_t *pa = zr, *pb = nullptr, *w = wr;
    bool sub = false, negx = false, mul = true;
    int sp = 0;
    uint32_t *dst = nullptr;
    if (step == 0) {
      pb = zi;
      sub = side;
    } else if (!special) {
      if (step == 1) {
        pa = zi;
        w = wd;
        negx = dn ^ (side == 0);
        sp = 1;
        dst = zi;
      } else {
        w = ws;
        negx = side == 0;
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
      const uint32_t xneg = big_addsub(AX, ss, pa, pb, plane, L, sub);
      big_cond_neg(AX, ss, L, xneg);
      if (!dst) big_mul_merge(AX, ss, w, tplane, L, xneg, false, nullptr, ss, 0, P, ss);
      else big_mul_merge(AX, ss, w, tplane, L, xneg, negx, P, ss, sp, dst, plane);
    } else {
      for (int i = 0; i < L; ++i) dst[(size_t)i * plane] = P[(size_t)i * ss];
    }
  }
  big_combine(u0, u1, zp, zm, plane, cim, L, true);
}

size_t mp_big_scratch_words(const MpDeviceTables &T, int L, int B) {
  long long most = 0;
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const long long th = (long long)T.level_count[lv] * (T.level_n[lv] / 4) * B;
    if (th > most) most = th;
  }
  const size_t words = (size_t)2 * L * (size_t)most;
  if (!mp_tc_used(T, L)) return words;
  const size_t tcw = mp_tc_scratch_words(T, L, B);
  return tcw > words ? tcw : words;
}

cudaError_t mp_big_run_transform(int L, const MpDeviceTables &T, const uint32_t *in, uint32_t *out, int B,
                                 uint32_t *scratch, cudaStream_t s, float *launch_ms) {
  LaunchTimer timer(launch_ms, s);
  {
    const long long total = (long long)T.nleaves * B;
    timer.begin();
    mp_big_leaf_kernel<<<(int)((total + 255) / 256), 256, 0, s>>>(in, out, T.N, B, L, T.leaves, T.nleaves);
    timer.end();
  }
  if (mp_tc_used(T, L)) return mp_tc_run_levels(L, T, out, B, scratch, s, timer);
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const int n = T.level_n[lv];
    const long long total = (long long)T.level_count[lv] * (n / 4) * B;
    timer.begin();
    mp_big_level_kernel<<<(int)((total + 127) / 128), 128, 0, s>>>(out, T.N, B, L, n, T.node_off + T.level_start[lv],
                                                                   T.level_count[lv], T.tw, T.dneg, T.tws, scratch);
    timer.end();
  }
  return cudaGetLastError();
}

}  // namespace mpfft
