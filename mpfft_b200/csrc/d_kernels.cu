// FP64 conjugate-pair split-radix 2/4 DIT FFT kernels (sm_100a).
//
// Bit-identical to the reference's double transform d_sr24_cp_fft
// (lab/serial/double/serial_d_fft6.c:93-429): the same n=8 and n=16 base
// cases, the same 4m2a butterfly for every k (twiddle (1,0) at k=0
// included), every IEEE operation with the same operands in the same
// association.  This file is compiled with --fmad=false so no multiply-add is
// contracted into an FMA (the reference's x86-64 build has no FMA either).
//
// Schedule: breadth-first over the reference's recursion tree -- one launch
// for all leaves (n = 16 and 8 for N >= 16; the whole transform for N <= 16),
// then one launch per node size n = 32 .. N.  Layout: word (c, p, b) at
// base[(c*N + p)*B + b]; consecutive threads are consecutive signals (or k).
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

__global__ void __launch_bounds__(128) d_leaf_kernel(const double *__restrict__ in, double *__restrict__ out, int N,
                                                      int B, const Leaf *__restrict__ leaves, int nleaves, DConst K,
                                                      double scale) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nleaves * B) return;
  const int b = (int)(t % B);
  const Leaf lf = leaves[t / B];
  const size_t cim = (size_t)N * B;
  double xr[16], xi[16], yr[16], yi[16];
  const int n = lf.n;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j < n) {
      const int idx = (j == 0 && lf.sn < 0) ? lf.sn + N : lf.sn + j * lf.s;
      xr[j] = in[(size_t)idx * B + b];
      xi[j] = in[(size_t)idx * B + b + cim];
    } else {
      xr[j] = 0.0;
      xi[j] = 0.0;
    }
  }
  if (n == 16) {
    D16 R, I;
    d16_part(K, xr, false, R);
    d16_part(K, xi, true, I);
    // output stage (reference :350-382)
    yr[0] = R.b5 + R.b11;  yr[8] = R.b5 - R.b11;
    yi[0] = I.b5 + I.b11;  yi[8] = I.b5 - I.b11;
    yr[4] = R.b6 - I.b12;  yr[12] = R.b6 + I.b12;
    yi[4] = I.b6 - R.b12;  yi[12] = I.b6 + R.b12;
    yr[1] = R.c9 - I.c17;  yr[15] = R.c9 + I.c17;
    yi[1] = I.c9 - R.c17;  yi[15] = I.c9 + R.c17;
    yr[2] = R.c1 - I.c3;   yr[14] = R.c1 + I.c3;
    yi[2] = I.c1 - R.c3;   yi[14] = I.c1 + R.c3;
    yr[3] = R.c12 + I.c20; yr[13] = R.c12 - I.c20;
    yi[3] = I.c12 + R.c20; yi[13] = I.c12 - R.c20;
    yr[5] = R.c11 - I.c19; yr[11] = R.c11 + I.c19;
    yi[5] = I.c11 - R.c19; yi[11] = I.c11 + R.c19;
    yr[6] = R.c2 - I.c4;   yr[10] = R.c2 + I.c4;
    yi[6] = I.c2 - R.c4;   yi[10] = I.c2 + R.c4;
    yr[7] = R.c10 + I.c18; yr[9] = R.c10 - I.c18;
    yi[7] = I.c10 + R.c18; yi[9] = I.c10 - R.c18;
  } else if (n == 8) {
    double R[8], I[8];
    d8_part(K, xr, R);
    d8_part(K, xi, I);
    // output stage (reference :193-209)
    yr[0] = R[1] + R[0]; yr[4] = R[1] - R[0];
    yi[0] = I[1] + I[0]; yi[4] = I[1] - I[0];
    yr[1] = R[4] + I[6]; yr[7] = R[4] - I[6];
    yi[1] = I[4] - R[6]; yi[7] = I[4] + R[6];
    yr[2] = R[2] + I[3]; yr[6] = R[2] - I[3];
    yi[2] = I[2] - R[3]; yi[6] = I[2] + R[3];
    yr[3] = R[5] - I[7]; yr[5] = R[5] + I[7];
    yi[3] = I[5] + R[7]; yi[5] = I[5] - R[7];
  } else if (n == 4) {
    // reference :121-147
    const double er = xr[0] + xr[2], fr = xr[0] - xr[2], gr = xr[1] + xr[3], hr = xr[1] - xr[3];
    const double ei = xi[0] + xi[2], fi = xi[0] - xi[2], gi = xi[1] + xi[3], hi = xi[1] - xi[3];
    yr[0] = er + gr; yr[1] = fr + hi; yr[2] = er - gr; yr[3] = fr - hi;
    yi[0] = ei + gi; yi[1] = fi - hr; yi[2] = ei - gi; yi[3] = fi + hr;
  } else if (n == 2) {
    yr[0] = xr[0] + xr[1]; yr[1] = xr[0] - xr[1];
    yi[0] = xi[0] + xi[1]; yi[1] = xi[0] - xi[1];
  } else {
    yr[0] = xr[0];
    yi[0] = xi[0];
  }
  double *y = out + (size_t)lf.out * B + b;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j < n) {
      y[(size_t)j * B] = yr[j] * scale;
      y[(size_t)j * B + cim] = yi[j] * scale;
    }
  }
}

// 4m2a butterflies of all nodes of size n (reference :392-427)
__global__ void __launch_bounds__(256) d_level_kernel(double *__restrict__ y, int N, int B, int n,
                                                       const int *__restrict__ node_off, int nnodes,
                                                       const double *__restrict__ wr, const double *__restrict__ wi,
                                                       double scale) {
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnodes * q * B) return;
  const int b = (int)(t % B);
  const long long r = t / B;
  const int k = (int)(r % q);
  const int off = node_off[r / q];
  const size_t cim = (size_t)N * B;
  double *p0 = y + (size_t)(off + k) * B + b;
  double *p1 = p0 + (size_t)q * B, *p2 = p0 + (size_t)2 * q * B, *p3 = p0 + (size_t)3 * q * B;
  const int kn = k * (N / n);
  const double w_r = wr[kn], w_i = wi[kn];
  const double u0r = p0[0], u1r = p1[0], zpr = p2[0], zmr = p3[0];
  const double u0i = p0[cim], u1i = p1[cim], zpi = p2[cim], zmi = p3[cim];
  const double pr = w_r * zpr + w_i * zpi, pi = w_r * zpi - w_i * zpr;
  const double mr = w_r * zmr - w_i * zmi, mi = w_r * zmi + w_i * zmr;
  const double sr = pr + mr, si = pi + mi, dr = pr - mr, di = pi - mi;
  p0[0] = (u0r + sr) * scale;
  p2[0] = (u0r - sr) * scale;
  p1[0] = (u1r + di) * scale;
  p3[0] = (u1r - di) * scale;
  p0[cim] = (u0i + si) * scale;
  p2[cim] = (u0i - si) * scale;
  p1[cim] = (u1i - dr) * scale;
  p3[cim] = (u1i + dr) * scale;
}

cudaError_t d_run_transform(const DDeviceTables &T, const double *in, double *out, int B, double scale,
                            cudaStream_t s) {
  const DConst K{T.c8, T.c16a, T.c16b, T.c16c, T.c16d};
  {
    const int threads = 128;
    const long long total = (long long)T.nleaves * B;
    const int blocks = (int)((total + threads - 1) / threads);
    d_leaf_kernel<<<blocks, threads, 0, s>>>(in, out, T.N, B, T.leaves, T.nleaves, K,
                                             T.nlevels == 0 ? scale : 1.0);
  }
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const int threads = 256;
    const int n = T.level_n[lv];
    const long long total = (long long)T.level_count[lv] * (n / 4) * B;
    const int blocks = (int)((total + threads - 1) / threads);
    d_level_kernel<<<blocks, threads, 0, s>>>(out, T.N, B, n, T.node_off + T.level_start[lv], T.level_count[lv],
                                              T.wr, T.wi, lv == T.nlevels - 1 ? scale : 1.0);
  }
  return cudaGetLastError();
}

}  // namespace mpfft
