// FP64 conjugate-pair split-radix 2/4 DIT FFT kernels (sm_100a).
//
// Bit-identical to the reference's double transform d_sr24_cp_fft
// (lab/serial/double/serial_d_fft6.c:93-429): the same n=8 and n=16 base
// cases, the same 4m2a butterfly for every k (twiddle (1,0) at k=0
// included), every IEEE operation with the same operands in the same
// association.  This file is compiled with --fmad=false so no multiply-add is
// contracted into an FMA (the reference's x86-64 build has no FMA either).
//
// Schedule: the reference's recursion tree, cut at T = min(N, 4096) points.
// Every maximal node of size <= T (size T or T/2) is one shared-memory
// sub-transform: one CTA gathers its input sequence in DIT order (so every
// leaf's inputs already sit where its outputs go), runs the leaves (n = 16 and
// 8; the whole transform for N <= 16) and all levels up to the node in place
// in shared memory, and writes the node's outputs once.  Levels above T run
// one launch per node size in global memory.  For N <= 4096 a transform is one
// launch that reads its input once and writes its output once.
//
// Layout: word (c, b, p) at base[(c*B + b)*N + p] -- each signal contiguous.
#include <algorithm>
#include <cstdint>

#include "d_core.cuh"
#include "mpfft_internal.h"

namespace mpfft {

template <bool SINGLE>
__global__ void __launch_bounds__(256, 3) d_sub_kernel(const double *__restrict__ in, double *__restrict__ out, int N,
                                                        int B, const SubRoot *__restrict__ roots, int nroots, int G,
                                                        SubSchedule big, SubSchedule small,
                                                        const double *__restrict__ wr, const double *__restrict__ wi,
                                                        DConst K, double scale, int swap_in, int swap_out) {
  extern __shared__ double sm[];
  if (SINGLE) {
    const int b0 = blockIdx.x * G;
    d_sub_instances<true>(in, out, N, B, b0, min(G, B - b0), roots[0], big, small, wr, wi, K, scale, swap_in, swap_out,
                          sm);
  } else {
    d_sub_instances<false>(in, out, N, B, blockIdx.x / nroots, 1, roots[blockIdx.x % nroots], big, small, wr, wi, K,
                           scale, swap_in, swap_out, sm);
  }
}

// 4m2a butterflies of all nodes of size n above the shared-memory
// sub-transforms; consecutive threads are consecutive k of one signal.
__global__ void __launch_bounds__(256) d_level_kernel(double *__restrict__ y, int N, int B, int n,
                                                       const int *__restrict__ node_off, int nnodes,
                                                       const double *__restrict__ wr, const double *__restrict__ wi,
                                                       double scale, int swap_out) {
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnodes * q * B) return;
  const int k = (int)(t % q);
  const long long r = t / q;
  const int node = (int)(r % nnodes);
  const int b = (int)(r / nnodes);
  const int kn = k * (N / n);
  d_butterfly(y + (size_t)b * N, y + ((size_t)B + b) * N, 1, node_off[node], k, q, wr[kn], wi[kn], scale,
              swap_out != 0);
}

// Split step of the FP64 real transforms (n = 2M real points; layouts [c][b][k]).
// Forward: Z = FFT_M(x_2m + i x_2m+1) (M points) -> X_0..X_M (M+1 points):
//   S = Z_k + conj Z_(M-k), D = Z_k - conj Z_(M-k), T = w^k D (w = exp(-2 pi i/n)),
//   X_k = (S_r + T_i, S_i - T_r) / 2,  X_(M-k) = (S_r - T_i, -(S_i + T_r)) / 2.
// Inverse: X (M+1 points) -> W = the planes-exchanged 2Z, with
//   S' = X_k + conj X_(M-k), D' = X_k - conj X_(M-k), T' = w^-k D',
//   2Z_k = (S'_r - T'_i, S'_i + T'_r), 2Z_(M-k) = (S'_r + T'_i, T'_r - S'_i),
// so that the forward transform of W is n * (x_2m+1 + i x_2m) (the swap
// identity); the imaginary parts of X_0 and X_M are ignored.  wc, ws: cos and
// sin of 2 pi k/n for k < M/2; scale multiplies the forward outputs.
__global__ void __launch_bounds__(256) d_r2c_post(const double *__restrict__ z, double *__restrict__ x, int M, int B,
                                                   const double *__restrict__ wc, const double *__restrict__ ws,
                                                   double scale) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)(M / 2 + 1) * B) return;
  const int k = (int)(t % (M / 2 + 1));
  const int b = (int)(t / (M / 2 + 1));
  const double *zr = z + (size_t)b * M, *zi = z + ((size_t)B + b) * M;
  double *xr = x + (size_t)b * (M + 1), *xi = x + ((size_t)B + b) * (M + 1);
  const double h = 0.5 * scale;
  if (k == 0) {
    xr[0] = (zr[0] + zi[0]) * scale;
    xi[0] = 0.0;
    xr[M] = (zr[0] - zi[0]) * scale;
    xi[M] = 0.0;
    return;
  }
  const double ar = zr[k], ai = zi[k], br = zr[M - k], bi = zi[M - k];
  const double sr = ar + br, si = ai - bi, dr = ar - br, di = ai + bi;
  const double c = 2 * k == M ? 0.0 : wc[k], s = 2 * k == M ? 1.0 : ws[k];
  const double tr = c * dr + s * di, ti = c * di - s * dr;
  xr[k] = (sr + ti) * h;
  xi[k] = (si - tr) * h;
  if (2 * k != M) {
    xr[M - k] = (sr - ti) * h;
    xi[M - k] = -(si + tr) * h;
  }
}

__global__ void __launch_bounds__(256) d_c2r_pre(const double *__restrict__ x, double *__restrict__ w, int M, int B,
                                                  const double *__restrict__ wc, const double *__restrict__ ws) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)(M / 2 + 1) * B) return;
  const int k = (int)(t % (M / 2 + 1));
  const int b = (int)(t / (M / 2 + 1));
  const double *xr = x + (size_t)b * (M + 1), *xi = x + ((size_t)B + b) * (M + 1);
  // W = (2Z_i, 2Z_r): real plane holds the imaginary parts
  double *wr = w + (size_t)b * M, *wi = w + ((size_t)B + b) * M;
  if (k == 0) {
    wi[0] = xr[0] + xr[M];
    wr[0] = xr[0] - xr[M];
    return;
  }
  const double ar = xr[k], ai = xi[k], br = xr[M - k], bi = xi[M - k];
  const double sr = ar + br, si = ai - bi, dr = ar - br, di = ai + bi;
  const double c = 2 * k == M ? 0.0 : wc[k], s = 2 * k == M ? 1.0 : ws[k];
  const double tr = c * dr - s * di, ti = c * di + s * dr;
  wi[k] = sr - ti;
  wr[k] = si + tr;
  if (2 * k != M) {
    wi[M - k] = sr + ti;
    wr[M - k] = tr - si;
  }
}

cudaError_t d_real_split(bool forward, const double *in, double *out, int M, int B, const double *wc,
                         const double *ws, double scale, cudaStream_t s) {
  const long long total = (long long)(M / 2 + 1) * B;
  const int blocks = (int)((total + 255) / 256);
  if (forward) d_r2c_post<<<blocks, 256, 0, s>>>(in, out, M, B, wc, ws, scale);
  else d_c2r_pre<<<blocks, 256, 0, s>>>(in, out, M, B, wc, ws);
  return cudaGetLastError();
}

// instances of the shared-memory kernel per CTA and its dynamic shared memory
static int d_sub_instances(const DDeviceTables &T) {
  if (T.nroots != 1) return 1;
  const int per = 2 * T.sub[0].size;
  return std::max(1, std::min(kDSubMax / std::max(T.sub[0].size, 1), 8192 / per));
}

cudaError_t d_run_transform(const DDeviceTables &T, const double *in, double *out, int B, double scale,
                            cudaStream_t s, bool swap_in, bool swap_out) {
  const DConst K{T.c8, T.c16a, T.c16b, T.c16c, T.c16d};
  const int size = T.sub[0].size;
  const int G = d_sub_instances(T);
  const size_t smem = ((size_t)G * 2 * size) * sizeof(double);
  static bool attr_set = false;  // idempotent; benign race
  if (!attr_set) {
    cudaFuncSetAttribute(d_sub_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    cudaFuncSetAttribute(d_sub_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr_set = true;
  }
  const bool final_sub = T.upper.nlevels == 0;
  if (T.nroots == 1) {
    const int blocks = (B + G - 1) / G;
    d_sub_kernel<true><<<blocks, 256, smem, s>>>(in, out, T.N, B, T.roots, T.nroots, G, T.sub[0], T.sub[1], T.wr,
                                                 T.wi, K, final_sub ? scale : 1.0, swap_in, final_sub && swap_out);
  } else {
    d_sub_kernel<false><<<T.nroots * B, 256, smem, s>>>(in, out, T.N, B, T.roots, T.nroots, 1, T.sub[0], T.sub[1],
                                                        T.wr, T.wi, K, final_sub ? scale : 1.0, swap_in,
                                                        final_sub && swap_out);
  }
  for (int lv = 0; lv < T.upper.nlevels; ++lv) {
    const int threads = 256;
    const int n = T.upper.level_n[lv];
    const long long total = (long long)T.upper.level_count[lv] * (n / 4) * B;
    const int lblocks = (int)((total + threads - 1) / threads);
    d_level_kernel<<<lblocks, threads, 0, s>>>(out, T.N, B, n, T.upper.node_off + T.upper.level_start[lv],
                                               T.upper.level_count[lv], T.wr, T.wi,
                                               lv == T.upper.nlevels - 1 ? scale : 1.0,
                                               lv == T.upper.nlevels - 1 && swap_out);
  }
  return cudaGetLastError();
}

}  // namespace mpfft
