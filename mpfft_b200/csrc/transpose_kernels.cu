// Batched matrix transposition for multi-dimensional transforms:
//     out[m][c][r][e] = in[m][r][c][e]
// for nmat matrices of R x C elements of E 32-bit words each.  In the
// multiprecision layout an element is the batch column of one point of one
// limb plane (E = batch, m = limb plane); in the FP64 layout an element is one
// double (E = 2, m = component x signal).  Rotating the last axis of a
// row-major multi-dimensional signal to the front is one such transposition
// with C = that axis' length and R = the product of the others.
//
// HBM-bound copies: elements of 16 words or more are copied by one warp each
// (both sides coalesced along e); smaller elements go through a shared-memory
// tile of T x T elements, T = floor(32 / E), so that tile rows are up to 32
// contiguous words on both sides.
#include <algorithm>
#include <cstdint>

#include "mpfft_internal.h"

namespace mpfft {

__global__ void __launch_bounds__(256) transpose_rows_kernel(const uint32_t *__restrict__ in,
                                                             uint32_t *__restrict__ out, long long nmat,
                                                             long long R, long long C, int E) {
  const long long nelem = nmat * R * C;
  const int lane = threadIdx.x & 31;
  for (long long o = (long long)blockIdx.x * 8 + (threadIdx.x >> 5); o < nelem; o += (long long)gridDim.x * 8) {
    // output element o = (m, c, r) row-major
    const long long r = o % R;
    const long long t = o / R;
    const long long c = t % C;
    const long long m = t / C;
    const uint32_t *src = in + ((m * R + r) * C + c) * E;
    uint32_t *dst = out + o * E;
    for (int e = lane; e < E; e += 32) dst[e] = src[e];
  }
}

__global__ void __launch_bounds__(256) transpose_tile_kernel(const uint32_t *__restrict__ in,
                                                             uint32_t *__restrict__ out, long long nmat,
                                                             long long R, long long C, int E, int T) {
  __shared__ uint32_t tile[32 * 33];
  const int W = T * E;  // words per tile row (<= 32)
  const long long tR = (R + T - 1) / T, tC = (C + T - 1) / T;
  const long long ntiles = nmat * tR * tC;
  for (long long tix = blockIdx.x; tix < ntiles; tix += gridDim.x) {
    const long long tc = tix % tC;
    const long long t2 = tix / tC;
    const long long tr = t2 % tR;
    const long long m = t2 / tR;
    const long long r0 = tr * T, c0 = tc * T;
    const int nr = (int)min((long long)T, R - r0), nc = (int)min((long long)T, C - c0);
    // load: tile row r = in row r0 + r, words of columns c0 .. c0 + nc - 1
    for (int q = threadIdx.x; q < T * W; q += blockDim.x) {
      const int r = q / W, w = q - r * W;
      if (r < nr && w < nc * E) tile[r * 33 + w] = in[((m * R + r0 + r) * C + c0) * E + w];
    }
    __syncthreads();
    // store: out row c = column c0 + c, words of rows r0 .. r0 + nr - 1
    for (int q = threadIdx.x; q < T * W; q += blockDim.x) {
      const int c = q / W, w = q - c * W;
      const int r = w / E, e = w - r * E;
      if (c < nc && r < nr) out[((m * C + c0 + c) * R + r0) * E + w] = tile[r * 33 + c * E + e];
    }
    __syncthreads();
  }
}

cudaError_t transpose_launch(const uint32_t *in, uint32_t *out, long long nmat, long long R, long long C, int E,
                             cudaStream_t s) {
  const long long nelem = nmat * R * C;
  if (nelem == 0) return cudaSuccess;
  if (E >= 16) {
    const long long blocks = std::min<long long>((nelem + 7) / 8, 148LL * 64);
    transpose_rows_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, out, nmat, R, C, E);
  } else {
    const int T = 32 / E;
    const long long ntiles = nmat * ((R + T - 1) / T) * ((C + T - 1) / T);
    const long long blocks = std::min<long long>(ntiles, 148LL * 32);
    transpose_tile_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, out, nmat, R, C, E, T);
  }
  return cudaGetLastError();
}

}  // namespace mpfft
