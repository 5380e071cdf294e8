// Launchers of the compensated floating-point tiers (double-double,
// quad-double, float-float): the per-launch kernels over float_tiers.cuh.
#include <algorithm>
#include <cstdint>

#include "float_tiers.cuh"
#include "mpfft_internal.h"

namespace mpfft {

template <class NT, bool SINGLE>
__global__ void __launch_bounds__(256) tier_sub_kernel(const typename NT::W *__restrict__ in,
                                                       typename NT::W *__restrict__ out, int N, int B,
                                                       const SubRoot *__restrict__ roots, int nroots, int G,
                                                       SubSchedule big, SubSchedule small, TierTw tw, double scale,
                                                       int swap_in, int swap_out) {
  extern __shared__ __align__(16) unsigned char tier_smem[];
  typename NT::W *sm = reinterpret_cast<typename NT::W *>(tier_smem);
  if (SINGLE) {
    const int b0 = blockIdx.x * G;
    tier_sub_instances<NT, true>(in, out, N, B, b0, min(G, B - b0), roots[0], big, small, tw, scale, swap_in, swap_out,
                                 sm);
  } else {
    tier_sub_instances<NT, false>(in, out, N, B, blockIdx.x / nroots, 1, roots[blockIdx.x % nroots], big, small, tw,
                                  scale, swap_in, swap_out, sm);
  }
}

template <class NT>
__global__ void __launch_bounds__(256) tier_level_kernel(typename NT::W *__restrict__ y, int N, int B, int n,
                                                         const int *__restrict__ node_off, int nnodes, TierTw tw,
                                                         double scale, int swap_out) {
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnodes * q * B) return;
  const long long r = t / q;
  tier_level_one<NT>(y, N, B, n, node_off[(int)(r % nnodes)], (int)(t % q), (int)(r / nnodes), tw, scale, swap_out);
}

constexpr size_t kTierSmemBytes = 64 * 1024;  // planes of one CTA

template <class NT>
static cudaError_t tier_run(const DDeviceTables &T, const void *in_, void *out_, int B, double scale, cudaStream_t s,
                            bool swap_in, bool swap_out) {
  using W = typename NT::W;
  const W *in = static_cast<const W *>(in_);
  W *out = static_cast<W *>(out_);
  const int size = T.sub[0].size;
  const size_t inst_bytes = (size_t)2 * NT::K * size * sizeof(W);
  const int G = T.nroots != 1 ? 1 : (int)std::max<size_t>(1, kTierSmemBytes / inst_bytes);
  const size_t smem = (size_t)G * inst_bytes;
  static bool attr_set = false;  // idempotent; benign race
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(tier_sub_kernel<NT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTierSmemBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tier_sub_kernel<NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kTierSmemBytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  TierTw tw{};
  for (int h = 0; h < 4; ++h) {
    tw.c[h] = T.tw_cos[h];
    tw.s[h] = T.tw_sin[h];
  }
  const bool final_sub = T.upper.nlevels == 0;
  if (T.nroots == 1) {
    tier_sub_kernel<NT, true><<<(B + G - 1) / G, 256, smem, s>>>(in, out, T.N, B, T.roots, T.nroots, G, T.sub[0],
                                                                 T.sub[1], tw, final_sub ? scale : 1.0, swap_in,
                                                                 final_sub && swap_out);
  } else {
    tier_sub_kernel<NT, false><<<T.nroots * B, 256, smem, s>>>(in, out, T.N, B, T.roots, T.nroots, 1, T.sub[0],
                                                               T.sub[1], tw, final_sub ? scale : 1.0, swap_in,
                                                               final_sub && swap_out);
  }
  for (int lv = 0; lv < T.upper.nlevels; ++lv) {
    const int n = T.upper.level_n[lv];
    const long long total = (long long)T.upper.level_count[lv] * (n / 4) * B;
    const bool last = lv == T.upper.nlevels - 1;
    tier_level_kernel<NT><<<(int)((total + 255) / 256), 256, 0, s>>>(
        out, T.N, B, n, T.upper.node_off + T.upper.level_start[lv], T.upper.level_count[lv], tw, last ? scale : 1.0,
        last && swap_out);
  }
  return cudaGetLastError();
}

int tier_words(int tier) { return tier == kTierQD ? 4 : 2; }
size_t tier_word_bytes(int tier) { return tier == kTierFF ? 4 : 8; }
int tier_sub_max(int tier) { return tier == kTierQD ? kQDSubMax : tier == kTierFF ? kFFSubMax : kDDSubMax; }

cudaError_t tier_run_transform(int tier, const DDeviceTables &T, const void *in, void *out, int B, double scale,
                               cudaStream_t s, bool swap_in, bool swap_out) {
  switch (tier) {
    case kTierDD:
      return tier_run<DDT>(T, in, out, B, scale, s, swap_in, swap_out);
    case kTierQD:
      return tier_run<QDT>(T, in, out, B, scale, s, swap_in, swap_out);
    case kTierFF:
      return tier_run<FFT_>(T, in, out, B, scale, s, swap_in, swap_out);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t dd_run_transform(const DDeviceTables &T, const double *in, double *out, int B, double scale,
                             cudaStream_t s, bool swap_in, bool swap_out) {
  return tier_run<DDT>(T, in, out, B, scale, s, swap_in, swap_out);
}

}  // namespace mpfft
