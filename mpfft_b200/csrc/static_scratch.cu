// A multiprecision entry point that allocates nothing.
//
// mpfft_mp_execute_significands_static transforms signals whose MPFR fields
// (significand limbs, exponents, signs) already live in device memory.  Its
// working storage -- the input and output limb planes and the per-signal
// block exponents -- comes from one file-scope device array instead of
// cudaMalloc, for callers that cannot allocate device memory at call time:
// services that reserve their whole device-memory budget at start-up, and
// code paths that must not pay cudaMalloc/cudaFree's implicit device-wide
// synchronisation.  Every GPU that loads this library holds the array
// (kStaticScratchBytes) until the process exits.
//
// In host code the name g_static_scratch is only a host-side stand-in for the
// device array, not a device address; the address is fetched once per device
// with cudaGetSymbolAddress (with that device current) and then passed to the
// kernels.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "mpfft_internal.h"

namespace mpfft {

constexpr size_t kStaticScratchBytes = 64ull << 20;  // 64 MiB per GPU

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

static std::mutex g_scratch_mu;
static void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device (set-up on the
// first call per device).
static cudaError_t static_scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

size_t static_scratch_bytes() { return kStaticScratchBytes; }

int mp_execute_significands_static(const MpPlanView &v, unsigned long batch, const uint64_t *d_mant_in,
                                   const int64_t *d_exp_in, const uint8_t *d_sign_in, int nl_in,
                                   uint64_t *d_mant_out, int64_t *d_exp_out, uint8_t *d_sign_out, long prec_out,
                                   unsigned scaled_shift, cudaStream_t stream, char *msg, size_t msglen) {
  // scratch layout: input planes | output planes | block exponents.  The
  // bound is a division, so that no product of the caller's sizes can wrap:
  // each signal takes 2 x (2 L n words) of planes plus an 8-byte exponent,
  // and the two planes' 256-byte roundings take at most 510 bytes more.
  const size_t per_signal = (size_t)2 * ((size_t)2 * v.L * v.N * 4) + 8;
  const size_t max_batch = (kStaticScratchBytes - 512) / per_signal;
  if (batch > max_batch) {
    snprintf(msg, msglen,
             "batch %lu of n=%lu exceeds the static scratch of %zu bytes (at most %zu signals at this size)",
             batch, v.N, kStaticScratchBytes, max_batch);
    return 2;  // MPFFT_EUNSUPPORTED
  }
  const size_t plane_words = (size_t)2 * v.L * v.N * batch;
  const size_t plane_bytes = (plane_words * 4 + 255) & ~(size_t)255;
  void *base = nullptr;
  cudaError_t e = static_scratch_address(&base);
  if (e == cudaSuccess) {
    uint32_t *in_planes = static_cast<uint32_t *>(base);
    uint32_t *out_planes = reinterpret_cast<uint32_t *>(static_cast<unsigned char *>(base) + plane_bytes);
    int64_t *es = reinterpret_cast<int64_t *>(static_cast<unsigned char *>(base) + 2 * plane_bytes);
    // import clears nothing it does not overwrite: every plane word and every
    // block exponent is written before it is read
    e = mp_import_launch(d_mant_in, d_exp_in, d_sign_in, nl_in, (int)v.N, (int)batch, v.L, v.F, es, in_planes,
                         stream);
    if (e == cudaSuccess) e = mp_run_transform(v.L, *v.tabs, in_planes, out_planes, (int)batch, stream);
    if (e == cudaSuccess)
      e = mp_export_launch(out_planes, (int)v.N, (int)batch, v.L, es, v.F + (long)scaled_shift, prec_out,
                           (int)((prec_out + 63) / 64), d_mant_out, d_exp_out, d_sign_out, stream);
  }
  if (e != cudaSuccess) {
    snprintf(msg, msglen, "CUDA error: %s", cudaGetErrorString(e));
    return 4;  // MPFFT_ECUDA
  }
  return 0;
}

}  // namespace mpfft
