// Persistent work-queue kernels for uneven batches: signals of different
// lengths and precisions in one graph launch.
//
// The reference transforms one signal per call and parallelises inside one
// butterfly loop with an OpenMP team per recursion node
// (lab/parallel/mp/parallel_mp_fft2.c:259-326).  Here a batch of signals is
// split into queues by form (fixed-point limbs of each limb count, FP64, and
// the compensated tiers); each queue is one persistent kernel whose CTAs pop
// whole signals from a device counter (atomicAdd) and transform them end to
// end, the largest first.  A CTA runs the same device functions as the
// per-launch kernels -- leaves and L-butterflies of mp_bfly.cuh, the FP64
// sub-transforms of d_core.cuh, the tier sub-transforms of float_tiers.cuh --
// level after level with a CTA barrier between levels, so every output is
// bit-identical to a single call of the same signal.  No CTA waits for
// another: the only shared state is the queue counter.
//
// Compiled with --fmad=false (FP64 bit-identity to the reference); the
// compensated tiers call fma() explicitly and the limb forms are integer
// arithmetic, so neither depends on contraction.
#include <algorithm>
#include <cstdint>

#include "d_core.cuh"
#include "float_tiers.cuh"
#include "mp_bfly.cuh"
#include "mpfft_internal.h"

namespace mpfft {

// the next item of this CTA's queue (all threads see the same value)
__device__ __forceinline__ int queue_next(int *head, int *slot) {
  __syncthreads();  // the previous item is finished before the slot changes
  if (threadIdx.x == 0) *slot = atomicAdd(head, 1);
  __syncthreads();
  return *slot;
}

// ---------------------------------------------------------------------------
// limb forms: one signal = the leaf stage and every level, in global memory
// ---------------------------------------------------------------------------
template <int L>
__global__ void __launch_bounds__(256) mp_queue_kernel(const QueueItem *__restrict__ items, int nitems, int *head) {
  extern __shared__ uint32_t Ps[];  // L x blockDim.x words: each thread's first product of a side
  __shared__ int slot;
  for (int i; (i = queue_next(head, &slot)) < nitems;) {
    const QueueItem it = items[i];
    const QueueTables &Q = *it.tab;
    const TreeTables &T = Q.tree;
    const uint32_t *in = static_cast<const uint32_t *>(it.in);
    uint32_t *out = static_cast<uint32_t *>(it.out);
    const int N = Q.N;
    for (int e = threadIdx.x; e < T.nleaves; e += blockDim.x) mp_leaf_one<L>(in, out, N, 1, 0, T.leaves[e]);
    for (int lv = 0; lv < T.nlevels; ++lv) {
      __syncthreads();  // the previous stage's outputs are visible to the whole CTA
      const int n = T.level_n[lv], q = n >> 2;
      const int total = T.level_count[lv] * q;
      const int *nodes = T.node_off + T.level_start[lv];
      for (int t = threadIdx.x; t < total; t += blockDim.x)
        mp_bfly_one<L, false>(out, N, 1, 0, n, nodes[t / q], t % q, Q.tw, Q.dneg, 1, Ps + threadIdx.x, blockDim.x,
                              nullptr);
    }
  }
}

// ---------------------------------------------------------------------------
// FP64: the sub-transform roots one after another in shared memory, then the
// levels above them in global memory
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) d_queue_kernel(const QueueItem *__restrict__ items, int nitems, int *head,
                                                      double scale) {
  extern __shared__ double dq_smem[];
  __shared__ int slot;
  for (int i; (i = queue_next(head, &slot)) < nitems;) {
    const QueueItem it = items[i];
    const DDeviceTables &T = it.tab->ft;
    const double *in = static_cast<const double *>(it.in);
    double *out = static_cast<double *>(it.out);
    const DConst K{T.c8, T.c16a, T.c16b, T.c16c, T.c16d};
    const bool final_sub = T.upper.nlevels == 0;
    for (int r = 0; r < T.nroots; ++r) {
      __syncthreads();  // shared memory of the previous root is free
      d_sub_instances<false>(in, out, T.N, 1, 0, 1, T.roots[r], T.sub[0], T.sub[1], T.wr, T.wi, K,
                             final_sub ? scale : 1.0, 0, 0, dq_smem);
    }
    for (int lv = 0; lv < T.upper.nlevels; ++lv) {
      __syncthreads();
      const int n = T.upper.level_n[lv], q = n >> 2;
      const int total = T.upper.level_count[lv] * q;
      const int *nodes = T.upper.node_off + T.upper.level_start[lv];
      const double sc = lv == T.upper.nlevels - 1 ? scale : 1.0;
      for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int k = t % q, kn = k * (T.N / n);
        d_butterfly(out, out + T.N, 1, nodes[t / q], k, q, T.wr[kn], T.wi[kn], sc, false);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// compensated tiers: the same pattern
// ---------------------------------------------------------------------------
template <class NT>
__global__ void __launch_bounds__(256) tier_queue_kernel(const QueueItem *__restrict__ items, int nitems, int *head,
                                                         double scale) {
  extern __shared__ __align__(16) unsigned char tq_smem[];
  typename NT::W *sm = reinterpret_cast<typename NT::W *>(tq_smem);
  __shared__ int slot;
  for (int i; (i = queue_next(head, &slot)) < nitems;) {
    const QueueItem it = items[i];
    const DDeviceTables &T = it.tab->ft;
    const auto *in = static_cast<const typename NT::W *>(it.in);
    auto *out = static_cast<typename NT::W *>(it.out);
    TierTw tw{};
    for (int h = 0; h < 4; ++h) {
      tw.c[h] = T.tw_cos[h];
      tw.s[h] = T.tw_sin[h];
    }
    const bool final_sub = T.upper.nlevels == 0;
    for (int r = 0; r < T.nroots; ++r) {
      __syncthreads();
      tier_sub_instances<NT, false>(in, out, T.N, 1, 0, 1, T.roots[r], T.sub[0], T.sub[1], tw,
                                    final_sub ? scale : 1.0, 0, 0, sm);
    }
    for (int lv = 0; lv < T.upper.nlevels; ++lv) {
      __syncthreads();
      const int n = T.upper.level_n[lv], q = n >> 2;
      const int total = T.upper.level_count[lv] * q;
      const int *nodes = T.upper.node_off + T.upper.level_start[lv];
      const double sc = lv == T.upper.nlevels - 1 ? scale : 1.0;
      for (int t = threadIdx.x; t < total; t += blockDim.x)
        tier_level_one<NT>(out, T.N, 1, n, nodes[t / q], t % q, 0, tw, sc, 0);
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
constexpr size_t kQueueSmemBytes = 64 * 1024;  // FP64 (4096 points) and every tier (64 KB planes)

template <int L>
static const void *mp_queue_fn() {
  return (const void *)mp_queue_kernel<L>;
}

static const void *queue_fn(int family, int L) {
  switch (family) {
    case kQueueDouble:
      return (const void *)d_queue_kernel;
    case kQueueTierDD:
      return (const void *)tier_queue_kernel<DDT>;
    case kQueueTierQD:
      return (const void *)tier_queue_kernel<QDT>;
    case kQueueTierFF:
      return (const void *)tier_queue_kernel<FFT_>;
    default:
      break;
  }
#define MPFFT_Q_CASE(LL) \
  case LL:               \
    return mp_queue_fn<LL>();
  switch (L) {
    MPFFT_Q_CASE(2) MPFFT_Q_CASE(3) MPFFT_Q_CASE(4) MPFFT_Q_CASE(5) MPFFT_Q_CASE(6) MPFFT_Q_CASE(7)
    MPFFT_Q_CASE(8) MPFFT_Q_CASE(9) MPFFT_Q_CASE(10) MPFFT_Q_CASE(11) MPFFT_Q_CASE(12) MPFFT_Q_CASE(13)
    MPFFT_Q_CASE(14) MPFFT_Q_CASE(15) MPFFT_Q_CASE(16) MPFFT_Q_CASE(17) MPFFT_Q_CASE(18) MPFFT_Q_CASE(19)
    MPFFT_Q_CASE(20) MPFFT_Q_CASE(21) MPFFT_Q_CASE(22) MPFFT_Q_CASE(23) MPFFT_Q_CASE(24) MPFFT_Q_CASE(25)
    MPFFT_Q_CASE(26) MPFFT_Q_CASE(27) MPFFT_Q_CASE(28) MPFFT_Q_CASE(29) MPFFT_Q_CASE(30) MPFFT_Q_CASE(31)
    MPFFT_Q_CASE(32) MPFFT_Q_CASE(33) MPFFT_Q_CASE(34)
    default:
      return nullptr;
  }
#undef MPFFT_Q_CASE
}

static size_t queue_smem(int family, int L, int threads) {
  return family == kQueueLimbs ? (size_t)L * threads * sizeof(uint32_t) : kQueueSmemBytes;
}

cudaError_t queue_prepare(int family, int L) {
  const void *fn = queue_fn(family, L);
  if (!fn) return cudaErrorInvalidValue;
  if (family == kQueueLimbs) return cudaSuccess;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQueueSmemBytes);
}

int queue_ctas_per_sm(int family, int L, int threads) {
  const void *fn = queue_fn(family, L);
  int n = 0;
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, queue_smem(family, L, threads)) !=
                 cudaSuccess)
    return 1;
  return std::max(1, n);
}

cudaError_t queue_launch(int family, int L, const QueueItem *items, int nitems, int *head, int ctas, int threads,
                         double scale, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  const void *fn = queue_fn(family, L);
  if (!fn) return cudaErrorInvalidValue;
  void *args_mp[] = {(void *)&items, (void *)&nitems, (void *)&head};
  void *args_fp[] = {(void *)&items, (void *)&nitems, (void *)&head, (void *)&scale};
  return cudaLaunchKernel(fn, dim3(ctas), dim3(threads), family == kQueueLimbs ? args_mp : args_fp,
                          queue_smem(family, L, threads), s);
}

}  // namespace mpfft
