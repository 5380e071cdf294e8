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
// limb forms, long signals: a group of signals of one (N, L) runs the
// per-level schedule over all its signals at once -- one launch for the
// leaves, one per node size, a thread per leaf or butterfly (consecutive
// threads consecutive k of one signal) -- instead of one CTA per signal.
// The same device functions: bit-identical to the queue and to single calls.
// The level launches read per-level copies of the twiddles (GroupTw), indexed
// by k: in the N/4-entry tables consecutive k of a level of size n are N/n
// entries apart, so a warp's twiddle loads would touch 32 sectors instead of
// four.
// ---------------------------------------------------------------------------
template <int L>
__global__ void __launch_bounds__(256) mp_group_leaf_kernel(const QueueItem *__restrict__ items, int nsig, int N,
                                                            const MpLeaf *__restrict__ leaves, int nleaves) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nsig * nleaves) return;
  const QueueItem it = items[t / nleaves];
  mp_leaf_one<L>(static_cast<const uint32_t *>(it.in), static_cast<uint32_t *>(it.out), N, 1, 0,
                 leaves[t % nleaves]);
}

template <int L>
__global__ void __launch_bounds__(128, level_min_blocks<L>())
    mp_group_level_kernel(const QueueItem *__restrict__ items, int nsig, int N, int n,
                          const int *__restrict__ node_off, int nnodes, const uint32_t *__restrict__ tw_level,
                          const uint8_t *__restrict__ dneg_level) {
  __shared__ uint32_t Ps[L * 128];  // each thread's first product of a side
  const int q = n >> 2;
  const long long per = (long long)nnodes * q;  // butterflies per signal
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nsig * per) return;
  const long long r = t % per;
  uint32_t *y = static_cast<uint32_t *>(items[t / per].out);
  mp_bfly_one<L, false, true>(y, N, 1, 0, n, node_off[r / q], (int)(r % q), tw_level, dneg_level, 1,
                              Ps + threadIdx.x, blockDim.x, nullptr);
}

// the level copy of the twiddles: out[(r*L + i)*q + k] = tw[(r*L + i)*N/4 + k*N/n]
__global__ void __launch_bounds__(256) mp_level_twiddle_kernel(const uint32_t *__restrict__ tw,
                                                               const uint8_t *__restrict__ dneg, int N, int n, int L,
                                                               uint32_t *__restrict__ out,
                                                               uint8_t *__restrict__ dout) {
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = N / n;
  if (t < 3LL * L * q) out[t] = tw[(t / q) * (N / 4) + (t % q) * stride];
  if (t < q) dout[t] = dneg[t * stride];
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

size_t group_twiddle_words(int L, const TreeTables &T) {
  size_t w = 0;
  for (int lv = 0; lv < T.nlevels; ++lv) w += (size_t)3 * L * (T.level_n[lv] / 4);
  return w;
}

cudaError_t group_twiddles(int L, const QueueTables &Q, uint32_t *d_tw, uint8_t *d_dneg, GroupTw &gt,
                           cudaStream_t s) {
  const TreeTables &T = Q.tree;
  size_t w = 0, d = 0;
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const int n = T.level_n[lv], q = n / 4;
    gt.tw[lv] = d_tw + w;
    gt.dneg[lv] = d_dneg + d;
    const long long cnt = 3LL * L * q;
    mp_level_twiddle_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(Q.tw, Q.dneg, Q.N, n, L, d_tw + w,
                                                                          d_dneg + d);
    w += (size_t)cnt;
    d += (size_t)q;
  }
  return cudaGetLastError();
}

template <int L>
static cudaError_t group_run(const QueueItem *items, int nsig, const QueueTables &Q, const GroupTw &gt,
                             cudaStream_t s) {
  const TreeTables &T = Q.tree;
  const long long leaves = (long long)nsig * T.nleaves;
  if (leaves > 0)
    mp_group_leaf_kernel<L><<<(unsigned)((leaves + 255) / 256), 256, 0, s>>>(items, nsig, Q.N, T.leaves, T.nleaves);
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const int n = T.level_n[lv];
    const long long total = (long long)nsig * T.level_count[lv] * (n / 4);
    mp_group_level_kernel<L><<<(unsigned)((total + 127) / 128), 128, 0, s>>>(
        items, nsig, Q.N, n, T.node_off + T.level_start[lv], T.level_count[lv], gt.tw[lv], gt.dneg[lv]);
  }
  return cudaGetLastError();
}

cudaError_t group_launch(int L, const QueueItem *items, int nsig, const QueueTables &T, const GroupTw &gt,
                         cudaStream_t s) {
  if (nsig <= 0) return cudaSuccess;
#define MPFFT_G_CASE(LL) \
  case LL:               \
    return group_run<LL>(items, nsig, T, gt, s);
  switch (L) {
    MPFFT_G_CASE(2) MPFFT_G_CASE(3) MPFFT_G_CASE(4) MPFFT_G_CASE(5) MPFFT_G_CASE(6) MPFFT_G_CASE(7)
    MPFFT_G_CASE(8) MPFFT_G_CASE(9) MPFFT_G_CASE(10) MPFFT_G_CASE(11) MPFFT_G_CASE(12) MPFFT_G_CASE(13)
    MPFFT_G_CASE(14) MPFFT_G_CASE(15) MPFFT_G_CASE(16) MPFFT_G_CASE(17) MPFFT_G_CASE(18) MPFFT_G_CASE(19)
    MPFFT_G_CASE(20) MPFFT_G_CASE(21) MPFFT_G_CASE(22) MPFFT_G_CASE(23) MPFFT_G_CASE(24) MPFFT_G_CASE(25)
    MPFFT_G_CASE(26) MPFFT_G_CASE(27) MPFFT_G_CASE(28) MPFFT_G_CASE(29) MPFFT_G_CASE(30) MPFFT_G_CASE(31)
    MPFFT_G_CASE(32) MPFFT_G_CASE(33) MPFFT_G_CASE(34)
    default:
      return cudaErrorInvalidValue;
  }
#undef MPFFT_G_CASE
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
