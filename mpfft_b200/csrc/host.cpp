// libmpfft_b200 host side: the C ABI declared in include/mpfft_b200.h.
//
// Responsibilities
//  - plans: one per (n, limb count) for the mp tier and per n for FP64, cached
//    process-wide; a plan owns the device twiddle tables, the breadth-first
//    schedule of the split-radix tree, device buffers and a CUDA stream;
//  - twiddles: built with MPFR at 32L+64 bits and rounded once to fixed point
//    (the reference builds its LUT with MPFR at P, lut() in
//    lab/parallel/mp/parallel_mp_fft2.c:71-82);
//  - conversion between mpfr_t arrays and device limb planes (block floating
//    point: one exponent per signal);
//  - error status for the void drop-in entry points.
#include <algorithm>
#include <climits>
#include <cmath>
#include <functional>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <string>
#include <atomic>
#include <condition_variable>
#include <thread>
#include <tuple>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <cuda_runtime.h>

#include "mpfr_abi.h"
#define MPFFT_MPFR_TYPES_PROVIDED 1
#include "../../include/mpfft_b200.h"
#include "mpfft_internal.h"

#define MPFFT_API extern "C" __attribute__((visibility("default")))

namespace mpfft {

// ---------------------------------------------------------------------------
// status
// ---------------------------------------------------------------------------
static thread_local int g_err = MPFFT_OK;
static thread_local char g_msg[256] = "";

static int set_err(int code, const char *fmt, ...) {
  g_err = code;
  if (code == MPFFT_OK) {
    g_msg[0] = 0;
    return code;
  }
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof g_msg, fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(expr)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (expr);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return set_err(MPFFT_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// ---------------------------------------------------------------------------
// allocations of execution buffers, with a test hook
// ---------------------------------------------------------------------------
// Every device or pinned-host buffer that an execution grows on demand comes
// from these two functions.  mpfft_diag_fail_allocations(k) makes the k-th
// such allocation from now on (0 = the next one), and every later one, fail as
// cudaMalloc would, so that the MPFFT_ENOMEM paths can be exercised without
// exhausting a real device; -1 switches the hook off.
static std::atomic<long> g_alloc_fail_after{-1};

static bool alloc_should_fail() {
  long v = g_alloc_fail_after.load();
  while (v > 0 && !g_alloc_fail_after.compare_exchange_weak(v, v - 1)) {
  }
  return v == 0;
}

static cudaError_t dev_alloc(void **p, size_t bytes) {
  if (alloc_should_fail()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

static cudaError_t host_alloc(void **p, size_t bytes) {
  if (alloc_should_fail()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(p, bytes);
}

static bool is_pow2(unsigned long n) { return n >= 1 && (n & (n - 1)) == 0; }
static int ilog2(unsigned long n) {
  int l = 0;
  while ((1UL << l) < n) ++l;
  return l;
}

// ---------------------------------------------------------------------------
// breadth-first schedule of the reference's recursion tree
// ---------------------------------------------------------------------------
struct HostTree {
  std::vector<Leaf> leaves;
  std::map<int, std::vector<int>> levels;  // node size -> output offsets
};

// Walks the recursion of mp_sr24_cp_fft (parallel_mp_fft2.c:180-182):
// (n/2, 2s, sn) -> out+0, (n/4, 4s, sn+s) -> out+n/2, (n/4, 4s, sn-s) -> out+3n/4.
static void walk(HostTree &t, int n, int s, int sn, int out, int leaf_max) {
  if (n <= leaf_max) {
    t.leaves.push_back(Leaf{out, sn, s, n});
    return;
  }
  walk(t, n / 2, 2 * s, sn, out, leaf_max);
  walk(t, n / 4, 4 * s, sn + s, out + n / 2, leaf_max);
  walk(t, n / 4, 4 * s, sn - s, out + 3 * n / 4, leaf_max);
  t.levels[n].push_back(out);
}

struct DeviceTree {
  TreeTables tabs;
  Leaf *d_leaves = nullptr;
  int *d_nodes = nullptr;
  int *d_pair_nodes = nullptr;
  ~DeviceTree() {
    if (d_leaves) cudaFree(d_leaves);
    if (d_nodes) cudaFree(d_nodes);
    if (d_pair_nodes) cudaFree(d_pair_nodes);
  }
};

static int build_tree(DeviceTree &dt, unsigned long N, int leaf_max) {
  HostTree t;
  walk(t, (int)N, 1, 0, 0, leaf_max);
  dt.tabs.N = (int)N;
  dt.tabs.nleaves = (int)t.leaves.size();
  for (const Leaf &lf : t.leaves)
    if (lf.n <= 4) ++dt.tabs.leaf_count[lf.n];
  std::vector<int> nodes;
  int lv = 0;
  for (auto &kv : t.levels) {
    if (lv >= kMaxLevels) return set_err(MPFFT_EUNSUPPORTED, "transform too large");
    dt.tabs.level_n[lv] = kv.first;
    dt.tabs.level_start[lv] = (int)nodes.size();
    dt.tabs.level_count[lv] = (int)kv.second.size();
    nodes.insert(nodes.end(), kv.second.begin(), kv.second.end());
    ++lv;
  }
  dt.tabs.nlevels = lv;
  // per level: its nodes that are not the first child of a node of the next
  // level (a first child starts at its parent's offset)
  std::vector<int> pair_nodes;
  for (int l = 0; l + 1 < lv; ++l) {
    const int *up = nodes.data() + dt.tabs.level_start[l + 1];
    std::set<int> parents(up, up + dt.tabs.level_count[l + 1]);
    dt.tabs.pair_start[l] = (int)pair_nodes.size();
    for (int j = 0; j < dt.tabs.level_count[l]; ++j) {
      const int o = nodes[dt.tabs.level_start[l] + j];
      if (!parents.count(o)) pair_nodes.push_back(o);
    }
    dt.tabs.pair_count[l] = (int)pair_nodes.size() - dt.tabs.pair_start[l];
  }
  CUDA_TRY(cudaMalloc(&dt.d_leaves, sizeof(Leaf) * t.leaves.size()));
  CUDA_TRY(cudaMemcpy(dt.d_leaves, t.leaves.data(), sizeof(Leaf) * t.leaves.size(), cudaMemcpyHostToDevice));
  if (!nodes.empty()) {
    CUDA_TRY(cudaMalloc(&dt.d_nodes, sizeof(int) * nodes.size()));
    CUDA_TRY(cudaMemcpy(dt.d_nodes, nodes.data(), sizeof(int) * nodes.size(), cudaMemcpyHostToDevice));
  }
  if (!pair_nodes.empty()) {
    CUDA_TRY(cudaMalloc(&dt.d_pair_nodes, sizeof(int) * pair_nodes.size()));
    CUDA_TRY(cudaMemcpy(dt.d_pair_nodes, pair_nodes.data(), sizeof(int) * pair_nodes.size(),
                        cudaMemcpyHostToDevice));
  }
  dt.tabs.leaves = dt.d_leaves;
  dt.tabs.node_off = dt.d_nodes;
  dt.tabs.pair_nodes = dt.d_pair_nodes;
  return MPFFT_OK;
}

// ---------------------------------------------------------------------------
// fixed point <-> MPFR
// ---------------------------------------------------------------------------

// 32 bits of the non-negative integer M (32-bit words, least significant
// first) starting at bit position pos (pos may be negative).
static inline uint32_t bits32(const uint32_t *M, int nw, long pos) {
  long w = pos >= 0 ? pos / 32 : -((-pos + 31) / 32);
  int off = (int)(pos - w * 32);
  uint64_t lo = (w >= 0 && w < nw) ? M[w] : 0;
  uint64_t hi = (w + 1 >= 0 && w + 1 < nw) ? M[w + 1] : 0;
  return (uint32_t)(((hi << 32) | lo) >> off);
}

// |x| * 2^(F - e_s), rounded to nearest (ties away), into L words; returns the
// sign (0 / 1).  x must be a regular number or zero.
static uint32_t mpfr_to_fixed(mpfr_srcptr x, int L, long F, long e_s, uint32_t *out) {
  for (int i = 0; i < L; ++i) out[i] = 0;
  if (mpfr_zero_p(x)) return 0;
  const long prec = x->_mpfr_prec;
  const int nl = (int)((prec + 63) / 64);
  const uint32_t *M = reinterpret_cast<const uint32_t *>(x->_mpfr_d);  // little-endian 64-bit limbs
  const int nw = 2 * nl;
  // value = M * 2^(exp - 64 nl);  A = M * 2^sh
  const long sh = (long)x->_mpfr_exp - 64L * nl + F - e_s;
  for (int i = 0; i < L; ++i) out[i] = bits32(M, nw, 32L * i - sh);
  if (sh < 0) {
    const long rb = -sh - 1;  // highest discarded bit
    uint32_t round_bit = (rb < 32L * nw) ? (bits32(M, nw, rb) & 1u) : 0u;
    uint32_t c = round_bit;
    for (int i = 0; i < L && c; ++i) {
      uint64_t t = (uint64_t)out[i] + c;
      out[i] = (uint32_t)t;
      c = (uint32_t)(t >> 32);
    }
  }
  return x->_mpfr_sign < 0 ? 1u : 0u;
}

// two's-complement L-word integer A -> y = A * 2^e2, rounded to y's precision.
static void fixed_to_mpfr(const uint32_t *A, int L, long e2, mpfr_ptr y) {
  uint32_t mag[kMaxLimbsBig + 2];
  const bool neg = (A[L - 1] >> 31) != 0;
  uint32_t c = neg ? 1u : 0u;
  const uint32_t m = neg ? 0xffffffffu : 0u;
  for (int i = 0; i < L; ++i) {
    uint64_t t = (uint64_t)(A[i] ^ m) + c;
    mag[i] = (uint32_t)t;
    c = (uint32_t)(t >> 32);
  }
  int nw = L;
  if (nw & 1) mag[nw++] = 0;
  while (nw > 0 && mag[nw - 1] == 0) --nw;
  if (nw == 0) {
    mpfr_set_zero(y, 1);
    return;
  }
  const int n64 = (nw + 1) / 2;
  if (nw & 1) mag[nw] = 0;
  __mpz_struct z;
  z._mp_alloc = n64;
  z._mp_size = neg ? -n64 : n64;
  z._mp_d = reinterpret_cast<mp_limb_t *>(mag);
  mpfr_set_z_2exp(y, &z, e2, MPFR_RNDN);
}

// A process-wide pool of hardware_concurrency - 1 workers for the host-side
// conversion loops (they run several times per call on large batches, so
// thread start-up would show).  One job at a time: a caller that finds the pool
// busy, or runs in a process forked after the pool was started (whose workers
// did not survive the fork), falls back to its own threads.
class WorkerPool {
 public:
  static WorkerPool &get() {
    static WorkerPool pool;
    return pool;
  }
  // fn over parts [i*chunk, min(n, (i+1)*chunk)), i < nparts; false when unavailable
  bool run(long n, long nparts, long chunk, const std::function<void(long, long)> &fn) {
    if (getpid() != pid_ || workers_.empty()) return false;
    std::unique_lock<std::mutex> busy(run_mu_, std::try_to_lock);
    if (!busy.owns_lock()) return false;
    {
      std::lock_guard<std::mutex> g(mu_);
      fn_ = &fn;
      n_ = n;
      nparts_ = nparts;
      chunk_ = chunk;
      next_.store(0);
      done_ = 0;
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> g(mu_);
    done_cv_.wait(g, [&] { return done_ == nparts_; });
    fn_ = nullptr;
    return true;
  }

 private:
  WorkerPool() : pid_(getpid()) {
    const unsigned hw = std::thread::hardware_concurrency();
    for (unsigned i = 1; i < hw; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~WorkerPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();
  }
  void work() {
    long ndone = 0;
    for (long i; (i = next_.fetch_add(1)) < nparts_;) {
      const long a = i * chunk_, b = std::min(n_, a + chunk_);
      if (a < b) (*fn_)(a, b);
      ++ndone;
    }
    if (ndone) {
      std::lock_guard<std::mutex> g(mu_);
      done_ += ndone;
      if (done_ == nparts_) done_cv_.notify_all();
    }
  }
  void loop() {
    unsigned long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
    }
  }
  const pid_t pid_;
  std::vector<std::thread> workers_;
  std::mutex run_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(long, long)> *fn_ = nullptr;
  long n_ = 0, nparts_ = 0, chunk_ = 0, done_ = 0;
  std::atomic<long> next_{0};
  unsigned long gen_ = 0;
  bool stop_ = false;
};

static void parallel_for(long n, long grain, const std::function<void(long, long)> &fn) {
  unsigned hw = std::thread::hardware_concurrency();
  long nthreads = std::min<long>(hw ? hw : 1, (n + grain - 1) / grain);
  if (nthreads <= 1) {
    fn(0, n);
    return;
  }
  // a few parts per thread balance uneven element costs
  const long nparts = std::min<long>((n + grain - 1) / grain, 4 * nthreads);
  const long chunk = (n + nparts - 1) / nparts;
  if (WorkerPool::get().run(n, nparts, chunk, fn)) return;
  std::vector<std::thread> th;
  const long tchunk = (n + nthreads - 1) / nthreads;
  for (long t = 0; t < nthreads; ++t) {
    long a = t * tchunk, b = std::min(n, a + tchunk);
    if (a >= b) break;
    th.emplace_back([&fn, a, b] { fn(a, b); });
  }
  for (auto &x : th) x.join();
}

// Copy `words` 64-bit limbs to pinned staging memory that the CPU will not read
// again: streaming stores when both ends allow 16-byte vectors (no
// read-for-ownership of the destination lines), memcpy otherwise.
static inline void stage_limbs(uint64_t *dst, const uint64_t *src, int words) {
#if defined(__x86_64__)
  if (((uintptr_t)dst & 15) == 0 && (words & 1) == 0) {
    for (int k = 0; k < words; k += 2)
      _mm_stream_si128(reinterpret_cast<__m128i *>(dst + k),
                       _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + k)));
    return;
  }
#endif
  memcpy(dst, src, (size_t)words * 8);
}

// Host copies of large arrays of doubles (to and from pinned staging) on the
// worker pool, 512 KB per piece; small copies stay on the calling thread.
constexpr long kParCopyGrain = 1L << 16;
constexpr size_t kCopyPiece = (size_t)1 << 18;  // doubles (2 MB) per overlapped staging piece
static void par_copy(double *dst, const double *src, size_t n) {
  parallel_for((long)n, kParCopyGrain, [&](long a, long b) { memcpy(dst + a, src + a, (size_t)(b - a) * sizeof(double)); });
}

static inline void stage_word(int64_t *dst, int64_t v) {
#if defined(__x86_64__)
  _mm_stream_si64(reinterpret_cast<long long *>(dst), (long long)v);
#else
  *dst = v;
#endif
}

static inline void stage_fence() {
#if defined(__x86_64__)
  _mm_sfence();
#endif
}

// ---------------------------------------------------------------------------
// mp plans
// ---------------------------------------------------------------------------

// Limb count for (N, P): one sign bit, H = log2 N + 2 headroom bits and at
// least P + log2 N + 4 fraction bits.
static int mp_limbs_for(unsigned long N, long P) {
  const long lg = ilog2(N);
  long L = (P + 2 * lg + 7 + 31) / 32;
  return (int)std::max<long>(L, kMinLimbs);
}

struct MpTwiddles {
  uint32_t *d_tw = nullptr;
  uint8_t *d_dneg = nullptr;
  ~MpTwiddles() {
    if (d_tw) cudaFree(d_tw);
    if (d_dneg) cudaFree(d_dneg);
  }
};

// Twiddle tables for (N, L): cos, cos+sin and |cos-sin| of 2 pi k/N, k < N/4,
// as unsigned L-limb fixed-point with 32L-1 fraction bits, plus sign(cos-sin).
static int build_twiddles(MpTwiddles &tw, unsigned long N, int L) {
  const unsigned long q = N / 4;
  if (q == 0) return MPFFT_OK;
  std::vector<uint32_t> h((size_t)3 * L * q);
  std::vector<uint8_t> neg(q);
  const long pw = 32L * L + 64;
  parallel_for((long)q, 16, [&](long a, long b) {
    mpfr_t pi2, th, s, c, t;
    mpfr_init2(pi2, pw + 32);
    mpfr_init2(th, pw + 32);
    mpfr_init2(s, pw);
    mpfr_init2(c, pw);
    mpfr_init2(t, pw);
    mpfr_const_pi(pi2, MPFR_RNDN);
    uint32_t tmp[kMaxLimbsBig + 2];
    for (long k = a; k < b; ++k) {
      mpfr_mul_ui(th, pi2, 2UL * (unsigned long)k, MPFR_RNDN);
      mpfr_div_ui(th, th, N, MPFR_RNDN);
      mpfr_sin_cos(s, c, th, MPFR_RNDN);
      for (int which = 0; which < 3; ++which) {
        if (which == 0) mpfr_set(t, c, MPFR_RNDN);
        else if (which == 1) mpfr_add(t, c, s, MPFR_RNDN);
        else mpfr_sub(t, c, s, MPFR_RNDN);
        uint32_t sg = mpfr_to_fixed(t, L, 32L * L - 1, 0, tmp);
        if (which == 2) neg[k] = (uint8_t)sg;
        for (int i = 0; i < L; ++i) h[((size_t)which * L + i) * q + k] = tmp[i];
      }
    }
    mpfr_clear(pi2);
    mpfr_clear(th);
    mpfr_clear(s);
    mpfr_clear(c);
    mpfr_clear(t);
    mpfr_free_cache();
  });
  CUDA_TRY(cudaMalloc(&tw.d_tw, h.size() * sizeof(uint32_t)));
  CUDA_TRY(cudaMemcpy(tw.d_tw, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMalloc(&tw.d_dneg, q));
  CUDA_TRY(cudaMemcpy(tw.d_dneg, neg.data(), q, cudaMemcpyHostToDevice));
  return MPFFT_OK;
}

}  // namespace mpfft

using namespace mpfft;

namespace mpfft {
static void d_plan_delete(mpfft_d_plan *p);
}

struct mpfft_mp_plan {
  unsigned long N = 0;
  long P = 0;
  int L = 0;
  long F = 0;  // fraction bits
  bool host_only = false;  // conversion-only plan: no device state
  bool force_host_conversion = false;  // convert mpfr_t <-> limbs on the host even when the GPU could
  bool real = false;          // real transform of n_real = 2N points: N-point complex transform + split step
  unsigned long n_real = 0;
  // points per signal the staging buffers hold (the half spectrum of a real plan has N+1)
  unsigned long pts_max() const { return real ? N + 1 : N; }
  // multi-dimensional plan: dims[0] x ... x dims[rank-1] = N points, row-major
  int rank = 1;
  unsigned long dims[3] = {0, 0, 0};
  std::unique_ptr<mpfft_mp_plan> axis[3];  // rank > 1: one-dimensional plan of each axis (same L)
  uint32_t *d_tmp = nullptr;               // rank > 1: transposition buffer, grown on demand
  size_t tmp_words = 0;
  uint32_t *d_big = nullptr;  // streaming-kernel scratch (L > kMaxLimbs), grown on demand
  size_t big_words = 0;
  // Device work that reads or writes d_tmp / d_big is ordered across calls:
  // each such call makes its stream wait for scratch_ev (recorded after the
  // previous such call's kernels) and records it again after its own, under mu.
  cudaEvent_t scratch_ev = nullptr;
  bool scratch_recorded = false;
  int device = -1;  // the CUDA device the plan's tables live on (-1: host-only plan)
  DeviceTree tree;
  MpTwiddles tw;
  MpDeviceTables tabs;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  // staging for host-array execution, grown on demand
  size_t cap_words = 0;
  uint32_t *d_in = nullptr, *d_out = nullptr;
  uint32_t *h_in = nullptr, *h_out = nullptr;
  std::vector<long> exps;
  // GPU-conversion pipeline (uniform-precision calls): two slots, each with
  // its own stream and staging for one chunk of signals, grown on demand
  struct ConvSlot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    uint32_t *d_in = nullptr, *d_out = nullptr;
    // raw MPFR fields in (i) and out (o), pinned host and device: one block
    // per direction laid out per chunk by stage_view (one copy each way)
    uint64_t *h_i = nullptr, *d_i = nullptr, *h_o = nullptr, *d_o = nullptr;
    int64_t *d_es = nullptr;
    // the chunk's copies and kernels captured as a CUDA graph, per chunk shape
    // (null: the shape runs its launches directly); uses[] counts the direct
    // runs before a shape is captured
    std::map<std::vector<long>, cudaGraphExec_t> graphs;
    std::map<std::vector<long>, int> uses;
    uint32_t *d_big = nullptr;  // streaming-kernel scratch of this slot (L > kMaxLimbs)
    uint32_t *d_tmp = nullptr;  // transposition buffer of this slot (multi-dimensional plans)
  };
  ConvSlot cv[2];
  unsigned long cv_chunk = 0;  // signals per chunk the slots hold
  int cv_nli = 0, cv_nlo = 0;
  void free_conv() {
    for (auto &c : cv) {
      for (auto &g : c.graphs)
        if (g.second) cudaGraphExecDestroy(g.second);
      for (void *q : {(void *)c.d_in, (void *)c.d_out, (void *)c.d_i, (void *)c.d_o, (void *)c.d_es,
                      (void *)c.d_big, (void *)c.d_tmp})
        if (q) cudaFree(q);
      for (void *q : {(void *)c.h_i, (void *)c.h_o})
        if (q) cudaFreeHost(q);
      if (c.st) cudaStreamDestroy(c.st);
      if (c.done) cudaEventDestroy(c.done);
      c = ConvSlot();
    }
    cv_chunk = 0;
  }
  // MPFFT_PLAN_FLOAT_TIERS: the compensated floating-point plan that runs this
  // plan's host-array transforms (null: the limb kernels run them), and the
  // form the plan reports (MPFFT_FORM_*)
  mpfft_d_plan *fplan = nullptr;
  int form = MPFFT_FORM_LIMBS;
  // device-layout executions (mpfft_mp_execute_device) replayed from CUDA
  // graphs, keyed by (batch, input, output); null: that call shape runs its
  // launches directly.  dev_uses counts the direct runs before a capture.
  using DevKey = std::tuple<unsigned long, const void *, const void *>;
  std::map<DevKey, cudaGraphExec_t> dev_graphs;
  std::map<DevKey, int> dev_uses;
  void free_dev_graphs() {
    for (auto &g : dev_graphs)
      if (g.second) cudaGraphExecDestroy(g.second);
    dev_graphs.clear();
    dev_uses.clear();
  }
  ~mpfft_mp_plan() {
    free_dev_graphs();
    free_conv();
    d_plan_delete(fplan);
    if (scratch_ev) cudaEventDestroy(scratch_ev);
    if (d_tmp) cudaFree(d_tmp);
    if (d_big) cudaFree(d_big);
    if (d_in) cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    if (h_in) cudaFreeHost(h_in);
    if (h_out) cudaFreeHost(h_out);
    if (stream) cudaStreamDestroy(stream);
  }
};

struct mpfft_d_plan {
  unsigned long N = 0;
  // multi-dimensional plan: dims[0] x ... x dims[rank-1] = N points, row-major
  int rank = 1;
  unsigned long dims[3] = {0, 0, 0};
  std::unique_ptr<mpfft_d_plan> axis[3];
  double *d_tmp = nullptr;  // rank > 1: transposition buffer; real plans: split-step output
  size_t tmp_cap = 0;
  cudaEvent_t scratch_ev = nullptr;  // orders the device work that uses d_tmp across calls (as mp plans)
  bool scratch_recorded = false;
  bool dd = false;          // double-double tier
  int tier = -1;            // compensated tier (kTierDD / kTierQD / kTierFF), -1 for FP64
  bool real = false;        // real transform of n_real = 2N points: N-point complex transform + split step
  unsigned long n_real = 0;
  double *d_wc = nullptr, *d_ws = nullptr;  // real plans: cos, sin of 2 pi k / n_real, k < N/2
  DeviceTree upper;                   // levels above the shared-memory sub-transforms
  std::vector<void *> dev_allocs;     // roots, perms, sub-schedule tables
  double *d_wr = nullptr, *d_wi = nullptr;
  DDeviceTables tabs;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  size_t cap = 0;
  double *d_in = nullptr, *d_out = nullptr, *h_in = nullptr, *h_out = nullptr;
  std::vector<cudaEvent_t> piece_done;  // chunked device-to-host copies (d_execute_impl)
  ~mpfft_d_plan() {
    if (scratch_ev) cudaEventDestroy(scratch_ev);
    for (cudaEvent_t e : piece_done) cudaEventDestroy(e);
    for (void *q : dev_allocs) cudaFree(q);
    if (d_wr) cudaFree(d_wr);
    if (d_wi) cudaFree(d_wi);
    if (d_in) cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    if (h_in) cudaFreeHost(h_in);
    if (h_out) cudaFreeHost(h_out);
    if (d_tmp) cudaFree(d_tmp);
    if (d_wc) cudaFree(d_wc);
    if (d_ws) cudaFree(d_ws);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace mpfft {

static int device_ready() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return set_err(MPFFT_ECUDA, "no CUDA device available: %s", cudaGetErrorString(e));
  return MPFFT_OK;
}

// Device work that uses a plan's shared scratch is ordered across calls and
// streams: the call's stream first waits for the previous such call's kernels
// (scratch_ev), and the event is recorded again after the call's own kernels.
// The caller holds the plan's lock from scratch_wait to scratch_record.
template <class Plan>
static int scratch_wait(Plan *p, cudaStream_t st) {
  if (!p->scratch_ev) CUDA_TRY(cudaEventCreateWithFlags(&p->scratch_ev, cudaEventDisableTiming));
  if (p->scratch_recorded) CUDA_TRY(cudaStreamWaitEvent(st, p->scratch_ev, 0));
  return MPFFT_OK;
}

template <class Plan>
static int scratch_record(Plan *p, cudaStream_t st) {
  CUDA_TRY(cudaEventRecord(p->scratch_ev, st));
  p->scratch_recorded = true;
  return MPFFT_OK;
}

// real: n real points, planned as an n/2-point complex transform whose limb
// format (L, F) and twiddle table are those of an n-point transform.
// force_L > 0: use that limb count (the axes of a multi-dimensional plan take the
// format of the whole signal)
static int mp_plan_init(mpfft_mp_plan *p, unsigned long n, long prec, bool host_only = false, bool real = false,
                        int force_L = 0) {
  if (!is_pow2(n)) return set_err(MPFFT_EINVAL, "n=%lu is not a power of two", n);
  if (real && n < 2) return set_err(MPFFT_EINVAL, "a real transform needs n >= 2 (n=%lu)", n);
  if (prec < 2) return set_err(MPFFT_EINVAL, "precision %ld < 2", prec);
  if (n > (1UL << 26)) return set_err(MPFFT_EUNSUPPORTED, "n=%lu too large", n);
  int L = force_L > 0 ? force_L : mp_limbs_for(n, prec);
  if (L > kMaxLimbsBig)
    return set_err(MPFFT_EUNSUPPORTED, "precision %ld at n=%lu needs %d limbs (> %d supported)", prec, n, L,
                   kMaxLimbsBig);
  if (real && L > kMaxLimbs)
    return set_err(MPFFT_EUNSUPPORTED, "real transforms support up to %d limbs (precision %ld at n=%lu needs %d)",
                   kMaxLimbs, prec, n, L);
  const unsigned long nt = real ? n / 2 : n;  // complex transform size
  p->N = nt;
  p->real = real;
  p->n_real = real ? n : 0;
  p->P = prec;
  p->L = L;
  p->F = 32L * L - 1 - (ilog2(n) + 2);
  p->host_only = host_only;
  if (host_only) return MPFFT_OK;
  if (int e = device_ready()) return e;
  CUDA_TRY(cudaGetDevice(&p->device));
  if (int e = build_tree(p->tree, nt, 4)) return e;
  if (int e = build_twiddles(p->tw, n, L)) return e;
  static_cast<TreeTables &>(p->tabs) = p->tree.tabs;
  p->tabs.tw = p->tw.d_tw;
  p->tabs.dneg = p->tw.d_dneg;
  p->tabs.tws = real ? 2 : 1;
  CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  return MPFFT_OK;
}

// Multi-dimensional plan (rank 1..3, row-major, last index fastest): the limb
// format of the whole N = prod(dims)-point signal, plus a one-dimensional
// plan per axis with that format.
static int mp_plan_init_nd(mpfft_mp_plan *p, int rank, const unsigned long *dims, long prec, bool host_only) {
  if (rank < 1 || rank > 3 || !dims) return set_err(MPFFT_EINVAL, "rank must be 1, 2 or 3");
  unsigned long n = 1;
  for (int i = 0; i < rank; ++i) {
    if (!is_pow2(dims[i])) return set_err(MPFFT_EINVAL, "dims[%d]=%lu is not a power of two", i, dims[i]);
    if (dims[i] > (1UL << 26) || n > (1UL << 26) / dims[i])
      return set_err(MPFFT_EUNSUPPORTED, "more than 2^26 points in total");
    n *= dims[i];
  }
  if (rank == 1) return mp_plan_init(p, n, prec, host_only);
  if (int e = mp_plan_init(p, n, prec, true)) return e;  // the format of the whole signal
  p->host_only = host_only;
  p->rank = rank;
  for (int i = 0; i < rank; ++i) p->dims[i] = dims[i];
  if (host_only) return MPFFT_OK;
  if (int e = device_ready()) return e;
  CUDA_TRY(cudaGetDevice(&p->device));
  for (int i = 0; i < rank; ++i) {
    p->axis[i].reset(new (std::nothrow) mpfft_mp_plan);
    if (!p->axis[i]) return set_err(MPFFT_ENOMEM, "out of host memory");
    if (int e = mp_plan_init(p->axis[i].get(), dims[i], prec, false, false, p->L)) return e;
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  return MPFFT_OK;
}

// ---------------------------------------------------------------------------
// dispatch of mp plans to the compensated floating-point tiers
// ---------------------------------------------------------------------------
//
// With MPFFT_PLAN_FLOAT_TIERS an mp plan whose precision a floating tier
// covers runs its host-array transforms on that tier instead of fixed-point
// limbs.  A tier covers P when its normwise error, measured against the 2P-bit
// oracle over N = 2 .. 2^16, stays within the mp contract 8 log2(N) 2^-P:
//   float-float (about 48 bits)  P <= 40
//   FP64 (the reference's double transform)  40 < P <= 48
//   double-double (about 106 bits)  48 < P <= 98
//   quad-double (about 212 bits)  98 < P <= 200
// Larger precisions keep the limb kernels.
// With MPFFT_PLAN_NATIVE_TIERS instead, P picks the smallest word format that
// holds P bits (float-float 48, FP64 53, double-double 106, quad-double 212)
// and the result carries that tier's own error, about log2(N) 2^-(bits-2).
static int float_form_for(long P, bool native = false) {
  if (native) {
    if (P <= 48) return MPFFT_FORM_FLOAT_FLOAT;
    if (P <= 53) return MPFFT_FORM_DOUBLE;
    if (P <= 106) return MPFFT_FORM_DOUBLE_DOUBLE;
    if (P <= 212) return MPFFT_FORM_QUAD_DOUBLE;
    return -1;
  }
  if (P <= 40) return MPFFT_FORM_FLOAT_FLOAT;
  if (P <= 48) return MPFFT_FORM_DOUBLE;
  if (P <= 98) return MPFFT_FORM_DOUBLE_DOUBLE;
  if (P <= 200) return MPFFT_FORM_QUAD_DOUBLE;
  return -1;
}

static int d_plan_init(mpfft_d_plan *p, unsigned long n, int sub_max = 0);
static int d_plan_init_tier(mpfft_d_plan *p, unsigned long n, int tier, int sub_max = 0);

static int mp_plan_attach_float_tier(mpfft_mp_plan *p, bool native) {
  const int form = float_form_for(p->P, native);
  if (form < 0 || p->rank > 1 || p->real || p->host_only) return MPFFT_OK;
  std::unique_ptr<mpfft_d_plan> f(new (std::nothrow) mpfft_d_plan);
  if (!f) return set_err(MPFFT_ENOMEM, "out of host memory");
  const int tier = form == MPFFT_FORM_FLOAT_FLOAT ? kTierFF : form == MPFFT_FORM_DOUBLE_DOUBLE ? kTierDD : kTierQD;
  if (int e = form == MPFFT_FORM_DOUBLE ? d_plan_init(f.get(), p->N) : d_plan_init_tier(f.get(), p->N, tier)) return e;
  p->fplan = f.release();
  p->form = form;
  return MPFFT_OK;
}

// process-wide cache used by the drop-in entry points
static std::mutex g_cache_mu;
static std::map<std::pair<unsigned long, int>, std::unique_ptr<mpfft_mp_plan>> g_mp_cache;
static std::map<unsigned long, std::unique_ptr<mpfft_d_plan>> g_d_cache;

static mpfft_mp_plan *mp_cached(unsigned long n, long prec) {
  std::lock_guard<std::mutex> g(g_cache_mu);
  const int L = mp_limbs_for(n, prec);
  auto key = std::make_pair(n, L);
  auto it = g_mp_cache.find(key);
  if (it != g_mp_cache.end()) return it->second.get();
  std::unique_ptr<mpfft_mp_plan> p(new mpfft_mp_plan);
  if (mp_plan_init(p.get(), n, prec) != MPFFT_OK) return nullptr;
  auto *raw = p.get();
  g_mp_cache[key] = std::move(p);
  return raw;
}

static int mp_reserve(mpfft_mp_plan *p, unsigned long batch) {
  const size_t words = (size_t)2 * p->L * p->pts_max() * batch;
  if (words <= p->cap_words) return MPFFT_OK;
  if (p->d_in) cudaFree(p->d_in);
  if (p->d_out) cudaFree(p->d_out);
  if (p->h_in) cudaFreeHost(p->h_in);
  if (p->h_out) cudaFreeHost(p->h_out);
  p->d_in = p->d_out = p->h_in = p->h_out = nullptr;
  p->cap_words = 0;
  if (dev_alloc((void **)&p->d_in, words * 4) != cudaSuccess || dev_alloc((void **)&p->d_out, words * 4) != cudaSuccess ||
      host_alloc((void **)&p->h_in, words * 4) != cudaSuccess || host_alloc((void **)&p->h_out, words * 4) != cudaSuccess) {
    cudaGetLastError();
    return set_err(MPFFT_ENOMEM, "cannot allocate %zu-byte staging buffers", words * 4);
  }
  p->cap_words = words;
  return MPFFT_OK;
}

// Geometry of a host mpfr_t array: element q < n of signal b is a[b*pitch + q*s].
// With per-signal bases (base[part] non-null) element q of signal b is
// base[part][b][q*s] instead (part 0 real, 1 imaginary), and the array
// arguments are ignored.
struct IoShape {
  unsigned long n, pitch, s;
  mpfr_t *const *base[2] = {nullptr, nullptr};
};
static inline IoShape io_signals(unsigned long n, unsigned long s) { return IoShape{n, n * s, s}; }
static inline mpfr_ptr elem(mpfr_t *a, int part, unsigned long b, const IoShape &io, unsigned long q) {
  if (io.base[part]) return io.base[part][b][q * io.s];
  return a[b * io.pitch + q * io.s];
}

// What runs between import and export on the device.
enum MpMode { kComplex = 0, kR2C = 1, kC2R = 2 };

static int mp_pack_impl(const mpfft_mp_plan *P, unsigned long batch, const IoShape &io, mpfr_t *inr, mpfr_t *ini,
                        uint32_t *planes, long *exps) {
  const unsigned long N = io.n;
  const int L = P->L;
  // block exponents and finiteness
  std::vector<int> bad(batch, 0);
  parallel_for((long)batch, 1, [&](long b0, long b1) {
    for (long b = b0; b < b1; ++b) {
      long e_s = LONG_MIN;
      for (unsigned long p = 0; p < N; ++p) {
        for (int c = 0; c < 2; ++c) {
          mpfr_srcptr x = elem(c ? ini : inr, c, b, io, p);
          if (!mpfr_number_p(x)) bad[b] = 1;
          else if (!mpfr_zero_p(x) && x->_mpfr_exp > e_s) e_s = x->_mpfr_exp;
        }
      }
      exps[b] = e_s == LONG_MIN ? 0 : e_s;
    }
  });
  for (unsigned long b = 0; b < batch; ++b)
    if (bad[b]) return set_err(MPFFT_ENONFINITE, "input signal %lu holds NaN or infinity", b);
  const size_t plane = (size_t)N * batch;
  parallel_for((long)(N * batch), 256, [&](long a0, long a1) {
    uint32_t tmp[kMaxLimbsBig + 2];
    for (long t = a0; t < a1; ++t) {
      const unsigned long p = t / batch, b = t % batch;
      for (int c = 0; c < 2; ++c) {
        uint32_t sg = mpfr_to_fixed(elem(c ? ini : inr, c, b, io, p), L, P->F, exps[b], tmp);
        if (sg) {  // two's complement
          uint32_t cy = 1;
          for (int i = 0; i < L; ++i) {
            uint64_t v = (uint64_t)(uint32_t)~tmp[i] + cy;
            tmp[i] = (uint32_t)v;
            cy = (uint32_t)(v >> 32);
          }
        }
        uint32_t *dst = planes + (size_t)c * L * plane + (size_t)p * batch + b;
        for (int i = 0; i < L; ++i) dst[(size_t)i * plane] = tmp[i];
      }
    }
  });
  return MPFFT_OK;
}

// fadj: the value of fixed-point integer A is A * 2^(exps[b] - F - fadj)
static void mp_unpack_impl(const mpfft_mp_plan *P, unsigned long batch, const uint32_t *planes, const long *exps,
                           const IoShape &io, mpfr_t *outr, mpfr_t *outi, long fadj) {
  const unsigned long N = io.n;
  const int L = P->L;
  const size_t plane = (size_t)N * batch;
  parallel_for((long)(N * batch), 256, [&](long a0, long a1) {
    uint32_t tmp[kMaxLimbsBig + 2];
    for (long t = a0; t < a1; ++t) {
      const unsigned long p = t / batch, b = t % batch;
      for (int c = 0; c < 2; ++c) {
        const uint32_t *src = planes + (size_t)c * L * plane + (size_t)p * batch + b;
        for (int i = 0; i < L; ++i) tmp[i] = src[(size_t)i * plane];
        fixed_to_mpfr(tmp, L, exps[b] - P->F - fadj, elem(c ? outi : outr, c, b, io, p));
      }
    }
  });
}

static void mp_fill_nan(mpfr_t *a, unsigned long n) {
  if (!a) return;
  for (unsigned long k = 0; k < n; ++k) mpfr_set_nan(a[k]);
}

// streaming/tensor-kernel scratch words of one transform of B signals (0 when unused)
static size_t mp_plan_big_words(const mpfft_mp_plan *p, unsigned long B) {
  const MpDeviceTables &T0 = p->rank > 1 ? p->axis[0]->tabs : p->tabs;
  if (p->L <= kMaxLimbs && !mp_tc_used(T0, p->L)) return 0;
  if (p->rank == 1) return mp_big_scratch_words(p->tabs, p->L, (int)B);
  size_t w = 0;
  for (int s = 0; s < p->rank; ++s)
    w = std::max(w, mp_big_scratch_words(p->axis[s]->tabs, p->L, (int)(B * (p->N / p->dims[s]))));
  return w;
}

// The plan's complex transform on device limb planes, any rank.  Rank > 1:
// per axis, last first: rotate that axis to the front (transposition of
// [N/d][d] elements of B words per limb plane, into tmp), then a batched
// one-dimensional transform of length d over the other N/d points x B
// signals (tmp -> out).  After the last round the planes are in natural
// order again.  tmp: 2*L*N*B words.
static cudaError_t mp_transform(const mpfft_mp_plan *p, const uint32_t *in, uint32_t *out, int B, cudaStream_t st,
                                uint32_t *big, uint32_t *tmp, float *launch_ms = nullptr) {
  if (p->rank == 1) return mp_run_transform(p->L, p->tabs, in, out, B, st, launch_ms, big);
  const uint32_t *src = in;
  for (int s = p->rank - 1; s >= 0; --s) {
    const long long d = (long long)p->dims[s], R = (long long)p->N / d;
    cudaError_t e = transpose_launch(src, tmp, 2LL * p->L, R, d, B, st);
    if (e != cudaSuccess) return e;
    if ((e = mp_run_transform(p->L, p->axis[s]->tabs, tmp, out, (int)(B * R), st, nullptr, big)) != cudaSuccess)
      return e;
    src = out;
  }
  return cudaSuccess;
}

// Raw MPFR fields of n components with nl significand limbs each, packed in
// one buffer: limbs [n][nl], then exponents [n], then sign bytes [n].  The
// same view of a pinned host block and of a device block makes each
// direction of a chunk one copy of `bytes`.
struct StageView {
  uint64_t *m;
  int64_t *e;
  uint8_t *s;
  size_t bytes;
};
static inline size_t stage_bytes(size_t n, int nl) { return n * ((size_t)nl * 8 + 8 + 1); }
static inline StageView stage_view(uint64_t *base, size_t n, int nl) {
  int64_t *e = reinterpret_cast<int64_t *>(base + n * (size_t)nl);
  return StageView{base, e, reinterpret_cast<uint8_t *>(e + n), stage_bytes(n, nl)};
}

using ConvSlotRef = mpfft_mp_plan::ConvSlot &;

static int mp_conv_reserve(mpfft_mp_plan *p, unsigned long chunk, int nli, int nlo) {
  if (chunk <= p->cv_chunk && nli <= p->cv_nli && nlo <= p->cv_nlo) return MPFFT_OK;
  p->free_conv();
  const size_t comp = (size_t)2 * p->pts_max() * chunk;
  const size_t words = (size_t)2 * p->L * p->pts_max() * chunk;
  bool ok = true;
  auto dm = [&](void **q, size_t bytes) { ok = ok && dev_alloc(q, bytes) == cudaSuccess; };
  auto hm = [&](void **q, size_t bytes) { ok = ok && host_alloc(q, bytes) == cudaSuccess; };
  for (auto &c : p->cv) {
    ok = ok && cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) == cudaSuccess;
    dm((void **)&c.d_in, words * 4);
    dm((void **)&c.d_out, words * 4);
    dm((void **)&c.d_i, stage_bytes(comp, nli));
    hm((void **)&c.h_i, stage_bytes(comp, nli));
    dm((void **)&c.d_o, stage_bytes(comp, nlo));
    hm((void **)&c.h_o, stage_bytes(comp, nlo));
    dm((void **)&c.d_es, chunk * 8);
    if (const size_t bw = mp_plan_big_words(p, chunk)) dm((void **)&c.d_big, bw * 4);
    if (p->rank > 1) dm((void **)&c.d_tmp, words * 4);
  }
  if (!ok) {
    cudaGetLastError();
    p->free_conv();
    return set_err(MPFFT_ENOMEM, "cannot allocate conversion staging for %lu-signal chunks", chunk);
  }
  p->cv_chunk = chunk;
  p->cv_nli = nli;
  p->cv_nlo = nlo;
  return MPFFT_OK;
}

static inline int nlimbs64(long prec) { return (int)((prec + 63) / 64); }

// Device work between import and export.  a holds the imported input; the
// result ends in *res (a or b).  complex: transform a -> b.  R2C: transform
// a -> b, split b -> a (half spectrum, value 2X).  C2R: split a -> b (2Z with
// planes exchanged), transform b -> a (planes exchanged: the inverse).
static cudaError_t mp_device_pipeline(const mpfft_mp_plan *p, int mode, uint32_t *a, uint32_t *b, int B,
                                      cudaStream_t st, uint32_t *big, uint32_t *tmp, uint32_t **res) {
  cudaError_t e = cudaSuccess;
  if (mode == kComplex) {
    *res = b;
    return mp_transform(p, a, b, B, st, big, tmp);
  }
  *res = a;
  if (mode == kR2C) {
    if ((e = mp_run_transform(p->L, p->tabs, a, b, B, st, nullptr, big)) != cudaSuccess) return e;
    return mp_real_split(true, p->L, b, a, (int)p->N, B, p->tabs.tw, p->tabs.dneg, st);
  }
  if ((e = mp_real_split(false, p->L, a, b, (int)p->N, B, p->tabs.tw, p->tabs.dneg, st)) != cudaSuccess) return e;
  return mp_run_transform(p->L, p->tabs, b, a, B, st, nullptr, big);
}

// Signals whose inputs share one limb count and whose outputs share one
// precision (those of signal 0): the conversion runs on the GPU and the host
// only moves raw significand limbs.  The batch is processed in chunks through
// two slots (stream + staging each): while the GPU copies and transforms chunk
// i, the host scatters chunk i-1's results and gathers chunk i+1's inputs.
// The precisions are checked chunk by chunk as the pipeline reaches them (the
// inputs' inside the gather, which reads the same mpfr_t fields anyway; the
// outputs' just before it), not in a separate pass over the whole batch.  At
// the first chunk that holds a different precision the pipeline drains and
// stops: *done = the number of leading signals it completed, all of them with
// their outputs written; the caller converts the rest on the host.
// fadj: output value = A * 2^(e_s - F - fadj).
static int mp_execute_gpuconv(mpfft_mp_plan *p, unsigned long batch, int mode, const IoShape &ii, mpfr_t *inr,
                              mpfr_t *ini, const IoShape &oo, mpfr_t *outr, mpfr_t *outi, long fadj,
                              unsigned long *done) {
  *done = 0;
  const unsigned long Ni = ii.n, No = oo.n;
  const long prec_out = mpfr_get_prec(elem(outr, 0, 0, oo, 0));
  const int nli = nlimbs64(mpfr_get_prec(elem(inr, 0, 0, ii, 0))), nlo = nlimbs64(prec_out);
  // chunks of up to 256 signals (a multiple of 32 keeps every warp on one
  // butterfly), and at most ~256 MiB of staging per slot
  const size_t per_signal = (size_t)2 * p->pts_max() * ((nli + nlo) * 8 + 2 * 4 * p->L + 18);
  unsigned long chunk = std::min<unsigned long>(256, std::max<size_t>(32, (256UL << 20) / per_signal));
  chunk = std::min<unsigned long>(chunk, (unsigned long)INT32_MAX / p->pts_max());  // batch x points fits an int
  if (chunk >= 32) chunk &= ~31UL;
  chunk = std::min(chunk, batch);
  if (int e = mp_conv_reserve(p, chunk, nli, nlo)) return e;
  const unsigned long nchunks = (batch + chunk - 1) / chunk;
  const long emin = mpfr_get_emin(), emax = mpfr_get_emax();
  std::vector<int> nonfin(nchunks, 0), mixed(nchunks, 0);

  // outputs of chunk ci all at prec_out (checked before any input of the chunk
  // is staged, so a chunk is either converted whole here or not at all)
  auto outputs_uniform = [&](unsigned long ci) {
    const unsigned long b0 = ci * chunk, cb = std::min(chunk, batch - b0);
    std::atomic<int> bad{0};
    parallel_for((long)(2 * cb * No), 4096, [&](long x0, long x1) {
      for (long u = x0; u < x1; ++u) {
        const long bb = u / (2 * (long)No), part = (u / (long)No) & 1;
        if (elem(part ? outi : outr, (int)part, b0 + bb, oo, (unsigned long)(u % (long)No))->_mpfr_prec != prec_out) {
          bad.store(1, std::memory_order_relaxed);
          return;
        }
      }
    });
    return bad.load() == 0;
  };
  // staging is signal-major: component u = (signal*2 + part)*Ni + q, the order
  // the host walks the mpfr_t arrays in, so both sides stream.  An input with
  // another limb count marks the chunk mixed; its significand is not read.
  auto gather = [&](unsigned long ci) {
    auto &c = p->cv[ci & 1];
    const unsigned long b0 = ci * chunk, cb = std::min(chunk, batch - b0);
    const StageView hv = stage_view(c.h_i, (size_t)2 * Ni * cb, nli);
    parallel_for((long)(2 * cb * Ni), 2048, [&](long x0, long x1) {
      constexpr long kAhead = 8;  // significands prefetched ahead of use
      auto at = [&](long u) {
        const long bb = u / (2 * (long)Ni), part = (u / (long)Ni) & 1;
        return elem(part ? ini : inr, (int)part, b0 + bb, ii, (unsigned long)(u % (long)Ni));
      };
      for (long u = x0; u < std::min(x1, x0 + kAhead); ++u) __builtin_prefetch(at(u)->_mpfr_d);
      for (long u = x0; u < x1; ++u) {
        if (u + kAhead < x1) {
          const mp_limb_t *d = at(u + kAhead)->_mpfr_d;
          __builtin_prefetch(d);
          __builtin_prefetch(d + nli - 1);
        }
        mpfr_srcptr x = at(u);
        if (nlimbs64(x->_mpfr_prec) != nli) {
          mixed[ci] = 1;
          break;
        }
        if (x->_mpfr_exp <= LONG_MIN + 3) {  // MPFR's reserved exponents: zero, NaN, infinity
          if (!mpfr_zero_p(x)) nonfin[ci] = 1;
          stage_word(hv.e + u, INT64_MIN);
          hv.s[u] = 0;
          memset(hv.m + u * nli, 0, nli * 8);
        } else {
          stage_word(hv.e + u, x->_mpfr_exp);
          hv.s[u] = x->_mpfr_sign < 0;
          stage_limbs(hv.m + u * nli, reinterpret_cast<const uint64_t *>(x->_mpfr_d), nli);
        }
      }
      stage_fence();
    });
  };
  // copy in, import, transform, export, copy out: one chunk on its slot's stream
  auto enqueue = [&](ConvSlotRef c, unsigned long cb) -> int {
    const size_t ci_n = (size_t)2 * Ni * cb, co_n = (size_t)2 * No * cb;
    const StageView di = stage_view(c.d_i, ci_n, nli), dout = stage_view(c.d_o, co_n, nlo);
    CUDA_TRY(cudaMemcpyAsync(c.d_i, c.h_i, di.bytes, cudaMemcpyHostToDevice, c.st));
    CUDA_TRY(mp_import_launch(di.m, di.e, di.s, nli, (int)Ni, (int)cb, p->L, p->F, c.d_es, c.d_in, c.st,
                              true));
    uint32_t *res = nullptr;
    CUDA_TRY(mp_device_pipeline(p, mode, c.d_in, c.d_out, (int)cb, c.st, c.d_big, c.d_tmp, &res));
    CUDA_TRY(mp_export_launch(res, (int)No, (int)cb, p->L, c.d_es, p->F + fadj, prec_out, nlo, dout.m, dout.e,
                              dout.s, c.st, true));
    CUDA_TRY(cudaMemcpyAsync(c.h_o, c.d_o, dout.bytes, cudaMemcpyDeviceToHost, c.st));
    return MPFFT_OK;
  };
  // Integer-pipe plans replay a chunk shape from a CUDA graph from its second
  // use on (one launch instead of a dozen; the first use runs directly so that
  // nothing is initialised inside a capture).  A capture that fails leaves
  // the shape on direct launches.
  const bool graphable = p->L <= kMaxLimbs && !mp_tc_used(p->tabs, p->L);
  auto launch = [&](unsigned long ci) -> int {
    auto &c = p->cv[ci & 1];
    const unsigned long b0 = ci * chunk, cb = std::min(chunk, batch - b0);
    if (graphable) {
      const std::vector<long> key{(long)cb, nli, nlo, mode, fadj, prec_out, (long)Ni, (long)No};
      auto it = c.graphs.find(key);
      if (it == c.graphs.end() && c.uses[key]++ >= 1) {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        if (cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
          const int e = enqueue(c, cb);
          const cudaError_t ce = cudaStreamEndCapture(c.st, &g);
          if (e != MPFFT_OK || ce != cudaSuccess || !g || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess)
            ge = nullptr;
          if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        it = c.graphs.emplace(key, ge).first;
      }
      if (it != c.graphs.end() && it->second) {
        CUDA_TRY(cudaGraphLaunch(it->second, c.st));
        CUDA_TRY(cudaEventRecord(c.done, c.st));
        return MPFFT_OK;
      }
    }
    if (int e = enqueue(c, cb)) return e;
    CUDA_TRY(cudaEventRecord(c.done, c.st));
    return MPFFT_OK;
  };
  auto scatter = [&](unsigned long ci) -> int {
    auto &c = p->cv[ci & 1];
    CUDA_TRY(cudaEventSynchronize(c.done));
    const unsigned long b0 = ci * chunk, cb = std::min(chunk, batch - b0);
    const StageView ho = stage_view(c.h_o, (size_t)2 * No * cb, nlo);
    parallel_for((long)(2 * cb * No), 2048, [&](long x0, long x1) {
      constexpr long kAhead = 8;  // destination significands prefetched ahead of use
      auto at = [&](long u) {
        const long bb = u / (2 * (long)No), part = (u / (long)No) & 1;
        return elem(part ? outi : outr, (int)part, b0 + bb, oo, (unsigned long)(u % (long)No));
      };
      for (long u = x0; u < std::min(x1, x0 + kAhead); ++u) __builtin_prefetch(at(u)->_mpfr_d, 1);
      for (long u = x0; u < x1; ++u) {
        if (u + kAhead < x1) {
          const mp_limb_t *d = at(u + kAhead)->_mpfr_d;
          __builtin_prefetch(d, 1);
          __builtin_prefetch(d + nlo - 1, 1);
        }
        mpfr_ptr y = at(u);
        const size_t t = (size_t)u;  // signal-major staging
        const int64_t e = ho.e[t];
        if (e == INT64_MIN) {
          mpfr_set_zero(y, 1);
        } else if (e >= emin && e <= emax) {
          memcpy(y->_mpfr_d, ho.m + t * nlo, nlo * 8);
          y->_mpfr_exp = e;
          y->_mpfr_sign = ho.s[t] ? -1 : 1;
        } else {  // outside the current exponent range: let MPFR overflow/underflow
          __mpz_struct z;
          z._mp_alloc = nlo;
          z._mp_size = ho.s[t] ? -nlo : nlo;
          z._mp_d = reinterpret_cast<mp_limb_t *>(ho.m + t * nlo);
          mpfr_set_z_2exp(y, &z, e - 64L * nlo, MPFR_RNDN);
        }
      }
    });
    return MPFFT_OK;
  };

  // chunks [0, scattered) have their outputs written
  unsigned long scattered = 0;
  auto drain = [&](unsigned long upto) -> int {
    for (; scattered < upto; ++scattered)
      if (int e = scatter(scattered)) return e;
    return MPFFT_OK;
  };
  int err = MPFFT_OK;
  unsigned long ci = 0;
  for (; ci < nchunks; ++ci) {
    if (ci >= 2 && (err = drain(ci - 1))) return err;  // chunk ci-2: frees slot ci&1
    if (!outputs_uniform(ci)) break;
    gather(ci);
    if (mixed[ci]) break;
    if (nonfin[ci]) {  // chunk 0: before any output is written
      cudaStreamSynchronize(p->cv[0].st);
      cudaStreamSynchronize(p->cv[1].st);
      return set_err(MPFFT_ENONFINITE, "input holds NaN or infinity");
    }
    if ((err = launch(ci))) return err;
  }
  if ((err = drain(ci))) return err;
  *done = std::min(batch, ci * chunk);
  return set_err(MPFFT_OK, "");
}

// streaming-kernel scratch for a batch (large limb counts only); null otherwise
static int mp_big_reserve(mpfft_mp_plan *p, unsigned long batch, uint32_t **out) {
  *out = nullptr;
  const size_t words = mp_plan_big_words(p, batch);
  if (words == 0) return MPFFT_OK;
  if (words > p->big_words) {
    if (p->d_big) cudaFree(p->d_big);
    p->d_big = nullptr;
    p->big_words = 0;
    if (dev_alloc((void **)&p->d_big, words * 4) != cudaSuccess) {
      cudaGetLastError();
      return set_err(MPFFT_ENOMEM, "cannot allocate %zu bytes of scratch", words * 4);
    }
    p->big_words = words;
  }
  *out = p->d_big;
  return MPFFT_OK;
}

// transposition buffer of a multi-dimensional plan for a batch; null for rank 1
static int mp_tmp_reserve(mpfft_mp_plan *p, unsigned long batch, uint32_t **out) {
  *out = nullptr;
  if (p->rank == 1) return MPFFT_OK;
  const size_t words = (size_t)2 * p->L * p->N * batch;
  if (words > p->tmp_words) {
    if (p->d_tmp) cudaFree(p->d_tmp);
    p->d_tmp = nullptr;
    p->tmp_words = 0;
    if (dev_alloc((void **)&p->d_tmp, words * 4) != cudaSuccess) {
      cudaGetLastError();
      return set_err(MPFFT_ENOMEM, "cannot allocate %zu bytes of transposition scratch", words * 4);
    }
    p->tmp_words = words;
  }
  *out = p->d_tmp;
  return MPFFT_OK;
}

// after a synchronous execution: a tensor-core wait that expired voids the results
static int mp_tc_check(const mpfft_mp_plan *p, int rc) {
  const MpDeviceTables &T = p->rank > 1 ? p->axis[0]->tabs : p->tabs;
  if (rc != MPFFT_OK || !mp_tc_used(T, p->L)) return rc;
  int code = 0;
  CUDA_TRY(mp_tc_take_error(&code));
  if (code) return set_err(MPFFT_ECUDA, "a tensor-core wait expired (code %d)", code);
  return rc;
}

static int mp_execute_hostconv(mpfft_mp_plan *p, unsigned long batch, int mode, const IoShape &ii, mpfr_t *inr,
                               mpfr_t *ini, const IoShape &oo, mpfr_t *outr, mpfr_t *outi, long fadj);
constexpr int kFloatOutOfRange = -1;
static int mp_execute_float(mpfft_mp_plan *p, unsigned long batch, const IoShape &ii, mpfr_t *inr, mpfr_t *ini,
                            const IoShape &oo, mpfr_t *outr, mpfr_t *outi, long fadj);

static int mp_execute_impl(mpfft_mp_plan *p, unsigned long batch, int mode, const IoShape &ii, mpfr_t *inr,
                           mpfr_t *ini, const IoShape &oo, mpfr_t *outr, mpfr_t *outi, long fadj) {
  if (p->host_only) return set_err(MPFFT_EINVAL, "plan was created host-only (conversion only)");
  std::lock_guard<std::mutex> g(p->mu);
  if (p->fplan && mode == kComplex) {
    const int r = mp_execute_float(p, batch, ii, inr, ini, oo, outr, outi, fadj);
    if (r != kFloatOutOfRange) return r;
  }
  if (!p->force_host_conversion) {
    unsigned long done = 0;
    const int r = mp_execute_gpuconv(p, batch, mode, ii, inr, ini, oo, outr, outi, fadj, &done);
    if (r != MPFFT_OK || done == batch) return mp_tc_check(p, r);
    if (done > 0) {  // signals [done, batch): the same arrays seen from signal `done` on
      IoShape ri = ii, ro = oo;
      for (int c = 0; c < 2; ++c) {
        if (ri.base[c]) ri.base[c] += done;
        if (ro.base[c]) ro.base[c] += done;
      }
      mpfr_t *r_inr = ii.base[0] ? inr : inr + done * ii.pitch, *r_ini = ii.base[1] ? ini : ini + done * ii.pitch;
      mpfr_t *r_outr = oo.base[0] ? outr : outr + done * oo.pitch;
      mpfr_t *r_outi = oo.base[1] ? outi : outi + done * oo.pitch;
      return mp_execute_hostconv(p, batch - done, mode, ri, r_inr, r_ini, ro, r_outr, r_outi, fadj);
    }
  }
  return mp_execute_hostconv(p, batch, mode, ii, inr, ini, oo, outr, outi, fadj);
}

// Host conversion (mpfr_t <-> limb planes on the CPU) of a whole batch; any mix
// of precisions.  The caller holds the plan's lock.
static int mp_execute_hostconv(mpfft_mp_plan *p, unsigned long batch, int mode, const IoShape &ii, mpfr_t *inr,
                               mpfr_t *ini, const IoShape &oo, mpfr_t *outr, mpfr_t *outi, long fadj) {
  if ((unsigned long long)batch * p->pts_max() > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large for host conversion");
  if (int e = mp_reserve(p, batch)) return e;
  p->exps.assign(batch, 0);
  if (int e = mp_pack_impl(p, batch, ii, inr, ini, p->h_in, p->exps.data())) return e;
  uint32_t *big = nullptr, *tmp = nullptr;
  if (int e = mp_big_reserve(p, batch, &big)) return e;
  if (int e = mp_tmp_reserve(p, batch, &tmp)) return e;
  if (big || tmp)
    if (int e = scratch_wait(p, p->stream)) return e;
  uint32_t *res = nullptr;
  CUDA_TRY(cudaMemcpyAsync(p->d_in, p->h_in, (size_t)2 * p->L * ii.n * batch * 4, cudaMemcpyHostToDevice,
                           p->stream));
  CUDA_TRY(mp_device_pipeline(p, mode, p->d_in, p->d_out, (int)batch, p->stream, big, tmp, &res));
  if (big || tmp)
    if (int e = scratch_record(p, p->stream)) return e;
  CUDA_TRY(cudaMemcpyAsync(p->h_out, res, (size_t)2 * p->L * oo.n * batch * 4, cudaMemcpyDeviceToHost, p->stream));
  CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (int e = mp_tc_check(p, MPFFT_OK)) return e;
  mp_unpack_impl(p, batch, p->h_out, p->exps.data(), oo, outr, outi, fadj);
  return set_err(MPFFT_OK, "");
}

// complex transform of strided host arrays (input stride s, contiguous output)
static int mp_execute_complex(mpfft_mp_plan *p, unsigned long batch, mpfr_t *inr, mpfr_t *ini, unsigned long s,
                              mpfr_t *outr, mpfr_t *outi, unsigned flags) {
  const long shift = (flags & MPFFT_SCALED) ? ilog2(p->N) : 0;
  return mp_execute_impl(p, batch, kComplex, io_signals(p->N, s), inr, ini, io_signals(p->N, 1), outr, outi, shift);
}

static long mp_call_prec(mpfr_t *inr, mpfr_t *ini, mpfr_t *outr, mpfr_t *outi) {
  long P = mpfr_get_prec(outr[0]);
  P = std::max<long>(P, mpfr_get_prec(outi[0]));
  P = std::max<long>(P, mpfr_get_prec(inr[0]));
  P = std::max<long>(P, mpfr_get_prec(ini[0]));
  return P;
}

static void mp_dropin(unsigned long n, unsigned long s, long sn, mpfr_t *inr, mpfr_t *ini, mpfr_t *outr,
                      mpfr_t *outi, unsigned flags) {
  if (!inr || !ini || !outr || !outi) {
    set_err(MPFFT_EINVAL, "NULL array");
    return;
  }
  if (flags & MPFFT_INVERSE) {  // ifft(X) = swap(FFT(swap(X))) (times 1/n if scaled)
    std::swap(inr, ini);
    std::swap(outr, outi);
    flags &= ~MPFFT_INVERSE;
  }
  int e = MPFFT_OK;
  if (!is_pow2(n)) e = set_err(MPFFT_EINVAL, "n=%lu is not a power of two", n);
  else if (s == 0) e = set_err(MPFFT_EINVAL, "stride s must be >= 1");
  else if (sn < 0)
    e = set_err(MPFFT_EINVAL, "sn=%ld < 0 addresses the reference's global array; only top-level calls (sn >= 0)", sn);
  if (e == MPFFT_OK) {
    mpfft_mp_plan *p = mp_cached(n, mp_call_prec(inr, ini, outr, outi));
    if (!p) e = g_err;
    else e = mp_execute_complex(p, 1, inr, ini, s, outr, outi, flags);
  }
  if (e != MPFFT_OK) {
    mp_fill_nan(outr, n);
    mp_fill_nan(outi, n);
  }
}

// ---------------------------------------------------------------------------
// FP64 plans
// ---------------------------------------------------------------------------
template <typename T>
static int upload(mpfft_d_plan *p, const std::vector<T> &v, const T **out) {
  T *d = nullptr;
  const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
  CUDA_TRY(cudaMalloc(&d, bytes));
  p->dev_allocs.push_back(d);
  if (!v.empty()) CUDA_TRY(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = d;
  return MPFFT_OK;
}

// Schedule of a shared-memory sub-transform of `size` points: the leaves and
// levels of its own recursion tree, and the DIT input order perm[m].
static int build_sub(mpfft_d_plan *p, int size, SubSchedule &S, int leaf_max = 16) {
  HostTree t;
  walk(t, size, 1, 0, 0, leaf_max);
  // invperm[j] = DIT position of element j of the sub-transform's input sequence
  std::vector<int> perm(size);
  for (const Leaf &lf : t.leaves)
    for (int j = 0; j < lf.n; ++j) perm[(j == 0 && lf.sn < 0) ? lf.sn + size : lf.sn + j * lf.s] = lf.out + j;
  std::vector<int> nodes;
  std::stable_sort(t.leaves.begin(), t.leaves.end(), [](const Leaf &a, const Leaf &b) { return a.n > b.n; });
  S.size = size;
  S.nleaves = (int)t.leaves.size();
  S.nleaf16 = (int)std::count_if(t.leaves.begin(), t.leaves.end(), [](const Leaf &l) { return l.n == 16; });
  S.nleaf8 = (int)std::count_if(t.leaves.begin(), t.leaves.end(), [](const Leaf &l) { return l.n == 8; });
  S.nlevels = 0;
  for (auto &kv : t.levels) {
    if (S.nlevels >= kMaxLevels) return set_err(MPFFT_EUNSUPPORTED, "sub-transform too large");
    S.level_n[S.nlevels] = kv.first;
    S.level_start[S.nlevels] = (int)nodes.size();
    S.level_count[S.nlevels] = (int)kv.second.size();
    nodes.insert(nodes.end(), kv.second.begin(), kv.second.end());
    ++S.nlevels;
  }
  // per level: its nodes that are not the first child of a node of the next
  // level (a first child starts at its parent's offset)
  std::vector<int> pair_nodes;
  for (int l = 0; l + 1 < S.nlevels; ++l) {
    const int *up = nodes.data() + S.level_start[l + 1];
    std::set<int> parents(up, up + S.level_count[l + 1]);
    S.pair_start[l] = (int)pair_nodes.size();
    for (int j = 0; j < S.level_count[l]; ++j) {
      const int o = nodes[S.level_start[l] + j];
      if (!parents.count(o)) pair_nodes.push_back(o);
    }
    S.pair_count[l] = (int)pair_nodes.size() - S.pair_start[l];
  }
  if (int e = upload(p, perm, &S.perm)) return e;
  if (int e = upload(p, t.leaves, &S.leaves)) return e;
  if (int e = upload(p, nodes, &S.node_off)) return e;
  if (int e = upload(p, pair_nodes, &S.pair_nodes)) return e;
  return MPFFT_OK;
}

// sub_max: largest shared-memory sub-transform (0: the default kDSubMax; the
// results do not depend on it, only where each butterfly runs)
static int d_plan_init(mpfft_d_plan *p, unsigned long n, int sub_max) {
  if (!is_pow2(n)) return set_err(MPFFT_EINVAL, "n=%lu is not a power of two", n);
  if (n > (1UL << 28)) return set_err(MPFFT_EUNSUPPORTED, "n=%lu too large", n);
  if (int e = device_ready()) return e;
  p->N = n;
  p->tabs.N = (int)n;
  // cut the tree at T points: maximal nodes of size <= T run in shared memory
  const int T = (int)std::min<unsigned long>(n, sub_max > 0 ? sub_max : kDSubMax);
  {
    HostTree t;
    walk(t, (int)n, 1, 0, 0, T);
    std::vector<SubRoot> roots;
    for (const Leaf &lf : t.leaves) roots.push_back(SubRoot{lf.sn, lf.s, lf.out, lf.n});
    p->tabs.nroots = (int)roots.size();
    if (int e = upload(p, roots, &p->tabs.roots)) return e;
    if (int e = build_tree(p->upper, n, T)) return e;  // its levels are the ones above T
    p->tabs.upper = p->upper.tabs;
  }
  if (int e = build_sub(p, T, p->tabs.sub[0])) return e;
  if (T >= 2) {
    if (int e = build_sub(p, T / 2, p->tabs.sub[1])) return e;
  } else {
    p->tabs.sub[1] = p->tabs.sub[0];
  }
  // twiddles exactly as the reference lut() (serial_d_fft6.c:52-62)
  const unsigned long q = n / 4;
  std::vector<double> wr(q ? q : 1), wi(q ? q : 1);
  for (unsigned long k = 0; k < q; ++k) {
    wr[k] = cos(2. * M_PI * k / n);
    wi[k] = sin(2. * M_PI * k / n);
  }
  CUDA_TRY(cudaMalloc(&p->d_wr, wr.size() * sizeof(double)));
  CUDA_TRY(cudaMalloc(&p->d_wi, wi.size() * sizeof(double)));
  CUDA_TRY(cudaMemcpy(p->d_wr, wr.data(), wr.size() * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(p->d_wi, wi.data(), wi.size() * sizeof(double), cudaMemcpyHostToDevice));
  p->tabs.wr = p->d_wr;
  p->tabs.wi = p->d_wi;
  p->tabs.c8 = cos(2. * M_PI * 1 / 8);
  p->tabs.c16a = cos(2. * M_PI * 1 / 16);
  p->tabs.c16b = cos(2. * M_PI * 1 / 16) - cos(2. * M_PI * 3 / 16);
  p->tabs.c16c = cos(2. * M_PI * 3 / 16);
  p->tabs.c16d = cos(2. * M_PI * 1 / 16) + cos(2. * M_PI * 3 / 16);
  CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  return MPFFT_OK;
}

static mpfft_d_plan *d_cached(unsigned long n) {
  std::lock_guard<std::mutex> g(g_cache_mu);
  auto it = g_d_cache.find(n);
  if (it != g_d_cache.end()) return it->second.get();
  std::unique_ptr<mpfft_d_plan> p(new mpfft_d_plan);
  if (d_plan_init(p.get(), n) != MPFFT_OK) return nullptr;
  auto *raw = p.get();
  g_d_cache[n] = std::move(p);
  return raw;
}

// words per real component and bytes per word of a plan's device layout
static int d_words(const mpfft_d_plan *p) { return p->tier < 0 ? 1 : tier_words(p->tier); }
static size_t d_word_bytes(const mpfft_d_plan *p) { return p->tier < 0 ? 8 : tier_word_bytes(p->tier); }

static int d_reserve(mpfft_d_plan *p, unsigned long batch) {
  // in doubles (float-float words take half a double each)
  const size_t words =
      ((size_t)2 * d_words(p) * (p->real ? p->N + 1 : p->N) * batch * d_word_bytes(p) + 7) / 8;
  if (words <= p->cap) return MPFFT_OK;
  if (p->d_in) cudaFree(p->d_in);
  if (p->d_out) cudaFree(p->d_out);
  if (p->h_in) cudaFreeHost(p->h_in);
  if (p->h_out) cudaFreeHost(p->h_out);
  p->d_in = p->d_out = p->h_in = p->h_out = nullptr;
  p->cap = 0;
  if (dev_alloc((void **)&p->d_in, words * 8) != cudaSuccess || dev_alloc((void **)&p->d_out, words * 8) != cudaSuccess ||
      host_alloc((void **)&p->h_in, words * 8) != cudaSuccess || host_alloc((void **)&p->h_out, words * 8) != cudaSuccess) {
    cudaGetLastError();
    return set_err(MPFFT_ENOMEM, "cannot allocate %zu-byte staging buffers", words * 8);
  }
  p->cap = words;
  return MPFFT_OK;
}

static double d_scale(const mpfft_d_plan *p, unsigned flags) {
  return (flags & MPFFT_SCALED) ? 1.0 / (double)p->N : 1.0;
}

static int d_plan_init_nd(mpfft_d_plan *p, int rank, const unsigned long *dims) {
  if (rank < 1 || rank > 3 || !dims) return set_err(MPFFT_EINVAL, "rank must be 1, 2 or 3");
  unsigned long n = 1;
  for (int i = 0; i < rank; ++i) {
    if (!is_pow2(dims[i])) return set_err(MPFFT_EINVAL, "dims[%d]=%lu is not a power of two", i, dims[i]);
    if (dims[i] > (1UL << 28) || n > (1UL << 28) / dims[i])
      return set_err(MPFFT_EUNSUPPORTED, "more than 2^28 points in total");
    n *= dims[i];
  }
  if (rank == 1) return d_plan_init(p, n);
  if (int e = device_ready()) return e;
  p->N = n;
  p->rank = rank;
  for (int i = 0; i < rank; ++i) {
    p->dims[i] = dims[i];
    p->axis[i].reset(new (std::nothrow) mpfft_d_plan);
    if (!p->axis[i]) return set_err(MPFFT_ENOMEM, "out of host memory");
    if (int e = d_plan_init(p->axis[i].get(), dims[i])) return e;
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  return MPFFT_OK;
}

// The plan's transform in the FP64 layout [c][b][p], any rank.  Rank > 1: per
// axis, last first: a batched one-dimensional transform along the innermost
// axis (in -> tmp; the other points are more signals), then a transposition
// of each component of each signal, [N/d][d] -> [d][N/d] (tmp -> out), which
// brings the next axis innermost; after the last round the points are in
// natural order again.  Every one-dimensional transform is the reference's
// (bit-identical), so the result equals the axis-by-axis application of
// d_sr24_cp_fft in this order.  Scaling by 1/d per axis is exact.
static cudaError_t d_transform(mpfft_d_plan *p, const double *in, double *out, int B, unsigned flags,
                               cudaStream_t st, double *tmp) {
  // MPFFT_INVERSE: the first launch reads the planes exchanged, the last writes
  // them exchanged (transpositions keep planes apart), i.e. swap(FFT(swap(x)))
  const bool inv = (flags & MPFFT_INVERSE) != 0;
  if (p->rank == 1) return d_run_transform(p->tabs, in, out, B, d_scale(p, flags), st, inv, inv);
  const double *src = in;
  for (int s = p->rank - 1; s >= 0; --s) {
    const long long d = (long long)p->dims[s], R = (long long)p->N / d;
    const double sc = (flags & MPFFT_SCALED) ? 1.0 / (double)d : 1.0;
    cudaError_t e = d_run_transform(p->axis[s]->tabs, src, tmp, (int)(B * R), sc, st, inv && s == p->rank - 1,
                                    inv && s == 0);
    if (e != cudaSuccess) return e;
    e = transpose_launch(reinterpret_cast<const uint32_t *>(tmp), reinterpret_cast<uint32_t *>(out), 2LL * B, R, d, 2,
                         st);
    if (e != cudaSuccess) return e;
    src = out;
  }
  return cudaSuccess;
}

static int d_tmp_reserve(mpfft_d_plan *p, unsigned long batch, double **out) {
  *out = nullptr;
  if (p->rank == 1 && !p->real) return MPFFT_OK;
  const size_t words = (size_t)2 * (p->real ? p->N + 1 : p->N) * batch;
  if (words > p->tmp_cap) {
    if (p->d_tmp) cudaFree(p->d_tmp);
    p->d_tmp = nullptr;
    p->tmp_cap = 0;
    if (dev_alloc((void **)&p->d_tmp, words * 8) != cudaSuccess) {
      cudaGetLastError();
      return set_err(MPFFT_ENOMEM, "cannot allocate %zu bytes of transposition scratch", words * 8);
    }
    p->tmp_cap = words;
  }
  *out = p->d_tmp;
  return MPFFT_OK;
}

static int d_execute_impl(mpfft_d_plan *p, unsigned long batch, const double *inr, const double *ini,
                          unsigned long s, double *outr, double *outi, unsigned flags) {
  std::lock_guard<std::mutex> g(p->mu);
  if ((unsigned long long)batch * p->N > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  if (int e = d_reserve(p, batch)) return e;
  double *tmp = nullptr;
  if (int e = d_tmp_reserve(p, batch, &tmp)) return e;
  // wait for device calls still using d_tmp; this call itself holds the lock
  // until its stream is synchronised, so later callers need no event from it
  if (tmp)
    if (int e = scratch_wait(p, p->stream)) return e;
  const unsigned long N = p->N;
  const size_t cim = (size_t)N * batch;
  // [c][b][p]: each signal contiguous
  const size_t bytes = 2 * cim * sizeof(double);
  if (s == 1 && 2 * cim > kCopyPiece) {
    // large arrays: pieces of the staging copies overlap the PCIe transfers
    // (piece i is copied into pinned memory while piece i-1 is in flight, and
    // copied out of it once its transfer has landed)
    const size_t total = 2 * cim, np = (total + kCopyPiece - 1) / kCopyPiece;
    while (p->piece_done.size() < np) {
      cudaEvent_t e;
      CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      p->piece_done.push_back(e);
    }
    // element o of the concatenated [re | im] staging lives in re[o] or im[o - cim]
    auto each_part = [&](size_t o, size_t len, const std::function<void(size_t, size_t, size_t)> &fn) {
      if (o < cim) fn(o, o, std::min(len, cim - o));
      if (o + len > cim) fn(std::max(o, cim), std::max(o, cim) - cim, o + len - std::max(o, cim));
    };
    for (size_t i = 0; i < np; ++i) {
      const size_t o = i * kCopyPiece, len = std::min(kCopyPiece, total - o);
      each_part(o, len, [&](size_t at, size_t src, size_t cnt) { par_copy(p->h_in + at, (at < cim ? inr : ini) + src, cnt); });
      CUDA_TRY(cudaMemcpyAsync(p->d_in + o, p->h_in + o, len * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    }
    CUDA_TRY(d_transform(p, p->d_in, p->d_out, (int)batch, flags, p->stream, tmp));
    for (size_t i = 0; i < np; ++i) {
      const size_t o = i * kCopyPiece, len = std::min(kCopyPiece, total - o);
      CUDA_TRY(cudaMemcpyAsync(p->h_out + o, p->d_out + o, len * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
      CUDA_TRY(cudaEventRecord(p->piece_done[i], p->stream));
    }
    for (size_t i = 0; i < np; ++i) {
      const size_t o = i * kCopyPiece, len = std::min(kCopyPiece, total - o);
      CUDA_TRY(cudaEventSynchronize(p->piece_done[i]));
      each_part(o, len, [&](size_t at, size_t dst, size_t cnt) { par_copy((at < cim ? outr : outi) + dst, p->h_out + at, cnt); });
    }
    return set_err(MPFFT_OK, "");
  }
  if (s == 1) {
    par_copy(p->h_in, inr, cim);
    par_copy(p->h_in + cim, ini, cim);
  } else {
    parallel_for((long)cim, kParCopyGrain, [&](long t0, long t1) {
      for (long t = t0; t < t1; ++t) {
        p->h_in[t] = inr[(size_t)t * s];
        p->h_in[cim + t] = ini[(size_t)t * s];
      }
    });
  }
  CUDA_TRY(cudaMemcpyAsync(p->d_in, p->h_in, bytes, cudaMemcpyHostToDevice, p->stream));
  CUDA_TRY(d_transform(p, p->d_in, p->d_out, (int)batch, flags, p->stream, tmp));
  CUDA_TRY(cudaMemcpyAsync(p->h_out, p->d_out, bytes, cudaMemcpyDeviceToHost, p->stream));
  CUDA_TRY(cudaStreamSynchronize(p->stream));
  par_copy(outr, p->h_out, cim);
  par_copy(outi, p->h_out + cim, cim);
  return set_err(MPFFT_OK, "");
}

// Compensated-tier plan (double-double, quad-double, float-float): the same
// tree, cut at T = min(n, tier_sub_max) points, base cases of at most 4
// points; cos and sin of 2 pi k/n computed by MPFR at 320 bits and split into
// the tier's words (each the nearest double to what the words above leave;
// float-float keeps one double: its products are formed in FP64).
static int d_plan_init_tier(mpfft_d_plan *p, unsigned long n, int tier, int sub_max) {
  if (!is_pow2(n)) return set_err(MPFFT_EINVAL, "n=%lu is not a power of two", n);
  if (n > (1UL << 26)) return set_err(MPFFT_EUNSUPPORTED, "n=%lu too large", n);
  if (int e = device_ready()) return e;
  p->N = n;
  p->tier = tier;
  p->dd = tier == kTierDD;
  p->tabs.N = (int)n;
  const int T = (int)std::min<unsigned long>(n, (unsigned long)(sub_max > 0 ? sub_max : tier_sub_max(tier)));
  {
    HostTree t;
    walk(t, (int)n, 1, 0, 0, T);
    std::vector<SubRoot> roots;
    for (const Leaf &lf : t.leaves) roots.push_back(SubRoot{lf.sn, lf.s, lf.out, lf.n});
    p->tabs.nroots = (int)roots.size();
    if (int e = upload(p, roots, &p->tabs.roots)) return e;
    if (int e = build_tree(p->upper, n, T)) return e;
    p->tabs.upper = p->upper.tabs;
  }
  if (int e = build_sub(p, T, p->tabs.sub[0], 4)) return e;
  if (T >= 2) {
    if (int e = build_sub(p, T / 2, p->tabs.sub[1], 4)) return e;
  } else {
    p->tabs.sub[1] = p->tabs.sub[0];
  }
  const int K = tier == kTierQD ? 4 : tier == kTierDD ? 2 : 1;  // twiddle words
  const unsigned long q = std::max<unsigned long>(1, n / 4);
  std::vector<double> w((size_t)2 * K * q);  // [cos words][sin words][k]
  parallel_for((long)q, 64, [&](long a, long b) {
    mpfr_t th, c, s;
    mpfr_init2(th, 360);
    mpfr_init2(c, 320);
    mpfr_init2(s, 320);
    for (long k = a; k < b; ++k) {
      mpfr_const_pi(th, MPFR_RNDN);
      mpfr_mul_ui(th, th, 2UL * (unsigned long)k, MPFR_RNDN);
      mpfr_div_ui(th, th, n, MPFR_RNDN);
      mpfr_sin_cos(s, c, th, MPFR_RNDN);
      for (int h = 0; h < K; ++h) {  // exact remainders at 320 bits
        w[(size_t)h * q + k] = mpfr_get_d(c, MPFR_RNDN);
        mpfr_sub_d(c, c, w[(size_t)h * q + k], MPFR_RNDN);
        w[(size_t)(K + h) * q + k] = mpfr_get_d(s, MPFR_RNDN);
        mpfr_sub_d(s, s, w[(size_t)(K + h) * q + k], MPFR_RNDN);
      }
    }
    mpfr_clear(th);
    mpfr_clear(c);
    mpfr_clear(s);
    mpfr_free_cache();
  });
  const double *dw = nullptr;
  if (int e = upload(p, w, &dw)) return e;
  for (int h = 0; h < K; ++h) {
    p->tabs.tw_cos[h] = dw + (size_t)h * q;
    p->tabs.tw_sin[h] = dw + (size_t)(K + h) * q;
  }
  p->tabs.wr = p->tabs.tw_cos[0];
  p->tabs.wi = p->tabs.tw_sin[0];
  if (K >= 2) {
    p->tabs.wrl = p->tabs.tw_cos[1];
    p->tabs.wil = p->tabs.tw_sin[1];
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  return MPFFT_OK;
}

// real transform of n >= 2 points: the n/2-point complex plan plus split twiddles
static int d_plan_init_real(mpfft_d_plan *p, unsigned long n) {
  if (!is_pow2(n) || n < 2) return set_err(MPFFT_EINVAL, "a real transform needs n >= 2, a power of two (n=%lu)", n);
  if (n > (1UL << 28)) return set_err(MPFFT_EUNSUPPORTED, "n=%lu too large", n);
  if (int e = d_plan_init(p, n / 2)) return e;
  p->real = true;
  p->n_real = n;
  const unsigned long q = std::max<unsigned long>(1, n / 4);
  std::vector<double> wc(q), ws(q);
  for (unsigned long k = 0; k < q; ++k) {
    wc[k] = cos(2. * M_PI * k / n);
    ws[k] = sin(2. * M_PI * k / n);
  }
  CUDA_TRY(cudaMalloc(&p->d_wc, q * sizeof(double)));
  CUDA_TRY(cudaMalloc(&p->d_ws, q * sizeof(double)));
  CUDA_TRY(cudaMemcpy(p->d_wc, wc.data(), q * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(p->d_ws, ws.data(), q * sizeof(double), cudaMemcpyHostToDevice));
  return MPFFT_OK;
}

// forward: in = batch x n reals -> outr/outi = batch x (n/2+1); else the inverse
static int d_execute_real(mpfft_d_plan *p, bool forward, unsigned long batch, const double *xin, const double *inr,
                          const double *ini, double *xout, double *outr, double *outi, unsigned flags) {
  std::lock_guard<std::mutex> g(p->mu);
  const unsigned long M = p->N, n = p->n_real, H = M + 1;
  if ((unsigned long long)batch * H > (unsigned long long)INT32_MAX) return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  if (int e = d_reserve(p, batch)) return e;
  double *tmp = nullptr;
  if (int e = d_tmp_reserve(p, batch, &tmp)) return e;
  if (int e = scratch_wait(p, p->stream)) return e;  // the real path always uses d_tmp
  const double scale = (flags & MPFFT_SCALED) ? 1.0 / (double)n : 1.0;
  if (forward) {
    // even samples -> real plane, odd samples -> imaginary plane ([c][b][m])
    for (unsigned long b = 0; b < batch; ++b)
      for (unsigned long m = 0; m < M; ++m) {
        p->h_in[b * M + m] = xin[b * n + 2 * m];
        p->h_in[(batch + b) * M + m] = xin[b * n + 2 * m + 1];
      }
    CUDA_TRY(cudaMemcpyAsync(p->d_in, p->h_in, 2 * M * batch * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    CUDA_TRY(d_run_transform(p->tabs, p->d_in, p->d_out, (int)batch, 1.0, p->stream));
    CUDA_TRY(d_real_split(true, p->d_out, tmp, (int)M, (int)batch, p->d_wc, p->d_ws, scale, p->stream));
    CUDA_TRY(cudaMemcpyAsync(p->h_out, tmp, 2 * H * batch * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    par_copy(outr, p->h_out, H * batch);
    par_copy(outi, p->h_out + H * batch, H * batch);
  } else {
    par_copy(p->h_in, inr, H * batch);
    par_copy(p->h_in + H * batch, ini, H * batch);
    CUDA_TRY(cudaMemcpyAsync(p->d_in, p->h_in, 2 * H * batch * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    CUDA_TRY(d_real_split(false, p->d_in, tmp, (int)M, (int)batch, p->d_wc, p->d_ws, 1.0, p->stream));
    CUDA_TRY(d_run_transform(p->tabs, tmp, p->d_out, (int)batch, scale, p->stream));
    CUDA_TRY(cudaMemcpyAsync(p->h_out, p->d_out, 2 * M * batch * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    // the transform of the exchanged planes: imaginary plane = even samples
    for (unsigned long b = 0; b < batch; ++b)
      for (unsigned long m = 0; m < M; ++m) {
        xout[b * n + 2 * m] = p->h_out[(batch + b) * M + m];
        xout[b * n + 2 * m + 1] = p->h_out[b * M + m];
      }
  }
  return set_err(MPFFT_OK, "");
}

static void d_plan_delete(mpfft_d_plan *p) { delete p; }

// The words of one real value x in a compensated tier (K words, floats when
// fl): the nearest word, then the nearest word to what is left, ... (exact
// down to the last word), word h stored at dst[at + h*stride].  t: scratch
// mpfr_t.  Returns 0, 1 for NaN/infinity, 2 for an exponent outside
// [emin, emax] (the window the words represent without underflow or overflow
// over N-point growth).
static inline int mpfr_to_words(mpfr_srcptr x, mpfr_ptr t, int K, bool fl, long emin, long emax, void *dst,
                                size_t at, size_t stride) {
  if (!mpfr_number_p(x)) return 1;
  if (!mpfr_zero_p(x) && (x->_mpfr_exp < emin || x->_mpfr_exp > emax)) return 2;
  if (mpfr_get_prec(t) < mpfr_get_prec(x)) mpfr_set_prec(t, mpfr_get_prec(x));
  mpfr_set(t, x, MPFR_RNDN);  // exact
  for (int h = 0; h < K; ++h) {
    const double w = fl ? (double)(float)mpfr_get_d(t, MPFR_RNDN) : mpfr_get_d(t, MPFR_RNDN);
    mpfr_sub_d(t, t, w, MPFR_RNDN);  // exact: the part of t below w
    if (fl) static_cast<float *>(dst)[at + (size_t)h * stride] = (float)w;
    else static_cast<double *>(dst)[at + (size_t)h * stride] = w;
  }
  return 0;
}

// y = (sum of the K words at src[at + h*stride]) * 2^-shift, rounded to nearest
// into y's precision; acc: a 320-bit scratch mpfr_t (the sum of a tier's words
// is exact at 320 bits)
static inline void words_to_mpfr(const void *src, size_t at, size_t stride, int K, bool fl, long shift, mpfr_ptr acc,
                                 mpfr_ptr y) {
  mpfr_set_zero(acc, 1);
  for (int h = 0; h < K; ++h)
    mpfr_add_d(acc, acc,
               fl ? (double)static_cast<const float *>(src)[at + (size_t)h * stride]
                  : static_cast<const double *>(src)[at + (size_t)h * stride],
               MPFR_RNDN);
  mpfr_mul_2si(acc, acc, -shift, MPFR_RNDN);
  mpfr_set(y, acc, MPFR_RNDN);
}

static inline void tier_window(const mpfft_d_plan *f, long *emin, long *emax) {
  const bool fl = d_word_bytes(f) == 4;
  *emin = fl ? -100 : -700;
  *emax = fl ? 90 : 900;
}

// A transform through the plan's compensated floating-point tier: every mpfr_t
// input is split on the host into the tier's words (mpfr_to_words), the
// tier's kernels run, and each output is the words' sum times 2^-fadj rounded
// into the output's precision (words_to_mpfr).  Returns kFloatOutOfRange,
// before writing any output, when an input exponent lies outside the tier's
// window; the caller then runs the limb kernels.
static int mp_execute_float(mpfft_mp_plan *p, unsigned long batch, const IoShape &ii, mpfr_t *inr, mpfr_t *ini,
                            const IoShape &oo, mpfr_t *outr, mpfr_t *outi, long fadj) {
  mpfft_d_plan *f = p->fplan;
  const unsigned long N = p->N;
  if ((unsigned long long)batch * N > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  std::lock_guard<std::mutex> g(f->mu);
  if (int e = d_reserve(f, batch)) return e;
  const int K = d_words(f);
  const bool fl = d_word_bytes(f) == 4;
  long emin, emax;
  tier_window(f, &emin, &emax);
  const size_t hplane = (size_t)N * batch;
  std::atomic<int> status{0};
  parallel_for((long)hplane, 1024, [&](long a0, long a1) {
    mpfr_t t;
    mpfr_init2(t, 64);
    int st = 0;
    for (long u = a0; u < a1; ++u) {
      const unsigned long b = (unsigned long)u / N, q = (unsigned long)u % N;
      for (int c = 0; c < 2; ++c)
        st |= mpfr_to_words(elem(c ? ini : inr, c, b, ii, q), t, K, fl, emin, emax, f->h_in,
                            ((size_t)c * K * batch + b) * N + q, hplane);
    }
    mpfr_clear(t);
    if (st) status.fetch_or(st);
  });
  if (status.load() & 2) return kFloatOutOfRange;
  if (status.load() & 1) return set_err(MPFFT_ENONFINITE, "input holds NaN or infinity");
  const size_t bytes = (size_t)2 * K * hplane * d_word_bytes(f);
  CUDA_TRY(cudaMemcpyAsync(f->d_in, f->h_in, bytes, cudaMemcpyHostToDevice, f->stream));
  if (f->tier < 0) CUDA_TRY(d_run_transform(f->tabs, f->d_in, f->d_out, (int)batch, 1.0, f->stream));
  else CUDA_TRY(tier_run_transform(f->tier, f->tabs, f->d_in, f->d_out, (int)batch, 1.0, f->stream));
  CUDA_TRY(cudaMemcpyAsync(f->h_out, f->d_out, bytes, cudaMemcpyDeviceToHost, f->stream));
  CUDA_TRY(cudaStreamSynchronize(f->stream));
  parallel_for((long)hplane, 1024, [&](long a0, long a1) {
    mpfr_t acc;
    mpfr_init2(acc, 320);
    for (long u = a0; u < a1; ++u) {
      const unsigned long b = (unsigned long)u / N, q = (unsigned long)u % N;
      for (int c = 0; c < 2; ++c)
        words_to_mpfr(f->h_out, ((size_t)c * K * batch + b) * N + q, hplane, K, fl, fadj, acc,
                      elem(c ? outi : outr, c, b, oo, q));
    }
    mpfr_clear(acc);
  });
  return set_err(MPFFT_OK, "");
}

static void d_dropin(unsigned long n, unsigned long s, long sn, double *inr, double *ini, double *outr,
                     double *outi, unsigned flags) {
  if (!inr || !ini || !outr || !outi) {
    set_err(MPFFT_EINVAL, "NULL array");
    return;
  }
  if (flags & MPFFT_INVERSE) {  // ifft(X) = swap(FFT(swap(X))) (times 1/n if scaled)
    std::swap(inr, ini);
    std::swap(outr, outi);
    flags &= ~MPFFT_INVERSE;
  }
  int e = MPFFT_OK;
  if (!is_pow2(n)) e = set_err(MPFFT_EINVAL, "n=%lu is not a power of two", n);
  else if (s == 0) e = set_err(MPFFT_EINVAL, "stride s must be >= 1");
  else if (sn < 0)
    e = set_err(MPFFT_EINVAL, "sn=%ld < 0 addresses the reference's global array; only top-level calls (sn >= 0)", sn);
  if (e == MPFFT_OK) {
    mpfft_d_plan *p = d_cached(n);
    if (!p) e = g_err;
    else e = d_execute_impl(p, 1, inr, ini, s, outr, outi, flags);
  }
  if (e != MPFFT_OK && is_pow2(n)) {
    for (unsigned long k = 0; k < n; ++k) outr[k] = outi[k] = NAN;
  }
}

}  // namespace mpfft

// ===========================================================================
// C ABI
// ===========================================================================

MPFFT_API void mp_sr24_cp_fft(unsigned long n, unsigned long s, long sn, mpfr_t *inr, mpfr_t *ini, mpfr_t *outr,
                              mpfr_t *outi) {
  mp_dropin(n, s, sn, inr, ini, outr, outi, 0);
}

MPFFT_API void mp_sr24_cp_fft_v2(unsigned long n, unsigned long log2n, unsigned long s, long sn, mpfr_t *inr,
                                 mpfr_t *ini, mpfr_t *outr, mpfr_t *outi) {
  if (log2n != 0) {
    set_err(MPFFT_EINVAL, "log2n=%lu != 0 is a sub-transform of the reference's global N", log2n);
    if (is_pow2(n) && outr && outi) {
      mp_fill_nan(outr, n);
      mp_fill_nan(outi, n);
    }
    return;
  }
  mp_dropin(n, s, sn, inr, ini, outr, outi, 0);
}

MPFFT_API void mp_sr24_cp_fft_scaled(unsigned long n, unsigned long s, long sn, mpfr_t *inr, mpfr_t *ini,
                                     mpfr_t *outr, mpfr_t *outi) {
  mp_dropin(n, s, sn, inr, ini, outr, outi, MPFFT_SCALED);
}

MPFFT_API void mp_sr24_cp_ifft(unsigned long n, unsigned long s, long sn, mpfr_t *inr, mpfr_t *ini, mpfr_t *outr,
                               mpfr_t *outi) {
  mp_dropin(n, s, sn, inr, ini, outr, outi, MPFFT_INVERSE | MPFFT_SCALED);
}

MPFFT_API void d_sr24_cp_ifft(unsigned long n, unsigned long s, long sn, double *inr, double *ini, double *outr,
                              double *outi) {
  d_dropin(n, s, sn, inr, ini, outr, outi, MPFFT_INVERSE | MPFFT_SCALED);
}

MPFFT_API void d_sr24_cp_fft(unsigned long n, unsigned long s, long sn, double *inr, double *ini, double *outr,
                             double *outi) {
  d_dropin(n, s, sn, inr, ini, outr, outi, 0);
}

MPFFT_API void d_sr24_cp_fft_v2(unsigned long n, unsigned long log2n, unsigned long s, long sn, double *inr,
                                double *ini, double *outr, double *outi) {
  if (log2n != 0) {
    set_err(MPFFT_EINVAL, "log2n=%lu != 0 is a sub-transform of the reference's global N", log2n);
    if (is_pow2(n) && outr && outi)
      for (unsigned long k = 0; k < n; ++k) outr[k] = outi[k] = NAN;
    return;
  }
  d_dropin(n, s, sn, inr, ini, outr, outi, 0);
}

MPFFT_API void d_sr24_cp_fft_scaled(unsigned long n, unsigned long s, long sn, double *inr, double *ini,
                                    double *outr, double *outi) {
  d_dropin(n, s, sn, inr, ini, outr, outi, MPFFT_SCALED);
}

MPFFT_API int mpfft_last_error(void) { return g_err; }
MPFFT_API const char *mpfft_last_error_string(void) { return g_msg; }

MPFFT_API int mpfft_mp_plan_create_flags(mpfft_mp_plan **plan, unsigned long n, long prec, unsigned flags) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  std::unique_ptr<mpfft_mp_plan> p(new (std::nothrow) mpfft_mp_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = mp_plan_init(p.get(), n, prec, (flags & MPFFT_PLAN_HOST_ONLY) != 0)) return e;
  p->force_host_conversion = (flags & MPFFT_PLAN_HOST_CONVERSION) != 0;
  if (flags & MPFFT_PLAN_NO_TENSOR) p->tabs.tc = 0;
  else if (flags & MPFFT_PLAN_TENSOR) p->tabs.tc = 2;
  if (!p->host_only && mp_tc_used(p->tabs, p->L)) p->form = MPFFT_FORM_TENSOR;
  if (flags & (MPFFT_PLAN_FLOAT_TIERS | MPFFT_PLAN_NATIVE_TIERS))
    if (int e = mp_plan_attach_float_tier(p.get(), (flags & MPFFT_PLAN_NATIVE_TIERS) != 0)) return e;
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_plan_create_nd(mpfft_mp_plan **plan, int rank, const unsigned long *dims, long prec,
                                      unsigned flags) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  std::unique_ptr<mpfft_mp_plan> p(new (std::nothrow) mpfft_mp_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = mp_plan_init_nd(p.get(), rank, dims, prec, (flags & MPFFT_PLAN_HOST_ONLY) != 0)) return e;
  p->force_host_conversion = (flags & MPFFT_PLAN_HOST_CONVERSION) != 0;
  if (flags & (MPFFT_PLAN_NO_TENSOR | MPFFT_PLAN_TENSOR)) {
    const int tc = (flags & MPFFT_PLAN_NO_TENSOR) ? 0 : 2;
    p->tabs.tc = tc;
    for (auto &a : p->axis)
      if (a) a->tabs.tc = tc;
  }
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_plan_create(mpfft_mp_plan **plan, unsigned long n, long prec) {
  return mpfft_mp_plan_create_flags(plan, n, prec, 0);
}

MPFFT_API int mpfft_mp_plan_destroy(mpfft_mp_plan *plan) {
  delete plan;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_plan_limbs(const mpfft_mp_plan *plan) { return plan ? plan->L : 0; }
MPFFT_API int mpfft_mp_plan_form(const mpfft_mp_plan *plan) { return plan ? plan->form : -1; }
MPFFT_API long mpfft_mp_plan_frac_bits(const mpfft_mp_plan *plan) { return plan ? plan->F : 0; }

MPFFT_API int mpfft_mp_execute(mpfft_mp_plan *plan, unsigned long batch, mpfr_t *inr, mpfr_t *ini, mpfr_t *outr,
                               mpfr_t *outi, unsigned flags) {
  if (!plan || !inr || !ini || !outr || !outi) return set_err(MPFFT_EINVAL, "NULL argument");
  if (batch == 0) return set_err(MPFFT_OK, "");
  if (flags & MPFFT_INVERSE) {  // ifft(X) = swap(FFT(swap(X))) (times 1/n if scaled)
    std::swap(inr, ini);
    std::swap(outr, outi);
    flags &= ~MPFFT_INVERSE;
  }
  if (plan->real) return set_err(MPFFT_EINVAL, "real plan: use mpfft_mp_execute_r2c / mpfft_mp_execute_c2r");
  int e = mp_execute_complex(plan, batch, inr, ini, 1, outr, outi, flags);
  if (e != MPFFT_OK) {
    mp_fill_nan(outr, plan->N * batch);
    mp_fill_nan(outi, plan->N * batch);
  }
  return e;
}

MPFFT_API int mpfft_mp_execute_mixed(unsigned long count, const unsigned long *n, mpfr_t *const *inr,
                                     mpfr_t *const *ini, mpfr_t *const *outr, mpfr_t *const *outi, unsigned flags) {
  if (!n || !inr || !ini || !outr || !outi) return set_err(MPFFT_EINVAL, "NULL argument");
  if (flags & MPFFT_INVERSE) {  // ifft(X) = swap(FFT(swap(X))) (times 1/n if scaled)
    std::swap(inr, ini);
    std::swap(outr, outi);
    flags &= ~MPFFT_INVERSE;
  }
  // group the signals by (length, limb count): each group is one batched execution of a cached plan
  std::map<std::pair<unsigned long, int>, std::vector<unsigned long>> groups;
  std::vector<long> prec(count);
  for (unsigned long i = 0; i < count; ++i) {
    if (!inr[i] || !ini[i] || !outr[i] || !outi[i]) return set_err(MPFFT_EINVAL, "NULL array of signal %lu", i);
    if (!is_pow2(n[i])) return set_err(MPFFT_EINVAL, "n[%lu]=%lu is not a power of two", i, n[i]);
    prec[i] = mp_call_prec(inr[i], ini[i], outr[i], outi[i]);
    if (prec[i] < 2) return set_err(MPFFT_EINVAL, "signal %lu: precision %ld < 2", i, prec[i]);
    groups[std::make_pair(n[i], mp_limbs_for(n[i], prec[i]))].push_back(i);
  }
  int first_err = MPFFT_OK;
  std::string first_msg;
  for (auto &kv : groups) {
    const unsigned long nn = kv.first.first;
    const std::vector<unsigned long> &ids = kv.second;
    long pg = 2;
    for (unsigned long i : ids) pg = std::max(pg, prec[i]);
    mpfft_mp_plan *p = mp_cached(nn, pg);
    int e = p ? MPFFT_OK : g_err;
    if (e == MPFFT_OK) {
      std::vector<mpfr_t *> bi[2], bo[2];
      for (unsigned long i : ids) {
        bi[0].push_back(inr[i]);
        bi[1].push_back(ini[i]);
        bo[0].push_back(outr[i]);
        bo[1].push_back(outi[i]);
      }
      IoShape ii = io_signals(nn, 1), oo = io_signals(nn, 1);
      ii.base[0] = bi[0].data();
      ii.base[1] = bi[1].data();
      oo.base[0] = bo[0].data();
      oo.base[1] = bo[1].data();
      const long shift = (flags & MPFFT_SCALED) ? ilog2(nn) : 0;
      e = mp_execute_impl(p, ids.size(), kComplex, ii, nullptr, nullptr, oo, nullptr, nullptr, shift);
    }
    if (e != MPFFT_OK) {
      if (first_err == MPFFT_OK) {
        first_err = e;
        first_msg = g_msg;
      }
      for (unsigned long i : ids) {
        mp_fill_nan(outr[i], nn);
        mp_fill_nan(outi[i], nn);
      }
    }
  }
  if (first_err != MPFFT_OK) return set_err(first_err, "%s", first_msg.c_str());
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_plan_create_real(mpfft_mp_plan **plan, unsigned long n, long prec, unsigned flags) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  if (flags & MPFFT_PLAN_HOST_ONLY) return set_err(MPFFT_EINVAL, "real plans have no host-only form");
  std::unique_ptr<mpfft_mp_plan> p(new (std::nothrow) mpfft_mp_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = mp_plan_init(p.get(), n, prec, false, true)) return e;
  p->force_host_conversion = (flags & MPFFT_PLAN_HOST_CONVERSION) != 0;
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_execute_r2c(mpfft_mp_plan *plan, unsigned long batch, mpfr_t *in, mpfr_t *outr,
                                   mpfr_t *outi, unsigned flags) {
  if (!plan || !in || !outr || !outi) return set_err(MPFFT_EINVAL, "NULL argument");
  if (!plan->real) return set_err(MPFFT_EINVAL, "not a real plan (mpfft_mp_plan_create_real)");
  if (flags & MPFFT_INVERSE) return set_err(MPFFT_EINVAL, "MPFFT_INVERSE: use mpfft_mp_execute_c2r");
  if (batch == 0) return set_err(MPFFT_OK, "");
  const unsigned long n = plan->n_real, m = plan->N;
  // x_(2j) -> real plane, x_(2j+1) -> imaginary plane of the m-point complex signal
  const IoShape ii{m, n, 2}, oo{m + 1, m + 1, 1};
  const long fadj = 1 + ((flags & MPFFT_SCALED) ? ilog2(n) : 0);  // the split step yields 2X
  int e = mp_execute_impl(plan, batch, kR2C, ii, in, in + 1, oo, outr, outi, fadj);
  if (e != MPFFT_OK) {
    mp_fill_nan(outr, (m + 1) * batch);
    mp_fill_nan(outi, (m + 1) * batch);
  }
  return e;
}

MPFFT_API int mpfft_mp_execute_c2r(mpfft_mp_plan *plan, unsigned long batch, mpfr_t *inr, mpfr_t *ini,
                                   mpfr_t *out, unsigned flags) {
  if (!plan || !inr || !ini || !out) return set_err(MPFFT_EINVAL, "NULL argument");
  if (!plan->real) return set_err(MPFFT_EINVAL, "not a real plan (mpfft_mp_plan_create_real)");
  if (batch == 0) return set_err(MPFFT_OK, "");
  const unsigned long n = plan->n_real, m = plan->N;
  // the result's real plane holds the odd samples, its imaginary plane the even ones
  const IoShape ii{m + 1, m + 1, 1}, oo{m, n, 2};
  const long fadj = (flags & MPFFT_SCALED) ? ilog2(n) : 0;
  int e = mp_execute_impl(plan, batch, kC2R, ii, inr, ini, oo, out + 1, out, fadj);
  if (e != MPFFT_OK) mp_fill_nan(out, n * batch);
  return e;
}

// One-dimensional integer-pipe plans replay a device-layout call shape
// (batch, input, output) from a CUDA graph from its second use on: one graph
// launch instead of one launch per level, which matters for single signals,
// whose levels are each a few microseconds of device work -- less than the
// host's cost of issuing them.  Captured on the plan's own stream (the
// caller's may be the legacy default stream, which cannot be captured) and
// launched on the caller's.  The first use runs directly, so that nothing is
// initialised inside a capture; a capture that fails leaves the shape on
// direct launches.  Called under plan->mu.
constexpr size_t kDeviceGraphsMax = 16;  // cached call shapes per plan

static cudaGraphExec_t mp_device_graph(mpfft_mp_plan *p, unsigned long batch, const uint32_t *in, uint32_t *out) {
  const mpfft_mp_plan::DevKey key{batch, in, out};
  auto it = p->dev_graphs.find(key);
  if (it != p->dev_graphs.end()) return it->second;
  if (p->dev_uses.size() >= 4 * kDeviceGraphsMax || p->dev_graphs.size() >= kDeviceGraphsMax) p->free_dev_graphs();
  if (p->dev_uses[key]++ < 1) return nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  if (cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    const cudaError_t e = mp_transform(p, in, out, (int)batch, p->stream, nullptr, nullptr);
    const cudaError_t ce = cudaStreamEndCapture(p->stream, &g);
    if (e != cudaSuccess || ce != cudaSuccess || !g || cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) ge = nullptr;
    if (g) cudaGraphDestroy(g);
  }
  cudaGetLastError();
  p->dev_graphs.emplace(key, ge);
  return ge;
}

MPFFT_API int mpfft_mp_execute_device(mpfft_mp_plan *plan, unsigned long batch, const uint32_t *d_in,
                                      uint32_t *d_out, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->host_only) return set_err(MPFFT_EINVAL, "plan was created host-only (conversion only)");
  if (plan->real) return set_err(MPFFT_EINVAL, "real plans have no device-layout entry point");
  if (batch == 0) return set_err(MPFFT_OK, "");
  const size_t bytes = (size_t)2 * plan->L * plan->N * batch * 4;
  const char *a = (const char *)d_in, *b = (const char *)d_out;
  if (a < b + bytes && b < a + bytes) return set_err(MPFFT_EINVAL, "input and output buffers overlap");
  if (batch > (unsigned long)INT32_MAX || (unsigned long long)batch * plan->N > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  std::lock_guard<std::mutex> g(plan->mu);
  uint32_t *big = nullptr, *tmp = nullptr;
  if (int e = mp_big_reserve(plan, batch, &big)) return e;
  if (int e = mp_tmp_reserve(plan, batch, &tmp)) return e;
  const cudaStream_t st = (cudaStream_t)stream;
  // (not while the caller's stream is being captured: its own graph takes the launches)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusActive;
  }
  if (cap == cudaStreamCaptureStatusNone && !big && !tmp && plan->rank == 1 && plan->L <= kMaxLimbs &&
      !mp_tc_used(plan->tabs, plan->L))
    if (cudaGraphExec_t ge = mp_device_graph(plan, batch, d_in, d_out)) {
      CUDA_TRY(cudaGraphLaunch(ge, st));
      return set_err(MPFFT_OK, "");
    }
  if (big || tmp)
    if (int e = scratch_wait(plan, st)) return e;
  CUDA_TRY(mp_transform(plan, d_in, d_out, (int)batch, st, big, tmp));
  if (big || tmp)
    if (int e = scratch_record(plan, st)) return e;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_pack(const mpfft_mp_plan *plan, unsigned long batch, mpfr_t *inr, mpfr_t *ini,
                            uint32_t *planes, long *exps) {
  if (!plan || !inr || !ini || !planes || !exps) return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->real) return set_err(MPFFT_EINVAL, "pack/unpack take complex plans");
  if (int e = mp_pack_impl(plan, batch, io_signals(plan->N, 1), inr, ini, planes, exps)) return e;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_unpack(const mpfft_mp_plan *plan, unsigned long batch, const uint32_t *planes,
                              const long *exps, mpfr_t *outr, mpfr_t *outi, unsigned flags) {
  if (!plan || !outr || !outi || !planes || !exps) return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->real) return set_err(MPFFT_EINVAL, "pack/unpack take complex plans");
  mp_unpack_impl(plan, batch, planes, exps, io_signals(plan->N, 1), outr, outi,
                 (flags & MPFFT_SCALED) ? ilog2(plan->N) : 0);
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_d_plan_create(mpfft_d_plan **plan, unsigned long n) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  std::unique_ptr<mpfft_d_plan> p(new (std::nothrow) mpfft_d_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = d_plan_init(p.get(), n)) return e;
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_dd_plan_create(mpfft_d_plan **plan, unsigned long n) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  std::unique_ptr<mpfft_d_plan> p(new (std::nothrow) mpfft_d_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = d_plan_init_tier(p.get(), n, kTierDD)) return e;
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

static int d_plan_create_tier(mpfft_d_plan **plan, unsigned long n, int tier) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  std::unique_ptr<mpfft_d_plan> p(new (std::nothrow) mpfft_d_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = d_plan_init_tier(p.get(), n, tier)) return e;
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_qd_plan_create(mpfft_d_plan **plan, unsigned long n) {
  return d_plan_create_tier(plan, n, kTierQD);
}

MPFFT_API int mpfft_ff_plan_create(mpfft_d_plan **plan, unsigned long n) {
  return d_plan_create_tier(plan, n, kTierFF);
}

MPFFT_API int mpfft_multiword_format(const mpfft_d_plan *plan, int *words, int *word_bytes) {
  if (!plan || !words || !word_bytes) return set_err(MPFFT_EINVAL, "NULL argument");
  *words = d_words(plan);
  *word_bytes = (int)d_word_bytes(plan);
  return set_err(MPFFT_OK, "");
}

static int multiword_check(const mpfft_d_plan *plan, unsigned long batch) {
  if (plan->tier < 0) return set_err(MPFFT_EINVAL, "not a double-double, quad-double or float-float plan");
  if (plan->real || plan->rank > 1) return set_err(MPFFT_EINVAL, "multiword plans are one-dimensional complex plans");
  if ((unsigned long long)batch * plan->N > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  return MPFFT_OK;
}

MPFFT_API int mpfft_multiword_execute(mpfft_d_plan *plan, unsigned long batch, const void *x, void *y,
                                      unsigned flags) {
  if (!plan || !x || !y) return set_err(MPFFT_EINVAL, "NULL argument");
  if (int e = multiword_check(plan, batch)) return e;
  if (batch == 0) return set_err(MPFFT_OK, "");
  std::lock_guard<std::mutex> g(plan->mu);
  if (int e = d_reserve(plan, batch)) return e;
  const size_t bytes = (size_t)2 * d_words(plan) * plan->N * batch * d_word_bytes(plan);
  const bool inv = (flags & MPFFT_INVERSE) != 0;
  memcpy(plan->h_in, x, bytes);
  CUDA_TRY(cudaMemcpyAsync(plan->d_in, plan->h_in, bytes, cudaMemcpyHostToDevice, plan->stream));
  CUDA_TRY(tier_run_transform(plan->tier, plan->tabs, plan->d_in, plan->d_out, (int)batch, d_scale(plan, flags),
                              plan->stream, inv, inv));
  CUDA_TRY(cudaMemcpyAsync(plan->h_out, plan->d_out, bytes, cudaMemcpyDeviceToHost, plan->stream));
  CUDA_TRY(cudaStreamSynchronize(plan->stream));
  memcpy(y, plan->h_out, bytes);
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_multiword_execute_device(mpfft_d_plan *plan, unsigned long batch, const void *d_in, void *d_out,
                                             unsigned flags, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(MPFFT_EINVAL, "NULL argument");
  if (int e = multiword_check(plan, batch)) return e;
  if (batch == 0) return set_err(MPFFT_OK, "");
  const size_t bytes = (size_t)2 * d_words(plan) * plan->N * batch * d_word_bytes(plan);
  const char *a = (const char *)d_in, *b = (const char *)d_out;
  if (a < b + bytes && b < a + bytes) return set_err(MPFFT_EINVAL, "input and output buffers overlap");
  const bool inv = (flags & MPFFT_INVERSE) != 0;
  CUDA_TRY(tier_run_transform(plan->tier, plan->tabs, d_in, d_out, (int)batch, d_scale(plan, flags),
                              (cudaStream_t)stream, inv, inv));
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_dd_execute(mpfft_d_plan *plan, unsigned long batch, const double *xr_hi, const double *xr_lo,
                               const double *xi_hi, const double *xi_lo, double *yr_hi, double *yr_lo,
                               double *yi_hi, double *yi_lo, unsigned flags) {
  if (!plan || !xr_hi || !xr_lo || !xi_hi || !xi_lo || !yr_hi || !yr_lo || !yi_hi || !yi_lo)
    return set_err(MPFFT_EINVAL, "NULL argument");
  if (!plan->dd) return set_err(MPFFT_EINVAL, "not a double-double plan (mpfft_dd_plan_create)");
  if (batch == 0) return set_err(MPFFT_OK, "");
  if ((unsigned long long)batch * plan->N > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  if (flags & MPFFT_INVERSE) {  // ifft(X) = swap(FFT(swap(X))) (times 1/n if scaled)
    std::swap(xr_hi, xi_hi);
    std::swap(xr_lo, xi_lo);
    std::swap(yr_hi, yi_hi);
    std::swap(yr_lo, yi_lo);
  }
  std::lock_guard<std::mutex> g(plan->mu);
  if (int e = d_reserve(plan, batch)) return e;
  const size_t pl = (size_t)plan->N * batch;
  const double *src[4] = {xr_hi, xr_lo, xi_hi, xi_lo};
  for (int i = 0; i < 4; ++i) par_copy(plan->h_in + i * pl, src[i], pl);
  CUDA_TRY(cudaMemcpyAsync(plan->d_in, plan->h_in, 4 * pl * sizeof(double), cudaMemcpyHostToDevice, plan->stream));
  CUDA_TRY(dd_run_transform(plan->tabs, plan->d_in, plan->d_out, (int)batch, d_scale(plan, flags), plan->stream));
  CUDA_TRY(cudaMemcpyAsync(plan->h_out, plan->d_out, 4 * pl * sizeof(double), cudaMemcpyDeviceToHost, plan->stream));
  CUDA_TRY(cudaStreamSynchronize(plan->stream));
  double *dst[4] = {yr_hi, yr_lo, yi_hi, yi_lo};
  for (int i = 0; i < 4; ++i) par_copy(dst[i], plan->h_out + i * pl, pl);
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_dd_execute_device(mpfft_d_plan *plan, unsigned long batch, const double *d_in, double *d_out,
                                      unsigned flags, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(MPFFT_EINVAL, "NULL argument");
  if (!plan->dd) return set_err(MPFFT_EINVAL, "not a double-double plan (mpfft_dd_plan_create)");
  if (batch == 0) return set_err(MPFFT_OK, "");
  if ((unsigned long long)batch * plan->N > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  const size_t bytes = (size_t)4 * plan->N * batch * 8;
  const char *a = (const char *)d_in, *b = (const char *)d_out;
  if (a < b + bytes && b < a + bytes) return set_err(MPFFT_EINVAL, "input and output buffers overlap");
  const bool inv = (flags & MPFFT_INVERSE) != 0;
  CUDA_TRY(dd_run_transform(plan->tabs, d_in, d_out, (int)batch, d_scale(plan, flags), (cudaStream_t)stream, inv,
                            inv));
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_d_plan_create_real(mpfft_d_plan **plan, unsigned long n) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  std::unique_ptr<mpfft_d_plan> p(new (std::nothrow) mpfft_d_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = d_plan_init_real(p.get(), n)) return e;
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_d_execute_r2c(mpfft_d_plan *plan, unsigned long batch, const double *in, double *outr,
                                  double *outi, unsigned flags) {
  if (!plan || !in || !outr || !outi) return set_err(MPFFT_EINVAL, "NULL argument");
  if (!plan->real) return set_err(MPFFT_EINVAL, "not a real plan (mpfft_d_plan_create_real)");
  if (batch == 0) return set_err(MPFFT_OK, "");
  return d_execute_real(plan, true, batch, in, nullptr, nullptr, nullptr, outr, outi, flags);
}

MPFFT_API int mpfft_d_execute_c2r(mpfft_d_plan *plan, unsigned long batch, const double *inr, const double *ini,
                                  double *out, unsigned flags) {
  if (!plan || !inr || !ini || !out) return set_err(MPFFT_EINVAL, "NULL argument");
  if (!plan->real) return set_err(MPFFT_EINVAL, "not a real plan (mpfft_d_plan_create_real)");
  if (batch == 0) return set_err(MPFFT_OK, "");
  return d_execute_real(plan, false, batch, nullptr, inr, ini, out, nullptr, nullptr, flags);
}

MPFFT_API int mpfft_d_plan_create_nd(mpfft_d_plan **plan, int rank, const unsigned long *dims) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL plan pointer");
  *plan = nullptr;
  std::unique_ptr<mpfft_d_plan> p(new (std::nothrow) mpfft_d_plan);
  if (!p) return set_err(MPFFT_ENOMEM, "out of host memory");
  if (int e = d_plan_init_nd(p.get(), rank, dims)) return e;
  *plan = p.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_d_plan_destroy(mpfft_d_plan *plan) {
  delete plan;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_d_execute(mpfft_d_plan *plan, unsigned long batch, const double *inr, const double *ini,
                              double *outr, double *outi, unsigned flags) {
  if (!plan || !inr || !ini || !outr || !outi) return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->real) return set_err(MPFFT_EINVAL, "real plan: use mpfft_d_execute_r2c / mpfft_d_execute_c2r");
  if (plan->tier >= 0) return set_err(MPFFT_EINVAL, "multiword plan: use mpfft_multiword_execute (or mpfft_dd_execute)");
  if (batch == 0) return set_err(MPFFT_OK, "");
  if (flags & MPFFT_INVERSE) {  // ifft(X) = swap(FFT(swap(X))) (times 1/n if scaled)
    std::swap(inr, ini);
    std::swap(outr, outi);
    flags &= ~MPFFT_INVERSE;
  }
  return d_execute_impl(plan, batch, inr, ini, 1, outr, outi, flags);
}

MPFFT_API int mpfft_d_execute_device(mpfft_d_plan *plan, unsigned long batch, const double *d_in, double *d_out,
                                     unsigned flags, void *stream) {
  if (!plan || !d_in || !d_out) return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->real) return set_err(MPFFT_EINVAL, "real plans have no device-layout entry point");
  if (plan->tier >= 0)
    return set_err(MPFFT_EINVAL, "multiword plan: use mpfft_multiword_execute_device (or mpfft_dd_execute_device)");
  if (batch == 0) return set_err(MPFFT_OK, "");
  const size_t bytes = (size_t)2 * plan->N * batch * 8;
  const char *a = (const char *)d_in, *b = (const char *)d_out;
  if (a < b + bytes && b < a + bytes) return set_err(MPFFT_EINVAL, "input and output buffers overlap");
  if ((unsigned long long)batch * plan->N > (unsigned long long)INT32_MAX)
    return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  std::lock_guard<std::mutex> g(plan->mu);
  double *tmp = nullptr;
  if (int e = d_tmp_reserve(plan, batch, &tmp)) return e;
  const cudaStream_t st = (cudaStream_t)stream;
  if (tmp)
    if (int e = scratch_wait(plan, st)) return e;
  CUDA_TRY(d_transform(plan, d_in, d_out, (int)batch, flags, st, tmp));
  if (tmp)
    if (int e = scratch_record(plan, st)) return e;
  return set_err(MPFFT_OK, "");
}

// ---------------------------------------------------------------------------
// diagnostics for benchmarks
// ---------------------------------------------------------------------------

MPFFT_API int mpfft_mp_plan_schedule(const mpfft_mp_plan *plan, int *level_n, int *level_nodes, int max_levels) {
  if (!plan || plan->host_only || plan->rank > 1) return -1;
  const int n = plan->tabs.nlevels;
  for (int i = 0; i < n && i < max_levels; ++i) {
    level_n[i] = plan->tabs.level_n[i];
    level_nodes[i] = plan->tabs.level_count[i];
  }
  return n;
}

MPFFT_API int mpfft_mp_execute_device_timed(mpfft_mp_plan *plan, unsigned long batch, const uint32_t *d_in,
                                            uint32_t *d_out, void *stream, float *launch_ms) {
  if (!plan || !d_in || !d_out || !launch_ms) return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->host_only) return set_err(MPFFT_EINVAL, "plan was created host-only (conversion only)");
  if (plan->real) return set_err(MPFFT_EINVAL, "real plans have no device-layout entry point");
  if (plan->rank > 1) return set_err(MPFFT_EINVAL, "per-launch timing is for one-dimensional plans");
  std::lock_guard<std::mutex> g(plan->mu);
  uint32_t *big = nullptr;
  if (int e = mp_big_reserve(plan, batch, &big)) return e;
  const cudaStream_t st = (cudaStream_t)stream;
  if (big)
    if (int e = scratch_wait(plan, st)) return e;
  CUDA_TRY(mp_run_transform(plan->L, plan->tabs, d_in, d_out, (int)batch, st, launch_ms, big));
  if (big)
    if (int e = scratch_record(plan, st)) return e;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_diag_tc_mul(int limbs, unsigned long batch, const uint32_t *d_x, const uint32_t *d_w,
                                uint32_t *d_out, void *stream) {
  if (!d_x || !d_w || !d_out) return set_err(MPFFT_EINVAL, "NULL argument");
  if (limbs < kTcMinLimbs || limbs > kTcMaxLimbs)
    return set_err(MPFFT_EUNSUPPORTED, "limbs must be in [%d, %d]", kTcMinLimbs, kTcMaxLimbs);
  if (batch == 0) return set_err(MPFFT_OK, "");
  if (batch > (unsigned long)INT32_MAX) return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  if (int e = device_ready()) return e;
  CUDA_TRY(mp_tc_mul(limbs, (int)batch, d_x, d_w, d_out, (cudaStream_t)stream));
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_diag_tc_set_wait_limit(unsigned long long ns) {
  if (int e = device_ready()) return e;
  CUDA_TRY(mp_tc_set_wait_limit(ns));
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_diag_fail_allocations(long after) {
  g_alloc_fail_after.store(after < 0 ? -1 : after);
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_mp_plan_counts(const mpfft_mp_plan *plan, unsigned long *mults, unsigned long *adds) {
  if (!plan || !mults || !adds) return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->host_only || plan->rank > 1 || plan->real)
    return set_err(MPFFT_EINVAL, "op counts are reported for one-dimensional complex device plans");
  const TreeTables &T = plan->tabs;
  // leaves: a 4-point DFT is 16 additions, a 2-point one 4 (reference base
  // cases, lab/parallel/mp/parallel_mp_fft2.c:136-177)
  unsigned long m = 0, a = 16UL * T.leaf_count[4] + 4UL * T.leaf_count[2];
  for (int lv = 0; lv < T.nlevels; ++lv) {
    // per node of size n (q = n/4 butterflies), as the level kernels' step
    // table runs them: k = 0 no product and 12 additions, k = q/2 four
    // products and 4 + 12 additions, every other k six products and 6 + 12
    const unsigned long q = (unsigned long)T.level_n[lv] / 4, cnt = (unsigned long)T.level_count[lv];
    m += cnt * (4 + 6 * (q - 2));
    a += cnt * (12 + 16 + 18 * (q - 2));
  }
  *mults = m;
  *adds = a;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_diag_tc_error(void) {
  int code = 0;
  CUDA_TRY(mp_tc_take_error(&code));
  return code ? set_err(MPFFT_ECUDA, "a tensor-core wait expired (code %d)", code) : set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_diag_tc_int8_rate(double *macs_per_s) {
  if (!macs_per_s) return set_err(MPFFT_EINVAL, "NULL argument");
  if (int e = device_ready()) return e;
  CUDA_TRY(mp_tc_int8_rate(macs_per_s));
  int code = 0;
  CUDA_TRY(mp_tc_take_error(&code));
  if (code) return set_err(MPFFT_ECUDA, "a tensor-core wait expired (code %d)", code);
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_diag_imad_rate(int wide, double *ops_per_s) {
  if (!ops_per_s) return set_err(MPFFT_EINVAL, "NULL argument");
  if (int e = device_ready()) return e;
  CUDA_TRY(diag_imad_rate(wide, ops_per_s));
  return set_err(MPFFT_OK, "");
}

// ---------------------------------------------------------------------------
// entry point without allocation (static scratch, static_scratch.cu)
// ---------------------------------------------------------------------------

MPFFT_API int mpfft_mp_execute_significands_static(const mpfft_mp_plan *plan, unsigned long batch,
                                                   const uint64_t *d_mant_in, const int64_t *d_exp_in,
                                                   const uint8_t *d_sign_in, int nl_in, uint64_t *d_mant_out,
                                                   int64_t *d_exp_out, uint8_t *d_sign_out, long prec_out,
                                                   unsigned flags, void *stream) {
  if (!plan || !d_mant_in || !d_exp_in || !d_sign_in || !d_mant_out || !d_exp_out || !d_sign_out)
    return set_err(MPFFT_EINVAL, "NULL argument");
  if (plan->host_only) return set_err(MPFFT_EINVAL, "plan was created host-only (conversion only)");
  if (plan->real) return set_err(MPFFT_EINVAL, "real plans have no device-layout entry point");
  if (plan->rank > 1) return set_err(MPFFT_EINVAL, "the static-scratch entry point takes one-dimensional plans");
  if (nl_in < 1 || prec_out < 2) return set_err(MPFFT_EINVAL, "nl_in must be >= 1 and prec_out >= 2");
  if (flags & ~MPFFT_SCALED) return set_err(MPFFT_EINVAL, "flags 0x%x: only MPFFT_SCALED is accepted here", flags);
  {
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != plan->device)
      return set_err(MPFFT_EINVAL, "the current device (%d) is not the plan's device (%d)", dev, plan->device);
  }
  if (batch == 0) return set_err(MPFFT_OK, "");
  if (batch > (unsigned long)INT32_MAX) return set_err(MPFFT_EUNSUPPORTED, "batch too large");
  if (plan->L > kMaxLimbs || mp_tc_used(plan->tabs, plan->L))
    return set_err(MPFFT_EUNSUPPORTED,
                   "the static-scratch entry point supports up to %d limbs on the integer kernels (plan has %d)",
                   kMaxLimbs, plan->L);
  MpPlanView v;
  v.device = plan->device;
  v.N = plan->N;
  v.L = plan->L;
  v.F = plan->F;
  v.tabs = &plan->tabs;
  char msg[200] = "";
  const unsigned shift = (flags & MPFFT_SCALED) ? (unsigned)ilog2(plan->N) : 0u;
  const int rc = mp_execute_significands_static(v, batch, d_mant_in, d_exp_in, d_sign_in, nl_in, d_mant_out,
                                                d_exp_out, d_sign_out, prec_out, shift, (cudaStream_t)stream, msg,
                                                sizeof msg);
  return set_err(rc, "%s", msg);
}

MPFFT_API size_t mpfft_static_scratch_bytes(void) { return static_scratch_bytes(); }

// ===========================================================================
// uneven batches as one graph launch of persistent work-queue kernels
// ===========================================================================

namespace mpfft {

// process-wide caches of FP64 / compensated-tier plans by (n, tier, sub size)
static std::map<std::tuple<unsigned long, int, int>, std::unique_ptr<mpfft_d_plan>> g_ft_cache;

static mpfft_d_plan *ft_cached(unsigned long n, int tier, int sub_max) {
  std::lock_guard<std::mutex> g(g_cache_mu);
  const auto key = std::make_tuple(n, tier, sub_max);
  auto it = g_ft_cache.find(key);
  if (it != g_ft_cache.end()) return it->second.get();
  std::unique_ptr<mpfft_d_plan> p(new mpfft_d_plan);
  if ((tier < 0 ? d_plan_init(p.get(), n, sub_max) : d_plan_init_tier(p.get(), n, tier, sub_max)) != MPFFT_OK)
    return nullptr;
  auto *raw = p.get();
  g_ft_cache[key] = std::move(p);
  return raw;
}

static int form_family(int form) {
  switch (form) {
    case MPFFT_FORM_DOUBLE: return kQueueDouble;
    case MPFFT_FORM_DOUBLE_DOUBLE: return kQueueTierDD;
    case MPFFT_FORM_QUAD_DOUBLE: return kQueueTierQD;
    case MPFFT_FORM_FLOAT_FLOAT: return kQueueTierFF;
    default: return kQueueLimbs;
  }
}
static int family_tier(int fam) {
  return fam == kQueueTierDD ? kTierDD : fam == kQueueTierQD ? kTierQD : fam == kQueueTierFF ? kTierFF : -1;
}
static int family_default_sub(int fam) { return fam == kQueueDouble ? kDSubMax : tier_sub_max(family_tier(fam)); }

// Limb signals of at least this length run as groups instead of in their
// queue: the signals of one (n, L) are transposed into the batch layout, run
// through the batched per-level kernels as one batch, and transposed back.
// One CTA per signal would make the longest signals the end of the launch (a
// 2^16-point signal at 34 limbs is ~10^9 limb products on one SM) and leave
// the products at one CTA's occupancy.
constexpr unsigned long kGroupMinN = 4096;

}  // namespace mpfft

struct mpfft_batch_plan {
  struct Sig {
    unsigned long n = 0;
    long prec = 0;
    int form = 0, L = 0, queue = 0, tab = 0;
    size_t off = 0, bytes = 0;  // place in the arenas
    mpfft_mp_plan *mp = nullptr;
    mpfft_d_plan *fp = nullptr;
  };
  struct Queue {
    int family = 0, L = 0;  // L: limb count of a limb queue
    int threads = 256, sub = 0, ctas = 1;
    std::vector<unsigned long> sigs;  // largest first
    QueueItem *d_items = nullptr;
  };
  // long limb signals (n >= kGroupMinN): the signals of one (n, L) run as one
  // batch of the per-level kernels
  struct Group {
    int L = 0, tab = 0;
    unsigned long n = 0;
    std::vector<unsigned long> sigs;  // contiguous in the arenas, in this order
    const mpfft_mp_plan *mp = nullptr;  // tables of (n, L)
  };
  std::vector<Sig> sig;
  std::vector<Queue> queues;
  std::vector<Group> groups;
  std::vector<QueueTables> tabs;
  QueueTables *d_tabs = nullptr;
  int *d_heads = nullptr;
  unsigned char *d_in = nullptr, *d_out = nullptr, *h_in = nullptr, *h_out = nullptr;
  size_t arena = 0;
  std::vector<long> exps;  // limb signals: block exponents of the last host-array call
  cudaStream_t stream = nullptr;
  uint32_t *d_gs = nullptr;  // groups: two signal-interleaved copies of the largest group
  std::vector<cudaStream_t> qstreams;  // one per queue, then one for the groups
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraphExec_t graph = nullptr;
  int device = -1;
  std::mutex mu;
  void free_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
  ~mpfft_batch_plan() {
    free_graph();
    for (auto &q : queues)
      if (q.d_items) cudaFree(q.d_items);
    if (d_gs) cudaFree(d_gs);
    for (void *p : {(void *)d_tabs, (void *)d_heads, (void *)d_in, (void *)d_out})
      if (p) cudaFree(p);
    for (void *p : {(void *)h_in, (void *)h_out})
      if (p) cudaFreeHost(p);
    for (cudaStream_t s : qstreams) cudaStreamDestroy(s);
    for (cudaEvent_t e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace mpfft {

// (Re)build a queue's tables and items for its current sub size, and its grid.
static int batch_build_queue(mpfft_batch_plan *bp, int qi) {
  auto &Q = bp->queues[qi];
  std::vector<QueueItem> items;
  for (unsigned long i : Q.sigs) {
    auto &s = bp->sig[i];
    if (Q.family != kQueueLimbs) {
      s.fp = ft_cached(s.n, family_tier(Q.family), Q.sub);
      if (!s.fp) return g_err;
      bp->tabs[s.tab].ft = s.fp->tabs;
    }
    items.push_back(QueueItem{bp->d_in + s.off, bp->d_out + s.off, bp->d_tabs + s.tab});
  }
  if (!Q.d_items) CUDA_TRY(cudaMalloc(&Q.d_items, std::max<size_t>(1, items.size()) * sizeof(QueueItem)));
  CUDA_TRY(cudaMemcpy(Q.d_items, items.data(), items.size() * sizeof(QueueItem), cudaMemcpyHostToDevice));
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, bp->device));
  CUDA_TRY(queue_prepare(Q.family, Q.L));
  Q.ctas = (int)std::min<size_t>(Q.sigs.size(), (size_t)sms * queue_ctas_per_sm(Q.family, Q.L, Q.threads));
  return MPFFT_OK;
}

// Capture the whole batch as one graph: zero the queue counters, fork one
// branch per queue, launch its persistent kernel, join.
static int batch_capture(mpfft_batch_plan *bp) {
  bp->free_graph();
  CUDA_TRY(cudaMemcpy(bp->d_tabs, bp->tabs.data(), bp->tabs.size() * sizeof(QueueTables), cudaMemcpyHostToDevice));
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(bp->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemsetAsync(bp->d_heads, 0, std::max<size_t>(1, bp->queues.size()) * sizeof(int), bp->stream);
  if (e == cudaSuccess) e = cudaEventRecord(bp->fork, bp->stream);
  for (size_t q = 0; q < bp->queues.size() && e == cudaSuccess; ++q) {
    const auto &Q = bp->queues[q];
    e = cudaStreamWaitEvent(bp->qstreams[q], bp->fork, 0);
    if (e == cudaSuccess)
      e = queue_launch(Q.family, Q.L, Q.d_items, (int)Q.sigs.size(), bp->d_heads + q, Q.ctas, Q.threads, 1.0,
                       bp->qstreams[q]);
    if (e == cudaSuccess) e = cudaEventRecord(bp->joins[q], bp->qstreams[q]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(bp->stream, bp->joins[q], 0);
  }
  // the groups, one after another on one branch (each fills the GPU): the
  // group's signals (contiguous, 2 L n words each) transposed into the
  // batch layout, the batched transform, transposed back
  if (!bp->groups.empty() && e == cudaSuccess) {
    const size_t b = bp->queues.size();
    const cudaStream_t st = bp->qstreams[b];
    e = cudaStreamWaitEvent(st, bp->fork, 0);
    for (const auto &G : bp->groups) {
      if (e != cudaSuccess) break;
      const long long W = 2LL * G.L * (long long)G.n, ns = (long long)G.sigs.size();
      const size_t off = bp->sig[G.sigs[0]].off;
      uint32_t *a = bp->d_gs, *c = bp->d_gs + (size_t)(W * ns);
      e = transpose_launch(reinterpret_cast<const uint32_t *>(bp->d_in + off), a, 1, ns, W, 1, st);
      if (e == cudaSuccess) e = mp_run_transform(G.L, G.mp->tabs, a, c, (int)ns, st, nullptr, nullptr);
      if (e == cudaSuccess) e = transpose_launch(c, reinterpret_cast<uint32_t *>(bp->d_out + off), 1, W, ns, 1, st);
    }
    if (e == cudaSuccess) e = cudaEventRecord(bp->joins[b], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(bp->stream, bp->joins[b], 0);
  }
  const cudaError_t ce = cudaStreamEndCapture(bp->stream, &g);
  if (e == cudaSuccess) e = ce;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&bp->graph, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    bp->graph = nullptr;
    cudaGetLastError();
    return set_err(MPFFT_ECUDA, "capturing the batch graph: %s", cudaGetErrorString(e));
  }
  return MPFFT_OK;
}

// ---- autotuning of the queue launches --------------------------------------
//
// Per queue the choices are the CTA size and, for the floating forms, the
// largest shared-memory sub-transform (a smaller one lets more CTAs share an
// SM at the price of more levels in global memory); neither changes any
// result.  mpfft_batch_autotune times every candidate on the batch's own
// queues and records the fastest per (device, queue kind, length mix) in a
// JSON file -- MPFFT_AUTOTUNE_FILE, else $XDG_CACHE_HOME/mpfft_b200/autotune.json,
// else ~/.cache/mpfft_b200/autotune.json -- which later plans read.

static std::string tune_path() {
  if (const char *p = getenv("MPFFT_AUTOTUNE_FILE")) return p;
  std::string base;
  if (const char *x = getenv("XDG_CACHE_HOME")) base = x;
  else if (const char *h = getenv("HOME")) base = std::string(h) + "/.cache";
  else return "";
  return base + "/mpfft_b200/autotune.json";
}

static std::string tune_key(const mpfft_batch_plan *bp, int qi) {
  const auto &Q = bp->queues[qi];
  cudaDeviceProp prop;
  std::string dev = cudaGetDeviceProperties(&prop, bp->device) == cudaSuccess ? prop.name : "gpu";
  for (auto &c : dev)
    if (c == '"' || c == ' ') c = '_';
  // length mix: the signal count per log2 N
  int hist[32] = {};
  for (unsigned long i : Q.sigs) ++hist[ilog2(bp->sig[i].n)];
  std::string mix;
  for (int l = 0; l < 32; ++l)
    if (hist[l]) mix += std::to_string(l) + "x" + std::to_string(hist[l]) + ".";
  return dev + "/" + std::to_string(Q.family) + "/" + std::to_string(Q.L) + "/" + mix;
}

// entries "key": [threads, sub] of the tune file
static std::map<std::string, std::pair<int, int>> tune_load() {
  std::map<std::string, std::pair<int, int>> m;
  const std::string path = tune_path();
  FILE *f = path.empty() ? nullptr : fopen(path.c_str(), "r");
  if (!f) return m;
  std::string txt;
  char buf[4096];
  for (size_t k; (k = fread(buf, 1, sizeof buf, f)) > 0;) txt.append(buf, k);
  fclose(f);
  for (size_t p = 0; (p = txt.find('"', p)) != std::string::npos;) {
    const size_t e = txt.find('"', p + 1);
    if (e == std::string::npos) break;
    const std::string key = txt.substr(p + 1, e - p - 1);
    int t = 0, s = 0;
    if (sscanf(txt.c_str() + e + 1, " : [ %d , %d ]", &t, &s) == 2) m[key] = std::make_pair(t, s);
    p = e + 1;
  }
  return m;
}

static void tune_save(const std::map<std::string, std::pair<int, int>> &m) {
  const std::string path = tune_path();
  if (path.empty()) return;
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {  // create the directory chain
    for (size_t p = 1; p <= slash; ++p)
      if (path[p] == '/' || p == slash) mkdir(path.substr(0, p == slash ? slash : p).c_str(), 0755);
  }
  const std::string tmp = path + ".tmp" + std::to_string(getpid());
  FILE *f = fopen(tmp.c_str(), "w");
  if (!f) return;
  fprintf(f, "{\n");
  size_t k = 0;
  for (auto &kv : m) fprintf(f, "  \"%s\": [%d, %d]%s\n", kv.first.c_str(), kv.second.first, kv.second.second,
                             ++k < m.size() ? "," : "");
  fprintf(f, "}\n");
  fclose(f);
  rename(tmp.c_str(), path.c_str());
}

}  // namespace mpfft

MPFFT_API int mpfft_batch_plan_create(mpfft_batch_plan **plan, unsigned long count, const unsigned long *n,
                                      const long *prec, unsigned flags) {
  if (!plan || !n || !prec) return set_err(MPFFT_EINVAL, "NULL argument");
  *plan = nullptr;
  if (count == 0) return set_err(MPFFT_EINVAL, "empty batch");
  if (int e = device_ready()) return e;
  std::unique_ptr<mpfft_batch_plan> bp(new (std::nothrow) mpfft_batch_plan);
  if (!bp) return set_err(MPFFT_ENOMEM, "out of host memory");
  CUDA_TRY(cudaGetDevice(&bp->device));
  bp->sig.resize(count);
  std::map<std::pair<int, int>, int> qindex;              // (family, L) -> queue
  std::map<std::pair<int, unsigned long>, int> gindex;    // (L, n) -> group
  std::map<std::tuple<int, int, unsigned long>, int> tindex;  // (family, L, n) -> tables
  for (unsigned long i = 0; i < count; ++i) {
    auto &s = bp->sig[i];
    if (!is_pow2(n[i])) return set_err(MPFFT_EINVAL, "n[%lu]=%lu is not a power of two", i, n[i]);
    if (prec[i] < 2) return set_err(MPFFT_EINVAL, "signal %lu: precision %ld < 2", i, prec[i]);
    if (n[i] > (1UL << 22)) return set_err(MPFFT_EUNSUPPORTED, "signal %lu: n=%lu above the queue limit 2^22", i, n[i]);
    s.n = n[i];
    s.prec = prec[i];
    const int ff = (flags & MPFFT_PLAN_NATIVE_TIERS)  ? float_form_for(prec[i], true)
                   : (flags & MPFFT_PLAN_FLOAT_TIERS) ? float_form_for(prec[i])
                                                      : -1;
    int fam;
    if (ff >= 0) {
      s.form = ff;
      fam = form_family(ff);
      const int K = fam == kQueueDouble ? 1 : tier_words(family_tier(fam));
      const size_t wb = fam == kQueueDouble ? 8 : tier_word_bytes(family_tier(fam));
      s.bytes = (size_t)2 * K * s.n * wb;
    } else {
      s.form = MPFFT_FORM_LIMBS;
      fam = kQueueLimbs;
      s.L = mp_limbs_for(s.n, s.prec);
      if (s.L > kMaxLimbs)
        return set_err(MPFFT_EUNSUPPORTED, "signal %lu: %d limbs; the queue kernels take up to %d", i, s.L,
                       kMaxLimbs);
      s.mp = mp_cached(s.n, s.prec);
      if (!s.mp) return g_err;
      s.bytes = (size_t)2 * s.L * s.n * 4;
    }
    const auto tk = std::make_tuple(fam, s.L, s.n);
    if (!tindex.count(tk)) {
      tindex[tk] = (int)bp->tabs.size();
      QueueTables t;
      t.N = (int)s.n;
      if (fam == kQueueLimbs) {
        t.tree = s.mp->tabs;
        t.tw = s.mp->tabs.tw;
        t.dneg = s.mp->tabs.dneg;
      }
      bp->tabs.push_back(t);
    }
    s.tab = tindex[tk];
    if (fam == kQueueLimbs && s.n >= kGroupMinN) {
      const auto gk = std::make_pair(s.L, s.n);
      if (!gindex.count(gk)) {
        gindex[gk] = (int)bp->groups.size();
        mpfft_batch_plan::Group G;
        G.L = s.L;
        G.n = s.n;
        G.tab = s.tab;
        G.mp = s.mp;
        bp->groups.push_back(G);
      }
      s.queue = -1;
      bp->groups[gindex[gk]].sigs.push_back(i);
      continue;
    }
    const auto qk = std::make_pair(fam, s.L);
    if (!qindex.count(qk)) {
      qindex[qk] = (int)bp->queues.size();
      mpfft_batch_plan::Queue Q;
      Q.family = fam;
      Q.L = s.L;
      Q.threads = fam == kQueueLimbs ? 128 : 256;
      Q.sub = fam == kQueueLimbs ? 0 : family_default_sub(fam);
      bp->queues.push_back(Q);
    }
    s.queue = qindex[qk];
    bp->queues[s.queue].sigs.push_back(i);
  }
  // largest first within each queue; arena offsets queue by queue (256-byte aligned)
  for (auto &Q : bp->queues) {
    std::stable_sort(Q.sigs.begin(), Q.sigs.end(), [&](unsigned long a, unsigned long b) {
      const auto &x = bp->sig[a], &y = bp->sig[b];
      return (double)x.n * (ilog2(x.n) + 1) > (double)y.n * (ilog2(y.n) + 1);
    });
    for (unsigned long i : Q.sigs) {
      bp->sig[i].off = bp->arena;
      bp->arena += (bp->sig[i].bytes + 255) & ~(size_t)255;
    }
  }
  for (auto &G : bp->groups)
    for (unsigned long i : G.sigs) {
      bp->sig[i].off = bp->arena;
      bp->arena += (bp->sig[i].bytes + 255) & ~(size_t)255;
    }
  CUDA_TRY(cudaMalloc(&bp->d_tabs, bp->tabs.size() * sizeof(QueueTables)));
  CUDA_TRY(cudaMalloc(&bp->d_heads, std::max<size_t>(1, bp->queues.size()) * sizeof(int)));
  if (dev_alloc((void **)&bp->d_in, bp->arena) != cudaSuccess || dev_alloc((void **)&bp->d_out, bp->arena) != cudaSuccess) {
    cudaGetLastError();
    return set_err(MPFFT_ENOMEM, "cannot allocate %zu-byte signal arenas", bp->arena);
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&bp->stream, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&bp->fork, cudaEventDisableTiming));
  const auto tuned = tune_load();
  for (size_t q = 0; q < bp->queues.size(); ++q) {
    cudaStream_t s;
    cudaEvent_t e;
    CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    bp->qstreams.push_back(s);
    CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    bp->joins.push_back(e);
    auto it = tuned.find(tune_key(bp.get(), (int)q));
    if (it != tuned.end()) {
      bp->queues[q].threads = it->second.first;
      if (bp->queues[q].family != kQueueLimbs) bp->queues[q].sub = it->second.second;
    }
    if (int e2 = batch_build_queue(bp.get(), (int)q)) return e2;
  }
  if (!bp->groups.empty()) {
    cudaStream_t s;
    cudaEvent_t e;
    CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    bp->qstreams.push_back(s);
    CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    bp->joins.push_back(e);
    size_t most = 0;
    for (const auto &G : bp->groups) most = std::max(most, (size_t)2 * G.L * G.n * G.sigs.size());
    if (dev_alloc((void **)&bp->d_gs, 2 * most * 4) != cudaSuccess) {
      cudaGetLastError();
      return set_err(MPFFT_ENOMEM, "cannot allocate %zu bytes of group scratch", 2 * most * 4);
    }
  }
  if (int e = batch_capture(bp.get())) return e;
  *plan = bp.release();
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_batch_plan_destroy(mpfft_batch_plan *plan) {
  delete plan;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_batch_signal_format(const mpfft_batch_plan *plan, unsigned long i, int *form, int *words,
                                        size_t *offset, size_t *bytes) {
  if (!plan || !form || !words || !offset || !bytes) return set_err(MPFFT_EINVAL, "NULL argument");
  if (i >= plan->sig.size()) return set_err(MPFFT_EINVAL, "signal %lu out of range", i);
  const auto &s = plan->sig[i];
  *form = s.form;
  *words = s.form == MPFFT_FORM_LIMBS ? s.L : (s.form == MPFFT_FORM_DOUBLE ? 1 : tier_words(family_tier(form_family(s.form))));
  *offset = s.off;
  *bytes = s.bytes;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_batch_arenas(const mpfft_batch_plan *plan, void **d_in, void **d_out, size_t *bytes) {
  if (!plan || !d_in || !d_out || !bytes) return set_err(MPFFT_EINVAL, "NULL argument");
  *d_in = plan->d_in;
  *d_out = plan->d_out;
  *bytes = plan->arena;
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_batch_execute_device(mpfft_batch_plan *plan, void *stream) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> g(plan->mu);
  CUDA_TRY(cudaGraphLaunch(plan->graph, (cudaStream_t)stream));
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_batch_execute(mpfft_batch_plan *plan, mpfr_t *const *inr, mpfr_t *const *ini,
                                  mpfr_t *const *outr, mpfr_t *const *outi, unsigned flags) {
  if (!plan || !inr || !ini || !outr || !outi) return set_err(MPFFT_EINVAL, "NULL argument");
  if (flags & ~(MPFFT_SCALED | MPFFT_INVERSE)) return set_err(MPFFT_EINVAL, "flags 0x%x", flags);
  if (flags & MPFFT_INVERSE) {  // ifft(X) = swap(FFT(swap(X)))
    std::swap(inr, ini);
    std::swap(outr, outi);
  }
  std::lock_guard<std::mutex> g(plan->mu);
  const unsigned long count = plan->sig.size();
  for (unsigned long i = 0; i < count; ++i)
    if (!inr[i] || !ini[i] || !outr[i] || !outi[i]) return set_err(MPFFT_EINVAL, "NULL array of signal %lu", i);
  if (!plan->h_in) {
    if (host_alloc((void **)&plan->h_in, plan->arena) != cudaSuccess ||
        host_alloc((void **)&plan->h_out, plan->arena) != cudaSuccess) {
      cudaGetLastError();
      return set_err(MPFFT_ENOMEM, "cannot allocate %zu bytes of pinned staging", plan->arena);
    }
  }
  plan->exps.assign(count, 0);
  // inputs -> arena layout (limb planes with a block exponent, or tier words)
  std::atomic<int> status{0};
  std::atomic<unsigned long> bad_sig{0};
  parallel_for((long)count, 1, [&](long a, long b) {
    mpfr_t t;
    mpfr_init2(t, 64);
    for (long i = a; i < b; ++i) {
      const auto &s = plan->sig[i];
      IoShape io = io_signals(s.n, 1);
      if (s.form == MPFFT_FORM_LIMBS) {
        mpfr_t *bi[2] = {inr[i], ini[i]};
        io.base[0] = &bi[0];
        io.base[1] = &bi[1];
        if (mp_pack_impl(s.mp, 1, io, nullptr, nullptr, reinterpret_cast<uint32_t *>(plan->h_in + s.off),
                         &plan->exps[i]) != MPFFT_OK) {
          status.fetch_or(1);
          bad_sig.store(i);
        }
      } else {
        const int K = s.form == MPFFT_FORM_DOUBLE ? 1 : tier_words(family_tier(form_family(s.form)));
        const bool fl = s.form == MPFFT_FORM_FLOAT_FLOAT;
        long emin, emax;
        tier_window(s.fp, &emin, &emax);
        int st = 0;
        for (unsigned long q = 0; q < s.n; ++q)
          for (int c = 0; c < 2; ++c)
            st |= mpfr_to_words((c ? ini : inr)[i][q], t, K, fl, emin, emax, plan->h_in + s.off,
                                (size_t)c * K * s.n + q, s.n);
        if (st) {
          status.fetch_or(st);
          bad_sig.store(i);
        }
      }
    }
    mpfr_clear(t);
  });
  if (status.load() & 1) return set_err(MPFFT_ENONFINITE, "signal %lu holds NaN or infinity", bad_sig.load());
  if (status.load() & 2)
    return set_err(MPFFT_EUNSUPPORTED, "signal %lu has exponents outside its floating tier's window",
                   bad_sig.load());
  CUDA_TRY(cudaMemcpyAsync(plan->d_in, plan->h_in, plan->arena, cudaMemcpyHostToDevice, plan->stream));
  CUDA_TRY(cudaGraphLaunch(plan->graph, plan->stream));
  CUDA_TRY(cudaMemcpyAsync(plan->h_out, plan->d_out, plan->arena, cudaMemcpyDeviceToHost, plan->stream));
  CUDA_TRY(cudaStreamSynchronize(plan->stream));
  parallel_for((long)count, 1, [&](long a, long b) {
    mpfr_t acc;
    mpfr_init2(acc, 320);
    for (long i = a; i < b; ++i) {
      const auto &s = plan->sig[i];
      const long shift = (flags & MPFFT_SCALED) ? ilog2(s.n) : 0;
      IoShape io = io_signals(s.n, 1);
      if (s.form == MPFFT_FORM_LIMBS) {
        mpfr_t *bo[2] = {outr[i], outi[i]};
        io.base[0] = &bo[0];
        io.base[1] = &bo[1];
        mp_unpack_impl(s.mp, 1, reinterpret_cast<const uint32_t *>(plan->h_out + s.off), &plan->exps[i], io, nullptr,
                       nullptr, shift);
      } else {
        const int K = s.form == MPFFT_FORM_DOUBLE ? 1 : tier_words(family_tier(form_family(s.form)));
        const bool fl = s.form == MPFFT_FORM_FLOAT_FLOAT;
        for (unsigned long q = 0; q < s.n; ++q)
          for (int c = 0; c < 2; ++c)
            words_to_mpfr(plan->h_out + s.off, (size_t)c * K * s.n + q, s.n, K, fl, shift, acc, (c ? outi : outr)[i][q]);
      }
    }
    mpfr_clear(acc);
  });
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_batch_autotune(mpfft_batch_plan *plan, int save) {
  if (!plan) return set_err(MPFFT_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> g(plan->mu);
  auto table = tune_load();
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  for (size_t q = 0; q < plan->queues.size(); ++q) {
    auto &Q = plan->queues[q];
    std::vector<std::pair<int, int>> cand;
    for (int th : {128, 256}) {
      if (Q.family == kQueueLimbs) {
        cand.emplace_back(th, 0);
        continue;
      }
      const int top = family_default_sub(Q.family);
      for (int sub : {top, top / 2, top / 4}) cand.emplace_back(th, sub);
    }
    float best = 1e30f;
    std::pair<int, int> pick(Q.threads, Q.sub);
    for (auto &c : cand) {
      Q.threads = c.first;
      Q.sub = c.second;
      if (int e = batch_build_queue(plan, (int)q)) return e;
      CUDA_TRY(cudaMemcpy(plan->d_tabs, plan->tabs.data(), plan->tabs.size() * sizeof(QueueTables),
                          cudaMemcpyHostToDevice));
      float ms = 0, tot = 0;
      for (int rep = 0; rep < 4; ++rep) {
        CUDA_TRY(cudaMemsetAsync(plan->d_heads + q, 0, sizeof(int), plan->stream));
        CUDA_TRY(cudaEventRecord(e0, plan->stream));
        CUDA_TRY(queue_launch(Q.family, Q.L, Q.d_items, (int)Q.sigs.size(), plan->d_heads + q, Q.ctas, Q.threads, 1.0,
                              plan->stream));
        CUDA_TRY(cudaEventRecord(e1, plan->stream));
        CUDA_TRY(cudaEventSynchronize(e1));
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (rep) tot += ms;  // the first run warms the caches
      }
      if (tot < best) {
        best = tot;
        pick = c;
      }
    }
    Q.threads = pick.first;
    Q.sub = pick.second;
    if (int e = batch_build_queue(plan, (int)q)) return e;
    table[tune_key(plan, (int)q)] = pick;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (int e = batch_capture(plan)) return e;
  if (save) tune_save(table);
  return set_err(MPFFT_OK, "");
}

MPFFT_API int mpfft_batch_queue_info(const mpfft_batch_plan *plan, int q, int *family, int *limbs, int *threads,
                                     int *sub, int *signals) {
  if (!plan || !family || !limbs || !threads || !sub || !signals) return set_err(MPFFT_EINVAL, "NULL argument");
  if (q < 0) return (int)(plan->queues.size() + plan->groups.size());
  if ((size_t)q >= plan->queues.size() + plan->groups.size()) return set_err(MPFFT_EINVAL, "queue %d out of range", q);
  if ((size_t)q >= plan->queues.size()) {  // a group of long limb signals: threads 0, sub = its length
    const auto &G = plan->groups[q - plan->queues.size()];
    *family = kQueueLimbs;
    *limbs = G.L;
    *threads = 0;
    *sub = (int)G.n;
    *signals = (int)G.sigs.size();
    return set_err(MPFFT_OK, "");
  }
  const auto &Q = plan->queues[q];
  *family = Q.family;
  *limbs = Q.L;
  *threads = Q.threads;
  *sub = Q.sub;
  *signals = (int)Q.sigs.size();
  return set_err(MPFFT_OK, "");
}
