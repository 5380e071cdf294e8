// Internal declarations shared by the host library and the kernel files.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace mpfft {

// One leaf of the split-radix tree (a node of size n <= 4 for the mp tier,
// n <= 16 for the FP64 tier): its input elements are x[(sn + j*s)], j < n,
// with the j = 0 element wrapped to sn + N when sn < 0, and its outputs go to
// y[out .. out+n).
struct Leaf {
  int out;
  int sn;
  int s;
  int n;
};
using MpLeaf = Leaf;

constexpr int kMaxLevels = 32;

// The breadth-first schedule of one transform size: every leaf, then for each
// node size n = first_level_n .. N (doubling) the output offsets of all nodes
// of that size.  Pointers are device pointers; the small arrays are host
// copies of the per-level metadata.
struct TreeTables {
  int N = 0;
  int nleaves = 0;
  int leaf_count[5] = {};  // leaves of size 1, 2, 4 (index = size; others unused)
  const Leaf *leaves = nullptr;
  int nlevels = 0;
  int level_n[kMaxLevels] = {};
  int level_start[kMaxLevels] = {};
  int level_count[kMaxLevels] = {};
  const int *node_off = nullptr;
  // for a launch of levels lv and lv+1 together (mp_level_pair_kernel): the
  // nodes of size level_n[lv] that are not the first child of a node of size
  // level_n[lv+1], at pair_nodes + pair_start[lv] (pair_count[lv] of them)
  const int *pair_nodes = nullptr;
  int pair_start[kMaxLevels] = {};
  int pair_count[kMaxLevels] = {};
};

struct MpDeviceTables : TreeTables {
  const uint32_t *tw = nullptr;   // [3][L][tws*N/4]: cos, cos+sin, |cos-sin| magnitudes
  const uint8_t *dneg = nullptr;  // [tws*N/4]: sign of cos-sin
  int tws = 1;  // the table is built for tws*N points (2 for a real transform of 2N points)
  int tc = 1;   // twiddle products on the tensor cores (mp_tc_kernels.cu): 0 never, 1 from
                // kTcMinLimbs limbs, 2 from kTcForceMinLimbs limbs
};

// Schedule of one shared-memory sub-transform of size `size` (FP64 tier):
// perm[j] = the position that element j of the sub-transform's input sequence
// takes (the DIT input order), then the leaves (n <= 16, in place over
// positions [out, out+n)) and the levels of the size-`size` tree.
struct SubSchedule {
  int size = 0;
  const int *perm = nullptr;
  int nleaves = 0;
  int nleaf16 = 0, nleaf8 = 0;   // leaves are sorted: 16-point, 8-point, then smaller
  const Leaf *leaves = nullptr;  // .sn/.s unused: inputs are already in place
  int nlevels = 0;
  int level_n[kMaxLevels] = {};
  int level_start[kMaxLevels] = {};
  int level_count[kMaxLevels] = {};
  const int *node_off = nullptr;
  // for levels lv and lv+1 run in one pass (each node of size level_n[lv+1]
  // with its first child): the nodes of size level_n[lv] that are not a first
  // child, at pair_nodes + pair_start[lv] (pair_count[lv] of them)
  const int *pair_nodes = nullptr;
  int pair_start[kMaxLevels] = {};
  int pair_count[kMaxLevels] = {};
};

// root of a shared-memory sub-transform: input elements x[(sn + j*s)] (j = 0
// wrapped to sn + N when sn < 0), outputs y[out .. out+size)
struct SubRoot {
  int sn, s, out, size;
};

struct DDeviceTables {
  int N = 0;
  const double *wr = nullptr;  // [N/4] cos(2 pi k/N)
  const double *wi = nullptr;  // [N/4] sin(2 pi k/N)
  const double *wrl = nullptr, *wil = nullptr;  // double-double plans: low parts of wr, wi
  // compensated tiers (float_tier_kernels.cu): the words of cos and sin of
  // 2 pi k/N, k < N/4 (double-double: 2, quad-double: 4, float-float: 1 double)
  const double *tw_cos[4] = {}, *tw_sin[4] = {};
  double c8 = 0, c16a = 0, c16b = 0, c16c = 0, c16d = 0;
  // shared-memory sub-transforms (sizes T and T/2) ...
  int nroots = 0;
  const SubRoot *roots = nullptr;
  SubSchedule sub[2];
  // ... and the levels above them, in global memory
  TreeTables upper;
};

constexpr int kMaxDevices = 64;
constexpr int kDSubMax = 4096;  // FP64: largest shared-memory sub-transform (64 KB)
constexpr int kDDSubMax = 2048; // double-double: largest shared-memory sub-transform (64 KB)
constexpr int kQDSubMax = 1024; // quad-double (64 KB)
constexpr int kFFSubMax = 4096; // float-float (64 KB)
// compensated floating-point tiers (float_tier_kernels.cu)
enum { kTierDD = 0, kTierQD = 1, kTierFF = 2 };

// What the static-scratch entry point needs to know about a plan.
struct MpPlanView {
  int device = -1;
  unsigned long N = 0;
  int L = 0;
  long F = 0;
  const MpDeviceTables *tabs = nullptr;
};

// largest limb count with register-resident kernels; above it (up to
// kMaxLimbsBig) the streaming kernels of mp_big_kernels.cu run
constexpr int kMaxLimbs = 34;
constexpr int kMaxLimbsBig = 520;
constexpr int kMinLimbs = 2;
// limb counts whose level kernels run their twiddle products as int8 tensor-core
// GEMMs: every count above the register kernels up to 260 (P from about 1050
// to 8200 bits at N = 1024); measured faster than the streaming integer kernels
// over the whole range
constexpr int kTcMinLimbs = 35;
constexpr int kTcMaxLimbs = 260;
constexpr int kTcForceMinLimbs = 8;

// launch_ms (optional, host array of >= 1 + nlevels floats): when non-null,
// each launch is bracketed by events on `s` and its duration written there
// (the call then synchronizes); used by benchmarks to attribute time.
// Optional per-launch timing with events on the launch stream.
struct LaunchTimer {
  float *ms;
  cudaStream_t s;
  cudaEvent_t ev[2 * (kMaxLevels + 1)] = {};
  int n = 0;
  LaunchTimer(float *ms_, cudaStream_t s_) : ms(ms_), s(s_) {}
  void begin() {
    if (!ms) return;
    cudaEventCreate(&ev[2 * n]);
    cudaEventCreate(&ev[2 * n + 1]);
    cudaEventRecord(ev[2 * n], s);
  }
  void end() {
    if (!ms) return;
    cudaEventRecord(ev[2 * n + 1], s);
    ++n;
  }
  // an entry without a launch of its own (a level run together with the previous one): 0 ms
  void none() {
    if (!ms) return;
    ++n;
  }
  ~LaunchTimer() {
    if (!ms) return;
    cudaStreamSynchronize(s);
    for (int i = 0; i < n; ++i) {
      ms[i] = 0.0f;
      if (!ev[2 * i]) continue;
      cudaEventElapsedTime(&ms[i], ev[2 * i], ev[2 * i + 1]);
      cudaEventDestroy(ev[2 * i]);
      cudaEventDestroy(ev[2 * i + 1]);
    }
  }
};

// big_scratch: device buffer of mp_big_scratch_words(T, L, B) words, needed
// (and only used) when L > kMaxLimbs.
cudaError_t mp_run_transform(int L, const MpDeviceTables &T, const uint32_t *in, uint32_t *out, int B,
                             cudaStream_t s, float *launch_ms = nullptr, uint32_t *big_scratch = nullptr);
size_t mp_big_scratch_words(const MpDeviceTables &T, int L, int B);
cudaError_t mp_big_run_transform(int L, const MpDeviceTables &T, const uint32_t *in, uint32_t *out, int B,
                                 uint32_t *scratch, cudaStream_t s, float *launch_ms);
cudaError_t diag_imad_rate(int wide, double *ops_per_s);
// tensor-core level kernels (kTcMinLimbs <= L <= kTcMaxLimbs); scratch of
// mp_tc_scratch_words words
size_t mp_tc_scratch_words(const MpDeviceTables &T, int L, int B);
cudaError_t mp_tc_run_levels(int L, const MpDeviceTables &T, uint32_t *out, int B, uint32_t *scratch, cudaStream_t s,
                             LaunchTimer &timer);
// diagnostics: B signed products x * w through the tensor-core product
cudaError_t mp_tc_mul(int L, int B, const uint32_t *x, const uint32_t *w, uint32_t *out, cudaStream_t s);
// reads and clears the device-side error flag of the tensor-core kernels
cudaError_t mp_tc_take_error(int *code);
// measured int8 tensor-core rate (multiply-adds per second, kind::i8 MMAs)
cudaError_t mp_tc_int8_rate(double *macs_per_s);
// limit of the tensor-core kernels' waits on their own MMAs (ns); tests only
cudaError_t mp_tc_set_wait_limit(unsigned long long ns);
size_t mp_tc_smem_bytes(int L);
inline bool mp_tc_used(const MpDeviceTables &T, int L) {
  return T.tc && L >= (T.tc == 2 ? kTcForceMinLimbs : kTcMinLimbs) && L <= kTcMaxLimbs;
}
// Split step of a real transform of 2M points (L <= kMaxLimbs; tw/dneg: the
// table of a 2M-point plan).  forward: Z (M points) -> 2X (M+1 points);
// otherwise half spectrum X (M+1 points) -> 2Z with its planes exchanged.
cudaError_t mp_real_split(bool forward, int L, const uint32_t *in, uint32_t *out, int M, int B, const uint32_t *tw,
                          const uint8_t *dneg, cudaStream_t s);

// GPU-side conversion between MPFR significands and limb planes.  Component
// (c, p, b) is index (c*N + p)*B + b of the mant/ex/sg arrays; ex = INT64_MIN
// marks zero.  import computes the per-signal block exponents into es[B].
// sig_major: component (c, p, b) at index (b*2 + c)*N + p instead
cudaError_t mp_import_launch(const uint64_t *mant, const int64_t *ex, const uint8_t *sg, int nl, int N, int B,
                             int L, long F, int64_t *es, uint32_t *planes, cudaStream_t s, bool sig_major = false);
cudaError_t mp_export_launch(const uint32_t *planes, int N, int B, int L, const int64_t *es, long F_plus_shift,
                             long prec, int nlo, uint64_t *out, int64_t *oex, uint8_t *osg, cudaStream_t s,
                             bool sig_major = false);
// out[m][c][r][e] = in[m][r][c][e]: nmat matrices of R x C elements of E words
cudaError_t transpose_launch(const uint32_t *in, uint32_t *out, long long nmat, long long R, long long C, int E,
                             cudaStream_t s);
// FP64 layout: word (c, b, p) at base[(c*B + b)*N + p]  (signal-contiguous)
// swap_in / swap_out: read the input's / write the output's real and imaginary
// planes exchanged (both: the unscaled inverse, swap(FFT(swap(x))))
cudaError_t d_run_transform(const DDeviceTables &T, const double *in, double *out, int B, double scale,
                            cudaStream_t s, bool swap_in = false, bool swap_out = false);
// double-double tier (dd_kernels.cu); layout word (c, h, b, p) at ((c*2 + h)*B + b)*N + p
cudaError_t dd_run_transform(const DDeviceTables &T, const double *in, double *out, int B, double scale,
                             cudaStream_t s, bool swap_in = false, bool swap_out = false);
// any compensated tier; layout word (c, h, b, p) at ((c*K + h)*B + b)*N + p with
// K = tier_words(tier) words of tier_word_bytes(tier) bytes per real component
cudaError_t tier_run_transform(int tier, const DDeviceTables &T, const void *in, void *out, int B, double scale,
                               cudaStream_t s, bool swap_in = false, bool swap_out = false);
int tier_words(int tier);
size_t tier_word_bytes(int tier);
int tier_sub_max(int tier);
// split step of the FP64 real transforms (n = 2M real points), d_kernels.cu
cudaError_t d_real_split(bool forward, const double *in, double *out, int M, int B, const double *wc,
                         const double *ws, double scale, cudaStream_t s);

// ---------------------------------------------------------------------------
// persistent work-queue kernels (queue_kernels.cu)
// ---------------------------------------------------------------------------
// What one CTA needs to transform one signal of a given form and length:
// limb forms use the breadth-first schedule and twiddles of an N-point mp
// plan (a single signal: limb planes [c][i][p]); floating forms use the
// sub-transform roots, schedules, upper levels and twiddles of an N-point
// FP64 / compensated-tier plan (layout [c][h][p]).
struct QueueTables {
  int N = 0;
  TreeTables tree;                 // limb forms
  const uint32_t *tw = nullptr;    // limb forms: [3][L][N/4]
  const uint8_t *dneg = nullptr;
  DDeviceTables ft;                // floating forms
};
// one signal of a queue: its input and output in the form's device layout
struct QueueItem {
  const void *in;
  void *out;
  const QueueTables *tab;
};
// Queue families: limb forms (one kernel per limb count), FP64, and the
// compensated tiers.  A launch runs `ctas` persistent CTAs of `threads`
// threads that pop items[0 .. nitems) through *head (an atomic counter the
// caller zeroes before the launch) until the queue is empty; no CTA ever
// waits for another.
enum { kQueueLimbs = 0, kQueueDouble = 1, kQueueTierDD = 2, kQueueTierQD = 3, kQueueTierFF = 4 };
cudaError_t queue_launch(int family, int L, const QueueItem *items, int nitems, int *head, int ctas, int threads,
                         double scale, cudaStream_t s);
// largest resident CTAs per SM of a family's kernel at `threads` threads
int queue_ctas_per_sm(int family, int L, int threads);
cudaError_t queue_prepare(int family, int L);  // kernel attributes, before any stream capture

// Import -> transform -> export of device-resident MPFR fields with all
// working storage in a file-scope device array (static_scratch.cu).  Returns an
// MPFFT_* status and writes a message on failure.
int mp_execute_significands_static(const MpPlanView &v, unsigned long batch, const uint64_t *d_mant_in,
                                   const int64_t *d_exp_in, const uint8_t *d_sign_in, int nl_in,
                                   uint64_t *d_mant_out, int64_t *d_exp_out, uint8_t *d_sign_out, long prec_out,
                                   unsigned scaled_shift, cudaStream_t stream, char *msg, size_t msglen);
size_t static_scratch_bytes();

}  // namespace mpfft
