// Multiprecision conjugate-pair split-radix 2/4 DIT FFT kernels (sm_100a).
//
// The reference computes the transform by depth-first recursion
// (lab/parallel/mp/parallel_mp_fft2.c:121-328): a node of size n runs its
// n/2 child on even samples, two n/4 children on samples 4m+1 and 4m-1 (the
// conjugate pair), then one L-shaped butterfly per k in [0, n/4).  Here the
// same tree is executed breadth-first: one launch runs every leaf (n = 4, 2 or
// 1), then one launch per node size n = 8, 16, ..., N runs every butterfly of
// every node of that size (for large batches one launch per two node sizes,
// mp_level_pair_kernel).  All nodes of one size are independent, so each
// launch is one flat grid over (node, k, signal); consecutive threads are
// consecutive signals of a batch (or consecutive k for a single signal),
// which makes every limb-plane access a coalesced 128-byte transaction and,
// for batches, makes the twiddle operand warp-uniform.
//
// Data layout (limb planes): word (c, i, p, b) of a batch of B signals of
// N points, c = 0 real / 1 imaginary, limb i < L, at
//   base[((c*L + i)*N + p)*B + b].
#include <cstdint>

#include "mp_bfly.cuh"
#include "mp_lanes.cuh"
#include "mp_limbs.cuh"
#include "mpfft_internal.h"

namespace mpfft {

// Programmatic dependent launch, for the kernels of launches too small to fill
// the GPU (one signal: a few microseconds of work each, comparable to the
// launch latency between them).  Launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, such a kernel may be
// scheduled while its predecessor in the stream still runs: it lets its own
// successor be scheduled at once (pdl_release) and, before its first access
// to global data that earlier work reads or writes, waits (pdl_wait) until the
// predecessor grid has completed and its memory is visible.  Plan constants
// (leaf table, node offsets, twiddles) are read before the wait.  Without the
// attribute both instructions do nothing.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---------------------------------------------------------------------------
// leaves: size-1, size-2 and size-4 DFTs of strided input subsequences
// (reference base cases, parallel_mp_fft2.c:125-177).  Exact in fixed point.
// ---------------------------------------------------------------------------
template <int L>
__global__ void __launch_bounds__(256) mp_leaf_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                       int N, int B, const MpLeaf *__restrict__ leaves,
                                                       int nleaves) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nleaves * B) return;
  mp_leaf_one<L>(in, out, N, B, (int)(t % B), leaves[t / B]);
}

// The same leaves for launches too small to fill the GPU: one thread per
// output component (8 for a 4-point leaf, 4 for a 2-point one, 2 for a copy),
// each loading its (at most four) input components for every limb at once and
// then running that output's carry chain -- the chains of mp_leaf_kernel are
// already one per output, so the results are bit-identical.  16 leaves per CTA.
template <int L>
__global__ void __launch_bounds__(128) mp_leaf_small_kernel(const uint32_t *__restrict__ in,
                                                            uint32_t *__restrict__ out, int N, int B,
                                                            const MpLeaf *__restrict__ leaves, int nleaves) {
  pdl_release();
  const long long t = (long long)blockIdx.x * 16 + (threadIdx.x >> 3);
  const int o = threadIdx.x & 7;
  if (t >= (long long)nleaves * B) return;
  const int b = (int)(t % B);
  const MpLeaf lf = leaves[t / B];
  if (o >= 2 * lf.n) return;
  pdl_wait();
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  // terms of output o: (input element j, imaginary part?, sign)
  int nt = 0, tj[4] = {0, 0, 0, 0}, ti[4] = {0, 0, 0, 0}, ts[4] = {1, 1, 1, 1};
  if (lf.n == 4) {
    // X0 = x0+x2 + (x1+x3)      X2 = x0+x2 - (x1+x3)
    // X1 = x0-x2 - i(x1-x3)     X3 = x0-x2 + i(x1-x3)
    const int im = o >= 4, q = o & 3;
    nt = 4;
    tj[0] = 0, ti[0] = im;
    tj[1] = 2, ti[1] = im, ts[1] = (q & 1) ? -1 : 1;
    tj[2] = 1, tj[3] = 3;
    if ((q & 1) == 0) {  // X0, X2: the same part of x1, x3
      ti[2] = ti[3] = im;
      ts[2] = ts[3] = q == 0 ? 1 : -1;
    } else {  // X1, X3: the other part of x1, x3
      ti[2] = ti[3] = !im;
      const int sg = ((q == 1) != (im != 0)) ? 1 : -1;  // X1r: +(x1i-x3i), X1i: -(x1r-x3r), X3 opposite
      ts[2] = sg, ts[3] = -sg;
    }
  } else if (lf.n == 2) {
    nt = 2;
    tj[1] = 1, ti[0] = ti[1] = o >= 2, ts[1] = (o & 1) ? -1 : 1;
  } else {
    nt = 1;
    ti[0] = o;
  }
  const uint32_t *src[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int j = e < nt ? tj[e] : 0;
    const int idx = (j == 0 && lf.sn < 0) ? lf.sn + N : lf.sn + j * lf.s;
    src[e] = in + (size_t)idx * B + b + (ti[e] ? cim : 0);
  }
  const int q = lf.n == 4 ? (o & 3) : (lf.n == 2 ? (o & 1) : 0);
  const bool im_out = lf.n == 4 ? o >= 4 : (lf.n == 2 ? o >= 2 : o == 1);
  uint32_t *y = out + ((size_t)lf.out + q) * B + b + (im_out ? cim : 0);
  uint32_t v[4][L];
#pragma unroll
  for (int e = 0; e < 4; ++e)
    if (e < nt) {
#pragma unroll
      for (int i = 0; i < L; ++i) v[e][i] = src[e][(size_t)i * plane];
    }
  int64_t c = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    int64_t acc = c;
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (e < nt) {
        const int64_t x = (i == L - 1) ? (int64_t)(int32_t)v[e][i] : (int64_t)v[e][i];
        acc += ts[e] > 0 ? x : -x;
      }
    y[(size_t)i * plane] = (uint32_t)acc;
    c = acc >> 32;
  }
}

// ---------------------------------------------------------------------------
// one launch = every butterfly of every node of size n
// ---------------------------------------------------------------------------
//
// Thread t handles signal b = t mod B of butterfly k of one node (q = n/4 at
// output offset `off`):
//   U0 = y[off+k], U1 = y[off+k+q], Z+ = y[off+k+2q], Z- = y[off+k+3q]
//   k = 0     : no twiddle (reference :184-201)
//   k = q/2   : w^k = (1-i)/sqrt 2, products by cos(pi/4) (:213-221)
//   otherwise : 3 products per complex multiply with cos, cos+sin, cos-sin
//               (3m3a, :222-236); twiddle index kn = k*(N/n) into the N/4 table.
// For a batch that is a multiple of 32 every warp shares (node, k), so the
// twiddle loads are warp-uniform broadcasts and no lane diverges.
//
// Both twiddled cases run as six steps of one rolled loop around a single
// inlined product (one copy of its ~L^2 instructions keeps the instruction
// cache warm).  Per side (Z+ then Z-), the step's operand, twiddle and the
// rule that merges the product with P (the first product of the side, kept in
// shared memory) are:
//            step 0           step 1                      step 2
//   general  P=(Zr+-Zi)c      m.r = P -+ d Zi -> im slot   m.i = +-(P - s Zr) -> re slot
//   k = q/2  P=(Zr+-Zi)c      m.i = (Zi-Zr)c | (Zr+Zi)c    m.r = P -> im slot
//                                   -> re slot
// so m.r ends in the imaginary slot and m.i in the real slot ("swapped").

// Batches that are a multiple of the CTA size give every CTA one (node, k):
// up to 31 limbs the CTA then stages its three twiddles in shared memory once
// and the products read them four limbs per load (measured at N=1024, batch
// 2048: +4.6 % at 9 limbs, +3.1 % at 17, +0.4 to +2.2 % at 31; -0.7 % at 33,
// where the 128-register product already spills, so the larger limb counts
// keep the per-row global loads).
constexpr int kPackedTwiddleMaxLimbs = 31;

template <int L, bool kPackedTw>
__global__ void __launch_bounds__(128, level_min_blocks<L>()) mp_level_kernel(uint32_t *__restrict__ y, int N, int B, int n,
                                                          const int *__restrict__ node_off, int nnodes,
                                                          const uint32_t *__restrict__ tw,
                                                          const uint8_t *__restrict__ dneg, int tws) {
  __shared__ uint32_t Ps[L * 128];
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnodes * q * B) return;
  const int b = (int)(t % B);
  const long long r = t / B;
  const int k = (int)(r % q);
  const int off = node_off[r / q];
  constexpr int Lp = (L + 3) & ~3;
  __shared__ __align__(16) uint32_t Tw[kPackedTw ? 3 * Lp : 4];
  if (kPackedTw && k != 0) {  // cos, cos+sin, |cos-sin| of this CTA's k (every thread of the CTA has it)
    const size_t tplane = (size_t)(N >> 2) * tws;
    const int kn = k * (N / n) * tws;
    for (int e = threadIdx.x; e < 3 * L; e += blockDim.x) {
      const int sel = e / L, j = e - sel * L;
      Tw[sel * Lp + j] = tw[(size_t)(sel * L + j) * tplane + kn];
    }
    __syncthreads();
  }
  mp_bfly_one<L, kPackedTw>(y, N, B, b, n, off, k, tw, dneg, tws, Ps + threadIdx.x, blockDim.x, Tw);
}

// ---------------------------------------------------------------------------
// two levels in one launch: a node of size 2n together with its first child
// ---------------------------------------------------------------------------
//
// A node Y of size 2n (quarter 2q, q = n/4) at offset off has as first child
// the node X of size n at the same offset, so X's butterfly k writes X[k],
// X[k+q], X[k+2q], X[k+3q] -- exactly the U inputs of Y's butterflies k
// (U0 = Y[k], U1 = Y[k+2q]) and k+q (U0 = Y[k+q], U1 = Y[k+3q]).  One thread
// runs all three butterflies of one signal: the twiddle steps of each (the
// products land in their Z slots as in mp_level_kernel), then one streamed
// pass of the three L-combines, in which X's outputs go straight into Y's
// combines and are never stored.  Per level pair the planes cross HBM once
// instead of twice, and a thread's loads and stores drop from 3 x 28 L to
// 68 L words.  The same modular sums and products of the same operands as
// two mp_level_kernel launches, so the results are bit-identical.
//
// Nodes of size n that are not a first child (the conjugate-pair children of
// nodes of size 4n) run in the same launch as ordinary butterflies, after the
// fused ones: thread t < ny*q*B is fused, the rest take unodes.

// Twelve carry chains of one L-combine (the operations of combine()), one limb
// at a time: o = u0r, zpr, u1r, zmr, u0i, zpi, u1i, zmi of that limb.
struct CombineChains {
  uint32_t ca1r = 0, ca1i = 0, ca2r = 1, ca2i = 1;
  uint32_t c0r = 0, c2r = 1, c1r = 0, c3r = 1, c0i = 0, c2i = 1, c1i = 1, c3i = 0;
  __device__ __forceinline__ void limb(uint32_t U0r, uint32_t U0i, uint32_t U1r, uint32_t U1i, uint32_t m1r,
                                       uint32_t m1i, uint32_t m2r, uint32_t m2i, uint32_t (&o)[8]) {
    const uint32_t a1r = addc(m1r, m2r, ca1r), a1i = addc(m1i, m2i, ca1i);
    const uint32_t a2r = addc(m1r, ~m2r, ca2r), a2i = addc(m1i, ~m2i, ca2i);
    o[0] = addc(U0r, a1r, c0r);
    o[1] = addc(U0r, ~a1r, c2r);
    o[2] = addc(U1r, a2i, c1r);
    o[3] = addc(U1r, ~a2i, c3r);
    o[4] = addc(U0i, a1i, c0i);
    o[5] = addc(U0i, ~a1i, c2i);
    o[6] = addc(U1i, ~a2r, c1i);
    o[7] = addc(U1i, a2r, c3i);
  }
};

// Limb counts up to which combine_pair's limb loop is unrolled; above, the
// unrolled loop's register demand next to the 128-register product costs more
// than it saves, and the rolled loop reads the Z slots through ld_hint (kept
// in program order; 33 limbs 3.02 -> 2.91 ms, 9 and 17 limbs 6 % slower that
// way).  N=1024, batch 2048, ms per transform batch, unrolled / rolled with
// plain loads: 9 limbs 0.517 / 0.601, 17 limbs 1.091 / 1.186, 25 limbs 1.886 /
// 1.886, 29 limbs 2.479 / 2.337, 33 limbs 3.265 / 3.010, 34 limbs 3.489 / 3.279.
constexpr int kPairUnrollMaxLimbs = 25;

// One limb of the three L-combines of a fused thread; p: limb i of position k
// of the pair's node Y (word stride qB = q*B between the positions k + j*q).
// X's Z slots are at 2q, 3q; Y_k's at 4q, 6q; Y_{k+q}'s at 5q, 7q (always
// twiddled: swapped).  The outputs are stored with L2 priority evict_first:
// the next launch reads them after the whole signal has passed through L2.
template <bool kOrderedLoads>
__device__ __forceinline__ void combine_pair_limb(uint32_t *p, size_t qB, size_t cim, size_t sre, size_t sim,
                                                  CombineChains &cx, CombineChains &cy0, CombineChains &cy1,
                                                  uint64_t ld_pol, uint64_t st_pol) {
  auto z = [&](size_t o) { return kOrderedLoads ? ld_hint(p + o, ld_pol) : p[o]; };
  uint32_t ox[8], o0[8], o1[8];
  cx.limb(p[0], p[cim], p[qB], p[qB + cim], z(2 * qB + sre), z(2 * qB + sim), z(3 * qB + sre), z(3 * qB + sim), ox);
  cy0.limb(ox[0], ox[4], ox[1], ox[5], z(4 * qB + sre), z(4 * qB + sim), z(6 * qB + sre), z(6 * qB + sim), o0);
  cy1.limb(ox[2], ox[6], ox[3], ox[7], z(5 * qB + cim), z(5 * qB), z(7 * qB + cim), z(7 * qB), o1);
  const uint32_t *v0 = o0, *v1 = o1;
  // output j of Y_k / Y_{k+q} (u0, zp, u1, zm) at positions 0, 4q, 2q, 6q / q, 5q, 3q, 7q
  const int pos0[4] = {0, 4, 2, 6}, pos1[4] = {1, 5, 3, 7};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    st_hint(p + pos0[j] * qB, v0[j], st_pol);
    st_hint(p + pos0[j] * qB + cim, v0[j + 4], st_pol);
    st_hint(p + pos1[j] * qB, v1[j], st_pol);
    st_hint(p + pos1[j] * qB + cim, v1[j + 4], st_pol);
  }
}

template <int L>
__device__ __forceinline__ void combine_pair(uint32_t *p, size_t qB, size_t plane, size_t cim, bool swapped) {
  const size_t sre = swapped ? cim : 0, sim = swapped ? 0 : cim;
  const uint64_t st_pol = l2_policy_evict_first();
  CombineChains cx, cy0, cy1;
  if constexpr (L <= kPairUnrollMaxLimbs) {
#pragma unroll
    for (int i = 0; i < L; ++i, p += plane)
      combine_pair_limb<false>(p, qB, cim, sre, sim, cx, cy0, cy1, 0, st_pol);
  } else {
    const uint64_t ld_pol = l2_policy_evict_normal();
#pragma unroll 1
    for (int i = 0; i < L; ++i, p += plane)
      combine_pair_limb<true>(p, qB, cim, sre, sim, cx, cy0, cy1, ld_pol, st_pol);
  }
}

// CTAs per SM of mp_level_pair_kernel: from 31 limbs three (up to 170
// registers, no spills) instead of the one-level kernel's four, whose
// 128-register product spills (N=1024, batch 2048, ms per batch, four / three
// CTAs: 21 limbs 1.435 / 1.519, 25 1.837 / 1.929, 29 2.299 / 2.319, 31 2.706 /
// 2.638, 33 2.913 / 2.833, 34 3.257 / 3.005).
template <int L>
constexpr int pair_min_blocks() {
  return L >= 31 ? 3 : level_min_blocks<L>();
}

template <int L>
__global__ void __launch_bounds__(128, pair_min_blocks<L>()) mp_level_pair_kernel(
    uint32_t *__restrict__ y, int N, int B, int n, const int *__restrict__ ynodes, int ny,
    const int *__restrict__ unodes, int nu, const uint32_t *__restrict__ tw, const uint8_t *__restrict__ dneg,
    int tws) {
  __shared__ uint32_t Ps[L * 128];
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nf = (long long)ny * q * B;
  const bool fused = t < nf;
  const long long u = fused ? t : t - nf;
  if (!fused && u >= (long long)nu * q * B) return;
  const int b = (int)(u % B);
  const long long r = u / B;
  const int k = (int)(r % q);
  const int off = fused ? ynodes[r / q] : unodes[r / q];
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  const size_t qB = (size_t)q * B;
  uint32_t *p = y + (size_t)(off + k) * B + b;
  // the twiddle steps: X's (or the unfused node's) butterfly k, then Y's
  // butterflies k and k+q; one inlined copy of the product
#pragma unroll 1
  for (int j = 0; j < (fused ? 3 : 1); ++j) {
    const int kk = j == 2 ? k + q : k;
    if (kk == 0) continue;
    const int zs = j == 0 ? 2 : (j == 1 ? 4 : 5);  // Z+ slot at zs*q, Z- at (zs+1)*q or (zs+2)*q
    mp_bfly_steps<L, false>(p + (size_t)zs * qB, p + (size_t)(j == 0 ? 3 : zs + 2) * qB, plane, cim, N,
                            j == 0 ? n : 2 * n, kk, tw, dneg, tws, Ps + threadIdx.x, blockDim.x, nullptr);
  }
  if (fused) combine_pair<L>(p, qB, plane, cim, k != 0);
  else combine<L>(p, p + qB, p + 2 * qB, p + 3 * qB, plane, cim, k != 0);
}

// ---------------------------------------------------------------------------
// the same launch for batches too small to fill the GPU
// ---------------------------------------------------------------------------
//
// mp_level_kernel runs a butterfly's six products one after another on one
// thread, so with few butterflies (one signal: n/4 per launch) each launch
// takes six product latencies.  Here the six steps of a butterfly run on six
// threads at once: every thread forms its step's product into shared memory;
// after a barrier the threads of steps 1 and 2 merge theirs with the side's
// first product and store it into the Z slot exactly as mp_level_kernel does;
// after a second barrier eight threads run the L-combine, one output
// component each (three loads per limb, all limbs in flight at once, instead
// of eight per limb on one thread: one signal at N=1024, P=1024 5.3k -> 7.7k
// transforms/s, 16 signals 71k -> 107k).  The same modular sums of the same
// operands, so the results are bit-identical.

// Step st (0..5) of a twiddled butterfly: side st/3 (0: Z+ at zp, 1: Z- at
// zm), step st%3.  X = pa (+ or - pb when pb is set), X *= the twiddle whose
// first limb w points at (cos, cos+sin or |cos-sin|) when mul, else X = 0;
// then either X becomes the side's first product P (dst null) or
// dst = (negx ? -X : X) + sp * P.  This is the step table of mp_level_kernel,
// which spells it out inline in its step loop (the struct form measured 4 %
// slower there); the two kernels are checked to be bit-identical.
struct BflyStep {
  const uint32_t *pa, *pb, *w;  // w: the twiddle row's first limb (planes)
  uint32_t *dst;
  int sp;
  bool sub, negx, mul;
};

__device__ __forceinline__ BflyStep bfly_step(int st_, bool special, bool dn, uint32_t *zp, uint32_t *zm,
                                              size_t cim, const uint32_t *wr, const uint32_t *ws,
                                              const uint32_t *wd) {
  const int side = st_ >= 3;
  const int step = st_ - 3 * side;
  uint32_t *zr = side ? zm : zp;
  uint32_t *zi = zr + cim;
  BflyStep S{zr, nullptr, wr, nullptr, 0, false, false, true};
  if (step == 0) {
    S.pb = zi;
    S.sub = side;
  } else if (!special) {
    if (step == 1) {
      S.pa = zi;
      S.w = wd;
      S.negx = dn ^ (side == 0);
      S.sp = 1;
      S.dst = zi;
    } else {
      S.w = ws;
      S.negx = (side == 0);
      S.sp = side ? -1 : 1;
      S.dst = zr;
    }
  } else {
    if (step == 1) {
      S.pa = side ? zr : zi;
      S.pb = side ? zi : zr;
      S.sub = !side;
      S.dst = zr;
    } else {
      S.mul = false;
      S.sp = 1;
      S.dst = zi;
    }
  }
  return S;
}

constexpr int kSmallBflies = 16;  // butterflies per CTA, 8 threads each (128 threads)

// Output component o (0..7) of the L-combine of mp_kernels.cu combine():
//   out = U -/+ (mA +/- mB)
// with U one of U0r, U0i, U1r, U1i, mA/mB the same component of the Z+ / Z-
// products (real or imaginary, read from the slots the twiddle steps wrote).
// All inputs of all limbs are loaded before the CTA barrier that precedes
// any store, because the outputs overwrite the inputs in place.
template <int L>
__device__ __forceinline__ void combine_one(int o, bool valid, uint32_t *u0, uint32_t *u1, uint32_t *zp,
                                            uint32_t *zm, size_t plane, size_t cim, bool swapped) {
  const size_t sre = swapped ? cim : 0, sim = swapped ? 0 : cim;
  const bool im_in = (o >= 2 && o <= 5);      // products' imaginary parts (else real)
  const bool inner_sub = (o == 2 || o == 3 || o == 6 || o == 7);
  const bool outer_sub = (o == 1 || o == 3 || o == 5 || o == 6);
  uint32_t *U = (o <= 1 || o == 4 || o == 5) ? u0 : u1;
  if (o >= 4) U += cim;
  uint32_t *dst = o == 0 ? u0 : o == 1 ? zp : o == 2 ? u1 : o == 3 ? zm : o == 4 ? u0 + cim
                : o == 5 ? zp + cim : o == 6 ? u1 + cim : zm + cim;
  const uint32_t *A = zp + (im_in ? sim : sre), *Bm = zm + (im_in ? sim : sre);
  uint32_t Uv[L], Av[L], Bv[L];
  if (valid) {
#pragma unroll
    for (int i = 0; i < L; ++i) {
      Uv[i] = U[(size_t)i * plane];
      Av[i] = A[(size_t)i * plane];
      Bv[i] = Bm[(size_t)i * plane];
    }
  }
  __syncthreads();
  if (!valid) return;
  const uint32_t mi = inner_sub ? 0xffffffffu : 0u, mo = outer_sub ? 0xffffffffu : 0u;
  uint32_t ci = inner_sub ? 1u : 0u, co = outer_sub ? 1u : 0u;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    const uint32_t a = addc(Av[i], Bv[i] ^ mi, ci);
    dst[(size_t)i * plane] = addc(Uv[i], a ^ mo, co);
  }
}

template <int L>
__global__ void __launch_bounds__(8 * kSmallBflies) mp_level_small_kernel(uint32_t *__restrict__ y, int N, int B,
                                                                          int n, const int *__restrict__ node_off,
                                                                          int nnodes, const uint32_t *__restrict__ tw,
                                                                          const uint8_t *__restrict__ dneg, int tws) {
  __shared__ uint32_t Qs[kSmallBflies * 6 * L];  // [butterfly][step][limb]
  pdl_release();
  const int lb = threadIdx.x >> 3, st_ = threadIdx.x & 7;  // steps 0..5; all 8 in the combine
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * kSmallBflies + lb;
  const bool valid = t < (long long)nnodes * q * B;
  int k = 0;
  uint32_t *u0 = nullptr, *u1 = nullptr, *zp = nullptr, *zm = nullptr;
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  BflyStep S{};
  uint32_t *Q = Qs + (size_t)(lb * 6 + (st_ < 6 ? st_ : 0)) * L;
  if (valid) {
    const int b = (int)(t % B);
    const long long r = t / B;
    k = (int)(r % q);
    const int off = node_off[r / q];
    u0 = y + (size_t)(off + k) * B + b;
    u1 = u0 + (size_t)q * B;
    zp = u0 + (size_t)2 * q * B;
    zm = u0 + (size_t)3 * q * B;
    if (k != 0 && st_ < 6) {
      const size_t tplane = (size_t)(N >> 2) * tws;
      const int kn = k * (N / n) * tws;
      const bool special = (2 * k == q);
      const bool dn = special ? false : (dneg[kn] != 0);
      S = bfly_step(st_, special, dn, zp, zm, cim, tw + kn, tw + (size_t)L * tplane + kn,
                    tw + (size_t)2 * L * tplane + kn);
      pdl_wait();
      uint32_t X[L];
      if (S.mul) {
        ld_addsub<L>(X, S.pa, S.pb, plane, S.sub);
        mul_tw<L>(X, S.w, tplane);
      } else {
#pragma unroll
        for (int i = 0; i < L; ++i) X[i] = 0;
      }
      st<L>(Q, 1, X);
    }
  }
  pdl_wait();  // (again, for the threads that skipped the product: returns at once)
  __syncthreads();
  if (valid && k != 0 && S.dst) {  // steps 1 and 2: merge with the side's first product
    uint32_t X[L];
    ld<L>(X, Q, 1);
    combine_p<L>(X, Qs + (size_t)(lb * 6 + (st_ >= 3 ? 3 : 0)) * L, 1, S.negx, S.sp);
    st<L>(S.dst, plane, X);
  }
  __syncthreads();  // the merged Z slots (global) are visible to the CTA
  combine_one<L>(st_, valid, u0, u1, zp, zm, plane, cim, k != 0);
}

// ---------------------------------------------------------------------------
// the same launch with each product spread over a warp (fewest butterflies)
// ---------------------------------------------------------------------------
//
// One CTA of eight warps per butterfly, every number's limbs across a warp's
// lanes (mp_lanes.cuh).  Warps 0..5 run the six twiddle steps of
// mp_level_small_kernel at once (step = warp), each product as L column sums
// side by side instead of one thread's ~L^2/2 chained multiply-adds; after a
// barrier the warps of steps 1, 2, 4, 5 merge with their side's first
// product, and after a second barrier warp o (0..7) forms output component o
// of the L-combine (combine_one's table).  The merged products stay in
// shared memory; every global input a warp needs (its step's operands, its
// output's U and, without twiddle, the Z slots) is loaded before the first
// barrier and every output is stored after the second, so the in-place update
// is safe.  The same sums of the same operands: bit-identical.
constexpr int kWarpBflyThreads = 256;

template <int L>
__global__ void __launch_bounds__(kWarpBflyThreads) mp_level_warp_kernel(uint32_t *__restrict__ y, int N, int B,
                                                                          int n, const int *__restrict__ node_off,
                                                                          const uint32_t *__restrict__ tw,
                                                                          const uint8_t *__restrict__ dneg,
                                                                          int tws) {
  constexpr bool kTwo = L + 2 > 32;
  constexpr int Lp = (L + 3) & ~3;
  constexpr int Wlen = lanes_tw_len<L>();
  __shared__ __align__(16) uint32_t Xs[6][Lp];  // each step's operand, for broadcast reads
  __shared__ uint32_t Ws[6][Wlen];              // each step's zero-padded twiddle row
  __shared__ uint32_t Rs[6][64];                // P (steps 0, 3) and the merged products
  pdl_release();
  const int warp = threadIdx.x >> 5;
  const unsigned lane = lane_index();
  const int q = n >> 2;
  const int b = (int)(blockIdx.x % (unsigned)B);
  const long long r = blockIdx.x / (unsigned)B;
  const int k = (int)(r % q);
  const int off = node_off[r / q];
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  uint32_t *u0 = y + (size_t)(off + k) * B + b;
  uint32_t *u1 = u0 + (size_t)q * B;
  uint32_t *zp = u0 + (size_t)2 * q * B;
  uint32_t *zm = u0 + (size_t)3 * q * B;

  // output component o = warp: dst = U -/+ (mA +/- mB)
  const int o = warp;
  const bool im_in = (o >= 2 && o <= 5);
  const bool inner_sub = (o == 2 || o == 3 || o == 6 || o == 7);
  const bool outer_sub = (o == 1 || o == 3 || o == 5 || o == 6);
  const uint32_t *U = ((o <= 1 || o == 4 || o == 5) ? u0 : u1) + (o >= 4 ? cim : 0);
  uint32_t *dst = o == 0 ? u0 : o == 1 ? zp : o == 2 ? u1 : o == 3 ? zm : o == 4 ? u0 + cim
                : o == 5 ? zp + cim : o == 6 ? u1 + cim : zm + cim;
  BflyStep S{};
  uint32_t Xa = 0, Xb = 0, Wa = 0, Wb = 0;
  const bool special = (2 * k == q);
  if (k != 0 && warp < 6) {  // the step and its twiddle row (plan constants)
    const size_t tplane = (size_t)(N >> 2) * tws;
    const int kn = k * (N / n) * tws;
    const bool dn = special ? false : (dneg[kn] != 0);
    S = bfly_step(warp, special, dn, zp, zm, cim, tw + kn, tw + (size_t)L * tplane + kn,
                  tw + (size_t)2 * L * tplane + kn);
    if (S.mul) lanes_ld<L, kTwo>(Wa, Wb, S.w, tplane);
  }
  pdl_wait();
  uint32_t Ua, Ub, Aa = 0, Ab = 0, Ba = 0, Bb = 0;
  lanes_ld<L, kTwo>(Ua, Ub, U, plane);
  if (k == 0) {  // no twiddle: the Z slots are the products, unswapped
    lanes_ld<L, kTwo>(Aa, Ab, zp + (im_in ? cim : 0), plane);
    lanes_ld<L, kTwo>(Ba, Bb, zm + (im_in ? cim : 0), plane);
  } else if (warp < 6) {
    if (S.mul) {
      uint32_t Pa = 0, Pb = 0;
      lanes_ld<L, kTwo>(Xa, Xb, S.pa, plane);
      if (S.pb) lanes_ld<L, kTwo>(Pa, Pb, S.pb, plane);
      uint32_t *W = Ws[warp];  // W[j + L-1] = w_j, zeros around
      for (int e = (int)lane; e < Wlen; e += 32)
        if (e < L - 1 || e >= 2 * L - 1) W[e] = 0u;
      if (lane < L) W[lane + L - 1] = Wa;
      if (kTwo && lane + 32 < L) W[lane + 32 + L - 1] = Wb;
      if (S.pb) {
        const uint32_t m = S.sub ? ~0u : 0u;
        lanes_add<kTwo>(Xa, Xb, Pa ^ m, Pb ^ m, S.sub ? 1u : 0u);
      }
      if (lane < L) Xs[warp][lane] = Xa;
      if (kTwo && lane + 32 < L) Xs[warp][lane + 32] = Xb;
      __syncwarp();
      lanes_mul_tw<L>(Xa, Xb, Xs[warp], W);
    }
    if (!S.dst) {  // the side's first product
      Rs[warp][lane] = Xa;
      Rs[warp][lane + 32] = Xb;
    }
  }
  __syncthreads();
  if (k != 0 && warp < 6 && S.dst) {  // steps 1, 2, 4, 5: (negx ? -X : X) + sp * P
    const int ps = warp >= 3 ? 3 : 0;
    const uint32_t mx = S.negx ? ~0u : 0u, mp = S.sp < 0 ? ~0u : 0u, keep = S.sp != 0 ? ~0u : 0u;
    const uint32_t c = (S.negx ? 1u : 0u) + (S.sp < 0 ? 1u : 0u);
    Xa ^= mx;
    Xb ^= mx;
    lanes_add<kTwo>(Xa, Xb, (Rs[ps][lane] & keep) ^ mp, (Rs[ps][lane + 32] & keep) ^ mp, c > 0 ? 1u : 0u);
    if (c > 1) lanes_add<kTwo>(Xa, Xb, 0u, 0u, 1u);
    Rs[warp][lane] = Xa;
    Rs[warp][lane + 32] = Xb;
  }
  __syncthreads();
  if (k != 0) {  // m.r / m.i of each side: steps 1 / 2 (general) or 2 / 1 (k = q/2)
    const int rstep = special ? 2 : 1, istep = special ? 1 : 2;
    const int sa = im_in ? istep : rstep;
    Aa = Rs[sa][lane];
    Ab = Rs[sa][lane + 32];
    Ba = Rs[3 + sa][lane];
    Bb = Rs[3 + sa][lane + 32];
  }
  const uint32_t mi = inner_sub ? ~0u : 0u, mo = outer_sub ? ~0u : 0u;
  lanes_add<kTwo>(Aa, Ab, Ba ^ mi, Bb ^ mi, inner_sub ? 1u : 0u);
  lanes_add<kTwo>(Ua, Ub, Aa ^ mo, Ab ^ mo, outer_sub ? 1u : 0u);
  lanes_st<L, kTwo>(dst, plane, Ua, Ub);
}

// ---------------------------------------------------------------------------
// host-side launchers, one instantiation per supported limb count
// ---------------------------------------------------------------------------

// Below this many butterflies mp_level_kernel would run at most one CTA per
// SM, and the level runs as mp_level_small_kernel.  Measured at N=1024,
// P=1024 (transforms/s): one signal 2.0k -> 5.2k; 32 signals 95k -> 126k
// (with 148 x 32 as the threshold instead of 148 x 128: 95k); 64 signals
// 180k -> 200k; at 128 signals within 3 % either way; 148 x 256 as the
// threshold loses 17 % at 128 signals, and with 256 signals (65k butterflies
// per launch) the one-thread-per-butterfly kernel is 1.5x faster.
constexpr long long kSmallLevelButterflies = 148LL * 128;

// Two levels run as one mp_level_pair_kernel launch when both would run on
// mp_level_kernel and, below 31 limbs, the pair's fused threads (three
// butterflies each) fill at least one wave of the GPU; with fewer the
// single-level launches keep more butterflies in flight there (N=1024, batch
// 256, where the top pair has 32768 fused threads: 3, 5, 9 and 17 limbs 4 %,
// 4.6 %, 5.6 % and 2.5 % slower as pairs).  From 31 limbs the pairs win at
// every such batch (33 limbs, ms per batch, one level per launch / pairs:
// 128 signals 0.430 / 0.423, 192 0.486 / 0.478, 256 0.619 / 0.564, 384
// 0.826 / 0.781, 512 1.056 / 0.906).
template <int L>
constexpr long long pair_min_fused_threads() {
  return L >= 31 ? 0 : 148LL * 128 * pair_min_blocks<L>();
}

// Below this many butterflies a level runs as mp_level_warp_kernel, from 9
// limbs up.  Whole transforms at N=1024, graph-replayed, with programmatic
// dependent launch (us, warp kernel for every level / small kernel):
//   one signal   4 limbs 22.6 / 20.5   9 limbs 22.6 / 26.6   17 limbs 26.7 / 35.0
//                33 limbs 36.6 / 60.0
//   two signals  9 limbs 25.9 / 26.7   33 limbs 45.1 / 61.5
//   four signals 9 limbs 33.7 / 26.7   33 limbs 68.9 / 63.5  (1024 butterflies
//                per level; 25 limbs 49.2 / 51.3 is the one case that still gains)
// A CTA of eight warps per butterfly keeps one butterfly's latency short but
// issues ~4x the instructions of the per-thread products, so it pays only
// while the launch leaves most of the GPU idle.
template <int L>
constexpr long long warp_level_butterflies() {
  return L >= 9 ? 640 : 0;
}

// Launches below this many butterflies (or leaves) use programmatic dependent
// launch (pdl_wait).  Above it the early-scheduled CTAs of the next level cost
// more than the launch latency they hide (small kernel, N=1024, 8 signals,
// 2048 butterflies per level: 33 limbs 71.8 -> 81.7 us, 25 limbs 59.5 -> 68.7).
constexpr long long kPdlMaxButterflies = 2048;

// a launch with (pdl) or without programmatic stream serialization (pdl_wait)
template <typename... P, typename... A>
static cudaError_t launch_pdl(bool pdl, void (*kern)(P...), unsigned grid, unsigned block, cudaStream_t s,
                              A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <int L>
static cudaError_t run_transform(const MpDeviceTables &T, const uint32_t *in, uint32_t *out, int B,
                                 cudaStream_t s, float *launch_ms) {
  const int threads = 256;
  LaunchTimer timer(launch_ms, s);
  {
    const long long total = (long long)T.nleaves * B;
    timer.begin();
    if (total < kSmallLevelButterflies) {
      const cudaError_t e = launch_pdl(total < kPdlMaxButterflies, mp_leaf_small_kernel<L>,
                                       (unsigned)((total + 15) / 16), 128u, s, in, out, (int)T.N, B,
                                       (const MpLeaf *)T.leaves, (int)T.nleaves);
      if (e != cudaSuccess) return e;
    } else
      mp_leaf_kernel<L><<<(int)((total + threads - 1) / threads), threads, 0, s>>>(in, out, T.N, B, T.leaves,
                                                                                    T.nleaves);
    timer.end();
  }
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const int n = T.level_n[lv];
    const long long total = (long long)T.level_count[lv] * (n / 4) * B;
    const int lthreads = 128;
    const int blocks = (int)((total + lthreads - 1) / lthreads);
    const long long fused = lv + 1 < T.nlevels ? (long long)T.level_count[lv + 1] * (n / 4) * B : 0;
    if (fused > 0 && fused >= pair_min_fused_threads<L>() && total >= kSmallLevelButterflies &&
        (long long)T.level_count[lv + 1] * (n / 2) * B >= kSmallLevelButterflies) {
      // levels lv and lv+1 in one launch; lv+1's timer entry stays 0
      const long long threads = fused + (long long)T.pair_count[lv] * (n / 4) * B;
      timer.begin();
      mp_level_pair_kernel<L><<<(unsigned)((threads + lthreads - 1) / lthreads), lthreads, 0, s>>>(
          out, T.N, B, n, T.node_off + T.level_start[lv + 1], T.level_count[lv + 1],
          T.pair_nodes + T.pair_start[lv], T.pair_count[lv], T.tw, T.dneg, T.tws);
      timer.end();
      timer.none();
      ++lv;
      continue;
    }
    timer.begin();
    const int *nodes = T.node_off + T.level_start[lv];
    cudaError_t e = cudaSuccess;
    const bool pdl = total < kPdlMaxButterflies;
    if (total < warp_level_butterflies<L>())
      e = launch_pdl(pdl, mp_level_warp_kernel<L>, (unsigned)total, (unsigned)kWarpBflyThreads, s, out, (int)T.N,
                     B, n, nodes, (const uint32_t *)T.tw, (const uint8_t *)T.dneg, (int)T.tws);
    else if (total < kSmallLevelButterflies)
      e = launch_pdl(pdl, mp_level_small_kernel<L>, (unsigned)((total + kSmallBflies - 1) / kSmallBflies),
                     (unsigned)(8 * kSmallBflies), s, out, (int)T.N, B, n, nodes, (int)T.level_count[lv],
                     (const uint32_t *)T.tw, (const uint8_t *)T.dneg, (int)T.tws);
    else if (L <= kPackedTwiddleMaxLimbs && B % lthreads == 0)
      mp_level_kernel<L, (L <= kPackedTwiddleMaxLimbs)><<<blocks, lthreads, 0, s>>>(
          out, T.N, B, n, T.node_off + T.level_start[lv], T.level_count[lv], T.tw, T.dneg, T.tws);
    else
      mp_level_kernel<L, false><<<blocks, lthreads, 0, s>>>(out, T.N, B, n, T.node_off + T.level_start[lv],
                                                            T.level_count[lv], T.tw, T.dneg, T.tws);
    if (e != cudaSuccess) return e;
    timer.end();
  }
  return cudaGetLastError();
}

#define MPFFT_MP_CASE(LL) \
  case LL:                \
    return run_transform<LL>(T, in, out, B, s, launch_ms);

cudaError_t mp_run_transform(int L, const MpDeviceTables &T, const uint32_t *in, uint32_t *out, int B,
                             cudaStream_t s, float *launch_ms, uint32_t *big_scratch) {
  if (L > kMaxLimbs || mp_tc_used(T, L)) {
    // transforms without butterfly levels (N <= 4) need no scratch
    if ((!big_scratch && T.nlevels > 0) || L > kMaxLimbsBig) return cudaErrorInvalidValue;
    return mp_big_run_transform(L, T, in, out, B, big_scratch, s, launch_ms);
  }
  switch (L) {
    MPFFT_MP_CASE(2) MPFFT_MP_CASE(3) MPFFT_MP_CASE(4) MPFFT_MP_CASE(5) MPFFT_MP_CASE(6) MPFFT_MP_CASE(7)
    MPFFT_MP_CASE(8) MPFFT_MP_CASE(9) MPFFT_MP_CASE(10) MPFFT_MP_CASE(11) MPFFT_MP_CASE(12)
    MPFFT_MP_CASE(13) MPFFT_MP_CASE(14) MPFFT_MP_CASE(15) MPFFT_MP_CASE(16) MPFFT_MP_CASE(17)
    MPFFT_MP_CASE(18) MPFFT_MP_CASE(19) MPFFT_MP_CASE(20) MPFFT_MP_CASE(21) MPFFT_MP_CASE(22)
    MPFFT_MP_CASE(23) MPFFT_MP_CASE(24) MPFFT_MP_CASE(25) MPFFT_MP_CASE(26) MPFFT_MP_CASE(27)
    MPFFT_MP_CASE(28) MPFFT_MP_CASE(29) MPFFT_MP_CASE(30) MPFFT_MP_CASE(31) MPFFT_MP_CASE(32)
    MPFFT_MP_CASE(33) MPFFT_MP_CASE(34)
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace mpfft
