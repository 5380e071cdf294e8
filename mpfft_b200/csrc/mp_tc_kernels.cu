// Multiprecision butterflies whose twiddle products run on the tensor cores
// (tcgen05.mma kind::i8: unsigned 8-bit operands, exact int32 accumulation
// in tensor memory), for large limb counts kTcMinLimbs <= L <= kTcMaxLimbs
// (P from about 1050 to 8200 bits at N = 1024).
//
// Product as a matrix product.  At one level and one butterfly index k every
// signal multiplies its operands by the same three twiddle constants (cos,
// cos+sin, |cos-sin| of 2 pi k/N).  Write an operand |x| as 4L bytes x_a and a
// twiddle w as 4L bytes w_c.  The byte columns of the product are
//     D[m][j] = sum_a x_m[a] * w[j - a]      (each < 4L * 255^2 < 2^27)
// i.e. the operand matrix X (signals m x bytes a) times a Toeplitz matrix of
// twiddle bytes: a dense int8 GEMM with M = 128 signals per CTA, N = output
// byte columns in tiles of 128, K = 4L operand bytes in steps of 32.
//
// The Toeplitz operand is never materialised.  In the no-swizzle K-major
// shared-memory layout an MMA operand is made of core matrices of 8 rows x 16
// bytes with a fixed 16-byte row stride; the descriptor gives the stride
// between the two 16-byte K halves (LBO) and between 8-row groups (SBO).  Row
// n = 8g + r of a tile is assigned output column j = J + g + 16(7 - r), and
// group g reads copy g of the reversed twiddle bytes, shifted by g:
//     copy_g[t] = w[Q + g - t],   B[n][a] = copy_g[Q - J - 112 + 16r + a]
// so consecutive rows are 16 bytes apart (row r+1 is column j-16), the K
// halves are 16 bytes apart (LBO = 16) and the groups are one copy apart
// (SBO = copy length).  Sixteen copies of ~4L+320 bytes describe every
// Toeplitz tile of every K step.
//
// Truncation and rounding.  Byte columns below J0 = 4L-8 (rounded down to a
// multiple of 16) are not formed; the product is
//     r = floor((sum_{j >= J0} D[j] 2^(8j) + 2^(32L-2)) / 2^(32L-1))
// (the dropped part is below 4L * 2^-64 units of r's last place), with the
// operand's sign applied afterwards.  The epilogue reads each signal's column
// sums from its tensor-memory lane, carries them in increasing j and streams
// the result limbs into their destination, merged with the first product of
// the same side exactly as the streaming kernels do (mp_big_kernels.cu).
//
// Pipeline inside a CTA (128 threads, one per signal): operand bytes are
// written to shared memory by all threads; thread 0 issues the MMAs of one
// output tile into one of two 128-column tensor-memory buffers and commits
// them to that buffer's mbarrier; while the threads drain tile t (32 columns
// at a time), the MMAs of tile t+1 run.  Every wait is bounded (about two seconds of %globaltimer); on
// expiry the kernel records an error code instead of hanging.
#include <cstdint>

#include "mp_stream.cuh"
#include "mpfft_internal.h"

namespace mpfft {

constexpr int kTcRows = 128;                    // signals per CTA (MMA M)

// Tensor memory per CTA: two 128-column accumulators (the MMAs of tile t+1
// overlap the drain of tile t).  At least 80 KB of shared memory per CTA keeps
// a third CTA off the SM, so 2 x 256 of the 512 columns suffice and an
// allocation never waits.  (Measured: four CTAs per SM with one accumulator
// each and at most 128 registers per thread was slower from 65 limbs up.)
constexpr uint32_t kTcMinSmem = 80u * 1024u;
constexpr uint32_t kTcTmemCols = 256;
// instruction descriptor: D = s32, A = B = u8, both K-major, N = 128, M = 128
constexpr uint32_t kTcIdesc = (2u << 4) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ int g_tc_error = 0;  // first error code of any CTA (0 = none)
// Limit of each wait on this CTA's own MMAs, in ns of %globaltimer.  Only a
// test changes it (mpfft_diag_tc_set_wait_limit), to make the waits give up.
__device__ unsigned long long g_tc_wait_ns = 2000000000ull;
// Limit of the wait that drains a CTA's MMAs before it frees tensor memory
// after another wait gave up; not affected by the test setting.
constexpr unsigned long long kTcDrainNs = 2000000000ull;

struct TcGeom {
  int L, Kpad, J0, nt, Q, CL, wzw;
  uint32_t offT, offWZ, offBar, offSlot, bytes;
};

__host__ __device__ inline TcGeom tc_geom(int L) {
  TcGeom g;
  g.L = L;
  g.Kpad = (4 * L + 31) & ~31;            // operand bytes, padded to the MMA K step
  g.J0 = (4 * L - 8) & ~15;               // first output byte column formed
  g.nt = (8 * L - g.J0 + 127) / 128;      // output tiles of 128 columns
  g.Q = (4 * L + 160 + 15) & ~15;         // reversal base of the twiddle copies
  g.CL = (g.Q + 160 + 15) & ~15;          // bytes per copy (covers every tile and K step)
  g.wzw = g.CL / 4 + 8;                   // words of a zero-padded twiddle
  g.offT = 128u * g.Kpad;                 // operand rows first, then 3 x 16 copies
  g.offWZ = g.offT + 48u * g.CL;
  g.offBar = (g.offWZ + 12u * g.wzw + 15) & ~15u;  // 3 mbarriers: two buffers, one drain
  g.offSlot = g.offBar + 32;
  g.bytes = g.offSlot + 16 > kTcMinSmem ? g.offSlot + 16 : kTcMinSmem;
  return g;
}

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: no swizzle, version 1 (sm_100)
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait for the phase with the given parity to complete; false once `limit` ns
// have passed (checked before each try, so a limit of 0 gives up at once)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit) {
  const uint64_t t0 = global_ns();
  for (;;) {
    if (global_ns() - t0 >= limit) return false;
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
}

#define MPFFT_TMEM_LD32(addr, v)                                                                                  \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"  \
               "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                        \
               : "=r"((v)[0]), "=r"((v)[1]), "=r"((v)[2]), "=r"((v)[3]), "=r"((v)[4]), "=r"((v)[5]),             \
                 "=r"((v)[6]), "=r"((v)[7]), "=r"((v)[8]), "=r"((v)[9]), "=r"((v)[10]), "=r"((v)[11]),           \
                 "=r"((v)[12]), "=r"((v)[13]), "=r"((v)[14]), "=r"((v)[15]), "=r"((v)[16]), "=r"((v)[17]),       \
                 "=r"((v)[18]), "=r"((v)[19]), "=r"((v)[20]), "=r"((v)[21]), "=r"((v)[22]), "=r"((v)[23]),       \
                 "=r"((v)[24]), "=r"((v)[25]), "=r"((v)[26]), "=r"((v)[27]), "=r"((v)[28]), "=r"((v)[29]),       \
                 "=r"((v)[30]), "=r"((v)[31])                                                                    \
               : "r"(addr))

// ---------------------------------------------------------------------------
// CTA context: shared-memory layout, tensor memory, barriers
// ---------------------------------------------------------------------------

struct TcCtx {
  TcGeom G;
  uint8_t *smem;
  uint32_t sA, sT, bar;  // shared addresses: operand rows, twiddle copies, 2 mbarriers
  uint32_t tmem;         // tensor-memory base (lane 0, first column)
  uint32_t ph;           // bit b: parity of the next completion of buffer b
  int counter;           // output tiles processed so far (selects the buffer)
  bool bad;              // a wait expired: stop waiting, results are void
  unsigned long long wait_ns;  // limit of each wait
};

// all threads; warp 0 allocates the tensor memory
__device__ void tc_setup(TcCtx &c, uint8_t *smem, int L) {
  c.G = tc_geom(L);
  c.smem = smem;
  c.sA = smem_addr(smem);
  c.sT = c.sA + c.G.offT;
  c.bar = c.sA + c.G.offBar;
  c.ph = 0;
  c.counter = 0;
  c.bad = false;
  c.wait_ns = *(volatile unsigned long long *)&g_tc_wait_ns;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(c.bar) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(c.bar + 8) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(c.bar + 16) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(c.sA + c.G.offSlot),
                 "r"(kTcTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  c.tmem = *reinterpret_cast<volatile uint32_t *>(smem + c.G.offSlot);
}

__device__ void tc_teardown(TcCtx &c, int *err) {
  // After a wait gave up, MMAs of this CTA may still be writing tensor memory:
  // thread 0 (which issued them all) commits every MMA it issued to the drain
  // barrier and waits for it, bounded, before the memory is freed.  A wait
  // gives up only at the test setting of the limit or after seconds without
  // progress, so in practice this wait ends within microseconds.
  if (__syncthreads_or(c.bad ? 1 : 0)) {
    c.bad = true;
    if (threadIdx.x == 0) {
      tc_fence_after();
      tc_commit(c.bar + 16);
      if (!mbar_wait(c.bar + 16, 0, kTcDrainNs)) atomicCAS(err, 0, 2);  // 2: the drain wait expired too
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(c.tmem), "r"(kTcTmemCols) : "memory");
  }
  if (c.bad) atomicCAS(err, 0, 1);  // 1: a tensor-core wait expired
}

// Twiddle `which` (magnitude limbs w[l * tplane]) as 16 shifted reversed byte
// copies: copy_g[t] = w_byte[Q + g - t] (zero outside 0 .. 4L-1).
__device__ void tc_build_twiddle(TcCtx &c, int which, const uint32_t *w, size_t tplane) {
  const TcGeom &G = c.G;
  uint32_t *wz = reinterpret_cast<uint32_t *>(c.smem + G.offWZ) + which * G.wzw;
  const int d4 = (G.CL - G.Q) / 4;  // wz byte u holds w_byte[u - (CL - Q)]
  for (int u = threadIdx.x; u < G.wzw; u += blockDim.x) {
    const int l = u - d4;
    wz[u] = (l >= 0 && l < G.L) ? w[(size_t)l * tplane] : 0u;
  }
  __syncthreads();
  uint32_t *T = reinterpret_cast<uint32_t *>(c.smem + G.offT + (size_t)which * 16 * G.CL);
  const int cw = G.CL / 4;
  for (int idx = threadIdx.x; idx < 16 * cw; idx += blockDim.x) {
    const int g = idx / cw, t4 = 4 * (idx - g * cw);
    const int u0 = G.CL + g - t4 - 3;  // bytes u0 .. u0+3 of wz, reversed
    const uint32_t x = __funnelshift_r(wz[u0 >> 2], wz[(u0 >> 2) + 1], 8 * (u0 & 3));
    T[idx] = __byte_perm(x, 0, 0x0123);
  }
}

// |pa +/- pb| (pb may be null) of this thread's signal into operand row m of
// the CTA (4L bytes, zero padded to Kpad); returns its sign (1 = negative).
// Rows of signals beyond the batch read signal 0 (the caller clamps the
// pointers); their products are never stored.  Loads are unconditional, kB
// limbs of each input in flight.
__device__ uint32_t tc_prep(TcCtx &c, const uint32_t *pa, const uint32_t *pb, size_t plane, bool sub) {
  const TcGeom &G = c.G;
  const int L = G.L, m = threadIdx.x;
  uint8_t *row = c.smem + (size_t)(m >> 3) * (8 * G.Kpad) + (m & 7) * 16;
  const bool two = pb != nullptr;
  const uint32_t *qb = two ? pb : pa;
  const uint32_t msk = sub ? 0xffffffffu : 0u;
  uint32_t cy = sub ? 1u : 0u, last = 0;
  int i0 = 0;
  constexpr int kB = 16;
  for (; i0 + kB <= L; i0 += kB) {
    uint32_t va[kB], vb[kB];
#pragma unroll
    for (int e = 0; e < kB; ++e) {
      va[e] = pa[(size_t)(i0 + e) * plane];
      vb[e] = qb[(size_t)(i0 + e) * plane];
    }
    if (two) {
#pragma unroll
      for (int e = 0; e < kB; ++e) va[e] = add_c(va[e], vb[e] ^ msk, cy);
    }
    last = va[kB - 1];
#pragma unroll
    for (int q4 = 0; q4 < kB / 4; ++q4)
      *reinterpret_cast<uint4 *>(row + ((i0 >> 2) + q4) * 128) =
          make_uint4(va[4 * q4], va[4 * q4 + 1], va[4 * q4 + 2], va[4 * q4 + 3]);
  }
  // tail (fewer than 8 limbs) and zero padding up to Kpad, one 16-byte chunk at a time
  for (int ch = i0 >> 2; ch < G.Kpad / 16; ++ch) {
    uint32_t w4[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = 4 * ch + e;
      uint32_t v = 0;
      if (i < L) {
        v = pa[(size_t)i * plane];
        if (two) v = add_c(v, qb[(size_t)i * plane] ^ msk, cy);
        last = v;
      }
      w4[e] = v;
    }
    *reinterpret_cast<uint4 *>(row + ch * 128) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
  }
  const uint32_t neg = last >> 31;
  if (neg) {  // two's complement -> magnitude (limbs below L only; the padding stays zero)
    uint32_t cc = 1;
    const int nfull = L >> 2;
    for (int ch = 0; ch < nfull; ++ch) {
      uint4 u = *reinterpret_cast<uint4 *>(row + ch * 128);
      u.x = add_c(~u.x, 0, cc);
      u.y = add_c(~u.y, 0, cc);
      u.z = add_c(~u.z, 0, cc);
      u.w = add_c(~u.w, 0, cc);
      *reinterpret_cast<uint4 *>(row + ch * 128) = u;
    }
    if (L & 3) {
      uint4 u = *reinterpret_cast<uint4 *>(row + nfull * 128);
      uint32_t w4[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (e < (L & 3)) w4[e] = add_c(~w4[e], 0, cc);
      *reinterpret_cast<uint4 *>(row + nfull * 128) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
  }
  return neg;
}

// thread 0: the MMAs of output tile t of twiddle `which` into buffer buf
__device__ void tc_issue(const TcCtx &c, int which, int t, int buf) {
  const TcGeom &G = c.G;
  const int J = G.J0 + 128 * t;
  const int s_lo = max(0, J - 4 * G.L + 1) >> 5;  // K steps that meet nonzero Toeplitz entries
  const int s_hi = min(G.Kpad >> 5, (J + 159) >> 5);
  const uint32_t tb = c.sT + (uint32_t)which * 16u * G.CL + (uint32_t)(G.Q - J - 112);
  const uint32_t d = c.tmem + (uint32_t)buf * 128u;
  for (int s = s_lo; s < s_hi; ++s)
    tc_mma(d, tc_desc(c.sA + 256u * s, 128u, 8u * G.Kpad), tc_desc(tb + 32u * s, 16u, G.CL), kTcIdesc,
           s > s_lo ? 1u : 0u);
  tc_commit(c.bar + 8u * buf);
}

// Where a product's result limbs go: dst[q] = sign * r_q (two's complement,
// streamed in increasing q; stores only, the merges happen in tc_combine)
struct TcEmit {
  uint32_t *p;
  size_t ds;
  uint32_t rm, cr;
  bool on;
  __device__ void init(bool valid, uint32_t neg, uint32_t *dst_, size_t ds_) {
    on = valid;
    p = dst_;
    ds = ds_;
    rm = neg ? 0xffffffffu : 0u;
    cr = neg ? 1u : 0u;
  }
  __device__ __forceinline__ void put(uint32_t r) {
    const uint32_t v = add_c(r ^ rm, 0, cr);
    if (on) *p = v;
    p += ds;
  }
};

// The 3m3a merges and the L-combine in one streamed pass, 8 limbs of all
// inputs in flight at a time.  Per side (Z+ in zp, Z- in zm) the twiddled
// value is
//     T_r = a_r P + b_r S_r,   T_i = a_i P + b_i S_i      (coefficients in {-1, 0, 1})
// with P the side's first product and S_r, S_i the side's two slots read as
// (imaginary, real) when `swapped` (the products' layout) or (real,
// imaginary) otherwise.  Then the outputs of mp_kernels.cu combine():
//     u0 = U0 + (T+ + T-),  zp = U0 - (T+ + T-),
//     u1 = U1 - i (T+ - T-), zm = U1 + i (T+ - T-).
struct TcSide {
  const uint32_t *P;  // may be null when a_r = a_i = 0
  int ar, br, ai, bi;
};

__device__ __forceinline__ uint32_t coef_mask(int a) { return a < 0 ? 0xffffffffu : 0u; }
__device__ __forceinline__ uint32_t coef_keep(int a) { return a != 0 ? 0xffffffffu : 0u; }

__device__ void tc_combine(uint32_t *u0, uint32_t *u1, uint32_t *zp, uint32_t *zm, size_t plane, size_t cim,
                           size_t ps, int L, bool swapped, const TcSide &sp, const TcSide &sm) {
  const size_t sre = swapped ? cim : 0, sim = swapped ? 0 : cim;
  // merge chains: T+r, T+i, T-r, T-i
  const TcSide *sd[2] = {&sp, &sm};
  uint32_t kP[2][2], mP[2][2], kS[2][2], mS[2][2], cT[2][2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int a[2] = {sd[h]->ar, sd[h]->ai}, bb[2] = {sd[h]->br, sd[h]->bi};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      kP[h][c] = coef_keep(a[c]);
      mP[h][c] = coef_mask(a[c]);
      kS[h][c] = coef_keep(bb[c]);
      mS[h][c] = coef_mask(bb[c]);
      cT[h][c] = (a[c] < 0 ? 1u : 0u) + (bb[c] < 0 ? 1u : 0u);
    }
  }
  // without a first product the coefficient of P is 0: read any valid word instead
  const uint32_t *p0 = sp.P ? sp.P : u0, *p1 = sm.P ? sm.P : u0;
  const size_t ps0 = sp.P ? ps : plane, ps1 = sm.P ? ps : plane;
  uint32_t ca1r = 0, ca1i = 0, ca2r = 1, ca2i = 1;
  uint32_t c0r = 0, c2r = 1, c1r = 0, c3r = 1, c0i = 0, c2i = 1, c1i = 1, c3i = 0;
  constexpr int U = 8;
  for (int i0 = 0; i0 < L; i0 += U) {
    uint32_t U0r[U], U0i[U], U1r[U], U1i[U], Ar[U], Ai[U], Br[U], Bi[U], P0[U], P1[U];
#pragma unroll
    for (int e = 0; e < U; ++e) {
      const int i = min(i0 + e, L - 1);  // tail: re-read the top limb, not stored
      const size_t o = (size_t)i * plane;
      U0r[e] = u0[o];
      U0i[e] = u0[o + cim];
      U1r[e] = u1[o];
      U1i[e] = u1[o + cim];
      Ar[e] = zp[o + sre];
      Ai[e] = zp[o + sim];
      Br[e] = zm[o + sre];
      Bi[e] = zm[o + sim];
      P0[e] = p0[(size_t)i * ps0];
      P1[e] = p1[(size_t)i * ps1];
    }
#pragma unroll
    for (int e = 0; e < U; ++e) {
      const int i = i0 + e;
      if (i >= L) break;
      const size_t o = (size_t)i * plane;
      const uint32_t m1r = add_c((P0[e] & kP[0][0]) ^ mP[0][0], (Ar[e] & kS[0][0]) ^ mS[0][0], cT[0][0]);
      const uint32_t m1i = add_c((P0[e] & kP[0][1]) ^ mP[0][1], (Ai[e] & kS[0][1]) ^ mS[0][1], cT[0][1]);
      const uint32_t m2r = add_c((P1[e] & kP[1][0]) ^ mP[1][0], (Br[e] & kS[1][0]) ^ mS[1][0], cT[1][0]);
      const uint32_t m2i = add_c((P1[e] & kP[1][1]) ^ mP[1][1], (Bi[e] & kS[1][1]) ^ mS[1][1], cT[1][1]);
      const uint32_t a1r = add_c(m1r, m2r, ca1r), a1i = add_c(m1i, m2i, ca1i);
      const uint32_t a2r = add_c(m1r, ~m2r, ca2r), a2i = add_c(m1i, ~m2i, ca2i);
      u0[o] = add_c(U0r[e], a1r, c0r);
      zp[o] = add_c(U0r[e], ~a1r, c2r);
      u1[o] = add_c(U1r[e], a2i, c1r);
      zm[o] = add_c(U1r[e], ~a2i, c3r);
      u0[o + cim] = add_c(U0i[e], a1i, c0i);
      zp[o + cim] = add_c(U0i[e], ~a1i, c2i);
      u1[o + cim] = add_c(U1i[e], ~a2r, c1i);
      zm[o + cim] = add_c(U1i[e], a2r, c3i);
    }
  }
}

// One product per signal of the CTA: operand rows (already in shared memory,
// made visible to the async proxy) times twiddle `which`; all threads.
__device__ void tc_product(TcCtx &c, int which, TcEmit &em) {
  const TcGeom &G = c.G;
  const int L = G.L;
  const uint32_t lane_addr = c.tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
  uint64_t carry = 0;
  uint32_t prev = 0;
  if (threadIdx.x == 0) {
    tc_fence_after();
    tc_issue(c, which, 0, c.counter & 1);
  }
  for (int t = 0; t < G.nt; ++t) {
    const int buf = (c.counter + t) & 1;
    if (threadIdx.x == 0 && t + 1 < G.nt) tc_issue(c, which, t + 1, buf ^ 1);
    __syncwarp();
    if (!c.bad && !mbar_wait(c.bar + 8u * buf, (c.ph >> buf) & 1u, c.wait_ns)) c.bad = true;
    c.ph ^= 1u << buf;
    tc_fence_after();
    // Tile column n = 8g + r holds output byte column J + g + 16(7 - r), so
    // 32-column chunk ch holds the 4 bytes e of the 8 limb columns
    // lc = ch + 4(7 - r) at columns 8e + r: fold each chunk into limb-column
    // sums S[lc] = sum_e D[4 lc + e] 2^(8e) (< 2^52) as it arrives.
    uint64_t S[32];
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      uint32_t v[32];
      MPFFT_TMEM_LD32(lane_addr + 128u * buf + 32u * ch, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int r = 0; r < 8; ++r)
        S[ch + 4 * (7 - r)] = (uint64_t)v[r] + (uint64_t)v[8 + r] * 0x100u + (uint64_t)v[16 + r] * 0x10000u +
                              (uint64_t)v[24 + r] * 0x1000000u;
    }
    const int mbase = (G.J0 >> 2) + 32 * t;  // limb column of this tile's first byte column
#pragma unroll
    for (int lc = 0; lc < 32; ++lc) {
      const int m = mbase + lc;
      if (m >= 2 * L) break;  // above the product's top limb
      uint64_t sum = S[lc] + carry;
      if (m == L - 1) sum += 1ull << 30;  // + 2^(32L-2): round to nearest
      const uint32_t limb = (uint32_t)sum;
      carry = sum >> 32;
      if (m >= L) em.put(__funnelshift_r(prev, limb, 31));  // result limb m - L
      prev = limb;
    }
    tc_fence_before();
    __syncthreads();
  }
  c.counter += G.nt;
}

// ---------------------------------------------------------------------------
// level kernel
// ---------------------------------------------------------------------------

// One CTA per (node, butterfly index k, group of 128 signals): the 3m3a
// products of mp_big_level_kernel (three per side, two at k = n/8) on the
// tensor cores, stored unmerged, then one streamed merge + L-combine pass.
// Scratch: 2L limb planes of gridDim.x*128 words (the first product of each
// side).
__global__ void __launch_bounds__(kTcRows, 1)
    mp_tc_level_kernel(uint32_t *__restrict__ y, int N, int B, int L, int n, const int *__restrict__ node_off,
                       const uint32_t *__restrict__ tw, const uint8_t *__restrict__ dneg, int tws,
                       uint32_t *__restrict__ scratch, int *err) {
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  const int q = n >> 2;
  const int nbg = (B + kTcRows - 1) / kTcRows;
  long long cta = blockIdx.x;
  const int bg = (int)(cta % nbg);
  cta /= nbg;
  const int k = (int)(cta % q);
  const int off = node_off[cta / q];
  const int b = bg * kTcRows + (int)threadIdx.x;
  const bool valid = b < B;
  const int bs = valid ? b : 0;
  const size_t plane = (size_t)N * B;
  const size_t cim = (size_t)L * plane;
  uint32_t *u0 = y + (size_t)(off + k) * B + bs;
  uint32_t *u1 = u0 + (size_t)q * B;
  uint32_t *zp = u0 + (size_t)2 * q * B;
  uint32_t *zm = u0 + (size_t)3 * q * B;
  if (k == 0) {  // no twiddle products: T = Z
    const TcSide id{nullptr, 0, 1, 0, 1};
    if (valid) tc_combine(u0, u1, zp, zm, plane, cim, 0, L, false, id, id);
    return;
  }
  TcCtx c;
  tc_setup(c, tc_smem, L);
  const size_t tplane = (size_t)(N >> 2) * tws;
  const int kn = k * (N / n) * tws;
  const bool special = 2 * k == q;
  const bool dn = special ? false : (dneg[kn] != 0);
  for (int which = 0; which < (special ? 1 : 3); ++which)
    tc_build_twiddle(c, which, tw + (size_t)which * L * tplane + kn, tplane);
  const size_t ss = (size_t)gridDim.x * kTcRows;  // scratch limb-plane stride
  uint32_t *P0 = scratch + (size_t)blockIdx.x * kTcRows + threadIdx.x;  // first product of Z+
  uint32_t *P1 = P0 + (size_t)L * ss;                                      // first product of Z-
  // Products of each side (as the steps of mp_big_level_kernel, but unmerged):
  //   P = c (Zr +/- Zi) -> scratch;  R1 = |cos-sin| Zi -> zi slot;  R2 = (cos+sin) Zr -> zr slot
  // k = n/8: P = c (Zr +/- Zi) -> scratch, R = c (Zi - Zr) resp. c (Zr + Zi) -> zr slot.
  for (int side = 0; side < 2; ++side) {
    uint32_t *zr = side ? zm : zp;
    uint32_t *zi = zr + cim;
    uint32_t *Pd = side ? P1 : P0;
    for (int step = 0; step < (special ? 2 : 3); ++step) {
      const uint32_t *pa = zr, *pb = nullptr;
      bool sub = false;
      int which = 0;
      uint32_t *dst = Pd;
      size_t ds = ss;
      if (step == 0) {
        pb = zi;
        sub = side;
      } else if (special) {
        pa = side ? zr : zi;
        pb = side ? zi : zr;
        sub = !side;
        dst = zr;
        ds = plane;
      } else if (step == 1) {
        pa = zi;
        which = 2;
        dst = zi;
        ds = plane;
      } else {
        which = 1;
        dst = zr;
        ds = plane;
      }
      const uint32_t xneg = tc_prep(c, pa, pb, plane, sub);
      fence_async_smem();
      __syncthreads();
      TcEmit em;
      em.init(valid, xneg, dst, ds);
      tc_product(c, which, em);
    }
  }
  // merge coefficients (T_r from the zi slot, T_i from the zr slot):
  //   Z+: T_r = P + (dn ? R1 : -R1), T_i = P - R2;   Z-: T_r = P + (dn ? -R1 : R1), T_i = R2 - P
  //   k = n/8: T_r = P, T_i = R
  TcSide s0, s1;
  if (special) {
    s0 = TcSide{P0, 1, 0, 0, 1};
    s1 = TcSide{P1, 1, 0, 0, 1};
  } else {
    s0 = TcSide{P0, 1, dn ? 1 : -1, 1, -1};
    s1 = TcSide{P1, 1, dn ? -1 : 1, -1, 1};
  }
  if (valid) tc_combine(u0, u1, zp, zm, plane, cim, ss, L, true, s0, s1);
  tc_teardown(c, err);
}

// products of B operands (limb planes x[i*B + b], two's complement) with one
// twiddle magnitude w[0 .. L-1]: out[i*B + b] = sign(x) * r (diagnostics)
__global__ void __launch_bounds__(kTcRows, 1)
    mp_tc_mul_kernel(const uint32_t *__restrict__ x, const uint32_t *__restrict__ w, uint32_t *__restrict__ out,
                     int L, int B, int *err) {
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  const int b = blockIdx.x * kTcRows + (int)threadIdx.x;
  const bool valid = b < B;
  const int bs = valid ? b : 0;
  TcCtx c;
  tc_setup(c, tc_smem, L);
  tc_build_twiddle(c, 0, w, 1);
  const uint32_t xneg = tc_prep(c, x + bs, nullptr, (size_t)B, false);
  fence_async_smem();
  __syncthreads();
  TcEmit em;
  em.init(valid, xneg, out + bs, (size_t)B);
  tc_product(c, 0, em);
  tc_teardown(c, err);
}

// ---------------------------------------------------------------------------
// the int8 tensor-core rate (the roofline denominator of the products above)
// ---------------------------------------------------------------------------
//
// Thread 0 of each CTA issues `count` MMAs of M=128, N=256, K=32 unsigned
// bytes into one 256-column tensor-memory accumulator (operands: zeroed
// shared-memory tiles, no-swizzle K-major as above), commits them to an
// mbarrier and waits for it (bounded); MACs = count * 128*256*32 per CTA.
static cudaError_t tc_prepare(const void *fn, uint32_t bytes, int **err);
constexpr uint32_t kTcPeakIdesc = (2u << 4) | ((256u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kTcPeakSmem = 80u * 1024u;  // keeps a third CTA off an SM (2 x 256 columns)

__global__ void __launch_bounds__(128, 1) mp_tc_peak_kernel(int count, int *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  // A: 128 rows x 32 bytes at 0, B: 256 rows x 32 bytes at 4096; slot and barrier after
  for (int i = threadIdx.x; i < (4096 + 8192) / 16; i += blockDim.x) reinterpret_cast<uint4 *>(sm)[i] = make_uint4(0, 0, 0, 0);
  const uint32_t base = smem_addr(sm), bar = base + 12288, slot = base + 12304;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(256u) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(sm + 12304);
  if (threadIdx.x == 0) {
    const uint64_t da = tc_desc(base, 128u, 256u), db = tc_desc(base + 4096u, 128u, 256u);
    for (int i = 0; i < count; ++i) tc_mma(tmem, da, db, kTcPeakIdesc, i > 0 ? 1u : 0u);
    tc_commit(bar);
    if (!mbar_wait(bar, 0, kTcDrainNs)) atomicCAS(err, 0, 2);
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u) : "memory");
  }
}

cudaError_t mp_tc_int8_rate(double *macs_per_s) {
  int *err = nullptr;
  cudaError_t e = tc_prepare((const void *)mp_tc_peak_kernel, kTcPeakSmem, &err);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int ctas = 2 * sms, count = 16384;
  mp_tc_peak_kernel<<<ctas, 128, kTcPeakSmem>>>(256, err);  // warm-up
  cudaEventRecord(e0);
  mp_tc_peak_kernel<<<ctas, 128, kTcPeakSmem>>>(count, err);
  cudaEventRecord(e1);
  e = cudaEventSynchronize(e1);
  float ms = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) *macs_per_s = (double)ctas * count * 128.0 * 256.0 * 32.0 / (ms * 1e-3);
  return e;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static cudaError_t tc_prepare(const void *fn, uint32_t bytes, int **err) {
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  return cudaGetSymbolAddress(reinterpret_cast<void **>(err), g_tc_error);
}

size_t mp_tc_scratch_words(const MpDeviceTables &T, int L, int B) {
  long long most = 0;
  const long long nbg = (B + kTcRows - 1) / kTcRows;
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const long long th = (long long)T.level_count[lv] * (T.level_n[lv] / 4) * nbg * kTcRows;
    if (th > most) most = th;
  }
  return (size_t)2 * L * (size_t)most;
}

cudaError_t mp_tc_run_levels(int L, const MpDeviceTables &T, uint32_t *out, int B, uint32_t *scratch,
                             cudaStream_t s, LaunchTimer &timer) {
  const TcGeom G = tc_geom(L);
  int *err = nullptr;
  cudaError_t e = tc_prepare((const void *)mp_tc_level_kernel, G.bytes, &err);
  if (e != cudaSuccess) return e;
  const long long nbg = (B + kTcRows - 1) / kTcRows;
  for (int lv = 0; lv < T.nlevels; ++lv) {
    const int n = T.level_n[lv];
    const long long ctas = (long long)T.level_count[lv] * (n / 4) * nbg;
    timer.begin();
    mp_tc_level_kernel<<<(unsigned)ctas, kTcRows, G.bytes, s>>>(out, T.N, B, L, n, T.node_off + T.level_start[lv],
                                                               T.tw, T.dneg, T.tws, scratch, err);
    timer.end();
  }
  return cudaGetLastError();
}

cudaError_t mp_tc_mul(int L, int B, const uint32_t *x, const uint32_t *w, uint32_t *out, cudaStream_t s) {
  const TcGeom G = tc_geom(L);
  int *err = nullptr;
  cudaError_t e = tc_prepare((const void *)mp_tc_mul_kernel, G.bytes, &err);
  if (e != cudaSuccess) return e;
  mp_tc_mul_kernel<<<(B + kTcRows - 1) / kTcRows, kTcRows, G.bytes, s>>>(x, w, out, L, B, err);
  return cudaGetLastError();
}

cudaError_t mp_tc_set_wait_limit(unsigned long long ns) {
  return cudaMemcpyToSymbol(g_tc_wait_ns, &ns, sizeof ns);
}

cudaError_t mp_tc_take_error(int *code) {
  int *err = nullptr;
  cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&err), g_tc_error);
  if (e != cudaSuccess) return e;
  const int zero = 0;
  if ((e = cudaMemcpy(code, err, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) return e;
  return cudaMemcpy(err, &zero, sizeof(int), cudaMemcpyHostToDevice);
}

size_t mp_tc_smem_bytes(int L) { return tc_geom(L).bytes; }

}  // namespace mpfft
