// Double-double (about 106-bit) conjugate-pair split-radix FFT kernels.
//
// A double-double is an unevaluated sum hi + lo of two doubles with
// |lo| <= ulp(hi)/2.  The arithmetic is the published error-free
// transformations (Knuth's TwoSum, Dekker's Fast2Sum, the FMA form of
// TwoProd) composed as in Hida, Li and Bailey's double-double library:
// additions are the accurate (IEEE-style) variant, multiplications use one
// TwoProd plus the two cross products; every operation has a relative error
// of a few units of 2^-104.
//
// Same tree and schedule as the FP64 kernels (d_kernels.cu): maximal nodes of
// up to T = min(N, 2048) points run in shared memory (DIT-order gather, base
// cases, all levels up to the node), levels above in global memory.  Base
// cases are the 4-, 2- and 1-point DFTs only; every level is the 4m2a
// butterfly with double-double twiddles (cos and sin of 2 pi k/N rounded to
// 106 bits by MPFR).  Layout: word (c, h, b, p) at base[((c*2 + h)*B + b)*N + p]
// -- c real/imaginary, h high/low part, each signal contiguous.
#include <cstdint>

#include "mpfft_internal.h"

namespace mpfft {

struct dd {
  double h, l;
};

__device__ __forceinline__ dd two_sum(double a, double b) {  // Knuth: s + e = a + b exactly
  const double s = a + b;
  const double bb = s - a;
  return dd{s, (a - (s - bb)) + (b - bb)};
}

__device__ __forceinline__ dd fast_two_sum(double a, double b) {  // Dekker, |a| >= |b|
  const double s = a + b;
  return dd{s, b - (s - a)};
}

__device__ __forceinline__ dd dd_add(dd x, dd y) {
  dd s = two_sum(x.h, y.h);
  const dd t = two_sum(x.l, y.l);
  s.l += t.h;
  s = fast_two_sum(s.h, s.l);
  s.l += t.l;
  return fast_two_sum(s.h, s.l);
}

__device__ __forceinline__ dd dd_neg(dd x) { return dd{-x.h, -x.l}; }
__device__ __forceinline__ dd dd_sub(dd x, dd y) { return dd_add(x, dd_neg(y)); }

__device__ __forceinline__ dd dd_mul(dd x, dd y) {
  const double p = x.h * y.h;
  double e = fma(x.h, y.h, -p);  // TwoProd: p + e = x.h * y.h exactly
  e = fma(x.h, y.l, e);
  e = fma(x.l, y.h, e);
  return fast_two_sum(p, e);
}

// times a power of two: exact
__device__ __forceinline__ dd dd_scale(dd x, double s) { return dd{x.h * s, x.l * s}; }

// shared-memory index: low 4 bits XOR-ed with bits 4-7 ^ 8-11, a permutation
// inside each 16-aligned block (17 % fewer wavefronts than padding on this
// schedule, counted by simulating its accesses)
__device__ __forceinline__ int ddidx(int m) { return m ^ (((m >> 4) ^ (m >> 8)) & 15); }

// shared-memory instance: four planes (re hi, re lo, im hi, im lo)
struct DDPlanes {
  double *rh, *rl, *ih, *il;
  __device__ dd re(int m) const { return dd{rh[ddidx(m)], rl[ddidx(m)]}; }
  __device__ dd im(int m) const { return dd{ih[ddidx(m)], il[ddidx(m)]}; }
  __device__ void set(int m, dd r, dd i) const {
    const int a = ddidx(m);
    rh[a] = r.h;
    rl[a] = r.l;
    ih[a] = i.h;
    il[a] = i.l;
  }
};

// base cases on positions [o, o+n), in place (n = 4, 2, 1)
__device__ void dd_leaf(const DDPlanes &P, int o, int n) {
  if (n == 4) {
    const dd x0r = P.re(o), x1r = P.re(o + 1), x2r = P.re(o + 2), x3r = P.re(o + 3);
    const dd x0i = P.im(o), x1i = P.im(o + 1), x2i = P.im(o + 2), x3i = P.im(o + 3);
    const dd er = dd_add(x0r, x2r), fr = dd_sub(x0r, x2r), gr = dd_add(x1r, x3r), hr = dd_sub(x1r, x3r);
    const dd ei = dd_add(x0i, x2i), fi = dd_sub(x0i, x2i), gi = dd_add(x1i, x3i), hi = dd_sub(x1i, x3i);
    P.set(o, dd_add(er, gr), dd_add(ei, gi));
    P.set(o + 1, dd_add(fr, hi), dd_sub(fi, hr));
    P.set(o + 2, dd_sub(er, gr), dd_sub(ei, gi));
    P.set(o + 3, dd_sub(fr, hi), dd_add(fi, hr));
  } else if (n == 2) {
    const dd x0r = P.re(o), x1r = P.re(o + 1), x0i = P.im(o), x1i = P.im(o + 1);
    P.set(o, dd_add(x0r, x1r), dd_add(x0i, x1i));
    P.set(o + 1, dd_sub(x0r, x1r), dd_sub(x0i, x1i));
  }
}

// the 4m2a butterfly on (U0, U1, Z+, Z-) with twiddle w = (c, s)
__device__ __forceinline__ void dd_bfly(dd &u0r, dd &u0i, dd &u1r, dd &u1i, dd &zpr, dd &zpi, dd &zmr, dd &zmi, dd c,
                                        dd s) {
  const dd pr = dd_add(dd_mul(c, zpr), dd_mul(s, zpi)), pi = dd_sub(dd_mul(c, zpi), dd_mul(s, zpr));
  const dd mr = dd_sub(dd_mul(c, zmr), dd_mul(s, zmi)), mi = dd_add(dd_mul(c, zmi), dd_mul(s, zmr));
  const dd sr = dd_add(pr, mr), si = dd_add(pi, mi), dr = dd_sub(pr, mr), di = dd_sub(pi, mi);
  const dd a0r = dd_add(u0r, sr), a0i = dd_add(u0i, si), a2r = dd_sub(u0r, sr), a2i = dd_sub(u0i, si);
  const dd a1r = dd_add(u1r, di), a1i = dd_sub(u1i, dr), a3r = dd_sub(u1r, di), a3i = dd_add(u1i, dr);
  u0r = a0r, u0i = a0i, u1r = a1r, u1i = a1i, zpr = a2r, zpi = a2i, zmr = a3r, zmi = a3i;
}

struct DDTw {
  const double *ch, *cl, *sh, *sl;  // cos, sin of 2 pi k/N, hi and lo parts, k < N/4
  __device__ dd c(size_t k) const { return dd{__ldg(ch + k), __ldg(cl + k)}; }
  __device__ dd s(size_t k) const { return dd{__ldg(sh + k), __ldg(sl + k)}; }
};

// One CTA = G instances (sub-transform root x signal) in shared memory; see
// d_sub_kernel (d_kernels.cu) for the schedule.  swap_in / swap_out: read the
// input's / write the output's real and imaginary planes exchanged.
template <bool SINGLE>
__global__ void __launch_bounds__(256) dd_sub_kernel(const double *__restrict__ in, double *__restrict__ out, int N,
                                                     int B, const SubRoot *__restrict__ roots, int nroots, int G,
                                                     SubSchedule big, SubSchedule small, DDTw tw, double scale,
                                                     int swap_in, int swap_out) {
  extern __shared__ double dsm[];
  const int Tmax = big.size;
  const int lgT = 31 - __clz(Tmax);
  const int pl = Tmax;  // plane length
  const int tws = N / Tmax;
  int G_here, b0;
  SubRoot rt;
  bool is_big = true;
  if (SINGLE) {
    b0 = blockIdx.x * G;
    G_here = min(G, B - b0);
    rt = roots[0];
  } else {
    const int root = blockIdx.x % nroots;
    b0 = blockIdx.x / nroots;
    G_here = 1;
    rt = roots[root];
    is_big = rt.size == Tmax;
  }
  const int T = rt.size;
  const int *perm = is_big ? big.perm : small.perm;
  const Leaf *leaves = is_big ? big.leaves : small.leaves;
  const int nleaves = is_big ? big.nleaves : small.nleaves;
  const int nlevels = is_big ? big.nlevels : small.nlevels;
  auto inst = [&](int g) {
    double *base = dsm + (size_t)g * 4 * pl;
    return DDPlanes{base, base + pl, base + 2 * pl, base + 3 * pl};
  };
  const size_t cplane = (size_t)2 * B * N;  // real -> imaginary component
  const size_t hplane = (size_t)B * N;      // high -> low part
  const size_t in_re = swap_in ? cplane : 0, in_im = swap_in ? 0 : cplane;
  const size_t out_re = swap_out ? cplane : 0, out_im = swap_out ? 0 : cplane;
  // gather: element j of instance g to DIT position perm[j], 4 elements per thread in flight
  const int total = G_here << lgT;
  for (int e0 = 0; e0 < total; e0 += 4 * 256) {
    double v[4][4];
    int dst[4], gg[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * 256 + (int)threadIdx.x;
      const int g = e >> lgT, j = e & (Tmax - 1);
      dst[u] = -1;
      gg[u] = g;
      if (e < total && (SINGLE || j < T)) {
        int idx = rt.sn + j * rt.s;
        if (idx < 0) idx += N;
        const size_t o = (size_t)(b0 + g) * N + idx;
        v[u][0] = in[in_re + o];
        v[u][1] = in[in_re + hplane + o];
        v[u][2] = in[in_im + o];
        v[u][3] = in[in_im + hplane + o];
        dst[u] = perm[j];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (dst[u] >= 0) inst(gg[u]).set(dst[u], dd{v[u][0], v[u][1]}, dd{v[u][2], v[u][3]});
  }
  __syncthreads();
  for (int e = threadIdx.x; e < G_here * nleaves; e += blockDim.x) {
    const int g = SINGLE ? e / nleaves : 0, l = SINGLE ? e - g * nleaves : e;
    const Leaf lf = leaves[l];
    dd_leaf(inst(g), lf.out, lf.n);
  }
  for (int lv = 0; lv < nlevels; ++lv) {
    __syncthreads();
    const int n = big.level_n[lv], q = n >> 2, lgq = 29 - __clz(n);
    const int cnt = is_big ? big.level_count[lv] : small.level_count[lv];
    const int *nodes = (is_big ? big.node_off : small.node_off) + (is_big ? big.level_start[lv] : small.level_start[lv]);
    const int per = cnt * q;
    for (int e = threadIdx.x; e < G_here * per; e += blockDim.x) {
      const int g = SINGLE ? e / per : 0, t = SINGLE ? e - g * per : e;
      const int node = t >> lgq, k = t & (q - 1);
      const size_t km = (size_t)(k << (lgT - (lgq + 2))) * tws;  // k * (N/n)
      const DDPlanes P = inst(g);
      const int off = nodes[node];
      dd u0r = P.re(off + k), u0i = P.im(off + k), u1r = P.re(off + k + q), u1i = P.im(off + k + q);
      dd zpr = P.re(off + k + 2 * q), zpi = P.im(off + k + 2 * q), zmr = P.re(off + k + 3 * q),
         zmi = P.im(off + k + 3 * q);
      dd_bfly(u0r, u0i, u1r, u1i, zpr, zpi, zmr, zmi, tw.c(km), tw.s(km));
      P.set(off + k, u0r, u0i);
      P.set(off + k + q, u1r, u1i);
      P.set(off + k + 2 * q, zpr, zpi);
      P.set(off + k + 3 * q, zmr, zmi);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int g = e >> lgT, m = e & (Tmax - 1);
    if (!SINGLE && m >= T) continue;
    const DDPlanes P = inst(g);
    const dd r = dd_scale(P.re(m), scale), i = dd_scale(P.im(m), scale);
    const size_t o = (size_t)(b0 + g) * N + rt.out + m;
    out[out_re + o] = r.h;
    out[out_re + hplane + o] = r.l;
    out[out_im + o] = i.h;
    out[out_im + hplane + o] = i.l;
  }
}

// butterflies of the levels above the shared-memory sub-transforms (in place)
__global__ void __launch_bounds__(256) dd_level_kernel(double *__restrict__ y, int N, int B, int n,
                                                       const int *__restrict__ node_off, int nnodes, DDTw tw,
                                                       double scale, int swap_out) {
  const int q = n >> 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnodes * q * B) return;
  const int k = (int)(t % q);
  const long long r = t / q;
  const int node = (int)(r % nnodes);
  const int b = (int)(r / nnodes);
  const size_t cplane = (size_t)2 * B * N, hplane = (size_t)B * N;
  double *re = y + (size_t)b * N, *im = y + cplane + (size_t)b * N;
  const int off = node_off[node] + k;
  auto ld = [&](const double *p, int m) { return dd{p[m], p[hplane + m]}; };
  dd u0r = ld(re, off), u0i = ld(im, off), u1r = ld(re, off + q), u1i = ld(im, off + q);
  dd zpr = ld(re, off + 2 * q), zpi = ld(im, off + 2 * q), zmr = ld(re, off + 3 * q), zmi = ld(im, off + 3 * q);
  const size_t km = (size_t)k * (N / n);
  dd_bfly(u0r, u0i, u1r, u1i, zpr, zpi, zmr, zmi, tw.c(km), tw.s(km));
  double *ore = swap_out ? im : re, *oim = swap_out ? re : im;
  auto st = [&](double *p, int m, dd v) {
    v = dd_scale(v, scale);
    p[m] = v.h;
    p[hplane + m] = v.l;
  };
  st(ore, off, u0r);
  st(oim, off, u0i);
  st(ore, off + q, u1r);
  st(oim, off + q, u1i);
  st(ore, off + 2 * q, zpr);
  st(oim, off + 2 * q, zpi);
  st(ore, off + 3 * q, zmr);
  st(oim, off + 3 * q, zmi);
}

static int dd_instances(const DDeviceTables &T) {
  if (T.nroots != 1) return 1;
  const int per = 4 * T.sub[0].size;
  return std::max(1, std::min(kDDSubMax / std::max(T.sub[0].size, 1), 8192 / per));
}

cudaError_t dd_run_transform(const DDeviceTables &T, const double *in, double *out, int B, double scale,
                             cudaStream_t s, bool swap_in, bool swap_out) {
  const int size = T.sub[0].size;
  const int G = dd_instances(T);
  const size_t smem = (size_t)G * 4 * size * sizeof(double);
  static bool attr_set = false;  // idempotent; benign race
  if (!attr_set) {
    cudaFuncSetAttribute(dd_sub_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    cudaFuncSetAttribute(dd_sub_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr_set = true;
  }
  const DDTw tw{T.wr, T.wrl, T.wi, T.wil};
  const bool final_sub = T.upper.nlevels == 0;
  if (T.nroots == 1) {
    dd_sub_kernel<true><<<(B + G - 1) / G, 256, smem, s>>>(in, out, T.N, B, T.roots, T.nroots, G, T.sub[0], T.sub[1],
                                                           tw, final_sub ? scale : 1.0, swap_in,
                                                           final_sub && swap_out);
  } else {
    dd_sub_kernel<false><<<T.nroots * B, 256, smem, s>>>(in, out, T.N, B, T.roots, T.nroots, 1, T.sub[0], T.sub[1],
                                                         tw, final_sub ? scale : 1.0, swap_in,
                                                         final_sub && swap_out);
  }
  for (int lv = 0; lv < T.upper.nlevels; ++lv) {
    const int n = T.upper.level_n[lv];
    const long long total = (long long)T.upper.level_count[lv] * (n / 4) * B;
    const bool last = lv == T.upper.nlevels - 1;
    dd_level_kernel<<<(int)((total + 255) / 256), 256, 0, s>>>(out, T.N, B, n, T.upper.node_off + T.upper.level_start[lv],
                                                              T.upper.level_count[lv], tw, last ? scale : 1.0,
                                                              last && swap_out);
  }
  return cudaGetLastError();
}

}  // namespace mpfft
