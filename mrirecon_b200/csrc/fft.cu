// Zero-pruned, fused oversampled 2D FFTs for the NUFFT (sm_100a).
//
// The oversampled grid of a coil-frame is zero outside the centred S0 x S1
// image band, and the adjoint keeps only that band.  Instead of the dense
// G0 x G1 transform (cuFFT: two read+write passes over the grid) plus separate
// pad and crop kernels, the forward runs
//   row pass    fused with SENSE x deapodisation x sign and the zero pad:
//               S0 band rows of length G1 per coil-frame, image -> T (vol, S0, G1)
//   column pass input-pruned (S0 of G0 inputs are non-zero): T -> grid
// and the adjoint
//   column pass output-pruned (only the S0 band rows are stored): grid -> T
//   row pass    fused with crop, deapodisation, sign and the conj(S_c) coil sum:
//               T -> image (nb, S0, S1)
// HBM traffic per direction: grid once (write or read) + T twice, about 40% of
// pad + cuFFT + crop.
//
// Each 1D transform is a Stockham autosort FFT over the radices 8, 4, 2, 3, 5
// (twiddles e^{-2 pi i r k / (p R)} tabulated on the host in double precision),
// computed in place in shared memory: a stage loads all of a thread's
// R-point butterflies into registers, synchronises, and writes them back.  The
// first stage loads straight from HBM and the last stage stores straight to
// HBM, so a length-512 transform costs two shared-memory round trips.
// Transform lengths are template parameters (the radix plan, twiddle offsets
// and per-thread work unroll at compile time); fft2_supported() lists them.
// Column kernels map consecutive threads to consecutive columns (128-byte
// global segments, odd shared-memory row stride => no bank conflicts); row
// kernels map consecutive threads along the row and pad shared memory by one
// element per 8.  Sign conventions follow nufft.cu: (-1)^(n0+n1) on the image
// side, the sample-side signs stay in the interp / spread weights.

#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <vector>

#include "mrb_common.cuh"
#include "fft.cuh"
#include "group.cuh"

namespace {

using mrb::VBlock;
using mrb::hw_block;

constexpr int ROW_NT = 256;   // threads per row-pass block
constexpr int COL_NT = 512;   // threads per column-pass block

// ---------------------------------------------------------------------------
// compile-time radix plan: 8s first, then 4, 2, 3, 5
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int next_radix(int g) {
  return g % 8 == 0 ? 8 : g % 4 == 0 ? 4 : g % 2 == 0 ? 2 : g % 3 == 0 ? 3 : g % 5 == 0 ? 5 : 0;
}
__host__ __device__ constexpr int n_stages(int G) {
  int n = 0;
  while (G > 1) {
    const int r = next_radix(G);
    if (r == 0) return -1;
    G /= r;
    ++n;
  }
  return n;
}
__host__ __device__ constexpr int radix_at(int G, int s) {
  for (int i = 0; i < s; ++i) G /= next_radix(G);
  return next_radix(G);
}
// product of the radices before stage s
__host__ __device__ constexpr int span_at(int G, int s) {
  int p = 1;
  for (int i = 0; i < s; ++i) {
    const int r = next_radix(G);
    p *= r;
    G /= r;
  }
  return p;
}
// offset of stage s in the twiddle table ([k][r-1] entries per stage)
__host__ __device__ constexpr int tw_offset(int G, int s) {
  int off = 0, p = 1;
  for (int i = 0; i < s; ++i) {
    const int r = next_radix(G);
    off += p * (r - 1);
    p *= r;
    G /= r;
  }
  return off;
}
__host__ __device__ constexpr int clamp_rows(int r) { return r < 1 ? 1 : r > 16 ? 16 : r; }
// transforms per block: about 8 (rows) / 16 (columns) complex values per thread
__host__ __device__ constexpr int rows_per_block(int G) { return clamp_rows(8 * ROW_NT / G); }
__host__ __device__ constexpr int cols_per_block(int G) { return clamp_rows(16 * COL_NT / G); }
// Row transforms keep their intermediate values in shared memory at the
// swizzled slot e ^ ((e >> 3) & 15) (a bijection inside each aligned group of
// 16), rows LD = roundup16(G) + 8 apart.  Against a plain layout this removes
// the 2-way bank conflicts of the radix-8 Stockham exchanges (stride-8 stores,
// runs of 8 at stride 64) for every compiled length; with the 64-bit accesses
// of a warp split in two 16-lane halves, G = 512 needs 128 wavefronts per row
// instead of 192 with the earlier "one pad slot per 8" layout.
__host__ __device__ constexpr int row_ld(int G) { return ((G + 15) & ~15) + 8; }
__host__ __device__ __forceinline__ int swz(int e) { return e ^ ((e >> 3) & 15); }

std::vector<float2> host_twiddles(int G) {
  std::vector<float2> t;
  const int ns = n_stages(G);
  for (int s = 0; s < ns; ++s) {
    const int R = radix_at(G, s), p = span_at(G, s);
    for (int k = 0; k < p; ++k)
      for (int r = 1; r < R; ++r) {
        const double a = -2.0 * M_PI * (double)r * (double)k / (double)(p * R);
        t.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
      }
  }
  t.push_back(make_float2(1.f, 0.f));
  return t;
}

// ---------------------------------------------------------------------------
// small DFTs: X_k = sum_n u_n e^{DIR 2 pi i k n / R}, in place
//
// Every floating-point operation of the passes is written with its rounding
// stated (fmaf, __fmul_rn, __fadd_rn, __fsub_rn and their packed pair forms;
// the file also compiles with -fmad=false), so the compiler fuses no multiply into an add on its own: a
// pass computes the same bits in every kernel that contains it (the named
// kernels and their grouped forms).  The butterflies fuse by hand where a
// scaled term is added (e +- h p).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -__fmul_rn(a.y, b.y)), fmaf(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(__fmul_rn(a.x, s), __fmul_rn(a.y, s)); }
template <int DIR>
__device__ __forceinline__ float2 cmul_di(float2 a) {   // a * (DIR i)
  return DIR > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// PK: the same sums, differences and scaled sums as packed pair instructions
// (sm_100 __fadd2_rn / __ffma2_rn, each component rounded as the scalar form; a - b
// as fma(b, -1, a), whose product is exact): the same bits in half the issue
// slots.  Only the inverse row pass uses them (measured 4.5% faster there; the
// column passes ran 1-4% slower with them).
template <bool PK>
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  if constexpr (PK) return __fadd2_rn(a, b);
  else return cadd(a, b);
}
template <bool PK>
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  if constexpr (PK) return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
  else return csub(a, b);
}
// a + h b, h real: one fused multiply-add per component
template <bool PK>
__device__ __forceinline__ float2 paxpy(float h, float2 b, float2 a) {
  if constexpr (PK) return __ffma2_rn(make_float2(h, h), b, a);
  else return make_float2(fmaf(h, b.x, a.x), fmaf(h, b.y, a.y));
}
// a + DIR i b, scalar (the sign of the exchanged component folds into the add)
template <int DIR>
__device__ __forceinline__ float2 cadd_di(float2 a, float2 b) {
  return DIR > 0 ? make_float2(__fsub_rn(a.x, b.y), __fadd_rn(a.y, b.x))
                 : make_float2(__fadd_rn(a.x, b.y), __fsub_rn(a.y, b.x));
}

template <int R, int DIR, bool PK = false>
struct Dft;

template <int DIR, bool PK>
struct Dft<2, DIR, PK> {
  __device__ __forceinline__ static void run(float2* u) {
    const float2 a = u[0], b = u[1];
    u[0] = padd<PK>(a, b);
    u[1] = psub<PK>(a, b);
  }
};

template <int DIR, bool PK>
struct Dft<4, DIR, PK> {
  __device__ __forceinline__ static void run(float2* u) {
    const float2 a0 = padd<PK>(u[0], u[2]), a1 = psub<PK>(u[0], u[2]);
    const float2 a2 = padd<PK>(u[1], u[3]), d = psub<PK>(u[1], u[3]);
    u[0] = padd<PK>(a0, a2);
    u[2] = psub<PK>(a0, a2);
    u[1] = cadd_di<DIR>(a1, d);    // a1 + DIR i d
    u[3] = cadd_di<-DIR>(a1, d);   // a1 - DIR i d
  }
};

template <int DIR, bool PK>
struct Dft<8, DIR, PK> {
  // radix-2 split into the 4-point DFTs of the even and odd samples
  __device__ __forceinline__ static void run(float2* u) {
    float2 e[4] = {u[0], u[2], u[4], u[6]};
    float2 o[4] = {u[1], u[3], u[5], u[7]};
    Dft<4, DIR, PK>::run(e);
    Dft<4, DIR, PK>::run(o);
    combine(e, o, u);
  }
  // u = (0, 0, u2, u3, u4, u5, 0, 0): the first stage of a transform whose input
  // is the centred half of its length (2x oversampled grid, even image size).
  // The 4-point DFTs of (0, u2, u4, 0) and (0, u3, u5, 0) without the terms in
  // the zeros: the same values as run() (up to the sign of an exact zero).
  __device__ __forceinline__ static void run_mid(float2* u) {
    float2 e[4], o[4];
    half4(u[2], u[4], e);
    half4(u[3], u[5], o);
    combine(e, o, u);
  }
  // Dft<4> of (0, b, c, 0): a0 = c, a1 = -c, a2 = b, a3 = DIR i b
  __device__ __forceinline__ static void half4(float2 b, float2 c, float2* x) {
    const float2 a3 = cmul_di<DIR>(b);
    x[0] = padd<PK>(c, b);
    x[2] = psub<PK>(c, b);
    x[1] = make_float2(__fsub_rn(a3.x, c.x), __fsub_rn(a3.y, c.y));
    x[3] = make_float2(-__fadd_rn(c.x, a3.x), -__fadd_rn(c.y, a3.y));
  }
  __device__ __forceinline__ static void combine(const float2* e, const float2* o, float2* u) {
    const float h = 0.707106781186547524f;
    // o_k * e^{DIR i pi k / 4}: o1 = h p1, p1 = o + DIR i o; o3 = h p3, p3 = DIR i o - o;
    // e_k +- h p_k as one fused multiply-add per component
    const float2 p1 = cadd_di<DIR>(o[1], o[1]);
    const float2 q3 = cmul_di<DIR>(o[3]);
    const float2 p3 = make_float2(__fsub_rn(q3.x, o[3].x), __fsub_rn(q3.y, o[3].y));
    u[0] = padd<PK>(e[0], o[0]);
    u[4] = psub<PK>(e[0], o[0]);
    u[1] = paxpy<PK>(h, p1, e[1]);
    u[5] = paxpy<PK>(-h, p1, e[1]);
    u[2] = cadd_di<DIR>(e[2], o[2]);    // e2 + DIR i o2
    u[6] = cadd_di<-DIR>(e[2], o[2]);   // e2 - DIR i o2
    u[3] = paxpy<PK>(h, p3, e[3]);
    u[7] = paxpy<PK>(-h, p3, e[3]);
  }
};

template <int DIR, bool PK>
struct Dft<3, DIR, PK> {
  __device__ __forceinline__ static void run(float2* u) {
    const float c1 = -0.5f, s1 = 0.866025403784438647f * (float)DIR;
    const float2 t1 = padd<PK>(u[1], u[2]), t2 = psub<PK>(u[1], u[2]);
    const float2 m = paxpy<PK>(c1, t1, u[0]);
    // m +- r, r = DIR i s1 t2, as fused multiply-adds
    u[0] = padd<PK>(u[0], t1);
    u[1] = make_float2(fmaf(-s1, t2.y, m.x), fmaf(s1, t2.x, m.y));
    u[2] = make_float2(fmaf(s1, t2.y, m.x), fmaf(-s1, t2.x, m.y));
  }
};

template <int DIR, bool PK>
struct Dft<5, DIR, PK> {
  __device__ __forceinline__ static void run(float2* u) {
    // cos / sin of 2 pi k / 5
    const float c1 = 0.309016994374947424f, c2 = -0.809016994374947424f;
    const float s1 = 0.951056516295153572f * (float)DIR, s2 = 0.587785252292473129f * (float)DIR;
    const float2 a1 = padd<PK>(u[1], u[4]), b1 = psub<PK>(u[1], u[4]);
    const float2 a2 = padd<PK>(u[2], u[3]), b2 = psub<PK>(u[2], u[3]);
    const float2 x0 = u[0];
    const float2 m1 = paxpy<PK>(c2, a2, paxpy<PK>(c1, a1, x0));
    const float2 m2 = paxpy<PK>(c1, a2, paxpy<PK>(c2, a1, x0));
    // m_k +- n_k with n1 = i (s1 b1 + s2 b2), n2 = i (s2 b1 - s1 b2), as fused multiply-adds
    u[0] = padd<PK>(x0, padd<PK>(a1, a2));
    u[1] = make_float2(fmaf(-s2, b2.y, fmaf(-s1, b1.y, m1.x)), fmaf(s2, b2.x, fmaf(s1, b1.x, m1.y)));
    u[4] = make_float2(fmaf(s2, b2.y, fmaf(s1, b1.y, m1.x)), fmaf(-s2, b2.x, fmaf(-s1, b1.x, m1.y)));
    u[2] = make_float2(fmaf(s1, b2.y, fmaf(-s2, b1.y, m2.x)), fmaf(-s1, b2.x, fmaf(s2, b1.x, m2.y)));
    u[3] = make_float2(fmaf(-s1, b2.y, fmaf(s2, b1.y, m2.x)), fmaf(s1, b2.x, fmaf(-s2, b1.x, m2.y)));
  }
};

// ---------------------------------------------------------------------------
// Stockham stages.  Item (q, i), i < T = G / R, of row q reads element
// i + r T and writes element (i - k) R + k + r P, k = i mod P.  QFAST maps
// consecutive threads to consecutive rows q (column kernels).
// ---------------------------------------------------------------------------
// WARP: the transform belongs to one warp (NT = 32, ROWS = 1) and the exchanges
// synchronise the warp only.
template <bool WARP>
__device__ __forceinline__ void stage_sync() {
  if (WARP) __syncwarp();
  else __syncthreads();
}

// MID: the first stage of a transform whose nonzero input is the centred half
// [G/4, 3G/4): with R = 8 and T = G/8 every butterfly's inputs i + r T are
// zero for r = 0, 1, 6, 7, so only r = 2..5 are loaded (Dft<8>::run_mid).
template <int G, int S, int ROWS, int NT, int DIR, bool QFAST, bool WARP, bool MID, bool PK, class LD, class ST>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ tw, LD load, ST store) {
  constexpr int R = radix_at(G, S);
  constexpr int P = span_at(G, S);
  constexpr int T = G / R;
  static_assert(!MID || (R == 8 && S == 0), "the centred-input stage is a first radix-8 stage");
  constexpr int TOTAL = ROWS * T;
  constexpr int NI = (TOTAL + NT - 1) / NT;
  static_assert(!WARP || (NT == 32 && ROWS == 1), "warp transforms are one row of 32 lanes");
  const int tid = WARP ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
  const float2* tws = tw + tw_offset(G, S);
  float2 v[NI][R];
#pragma unroll
  for (int c = 0; c < NI; ++c) {
    const int w = tid + c * NT;
    if (TOTAL % NT == 0 || w < TOTAL) {
      const int q = QFAST ? w % ROWS : w / T;
      const int i = QFAST ? w / ROWS : w % T;
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (!MID || (r >= 2 && r <= 5)) v[c][r] = load(q, i + r * T);
    }
  }
  stage_sync<WARP>();
#pragma unroll
  for (int c = 0; c < NI; ++c) {
    const int w = tid + c * NT;
    if (TOTAL % NT == 0 || w < TOTAL) {
      const int q = QFAST ? w % ROWS : w / T;
      const int i = QFAST ? w / ROWS : w % T;
      const int k = i % P;
      if (P > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 t = __ldg(tws + k * (R - 1) + r - 1);
          if (DIR > 0) t.y = -t.y;
          v[c][r] = cmul(v[c][r], t);
        }
      }
      if constexpr (MID) Dft<8, DIR, PK>::run_mid(v[c]);
      else Dft<R, DIR, PK>::run(v[c]);
      const int j = (i - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        // a store that takes (q, j, r P) gets the element j + r P with its
        // thread-dependent part j apart from the compile-time offset r P
        if constexpr (std::is_invocable_v<ST, int, int, int, float2>) store(q, j, r * P, v[c][r]);
        else store(q, j + r * P, v[c][r]);
      }
    }
  }
  stage_sync<WARP>();
}

// All stages of a length-G transform of ROWS rows: the first stage loads
// through load0, the last stores through store_last, and intermediate results
// live in buf (row q at q * LD, element e at slot swz(e) when PAD).
template <int G, int S, int ROWS, int NT, int DIR, bool QFAST, bool PAD, int LD, bool WARP = false, bool MID = false,
          bool PK = false, class LD0, class STL>
__device__ __forceinline__ void fft_stages(float2* buf, const float2* tw, LD0 load0, STL store_last) {
  constexpr int NS = n_stages(G);
  constexpr bool MID0 = MID && S == 0;
  if constexpr (S < NS) {
    auto sload = [&](int q, int e) { return buf[q * LD + (PAD ? swz(e) : e)]; };
    auto sstore = [&](int q, int e, float2 v) { buf[q * LD + (PAD ? swz(e) : e)] = v; };
    if constexpr (S == 0 && S == NS - 1) fft_stage<G, S, ROWS, NT, DIR, QFAST, WARP, MID0, PK>(tw, load0, store_last);
    else if constexpr (S == 0) fft_stage<G, S, ROWS, NT, DIR, QFAST, WARP, MID0, PK>(tw, load0, sstore);
    else if constexpr (S == NS - 1) fft_stage<G, S, ROWS, NT, DIR, QFAST, WARP, false, PK>(tw, sload, store_last);
    else fft_stage<G, S, ROWS, NT, DIR, QFAST, WARP, false, PK>(tw, sload, sstore);
    fft_stages<G, S + 1, ROWS, NT, DIR, QFAST, PAD, LD, WARP, MID, PK>(buf, tw, load0, store_last);
  }
}

// the nonzero input of a length-G transform is its centred half [G/4, 3G/4)
// and the transform starts with radix 8: the first stage may skip the zeros
template <int G>
__device__ __forceinline__ bool centred_half(int S, int off) {
  return radix_at(G, 0) == 8 && 2 * S == G && 4 * off == G;
}

struct Geo2 {
  int S0, S1, G0, G1, off0, off1, C;
  long long stot, gtot;
  const double* skip;   // when non-null and non-zero the kernels return at once
  int nvol;             // volumes of the pass (the forward column pass: nb x C)
};

// forward row pass: T[row][:] = FFT_G1(pad(x[be][r][:] * S_c * deapod * sign)),
// row = vol * S0 + r; one warp per row (warp-scope exchanges), ROW_WARPS rows per block
constexpr int ROW_WARPS = ROW_NT / 32;

template <int G1>
struct FwdRows {
  static constexpr int NT = ROW_NT, MINB = (G1 <= 256 ? 5 : G1 <= 512 ? 4 : G1 <= 640 ? 3 : G1 <= 768 ? 2 : 1);
  static constexpr const char* FAMILY = "fwd_rows";
  static __device__ __forceinline__ void run(const VBlock& vb, const float2* __restrict__ x,
      const float2* __restrict__ maps, const float* __restrict__ rowfac, const float* __restrict__ coldeap,
      float2* __restrict__ Tb, const float2* __restrict__ tw, const Geo2& g, long long nrows, int coil_images) {
    constexpr int LD = row_ld(G1);
    extern __shared__ float2 sm[];
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    const int warp = threadIdx.x >> 5;
    const long long row = (long long)vb.x * ROW_WARPS + warp;
    if (row >= nrows) return;                          // no block-wide barrier below
    float2* buf = sm + warp * LD;
    const long long vol = row / g.S0;
    const int r = (int)(row - vol * g.S0);
    const long long be = vol / g.C;
    const int c = (int)(vol - be * g.C);
    const float2* xr = x + (coil_images ? vol : be) * g.stot + (long long)r * g.S1;
    const float2* mr = maps + (long long)c * g.stot + (long long)r * g.S1;
    const float dr = __ldg(rowfac + r);   // signed deapodisation of the row
    float2* out = Tb + row * G1;
    auto load0 = [&](int, int n1) -> float2 {
      const int i1 = n1 - g.off1;
      if ((unsigned)i1 >= (unsigned)g.S1) return make_float2(0.f, 0.f);
      const float2 xv = xr[i1];
      const float2 mv = coil_images ? make_float2(1.f, 0.f) : __ldg(mr + i1);
      float s = __fmul_rn(dr, __ldg(coldeap + i1));
      if (n1 & 1) s = -s;
      return cscale(cmul(xv, mv), s);
    };
    auto store = [&](int, int k1, float2 v) { out[k1] = v; };
    if constexpr (radix_at(G1, 0) == 8) {
      if (centred_half<G1>(g.S1, g.off1)) {
        fft_stages<G1, 0, 1, 32, -1, false, true, LD, true, true>(buf, tw, load0, store);
        return;
      }
    }
    fft_stages<G1, 0, 1, 32, -1, false, true, LD, true>(buf, tw, load0, store);
  }
};
template <int G1>
__global__ void __launch_bounds__(ROW_NT, FwdRows<G1>::MINB) fwd_rows_kernel(const float2* __restrict__ x,
    const float2* __restrict__ maps, const float* __restrict__ rowfac, const float* __restrict__ coldeap,
    float2* __restrict__ Tb, const float2* __restrict__ tw, Geo2 g, long long nrows, int coil_images) {
  FwdRows<G1>::run(hw_block(), x, maps, rowfac, coldeap, Tb, tw, g, nrows, coil_images);
}

// forward column pass: grid[vol][:][k1] = FFT_G0(band rows of T[vol][:][k1]),
// COLS consecutive columns per block.  BLK: the grid is stored in blocks of
// 2 x 8 cells (fft.cuh: cell (n0, n1) of a volume at
// ((n0 / 2) * (G1 / 8) + n1 / 8) * 16 + (n0 % 2) * 8 + n1 % 8, G0 even, G1 a
// multiple of 8), the 2D interp's layout: a sample's 4 x 4 taps then meet 2
// to 6 128-byte lines instead of 4 to 8.  The last stage's stores of a warp
// cover rows 2m and 2m + 1 of 16 columns: whole blocks, as whole rows' lines
// in the row-major layout.
// 16-byte asynchronous copy global -> shared (completes at cp_async_wait_all)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Forward column pass: a block transforms two column tiles (COLS columns of a
// volume each, tiles 2 x and 2 x + 1 of the pass): the second tile's band rows
// are copied into shared memory (cp.async, S0 x COLS values after the exchange
// buffer) while the first is transformed, so its first stage reads them there
// instead of waiting for global loads.
template <int G0, bool BLK = false>
struct FwdCols {
  static constexpr int NT = COL_NT, MINB = (G0 <= 256 ? 3 : 2);
  static constexpr const char* FAMILY = "fwd_cols";
  static __device__ __forceinline__ void run(const VBlock& vb, const float2* __restrict__ Tb,
      float2* __restrict__ grid, const float2* __restrict__ tw, const Geo2& g) {
    constexpr int COLS = cols_per_block(G0);
    constexpr int LD = G0 | 1;
    extern __shared__ float2 sm[];
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    const int cblocks = (g.G1 + COLS - 1) / COLS;
    const long long ntile = (long long)g.nvol * cblocks;
    const long long t0 = 2LL * vb.x, t1 = t0 + 1;
    const bool has1 = t1 < ntile;
    // 32-bit offsets inside one volume (at most 1024^3 = 2^30 cells for the compiled lengths)
    const int G1 = g.G1;
    float2* stg = sm + COLS * LD;   // the second tile's band rows, (S0, COLS)
    if (has1) {
      const int vol = (int)(t1 / cblocks);
      const int k0 = (int)(t1 - (long long)vol * cblocks) * COLS;
      const float2* tv = Tb + (long long)vol * g.S0 * G1 + k0;
      constexpr int HC = COLS / 2;   // 16-byte pieces per band row (COLS is even)
      for (int c = threadIdx.x; c < g.S0 * HC; c += COL_NT) {
        const int r = c / HC, col = 2 * (c - r * HC);
        if (k0 + col < G1) cp_async16(stg + r * COLS + col, tv + r * G1 + col);
      }
    }
    auto tile = [&](long long t, bool staged) {
      const int vol = (int)(t / cblocks);
      const int k0 = (int)(t - (long long)vol * cblocks) * COLS;
      const bool full = k0 + COLS <= G1;
      const float2* tv = Tb + (long long)vol * g.S0 * G1 + k0;
      float2* gv = grid + (long long)vol * g.gtot + k0;
      auto load0 = [&](int q, int n0) -> float2 {
        const int r = n0 - g.off0;
        if ((unsigned)r >= (unsigned)g.S0 || (!full && k0 + q >= G1)) return make_float2(0.f, 0.f);
        return staged ? stg[r * COLS + q] : tv[r * G1 + q];
      };
      // BLK: 2 x 8 cell blocks; a thread's column k0 + q is fixed and its rows of the
      // last stage are n0 = j + r P (P even), so the address is a per-thread base plus
      // a multiple of 2 G1 per r
      float2* gb = grid + (long long)vol * g.gtot + ((k0 >> 3) << 4);
      auto store = [&](int q, int n0, float2 v) {
        if (full || k0 + q < G1) gv[n0 * G1 + q] = v;
      };
      // row n0 = j + rP of the last stage (P even): block row j / 2 + rP / 2, row in block j % 2
      auto store_blk = [&](int q, int j, int rP, float2 v) {
        if (full || k0 + q < G1) {
          const int c = (k0 & 7) + q;   // column k0 + q = 8 (k0 / 8) + c
          gb[((j >> 1) + (rP >> 1)) * (2 * G1) + (j & 1) * 8 + ((c >> 3) << 4) + (c & 7)] = v;
        }
      };
      auto go = [&](auto st) {
        if constexpr (radix_at(G0, 0) == 8) {
          if (centred_half<G0>(g.S0, g.off0)) {
            fft_stages<G0, 0, COLS, COL_NT, -1, true, false, LD, false, true>(sm, tw, load0, st);
            return;
          }
        }
        fft_stages<G0, 0, COLS, COL_NT, -1, true, false, LD>(sm, tw, load0, st);
      };
      if constexpr (BLK) {
        static_assert(span_at(G0, n_stages(G0) - 1) % 2 == 0, "the last stage's span must be even");
        go(store_blk);
      } else {
        go(store);
      }
    };
    tile(t0, false);
    if (has1) {
      cp_async_wait_all();
      __syncthreads();   // every thread's copies landed (the last stage ended with a barrier)
      tile(t1, true);
    }
  }
};
template <int G0, bool BLK>
__global__ void __launch_bounds__(COL_NT, FwdCols<G0, BLK>::MINB) fwd_cols_kernel(const float2* __restrict__ Tb,
    float2* __restrict__ grid, const float2* __restrict__ tw, Geo2 g) {
  FwdCols<G0, BLK>::run(hw_block(), Tb, grid, tw, g);
}

// forward column pass with a coil-interleaved output (3D x pass, see fft.cuh):
// a block transforms IL_ROWS (column, coil) pairs, coil fastest, so that each
// output row holds runs of contiguous values of the (cell, coil) layout
constexpr int IL_ROWS = 32;

// A block takes IL_CG coils of its frame (groups of 8): its band reads per coil
// and row are IL_ROWS / 8 = 4 consecutive columns, one whole 32-byte sector
// (with all CT coils in one block they were 2 columns, half a sector), and its
// stores per cell are IL_CG coils, 64 contiguous bytes of the cell's CT.
template <int CT>
__host__ __device__ constexpr int il_cg() { return CT < 8 ? CT : 8; }

template <int G0, int CT>
__global__ void __launch_bounds__(COL_NT, G0 <= 320 ? 2 : 1) fwd_cols_il_kernel(const float2* __restrict__ Tb, float2* __restrict__ out,
                                                             const float2* __restrict__ tw, Geo2 g) {
  constexpr int LD = G0 | 1;
  constexpr int CG = il_cg<CT>();    // coils per block
  constexpr int CB = IL_ROWS / CG;   // columns per block
  extern __shared__ float2 sm[];
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  const int cblocks = (g.G1 + CB - 1) / CB;
  const int vg = blockIdx.x / cblocks;   // (frame, coil group)
  const int k0 = (blockIdx.x - vg * cblocks) * CB;
  const int be = vg / (CT / CG), c0 = (vg - be * (CT / CG)) * CG;
  const float2* tb = Tb + ((long long)be * CT + c0) * g.S0 * g.G1;   // (coil, band row, column)
  float2* ob = out + (long long)be * g.gtot * CT + c0;               // (cell, coil)
  auto load0 = [&](int q, int n0) -> float2 {
    const int j = q / CG, c = q - j * CG;
    const int r = n0 - g.off0;
    if ((unsigned)r >= (unsigned)g.S0 || k0 + j >= g.G1) return make_float2(0.f, 0.f);
    return tb[((long long)c * g.S0 + r) * g.G1 + k0 + j];
  };
  auto store = [&](int q, int n0, float2 v) {
    const int j = q / CG, c = q - j * CG;
    if (k0 + j < g.G1) ob[((long long)n0 * g.G1 + k0 + j) * CT + c] = v;
  };
  fft_stages<G0, 0, IL_ROWS, COL_NT, -1, true, false, LD>(sm, tw, load0, store);
}

// forward column pass writing a coil-quad grid (2D, see fft.cuh): a block
// transforms its COLS (column, coil) pairs as CJ consecutive columns of CG
// consecutive coils of one frame, so that its band reads are runs of CJ
// columns of a coil (32 bytes for CJ = 4) and its grid stores, in the layout
// (frame, coil quad, cell, coil in quad), runs of CJ cells x 4 coils (one
// 128-byte line for CJ = CG = 4).  Same transforms as fwd_cols_kernel: the
// grid values are identical, only their order in memory differs.  C % 4 == 0.
template <int G0>
struct ColGroups {
  static constexpr int COLS = cols_per_block(G0);
  static constexpr int CG = COLS % 4 == 0 ? 4 : COLS % 2 == 0 ? 2 : 1;
  static constexpr int CJ = COLS / CG;
};

template <int G0>
__global__ void __launch_bounds__(COL_NT) fwd_cols_cg_kernel(const float2* __restrict__ Tb, float2* __restrict__ out,
                                                             const float2* __restrict__ tw, Geo2 g) {
  constexpr int COLS = ColGroups<G0>::COLS;
  constexpr int CG = ColGroups<G0>::CG;
  constexpr int CJ = ColGroups<G0>::CJ;
  constexpr int LD = G0 | 1;
  extern __shared__ float2 sm[];
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  const int G1 = g.G1, C = g.C;
  const int cblocks = (G1 + CJ - 1) / CJ;
  const int cgroups = (C + CG - 1) / CG;
  int blk = blockIdx.x;
  const int cb = blk % cblocks;
  blk /= cblocks;
  const int cgi = blk % cgroups;
  const int be = blk / cgroups;
  const int k0 = cb * CJ, c0 = cgi * CG;
  const float2* tb = Tb + ((long long)be * C + c0) * g.S0 * G1 + k0;          // (coil, band row, column)
  // quad plane of coil c0 (4 coils x gtot cells), then (cell, coil in quad)
  float2* ob = out + ((long long)be * C + (c0 & ~3)) * g.gtot + (long long)k0 * 4 + (c0 & 3);
  // 32-bit offsets inside one frame's band and quad (C * S0 * G1 and 4 * G0 * G1 < 2^31,
  // checked on the host); a thread's (column, coil) pair is fixed across its elements
  const int S0G1 = g.S0 * G1;
  const bool full = k0 + CJ <= G1 && c0 + CG <= C;
  auto load0 = [&](int q, int n0) -> float2 {
    const int j = q % CJ, cc = q / CJ;
    const int r = n0 - g.off0;
    if ((unsigned)r >= (unsigned)g.S0 || (!full && (k0 + j >= G1 || c0 + cc >= C))) return make_float2(0.f, 0.f);
    return tb[cc * S0G1 + r * G1 + j];
  };
  auto store = [&](int q, int n0, float2 v) {
    const int j = q % CJ, cc = q / CJ;
    if (full || (k0 + j < G1 && c0 + cc < C)) ob[(n0 * G1 + j) * 4 + cc] = v;
  };
  fft_stages<G0, 0, COLS, COL_NT, -1, true, false, LD>(sm, tw, load0, store);
}

// forward column pass fused with the interp (see fft.cuh): COLS columns per
// block, the first COLS - 3 owned by the block's strip, the last three its
// halo; the column transforms end in shared memory, then the threads walk the
// strip's sample list.  Taps, signs, weights and the summation order are those
// of the gridded interp (rows i0 outer, columns i1 inner), so the samples are
// the same bit for bit.
template <int G0>
__global__ void __launch_bounds__(COL_NT, 2) fwd_cols_interp_kernel(const float2* __restrict__ Tb,
                                                                 const float2* __restrict__ tw, Geo2 g,
                                                                 mrb::ColInterp ci) {
  constexpr int COLS = cols_per_block(G0);
  constexpr int SW = COLS - 3;
  constexpr int LD = G0 | 1;
  constexpr int W = 4;
  extern __shared__ float2 sm[];
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  const int vol = blockIdx.x / ci.nstrips;
  const int strip = blockIdx.x - vol * ci.nstrips;
  const int k0 = strip * SW;
  const float2* tv = Tb + (long long)vol * g.S0 * g.G1;
  // the strip's first COL_NT samples (index and coordinates) are loaded while
  // the columns transform
  const int be = vol / g.C;
  const int b = ci.B == 1 ? 0 : be / (ci.nb / ci.B);
  const int key = b * ci.nstrips + strip;
  const int e0 = ci.strip_start[key], e1 = ci.strip_start[key + 1];
  const float* gx0 = ci.gx + (long long)b * 2 * ci.K;
  int pk = 0;
  float px[2] = {0.f, 0.f};
  if (e0 + (int)threadIdx.x < e1) {
    pk = ci.strip_entries[e0 + threadIdx.x];
    px[0] = gx0[pk];
    px[1] = gx0[ci.K + pk];
  }
  auto load0 = [&](int q, int n0) -> float2 {
    const int r = n0 - g.off0;
    if ((unsigned)r >= (unsigned)g.S0) return make_float2(0.f, 0.f);
    int col = k0 + q;
    col -= col >= g.G1 ? g.G1 : 0;
    return tv[(long long)r * g.G1 + col];
  };
  auto store = [&](int q, int n0, float2 v) { sm[q * LD + n0] = v; };
  fft_stages<G0, 0, COLS, COL_NT, -1, true, false, LD>(sm, tw, load0, store);
  __syncthreads();
  float2* yo = ci.y + (long long)vol * ci.K;
  for (int e = e0 + threadIdx.x; e < e1; e += COL_NT) {
    const bool first = e < e0 + COL_NT;
    const int k = first ? pk : ci.strip_entries[e];
    float w[2][W];
    int row[W], cq[W];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const float x = first ? px[d] : gx0[(long long)d * ci.K + k];
      const int base = (int)floorf(x);
      const float fx = x - (float)base;
#pragma unroll
      for (int o = 0; o < W; ++o) {
        const int n = base - (W / 2 - 1) + o;
        const float wd = mrb::kb_tap(ci.kb, o, fx);
        w[d][o] = (n & 1) ? -wd : wd;
        if (d == 0) {
          row[o] = mrb::wrap_i(n, g.G0);
        } else {
          int q = mrb::wrap_i(n, g.G1) - k0;
          q += q < 0 ? g.G1 : 0;
          cq[o] = q * LD;
        }
      }
    }
    float s = ci.scale;
    if (ci.wfwd) s *= ci.wfwd[(long long)b * ci.K + k];
    float re = 0.f, im = 0.f;
#pragma unroll
    for (int i0 = 0; i0 < W; ++i0) {
      float a0 = 0.f, b0 = 0.f;
#pragma unroll
      for (int i1 = 0; i1 < W; ++i1) {
        const float2 v = sm[cq[i1] + row[i0]];
        a0 = fmaf(w[1][i1], v.x, a0);
        b0 = fmaf(w[1][i1], v.y, b0);
      }
      re = fmaf(w[0][i0], a0, re);
      im = fmaf(w[0][i0], b0, im);
    }
    yo[k] = make_float2(re * s, im * s);
  }
}

// adjoint column pass: T[vol][r][k1] = IFFT_G0(grid[vol][:][k1])[r + off0]
template <int G0>
struct AdjCols {
  static constexpr int NT = COL_NT, MINB = (G0 <= 256 ? 3 : 2);
  static constexpr const char* FAMILY = "adj_cols";
  static __device__ __forceinline__ void run(const VBlock& vb, const float2* __restrict__ grid,
      float2* __restrict__ Tb, const float2* __restrict__ tw, const Geo2& g) {
    constexpr int COLS = cols_per_block(G0);
    constexpr int LD = G0 | 1;
    extern __shared__ float2 sm[];
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    const int cblocks = (g.G1 + COLS - 1) / COLS;
    const int vol = vb.x / cblocks;
    const int k0 = (vb.x - vol * cblocks) * COLS;
    // 32-bit offsets inside one volume (at most 1024^3 = 2^30 cells for the compiled lengths)
    const int G1 = g.G1;
    const bool full = k0 + COLS <= G1;
    const float2* gv = grid + (long long)vol * g.gtot + k0;
    float2* tv = Tb + (long long)vol * g.S0 * G1 + k0;
    auto load0 = [&](int q, int n0) -> float2 {
      if (!full && k0 + q >= G1) return make_float2(0.f, 0.f);
      return gv[n0 * G1 + q];
    };
    auto store = [&](int q, int n0, float2 v) {
      const int r = n0 - g.off0;
      if ((unsigned)r < (unsigned)g.S0 && (full || k0 + q < G1)) tv[r * G1 + q] = v;
    };
    fft_stages<G0, 0, COLS, COL_NT, +1, true, false, LD>(sm, tw, load0, store);
  }
};
template <int G0>
__global__ void __launch_bounds__(COL_NT) adj_cols_kernel(const float2* __restrict__ grid,
    float2* __restrict__ Tb, const float2* __restrict__ tw, Geo2 g) {
  AdjCols<G0>::run(hw_block(), grid, Tb, tw, g);
}

// Toeplitz column pass (normal operator A^H A by circular convolution on the
// 2x grid): for each column of the band, T <- IFFT_G0(P[frame] * FFT_G0(T)),
// band rows in, band rows out, the column never leaves shared memory.
// P (B, G0, G1) float is the real transfer function, already rolled by G/2 in
// both dims (the row passes' (-1)^n signs) and scaled.
template <int G0>
__global__ void __launch_bounds__(COL_NT) toeplitz_cols_kernel(float2* __restrict__ Tb,
                                                               const float* __restrict__ P,
                                                               const float2* __restrict__ tw, Geo2 g, int nb,
                                                               int B) {
  constexpr int COLS = cols_per_block(G0);
  constexpr int LD = G0 | 1;
  extern __shared__ float2 sm[];
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  const int cblocks = (g.G1 + COLS - 1) / COLS;
  const int vol = blockIdx.x / cblocks;
  const int k0 = (blockIdx.x - vol * cblocks) * COLS;
  const int be = vol / g.C;
  const int b = (B == 1) ? 0 : be / (nb / B);
  float2* tv = Tb + (long long)vol * g.S0 * g.G1;
  const float* pb = P + (long long)b * g.gtot;
  auto load0 = [&](int q, int n0) -> float2 {
    const int r = n0 - g.off0;
    if ((unsigned)r >= (unsigned)g.S0 || k0 + q >= g.G1) return make_float2(0.f, 0.f);
    return tv[(long long)r * g.G1 + k0 + q];
  };
  auto sload = [&](int q, int e) { return sm[q * LD + e]; };
  auto sstore = [&](int q, int e, float2 v) { sm[q * LD + e] = v; };
  fft_stages<G0, 0, COLS, COL_NT, -1, true, false, LD>(sm, tw, load0, sstore);
  for (int e = threadIdx.x; e < COLS * G0; e += COL_NT) {
    const int q = e % COLS, kr = e / COLS;
    const float p = k0 + q < g.G1 ? __ldg(pb + (long long)kr * g.G1 + k0 + q) : 0.f;
    float2 v = sm[q * LD + kr];
    sm[q * LD + kr] = cscale(v, p);
  }
  __syncthreads();
  auto store = [&](int q, int n0, float2 v) {
    const int r = n0 - g.off0;
    if ((unsigned)r < (unsigned)g.S0 && k0 + q < g.G1) tv[(long long)r * g.G1 + k0 + q] = v;
  };
  fft_stages<G0, 0, COLS, COL_NT, +1, true, false, LD>(sm, tw, sload, store);
}

// adjoint row pass: x[be][r][i1] = scale * deapod * sign *
//   sum_c conj(S_c) IFFT_G1(T[(be, c)][r][:])[i1 + off1], one block per (be, r).
// Each of the ARW_WARPS warps transforms one coil row (warp-synchronous stages,
// no block barrier inside a transform, as the forward row pass); after each pass
// of ARW_WARPS coils the block adds them to the row's accumulators in coil order.
constexpr int ARW_WARPS = 4;

template <int G1>
struct AdjRows {
  static constexpr int NT = ARW_WARPS * 32, MINB = (G1 <= 256 ? 8 : G1 <= 512 ? 6 : 4);
  static constexpr const char* FAMILY = "adj_rows";
  static __device__ __forceinline__ void run(const VBlock& vb, const float2* __restrict__ Tb,
      const float2* __restrict__ maps, const float* __restrict__ rowfac, const float* __restrict__ coldeap,
      float2* __restrict__ x, const float2* __restrict__ tw, const Geo2& g, float scale) {
    constexpr int LD = row_ld(G1);
    extern __shared__ float2 sm[];
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    float2* acc = sm + ARW_WARPS * LD;   // S1 accumulators
    const int warp = threadIdx.x >> 5;
    const int row = vb.x;
    const int be = row / g.S0;
    const int r = row - be * g.S0;
    float2* buf = sm + warp * LD;
    for (int i = threadIdx.x; i < g.S1; i += NT) acc[i] = make_float2(0.f, 0.f);
    for (int c0 = 0; c0 < g.C; c0 += ARW_WARPS) {
      const int ncl = min(ARW_WARPS, g.C - c0);
      if (warp < ncl) {
        const float2* tb = Tb + (((long long)be * g.C + c0 + warp) * g.S0 + r) * G1;
        auto load0 = [&](int, int n1) -> float2 { return tb[n1]; };
        auto sstore = [&](int, int e, float2 v) { buf[swz(e)] = v; };
        fft_stages<G1, 0, 1, 32, +1, false, true, LD, true, false, true>(buf, tw, load0, sstore);
      }
      __syncthreads();
      for (int i = threadIdx.x; i < g.S1; i += NT) {
        float2 s = acc[i];
        const int e = i + g.off1;
        const int pe = swz(e);
        const float2* mp = maps + (long long)c0 * g.stot + (long long)r * g.S1 + i;
        for (int q = 0; q < ncl; ++q) {
          const float2 v = sm[q * LD + pe];
          const float2 m = __ldg(mp + (long long)q * g.stot);
          // s += conj(m) v
          s.x = __fadd_rn(s.x, fmaf(m.x, v.x, __fmul_rn(m.y, v.y)));
          s.y = __fadd_rn(s.y, fmaf(m.x, v.y, -__fmul_rn(m.y, v.x)));
        }
        acc[i] = s;
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < g.S1; i += NT) {
      float d = __fmul_rn(__fmul_rn(scale, __ldg(rowfac + r)), __ldg(coldeap + i));
      if ((i + g.off1) & 1) d = -d;
      const float2 s = acc[i];
      x[((long long)be * g.S0 + r) * g.S1 + i] = make_float2(s.x * d, s.y * d);
    }
  }
};
template <int G1>
__global__ void __launch_bounds__(AdjRows<G1>::NT, AdjRows<G1>::MINB) adj_rows_kernel(const float2* __restrict__ Tb,
    const float2* __restrict__ maps, const float* __restrict__ rowfac, const float* __restrict__ coldeap,
    float2* __restrict__ x, const float2* __restrict__ tw, Geo2 g, float scale) {
  AdjRows<G1>::run(hw_block(), Tb, maps, rowfac, coldeap, x, tw, g, scale);
}

Geo2 make_geo2(int S0, int S1, int G0, int G1, int C, const double* skip) {
  return Geo2{S0, S1, G0, G1, G0 / 2 - S0 / 2, G1 / 2 - S1 / 2, C, (long long)S0 * S1, (long long)G0 * G1, skip, 0};
}

int set_smem(const void* fn, size_t bytes) {
  MRB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return 0;
}

// the transform lengths with compiled kernels
#define MRB_FFT_LENGTHS(X) \
  X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(160) X(192) X(256) X(320) X(384) X(512) X(640) X(768) X(1024)

bool length_supported(int G) {
  switch (G) {
#define MRB_CASE(n) case n:
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    return true;
    default:
      return false;
  }
}

template <int G1>
int launch_fwd_rows(const void* x, const float2* maps, const float* rowfac, const float* coldeap, float2* Tb,
                    const float2* tw,
                    const Geo2& g, int nb, int coil_images, cudaStream_t st) {
  const size_t smem = (size_t)ROW_WARPS * row_ld(G1) * sizeof(float2);
  int rc;
  if ((rc = set_smem((const void*)fwd_rows_kernel<G1>, smem))) return rc;
  const long long nrows = (long long)nb * g.C * g.S0;
  const long long blocks = (nrows + ROW_WARPS - 1) / ROW_WARPS;
  MRB_REQUIRE(blocks < (1LL << 31), "too many rows");
  return mrb::launch<FwdRows<G1>>(fwd_rows_kernel<G1>, dim3((unsigned)blocks), smem, st, (const float2*)x, maps, rowfac,
                                  coldeap, Tb, tw, g, nrows, coil_images);
}

template <int G0>
int launch_cols(bool forward, const float2* in, float2* out, const float2* tw, const Geo2& g, int nb, bool blocked,
                cudaStream_t st) {
  constexpr int COLS = cols_per_block(G0);
  const size_t smem = (size_t)COLS * (G0 | 1) * sizeof(float2);
  const long long blocks = (long long)nb * g.C * ((g.G1 + COLS - 1) / COLS);
  MRB_REQUIRE(blocks < (1LL << 31), "too many columns");
  int rc;
  if (forward) {
    // two column tiles per block, the second one's band rows staged in shared memory
    Geo2 gf = g;
    gf.nvol = nb * g.C;
    const size_t smem_f = smem + (size_t)g.S0 * COLS * sizeof(float2);
    const long long fblocks = (blocks + 1) / 2;
    MRB_REQUIRE(g.G1 % 2 == 0, "the forward column pass needs an even row length");
    if (blocked) {
      MRB_REQUIRE(G0 % 2 == 0 && g.G1 % 8 == 0, "2 x 8 cell blocks need G0 even and G1 divisible by 8");
      if ((rc = set_smem((const void*)fwd_cols_kernel<G0, true>, smem_f))) return rc;
      return mrb::launch<FwdCols<G0, true>>(fwd_cols_kernel<G0, true>, dim3((unsigned)fblocks), smem_f, st, in, out,
                                            tw, gf);
    }
    if ((rc = set_smem((const void*)fwd_cols_kernel<G0, false>, smem_f))) return rc;
    return mrb::launch<FwdCols<G0>>(fwd_cols_kernel<G0, false>, dim3((unsigned)fblocks), smem_f, st, in, out, tw,
                                    gf);
  }
  if ((rc = set_smem((const void*)adj_cols_kernel<G0>, smem))) return rc;
  return mrb::launch<AdjCols<G0>>(adj_cols_kernel<G0>, dim3((unsigned)blocks), smem, st, in, out, tw, g);
}

template <int G0, int CT>
int launch_cols_il(const float2* in, float2* out, const float2* tw, const Geo2& g, int nb, cudaStream_t st) {
  constexpr int CG = il_cg<CT>();
  constexpr int CB = IL_ROWS / CG;
  const size_t smem = (size_t)IL_ROWS * (G0 | 1) * sizeof(float2);
  MRB_REQUIRE(smem <= 200 * 1024, "interleaved column pass needs %zu bytes of shared memory", smem);
  const long long blocks = (long long)nb * (CT / CG) * ((g.G1 + CB - 1) / CB);
  MRB_REQUIRE(blocks < (1LL << 31), "too many columns");
  int rc;
  if ((rc = set_smem((const void*)fwd_cols_il_kernel<G0, CT>, smem))) return rc;
  fwd_cols_il_kernel<G0, CT><<<(unsigned)blocks, COL_NT, smem, st>>>(in, out, tw, g);
  MRB_LAUNCH_CHECK();
  return 0;
}

template <int G0>
int launch_cols_cg(const float2* in, float2* out, const float2* tw, const Geo2& g, int nb, cudaStream_t st) {
  constexpr int COLS = ColGroups<G0>::COLS;
  constexpr int CG = ColGroups<G0>::CG;
  constexpr int CJ = ColGroups<G0>::CJ;
  const size_t smem = (size_t)COLS * (G0 | 1) * sizeof(float2);
  const long long blocks = (long long)nb * ((g.C + CG - 1) / CG) * ((g.G1 + CJ - 1) / CJ);
  MRB_REQUIRE(blocks < (1LL << 31), "too many columns");
  MRB_REQUIRE((long long)g.C * g.S0 * g.G1 < (1LL << 31) && 4LL * g.gtot < (1LL << 31),
              "frame too large for the coil-quad column pass");
  int rc;
  if ((rc = set_smem((const void*)fwd_cols_cg_kernel<G0>, smem))) return rc;
  fwd_cols_cg_kernel<G0><<<(unsigned)blocks, COL_NT, smem, st>>>(in, out, tw, g);
  MRB_LAUNCH_CHECK();
  return 0;
}

template <int G0>
int launch_cols_interp(const float2* in, const float2* tw, const Geo2& g, int nb, const mrb::ColInterp& ci,
                       cudaStream_t st) {
  constexpr int COLS = cols_per_block(G0);
  static_assert(COLS >= 4, "a strip needs at least one own column besides the 3 halo columns");
  const size_t smem = (size_t)COLS * (G0 | 1) * sizeof(float2);
  const long long blocks = (long long)nb * g.C * ci.nstrips;
  MRB_REQUIRE(blocks < (1LL << 31), "too many column strips");
  MRB_REQUIRE(g.G1 >= COLS, "grid narrower than a column block");
  int rc;
  if ((rc = set_smem((const void*)fwd_cols_interp_kernel<G0>, smem))) return rc;
  fwd_cols_interp_kernel<G0><<<(unsigned)blocks, COL_NT, smem, st>>>(in, tw, g, ci);
  MRB_LAUNCH_CHECK();
  return 0;
}

template <int G0>
int launch_toeplitz_cols(float2* Tb, const float* P, const float2* tw, const Geo2& g, int nb, int B,
                         cudaStream_t st) {
  constexpr int COLS = cols_per_block(G0);
  const size_t smem = (size_t)COLS * (G0 | 1) * sizeof(float2);
  const long long blocks = (long long)nb * g.C * ((g.G1 + COLS - 1) / COLS);
  MRB_REQUIRE(blocks < (1LL << 31), "too many columns");
  int rc;
  if ((rc = set_smem((const void*)toeplitz_cols_kernel<G0>, smem))) return rc;
  toeplitz_cols_kernel<G0><<<(unsigned)blocks, COL_NT, smem, st>>>(Tb, P, tw, g, nb, B);
  MRB_LAUNCH_CHECK();
  return 0;
}

template <int G1>
int launch_adj_rows(const float2* Tb, const float2* maps, const float* rowfac, const float* coldeap, void* x,
                    const float2* tw,
                    const Geo2& g, int nb, float scale, cudaStream_t st) {
  const size_t smem = ((size_t)ARW_WARPS * row_ld(G1) + g.S1) * sizeof(float2);
  int rc;
  if ((rc = set_smem((const void*)adj_rows_kernel<G1>, smem))) return rc;
  const long long blocks = (long long)nb * g.S0;
  MRB_REQUIRE(blocks < (1LL << 31), "too many rows");
  return mrb::launch<AdjRows<G1>>(adj_rows_kernel<G1>, dim3((unsigned)blocks), smem, st, Tb, maps, rowfac, coldeap,
                                  (float2*)x, tw, g, scale);
}

}  // namespace

namespace mrb {

bool fft2_supported(int S0, int S1, int G0, int G1) {
  return length_supported(G0) && length_supported(G1) && S0 <= G0 && S1 <= G1;
}

size_t fft2_tmp_bytes(int S0, int G1, int C, int nb) { return (size_t)nb * C * S0 * G1 * sizeof(float2); }

int fft2_twiddles(DevBuf& tw, int G, const float2** out) {
  std::vector<float2> t = host_twiddles(G);
  int rc = tw.ensure(t.size() * sizeof(float2));
  if (rc) return rc;
  MRB_CUDA_TRY(cudaMemcpy(tw.p, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice));
  *out = tw.as<float2>();
  return 0;
}

int fft2_forward_rows(const void* x, const float2* maps, const float* rowfac, const float* coldeap, float2* Tb,
                      const float2* tw1, int S0,
                      int S1, int G0, int G1, int C, int nb, int coil_images, const double* skip,
                      cudaStream_t st) {
  const Geo2 g = make_geo2(S0, S1, G0, G1, C, skip);
  switch (G1) {
#define MRB_CASE(n) \
  case n: return launch_fwd_rows<n>(x, maps, rowfac, coldeap, Tb, tw1, g, nb, coil_images, st);
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      return fail(MRB_EINVAL, "no fused FFT for length %d", G1);
  }
}

int fft2_columns(int forward, const float2* in, float2* out, const float2* tw0, int S0, int S1, int G0, int G1, int C,
                 int nb, const double* skip, cudaStream_t st, int blocked) {
  const Geo2 g = make_geo2(S0, S1, G0, G1, C, skip);
  switch (G0) {
#define MRB_CASE(n) \
  case n: return launch_cols<n>(forward != 0, in, out, tw0, g, nb, blocked != 0, st);
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      return fail(MRB_EINVAL, "no fused FFT for length %d", G0);
  }
}

bool fft2_columns_il_supported(int G0, int C) {
  return (C == 8 || C == 16 || C == 32) && length_supported(G0) && (size_t)IL_ROWS * (G0 | 1) * 8 <= 200 * 1024;
}

int fft2_columns_il(const float2* Tb, float2* out, const float2* tw0, int S0, int G0, int G1, int C, int nb,
                    const double* skip, cudaStream_t st) {
  const Geo2 g = make_geo2(S0, G1, G0, G1, C, skip);
  switch (G0) {
#define MRB_CASE(n)                                                             \
  case n:                                                                       \
    if (C == 8) return launch_cols_il<n, 8>(Tb, out, tw0, g, nb, st);           \
    if (C == 16) return launch_cols_il<n, 16>(Tb, out, tw0, g, nb, st);         \
    if (C == 32) return launch_cols_il<n, 32>(Tb, out, tw0, g, nb, st);         \
    break;
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      break;
  }
  return fail(MRB_EINVAL, "no interleaved column pass for length %d and %d coils", G0, C);
}

int fft2_columns_cg(const float2* Tb, float2* out, const float2* tw0, int S0, int S1, int G0, int G1, int C, int nb,
                    const double* skip, cudaStream_t st) {
  const Geo2 g = make_geo2(S0, S1, G0, G1, C, skip);
  switch (G0) {
#define MRB_CASE(n) \
  case n: return launch_cols_cg<n>(Tb, out, tw0, g, nb, st);
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      return fail(MRB_EINVAL, "no fused FFT for length %d", G0);
  }
}

int interp_strip_width(int G0) {
  switch (G0) {
#define MRB_CASE(n) \
  case n: return cols_per_block(n) - 3;
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      return 0;
  }
}

int fft2_columns_interp(const float2* Tb, const float2* tw0, int S0, int S1, int G0, int G1, int C, int nb,
                        const ColInterp& ci, const double* skip, cudaStream_t st) {
  const Geo2 g = make_geo2(S0, S1, G0, G1, C, skip);
  switch (G0) {
#define MRB_CASE(n) \
  case n: return launch_cols_interp<n>(Tb, tw0, g, nb, ci, st);
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      return fail(MRB_EINVAL, "no fused FFT for length %d", G0);
  }
}

int fft2_toeplitz_columns(float2* Tb, const float* P, const float2* tw0, int S0, int S1, int G0, int G1, int C, int nb,
                          int B, const double* skip, cudaStream_t st) {
  const Geo2 g = make_geo2(S0, S1, G0, G1, C, skip);
  switch (G0) {
#define MRB_CASE(n) \
  case n: return launch_toeplitz_cols<n>(Tb, P, tw0, g, nb, B, st);
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      return fail(MRB_EINVAL, "no fused FFT for length %d", G0);
  }
}

int fft2_adjoint_rows(const float2* Tb, const float2* maps, const float* rowfac, const float* coldeap, void* x,
                      const float2* tw1, int S0,
                      int S1, int G0, int G1, int C, int nb, float scale, const double* skip,
                      cudaStream_t st) {
  const Geo2 g = make_geo2(S0, S1, G0, G1, C, skip);
  switch (G1) {
#define MRB_CASE(n) \
  case n: return launch_adj_rows<n>(Tb, maps, rowfac, coldeap, x, tw1, g, nb, scale, st);
    MRB_FFT_LENGTHS(MRB_CASE)
#undef MRB_CASE
    default:
      return fail(MRB_EINVAL, "no fused FFT for length %d", G1);
  }
}

}  // namespace mrb
