// Kaiser-Bessel NUFFT for B200 (sm_100a): binning, forward interp, adjoint
// spread, fused SENSE/deapodisation/pad and crop/coil-combine, cuFFT for the
// dense oversampled transform.
//
// Conventions (corrected form of graspcg/nufft/backends/ptnufft.py):
//   gx_d   = clamp((w_d / float32(2pi) + 0.5) * G_d, 0, float32(G_d - 1e-6))
//            in float32, same operation order as ptnufft.py:151-153;
//   nodes  n = floor(gx) + o, o in [-W/2+1, W/2], distance d = gx - n,
//            weight phi(d) (KB, ptnufft.py:79-90 / :125), index n mod G;
//   image pixel i sits at node i + G/2 - S//2 (centred coordinate i - S//2);
//   fftshift o FFT o ifftshift is applied as (-1)^(sum n) on the input and
//   (-1)^(sum k) * prod (-1)^(G_d/2) on the output of the unshifted FFT.
//
// Layouts: x (nb, 1, *S), maps (C, *S), y (nb, C, K), grid (nb, C, *G), all
// complex64 row-major.  Frame be of an nb-batch uses trajectory frame
// be / (nb / B) (graspcg/nufft/backends/torchkb.py:151-166).

#include <cuda_runtime.h>
#include <cufft.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mrb_common.cuh"
#include "fft.cuh"
#include "group.cuh"

using mrb::DevBuf;
using mrb::KBPoly;
using mrb::VBlock;
using mrb::hw_block;

struct mrb_plan {
  int nd = 2;
  int S[3] = {1, 1, 1};
  int G[3] = {1, 1, 1};
  int C = 1;
  int B = 1;
  int64_t K = 0;
  int W = 4;
  double osf = 2.0;
  int ortho = 1;
  float scale = 1.f;
  float gsign = 1.f;
  KBPoly kb{};
  double beta = 0.0;
  // options
  int tile = 16;
  int coils_per_item = 4;
  int interp_mode = 0;
  int spread_kernel = 1;   // 1: block-per-tile kernels (2D tile 16, 3D tile 8) where they apply (3D default)
  int grid_mask = 1;       // fused FFT mode: the spread stores only cell pairs inside some support
  int col_interp = 0;      // fused 2D mode: forward column pass and interp in one kernel (option key 8)
  int grid_blk = 1;        // fused 2D mode: the forward grid in 2 x 8 cell blocks (option key 9)
  int tap_table = 1;       // 2D: spread and interp read the per-sample tap table (option key 10)
  DevBuf strip_start;      // (B * nstrips + 1) per-frame lists of the samples starting in each column strip
  DevBuf strip_entries;    // (B * K) sample indices
  int nstrips = 0;
  DevBuf touch;            // (B, twords) bitmaps of the cells inside some sample's support
  long long twords = 0;
  DevBuf grid_adj;         // fused mode with the mask: the spread's own grid, zero outside the supports
  bool adj_zero = false;   // grid_adj holds zeros outside the current supports
  int adj_nb = 0;          // ... for this batch (the frame of slot be depends on it)
  int chunk = 128;     // samples per spread work item (heavy tiles are split)
  // state
  bool have_points = false;
  bool have_maps = false;
  DevBuf gx;          // (B, nd, K) float
  DevBuf tapw;        // 2D: (B, K, 2) float4, the signed kernel weights of each sample's 4 nodes per dim
  DevBuf tapb;        // 2D: (B, K) int2, each sample's first node floor(x) - 1 per dim
  DevBuf entries;     // (n_entries) int32 sample index, sorted by (frame, tile)
  DevBuf tile_start;  // (B * ntiles + 1) int32
  DevBuf items;      // spread work items int4 (key, chunk, partial slot or -1, chunks of key), heaviest first
  DevBuf multi;      // int4 (key, chunks, first partial slot, 0) for tiles split into several chunks
  DevBuf partials;   // chunk partial tiles (rep, slot, C, T^nd) float2
  int n_items = 0, n_multi = 0, n_slots = 0;
  DevBuf empty_keys; // (frame, tile) keys with no sample: zero-filled by a store-only kernel
  DevBuf seg_order;  // 3D interp: (B, nseg) segments of IL_SEG consecutive samples in Morton order
  long long nseg = 0;
  int n_empty = 0;
  int64_t n_entries = 0;
  int64_t touched = 0;
  int ntile_d[3] = {1, 1, 1};
  int ntiles = 1;
  DevBuf maps;        // (C, *S) float2
  DevBuf invdeap;     // concatenated per-dim 1/Phi, S[0] + S[1] (+ S[2]) floats
  DevBuf wfwd, wadj;  // (B, K) float
  bool has_wfwd = false, has_wadj = false;
  DevBuf grid;        // (nb, C, *G) float2
  cufftHandle fft = 0;
  int fft_batch = 0;
  int fft_mode = 0;   // 0 cuFFT dense transform + pad/crop kernels, 1 fused zero-pruned passes (fft.cu)
  DevBuf band;        // fused mode: (nb, C, S0, G1) float2 row-transformed band
                      //             3D: (nb, C, S0, S1, G2) after the z pass
  DevBuf band2;       // fused mode, 3D: (nb, C, S0, G1, G2) after the y pass
  DevBuf tw0, tw1, tw2;   // fused mode: twiddle tables of G0, G1 (and G2)
  const float2* tw0p = nullptr;
  const float2* tw1p = nullptr;
  const float2* tw2p = nullptr;
  DevBuf rowfac;      // fused mode: signed deapodisation of each image row (S0, or S0*S1 in 3D)
  const double* skip = nullptr;   // device flag: operator kernels return when it is non-zero
  int il = 0;         // 1: forward interp on a coil-interleaved grid (3D: a copy of the grid; 2D fused mode:
                      // the forward column pass writes the grid itself in coil quads (cell, 4 coils))
  DevBuf grid_il;     // (nb, gtot, C) float2, written by the transpose at the start of the interp stage
  DevBuf psf;         // Toeplitz transfer functions (B, G0, G1) float (mrb_plan_set_toeplitz)
  DevBuf ones;        // 2D: S0 signs (-1)^(r + G0/2 - S0/2), then S1 ones: the row passes without deapodisation
  bool have_psf = false;
  DevBuf tmp;         // scratch for set_points

  int64_t gtot() const {
    int64_t t = 1;
    for (int d = 0; d < nd; ++d) t *= G[d];
    return t;
  }
  int64_t stot() const {
    int64_t t = 1;
    for (int d = 0; d < nd; ++d) t *= S[d];
    return t;
  }
};

namespace {

struct Geo {
  int nd;
  int S[3];
  int G[3];
  float Gf[3];
  float gmax[3];
  int off[3];        // G/2 - S//2
  int C;
  int B;
  long long K;
  long long gtot;
  long long stot;
  const double* skip;   // when non-null and non-zero the operator kernels return at once
};

Geo make_geo(const mrb_plan* p) {
  Geo g{};
  g.nd = p->nd;
  for (int d = 0; d < 3; ++d) {
    g.S[d] = p->S[d];
    g.G[d] = p->G[d];
    g.Gf[d] = (float)p->G[d];
    g.gmax[d] = (float)((double)p->G[d] - 1e-6);
    g.off[d] = p->G[d] / 2 - p->S[d] / 2;
  }
  g.C = p->C;
  g.B = p->B;
  g.K = p->K;
  g.gtot = p->gtot();
  g.stot = p->stot();
  g.skip = p->skip;
  return g;
}

__device__ __forceinline__ int frame_of(int be, int nb, int B) {
  if (B == 1) return 0;
  return be / (nb / B);
}

// ---------------------------------------------------------------------------
// set-up kernels
// ---------------------------------------------------------------------------
__global__ void coords_kernel(const float* __restrict__ traj, float* __restrict__ gx, Geo g) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.B * g.nd * g.K;
  if (i >= n) return;
  int d = (int)((i / g.K) % g.nd);
  gx[i] = mrb::ref_grid_coord(traj[i], g.Gf[d], g.gmax[d]);
}

// Per-sample tap table (2D, built with the coordinates): the first node
// floor(x) - 1 and the weights of the 4 nodes n along each dim, with the
// sample-side sign (-1)^n.  The trajectory is fixed across the operator calls
// of a solve, so the default spread and interp read 40 bytes per sample
// instead of evaluating 8 kernel polynomials (the interp once per coil pair).
// Same fx = x - floor(x), polynomials and sign as the inline evaluation: the
// same weights bit for bit.
__global__ void taps2_kernel(const float* __restrict__ gx, float4* __restrict__ tapw, int2* __restrict__ tapb,
                             Geo g, KBPoly kb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // b * K + k
  if (i >= (long long)g.B * g.K) return;
  const long long b = i / g.K, k = i - b * g.K;
  int base[2];
  float w[2][4];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const float x = gx[(b * 2 + d) * g.K + k];
    const int fb = (int)floorf(x);
    const float fx = x - (float)fb;
    base[d] = fb - 1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float wd = mrb::kb_tap(kb, q, fx);
      w[d][q] = ((base[d] + q) & 1) ? -wd : wd;
    }
  }
  tapw[2 * i] = make_float4(w[0][0], w[0][1], w[0][2], w[0][3]);
  tapw[2 * i + 1] = make_float4(w[1][0], w[1][1], w[1][2], w[1][3]);
  tapb[i] = make_int2(base[0], base[1]);
}

constexpr int MAX_TOUCH = 4;   // W = 4 nodes per dim touch at most 4 tiles

struct TileGeo {
  int T;
  int nt[3];
  int ntiles;
  int lo_off;   // W/2 - 1
  int hi_off;   // W/2
};

// distinct tiles touched along one dim by nodes base-lo_off .. base+hi_off
// (wrapped); up to 3 when a narrow partial last tile sits inside the span.
__device__ __forceinline__ int dim_tiles(int base, int G, int T, int nt, int lo_off, int hi_off, int* ts) {
  int n = 0;
  for (int v = base - lo_off; v <= base + hi_off; ++v) {
    int t = mrb::wrap_i(v, G) / T;
    bool seen = false;
    for (int j = 0; j < n; ++j) seen = seen || (ts[j] == t);
    if (!seen) ts[n++] = t;
  }
  return n;
}

__global__ void entry_count_kernel(const float* __restrict__ gx, int* __restrict__ cnt, Geo g, TileGeo tg) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.B * g.K;
  if (i >= n) return;
  int b = (int)(i / g.K);
  long long k = i - (long long)b * g.K;
  int c = 1;
  int ts[MAX_TOUCH];
  for (int d = 0; d < g.nd; ++d) {
    int base = (int)floorf(gx[((long long)b * g.nd + d) * g.K + k]);
    c *= dim_tiles(base, g.G[d], tg.T, tg.nt[d], tg.lo_off, tg.hi_off, ts);
  }
  cnt[i] = c;
}

__global__ void entry_fill_kernel(const float* __restrict__ gx, const int* __restrict__ offs,
                                  unsigned* __restrict__ keys, int* __restrict__ vals, Geo g, TileGeo tg) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.B * g.K;
  if (i >= n) return;
  int b = (int)(i / g.K);
  int k = (int)(i - (long long)b * g.K);
  int ts[3][MAX_TOUCH], nn[3];
  for (int d = 0; d < 3; ++d) { ts[d][0] = 0; nn[d] = 1; }
  for (int d = 0; d < g.nd; ++d) {
    int base = (int)floorf(gx[((long long)b * g.nd + d) * g.K + k]);
    nn[d] = dim_tiles(base, g.G[d], tg.T, tg.nt[d], tg.lo_off, tg.hi_off, ts[d]);
  }
  int o = offs[i];
  for (int a0 = 0; a0 < nn[0]; ++a0)
    for (int a1 = 0; a1 < nn[1]; ++a1)
      for (int a2 = 0; a2 < nn[2]; ++a2) {
        int t = ts[0][a0];
        if (g.nd > 1) t = t * tg.nt[1] + ts[1][a1];
        if (g.nd > 2) t = t * tg.nt[2] + ts[2][a2];
        keys[o] = (unsigned)(b * tg.ntiles + t);
        vals[o] = k;
        ++o;
      }
}

__global__ void tile_start_kernel(const unsigned* __restrict__ keys, long long n, int* __restrict__ start,
                                  int nkeys) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  int key = (int)keys[e];
  int prev = e ? (int)keys[e - 1] : -1;
  for (int t = prev + 1; t <= key; ++t) start[t] = (int)e;
  if (e == n - 1)
    for (int t = key + 1; t <= nkeys; ++t) start[t] = (int)n;
}

__global__ void fill_int_kernel(int* p, long long n, int v) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// touched-cell count (for roofline bookkeeping): marks cells in a bitmap
// frame b = blockIdx.y marks the cells of its samples' supports in its bitmap
__global__ void touch_kernel(const float* __restrict__ gx, unsigned* __restrict__ bits_all, long long nwords, Geo g,
                             int W) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= g.K) return;
  const int b = blockIdx.y;
  unsigned* bits = bits_all + (long long)b * nwords;
  int base[3] = {0, 0, 0};
  for (int d = 0; d < g.nd; ++d) base[d] = (int)floorf(gx[((long long)b * g.nd + d) * g.K + k]);
  int lo = W / 2 - 1;
  int n2 = g.nd > 2 ? W : 1, n1 = g.nd > 1 ? W : 1;
  for (int a = 0; a < W; ++a)
    for (int c = 0; c < n1; ++c)
      for (int e = 0; e < n2; ++e) {
        long long idx = mrb::wrap_i(base[0] - lo + a, g.G[0]);
        if (g.nd > 1) idx = idx * g.G[1] + mrb::wrap_i(base[1] - lo + c, g.G[1]);
        if (g.nd > 2) idx = idx * g.G[2] + mrb::wrap_i(base[2] - lo + e, g.G[2]);
        atomicOr(&bits[idx >> 5], 1u << (idx & 31));
      }
}

__global__ void popc_kernel(const unsigned* __restrict__ bits, long long nwords,
                            unsigned long long* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  if (i < nwords) c = __popc(bits[i]);
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

__global__ void dcf_weight_kernel(const float* __restrict__ dcf, float* __restrict__ w, long long n, int sq) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v = dcf[i];
  w[i] = sq ? sqrtf(fmaxf(v, 0.f)) : v;
}

// ---------------------------------------------------------------------------
// forward: SENSE * deapod * sign, zero-padded into the grid
// ---------------------------------------------------------------------------
// grid: x = pairs along the last dim, y = G0 (2D) or G1 (3D), z = volume
// (2D: be*C + c; 3D: (be*C + c)*G0 + n0).  No 64-bit division.
template <int ND>
__global__ void __launch_bounds__(128) pre_fft_kernel(const float2* __restrict__ x, const float2* __restrict__ maps,
                                                     const float* __restrict__ invdeap, float4* __restrict__ grid,
                                                     Geo g, int nb, int coil_images) {
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  const int Gl = g.G[ND - 1];
  const int pair = blockIdx.x * blockDim.x + threadIdx.x;
  if (pair >= (Gl >> 1)) return;
  int n[3];
  unsigned vol;
  if (ND == 2) {
    n[0] = blockIdx.y;
    vol = blockIdx.z;
  } else {
    n[1] = blockIdx.y;
    n[0] = blockIdx.z % g.G[0];
    vol = blockIdx.z / g.G[0];
  }
  const int c = vol % g.C;
  const int be = vol / g.C;
  const int nl = pair * 2;
  long long row = (ND == 2) ? (long long)n[0] : (long long)n[0] * g.G[1] + n[1];
  float4* out = grid + ((long long)vol * g.gtot + row * Gl + nl) / 2;
  float4 o4 = make_float4(0.f, 0.f, 0.f, 0.f);
  bool inside = true;
  int ii[3];
  float dap = 1.f;
  int dap_off = 0, parity = 0;
#pragma unroll
  for (int d = 0; d < ND - 1; ++d) {
    ii[d] = n[d] - g.off[d];
    inside = inside && (unsigned)ii[d] < (unsigned)g.S[d];
    if (inside) dap *= invdeap[dap_off + ii[d]];
    dap_off += g.S[d];
    parity += n[d];
  }
  if (inside) {
    long long base = ii[0];
    if (ND == 3) base = base * g.S[1] + ii[1];
    const int Sl = g.S[ND - 1];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int il = nl + h - g.off[ND - 1];
      if ((unsigned)il < (unsigned)Sl) {
        long long pix = base * Sl + il;
        float2 xv, mv;
        if (coil_images) {
          xv = x[((long long)be * g.C + c) * g.stot + pix];
          mv = make_float2(1.f, 0.f);
        } else {
          xv = x[(long long)be * g.stot + pix];
          mv = maps[(long long)c * g.stot + pix];
        }
        float sc = dap * invdeap[dap_off + il] * (((parity + nl + h) & 1) ? -1.f : 1.f);
        float re = (xv.x * mv.x - xv.y * mv.y) * sc;
        float im = (xv.x * mv.y + xv.y * mv.x) * sc;
        if (h == 0) { o4.x = re; o4.y = im; } else { o4.z = re; o4.w = im; }
      }
    }
  }
  *out = o4;
}

// ---------------------------------------------------------------------------
// adjoint: crop * deapod * sign * conj(maps), summed over coils
// grid: x = pixels along the last dim, y = S0 (2D) or S1 (3D), z = be (2D)
// or be*S0 + i0 (3D).
// ---------------------------------------------------------------------------
template <int ND>
__global__ void __launch_bounds__(128) post_ifft_kernel(const float2* __restrict__ grid, const float2* __restrict__ maps,
                                                       const float* __restrict__ invdeap, float2* __restrict__ x,
                                                       Geo g, int nb, float scale) {
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  const int Sl = g.S[ND - 1];
  const int il = blockIdx.x * blockDim.x + threadIdx.x;
  if (il >= Sl) return;
  int ii[3];
  int be;
  if (ND == 2) {
    ii[0] = blockIdx.y;
    be = blockIdx.z;
  } else {
    ii[1] = blockIdx.y;
    ii[0] = blockIdx.z % g.S[0];
    be = blockIdx.z / g.S[0];
  }
  ii[ND - 1] = il;
  float dap = scale;
  int dap_off = 0, parity = 0;
  long long cell = 0, pix = 0;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    dap *= invdeap[dap_off + ii[d]];
    dap_off += g.S[d];
    int n = ii[d] + g.off[d];
    parity += n;
    cell = cell * g.G[d] + n;
    pix = pix * g.S[d] + ii[d];
  }
  if (parity & 1) dap = -dap;
  float re = 0.f, im = 0.f;
  const float2* gp = grid + (long long)be * g.C * g.gtot + cell;
  for (int c = 0; c < g.C; ++c) {
    float2 v = gp[(long long)c * g.gtot];
    float2 m = maps[(long long)c * g.stot + pix];
    re += m.x * v.x + m.y * v.y;
    im += m.x * v.y - m.y * v.x;
  }
  x[(long long)be * g.stot + pix] = make_float2(re * dap, im * dap);
}

// ---------------------------------------------------------------------------
// forward interp: one thread per sample, all coils (W = 4)
// ---------------------------------------------------------------------------
struct InterpArgs {
  const float2* grid;
  const float* gx;
  const float* wfwd;   // (B, K) or null
  const int* order;    // (B, K) sample order or null (acquisition order)
  float2* y;
  int nb;
  float scale;
  float gsign;
  const int* seg;      // 3D interleaved interp: segment visiting order (B, nseg) or null
  long long nseg;
  int blk;             // 2D pair-parallel interp: the grid is in 2 x 8 cell blocks (fwd_cols_kernel<G0, true>)
  const float4* tapw;  // 2D pair-parallel interp: tap table (taps2_kernel) or null
  const int2* tapb;
};

template <int ND>
struct InterpGen {
  static constexpr int NT = 256, MINB = (ND == 2 ? 4 : 1);
  static constexpr const char* FAMILY = "interp";
  static __device__ __forceinline__ void run(const VBlock& vb, const InterpArgs& a, const Geo& g,
      const KBPoly& kb) {
    constexpr int W = 4;
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    long long kk = (long long)vb.x * blockDim.x + threadIdx.x;
    int be = vb.y;
    if (kk >= g.K) return;
    int b = frame_of(be, a.nb, g.B);
    long long k = a.order ? a.order[(long long)b * g.K + kk] : kk;
    float w[ND][W];
    int nidx[ND][W];
  #pragma unroll
    for (int d = 0; d < ND; ++d) {
      float x = a.gx[((long long)b * ND + d) * g.K + k];
      int base = (int)floorf(x);
      const float fx = x - (float)base;
  #pragma unroll
      for (int o = 0; o < W; ++o) {
        int n = base - (W / 2 - 1) + o;
        float wd = mrb::kb_tap(kb, o, fx);
        w[d][o] = (n & 1) ? -wd : wd;
        nidx[d][o] = mrb::wrap_i(n, g.G[d]);
      }
    }
    float s = a.scale * a.gsign;
    if (a.wfwd) s *= a.wfwd[(long long)b * g.K + k];
    const float2* gb = a.grid + (long long)be * g.C * g.gtot;
    float2* yo = a.y + (long long)be * g.C * g.K + k;
    if (ND == 2) {
      // row offsets shared by all coils
      long long roff[W];
  #pragma unroll
      for (int i0 = 0; i0 < W; ++i0) roff[i0] = (long long)nidx[0][i0] * g.G[1];
      // two coils per pass: 32 independent loads in flight per thread
      int c = 0;
      for (; c + 1 < g.C; c += 2) {
        const float2* g0 = gb + (long long)c * g.gtot;
        const float2* g1 = g0 + g.gtot;
        float2 v0[W][W], v1[W][W];
  #pragma unroll
        for (int i0 = 0; i0 < W; ++i0)
  #pragma unroll
          for (int i1 = 0; i1 < W; ++i1) {
            v0[i0][i1] = __ldg(g0 + roff[i0] + nidx[1][i1]);
            v1[i0][i1] = __ldg(g1 + roff[i0] + nidx[1][i1]);
          }
        float r0 = 0.f, m0 = 0.f, r1 = 0.f, m1 = 0.f;
  #pragma unroll
        for (int i0 = 0; i0 < W; ++i0) {
          float a0 = 0.f, b0 = 0.f, a1 = 0.f, b1 = 0.f;
  #pragma unroll
          for (int i1 = 0; i1 < W; ++i1) {
            a0 = fmaf(w[1][i1], v0[i0][i1].x, a0);
            b0 = fmaf(w[1][i1], v0[i0][i1].y, b0);
            a1 = fmaf(w[1][i1], v1[i0][i1].x, a1);
            b1 = fmaf(w[1][i1], v1[i0][i1].y, b1);
          }
          r0 = fmaf(w[0][i0], a0, r0);
          m0 = fmaf(w[0][i0], b0, m0);
          r1 = fmaf(w[0][i0], a1, r1);
          m1 = fmaf(w[0][i0], b1, m1);
        }
        yo[(long long)c * g.K] = make_float2(r0 * s, m0 * s);
        yo[(long long)(c + 1) * g.K] = make_float2(r1 * s, m1 * s);
      }
      for (; c < g.C; ++c) {
        const float2* g0 = gb + (long long)c * g.gtot;
        float r0 = 0.f, m0 = 0.f;
  #pragma unroll
        for (int i0 = 0; i0 < W; ++i0) {
          float a0 = 0.f, b0 = 0.f;
  #pragma unroll
          for (int i1 = 0; i1 < W; ++i1) {
            float2 v = __ldg(g0 + roff[i0] + nidx[1][i1]);
            a0 = fmaf(w[1][i1], v.x, a0);
            b0 = fmaf(w[1][i1], v.y, b0);
          }
          r0 = fmaf(w[0][i0], a0, r0);
          m0 = fmaf(w[0][i0], b0, m0);
        }
        yo[(long long)c * g.K] = make_float2(r0 * s, m0 * s);
      }
    } else {
      for (int c = 0; c < g.C; ++c) {
        const float2* gc = gb + (long long)c * g.gtot;
        float re = 0.f, im = 0.f;
  #pragma unroll
        for (int i0 = 0; i0 < W; ++i0) {
          float r1 = 0.f, im1 = 0.f;
  #pragma unroll
          for (int i1 = 0; i1 < W; ++i1) {
            const float2* row = gc + ((long long)nidx[0][i0] * g.G[1] + nidx[1][i1]) * g.G[ND - 1];
            float r2 = 0.f, i2 = 0.f;
  #pragma unroll
            for (int i2x = 0; i2x < W; ++i2x) {
              float2 v = __ldg(row + nidx[ND - 1][i2x]);
              r2 = fmaf(w[ND - 1][i2x], v.x, r2);
              i2 = fmaf(w[ND - 1][i2x], v.y, i2);
            }
            r1 = fmaf(w[1][i1], r2, r1);
            im1 = fmaf(w[1][i1], i2, im1);
          }
          re = fmaf(w[0][i0], r1, re);
          im = fmaf(w[0][i0], im1, im);
        }
        yo[(long long)c * g.K] = make_float2(re * s, im * s);
      }
    }
  }
};
template <int ND>
__global__ void __launch_bounds__(256) interp_kernel(InterpArgs a, Geo g, KBPoly kb) {
  InterpGen<ND>::run(hw_block(), a, g, kb);
}

// 2D forward interp, one thread per (sample, coil pair): the 16 taps of both
// coils (32 independent 8-byte loads) in flight at once, and a grid of
// C/2 times more threads than samples, so the latency of the scattered reads
// is hidden by parallelism rather than by a per-thread loop over the coils.
// Blocks cover 256 consecutive samples of one coil pair (coalesced sample
// reads and result writes).  Same summation order as interp_kernel<2>.
struct Interp2p {
  static constexpr int NT = 256, MINB = 4;
  static constexpr const char* FAMILY = "interp";
  static __device__ __forceinline__ void run(const VBlock& vb, const InterpArgs& a, const Geo& g,
      const KBPoly& kb) {
    constexpr int W = 4;
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    const int kblocks = (int)((g.K + 255) / 256);
    const int pr = vb.x / kblocks;
    const long long k = (long long)(vb.x - pr * kblocks) * 256 + threadIdx.x;
    const int be = vb.y;
    if (k >= g.K) return;
    const int b = frame_of(be, a.nb, g.B);
    float w[2][W];
    int nidx[2][W];
    if (a.tapw) {
      // the tap table: first node floor(x) - 1 >= -1 and nodes up to G + 1, so
      // one conditional add or subtract wraps them
      const long long i = (long long)b * g.K + k;
      const float4 w0 = __ldg(a.tapw + 2 * i), w1 = __ldg(a.tapw + 2 * i + 1);
      const int2 bb = __ldg(a.tapb + i);
      w[0][0] = w0.x; w[0][1] = w0.y; w[0][2] = w0.z; w[0][3] = w0.w;
      w[1][0] = w1.x; w[1][1] = w1.y; w[1][2] = w1.z; w[1][3] = w1.w;
  #pragma unroll
      for (int o = 0; o < W; ++o) {
        const int n0 = bb.x + o, n1 = bb.y + o;
        nidx[0][o] = n0 < 0 ? n0 + g.G[0] : n0 >= g.G[0] ? n0 - g.G[0] : n0;
        nidx[1][o] = n1 < 0 ? n1 + g.G[1] : n1 >= g.G[1] ? n1 - g.G[1] : n1;
      }
    } else {
  #pragma unroll
      for (int d = 0; d < 2; ++d) {
        const float x = a.gx[((long long)b * 2 + d) * g.K + k];
        const int base = (int)floorf(x);
        const float fx = x - (float)base;
  #pragma unroll
        for (int o = 0; o < W; ++o) {
          const int n = base - (W / 2 - 1) + o;
          const float wd = mrb::kb_tap(kb, o, fx);
          w[d][o] = (n & 1) ? -wd : wd;
          nidx[d][o] = mrb::wrap_i(n, g.G[d]);
        }
      }
    }
    // offsets of the tap rows and columns: row-major, or 2 x 8 cell blocks
    int roff[W], coff[W];
  #pragma unroll
    for (int o = 0; o < W; ++o) {
      const int n0 = nidx[0][o], n1 = nidx[1][o];
      roff[o] = a.blk ? (n0 >> 1) * (2 * g.G[1]) + (n0 & 1) * 8 : n0 * g.G[1];
      coff[o] = a.blk ? ((n1 >> 3) << 4) + (n1 & 7) : n1;
    }
    float s = a.scale * a.gsign;
    if (a.wfwd) s *= a.wfwd[(long long)b * g.K + k];
    const int c = 2 * pr;
    const bool two = c + 1 < g.C;
    const float2* g0 = a.grid + ((long long)be * g.C + c) * g.gtot;
    const float2* g1 = two ? g0 + g.gtot : g0;
    float2 v0[W][W], v1[W][W];
  #pragma unroll
    for (int i0 = 0; i0 < W; ++i0) {
  #pragma unroll
      for (int i1 = 0; i1 < W; ++i1) {
        v0[i0][i1] = __ldg(g0 + roff[i0] + coff[i1]);
        v1[i0][i1] = two ? __ldg(g1 + roff[i0] + coff[i1]) : make_float2(0.f, 0.f);
      }
    }
    float r0 = 0.f, m0 = 0.f, r1 = 0.f, m1 = 0.f;
  #pragma unroll
    for (int i0 = 0; i0 < W; ++i0) {
      float a0 = 0.f, b0 = 0.f, a1 = 0.f, b1 = 0.f;
  #pragma unroll
      for (int i1 = 0; i1 < W; ++i1) {
        a0 = fmaf(w[1][i1], v0[i0][i1].x, a0);
        b0 = fmaf(w[1][i1], v0[i0][i1].y, b0);
        a1 = fmaf(w[1][i1], v1[i0][i1].x, a1);
        b1 = fmaf(w[1][i1], v1[i0][i1].y, b1);
      }
      r0 = fmaf(w[0][i0], a0, r0);
      m0 = fmaf(w[0][i0], b0, m0);
      r1 = fmaf(w[0][i0], a1, r1);
      m1 = fmaf(w[0][i0], b1, m1);
    }
    float2* yo = a.y + ((long long)be * g.C + c) * g.K + k;
    yo[0] = make_float2(r0 * s, m0 * s);
    if (two) yo[g.K] = make_float2(r1 * s, m1 * s);
  }
};
__global__ void __launch_bounds__(256) interp2p_kernel(InterpArgs a, Geo g, KBPoly kb) {
  Interp2p::run(hw_block(), a, g, kb);
}

// 2D forward interp on the coil-quad grid (be, coil quad, cell, coil in quad)
// that the coil-grouped forward column pass writes.  One thread per (sample,
// coil pair) with the P pairs of a sample on adjacent threads and 128-bit
// loads: a 4-cell tap row of a quad is one 128-byte run (at most two lines),
// where on the coil-planar grid every 4-cell tap row of a coil is a 32-byte
// piece that straddles two sectors three times in four.  A block covers
// S = 256 / P consecutive samples; the results go through shared memory so
// that each coil's samples are stored as one run.  Taps, weights and summation
// order are those of interp2p_kernel: identical samples.  C % 4 == 0.
struct Interp2Quad {
  static constexpr int NT = 256, MINB = 4;
  static constexpr const char* FAMILY = "interp";
  static __device__ __forceinline__ void run(const VBlock& vb, const InterpArgs& a, const Geo& g,
      const KBPoly& kb) {
    constexpr int W = 4;
    __shared__ float2 ys[512];   // [coil][sample]: C * S <= 2 * P * S <= 512
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    const int C = g.C;
    const int P = (C + 1) >> 1;
    const int S = 256 / P;
    const long long k0 = (long long)vb.x * S;
    const int be = vb.y;
    const int b = frame_of(be, a.nb, g.B);
    const int ks = threadIdx.x / P, pr = threadIdx.x - ks * P;
    const long long k = k0 + ks;
    if (ks < S && k < g.K) {
      float w[2][W];
      int nidx[2][W];
  #pragma unroll
      for (int d = 0; d < 2; ++d) {
        const float x = a.gx[((long long)b * 2 + d) * g.K + k];
        const int base = (int)floorf(x);
        const float fx = x - (float)base;
  #pragma unroll
        for (int o = 0; o < W; ++o) {
          const int n = base - (W / 2 - 1) + o;
          const float wd = mrb::kb_tap(kb, o, fx);
          w[d][o] = (n & 1) ? -wd : wd;
          nidx[d][o] = mrb::wrap_i(n, g.G[d]);
        }
      }
      float s = a.scale * a.gsign;
      if (a.wfwd) s *= a.wfwd[(long long)b * g.K + k];
      const int c = 2 * pr;
      const bool two = true;   // C % 4 == 0: every pair is whole
      const float2* gb = a.grid + ((long long)be * C + (c & ~3)) * g.gtot + (c & 3);
      float4 v[W][W];
  #pragma unroll
      for (int i0 = 0; i0 < W; ++i0) {
        const long long roff = (long long)nidx[0][i0] * g.G[1];
  #pragma unroll
        for (int i1 = 0; i1 < W; ++i1)
          v[i0][i1] = __ldg(reinterpret_cast<const float4*>(gb + (roff + nidx[1][i1]) * 4));
      }
      float r0 = 0.f, m0 = 0.f, r1 = 0.f, m1 = 0.f;
  #pragma unroll
      for (int i0 = 0; i0 < W; ++i0) {
        float a0 = 0.f, b0 = 0.f, a1 = 0.f, b1 = 0.f;
  #pragma unroll
        for (int i1 = 0; i1 < W; ++i1) {
          a0 = fmaf(w[1][i1], v[i0][i1].x, a0);
          b0 = fmaf(w[1][i1], v[i0][i1].y, b0);
          a1 = fmaf(w[1][i1], v[i0][i1].z, a1);
          b1 = fmaf(w[1][i1], v[i0][i1].w, b1);
        }
        r0 = fmaf(w[0][i0], a0, r0);
        m0 = fmaf(w[0][i0], b0, m0);
        r1 = fmaf(w[0][i0], a1, r1);
        m1 = fmaf(w[0][i0], b1, m1);
      }
      ys[c * S + ks] = make_float2(r0 * s, m0 * s);
      if (two) ys[(c + 1) * S + ks] = make_float2(r1 * s, m1 * s);
    }
    __syncthreads();
    const int ns = (int)min((long long)S, g.K - k0);
    float2* yo = a.y + (long long)be * C * g.K + k0;
    for (int e = threadIdx.x; e < C * S; e += blockDim.x) {
      const int c = e / S, j = e - c * S;
      if (j < ns) yo[(long long)c * g.K + j] = ys[c * S + j];
    }
  }
};
__global__ void __launch_bounds__(256) interp2_il_kernel(InterpArgs a, Geo g, KBPoly kb) {
  Interp2Quad::run(hw_block(), a, g, kb);
}

// ---------------------------------------------------------------------------
// 3D forward interp on a coil-interleaved grid.  The dense cuFFT leaves the
// oversampled grid planar, (be, coil, cell); a 64-tap gather from it touches
// 64 x C scattered 8-byte values per sample, a quarter of every 32-byte sector.
// The interp stage first rewrites the grid as (be, cell, coil) with a
// shared-memory tiled transpose (one read and one write of the grid, both
// coalesced), then gathers with one thread per (sample, coil pair): the
// threads of a sample read the C coils of a cell as one contiguous run
// (C = 16: one 128-byte line per tap), 128-bit loads when C is even.
// ---------------------------------------------------------------------------
constexpr int TR_CELLS = 64;    // cells per transpose block
constexpr int IL_SEG = 8;       // samples per interp visiting segment

// 3D visiting-order key of a segment: frame, then the Morton code of the
// 8-cell tile holding its middle sample
__global__ void seg_key_kernel(const float* __restrict__ gx, unsigned long long* __restrict__ keys,
                               int* __restrict__ vals, Geo g, long long nseg, int bits) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)g.B * nseg) return;
  const int b = (int)(i / nseg);
  const long long s = i - (long long)b * nseg;
  const long long k = min(s * IL_SEG + IL_SEG / 2, g.K - 1);
  unsigned long long m = 0;
  for (int d = 0; d < 3; ++d) {
    int c = (int)floorf(gx[((long long)b * 3 + d) * g.K + k]);
    c = min(max(c, 0), g.G[d] - 1) >> 3;
    for (int q = 0; q < bits; ++q) m |= (unsigned long long)((c >> q) & 1) << (3 * q + (2 - d));
  }
  keys[i] = ((unsigned long long)b << (3 * bits)) | m;
  vals[i] = (int)s;
}
constexpr int TR_COILS = 16;    // coils per shared tile pass

__global__ void __launch_bounds__(256) coil_interleave_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                              long long gtot, int C, const double* skip) {
  if (skip != nullptr && *skip != 0.0) return;   // solve already finished
  __shared__ float2 tile[TR_COILS][TR_CELLS + 1];
  const long long cell0 = (long long)blockIdx.x * TR_CELLS;
  const long long be = blockIdx.y;
  const float2* src = in + be * C * gtot;
  float2* dst = out + be * C * gtot;
  const int ncell = (int)min((long long)TR_CELLS, gtot - cell0);
  for (int c0 = 0; c0 < C; c0 += TR_COILS) {
    const int cc = min(TR_COILS, C - c0);
    for (int e = threadIdx.x; e < cc * TR_CELLS; e += blockDim.x) {
      const int c = e / TR_CELLS, l = e - c * TR_CELLS;
      if (l < ncell) tile[c][l] = src[(long long)(c0 + c) * gtot + cell0 + l];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < cc * TR_CELLS; e += blockDim.x) {
      const int l = e / cc, c = e - l * cc;
      if (l < ncell) dst[(cell0 + l) * C + c0 + c] = tile[c][l];
    }
    __syncthreads();
  }
}

template <bool V4>
__global__ void __launch_bounds__(256, 4) interp3_il_kernel(InterpArgs a, Geo g, KBPoly kb) {
  constexpr int W = 4;
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  const int P = (g.C + 1) >> 1;   // coil pairs
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int be = blockIdx.y;
  const int b = frame_of(be, a.nb, g.B);
  long long k = t / P;
  const int pr = (int)(t - k * P);
  if (a.seg) {
    // segments of IL_SEG consecutive samples (whole 32-byte pieces of every
    // coil row of y) visited in the Morton order of their middle sample's tile
    const long long ss = k / IL_SEG;
    if (ss >= a.nseg) return;
    k = (long long)a.seg[(long long)b * a.nseg + ss] * IL_SEG + (k - ss * IL_SEG);
  }
  if (k >= g.K) return;
  float w[3][W];
  int nidx[3][W];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float x = a.gx[((long long)b * 3 + d) * g.K + k];
    const int base = (int)floorf(x);
    const float fx = x - (float)base;
#pragma unroll
    for (int o = 0; o < W; ++o) {
      const int n = base - (W / 2 - 1) + o;
      const float wd = mrb::kb_tap(kb, o, fx);
      w[d][o] = (n & 1) ? -wd : wd;
      nidx[d][o] = mrb::wrap_i(n, g.G[d]);
    }
  }
  float s = a.scale * a.gsign;
  if (a.wfwd) s *= a.wfwd[(long long)b * g.K + k];
  const int c0 = 2 * pr;
  const bool two = c0 + 1 < g.C;
  const float2* gb = a.grid + (long long)be * g.C * g.gtot + c0;
  // 32-bit element offsets within a frame (gtot * C < 2^31, checked on the host)
  int off2[W];
#pragma unroll
  for (int i2 = 0; i2 < W; ++i2) off2[i2] = nidx[2][i2] * g.C;
  float re0 = 0.f, im0 = 0.f, re1 = 0.f, im1 = 0.f;
#pragma unroll
  for (int i0 = 0; i0 < W; ++i0) {
    float4 v[W][W];
#pragma unroll
    for (int i1 = 0; i1 < W; ++i1) {
      const int row = (nidx[0][i0] * g.G[1] + nidx[1][i1]) * g.G[2] * g.C;
#pragma unroll
      for (int i2 = 0; i2 < W; ++i2) {
        const float2* q = gb + (row + off2[i2]);
        if (V4) {
          v[i1][i2] = __ldg(reinterpret_cast<const float4*>(q));
        } else {
          const float2 u0 = __ldg(q);
          const float2 u1 = two ? __ldg(q + 1) : make_float2(0.f, 0.f);
          v[i1][i2] = make_float4(u0.x, u0.y, u1.x, u1.y);
        }
      }
    }
    float r0 = 0.f, m0 = 0.f, r1 = 0.f, m1 = 0.f;
#pragma unroll
    for (int i1 = 0; i1 < W; ++i1) {
      float a0 = 0.f, b0 = 0.f, a1 = 0.f, b1 = 0.f;
#pragma unroll
      for (int i2 = 0; i2 < W; ++i2) {
        a0 = fmaf(w[2][i2], v[i1][i2].x, a0);
        b0 = fmaf(w[2][i2], v[i1][i2].y, b0);
        a1 = fmaf(w[2][i2], v[i1][i2].z, a1);
        b1 = fmaf(w[2][i2], v[i1][i2].w, b1);
      }
      r0 = fmaf(w[1][i1], a0, r0);
      m0 = fmaf(w[1][i1], b0, m0);
      r1 = fmaf(w[1][i1], a1, r1);
      m1 = fmaf(w[1][i1], b1, m1);
    }
    re0 = fmaf(w[0][i0], r0, re0);
    im0 = fmaf(w[0][i0], m0, im0);
    re1 = fmaf(w[0][i0], r1, re1);
    im1 = fmaf(w[0][i0], m1, im1);
  }
  float2* yo = a.y + ((long long)be * g.C + c0) * g.K + k;
  yo[0] = make_float2(re0 * s, im0 * s);
  if (two) yo[g.K] = make_float2(re1 * s, im1 * s);
}

// ---------------------------------------------------------------------------
// adjoint spread (W = 4).  One warp owns one output tile (T x T cells in 2D,
// T^3 in 3D) for a group of coils and is the only writer of those cells:
// it walks the tile's sample list (samples whose 4-node support meets the
// tile, in sample order), accumulates into shared memory without atomics and
// writes every cell of the tile once (zeros included).  Deterministic.
// Samples are staged 32 at a time: lane i loads sample i's coordinates,
// kernel weights and coil values (independent loads, one latency per batch),
// then the warp applies them one by one from shared memory, lanes = taps x
// coil lanes, with a __syncwarp between samples to order the read-modify-
// writes of cells shared by consecutive samples.  Empty tiles only store zeros.
// ---------------------------------------------------------------------------
struct SpreadArgs {
  const float2* y;
  const float* gx;
  const float* wadj;
  const int* entries;
  const int* tile_start;
  const int4* items;   // (key, chunk, partial slot or -1, chunks), heaviest first
  int n_items;
  int chunk;
  float2* partials;    // (rep, slot, C, T^nd) partial tiles of split keys
  int n_slots;
  float2* grid;
  int nb;
  int cpi;     // coils per work item
  int ngroups; // ceil(C / cpi)
  float gsign;
  const unsigned* touch;   // per-frame touched-cell bitmaps: grid cells outside them are not stored
  long long twords;
  const float4* tapw;      // 2D tap table (taps2_kernel) or null: the weights are evaluated inline
  const int2* tapb;
};

// a tile's cell pair (cell, cell + 1; cell even) is stored: no bitmap is in use, or
// the aligned group of 4 cells around it (one 32-byte sector of a coil row, both
// pairs in the same tile) holds a touched cell.  The pair's cells that no support
// reaches hold zeros, so the sector is written whole (no partial-sector write
// for the memory to merge) and the grid stays the same.
__device__ __forceinline__ bool pair_touched(const SpreadArgs& a, int b, long long cell) {
  if (a.touch == nullptr) return true;
  return (__ldg(a.touch + (long long)b * a.twords + (cell >> 5)) >> (cell & 28)) & 15u;
}

constexpr int SPREAD_WARPS = 4;
constexpr int SPREAD_BATCH = 32;

// first grid node of a staged sample along each dim (2D: two ints, 3D: three in an int4)
__device__ __forceinline__ int2 stage_base(const int* b, int2*) { return make_int2(b[0], b[1]); }
__device__ __forceinline__ int4 stage_base(const int* b, int4*) { return make_int4(b[0], b[1], b[2], 0); }
__device__ __forceinline__ int base_z(const int2&) { return 0; }
__device__ __forceinline__ int base_z(const int4& b) { return b.z; }

template <int ND, int T>
struct SpreadSmem {
  static constexpr int CELLS = ND == 2 ? T * T : T * T * T;
  static constexpr int NW = 4 * ND;                               // staged weights per sample
  static constexpr int NWP = NW + 1;                              // their stride (odd: no bank conflicts)
  static constexpr int NTAP = ND == 2 ? 16 : 64;
  // samples staged per batch: 2D tiles hold ~15 samples a frame in radial
  // acquisitions, and the smaller staging area lets 6 instead of 5 blocks of
  // 4 coils per item share an SM
  static constexpr int BATCH = ND == 2 ? 16 : SPREAD_BATCH;
  using Base = typename std::conditional<ND == 2, int2, int4>::type;
  // the shared tile is coil-interleaved, [cell][coil] with an even coil stride, so
  // one lane updates a pair of coils with one 128-bit read-modify-write
  __host__ __device__ static int cstride(int cpi) { return (cpi + 1) & ~1; }
  __host__ __device__ static size_t warp_bytes(int cpi) {
    return (size_t)cstride(cpi) * CELLS * sizeof(float2) + BATCH * (sizeof(Base) + NWP * sizeof(float)) +
           (size_t)BATCH * cstride(cpi) * sizeof(float2);
  }
};

template <int ND, int T>
struct SpreadWarp {
  static constexpr int NT = SPREAD_WARPS * 32, MINB = 6;
  static constexpr const char* FAMILY = "spread";
  static __device__ __forceinline__ void run(const VBlock& vb, const SpreadArgs& a, const Geo& g,
      const TileGeo& tg, const KBPoly& kb) {
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    using SM = SpreadSmem<ND, T>;
    constexpr int CELLS = SM::CELLS;
    constexpr int NW = SM::NWP;   // stride of the staged weights
    constexpr int NTAP = SM::NTAP;
    extern __shared__ float4 smem4[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    long long item = (long long)vb.x * SPREAD_WARPS + warp;
    const long long reps = g.B == 1 ? a.nb : a.nb / g.B;
    const long long nitems = reps * a.n_items * a.ngroups;
    if (item >= nitems) return;
    // work items run heaviest (frame, tile) first; every frame of a B_eff batch
    // that shares the trajectory frame repeats the same item list
    const int grp = (int)(item % a.ngroups);
    const long long oi = item / a.ngroups;
    const int4 it = a.items[oi % a.n_items];
    const int rep = (int)(oi / a.n_items);
    const int okey = it.x;
    const int b = okey / tg.ntiles;
    const int tile = okey - b * tg.ntiles;
    const int be = (g.B == 1) ? rep : b * (a.nb / g.B) + rep;
    const int c0 = grp * a.cpi;
    const int nc = min(a.cpi, g.C - c0);
    int o[3];
    if (ND == 2) {
      o[0] = (tile / tg.nt[1]) * T;
      o[1] = (tile % tg.nt[1]) * T;
      o[2] = 0;
    } else {
      o[2] = (tile % tg.nt[2]) * T;
      o[1] = ((tile / tg.nt[2]) % tg.nt[1]) * T;
      o[0] = (tile / (tg.nt[2] * tg.nt[1])) * T;
    }
    const int key = okey;
    const int k0 = a.tile_start[key], k1 = a.tile_start[key + 1];
    const int e0 = min(k1, k0 + it.y * a.chunk), e1 = min(k1, e0 + a.chunk);
    float2* gout = a.grid + ((long long)be * g.C + c0) * g.gtot;
    const int Gl = g.G[ND - 1];
    // split keys write their partial tile (unpadded T^nd per coil) to a slot
    constexpr int TN = ND == 2 ? T * T : T * T * T;
    float2* pout = it.z >= 0 ? a.partials + (((long long)rep * a.n_slots + it.z) * g.C + c0) * TN : nullptr;

    // cells of the tile as float4 pairs along the last dim
    constexpr int PAIRS = (ND == 2 ? T * T : T * T * T) / 2;
    auto cell_of_pair = [&](int r, int* n) -> long long {
      int l = (r % (T / 2)) * 2;
      int rr = r / (T / 2);
      if (ND == 2) {
        n[0] = o[0] + rr;
        n[1] = o[1] + l;
        return (long long)n[0] * Gl + n[1];
      } else {
        n[0] = o[0] + rr / T;
        n[1] = o[1] + rr % T;
        n[2] = o[2] + l;
        return ((long long)n[0] * g.G[1] + n[1]) * Gl + n[2];
      }
    };
    auto in_grid = [&](const int* n) {
      bool ok = n[0] < g.G[0];
      if (ND >= 2) ok = ok && n[1] < g.G[1];
      if (ND == 3) ok = ok && n[2] < g.G[2];
      return ok;
    };

    if (e0 == e1 && !pout) {   // no sample touches this tile: zeros
      if (a.touch) return;     // its cells are outside every support and never read
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int i = lane; i < nc * PAIRS; i += 32) {
        int cl = i / PAIRS, r = i - cl * PAIRS;
        int n[3];
        long long cell = cell_of_pair(r, n);
        if (in_grid(n)) *reinterpret_cast<float4*>(gout + (long long)cl * g.gtot + cell) = z4;
      }
      return;
    }

    const int cps = SM::cstride(a.cpi);   // coils per shared cell (even)
    const int npair = cps >> 1;
    char* wbase = reinterpret_cast<char*>(smem4) + (size_t)warp * SM::warp_bytes(a.cpi);
    float2* acc = reinterpret_cast<float2*>(wbase);
    constexpr int SB = SM::BATCH;
    using Base = typename SM::Base;
    Base* sb = reinterpret_cast<Base*>(wbase + (size_t)cps * CELLS * sizeof(float2));
    float* sw = reinterpret_cast<float*>(sb + SB);
    float2* sy = reinterpret_cast<float2*>(sw + SB * NW);

    {
      float4* acc4 = reinterpret_cast<float4*>(acc);
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int i = lane; i < cps * CELLS / 2; i += 32) acc4[i] = z4;
    }
    __syncwarp();

    const float* gxp = a.gx + (long long)b * ND * g.K;
    const float2* yb = a.y + ((long long)be * g.C + c0) * g.K;
    const int ntask = NTAP * npair;
    // the next batch's sample index, coordinates, weight and first coil values
    // are loaded into registers while the warp works on the current batch
    constexpr int PF = 4;
    // 2D with the tap table: the sample's weights and first nodes instead of its coordinates
    const bool tab = ND == 2 && a.tapw != nullptr;
    int pk = 0;
    float px[ND], pwa = 1.f;
    float4 pw0 = make_float4(0.f, 0.f, 0.f, 0.f), pw1 = pw0;
    int2 pb = make_int2(0, 0);
    float2 py[PF];
    auto fetch = [&](int e, int nbat) {
      if (lane < nbat) {
        pk = a.entries[e + lane];
        if (tab) {
          const long long i = (long long)b * g.K + pk;
          pw0 = __ldg(a.tapw + 2 * i);
          pw1 = __ldg(a.tapw + 2 * i + 1);
          pb = __ldg(a.tapb + i);
        } else {
  #pragma unroll
          for (int d = 0; d < ND; ++d) px[d] = gxp[(long long)d * g.K + pk];
        }
        if (a.wadj) pwa = a.wadj[(long long)b * g.K + pk];
  #pragma unroll
        for (int cl = 0; cl < PF; ++cl) py[cl] = cl < nc ? yb[(long long)cl * g.K + pk] : make_float2(0.f, 0.f);
      }
    };
    if (e0 < e1) fetch(e0, min(SB, e1 - e0));
    for (int e = e0; e < e1; e += SB) {
      const int nbat = min(SB, e1 - e);
      if (lane < nbat) {
        const int k = pk;
        float ws = a.gsign;
        if (a.wadj) ws *= pwa;
        int base[3] = {0, 0, 0};
        if (tab) {
          // the table's signed weights; dim 0 times the sample's scale, as below
          const float t0[4] = {pw0.x, pw0.y, pw0.z, pw0.w}, t1[4] = {pw1.x, pw1.y, pw1.z, pw1.w};
  #pragma unroll
          for (int q = 0; q < 4; ++q) {
            sw[lane * NW + q] = t0[q] * ws;
            sw[lane * NW + 4 + q] = t1[q];
          }
          base[0] = pb.x;
          base[1] = pb.y;
        } else {
  #pragma unroll
          for (int d = 0; d < ND; ++d) {
            const float x = px[d];
            base[d] = (int)floorf(x) - 1;
            const float fx = x - (float)(base[d] + 1);
  #pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int n = base[d] + q;
              float w = mrb::kb_tap(kb, q, fx);
              if (n & 1) w = -w;
              if (d == 0) w *= ws;
              sw[lane * NW + d * 4 + q] = w;
            }
          }
        }
        // tile-relative first node r = base - o, taken modulo G into [-3, G - 4]:
        // tap t of the sample then sits at local index r + t (+ G when negative),
        // without the per-tap wrap into the grid
  #pragma unroll
        for (int d = 0; d < ND; ++d) {
          int r = base[d] - o[d];
          r += r < -3 ? g.G[d] : 0;
          r -= r > g.G[d] - 4 ? g.G[d] : 0;
          base[d] = r;
        }
        sb[lane] = stage_base(base, (Base*)nullptr);
  #pragma unroll
        for (int cl = 0; cl < PF; ++cl)
          if (cl < cps) sy[lane * cps + cl] = py[cl];
        for (int cl = PF; cl < cps; ++cl)
          sy[lane * cps + cl] = cl < nc ? yb[(long long)cl * g.K + k] : make_float2(0.f, 0.f);
      }
      __syncwarp();
      if (e + SB < e1) fetch(e + SB, min(SB, e1 - e - SB));
      if (ND == 2 && ntask <= 32) {
        // one task per lane (coil groups of up to 4 coils): the task's coil pair and
        // tap are fixed for the whole batch; same cells, weights and order as below.
        // A tap at local index r + t < 0 wraps to G + r + t >= G - 3, inside the
        // tile only on grids narrower than T + 3: the wrap is skipped on the others.
        const bool act = lane < ntask;
        const int pr = npair == 2 ? (lane & 1) : lane % npair;
        const int tap = npair == 2 ? (lane >> 1) : lane / npair;
        const int ox = tap >> 2, oy = tap & 3;
        float4* accp = reinterpret_cast<float4*>(acc) + pr;
        auto visit = [&](auto wrap_t) {
        constexpr bool WRAP = decltype(wrap_t)::value;
        for (int j = 0; j < nbat; ++j) {
          const Base bb = sb[j];
          int lx = bb.x + ox, ly = bb.y + oy;
          if (WRAP) {
            lx += lx < 0 ? g.G[0] : 0;
            ly += ly < 0 ? g.G[1] : 0;
          }
          if (act && (unsigned)lx < (unsigned)T && (unsigned)ly < (unsigned)T) {
            const float* wj = sw + j * NW;
            const float w = wj[ox] * wj[4 + oy];
            const float4 v = reinterpret_cast<const float4*>(sy + j * cps)[pr];
            float4* p = accp + (lx * T + ly) * npair;
            float4 t = *p;
            t.x = fmaf(w, v.x, t.x);
            t.y = fmaf(w, v.y, t.y);
            t.z = fmaf(w, v.z, t.z);
            t.w = fmaf(w, v.w, t.w);
            *p = t;
          }
          __syncwarp();
        }
        };
        if (g.G[0] < T + 3 || g.G[1] < T + 3) visit(std::true_type{});
        else visit(std::false_type{});
        continue;
      }
      for (int j = 0; j < nbat; ++j) {
        const Base bb = sb[j];
        const float* wj = sw + j * NW;
        const float4* yj = reinterpret_cast<const float4*>(sy + j * cps);
        // lane tasks: (tap, coil pair), every task of a sample touches a distinct float4;
        // coil pair fastest, so that the 8 lanes of a 128-bit access phase cover
        // consecutive (cell, pair) slots (taps first: all 4 taps of a row land on
        // the same bank group and conflict 2-way)
        for (int tk = lane; tk < ntask; tk += 32) {
          const int pr = npair == 2 ? (tk & 1) : tk % npair;
          const int tap = npair == 2 ? (tk >> 1) : tk / npair;
          int cell;
          float w;
          bool inside;
          if (ND == 2) {
            const int ox = tap >> 2, oy = tap & 3;
            int lx = bb.x + ox, ly = bb.y + oy;
            lx += lx < 0 ? g.G[0] : 0;
            ly += ly < 0 ? g.G[1] : 0;
            inside = (unsigned)lx < (unsigned)T && (unsigned)ly < (unsigned)T;
            cell = lx * T + ly;
            w = inside ? wj[ox] * wj[4 + oy] : 0.f;
          } else {
            const int a0 = tap >> 4, a1 = (tap >> 2) & 3, a2 = tap & 3;
            int l0 = bb.x + a0, l1 = bb.y + a1, l2 = base_z(bb) + a2;
            l0 += l0 < 0 ? g.G[0] : 0;
            l1 += l1 < 0 ? g.G[1] : 0;
            l2 += l2 < 0 ? g.G[2] : 0;
            inside = (unsigned)l0 < (unsigned)T && (unsigned)l1 < (unsigned)T && (unsigned)l2 < (unsigned)T;
            cell = (l0 * T + l1) * T + l2;
            w = inside ? wj[a0] * wj[4 + a1] * wj[8 + a2] : 0.f;
          }
          if (inside) {
            const float4 v = yj[pr];
            float4* p = reinterpret_cast<float4*>(acc + cell * cps) + pr;
            float4 t = *p;
            t.x = fmaf(w, v.x, t.x);
            t.y = fmaf(w, v.y, t.y);
            t.z = fmaf(w, v.z, t.z);
            t.w = fmaf(w, v.w, t.w);
            *p = t;
          }
        }
        __syncwarp();
      }
    }
    // write the whole tile once (or this chunk's partial tile): lane task = (cell
    // pair along the last dim, coil pair); two 128-bit shared loads, one 128-bit
    // global store per coil
    for (int i = lane; i < PAIRS * npair; i += 32) {
      // (cell pair, coil pair) of the task: shifts for 1 or 2 coil pairs (up to 4 coils per item)
      const int pr = npair == 2 ? (i & 1) : npair == 1 ? 0 : i % npair;
      const int r = npair == 2 ? (i >> 1) : npair == 1 ? i : i / npair;
      const int l = (r % (T / 2)) * 2;
      const int rr = r / (T / 2);
      const int cl0 = rr * T + l;
      const float4 a0 = reinterpret_cast<const float4*>(acc + cl0 * cps)[pr];
      const float4 a1 = reinterpret_cast<const float4*>(acc + (cl0 + 1) * cps)[pr];
      int n[3];
      const long long cell = cell_of_pair(r, n);
      const bool ok = in_grid(n) && (pout || pair_touched(a, b, cell));
  #pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int cl = 2 * pr + h;
        if (cl >= nc) continue;
        const float4 v = h == 0 ? make_float4(a0.x, a0.y, a1.x, a1.y) : make_float4(a0.z, a0.w, a1.z, a1.w);
        if (pout) {
          *reinterpret_cast<float4*>(pout + (long long)cl * TN + rr * T + l) = v;
        } else if (ok) {
          *reinterpret_cast<float4*>(gout + (long long)cl * g.gtot + cell) = v;
        }
      }
    }
  }
};
template <int ND, int T>
__global__ void __launch_bounds__(SPREAD_WARPS * 32) spread_kernel(SpreadArgs a, Geo g, TileGeo tg, KBPoly kb) {
  SpreadWarp<ND, T>::run(hw_block(), a, g, tg, kb);
}

// 2D per-warp spread with per-sample tap tables.  Ownership, sample order and
// arithmetic are those of spread_kernel<2, T> (identical grids); what moves is
// the per-tap work.  While a batch is staged, lane j computes sample j's taps
// that fall inside the tile once (wrapped node, cell offset, weight product)
// and stores them compacted, so that the per-sample loop runs over the inside
// taps x coil pairs only and a lane task is two table reads and one 128-bit
// shared read-modify-write; (tap, coil pair) of a lane per round is fixed for
// the work item.  A listing of a sample whose support straddles tiles holds
// fewer than 16 inside taps.  The tile's touched-cell bitmap rows are read
// once per work item.  Coil groups of up to 16 coils (8 pairs).
constexpr int SW2_MAXR = 4;   // rounds of 32 lane tasks per sample: 16 taps x 8 pairs

template <int T>
struct Spread2wSmem {
  static constexpr int CELLS = T * T;
  __host__ __device__ static int cstride(int cpi) { return (cpi + 1) & ~1; }
  // acc [cell][coil] | tap cells (short) | tap weights | tap counts | bitmap rows | staged coil values
  __host__ __device__ static size_t acc_bytes(int cpi) { return (size_t)cstride(cpi) * CELLS * sizeof(float2); }
  static constexpr size_t TAB = SPREAD_BATCH * 16 * (sizeof(short) + sizeof(float)) + SPREAD_BATCH * sizeof(int) +
                                ((T * sizeof(unsigned) + 15) & ~(size_t)15);
  __host__ __device__ static size_t warp_bytes(int cpi) {
    return acc_bytes(cpi) + TAB + (size_t)SPREAD_BATCH * cstride(cpi) * sizeof(float2);
  }
};

template <int T>
struct Spread2Taps {
  static constexpr int NT = SPREAD_WARPS * 32, MINB = 5;
  static constexpr const char* FAMILY = "spread";
  static __device__ __forceinline__ void run(const VBlock& vb, const SpreadArgs& a, const Geo& g,
      const TileGeo& tg, const KBPoly& kb) {
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    using SM = Spread2wSmem<T>;
    constexpr int CELLS = SM::CELLS;
    constexpr int PAIRS = CELLS / 2;
    extern __shared__ float4 smem4[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long item = (long long)vb.x * SPREAD_WARPS + warp;
    const long long reps = g.B == 1 ? a.nb : a.nb / g.B;
    const long long nitems = reps * a.n_items * a.ngroups;
    if (item >= nitems) return;
    const int grp = (int)(item % a.ngroups);
    const long long oi = item / a.ngroups;
    const int4 it = a.items[oi % a.n_items];
    const int rep = (int)(oi / a.n_items);
    const int okey = it.x;
    const int b = okey / tg.ntiles;
    const int tile = okey - b * tg.ntiles;
    const int be = (g.B == 1) ? rep : b * (a.nb / g.B) + rep;
    const int c0 = grp * a.cpi;
    const int nc = min(a.cpi, g.C - c0);
    const int o0 = (tile / tg.nt[1]) * T, o1 = (tile % tg.nt[1]) * T;
    const int k0 = a.tile_start[okey], k1 = a.tile_start[okey + 1];
    const int e0 = min(k1, k0 + it.y * a.chunk), e1 = min(k1, e0 + a.chunk);
    float2* gout = a.grid + ((long long)be * g.C + c0) * g.gtot;
    const int G0 = g.G[0], G1 = g.G[1];
    float2* pout = it.z >= 0 ? a.partials + (((long long)rep * a.n_slots + it.z) * g.C + c0) * CELLS : nullptr;

    if (e0 == e1 && !pout) {   // no sample touches this tile: zeros
      if (a.touch) return;     // its cells are outside every support and never read
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int i = lane; i < nc * PAIRS; i += 32) {
        const int cl = i / PAIRS, r = i - cl * PAIRS;
        const int n0 = o0 + r / (T / 2), n1 = o1 + (r % (T / 2)) * 2;
        if (n0 < G0 && n1 < G1) *reinterpret_cast<float4*>(gout + (long long)cl * g.gtot + (long long)n0 * G1 + n1) = z4;
      }
      return;
    }

    const int cps = SM::cstride(a.cpi);
    const int npair = cps >> 1;
    char* wbase = reinterpret_cast<char*>(smem4) + (size_t)warp * SM::warp_bytes(a.cpi);
    float2* acc = reinterpret_cast<float2*>(wbase);
    short* tcell = reinterpret_cast<short*>(wbase + SM::acc_bytes(a.cpi));
    float* tw = reinterpret_cast<float*>(tcell + SPREAD_BATCH * 16);
    int* tcnt = reinterpret_cast<int*>(tw + SPREAD_BATCH * 16);
    unsigned* tbits = reinterpret_cast<unsigned*>(tcnt + SPREAD_BATCH);
    float2* sy = reinterpret_cast<float2*>(wbase + SM::acc_bytes(a.cpi) + SM::TAB);

    {
      float4* acc4 = reinterpret_cast<float4*>(acc);
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int i = lane; i < cps * CELLS / 2; i += 32) acc4[i] = z4;
    }
    // the touched-cell bits of the tile's rows (bit l of row r = cell (o0 + r, o1 + l))
    if (!pout && a.touch && lane < T) {
      unsigned m = 0;
      const int n0 = o0 + lane;
      if (n0 < G0) {
        const long long cell = (long long)n0 * G1 + o1;
        const unsigned* tb = a.touch + (long long)b * a.twords;
        const long long wi = cell >> 5;
        const int sh = (int)(cell & 31);
        unsigned long long v = __ldg(tb + wi);
        if (sh + T > 32 && wi + 1 < a.twords) v |= (unsigned long long)__ldg(tb + wi + 1) << 32;
        m = (unsigned)(v >> sh);
      }
      tbits[lane] = m;
    }
    // this lane's (tap, coil pair) in each round of a sample's tasks
    int tap_r[SW2_MAXR], pr_r[SW2_MAXR];
  #pragma unroll
    for (int r = 0; r < SW2_MAXR; ++r) {
      tap_r[r] = (lane + 32 * r) / npair;
      pr_r[r] = (lane + 32 * r) - tap_r[r] * npair;
    }
    __syncwarp();

    const float* gxp = a.gx + (long long)b * 2 * g.K;
    const float2* yb = a.y + ((long long)be * g.C + c0) * g.K;
    // the next batch's sample index, coordinates, weight and first coil values
    // are loaded into registers while the warp works on the current batch
    constexpr int PF = 4;
    int pk = 0;
    float px[2], pwa = 1.f;
    float2 py[PF];
    auto fetch = [&](int e, int nbat) {
      if (lane < nbat) {
        pk = a.entries[e + lane];
        px[0] = gxp[pk];
        px[1] = gxp[g.K + pk];
        if (a.wadj) pwa = a.wadj[(long long)b * g.K + pk];
  #pragma unroll
        for (int cl = 0; cl < PF; ++cl) py[cl] = cl < nc ? yb[(long long)cl * g.K + pk] : make_float2(0.f, 0.f);
      }
    };
    if (e0 < e1) fetch(e0, min(SPREAD_BATCH, e1 - e0));
    for (int e = e0; e < e1; e += SPREAD_BATCH) {
      const int nbat = min(SPREAD_BATCH, e1 - e);
      if (lane < nbat) {
        const int k = pk;
        float ws = a.gsign;
        if (a.wadj) ws *= pwa;
        float wv[2][4];
        int base[2];
  #pragma unroll
        for (int d = 0; d < 2; ++d) {
          const float x = px[d];
          base[d] = (int)floorf(x) - 1;
          const float fx = x - (float)(base[d] + 1);
  #pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int n = base[d] + q;
            float w = mrb::kb_tap(kb, q, fx);
            if (n & 1) w = -w;
            if (d == 0) w *= ws;
            wv[d][q] = w;
          }
        }
        short* tc = tcell + lane * 16;
        float* tww = tw + lane * 16;
        int m = 0;
  #pragma unroll
        for (int ox = 0; ox < 4; ++ox) {
          int n0 = base[0] + ox;
          n0 += n0 < 0 ? G0 : 0;
          n0 -= n0 >= G0 ? G0 : 0;
          const int lx = n0 - o0;
          if ((unsigned)lx < (unsigned)T) {
  #pragma unroll
            for (int oy = 0; oy < 4; ++oy) {
              int n1 = base[1] + oy;
              n1 += n1 < 0 ? G1 : 0;
              n1 -= n1 >= G1 ? G1 : 0;
              const int ly = n1 - o1;
              if ((unsigned)ly < (unsigned)T) {
                tc[m] = (short)(lx * T + ly);
                tww[m] = wv[0][ox] * wv[1][oy];
                ++m;
              }
            }
          }
        }
        tcnt[lane] = m;
  #pragma unroll
        for (int cl = 0; cl < PF; ++cl)
          if (cl < cps) sy[lane * cps + cl] = py[cl];
        for (int cl = PF; cl < cps; ++cl)
          sy[lane * cps + cl] = cl < nc ? yb[(long long)cl * g.K + k] : make_float2(0.f, 0.f);
      }
      __syncwarp();
      if (e + SPREAD_BATCH < e1) fetch(e + SPREAD_BATCH, min(SPREAD_BATCH, e1 - e - SPREAD_BATCH));
      for (int j = 0; j < nbat; ++j) {
        const int nt = tcnt[j] * npair;
        const short* tc = tcell + j * 16;
        const float* twj = tw + j * 16;
        const float4* yj = reinterpret_cast<const float4*>(sy + j * cps);
  #pragma unroll
        for (int r = 0; r < SW2_MAXR; ++r) {
          if (lane + 32 * r < nt) {
            const int cell = tc[tap_r[r]];
            const float w = twj[tap_r[r]];
            const float4 v = yj[pr_r[r]];
            float4* p = reinterpret_cast<float4*>(acc + cell * cps) + pr_r[r];
            float4 t = *p;
            t.x = fmaf(w, v.x, t.x);
            t.y = fmaf(w, v.y, t.y);
            t.z = fmaf(w, v.z, t.z);
            t.w = fmaf(w, v.w, t.w);
            *p = t;
          }
        }
        __syncwarp();
      }
    }
    // write the whole tile once (or this chunk's partial tile): lane task = (cell
    // pair along the row, coil pair), coil pair fastest; two 128-bit shared loads,
    // one 128-bit global store per coil
    const int qd = 32 / npair, qr = 32 - qd * npair;
    int pr = lane % npair, r = lane / npair;
    for (int i = lane; i < PAIRS * npair; i += 32) {
      const int l = (r % (T / 2)) * 2;
      const int rr = r / (T / 2);
      const int cl0 = rr * T + l;
      const float4 a0 = reinterpret_cast<const float4*>(acc + cl0 * cps)[pr];
      const float4 a1 = reinterpret_cast<const float4*>(acc + (cl0 + 1) * cps)[pr];
      const int n0 = o0 + rr, n1 = o1 + l;
      const long long cell = (long long)n0 * G1 + n1;
      const bool ok = n0 < G0 && n1 < G1 && (pout || !a.touch || ((tbits[rr] >> (l & ~3)) & 15u));
  #pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int cl = 2 * pr + h;
        if (cl >= nc) continue;
        const float4 v = h == 0 ? make_float4(a0.x, a0.y, a1.x, a1.y) : make_float4(a0.z, a0.w, a1.z, a1.w);
        if (pout) {
          *reinterpret_cast<float4*>(pout + (long long)cl * CELLS + cl0) = v;
        } else if (ok) {
          *reinterpret_cast<float4*>(gout + (long long)cl * g.gtot + cell) = v;
        }
      }
      pr += qr;
      r += qd;
      if (pr >= npair) {
        pr -= npair;
        ++r;
      }
    }
  }
};
template <int T>
__global__ void __launch_bounds__(SPREAD_WARPS * 32) spread2w_kernel(SpreadArgs a, Geo g, TileGeo tg, KBPoly kb) {
  Spread2Taps<T>::run(hw_block(), a, g, tg, kb);
}

// 3D adjoint spread, one block per work item (8^3 tile, chunk of its sample
// list, group of up to 16 coils).  The per-warp kernel above repeats the tap
// arithmetic once per coil group and walks all 64 taps of every sample visit;
// in 3D that is most of its time.  Here the coils of a group share one
// shared-memory tile [cell][coil pair] and the sample staging: each batch of
// samples is loaded once per block (weights computed once, 64 x (dim) kernel
// evaluations per batch, coil values read coalesced along the sample list).
// Warp w owns the tile plane l0 = w, so warps never write the same cell and
// need no atomics: for a sample whose support meets plane w, lanes are
// (coil pair p, tap a2) and the loop runs over a1 (a warp-uniform row test
// skips rows outside the tile).  A quarter warp updates the PPL coil pairs of
// one cell: 16 * PPL contiguous bytes, free of bank conflicts.  The staged
// coil values are XOR-swizzled by sample so that the staging stores conflict
// at most 4-way.  Summation order per (cell, coil) is the sample-list order,
// as in the per-warp kernel: both give identical grids.
// ---------------------------------------------------------------------------
constexpr int S3_T = 8;         // tile edge (cells)
constexpr int S3_WARPS = 8;     // one warp per tile plane
constexpr int S3_BATCH = 64;    // samples staged per pass (two ballots of 32)
constexpr int S3_CPB = 16;      // coils per block (group)

template <int PPL>
struct Spread3Smem {
  static constexpr int CELLS = S3_T * S3_T * S3_T;
  static constexpr int CPS = 2 * PPL;   // float2 per cell
  static constexpr size_t ACC = (size_t)CELLS * CPS * sizeof(float2);
  static constexpr size_t BYTES = ACC + S3_BATCH * (sizeof(int4) + 12 * sizeof(float)) +
                                  (size_t)S3_BATCH * CPS * sizeof(float2);
};

template <int PPL>
__global__ void __launch_bounds__(S3_WARPS * 32) spread3_kernel(SpreadArgs a, Geo g, TileGeo tg, KBPoly kb) {
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  using SM = Spread3Smem<PPL>;
  constexpr int T = S3_T;
  constexpr int CPS = SM::CPS;
  constexpr int TPI = 32 / PPL;        // taps (a1, a2) per lane pass
  constexpr int ROWS = TPI / 4;        // a1 rows per lane pass
  extern __shared__ float4 smem4[];
  float4* acc4 = smem4;                                             // [cell][pair]
  int4* sb = reinterpret_cast<int4*>(reinterpret_cast<char*>(smem4) + SM::ACC);
  float* sw = reinterpret_cast<float*>(sb + S3_BATCH);
  float4* sy4 = reinterpret_cast<float4*>(sw + S3_BATCH * 12);     // [sample][pair slot]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long item = blockIdx.x;
  const int grp = (int)(item % a.ngroups);
  const long long oi = item / a.ngroups;
  const int4 it = a.items[oi % a.n_items];
  const int rep = (int)(oi / a.n_items);
  const int b = it.x / tg.ntiles;
  const int tile = it.x - b * tg.ntiles;
  const int be = (g.B == 1) ? rep : b * (a.nb / g.B) + rep;
  const int c0 = grp * a.cpi;
  const int nc = min(a.cpi, g.C - c0);
  const int o2 = (tile % tg.nt[2]) * T;
  const int o1 = ((tile / tg.nt[2]) % tg.nt[1]) * T;
  const int o0 = (tile / (tg.nt[2] * tg.nt[1])) * T;
  const int k0 = a.tile_start[it.x], k1 = a.tile_start[it.x + 1];
  const int e0 = min(k1, k0 + it.y * a.chunk), e1 = min(k1, e0 + a.chunk);
  constexpr int TN = T * T * T;
  float2* pout = it.z >= 0 ? a.partials + (((long long)rep * a.n_slots + it.z) * g.C + c0) * TN : nullptr;

  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = threadIdx.x; i < SM::CELLS * PPL; i += blockDim.x) acc4[i] = z4;

  // this warp's plane; lanes (pair p, tap sub q)
  const int P0 = o0 + warp;
  const int p = lane % PPL, q = lane / PPL;
  const int a2 = q & 3, arow = q >> 2;
  const float* gxp = a.gx + (long long)b * 3 * g.K;
  const float2* yb = a.y + ((long long)be * g.C + c0) * g.K;

  for (int e = e0; e < e1; e += S3_BATCH) {
    const int nbat = min(S3_BATCH, e1 - e);
    __syncthreads();   // previous batch consumed (and the zero fill done)
    // stage: (sample, dim) weights, then coil values
    for (int i = threadIdx.x; i < nbat * 3; i += blockDim.x) {
      const int j = i / 3, d = i - 3 * j;
      const int k = a.entries[e + j];
      const float x = gxp[(long long)d * g.K + k];
      const int base = (int)floorf(x) - 1;
      float ws = 1.f;
      if (d == 0) {
        ws = a.gsign;
        if (a.wadj) ws *= a.wadj[(long long)b * g.K + k];
      }
      const float fx = x - (float)(base + 1);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int n = base + t;
        float w = mrb::kb_tap(kb, t, fx);
        if (n & 1) w = -w;
        sw[j * 12 + d * 4 + t] = w * ws;
      }
      // tile-relative first node, modulo G in [-3, G - 4] (grid sides >= T + 3):
      // tap t of the sample lies at local index rel + t, or outside the tile
      const int od = d == 0 ? o0 : d == 1 ? o1 : o2;
      int rel = base - od;
      rel += rel < -3 ? g.G[d] : 0;
      rel -= rel > g.G[d] - 4 ? g.G[d] : 0;
      reinterpret_cast<int*>(sb + j)[d] = rel;
    }
    for (int i = threadIdx.x; i < S3_BATCH * CPS; i += blockDim.x) {
      const int j = i % S3_BATCH, c = i / S3_BATCH;   // lanes along the sample list
      float2 v = make_float2(0.f, 0.f);
      if (j < nbat && c < nc) v = yb[(long long)c * g.K + a.entries[e + j]];
      const int slot = (c >> 1) ^ (j & (PPL - 1));
      reinterpret_cast<float2*>(sy4 + j * PPL + slot)[c & 1] = v;
    }
    __syncthreads();
    if (P0 >= g.G[0]) continue;   // plane beyond a partial last tile: nothing lands here
    // lane j tests sample h + j against this warp's plane; the warp then
    // visits only the samples whose support meets it
    for (int h = 0; h < nbat; h += 32) {
    int myd0 = 4;
    if (h + lane < nbat) myd0 = warp - sb[h + lane].x;   // tap a0 on this plane
    unsigned todo = __ballot_sync(0xffffffffu, (unsigned)myd0 < 4u);
    while (todo) {
      const int jl = __ffs(todo) - 1;
      todo &= todo - 1;
      const int j = h + jl;
      const int4 bb = sb[j];
      const int d0 = __shfl_sync(0xffffffffu, myd0, jl);
      const int l2 = bb.z + a2;   // below 0 only outside the tile
      const bool in2 = (unsigned)l2 < (unsigned)T && p < (nc + 1) / 2;
      const float* wj = sw + j * 12;
      const float w0 = wj[d0], w2 = wj[8 + a2];
      const float4 v = sy4[j * PPL + (p ^ (j & (PPL - 1)))];
#pragma unroll
      for (int r = 0; r < 4 / ROWS; ++r) {
        const int a1 = r * ROWS + arow;
        const int l1 = bb.y + a1;
        if (in2 && (unsigned)l1 < (unsigned)T) {
          const float w = w0 * wj[4 + a1] * w2;   // the per-warp kernel's product order
          float4* c4 = acc4 + ((warp * T + l1) * T + l2) * PPL + p;
          float4 t = *c4;
          t.x = fmaf(w, v.x, t.x);
          t.y = fmaf(w, v.y, t.y);
          t.z = fmaf(w, v.z, t.z);
          t.w = fmaf(w, v.w, t.w);
          *c4 = t;
        }
      }
      __syncwarp();
    }
    }
  }
  __syncthreads();
  // write-out: lanes (coil, cell pair along l2) read whole cells from shared
  // memory; each coil row gets 32-byte pieces
  const float2* acc = reinterpret_cast<const float2*>(acc4);
  float2* gout = a.grid + ((long long)be * g.C + c0) * g.gtot;
  for (int i = threadIdx.x; i < (TN / 2) * CPS; i += blockDim.x) {
    const int c = i % CPS, r = i / CPS;   // r: cell pair
    if (c >= nc) continue;
    const int cl = 2 * r;                  // local cell (l0, l1, l2 even)
    const float2 u0 = acc[cl * CPS + c], u1 = acc[(cl + 1) * CPS + c];
    const float4 v = make_float4(u0.x, u0.y, u1.x, u1.y);
    if (pout) {
      *reinterpret_cast<float4*>(pout + (long long)c * TN + cl) = v;
    } else {
      const int l0 = cl / (T * T), l1 = (cl / T) % T, l2 = cl % T;
      const int n0 = o0 + l0, n1 = o1 + l1, n2 = o2 + l2;
      if (n0 < g.G[0] && n1 < g.G[1] && n2 < g.G[2])
        *reinterpret_cast<float4*>(gout + (long long)c * g.gtot + ((long long)n0 * g.G[1] + n1) * g.G[2] + n2) = v;
    }
  }
}

// 3D adjoint spread with shared staging for two coil groups and per-sample tap
// tables (option key 6 = 2 in 3D).  One block per work item (8^3 tile, chunk,
// up to 8 * NG coils) of NG x 8 warps: warp w owns tile plane w % 8 for coil
// group w / 8 (4 pairs), so the staging of a batch (coordinates, 12 kernel
// weights, the in-tile row and column of every tap, the coil values) is done
// once for all 8 * NG coils instead of once per group of 8, and a lane task
// reads its row and column from the tables instead of wrapping and testing
// them.  With two groups the pair slots of odd cells are swapped between the
// groups, so that the 128-bit updates of neighbouring cells by one warp land
// in different bank halves.  Summation order per (cell, coil) and the weight
// product are spread3_kernel's: identical grids.
template <int NG>
struct Spread3tSmem {
  static constexpr int CELLS = S3_T * S3_T * S3_T;
  static constexpr int PT = 4 * NG;     // coil pairs per cell
  static constexpr int CPS = 2 * PT;    // float2 per cell
  static constexpr size_t ACC = (size_t)CELLS * CPS * sizeof(float2);
  static constexpr size_t TAB = S3_BATCH * (sizeof(int4) + 12 * sizeof(float) + 8);
  static constexpr size_t BYTES = ACC + TAB + (size_t)S3_BATCH * CPS * sizeof(float2);
};

template <int NG>
__global__ void __launch_bounds__(NG * S3_WARPS * 32) spread3t_kernel(SpreadArgs a, Geo g, TileGeo tg, KBPoly kb) {
  if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
  using SM = Spread3tSmem<NG>;
  constexpr int T = S3_T;
  constexpr int PPL = 4;                // pairs per warp group
  constexpr int PT = SM::PT, CPS = SM::CPS;
  constexpr int ROWS = (32 / PPL) / 4;  // a1 rows per lane pass (2)
  extern __shared__ float4 smem4[];
  float4* acc4 = smem4;                                             // [cell][pair slot]
  int4* sb = reinterpret_cast<int4*>(reinterpret_cast<char*>(smem4) + SM::ACC);
  float* sw = reinterpret_cast<float*>(sb + S3_BATCH);
  signed char* st1 = reinterpret_cast<signed char*>(sw + S3_BATCH * 12);   // [sample][a1]: in-tile row or -1
  signed char* st2 = st1 + S3_BATCH * 4;                                  // [sample][a2]: in-tile column or -1
  float4* sy4 = reinterpret_cast<float4*>(reinterpret_cast<char*>(smem4) + SM::ACC + SM::TAB);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int plane = warp % S3_WARPS, grp = warp / S3_WARPS;
  const long long item = blockIdx.x;
  const int igrp = (int)(item % a.ngroups);
  const long long oi = item / a.ngroups;
  const int4 it = a.items[oi % a.n_items];
  const int rep = (int)(oi / a.n_items);
  const int b = it.x / tg.ntiles;
  const int tile = it.x - b * tg.ntiles;
  const int be = (g.B == 1) ? rep : b * (a.nb / g.B) + rep;
  const int c0 = igrp * a.cpi;
  const int nc = min(a.cpi, g.C - c0);
  const int o2 = (tile % tg.nt[2]) * T;
  const int o1 = ((tile / tg.nt[2]) % tg.nt[1]) * T;
  const int o0 = (tile / (tg.nt[2] * tg.nt[1])) * T;
  const int k0 = a.tile_start[it.x], k1 = a.tile_start[it.x + 1];
  const int e0 = min(k1, k0 + it.y * a.chunk), e1 = min(k1, e0 + a.chunk);
  constexpr int TN = T * T * T;
  float2* pout = it.z >= 0 ? a.partials + (((long long)rep * a.n_slots + it.z) * g.C + c0) * TN : nullptr;

  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = threadIdx.x; i < SM::CELLS * PT; i += blockDim.x) acc4[i] = z4;

  const int P0 = o0 + plane;
  const int p = lane % PPL, q = lane / PPL;
  const int pg = grp * PPL + p;                 // this lane's pair within the block's coils
  const bool pair_ok = pg < (nc + 1) / 2;
  const int a2 = q & 3, arow = q >> 2;
  const float* gxp = a.gx + (long long)b * 3 * g.K;
  const float2* yb = a.y + ((long long)be * g.C + c0) * g.K;
  for (int e = e0; e < e1; e += S3_BATCH) {
    const int nbat = min(S3_BATCH, e1 - e);
    __syncthreads();   // previous batch consumed (and the zero fill done)
    // stage: (sample, dim) weights and, for dims 1 and 2, the in-tile node of each tap
    for (int i = threadIdx.x; i < nbat * 3; i += blockDim.x) {
      const int j = i / 3, d = i - 3 * j;
      const int k = a.entries[e + j];
      const float x = gxp[(long long)d * g.K + k];
      const int base = (int)floorf(x) - 1;
      float ws = 1.f;
      if (d == 0) {
        ws = a.gsign;
        if (a.wadj) ws *= a.wadj[(long long)b * g.K + k];
      }
      const float fx = x - (float)(base + 1);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int n = base + t;
        float w = mrb::kb_tap(kb, t, fx);
        if (n & 1) w = -w;
        sw[j * 12 + d * 4 + t] = w * ws;
        if (d > 0) {
          int nn = n;
          nn += nn < 0 ? g.G[d] : 0;
          nn -= nn >= g.G[d] ? g.G[d] : 0;
          const int l = nn - (d == 1 ? o1 : o2);
          (d == 1 ? st1 : st2)[j * 4 + t] = (signed char)((unsigned)l < (unsigned)T ? l : -1);
        }
      }
      reinterpret_cast<int*>(sb + j)[d] = base;
    }
    for (int i = threadIdx.x; i < S3_BATCH * CPS; i += blockDim.x) {
      const int j = i % S3_BATCH, c = i / S3_BATCH;   // lanes along the sample list
      float2 v = make_float2(0.f, 0.f);
      if (j < nbat && c < nc) v = yb[(long long)c * g.K + a.entries[e + j]];
      const int slot = (c >> 1) ^ (j & (PT - 1));
      reinterpret_cast<float2*>(sy4 + j * PT + slot)[c & 1] = v;
    }
    __syncthreads();
    if (P0 >= g.G[0]) continue;   // plane beyond a partial last tile: nothing lands here
    for (int h = 0; h < nbat; h += 32) {
      int myd0 = 4;
      if (h + lane < nbat) {
        myd0 = P0 - sb[h + lane].x;
        myd0 += myd0 < 0 ? g.G[0] : 0;
        myd0 -= myd0 >= g.G[0] ? g.G[0] : 0;
      }
      unsigned todo = __ballot_sync(0xffffffffu, myd0 < 4);
      while (todo) {
        const int jl = __ffs(todo) - 1;
        todo &= todo - 1;
        const int j = h + jl;
        const int d0 = __shfl_sync(0xffffffffu, myd0, jl);
        const int l2 = st2[j * 4 + a2];
        const float* wj = sw + j * 12;
        const float w0 = wj[d0], w2 = wj[8 + a2];
        const float4 v = sy4[j * PT + (pg ^ (j & (PT - 1)))];
#pragma unroll
        for (int r = 0; r < 4 / ROWS; ++r) {
          const int a1 = r * ROWS + arow;
          const int l1 = st1[j * 4 + a1];
          if (pair_ok && l2 >= 0 && l1 >= 0) {
            const float w = w0 * wj[4 + a1] * w2;   // the per-warp kernel's product order
            const int cell = (plane * T + l1) * T + l2;
            const int slot = NG == 2 ? (pg ^ ((cell & 1) << 2)) : pg;
            float4* c4 = acc4 + cell * PT + slot;
            float4 t = *c4;
            t.x = fmaf(w, v.x, t.x);
            t.y = fmaf(w, v.y, t.y);
            t.z = fmaf(w, v.z, t.z);
            t.w = fmaf(w, v.w, t.w);
            *c4 = t;
          }
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();
  // write-out: lanes (coil, cell pair along l2) read whole cells from shared
  // memory; each coil row gets 32-byte pieces
  const float2* acc = reinterpret_cast<const float2*>(acc4);
  float2* gout = a.grid + ((long long)be * g.C + c0) * g.gtot;
  for (int i = threadIdx.x; i < (TN / 2) * CPS; i += blockDim.x) {
    const int c = i % CPS, r = i / CPS;   // r: cell pair
    if (c >= nc) continue;
    const int cl = 2 * r;                  // local cell (l0, l1, l2 even)
    const int s0 = NG == 2 ? ((c >> 1) ^ ((cl & 1) << 2)) : (c >> 1);
    const int s1 = NG == 2 ? ((c >> 1) ^ (((cl + 1) & 1) << 2)) : (c >> 1);
    const float2 u0 = acc[cl * CPS + 2 * s0 + (c & 1)], u1 = acc[(cl + 1) * CPS + 2 * s1 + (c & 1)];
    const float4 v = make_float4(u0.x, u0.y, u1.x, u1.y);
    if (pout) {
      *reinterpret_cast<float4*>(pout + (long long)c * TN + cl) = v;
    } else {
      const int l0 = cl / (T * T), l1 = (cl / T) % T, l2 = cl % T;
      const int n0 = o0 + l0, n1 = o1 + l1, n2 = o2 + l2;
      if (n0 < g.G[0] && n1 < g.G[1] && n2 < g.G[2])
        *reinterpret_cast<float4*>(gout + (long long)c * g.gtot + ((long long)n0 * g.G[1] + n1) * g.G[2] + n2) = v;
    }
  }
}

// 2D adjoint spread, one block per work item (16x16 tile, chunk of its sample
// list, group of up to 16 coils): the 2D counterpart of spread3_kernel.  Warp
// w owns tile rows 2w and 2w+1; lanes are (coil pair p, tap column a1) and a
// lane pass covers 8 / PPL tap rows.  Staging (coordinates, 8 kernel weights,
// coil values) is done once per block for all coils of the group.  Per
// (cell, coil) the samples are summed in sample-list order with the per-warp
// kernel's weight product, so both kernels give identical grids.
// ---------------------------------------------------------------------------
constexpr int S2_T = 16;
constexpr int S2_WARPS = 8;
constexpr int S2_RPW = S2_T / S2_WARPS;   // tile rows per warp
constexpr int S2_BATCH = 32;

template <int PPL>
struct Spread2Smem {
  static constexpr int CELLS = S2_T * S2_T;
  static constexpr int CPS = 2 * PPL;
  static constexpr size_t ACC = (size_t)CELLS * CPS * sizeof(float2);
  static constexpr size_t BYTES = ACC + S2_BATCH * (sizeof(int4) + 8 * sizeof(float)) +
                                  (size_t)S2_BATCH * CPS * sizeof(float2);
};

template <int PPL>
struct Spread2Block {
  static constexpr int NT = S2_WARPS * 32, MINB = (PPL <= 4 ? 2 : 1);
  static constexpr const char* FAMILY = "spread";
  static __device__ __forceinline__ void run(const VBlock& vb, const SpreadArgs& a, const Geo& g,
      const TileGeo& tg, const KBPoly& kb) {
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    using SM = Spread2Smem<PPL>;
    constexpr int T = S2_T;
    constexpr int CPS = SM::CPS;
    constexpr int RI = 8 / PPL;   // tap rows per lane pass
    extern __shared__ float4 smem4[];
    float4* acc4 = smem4;                                             // [cell][pair]
    int4* sb = reinterpret_cast<int4*>(reinterpret_cast<char*>(smem4) + SM::ACC);
    float* sw = reinterpret_cast<float*>(sb + S2_BATCH);
    float4* sy4 = reinterpret_cast<float4*>(sw + S2_BATCH * 8);      // [sample][pair slot]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long item = vb.x;
    const int grp = (int)(item % a.ngroups);
    const long long oi = item / a.ngroups;
    const int4 it = a.items[oi % a.n_items];
    const int rep = (int)(oi / a.n_items);
    const int b = it.x / tg.ntiles;
    const int tile = it.x - b * tg.ntiles;
    const int be = (g.B == 1) ? rep : b * (a.nb / g.B) + rep;
    const int c0 = grp * a.cpi;
    const int nc = min(a.cpi, g.C - c0);
    const int o0 = (tile / tg.nt[1]) * T;
    const int o1 = (tile % tg.nt[1]) * T;
    const int k0 = a.tile_start[it.x], k1 = a.tile_start[it.x + 1];
    const int e0 = min(k1, k0 + it.y * a.chunk), e1 = min(k1, e0 + a.chunk);
    constexpr int TN = T * T;
    float2* pout = it.z >= 0 ? a.partials + (((long long)rep * a.n_slots + it.z) * g.C + c0) * TN : nullptr;

    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = threadIdx.x; i < SM::CELLS * PPL; i += blockDim.x) acc4[i] = z4;

    const int R0 = o0 + warp * S2_RPW;   // the warp's first grid row
    const int p = lane % PPL, q = lane / PPL;
    const int a1 = q & 3, rsub = q >> 2;
    const bool pair_ok = p < (nc + 1) / 2;
    const float* gxp = a.gx + (long long)b * 2 * g.K;
    const float2* yb = a.y + ((long long)be * g.C + c0) * g.K;

    for (int e = e0; e < e1; e += S2_BATCH) {
      const int nbat = min(S2_BATCH, e1 - e);
      __syncthreads();   // previous batch consumed (and the zero fill done)
      for (int i = threadIdx.x; i < nbat * 2; i += blockDim.x) {
        const int j = i >> 1, d = i & 1;
        const int k = a.entries[e + j];
        const float x = gxp[(long long)d * g.K + k];
        const int base = (int)floorf(x) - 1;
        float ws = 1.f;
        if (d == 0) {
          ws = a.gsign;
          if (a.wadj) ws *= a.wadj[(long long)b * g.K + k];
        }
        const float fx = x - (float)(base + 1);
  #pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int n = base + t;
          float w = mrb::kb_tap(kb, t, fx);
          if (n & 1) w = -w;
          sw[j * 8 + d * 4 + t] = w * ws;
        }
        reinterpret_cast<int*>(sb + j)[d] = base;
      }
      for (int i = threadIdx.x; i < S2_BATCH * CPS; i += blockDim.x) {
        const int j = i % S2_BATCH, c = i / S2_BATCH;   // lanes along the sample list
        float2 v = make_float2(0.f, 0.f);
        if (j < nbat && c < nc) v = yb[(long long)c * g.K + a.entries[e + j]];
        const int slot = (c >> 1) ^ (j & (PPL - 1));
        reinterpret_cast<float2*>(sy4 + j * PPL + slot)[c & 1] = v;
      }
      __syncthreads();
      if (R0 >= g.G[0]) continue;   // rows beyond a partial last tile: nothing lands here
      // lane j tests sample j against this warp's rows; the warp then visits
      // only the samples whose support meets them
      int myd0 = 4;
      bool hit = false;
      if (lane < nbat) {
        myd0 = R0 - sb[lane].x;
        myd0 += myd0 < 0 ? g.G[0] : 0;
        myd0 -= myd0 >= g.G[0] ? g.G[0] : 0;
        hit = myd0 < 4 || myd0 + S2_RPW - 1 >= g.G[0];
      }
      unsigned todo = __ballot_sync(0xffffffffu, hit);
      while (todo) {
        const int j = __ffs(todo) - 1;
        todo &= todo - 1;
        const int4 bb = sb[j];
        const int d0 = __shfl_sync(0xffffffffu, myd0, j);
        int n1 = bb.y + a1;
        n1 += n1 < 0 ? g.G[1] : 0;
        n1 -= n1 >= g.G[1] ? g.G[1] : 0;
        const int l1 = n1 - o1;
        const bool in1 = pair_ok && (unsigned)l1 < (unsigned)T;
        const float* wj = sw + j * 8;
        const float w1 = wj[4 + a1];
        const float4 v = sy4[j * PPL + (p ^ (j & (PPL - 1)))];
  #pragma unroll
        for (int r0 = 0; r0 < S2_RPW; r0 += RI) {
          const int r = r0 + rsub;
          int a0 = d0 + r;
          a0 -= a0 >= g.G[0] ? g.G[0] : 0;
          if (in1 && r < S2_RPW && a0 < 4 && R0 + r < g.G[0]) {
            const float w = wj[a0] * w1;   // the per-warp kernel's product order
            float4* c4 = acc4 + ((warp * S2_RPW + r) * T + l1) * PPL + p;
            float4 t = *c4;
            t.x = fmaf(w, v.x, t.x);
            t.y = fmaf(w, v.y, t.y);
            t.z = fmaf(w, v.z, t.z);
            t.w = fmaf(w, v.w, t.w);
            *c4 = t;
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // write-out: lanes (coil, cell pair along the row) read whole cells from
    // shared memory; each coil row gets 32-byte pieces
    const float2* acc = reinterpret_cast<const float2*>(acc4);
    float2* gout = a.grid + ((long long)be * g.C + c0) * g.gtot;
    for (int i = threadIdx.x; i < (TN / 2) * CPS; i += blockDim.x) {
      const int c = i % CPS, r = i / CPS;
      if (c >= nc) continue;
      const int cl = 2 * r;
      const float2 u0 = acc[cl * CPS + c], u1 = acc[(cl + 1) * CPS + c];
      const float4 v = make_float4(u0.x, u0.y, u1.x, u1.y);
      if (pout) {
        *reinterpret_cast<float4*>(pout + (long long)c * TN + cl) = v;
      } else {
        const int n0 = o0 + cl / T, n1 = o1 + cl % T;
        const long long cell = (long long)n0 * g.G[1] + n1;
        if (n0 < g.G[0] && n1 < g.G[1] && pair_touched(a, b, cell))
          *reinterpret_cast<float4*>(gout + (long long)c * g.gtot + cell) = v;
      }
    }
  }
};
template <int PPL>
__global__ void __launch_bounds__(S2_WARPS * 32) spread2_kernel(SpreadArgs a, Geo g, TileGeo tg, KBPoly kb) {
  Spread2Block<PPL>::run(hw_block(), a, g, tg, kb);
}

// Zeros for the tiles no sample touches: a store-only grid-stride pass, one
// float4 (two cells) per thread, consecutive threads along tile rows.
template <int ND, int T>
struct ZeroTiles {
  static constexpr int NT = 256, MINB = 6;
  static constexpr const char* FAMILY = "zero_tiles";
  static __device__ __forceinline__ void run(const VBlock& vb, const int* __restrict__ keys, int n_empty,
      float2* __restrict__ grid, const Geo& g, const TileGeo& tg, int nb) {
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    // block = one (rep, empty key); threads over (coil, cell pair)
    constexpr int PAIRS = (ND == 2 ? T * T : T * T * T) / 2;
    const int key = keys[vb.x % n_empty];
    const int rep = vb.x / n_empty;
    const int b = key / tg.ntiles;
    const int tile = key - b * tg.ntiles;
    const int be = (g.B == 1) ? rep : b * (nb / g.B) + rep;
    int o0, o1, o2 = 0;
    if (ND == 2) {
      o0 = (tile / tg.nt[1]) * T;
      o1 = (tile % tg.nt[1]) * T;
    } else {
      o2 = (tile % tg.nt[2]) * T;
      o1 = ((tile / tg.nt[2]) % tg.nt[1]) * T;
      o0 = (tile / (tg.nt[2] * tg.nt[1])) * T;
    }
    float2* base = grid + (long long)be * g.C * g.gtot;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = threadIdx.x; i < g.C * PAIRS; i += blockDim.x) {
      const int c = i / PAIRS, r = i - c * PAIRS;
      const int l = (r % (T / 2)) * 2;
      const int rr = r / (T / 2);
      int n0, n1, n2;
      long long idx;
      if (ND == 2) {
        n0 = o0 + rr;
        n1 = o1 + l;
        if (n0 >= g.G[0] || n1 >= g.G[1]) continue;
        idx = (long long)n0 * g.G[1] + n1;
      } else {
        n0 = o0 + rr / T;
        n1 = o1 + rr % T;
        n2 = o2 + l;
        if (n0 >= g.G[0] || n1 >= g.G[1] || n2 >= g.G[2]) continue;
        idx = ((long long)n0 * g.G[1] + n1) * g.G[2] + n2;
      }
      *reinterpret_cast<float4*>(base + (long long)c * g.gtot + idx) = z4;
    }
  }
};
template <int ND, int T>
__global__ void __launch_bounds__(256) zero_tiles_kernel(const int* __restrict__ keys, int n_empty,
    float2* __restrict__ grid, Geo g, TileGeo tg, int nb) {
  ZeroTiles<ND, T>::run(hw_block(), keys, n_empty, grid, g, tg, nb);
}

// Sum of the chunk partial tiles of split keys, in chunk order, written once
// into the grid.  Block = (rep, split key, coil); threads over the tile cells.
template <int ND, int T>
struct SpreadReduce {
  static constexpr int NT = 256, MINB = 6;
  static constexpr const char* FAMILY = "spread_reduce";
  static __device__ __forceinline__ void run(const VBlock& vb, const float2* __restrict__ partials,
      const int4* __restrict__ multi, int n_multi, int n_slots, float2* __restrict__ grid, const Geo& g,
      const TileGeo& tg, int nb) {
    if (g.skip != nullptr && *g.skip != 0.0) return;   // solve already finished
    constexpr int TN = ND == 2 ? T * T : T * T * T;
    const int c = vb.y;
    const int rep = vb.z;
    const int4 m = multi[vb.x];
    const int b = m.x / tg.ntiles;
    const int tile = m.x - b * tg.ntiles;
    const int be = (g.B == 1) ? rep : b * (nb / g.B) + rep;
    int o[3];
    if (ND == 2) {
      o[0] = (tile / tg.nt[1]) * T;
      o[1] = (tile % tg.nt[1]) * T;
      o[2] = 0;
    } else {
      o[2] = (tile % tg.nt[2]) * T;
      o[1] = ((tile / tg.nt[2]) % tg.nt[1]) * T;
      o[0] = (tile / (tg.nt[2] * tg.nt[1])) * T;
    }
    for (int cell = threadIdx.x; cell < TN; cell += blockDim.x) {
      float sx = 0.f, sy = 0.f;
      for (int j = 0; j < m.y; ++j) {
        float2 v = partials[(((long long)rep * n_slots + m.z + j) * g.C + c) * TN + cell];
        sx += v.x;
        sy += v.y;
      }
      int n0, n1, n2 = 0;
      long long idx;
      if (ND == 2) {
        n0 = o[0] + cell / T;
        n1 = o[1] + cell % T;
        if (n0 >= g.G[0] || n1 >= g.G[1]) continue;
        idx = (long long)n0 * g.G[1] + n1;
      } else {
        n0 = o[0] + cell / (T * T);
        n1 = o[1] + (cell / T) % T;
        n2 = o[2] + cell % T;
        if (n0 >= g.G[0] || n1 >= g.G[1] || n2 >= g.G[2]) continue;
        idx = ((long long)n0 * g.G[1] + n1) * g.G[2] + n2;
      }
      grid[((long long)be * g.C + c) * g.gtot + idx] = make_float2(sx, sy);
    }
  }
};
template <int ND, int T>
__global__ void __launch_bounds__(256) spread_reduce_kernel(const float2* __restrict__ partials,
    const int4* __restrict__ multi, int n_multi, int n_slots, float2* __restrict__ grid, Geo g, TileGeo tg,
    int nb) {
  SpreadReduce<ND, T>::run(hw_block(), partials, multi, n_multi, n_slots, grid, g, tg, nb);
}

// literal / corrected index tables for one frame
__global__ void grid_index_kernel(const float* __restrict__ traj, int nd, int G0, int G1, int G2, long long K,
                                  int W, int conv, long long* __restrict__ out) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  int G[3] = {G0, G1, G2};
  long long n[3][16];
  for (int d = 0; d < nd; ++d) {
    float gx = mrb::ref_grid_coord(traj[(long long)d * K + k], (float)G[d], (float)((double)G[d] - 1e-6));
    for (int o = 0; o < W; ++o) {
      long long v;
      if (conv == MRB_IDX_REFERENCE) {
        float off = (float)(o - W / 2);
        v = (long long)floorf(__fadd_rn(gx, off));
      } else {
        v = (long long)floorf(gx) + (o - (W / 2 - 1));
      }
      long long r = v % G[d];
      n[d][o] = r < 0 ? r + G[d] : r;
    }
  }
  long long W2 = (long long)W * W;
  long long per = nd == 2 ? W2 : W2 * W;
  long long* row = out + k * per;
  if (nd == 2) {
    for (int a = 0; a < W; ++a)
      for (int b = 0; b < W; ++b)
        row[a * W + b] = conv == MRB_IDX_REFERENCE ? n[0][a] + (long long)G0 * n[1][b]
                                                   : n[0][a] * G1 + n[1][b];
  } else {
    for (int a = 0; a < W; ++a)
      for (int b = 0; b < W; ++b)
        for (int c = 0; c < W; ++c)
          row[(a * W + b) * W + c] = conv == MRB_IDX_REFERENCE
                                         ? n[0][a] + (long long)G0 * n[1][b] + (long long)G0 * G1 * n[2][c]
                                         : (n[0][a] * G1 + n[1][b]) * G2 + n[2][c];
  }
}

__global__ void cell_base_kernel(const float* __restrict__ gx, int* __restrict__ out, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int)floorf(gx[i]);
}

int grid_blocks(long long n, int bs) { return (int)((n + bs - 1) / bs); }

// 2D column-strip key of each sample: frame, then the strip of sw columns that
// holds its first tap column floor(gx1) - 1 (wrapped)
__global__ void strip_key_kernel(const float* __restrict__ gx, unsigned* __restrict__ keys, int* __restrict__ vals,
                                 long long K, int B, int G1, int sw, int nstrips) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)B * K) return;
  const int b = (int)(i / K);
  const long long k = i - (long long)b * K;
  const int c = mrb::wrap_i((int)floorf(gx[((long long)b * 2 + 1) * K + k]) - 1, G1);
  keys[i] = (unsigned)(b * nstrips + c / sw);
  vals[i] = (int)k;
}

int ensure_fft(mrb_plan* p, int nb) {
  int batch = nb * p->C;
  if (p->fft && p->fft_batch == batch) return 0;
  if (p->fft) {
    cufftDestroy(p->fft);
    p->fft = 0;
  }
  int n[3] = {p->G[0], p->G[1], p->G[2]};
  int dist = (int)p->gtot();
  cufftResult r = cufftPlanMany(&p->fft, p->nd, n, nullptr, 1, dist, nullptr, 1, dist, CUFFT_C2C, batch);
  if (r != CUFFT_SUCCESS) {
    p->fft = 0;
    return mrb::fail(MRB_ECUFFT, "cufftPlanMany failed (%d) for batch %d", (int)r, batch);
  }
  p->fft_batch = batch;
  return 0;
}

int check_ready(mrb_plan* p) {
  if (!p) return mrb::fail(MRB_EINVAL, "null plan");
  if (!p->have_points) return mrb::fail(MRB_ESTATE, "plan has no trajectory (call mrb_plan_set_points)");
  if (!p->have_maps) return mrb::fail(MRB_ESTATE, "plan has no coil maps (call mrb_plan_set_maps)");
  return 0;
}

int check_nb(mrb_plan* p, int nb) {
  if (nb <= 0) return mrb::fail(MRB_EINVAL, "batch must be positive (got %d)", nb);
  if (p->B != 1 && nb % p->B != 0)
    return mrb::fail(MRB_EINVAL, "omega batch %d incompatible with requested %d", p->B, nb);
  return 0;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
// compiled zero-pruned passes exist for every dim of this grid
static bool fused_supported(const mrb_plan* p) {
  if (p->nd == 2) return mrb::fft2_supported(p->S[0], p->S[1], p->G[0], p->G[1]);
  return mrb::fft2_supported(p->S[0], p->S[1], p->G[0], p->G[1]) && mrb::fft2_supported(p->S[1], p->S[2], p->G[1], p->G[2]);
}

extern "C" int mrb_plan_create(mrb_plan** out, int nd, const int* S, int C, int B, int64_t K, int W, double osf,
                               int norm_ortho) {
  if (!out) return mrb::fail(MRB_EINVAL, "null output pointer");
  *out = nullptr;
  MRB_REQUIRE(nd == 2 || nd == 3, "nd must be 2 or 3 (got %d)", nd);
  MRB_REQUIRE(S != nullptr, "null image shape");
  MRB_REQUIRE(C >= 1 && B >= 1 && K >= 1, "C, B, K must be positive");
  MRB_REQUIRE(W == 4, "kernel width %d not supported (W = 4)", W);
  MRB_REQUIRE(osf >= 1.0 && osf <= 4.0, "osf out of range");
  mrb_plan* p = new mrb_plan();
  p->nd = nd;
  for (int d = 0; d < nd; ++d) {
    if (S[d] < 2) {
      delete p;
      return mrb::fail(MRB_EINVAL, "image dim %d must be >= 2", d);
    }
    p->S[d] = S[d];
    p->G[d] = (int)std::ceil(osf * (double)S[d]);
    if (p->G[d] % 2) {
      delete p;
      return mrb::fail(MRB_EINVAL, "oversampled grid dim %d = %d must be even", d, p->G[d]);
    }
  }
  p->C = C;
  p->B = B;
  p->K = K;
  p->W = W;
  p->osf = osf;
  p->ortho = norm_ortho ? 1 : 0;
  p->scale = norm_ortho ? (float)(1.0 / std::sqrt((double)p->gtot())) : 1.f;
  int hs = 0;
  for (int d = 0; d < nd; ++d) hs += p->G[d] / 2;
  p->gsign = (hs & 1) ? -1.f : 1.f;
  p->beta = M_PI * std::sqrt(std::pow((W / osf) * (osf - 0.5), 2) - 0.8);   // ptnufft.py:125
  mrb::kb_poly_init(p->kb, W, p->beta);
  p->tile = nd == 2 ? 16 : 8;
  p->chunk = nd == 2 ? 128 : 4096;   // 3D: a block per item, only the centre tiles need splitting
  p->interp_mode = 1;
  p->spread_kernel = nd == 3 ? 1 : 0;   // 2D: the per-warp kernel is faster at typical coil counts
  p->coils_per_item = nd == 2 ? std::min(C, 4) : std::min(C, 8);
  // deapodisation: closed-form FT of the truncated KB window
  std::vector<float> dap;
  double i0b = 0.0;
  {
    double q = 0.25 * p->beta * p->beta, term = 1.0, sum = 1.0;
    for (int k = 1; k < 200; ++k) {
      term *= q / ((double)k * k);
      sum += term;
      if (term < 1e-18 * sum) break;
    }
    i0b = sum;
  }
  for (int d = 0; d < nd; ++d) {
    for (int i = 0; i < S[d]; ++i) {
      double r = (double)(i - S[d] / 2);
      double a = p->beta * p->beta - std::pow(M_PI * W * r / p->G[d], 2);
      double ph;
      if (a > 0) ph = std::sinh(std::sqrt(a)) / std::sqrt(a);
      else if (a < 0) ph = std::sin(std::sqrt(-a)) / std::sqrt(-a);
      else ph = 1.0;
      ph *= W / i0b;
      dap.push_back((float)(1.0 / ph));
    }
  }
  int rc = p->invdeap.ensure(dap.size() * sizeof(float));
  if (!rc && cudaMemcpy(p->invdeap.p, dap.data(), dap.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = mrb::fail(MRB_ECUDA, "copying deapodisation failed");
  // the fused row passes see a frame as rows of the last dim: each row's
  // deapodisation over the leading dims with the sign (-1)^(sum of their
  // centred indices)
  if (!rc) {
    std::vector<float> rf;
    const int off0 = p->G[0] / 2 - S[0] / 2;
    if (nd == 2) {
      for (int r = 0; r < S[0]; ++r) rf.push_back(((r + off0) & 1) ? -dap[r] : dap[r]);
    } else {
      const int off1 = p->G[1] / 2 - S[1] / 2;
      for (int a = 0; a < S[0]; ++a)
        for (int b = 0; b < S[1]; ++b) {
          const float v = dap[a] * dap[S[0] + b];
          rf.push_back(((a + off0 + b + off1) & 1) ? -v : v);
        }
    }
    rc = p->rowfac.ensure(rf.size() * sizeof(float));
    if (!rc && cudaMemcpy(p->rowfac.p, rf.data(), rf.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = mrb::fail(MRB_ECUDA, "copying row deapodisation failed");
  }
  if (!rc && fused_supported(p)) rc = mrb_plan_set_option(p, 4, 1);
  if (!rc && nd == 3) p->il = 1;   // 2D: the planar column pass + interp is faster overall
  if (rc) {
    delete p;
    return rc;
  }
  *out = p;
  return 0;
}

extern "C" int mrb_plan_destroy(mrb_plan* p) {
  if (!p) return 0;
  if (p->fft) cufftDestroy(p->fft);
  for (DevBuf* b : {&p->gx, &p->entries, &p->tile_start, &p->items, &p->multi, &p->partials, &p->empty_keys, &p->maps, &p->invdeap, &p->wfwd,
                    &p->wadj, &p->grid, &p->tmp, &p->band, &p->tw0, &p->tw1, &p->psf, &p->ones, &p->grid_il,
                    &p->band2, &p->tw2, &p->rowfac,
                    &p->seg_order, &p->touch, &p->grid_adj,
                    &p->strip_start, &p->strip_entries, &p->tapw, &p->tapb})
    b->release();
  delete p;
  return 0;
}

extern "C" int mrb_plan_set_option(mrb_plan* p, int key, int64_t value) {
  MRB_REQUIRE(p != nullptr, "null plan");
  switch (key) {
    case 0:
      MRB_REQUIRE(value == 4 || value == 8 || value == 16 || value == 32, "tile edge must be 4, 8, 16 or 32");
      MRB_REQUIRE(p->nd == 2 || value <= 8, "3D tile edge must be <= 8");
      if (p->tile != (int)value) p->have_points = false;   // lists depend on the tile
      p->tile = (int)value;
      return 0;
    case 1:
      MRB_REQUIRE(value >= 1 && value <= 64, "coils per item out of range");
      p->coils_per_item = (int)std::min<int64_t>(value, p->C);
      return 0;
    case 2:
      MRB_REQUIRE(value == 0 || value == 1, "interp mode must be 0 or 1");
      p->interp_mode = (int)value;
      return 0;
    case 3:
      MRB_REQUIRE(value >= 16 && value <= (1 << 20), "chunk must be 16 .. 2^20 samples");
      if (p->chunk != (int)value) p->have_points = false;   // the item table depends on it
      p->chunk = (int)value;
      return 0;
    case 4:
      MRB_REQUIRE(value == 0 || value == 1, "fft mode must be 0 (cuFFT) or 1 (fused)");
      if (value == 1) {
        MRB_REQUIRE(fused_supported(p), "no fused FFT kernels for this grid (%d x %d x %d)", p->G[0], p->G[1],
                    p->nd == 3 ? p->G[2] : 1);
        if (!p->tw0p) {
          int rc;
          if ((rc = mrb::fft2_twiddles(p->tw0, p->G[0], &p->tw0p))) return rc;
          if ((rc = mrb::fft2_twiddles(p->tw1, p->G[1], &p->tw1p))) return rc;
          if (p->nd == 3 && (rc = mrb::fft2_twiddles(p->tw2, p->G[2], &p->tw2p))) return rc;
        }
      }
      p->fft_mode = (int)value;
      return 0;
    case 6:
      MRB_REQUIRE(value >= 0 && value <= 2,
                  "spread kernel must be 0 (per-warp), 1 (block per tile) or 2 (per-warp with tap tables)");
      p->spread_kernel = (int)value;
      return 0;
    case 8:
      MRB_REQUIRE(value == 0 || value == 1, "column interp must be 0 or 1");
      if (value == 1 && p->nstrips == 0) p->have_points = false;   // set_points builds the strip lists
      p->col_interp = (int)value;
      return 0;
    case 7:
      MRB_REQUIRE(value == 0 || value == 1, "grid mask must be 0 or 1");
      if (value != p->grid_mask) p->adj_zero = false;
      p->grid_mask = (int)value;
      return 0;
    case 5:
      MRB_REQUIRE(value == 0 || value == 1, "interleaved interp must be 0 or 1");
      p->il = (int)value;
      return 0;
    case 9:
      MRB_REQUIRE(value == 0 || value == 1, "blocked forward grid must be 0 or 1");
      p->grid_blk = (int)value;
      return 0;
    case 10:
      MRB_REQUIRE(value == 0 || value == 1, "tap table must be 0 or 1");
      p->tap_table = (int)value;
      return 0;
    default:
      return mrb::fail(MRB_EINVAL, "unknown option %d", key);
  }
}

extern "C" int mrb_plan_set_points(mrb_plan* p, const float* traj, mrb_stream_t stream) {
  MRB_REQUIRE(p != nullptr && traj != nullptr, "null plan or trajectory");
  cudaStream_t st = (cudaStream_t)stream;
  Geo g = make_geo(p);
  const long long nBK = (long long)p->B * p->K;
  const long long nall = nBK * p->nd;
  int rc;
  if ((rc = p->gx.ensure(nall * sizeof(float)))) return rc;
  coords_kernel<<<grid_blocks(nall, 256), 256, 0, st>>>(traj, p->gx.as<float>(), g);
  MRB_LAUNCH_CHECK();
  if (p->nd == 2 && p->W == 4) {
    if ((rc = p->tapw.ensure(nBK * 2 * sizeof(float4)))) return rc;
    if ((rc = p->tapb.ensure(nBK * sizeof(int2)))) return rc;
    taps2_kernel<<<grid_blocks(nBK, 256), 256, 0, st>>>(p->gx.as<float>(), p->tapw.as<float4>(), p->tapb.as<int2>(),
                                                        g, p->kb);
    MRB_LAUNCH_CHECK();
  }

  TileGeo tg{};
  tg.T = p->tile;
  tg.ntiles = 1;
  for (int d = 0; d < 3; ++d) tg.nt[d] = 1;
  for (int d = 0; d < p->nd; ++d) {
    tg.nt[d] = (p->G[d] + tg.T - 1) / tg.T;
    tg.ntiles *= tg.nt[d];
  }
  tg.lo_off = p->W / 2 - 1;
  tg.hi_off = p->W / 2;
  MRB_REQUIRE((long long)p->B * tg.ntiles < (1LL << 31), "too many tiles");
  p->ntiles = tg.ntiles;
  for (int d = 0; d < 3; ++d) p->ntile_d[d] = tg.nt[d];

  // counts + exclusive scan
  DevBuf cnt, offs;
  if ((rc = cnt.ensure((nBK + 1) * sizeof(int)))) return rc;
  if ((rc = offs.ensure((nBK + 1) * sizeof(int)))) { cnt.release(); return rc; }
  entry_count_kernel<<<grid_blocks(nBK, 256), 256, 0, st>>>(p->gx.as<float>(), cnt.as<int>(), g, tg);
  fill_int_kernel<<<1, 1, 0, st>>>(cnt.as<int>() + nBK, 1, 0);
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.as<int>(), offs.as<int>(), (int)(nBK + 1), st);
  if ((rc = p->tmp.ensure(tmp_bytes))) return rc;
  cub::DeviceScan::ExclusiveSum(p->tmp.p, tmp_bytes, cnt.as<int>(), offs.as<int>(), (int)(nBK + 1), st);
  MRB_LAUNCH_CHECK();
  int n_entries = 0;
  MRB_CUDA_TRY(cudaMemcpyAsync(&n_entries, offs.as<int>() + nBK, sizeof(int), cudaMemcpyDeviceToHost, st));
  MRB_CUDA_TRY(cudaStreamSynchronize(st));
  p->n_entries = n_entries;

  DevBuf keys, keys_sorted, vals;
  if ((rc = keys.ensure((size_t)std::max(n_entries, 1) * sizeof(unsigned)))) return rc;
  if ((rc = keys_sorted.ensure((size_t)std::max(n_entries, 1) * sizeof(unsigned)))) return rc;
  if ((rc = vals.ensure((size_t)std::max(n_entries, 1) * sizeof(int)))) return rc;
  if ((rc = p->entries.ensure((size_t)std::max(n_entries, 1) * sizeof(int)))) return rc;
  if ((rc = p->tile_start.ensure(((size_t)p->B * tg.ntiles + 1) * sizeof(int)))) return rc;
  entry_fill_kernel<<<grid_blocks(nBK, 256), 256, 0, st>>>(p->gx.as<float>(), offs.as<int>(), keys.as<unsigned>(),
                                                           vals.as<int>(), g, tg);
  MRB_LAUNCH_CHECK();
  int nkeys = p->B * tg.ntiles;
  int end_bit = 1;
  while ((1LL << end_bit) <= nkeys) ++end_bit;
  tmp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.as<unsigned>(), keys_sorted.as<unsigned>(),
                                  vals.as<int>(), p->entries.as<int>(), n_entries, 0, end_bit, st);
  if ((rc = p->tmp.ensure(tmp_bytes))) return rc;
  cub::DeviceRadixSort::SortPairs(p->tmp.p, tmp_bytes, keys.as<unsigned>(), keys_sorted.as<unsigned>(),
                                  vals.as<int>(), p->entries.as<int>(), n_entries, 0, end_bit, st);
  MRB_LAUNCH_CHECK();
  if (n_entries > 0) {
    tile_start_kernel<<<grid_blocks(n_entries, 256), 256, 0, st>>>(keys_sorted.as<unsigned>(), n_entries,
                                                                   p->tile_start.as<int>(), nkeys);
  } else {
    fill_int_kernel<<<grid_blocks(nkeys + 1, 256), 256, 0, st>>>(p->tile_start.as<int>(), nkeys + 1, 0);
  }
  MRB_LAUNCH_CHECK();
  // spread work items: (frame, tile) keys heaviest first, each split into
  // chunks of at most p->chunk samples; a key with several chunks gets
  // partial-tile slots that a second pass sums in chunk order
  {
    std::vector<int> ts((size_t)nkeys + 1);
    MRB_CUDA_TRY(cudaMemcpyAsync(ts.data(), p->tile_start.p, ts.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    MRB_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<int> order((size_t)nkeys);
    for (int k = 0; k < nkeys; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return ts[a + 1] - ts[a] > ts[b + 1] - ts[b]; });
    std::vector<int4> items, multi;
    std::vector<int> empty;
    items.reserve((size_t)nkeys);
    int slots = 0;
    for (int key : order) {
      int cnt = ts[key + 1] - ts[key];
      if (cnt == 0) {
        empty.push_back(key);
        continue;
      }
      int nch = (cnt + p->chunk - 1) / p->chunk;
      int base = -1;
      if (nch > 1) {
        base = slots;
        slots += nch;
        multi.push_back(make_int4(key, nch, base, 0));
      }
      for (int c = 0; c < nch; ++c) items.push_back(make_int4(key, c, nch > 1 ? base + c : -1, nch));
    }
    MRB_REQUIRE(items.size() < (1u << 31), "too many spread work items");
    std::sort(empty.begin(), empty.end());
    p->n_empty = (int)empty.size();
    if (!empty.empty()) {
      if ((rc = p->empty_keys.ensure(empty.size() * sizeof(int)))) return rc;
      MRB_CUDA_TRY(cudaMemcpy(p->empty_keys.p, empty.data(), empty.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    p->n_items = (int)items.size();
    p->n_multi = (int)multi.size();
    p->n_slots = slots;
    if (!items.empty()) {
      if ((rc = p->items.ensure(items.size() * sizeof(int4)))) return rc;
      MRB_CUDA_TRY(cudaMemcpy(p->items.p, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    if (!multi.empty()) {
      if ((rc = p->multi.ensure(multi.size() * sizeof(int4)))) return rc;
      MRB_CUDA_TRY(cudaMemcpy(p->multi.p, multi.data(), multi.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
  }

  // 3D interp visiting order: segments of IL_SEG samples sorted by (frame,
  // Morton code of the middle sample's tile), so that concurrently running
  // blocks gather from neighbouring cells instead of re-reading each spoke's
  // whole tube of the grid from HBM
  p->nseg = 0;
  if (p->nd == 3) {
    const long long nseg = (p->K + IL_SEG - 1) / IL_SEG;
    const long long n = (long long)p->B * nseg;
    MRB_REQUIRE(n < (1LL << 31) && nseg < (1LL << 31), "too many interp segments");
    int bits = 1;
    while ((1 << bits) < (std::max(p->G[0], std::max(p->G[1], p->G[2])) + 7) / 8) ++bits;
    int bbits = 1;
    while ((1LL << bbits) < p->B) ++bbits;
    const int end_bit2 = 3 * bits + bbits;
    MRB_REQUIRE(end_bit2 <= 64, "interp order key too wide");
    DevBuf k_in, k_out, v_in;
    if ((rc = k_in.ensure(n * sizeof(unsigned long long)))) return rc;
    if ((rc = k_out.ensure(n * sizeof(unsigned long long)))) return rc;
    if ((rc = v_in.ensure(n * sizeof(int)))) return rc;
    if ((rc = p->seg_order.ensure(n * sizeof(int)))) return rc;
    seg_key_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(p->gx.as<float>(), k_in.as<unsigned long long>(),
                                                         v_in.as<int>(), g, nseg, bits);
    MRB_LAUNCH_CHECK();
    size_t tb2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb2, k_in.as<unsigned long long>(), k_out.as<unsigned long long>(),
                                    v_in.as<int>(), p->seg_order.as<int>(), (int)n, 0, end_bit2, st);
    if ((rc = p->tmp.ensure(tb2))) return rc;
    cub::DeviceRadixSort::SortPairs(p->tmp.p, tb2, k_in.as<unsigned long long>(), k_out.as<unsigned long long>(),
                                    v_in.as<int>(), p->seg_order.as<int>(), (int)n, 0, end_bit2, st);
    MRB_LAUNCH_CHECK();
    MRB_CUDA_TRY(cudaStreamSynchronize(st));   // the temporaries are freed on return
    p->nseg = nseg;
  }

  // touched cells (sum over frames), for the roofline bookkeeping
  {
    // kept per frame: the fused column passes and the spread write-out use them
    long long nwords = (p->gtot() + 31) / 32;
    DevBuf cntd;
    if ((rc = p->touch.ensure((size_t)p->B * nwords * sizeof(unsigned)))) return rc;
    if ((rc = cntd.ensure(sizeof(unsigned long long)))) return rc;
    MRB_CUDA_TRY(cudaMemsetAsync(cntd.p, 0, sizeof(unsigned long long), st));
    MRB_CUDA_TRY(cudaMemsetAsync(p->touch.p, 0, (size_t)p->B * nwords * sizeof(unsigned), st));
    MRB_REQUIRE(p->B <= 65535, "too many trajectory frames");
    touch_kernel<<<dim3(grid_blocks(p->K, 256), p->B), 256, 0, st>>>(p->gx.as<float>(), p->touch.as<unsigned>(),
                                                                      nwords, g, p->W);
    popc_kernel<<<grid_blocks((long long)p->B * nwords, 256), 256, 0, st>>>(p->touch.as<unsigned>(),
                                                                           (long long)p->B * nwords,
                                                                           cntd.as<unsigned long long>());
    p->twords = nwords;
    // 2D: per-frame lists of the samples of each column strip (the fused
    // forward column pass interpolates a strip's samples from shared memory)
    p->nstrips = 0;
    const int sw = p->nd == 2 && p->col_interp == 1 ? mrb::interp_strip_width(p->G[0]) : 0;
    if (sw > 0 && p->G[1] >= sw + 3) {
      const int nstrips = (p->G[1] + sw - 1) / sw;
      const long long n = (long long)p->B * p->K;
      MRB_REQUIRE(n < (1LL << 31) && (long long)p->B * nstrips < (1LL << 31), "too many samples for strip lists");
      int nkeys = p->B * nstrips;
      int eb = 1;
      while ((1LL << eb) <= nkeys) ++eb;
      DevBuf sk, sks, sv;
      if ((rc = sk.ensure(n * sizeof(unsigned)))) return rc;
      if ((rc = sks.ensure(n * sizeof(unsigned)))) return rc;
      if ((rc = sv.ensure(n * sizeof(int)))) return rc;
      if ((rc = p->strip_entries.ensure(n * sizeof(int)))) return rc;
      if ((rc = p->strip_start.ensure(((size_t)nkeys + 1) * sizeof(int)))) return rc;
      strip_key_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(p->gx.as<float>(), sk.as<unsigned>(), sv.as<int>(), p->K,
                                                             p->B, p->G[1], sw, nstrips);
      MRB_LAUNCH_CHECK();
      size_t tb3 = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, tb3, sk.as<unsigned>(), sks.as<unsigned>(), sv.as<int>(),
                                      p->strip_entries.as<int>(), (int)n, 0, eb, st);
      if ((rc = p->tmp.ensure(tb3))) return rc;
      cub::DeviceRadixSort::SortPairs(p->tmp.p, tb3, sk.as<unsigned>(), sks.as<unsigned>(), sv.as<int>(),
                                      p->strip_entries.as<int>(), (int)n, 0, eb, st);
      tile_start_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(sks.as<unsigned>(), n, p->strip_start.as<int>(), nkeys);
      MRB_LAUNCH_CHECK();
      MRB_CUDA_TRY(cudaStreamSynchronize(st));   // the temporaries are freed on return
      p->nstrips = nstrips;
    }
    p->adj_zero = false;   // the supports changed: the spread grid is zeroed again before its next use
    MRB_LAUNCH_CHECK();
    unsigned long long touched = 0;
    MRB_CUDA_TRY(cudaMemcpyAsync(&touched, cntd.p, sizeof(touched), cudaMemcpyDeviceToHost, st));
    MRB_CUDA_TRY(cudaStreamSynchronize(st));
    p->touched = (int64_t)touched;
  }
  MRB_CUDA_TRY(cudaStreamSynchronize(st));
  p->have_points = true;
  return 0;
}

extern "C" int mrb_plan_set_dcf(mrb_plan* p, const float* dcf, int mode, int apply_fwd, int apply_adj,
                                mrb_stream_t stream) {
  MRB_REQUIRE(p != nullptr, "null plan");
  MRB_REQUIRE(mode >= 0 && mode <= 2, "bad dcf mode %d", mode);
  cudaStream_t st = (cudaStream_t)stream;
  p->has_wfwd = p->has_wadj = false;
  if (!dcf || mode == MRB_DCF_NONE) return 0;
  long long n = (long long)p->B * p->K;
  int rc;
  if (mode == MRB_DCF_BALANCED) {
    if ((rc = p->wfwd.ensure(n * sizeof(float)))) return rc;
    dcf_weight_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(dcf, p->wfwd.as<float>(), n, 1);
    if ((rc = p->wadj.ensure(n * sizeof(float)))) return rc;
    dcf_weight_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(dcf, p->wadj.as<float>(), n, 1);
    p->has_wfwd = p->has_wadj = true;
  } else {
    if (apply_fwd) {
      if ((rc = p->wfwd.ensure(n * sizeof(float)))) return rc;
      dcf_weight_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(dcf, p->wfwd.as<float>(), n, 0);
      p->has_wfwd = true;
    }
    if (apply_adj) {
      if ((rc = p->wadj.ensure(n * sizeof(float)))) return rc;
      dcf_weight_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(dcf, p->wadj.as<float>(), n, 0);
      p->has_wadj = true;
    }
  }
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_plan_set_maps(mrb_plan* p, const void* maps, mrb_stream_t stream) {
  MRB_REQUIRE(p != nullptr && maps != nullptr, "null plan or maps");
  size_t bytes = (size_t)p->C * p->stot() * sizeof(float2);
  int rc;
  if ((rc = p->maps.ensure(bytes))) return rc;
  MRB_CUDA_TRY(cudaMemcpyAsync(p->maps.p, maps, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  p->have_maps = true;
  return 0;
}

static int ensure_grid(mrb_plan* p, int nb, cudaStream_t st) {
  size_t bytes = (size_t)nb * p->C * p->gtot() * sizeof(float2);
  int rc = p->grid.ensure(bytes);
  if (rc) return rc;
  if (p->fft_mode == 1 && p->grid_mask == 1) {
    if (p->grid_adj.bytes < bytes) {
      if ((rc = p->grid_adj.ensure(bytes))) return rc;
      p->adj_zero = false;
    }
    if (p->adj_nb != nb) p->adj_zero = false;
    p->adj_nb = nb;
    if (!p->adj_zero) {
      // once per trajectory and size, in stream order: afterwards the spread
      // only ever writes cell pairs inside the supports.  Inside a stream
      // capture the fill becomes part of the graph (run on every replay).
      MRB_CUDA_TRY(cudaMemsetAsync(p->grid_adj.p, 0, p->grid_adj.bytes, st));
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      MRB_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
      if (cs == cudaStreamCaptureStatusNone) p->adj_zero = true;
    }
  }
  if (p->fft_mode == 1 && p->nd == 3) {
    const size_t vol = (size_t)nb * p->C * sizeof(float2);
    if ((rc = p->band.ensure(vol * p->S[0] * p->S[1] * p->G[2]))) return rc;
    if ((rc = p->band2.ensure(vol * p->S[0] * p->G[1] * p->G[2]))) return rc;
    if (p->il && (rc = p->grid_il.ensure(bytes))) return rc;
    return 0;
  }
  if (p->fft_mode == 1) return p->band.ensure(mrb::fft2_tmp_bytes(p->S[0], p->G[1], p->C, nb));
  if (p->il && p->nd == 3 && (rc = p->grid_il.ensure(bytes))) return rc;
  return ensure_fft(p, nb);
}

// fused 3D mode with the interleaved interp: the x column pass writes the
// (cell, coil) copy itself, the interp stage needs no transpose
static bool il_direct(const mrb_plan* p) {
  return p->fft_mode == 1 && p->nd == 3 && p->il == 1 && mrb::fft2_columns_il_supported(p->G[0], p->C);
}

// the forward column pass also interpolates (fused 2D mode with strip lists)
static bool col_interp_active(const mrb_plan* p) {
  return p->fft_mode == 1 && p->nd == 2 && p->col_interp == 1 && p->nstrips > 0;
}

// fused 2D mode with the interleaved interp (coil counts divisible by 4): the
// forward column pass writes the grid in coil quads (cell, 4 coils) and the
// interp gathers coil pairs with 128-bit loads
static bool il2_active(const mrb_plan* p) {
  return p->fft_mode == 1 && p->nd == 2 && p->il == 1 && p->C % 4 == 0 && p->C <= 512 && !col_interp_active(p);
}

// fused 2D mode with the pair-parallel interp on a planar-coil grid: the
// forward column pass stores each coil-frame's grid in blocks of 2 x 8 cells
// (one 128-byte line each), where a sample's 4 x 4 taps meet 2 to 6 lines
// instead of 4 to 8 lines of 16 cells of a row
static bool grid_blocked(const mrb_plan* p) {
  return p->fft_mode == 1 && p->nd == 2 && p->grid_blk == 1 && p->interp_mode == 1 && !il2_active(p) &&
         !col_interp_active(p) && p->G[0] % 2 == 0 && p->G[1] % 8 == 0;
}

// the spread writes only touched cell pairs into a grid of its own (fused FFT mode)
static bool spread_masked(const mrb_plan* p) {
  return p->fft_mode == 1 && p->grid_mask == 1 && p->touch.p != nullptr && p->adj_zero;
}

// the grid the spread writes and the adjoint column pass reads
static float2* adj_grid(mrb_plan* p) { return spread_masked(p) ? p->grid_adj.as<float2>() : p->grid.as<float2>(); }

// raise a kernel's dynamic shared-memory limit once per (kernel, size)
static int ensure_smem(const void* fn, size_t smem) {
  static const void* fns[32];
  static size_t set[32];
  static int n = 0;
  if (smem <= 48 * 1024) return 0;
  int i = 0;
  while (i < n && fns[i] != fn) ++i;
  if (i < n && set[i] >= smem) return 0;
  MRB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (i == n && n < 32) fns[n++] = fn;
  if (i < n) set[i] = smem;
  return 0;
}

// spread launch of a selected variant; every variant takes (SpreadArgs, Geo, TileGeo, KBPoly)
using SpreadKern = void (*)(SpreadArgs, Geo, TileGeo, KBPoly);
using SpreadGo = int (*)(SpreadKern, int, int, size_t, cudaStream_t, const SpreadArgs&, const Geo&, const TileGeo&,
                         const KBPoly&);

// variants written as bodies (group.cuh): recordable, K::NT threads
template <class K>
static int spread_go(SpreadKern fn, int blocks, int, size_t smem, cudaStream_t st, const SpreadArgs& a, const Geo& g,
                     const TileGeo& tg, const KBPoly& kb) {
  return mrb::launch<K>(fn, dim3(blocks), smem, st, a, g, tg, kb);
}

// the 3D block variants: plain launches
static int spread_go_plain(SpreadKern fn, int blocks, int threads, size_t smem, cudaStream_t st, const SpreadArgs& a,
                           const Geo& g, const TileGeo& tg, const KBPoly& kb) {
  SpreadArgs a2 = a;
  Geo g2 = g;
  TileGeo tg2 = tg;
  KBPoly kb2 = kb;
  void* args[] = {&a2, &g2, &tg2, &kb2};
  MRB_CUDA_TRY(cudaLaunchKernel((const void*)fn, dim3(blocks), dim3(threads), args, smem, st));
  MRB_LAUNCH_CHECK();
  return 0;
}

// one stage of the forward/adjoint pipeline; x/y are the user image / samples
static int run_stage(mrb_plan* p, int stage, const void* x, void* y, int nb, cudaStream_t st, int coil_images) {
  Geo g = make_geo(p);
  if (p->fft_mode == 1 && p->nd == 3) {
    // fused 3D passes on (vol, x, y, z): 0 = SENSE/deapod/pad + z transforms of
    // the S0*S1 image rows -> band (vol, S0, S1, G2); 1 = input-pruned y
    // transforms (the y columns of each (vol, x) slab) -> band2 (vol, S0, G1, G2),
    // then input-pruned x transforms (band2 as S0 rows of G1*G2 columns) -> grid;
    // 4 and 5 the same in reverse, output-pruned, with crop, deapodisation and
    // the conj(S_c) coil sum in the z pass
    const float* rowfac = p->rowfac.as<float>();
    const float* coldeap = p->invdeap.as<float>() + p->S[0] + p->S[1];
    const int R = p->S[0] * p->S[1];
    const int GG = p->G[1] * p->G[2];
    MRB_REQUIRE((long long)p->C * p->S[0] < (1LL << 31), "too many coil slabs");
    float2* b1 = p->band.as<float2>();
    float2* b2 = p->band2.as<float2>();
    int rc3;
    if (stage == 0)
      return mrb::fft2_forward_rows(x, p->maps.as<float2>(), rowfac, coldeap, b1, p->tw2p, R, p->S[2], R, p->G[2],
                                    p->C, nb, coil_images, p->skip, st);
    if (stage == 1) {
      if ((rc3 = mrb::fft2_columns(1, b1, b2, p->tw1p, p->S[1], p->S[2], p->G[1], p->G[2], p->C * p->S[0], nb,
                                   p->skip, st)))
        return rc3;
      if (il_direct(p))
        return mrb::fft2_columns_il(b2, p->grid_il.as<float2>(), p->tw0p, p->S[0], p->G[0], GG, p->C, nb, p->skip,
                                    st);
      return mrb::fft2_columns(1, b2, p->grid.as<float2>(), p->tw0p, p->S[0], GG, p->G[0], GG, p->C, nb, p->skip,
                               st);
    }
    if (stage == 4) {
      if ((rc3 = mrb::fft2_columns(0, adj_grid(p), b2, p->tw0p, p->S[0], GG, p->G[0], GG, p->C, nb, p->skip, st)))
        return rc3;
      return mrb::fft2_columns(0, b2, b1, p->tw1p, p->S[1], p->S[2], p->G[1], p->G[2], p->C * p->S[0], nb, p->skip,
                               st);
    }
    if (stage == 5)
      return mrb::fft2_adjoint_rows(b1, p->maps.as<float2>(), rowfac, coldeap, (void*)x, p->tw2p, R, p->S[2], R,
                                    p->G[2], p->C, nb, p->scale, p->skip, st);
  }
  if (p->fft_mode == 1) {
    // fused passes: 0 = SENSE/deapod/pad + row FFTs, 1 = column FFTs,
    // 4 = inverse column FFTs, 5 = inverse row FFTs + crop/deapod/coil sum
    if (stage == 0)
      return mrb::fft2_forward_rows(x, p->maps.as<float2>(), p->rowfac.as<float>(), p->invdeap.as<float>() + p->S[0],
                                    p->band.as<float2>(), p->tw1p, p->S[0], p->S[1], p->G[0], p->G[1], p->C, nb,
                                    coil_images, p->skip, st);
    if (stage == 1 && y != nullptr && col_interp_active(p)) {
      mrb::ColInterp ci{};
      ci.gx = p->gx.as<float>();
      ci.wfwd = p->has_wfwd ? p->wfwd.as<float>() : nullptr;
      ci.strip_start = p->strip_start.as<int>();
      ci.strip_entries = p->strip_entries.as<int>();
      ci.y = (float2*)y;
      ci.K = p->K;
      ci.B = p->B;
      ci.nb = nb;
      ci.nstrips = p->nstrips;
      ci.scale = p->scale * p->gsign;
      ci.kb = p->kb;
      return mrb::fft2_columns_interp(p->band.as<float2>(), p->tw0p, p->S[0], p->S[1], p->G[0], p->G[1], p->C, nb,
                                      ci, p->skip, st);
    }
    if (stage == 1 && il2_active(p))
      return mrb::fft2_columns_cg(p->band.as<float2>(), p->grid.as<float2>(), p->tw0p, p->S[0], p->S[1], p->G[0],
                                  p->G[1], p->C, nb, p->skip, st);
    if (stage == 1)
      return mrb::fft2_columns(1, p->band.as<float2>(), p->grid.as<float2>(), p->tw0p, p->S[0], p->S[1], p->G[0],
                               p->G[1], p->C, nb, p->skip, st, grid_blocked(p) ? 1 : 0);
    if (stage == 4)
      return mrb::fft2_columns(0, adj_grid(p), p->band.as<float2>(), p->tw0p, p->S[0], p->S[1], p->G[0],
                               p->G[1], p->C, nb, p->skip, st);
    if (stage == 5)
      return mrb::fft2_adjoint_rows(p->band.as<float2>(), p->maps.as<float2>(), p->rowfac.as<float>(),
                                    p->invdeap.as<float>() + p->S[0], (void*)x, p->tw1p, p->S[0], p->S[1], p->G[0],
                                    p->G[1], p->C, nb, p->scale, p->skip, st);
  }
  if (stage == 0) {
    const int Gl = p->G[p->nd - 1];
    const long long nvol = (long long)nb * p->C;
    dim3 blk(128);
    dim3 grd((Gl / 2 + 127) / 128, p->nd == 2 ? p->G[0] : p->G[1],
             (unsigned)(p->nd == 2 ? nvol : nvol * p->G[0]));
    MRB_REQUIRE(grd.z <= 65535, "too many coil volumes in one call (%u)", grd.z);
    if (p->nd == 2)
      pre_fft_kernel<2><<<grd, blk, 0, st>>>(
          (const float2*)x, p->maps.as<float2>(), p->invdeap.as<float>(), p->grid.as<float4>(), g, nb, coil_images);
    else
      pre_fft_kernel<3><<<grd, blk, 0, st>>>(
          (const float2*)x, p->maps.as<float2>(), p->invdeap.as<float>(), p->grid.as<float4>(), g, nb, coil_images);
    MRB_LAUNCH_CHECK();
    return 0;
  }
  if (stage == 1 || stage == 4) {
    // a library transform cannot be recorded: it would run ahead of the recorded launches
    MRB_REQUIRE(!mrb::group_recording(), "the cuFFT mode cannot run inside a grouped recording");
    cufftResult r = cufftSetStream(p->fft, st);
    if (r == CUFFT_SUCCESS)
      r = cufftExecC2C(p->fft, p->grid.as<cufftComplex>(), p->grid.as<cufftComplex>(),
                       stage == 1 ? CUFFT_FORWARD : CUFFT_INVERSE);
    if (r != CUFFT_SUCCESS) return mrb::fail(MRB_ECUFFT, "cufftExecC2C failed (%d)", (int)r);
    return 0;
  }
  if (stage == 2) {
    InterpArgs a{};
    a.grid = p->grid.as<float2>();
    a.gx = p->gx.as<float>();
    a.wfwd = p->has_wfwd ? p->wfwd.as<float>() : nullptr;
    a.order = nullptr;
    a.y = (float2*)y;
    a.nb = nb;
    a.scale = p->scale;
    a.gsign = p->gsign;
    if (p->il && p->nd == 3) {
      MRB_REQUIRE(nb <= 65535, "too many frames in one call");
      MRB_REQUIRE(p->gtot() * p->C < (1LL << 31), "interleaved grid of one frame exceeds 2^31 elements");
      if (!il_direct(p)) {   // else the x column pass wrote the interleaved copy
        const long long tb = (p->gtot() + TR_CELLS - 1) / TR_CELLS;
        MRB_REQUIRE(tb < (1LL << 31), "grid too large for the coil transpose");
        coil_interleave_kernel<<<dim3((unsigned)tb, nb), 256, 0, st>>>(p->grid.as<float2>(), p->grid_il.as<float2>(),
                                                                       p->gtot(), p->C, p->skip);
        MRB_LAUNCH_CHECK();
      }
      a.grid = p->grid_il.as<float2>();
      a.seg = p->nseg > 0 && p->interp_mode == 1 ? p->seg_order.as<int>() : nullptr;
      a.nseg = p->nseg;
      const long long nt = (a.seg ? p->nseg * IL_SEG : p->K) * ((p->C + 1) / 2);
      MRB_REQUIRE((nt + 255) / 256 < (1LL << 31), "too many samples for the interleaved interp");
      dim3 grid(grid_blocks(nt, 256), nb);
      if (p->C % 2 == 0) interp3_il_kernel<true><<<grid, 256, 0, st>>>(a, g, p->kb);
      else interp3_il_kernel<false><<<grid, 256, 0, st>>>(a, g, p->kb);
      MRB_LAUNCH_CHECK();
      return 0;
    }
    if (il2_active(p)) {
      const int S = 256 / ((p->C + 1) / 2);
      const long long nbx = (p->K + S - 1) / S;
      MRB_REQUIRE(nbx < (1LL << 31) && nb <= 65535, "too many samples for the interp");
      return mrb::launch<Interp2Quad>(interp2_il_kernel, dim3((unsigned)nbx, nb), 0, st, a, g, p->kb);
    }
    if (p->nd == 2 && p->interp_mode == 1) {
      a.blk = grid_blocked(p) ? 1 : 0;
      a.tapw = p->tap_table ? p->tapw.as<float4>() : nullptr;
      a.tapb = p->tap_table ? p->tapb.as<int2>() : nullptr;
      const long long nbx = (long long)grid_blocks(p->K, 256) * ((p->C + 1) / 2);
      MRB_REQUIRE(nbx < (1LL << 31) && nb <= 65535, "too many samples for the interp");
      return mrb::launch<Interp2p>(interp2p_kernel, dim3((unsigned)nbx, nb), 0, st, a, g, p->kb);
    }
    dim3 grid(grid_blocks(p->K, 256), nb);
    if (p->nd == 2) return mrb::launch<InterpGen<2>>(interp_kernel<2>, grid, 0, st, a, g, p->kb);
    return mrb::launch<InterpGen<3>>(interp_kernel<3>, grid, 0, st, a, g, p->kb);
  }
  if (stage == 3) {
    TileGeo tg{};
    tg.T = p->tile;
    tg.ntiles = p->ntiles;
    for (int d = 0; d < 3; ++d) tg.nt[d] = p->ntile_d[d];
    tg.lo_off = p->W / 2 - 1;
    tg.hi_off = p->W / 2;
    SpreadArgs a{};
    a.y = (const float2*)y;
    a.gx = p->gx.as<float>();
    a.wadj = p->has_wadj ? p->wadj.as<float>() : nullptr;
    a.entries = p->entries.as<int>();
    a.tile_start = p->tile_start.as<int>();
    a.items = p->items.as<int4>();
    a.n_items = p->n_items;
    a.chunk = p->chunk;
    a.n_slots = p->n_slots;
    a.grid = p->grid.as<float2>();
    const int reps = p->B == 1 ? nb : nb / p->B;
    if (p->n_slots > 0) {
      int rc2 = p->partials.ensure((size_t)reps * p->n_slots * p->C * (p->nd == 2 ? tg.T * tg.T : tg.T * tg.T * tg.T) *
                                   sizeof(float2));
      if (rc2) return rc2;
    }
    a.partials = p->partials.as<float2>();
    a.nb = nb;
    // fused mode with the bitmaps: the spread has a grid of its own whose
    // cells outside every support were zeroed once; it stores only the cell
    // pairs that hold a touched cell and no zero tiles
    const bool masked = spread_masked(p);
    a.touch = masked ? p->touch.as<unsigned>() : nullptr;
    a.twords = p->twords;
    a.grid = adj_grid(p);
    a.tapw = p->nd == 2 && p->tap_table ? p->tapw.as<float4>() : nullptr;
    a.tapb = p->nd == 2 && p->tap_table ? p->tapb.as<int2>() : nullptr;
    const bool blk3t = p->spread_kernel == 2 && p->nd == 3 && tg.T == S3_T;  // shared-staging 3D kernel
    // block-per-tile kernels (the plain block kernel stages tile-relative bases: grid sides >= T + 3)
    const bool blk3 = (p->spread_kernel == 1 || blk3t) && p->nd == 3 && tg.T == S3_T &&
                      (blk3t || (p->G[0] >= S3_T + 3 && p->G[1] >= S3_T + 3 && p->G[2] >= S3_T + 3));
    const bool blk2 = p->spread_kernel == 1 && p->nd == 2 && tg.T == S2_T;
    a.cpi = blk3 || blk2 ? std::min(std::min(p->C, S3_CPB), p->coils_per_item) : p->coils_per_item;
    a.ngroups = (p->C + a.cpi - 1) / a.cpi;
    a.gsign = p->gsign;
    long long items = (long long)reps * p->n_items * a.ngroups;
    MRB_REQUIRE(items < (1LL << 31), "too many spread work items");
    int blocks = blk3 || blk2 ? (int)items : grid_blocks(items, SPREAD_WARPS);
    SpreadKern fn = nullptr;
    SpreadGo go = spread_go_plain;   // kernels without a grouped form
    size_t smem = 0;
    int threads = SPREAD_WARPS * 32;
    if (blk3t) {
      if (a.cpi > 8) {
        fn = spread3t_kernel<2>;
        smem = Spread3tSmem<2>::BYTES;
        threads = 2 * S3_WARPS * 32;
      } else {
        fn = spread3t_kernel<1>;
        smem = Spread3tSmem<1>::BYTES;
        threads = S3_WARPS * 32;
      }
    } else if (blk3) {
      const int pairs = (a.cpi + 1) / 2;
      threads = S3_WARPS * 32;
      if (pairs <= 2) {
        fn = spread3_kernel<2>;
        smem = Spread3Smem<2>::BYTES;
      } else if (pairs <= 4) {
        fn = spread3_kernel<4>;
        smem = Spread3Smem<4>::BYTES;
      } else {
        fn = spread3_kernel<8>;
        smem = Spread3Smem<8>::BYTES;
      }
    }
    if (blk2) {
      const int pairs = (a.cpi + 1) / 2;
      threads = S2_WARPS * 32;
      if (pairs <= 2) {
        fn = spread2_kernel<2>;
        go = spread_go<Spread2Block<2>>;
        smem = Spread2Smem<2>::BYTES;
      } else if (pairs <= 4) {
        fn = spread2_kernel<4>;
        go = spread_go<Spread2Block<4>>;
        smem = Spread2Smem<4>::BYTES;
      } else {
        fn = spread2_kernel<8>;
        go = spread_go<Spread2Block<8>>;
        smem = Spread2Smem<8>::BYTES;
      }
    }
    // 2D per-warp work items with option key 6 = 2: the tap-table kernel (coil
    // groups of up to 16); key 6 = 0 the kernel that evaluates every tap per lane task
#define MRB_SPREAD2W_CASE(T_)                                                                 \
  if (!fn && p->nd == 2 && tg.T == T_ && p->spread_kernel == 2 && a.cpi <= 16) {             \
    fn = spread2w_kernel<T_>;                                                                \
    go = spread_go<Spread2Taps<T_>>;                                                         \
    smem = SPREAD_WARPS * Spread2wSmem<T_>::warp_bytes(a.cpi);                               \
  }
    MRB_SPREAD2W_CASE(4)
    MRB_SPREAD2W_CASE(8)
    MRB_SPREAD2W_CASE(16)
    MRB_SPREAD2W_CASE(32)
#undef MRB_SPREAD2W_CASE
#define MRB_SPREAD_CASE(ND_, T_)                                                             \
  if (!fn && p->nd == ND_ && tg.T == T_) {                                                   \
    fn = spread_kernel<ND_, T_>;                                                             \
    go = spread_go<SpreadWarp<ND_, T_>>;                                                     \
    smem = SPREAD_WARPS * SpreadSmem<ND_, T_>::warp_bytes(a.cpi);                            \
  }
    MRB_SPREAD_CASE(2, 4)
    MRB_SPREAD_CASE(2, 8)
    MRB_SPREAD_CASE(2, 16)
    MRB_SPREAD_CASE(2, 32)
    MRB_SPREAD_CASE(3, 4)
    MRB_SPREAD_CASE(3, 8)
#undef MRB_SPREAD_CASE
    MRB_REQUIRE(fn != nullptr, "no spread kernel for nd=%d tile=%d", p->nd, tg.T);
    MRB_REQUIRE(smem <= 227 * 1024, "spread tile needs %zu bytes of shared memory", smem);
    if (int rc3 = ensure_smem((const void*)fn, smem)) return rc3;
    if (p->n_empty > 0 && !masked) {
      long long zbl = (long long)reps * p->n_empty;
      MRB_REQUIRE(zbl < (1LL << 31), "too many empty tiles");
      int zb = (int)zbl;
      const int* ek = p->empty_keys.as<int>();
      float2* gridp = a.grid;
      int rz = 0;
#define MRB_ZERO_CASE(ND_, T_)                                                                      \
  if (p->nd == ND_ && tg.T == T_)                                                                   \
    rz = mrb::launch<ZeroTiles<ND_, T_>>(zero_tiles_kernel<ND_, T_>, dim3(zb), 0, st, ek, p->n_empty, gridp, g, \
                                         tg, nb);
      MRB_ZERO_CASE(2, 4)
      MRB_ZERO_CASE(2, 8)
      MRB_ZERO_CASE(2, 16)
      MRB_ZERO_CASE(2, 32)
      MRB_ZERO_CASE(3, 4)
      MRB_ZERO_CASE(3, 8)
#undef MRB_ZERO_CASE
      if (rz) return rz;
    }
    if (items > 0) {
      if (int rs = go(fn, blocks, threads, smem, st, a, g, tg, p->kb)) return rs;
    }
    if (p->n_multi > 0) {
      MRB_REQUIRE(reps <= 65535 && p->C <= 65535, "too many frames for the split-tile reduction");
      dim3 rg(p->n_multi, p->C, reps);
      const float2* part = p->partials.as<float2>();
      const int4* mt = p->multi.as<int4>();
      float2* gridp = a.grid;
#define MRB_REDUCE_CASE(ND_, T_)                                                                      \
  if (p->nd == ND_ && tg.T == T_)                                                                     \
    return mrb::launch<SpreadReduce<ND_, T_>>(spread_reduce_kernel<ND_, T_>, rg, 0, st, part, mt, p->n_multi, \
                                              p->n_slots, gridp, g, tg, nb);
      MRB_REDUCE_CASE(2, 4)
      MRB_REDUCE_CASE(2, 8)
      MRB_REDUCE_CASE(2, 16)
      MRB_REDUCE_CASE(2, 32)
      MRB_REDUCE_CASE(3, 4)
      MRB_REDUCE_CASE(3, 8)
#undef MRB_REDUCE_CASE
      return mrb::fail(MRB_EINVAL, "no split-tile reduction for nd=%d tile=%d", p->nd, tg.T);
    }
    return 0;
  }
  if (stage == 5) {
    const int Sl = p->S[p->nd - 1];
    dim3 blk(128);
    dim3 grd((Sl + 127) / 128, p->nd == 2 ? p->S[0] : p->S[1],
             (unsigned)(p->nd == 2 ? (long long)nb : (long long)nb * p->S[0]));
    MRB_REQUIRE(grd.z <= 65535, "too many frames in one call");
    if (p->nd == 2)
      post_ifft_kernel<2><<<grd, blk, 0, st>>>(p->grid.as<float2>(), p->maps.as<float2>(), p->invdeap.as<float>(),
                                               (float2*)x, g, nb, p->scale);
    else
      post_ifft_kernel<3><<<grd, blk, 0, st>>>(p->grid.as<float2>(), p->maps.as<float2>(), p->invdeap.as<float>(),
                                               (float2*)x, g, nb, p->scale);
    MRB_LAUNCH_CHECK();
    return 0;
  }
  return mrb::fail(MRB_EINVAL, "unknown stage %d", stage);
}

static int forward_impl(mrb_plan* p, const void* x, void* y, int nb, cudaStream_t st, int coil_images) {
  int rc;
  if ((rc = check_ready(p))) return rc;
  if ((rc = check_nb(p, nb))) return rc;
  MRB_REQUIRE(x != nullptr && y != nullptr, "null x or y");
  if ((rc = ensure_grid(p, nb, st))) return rc;
  const bool fused_interp = col_interp_active(p);   // stage 1 interpolates as well
  for (int stage : {0, 1, 2}) {
    if (stage == 2 && fused_interp) break;
    if ((rc = run_stage(p, stage, x, y, nb, st, coil_images))) return rc;
  }
  return 0;
}

extern "C" int mrb_nufft_forward(mrb_plan* p, const void* x, void* y, int nb, mrb_stream_t stream) {
  return forward_impl(p, x, y, nb, (cudaStream_t)stream, 0);
}

extern "C" int mrb_nufft_forward_coils(mrb_plan* p, const void* x, void* y, int nb, mrb_stream_t stream) {
  return forward_impl(p, x, y, nb, (cudaStream_t)stream, 1);
}

extern "C" int mrb_nufft_adjoint(mrb_plan* p, const void* y, void* x, int nb, mrb_stream_t stream) {
  int rc;
  if ((rc = check_ready(p))) return rc;
  if ((rc = check_nb(p, nb))) return rc;
  MRB_REQUIRE(x != nullptr && y != nullptr, "null x or y");
  if ((rc = ensure_grid(p, nb, (cudaStream_t)stream))) return rc;
  for (int stage : {3, 4, 5})
    if ((rc = run_stage(p, stage, x, (void*)y, nb, (cudaStream_t)stream, 0))) return rc;
  return 0;
}

extern "C" int mrb_nufft_stage(mrb_plan* p, int stage, const void* x, void* y, int nb, mrb_stream_t stream) {
  int rc;
  if ((rc = check_ready(p))) return rc;
  if ((rc = check_nb(p, nb))) return rc;
  MRB_REQUIRE(stage >= 0 && stage <= 5, "stage must be 0..5");
  MRB_REQUIRE((stage == 1 || stage == 4) || (stage == 0 || stage == 5 ? x != nullptr : y != nullptr),
              "null x or y for stage %d", stage);
  if ((rc = ensure_grid(p, nb, (cudaStream_t)stream))) return rc;
  return run_stage(p, stage, x, y, nb, (cudaStream_t)stream, 0);
}

extern "C" int mrb_plan_info(mrb_plan* p, int64_t* out, int nout) {
  MRB_REQUIRE(p != nullptr && out != nullptr, "null plan or output");
  const int blk = (p->spread_kernel == 1 && ((p->nd == 2 && p->tile == S2_T) || (p->nd == 3 && p->tile == S3_T))) ||
                  (p->spread_kernel == 2 && p->nd == 3 && p->tile == S3_T);
  int64_t v[10] = {p->n_entries, p->ntiles,  p->touched, p->tile, p->coils_per_item, p->gtot(), p->fft_mode, blk,
                   col_interp_active(p), p->have_points ? 1 : 0};
  for (int i = 0; i < nout && i < 10; ++i) out[i] = v[i];
  return 0;
}

extern "C" int mrb_plan_set_toeplitz(mrb_plan* p, const float* psf, mrb_stream_t stream) {
  MRB_REQUIRE(p != nullptr && psf != nullptr, "null plan or transfer function");
  MRB_REQUIRE(p->nd == 2 && p->fft_mode == 1,
              "the Toeplitz normal operator needs a 2D plan in the fused FFT mode (compiled grid sizes)");
  const size_t bytes = (size_t)p->B * p->gtot() * sizeof(float);
  int rc;
  if ((rc = p->psf.ensure(bytes))) return rc;
  MRB_CUDA_TRY(cudaMemcpyAsync(p->psf.p, psf, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  if (!p->ones.p) {
    std::vector<float> one((size_t)p->S[0] + p->S[1], 1.f);
    const int off0 = p->G[0] / 2 - p->S[0] / 2;
    for (int r = 0; r < p->S[0]; ++r)
      if ((r + off0) & 1) one[r] = -1.f;   // the row sign the deapodisation table would carry
    if ((rc = p->ones.ensure(one.size() * sizeof(float)))) return rc;
    MRB_CUDA_TRY(cudaMemcpy(p->ones.p, one.data(), one.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  p->have_psf = true;
  return 0;
}

extern "C" int mrb_nufft_normal(mrb_plan* p, const void* x, void* out, int nb, mrb_stream_t stream) {
  int rc;
  if ((rc = check_ready(p))) return rc;
  if ((rc = check_nb(p, nb))) return rc;
  MRB_REQUIRE(x != nullptr && out != nullptr, "null x or out");
  if (!p->have_psf) return mrb::fail(MRB_ESTATE, "plan has no Toeplitz transfer function (mrb_plan_set_toeplitz)");
  if ((rc = ensure_grid(p, nb, (cudaStream_t)stream))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const float* one = p->ones.as<float>();
  float2* band = p->band.as<float2>();
  if ((rc = mrb::fft2_forward_rows(x, p->maps.as<float2>(), one, one + p->S[0], band, p->tw1p, p->S[0], p->S[1],
                                   p->G[0], p->G[1], p->C, nb, 0, p->skip, st)))
    return rc;
  if ((rc = mrb::fft2_toeplitz_columns(band, p->psf.as<float>(), p->tw0p, p->S[0], p->S[1], p->G[0], p->G[1], p->C,
                                       nb, p->B, p->skip, st)))
    return rc;
  return mrb::fft2_adjoint_rows(band, p->maps.as<float2>(), one, one + p->S[0], out, p->tw1p, p->S[0], p->S[1],
                                p->G[0], p->G[1], p->C, nb, 1.f, p->skip, st);
}

extern "C" int mrb_plan_set_skip_flag(mrb_plan* p, const double* flag) {
  MRB_REQUIRE(p != nullptr, "null plan");
  p->skip = flag;
  return 0;
}

extern "C" int mrb_plan_cell_base(mrb_plan* p, int32_t* out, mrb_stream_t stream) {
  MRB_REQUIRE(p != nullptr && out != nullptr, "null plan or output");
  if (!p->have_points) return mrb::fail(MRB_ESTATE, "plan has no trajectory");
  long long n = (long long)p->B * p->nd * p->K;
  cell_base_kernel<<<grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(p->gx.as<float>(), out, n);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_grid_indices(const float* traj, int nd, const int* G, int64_t K, int W, int convention,
                                int64_t* idx, mrb_stream_t stream) {
  MRB_REQUIRE(traj != nullptr && G != nullptr && idx != nullptr, "null pointer");
  MRB_REQUIRE(nd == 2 || nd == 3, "nd must be 2 or 3");
  MRB_REQUIRE(W >= 2 && W <= 16 && W % 2 == 0, "W must be even and <= 16");
  MRB_REQUIRE(convention == MRB_IDX_REFERENCE || convention == MRB_IDX_CORRECTED, "bad convention");
  for (int d = 0; d < nd; ++d) MRB_REQUIRE(G[d] >= 1, "bad grid");
  grid_index_kernel<<<grid_blocks(K, 128), 128, 0, (cudaStream_t)stream>>>(
      traj, nd, G[0], G[1], nd > 2 ? G[2] : 1, K, W, convention, (long long*)idx);
  MRB_LAUNCH_CHECK();
  return 0;
}
