// Learned warm start: BF16 2D+t convolutional network kernels (sm_100a).
//
// Activations are channels-last BF16 tensors (Nb, D, H, W, C) with D = frames,
// (H, W) = image; a tensor may hold several logical tensors side by side in its
// channel dimension (channel stride + offset), which makes U-Net skip
// concatenation free.  Gradients are FP32 in the same layout.
//
// conv3d (3x3x3, stride 1, zero padding 1) is an implicit GEMM on the tensor
// cores: M = output voxels, N = output channels, K = 27 taps x input channels,
// mma.sync m16n8k16 BF16 x BF16 -> FP32.  The data gradient is the same
// forward convolution with the tap-flipped, channel-transposed weights; the
// weight gradient is a GEMM over voxels split into fixed chunks whose partial
// sums are reduced in a fixed order (deterministic).
// No reference counterpart: the reference has no learned component.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "mrb_common.cuh"

namespace {

typedef __nv_bfloat16 bf16;

struct Vol {
  int Nb, D, H, W;
  __host__ __device__ long long voxels() const { return (long long)Nb * D * H * W; }
};

__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// ---------------------------------------------------------------------------
// forward convolution
// ---------------------------------------------------------------------------
constexpr int CBM = 64;    // voxels per CTA
constexpr int CBN = 32;    // output channels per CTA
constexpr int KST = 24;    // padded smem row (bf16) for conflict-free fragment loads

struct ConvArgs {
  const bf16* x;     // input (voxels, cx) channels [ci_off, ci_off + cin)
  int cx, ci_off, cin;
  const bf16* w;     // [27][cin][coutp]
  int coutp;         // padded output channels (multiple of 32)
  int cout;          // real output channels written
  const float* bias; // [coutp] or null
  int relu;
  bf16* yb;          // optional BF16 output (voxels, cyb) at offset yb_off
  int cyb, yb_off;
  float* yf;         // optional FP32 output (voxels, cyf) at offset yf_off
  int cyf, yf_off, yf_acc;
  Vol v;
};

__global__ void __launch_bounds__(128) conv3d_fwd_kernel(ConvArgs a) {
  __shared__ __align__(16) bf16 As[CBM][KST];
  __shared__ __align__(16) bf16 Bs[CBN][KST];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const long long M = a.v.voxels();
  const long long m0 = (long long)blockIdx.x * CBM;
  const int co0 = blockIdx.y * CBN;
  // this thread's A-load voxel and channel half
  const int am = tid >> 1, ah = tid & 1;
  const long long vox = m0 + am;
  int vn = 0, vd = 0, vh = 0, vw = 0;
  const bool vok = vox < M;
  if (vok) {
    long long r = vox;
    vw = (int)(r % a.v.W); r /= a.v.W;
    vh = (int)(r % a.v.H); r /= a.v.H;
    vd = (int)(r % a.v.D);
    vn = (int)(r / a.v.D);
  }
  float acc[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
  // B-load mapping: k = tid / 8, four output channels at (tid % 8) * 4
  const int bk = tid >> 3, bn = (tid & 7) * 4;
  for (int tap = 0; tap < 27; ++tap) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int nd = vd + dz, nh = vh + dy, nw = vw + dx;
    const bool inb = vok && (unsigned)nd < (unsigned)a.v.D && (unsigned)nh < (unsigned)a.v.H &&
                     (unsigned)nw < (unsigned)a.v.W;
    const long long nvox = (((long long)vn * a.v.D + nd) * a.v.H + nh) * a.v.W + nw;
    for (int ci0 = 0; ci0 < a.cin; ci0 += 16) {
      uint4 av = make_uint4(0u, 0u, 0u, 0u);
      if (inb) av = *reinterpret_cast<const uint4*>(a.x + nvox * a.cx + a.ci_off + ci0 + ah * 8);
      *reinterpret_cast<uint4*>(&As[am][ah * 8]) = av;
      const bf16* wp = a.w + ((long long)tap * a.cin + ci0 + bk) * a.coutp + co0 + bn;
      uint2 bv = *reinterpret_cast<const uint2*>(wp);
      const bf16* bb = reinterpret_cast<const bf16*>(&bv);
#pragma unroll
      for (int q = 0; q < 4; ++q) Bs[bn + q][bk] = bb[q];
      __syncthreads();
      const int r0 = warp * 16 + g;
      const uint32_t a0 = ld32(&As[r0][t4 * 2]), a1 = ld32(&As[r0 + 8][t4 * 2]);
      const uint32_t a2 = ld32(&As[r0][t4 * 2 + 8]), a3 = ld32(&As[r0 + 8][t4 * 2 + 8]);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t b0 = ld32(&Bs[j * 8 + g][t4 * 2]), b1 = ld32(&Bs[j * 8 + g][t4 * 2 + 8]);
        mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
      }
      __syncthreads();
    }
  }
  // epilogue
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const long long m = m0 + warp * 16 + g + half * 8;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int co = co0 + j * 8 + t4 * 2 + e;
        if (co >= a.cout) continue;
        float val = acc[j][half * 2 + e];
        if (a.bias) val += a.bias[co];
        if (a.relu) val = fmaxf(val, 0.f);
        if (a.yb) a.yb[m * a.cyb + a.yb_off + co] = __float2bfloat16_rn(val);
        if (a.yf) {
          float* p = a.yf + m * a.cyf + a.yf_off + co;
          *p = a.yf_acc ? *p + val : val;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// weight gradient: dW[tap][ci][co] = sum_v x[v + off(tap)][ci] * gz[v][co]
// grid (27, cin/32, coutp/32, nsplit); partials [split][27][cin][coutp]
// ---------------------------------------------------------------------------
struct WgradArgs {
  const bf16* x;
  int cx, ci_off, cin;
  const bf16* gz;
  int cg, cg_off, coutp;
  float* part;
  long long chunk;   // voxels per split
  Vol v;
};

__global__ void __launch_bounds__(128) conv3d_wgrad_kernel(WgradArgs a) {
  __shared__ __align__(16) bf16 As[32][KST];   // A[m = ci][k = voxel]
  __shared__ __align__(16) bf16 Bs[32][KST];   // B[n = co][k = voxel]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int tap = blockIdx.x % 27;
  const int split = blockIdx.x / 27;
  const int ci0 = blockIdx.y * 32, co0 = blockIdx.z * 32;
  const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const long long M = a.v.voxels();
  const long long v0 = (long long)split * a.chunk;
  const long long v1 = v0 + a.chunk < M ? v0 + a.chunk : M;
  const int mo = (warp >> 1) * 16, no = (warp & 1) * 16;
  float acc[2][4];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
  // loads: voxel k = tid / 8, 4 channels at (tid % 8) * 4
  const int lk = tid >> 3, lc = (tid & 7) * 4;
  for (long long vb = v0; vb < v1; vb += 16) {
    const long long vox = vb + lk;
    uint2 xa = make_uint2(0u, 0u), gb = make_uint2(0u, 0u);
    if (vox < v1) {
      long long r = vox;
      const int vw = (int)(r % a.v.W); r /= a.v.W;
      const int vh = (int)(r % a.v.H); r /= a.v.H;
      const int vd = (int)(r % a.v.D);
      const int vn = (int)(r / a.v.D);
      const int nd = vd + dz, nh = vh + dy, nw = vw + dx;
      if ((unsigned)nd < (unsigned)a.v.D && (unsigned)nh < (unsigned)a.v.H && (unsigned)nw < (unsigned)a.v.W) {
        const long long nv = (((long long)vn * a.v.D + nd) * a.v.H + nh) * a.v.W + nw;
        xa = *reinterpret_cast<const uint2*>(a.x + nv * a.cx + a.ci_off + ci0 + lc);
      }
      gb = *reinterpret_cast<const uint2*>(a.gz + vox * a.cg + a.cg_off + co0 + lc);
    }
    const bf16* xe = reinterpret_cast<const bf16*>(&xa);
    const bf16* ge = reinterpret_cast<const bf16*>(&gb);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      As[lc + q][lk] = xe[q];
      Bs[lc + q][lk] = ge[q];
    }
    __syncthreads();
    const uint32_t a0 = ld32(&As[mo + g][t4 * 2]), a1 = ld32(&As[mo + g + 8][t4 * 2]);
    const uint32_t a2 = ld32(&As[mo + g][t4 * 2 + 8]), a3 = ld32(&As[mo + g + 8][t4 * 2 + 8]);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint32_t b0 = ld32(&Bs[no + j * 8 + g][t4 * 2]), b1 = ld32(&Bs[no + j * 8 + g][t4 * 2 + 8]);
      mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
    }
    __syncthreads();
  }
  float* out = a.part + (((long long)split * 27 + tap) * a.cin + ci0) * a.coutp + co0;
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int half = 0; half < 2; ++half)
#pragma unroll
      for (int e = 0; e < 2; ++e)
        out[(long long)(mo + g + half * 8) * a.coutp + no + j * 8 + t4 * 2 + e] = acc[j][half * 2 + e];
}

// dW = sum over splits in order (and dbias from its own partials)
__global__ void sum_splits_kernel(const float* __restrict__ part, int nsplit, long long n, float* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int k = 0; k < nsplit; ++k) s += part[(long long)k * n + i];
  out[i] = s;
}

// bias gradient partials: one block per (split, 32 channels)
__global__ void bias_grad_kernel(const bf16* __restrict__ gz, int cg, int cg_off, int coutp, long long M,
                                 long long chunk, float* __restrict__ part) {
  const int split = blockIdx.x;
  const int co = blockIdx.y * 32 + (threadIdx.x & 31);
  const int row = threadIdx.x >> 5;
  const long long v0 = (long long)split * chunk, v1 = v0 + chunk < M ? v0 + chunk : M;
  float s = 0.f;
  for (long long v = v0 + row; v < v1; v += blockDim.x >> 5) s += __bfloat162float(gz[v * cg + cg_off + co]);
  __shared__ float sh[8][32];
  sh[row][threadIdx.x & 31] = s;
  __syncthreads();
  if (row == 0) {
    float t = 0.f;
    for (int r = 0; r < (int)(blockDim.x >> 5); ++r) t += sh[r][threadIdx.x & 31];
    part[(long long)split * coutp + co] = t;
  }
}

// Wd[tap][co][ci] = W[26 - tap][ci][co]  (data-gradient weights), both padded
__global__ void flip_weights_kernel(const bf16* __restrict__ w, int cin, int coutp, bf16* __restrict__ wd, int cinp) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = 27LL * coutp * cinp;
  if (i >= n) return;
  const int ci = (int)(i % cinp);
  const int co = (int)((i / cinp) % coutp);
  const int tap = (int)(i / ((long long)cinp * coutp));
  wd[i] = ci < cin ? w[((long long)(26 - tap) * cin + ci) * coutp + co] : __float2bfloat16_rn(0.f);
}

// gz = (act > 0 ? g : 0) in BF16 (ReLU backward), channel slices
__global__ void relu_bwd_kernel(const float* __restrict__ g, int cgs, int g_off, const bf16* __restrict__ act,
                                int cas, int a_off, int nch, long long M, bf16* __restrict__ gz, int czs, int z_off,
                                int nchp) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * nchp) return;
  const long long v = i / nchp;
  const int c = (int)(i % nchp);
  float val = 0.f;
  if (c < nch) {
    const bool on = act ? __bfloat162float(act[v * cas + a_off + c]) > 0.f : true;
    val = on ? g[v * cgs + g_off + c] : 0.f;
  }
  gz[v * czs + z_off + c] = __float2bfloat16_rn(val);
}

// 2x2 average pool over (H, W); out (Nb, D, H/2, W/2, c)
__global__ void pool2_fwd_kernel(const bf16* __restrict__ x, int cx, int x_off, int nch, Vol vi, bf16* __restrict__ y,
                                 int cy, int y_off) {
  const int Ho = vi.H / 2, Wo = vi.W / 2;
  long long n = (long long)vi.Nb * vi.D * Ho * Wo * nch;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = (int)(i % nch);
  long long r = i / nch;
  const int wo = (int)(r % Wo); r /= Wo;
  const int ho = (int)(r % Ho); r /= Ho;
  const long long nd = r;                       // (n, d) flattened
  float s = 0.f;
#pragma unroll
  for (int dy = 0; dy < 2; ++dy)
#pragma unroll
    for (int dxx = 0; dxx < 2; ++dxx) {
      const long long v = (nd * vi.H + 2 * ho + dy) * vi.W + 2 * wo + dxx;
      s += __bfloat162float(x[v * cx + x_off + c]);
    }
  const long long vo = (nd * Ho + ho) * Wo + wo;
  y[vo * cy + y_off + c] = __float2bfloat16_rn(0.25f * s);
}

// pool backward: gx (fine, FP32, accumulate) += 0.25 * gy (coarse, FP32)
__global__ void pool2_bwd_kernel(const float* __restrict__ gy, int cgy, int gy_off, int nch, Vol vi,
                                 float* __restrict__ gx, int cgx, int gx_off) {
  long long n = vi.voxels() * nch;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = (int)(i % nch);
  long long r = i / nch;
  const int w = (int)(r % vi.W); r /= vi.W;
  const int h = (int)(r % vi.H); r /= vi.H;
  const long long vo = (r * (vi.H / 2) + h / 2) * (vi.W / 2) + w / 2;
  const long long v = (r * vi.H + h) * vi.W + w;
  gx[v * cgx + gx_off + c] += 0.25f * gy[vo * cgy + gy_off + c];
}

// nearest 2x upsample over (H, W): out (Nb, D, 2H, 2W) from coarse vi
__global__ void up2_fwd_kernel(const bf16* __restrict__ x, int cx, int x_off, int nch, Vol vi, bf16* __restrict__ y,
                               int cy, int y_off) {
  const int Ho = vi.H * 2, Wo = vi.W * 2;
  long long n = (long long)vi.Nb * vi.D * Ho * Wo * nch;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = (int)(i % nch);
  long long r = i / nch;
  const int wo = (int)(r % Wo); r /= Wo;
  const int ho = (int)(r % Ho); r /= Ho;
  const long long v = (r * vi.H + ho / 2) * vi.W + wo / 2;
  y[((r * Ho + ho) * Wo + wo) * cy + y_off + c] = x[v * cx + x_off + c];
}

// upsample backward: gx (coarse, FP32, overwrite) = sum of the 4 fine gradients
__global__ void up2_bwd_kernel(const float* __restrict__ gy, int cgy, int gy_off, int nch, Vol vi,
                               float* __restrict__ gx, int cgx, int gx_off) {
  long long n = vi.voxels() * nch;          // coarse
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = (int)(i % nch);
  long long r = i / nch;
  const int w = (int)(r % vi.W); r /= vi.W;
  const int h = (int)(r % vi.H); r /= vi.H;
  const int Wf = vi.W * 2, Hf = vi.H * 2;
  float s = 0.f;
#pragma unroll
  for (int dy = 0; dy < 2; ++dy)
#pragma unroll
    for (int dxx = 0; dxx < 2; ++dxx) s += gy[((r * Hf + 2 * h + dy) * Wf + 2 * w + dxx) * cgy + gy_off + c];
  gx[((r * vi.H + h) * vi.W + w) * cgx + gx_off + c] = s;
}

// The same three data movements with 16-byte accesses: a thread moves 8
// channels (one uint4) of one voxel, a block row covers one image row, and the
// voxel index is rebuilt with 32-bit arithmetic from the row (blockIdx.y, grid-
// strided).  For channel counts, strides and offsets that are multiples of 8
// (16-byte aligned rows); 1 << lg8 = channels / 8.  Same values as the
// element kernels above (pooling sums in the same order).
__device__ __forceinline__ void bf16x8_to_f32(const uint4& u, float* f) {
  const bf16* h = reinterpret_cast<const bf16*>(&u);
#pragma unroll
  for (int k = 0; k < 8; ++k) f[k] = __bfloat162float(h[k]);
}

// nearest 2x upsample over (H, W): fine row `row` of (Nb, D, 2H) rows
__global__ void up2_fwd_vec_kernel(const bf16* __restrict__ x, int cx, int x_off, int lg8, Vol vi,
                                   bf16* __restrict__ y, int cy, int y_off) {
  const int Ho = vi.H * 2, Wo = vi.W * 2;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (Wo << lg8)) return;
  const int wo = e >> lg8, c = (e & ((1 << lg8) - 1)) * 8;
  const int rows = vi.Nb * vi.D * Ho;
  for (int row = blockIdx.y; row < rows; row += gridDim.y) {
    const int nd = row / Ho, ho = row - nd * Ho;
    const long long src = (((long long)nd * vi.H + ho / 2) * vi.W + wo / 2) * cx + x_off + c;
    const long long dst = ((long long)row * Wo + wo) * cy + y_off + c;
    *reinterpret_cast<uint4*>(y + dst) = __ldg(reinterpret_cast<const uint4*>(x + src));
  }
}

// 2x2 average pool over (H, W): coarse row `row` of (Nb, D, H/2) rows
__global__ void pool2_fwd_vec_kernel(const bf16* __restrict__ x, int cx, int x_off, int lg8, Vol vi,
                                     bf16* __restrict__ y, int cy, int y_off) {
  const int Ho = vi.H / 2, Wo = vi.W / 2;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (Wo << lg8)) return;
  const int wo = e >> lg8, c = (e & ((1 << lg8) - 1)) * 8;
  const int rows = vi.Nb * vi.D * Ho;
  for (int row = blockIdx.y; row < rows; row += gridDim.y) {
    const int nd = row / Ho, ho = row - nd * Ho;
    float s[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] = 0.f;
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dxx = 0; dxx < 2; ++dxx) {
        const long long v = ((long long)nd * vi.H + 2 * ho + dy) * vi.W + 2 * wo + dxx;
        float f[8];
        bf16x8_to_f32(__ldg(reinterpret_cast<const uint4*>(x + v * cx + x_off + c)), f);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] += f[k];
      }
    uint4 out;
    bf16* h = reinterpret_cast<bf16*>(&out);
#pragma unroll
    for (int k = 0; k < 8; ++k) h[k] = __float2bfloat16_rn(0.25f * s[k]);
    *reinterpret_cast<uint4*>(y + ((long long)row * Wo + wo) * cy + y_off + c) = out;
  }
}

// complex -> channels-last BF16 with cx % 8 == 0: frame `fr` = blockIdx.y (grid-strided) of Nb * D
__global__ void pack_vec_kernel(const float2* __restrict__ z, const float* __restrict__ scale, Vol v,
                                bf16* __restrict__ x, int cx) {
  const int hw = v.H * v.W;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= hw) return;
  const int frames = v.Nb * v.D;
  for (int fr = blockIdx.y; fr < frames; fr += gridDim.y) {
    const long long vox = (long long)fr * hw + p;
    const float sc = scale[fr / v.D];
    const float2 zz = z[vox];
    uint4 first = make_uint4(0u, 0u, 0u, 0u);
    bf16* h = reinterpret_cast<bf16*>(&first);
    h[0] = __float2bfloat16_rn(zz.x * sc);
    h[1] = __float2bfloat16_rn(zz.y * sc);
    uint4* dst = reinterpret_cast<uint4*>(x + vox * cx);
    dst[0] = first;
    for (int k = 1; k < cx / 8; ++k) dst[k] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// complex (Nb, D, H, W) -> channels-last BF16 (.., cx) channels 0/1 = re/im * scale[n], rest zero
__global__ void pack_kernel(const float2* __restrict__ z, const float* __restrict__ scale, Vol v, bf16* __restrict__ x,
                            int cx) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long M = v.voxels();
  if (i >= M * cx) return;
  const long long vox = i / cx;
  const int c = (int)(i % cx);
  const int n = (int)(vox / ((long long)v.D * v.H * v.W));
  float val = 0.f;
  if (c < 2) {
    float2 zz = z[vox];
    val = (c == 0 ? zz.x : zz.y) * scale[n];
  }
  x[i] = __float2bfloat16_rn(val);
}

// out = (x_in + net) / scale[n] as complex; net is FP32 (.., cy) channels 0/1
__global__ void unpack_kernel(const float2* __restrict__ zin, const float* __restrict__ net, int cy,
                              const float* __restrict__ scale, Vol v, float2* __restrict__ zout) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.voxels()) return;
  const int n = (int)(i / ((long long)v.D * v.H * v.W));
  const float s = 1.f / scale[n];
  float2 a = zin[i];
  zout[i] = make_float2(a.x + net[i * cy] * s, a.y + net[i * cy + 1] * s);
}

// loss = sum |x_in*scale + net - target*scale|^2 / count ; grad (FP32, .., cy) = 2 (pred - target) / count
__global__ void mse_kernel(const float2* __restrict__ zin, const float2* __restrict__ target,
                           const float* __restrict__ net, int cy, const float* __restrict__ scale, Vol v,
                           float inv_count, float* __restrict__ grad, double* __restrict__ loss_part) {
  __shared__ double sh[256];
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < v.voxels()) {
    const int n = (int)(i / ((long long)v.D * v.H * v.W));
    const float s = scale[n];
    float2 a = zin[i], t = target[i];
    const float er = a.x * s + net[i * cy] - t.x * s;
    const float ei = a.y * s + net[i * cy + 1] - t.y * s;
    l = (double)(er * er + ei * ei) * inv_count;
    grad[i * cy] = 2.f * er * inv_count;
    grad[i * cy + 1] = 2.f * ei * inv_count;
    for (int c = 2; c < cy; ++c) grad[i * cy + c] = 0.f;
  }
  sh[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = sh[0];
}

__global__ void sum_double_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += part[i];
  *out = s;
}

// Adam (Kingma & Ba 2015) on FP32 master weights; refreshes the BF16 copy.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps,
                            float bc1, float bc2, bf16* __restrict__ wb) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ a, long long n, bf16* __restrict__ b) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

Vol mkvol(const int* v) { return Vol{v[0], v[1], v[2], v[3]}; }

}  // namespace

// ===========================================================================
// C ABI (learned warm start; no counterpart in the reference)
// ===========================================================================
extern "C" int mrb_cnn_conv3d_fwd(const void* x, int cx, int ci_off, int cin, const void* w, int coutp, int cout,
                                  const float* bias, int relu, void* yb, int cyb, int yb_off, float* yf, int cyf,
                                  int yf_off, int yf_acc, const int* vol, mrb_stream_t stream) {
  MRB_REQUIRE(x && w && vol && (yb || yf), "null pointer");
  MRB_REQUIRE(cin > 0 && cin % 16 == 0, "cin must be a positive multiple of 16");
  MRB_REQUIRE(coutp > 0 && coutp % 32 == 0 && cout <= coutp, "coutp must be a multiple of 32 >= cout");
  MRB_REQUIRE(cx % 8 == 0 && ci_off % 8 == 0 && ci_off + cin <= cx, "input channel stride/offset must be x8");
  ConvArgs a{};
  a.x = (const bf16*)x;
  a.cx = cx;
  a.ci_off = ci_off;
  a.cin = cin;
  a.w = (const bf16*)w;
  a.coutp = coutp;
  a.cout = cout;
  a.bias = bias;
  a.relu = relu;
  a.yb = (bf16*)yb;
  a.cyb = cyb;
  a.yb_off = yb_off;
  a.yf = yf;
  a.cyf = cyf;
  a.yf_off = yf_off;
  a.yf_acc = yf_acc;
  a.v = mkvol(vol);
  long long M = a.v.voxels();
  dim3 grid(nblk(M, CBM), coutp / CBN);
  conv3d_fwd_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(a);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_conv3d_wgrad(const void* x, int cx, int ci_off, int cin, const void* gz, int cg, int cg_off,
                                    int coutp, float* dw, float* dbias, float* part, int64_t part_floats,
                                    const int* vol, mrb_stream_t stream) {
  MRB_REQUIRE(x && gz && dw && part && vol, "null pointer");
  MRB_REQUIRE(cin % 32 == 0 && coutp % 32 == 0, "wgrad needs cin and coutp multiples of 32");
  MRB_REQUIRE(cx % 4 == 0 && ci_off % 4 == 0 && cg % 4 == 0 && cg_off % 4 == 0, "channel strides must be x4");
  cudaStream_t st = (cudaStream_t)stream;
  WgradArgs a{};
  a.x = (const bf16*)x;
  a.cx = cx;
  a.ci_off = ci_off;
  a.cin = cin;
  a.gz = (const bf16*)gz;
  a.cg = cg;
  a.cg_off = cg_off;
  a.coutp = coutp;
  a.v = mkvol(vol);
  const long long M = a.v.voxels();
  const long long wsz = 27LL * cin * coutp;
  // fixed split: chunks of 4096 voxels, at most part_floats / wsz of them
  long long nsplit = (M + 4095) / 4096;
  const long long cap = part_floats / wsz;
  MRB_REQUIRE(cap >= 1, "partial buffer too small");
  if (nsplit > cap) nsplit = cap;
  if (nsplit > 65535 / 27) nsplit = 65535 / 27;
  a.chunk = ((M + nsplit - 1) / nsplit + 15) / 16 * 16;
  nsplit = (M + a.chunk - 1) / a.chunk;
  a.part = part;
  dim3 grid((unsigned)(27 * nsplit), cin / 32, coutp / 32);
  conv3d_wgrad_kernel<<<grid, 128, 0, st>>>(a);
  MRB_LAUNCH_CHECK();
  sum_splits_kernel<<<nblk(wsz, 256), 256, 0, st>>>(part, (int)nsplit, wsz, dw);
  MRB_LAUNCH_CHECK();
  if (dbias) {
    MRB_REQUIRE(nsplit * coutp <= part_floats, "partial buffer too small for the bias");
    bias_grad_kernel<<<dim3((unsigned)nsplit, coutp / 32), 256, 0, st>>>((const bf16*)gz, cg, cg_off, coutp, M,
                                                                         a.chunk, part);
    MRB_LAUNCH_CHECK();
    sum_splits_kernel<<<nblk(coutp, 256), 256, 0, st>>>(part, (int)nsplit, coutp, dbias);
    MRB_LAUNCH_CHECK();
  }
  return 0;
}

extern "C" int mrb_cnn_flip_weights(const void* w, int cin, int coutp, void* wd, int cinp, mrb_stream_t stream) {
  MRB_REQUIRE(w && wd && cinp >= cin, "bad arguments");
  long long n = 27LL * coutp * cinp;
  flip_weights_kernel<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)w, cin, coutp, (bf16*)wd, cinp);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_relu_bwd(const float* g, int cgs, int g_off, const void* act, int cas, int a_off, int nch,
                                int64_t voxels, void* gz, int czs, int z_off, int nchp, mrb_stream_t stream) {
  MRB_REQUIRE(g && gz && nchp >= nch, "bad arguments");
  relu_bwd_kernel<<<nblk(voxels * nchp, 256), 256, 0, (cudaStream_t)stream>>>(
      g, cgs, g_off, (const bf16*)act, cas, a_off, nch, voxels, (bf16*)gz, czs, z_off, nchp);
  MRB_LAUNCH_CHECK();
  return 0;
}

// 16-byte channel groups possible: nch = 8 * 2^lg8, strides and offsets multiples of 8, aligned bases
static bool vec8(int nch, int cin_s, int in_off, int cout_s, int out_off, const void* in, const void* out, int* lg8) {
  if (nch <= 0 || nch % 8 || cin_s % 8 || in_off % 8 || cout_s % 8 || out_off % 8) return false;
  if (((uintptr_t)in & 15) || ((uintptr_t)out & 15)) return false;
  const int g = nch / 8;
  if (g & (g - 1)) return false;
  int l = 0;
  while ((1 << l) < g) ++l;
  *lg8 = l;
  return true;
}

extern "C" int mrb_cnn_pool2(int dir, const void* in, int cin_s, int in_off, int nch, const int* fine_vol, void* out,
                             int cout_s, int out_off, mrb_stream_t stream) {
  MRB_REQUIRE(in && out && fine_vol, "null pointer");
  Vol v = mkvol(fine_vol);
  MRB_REQUIRE(v.H % 2 == 0 && v.W % 2 == 0, "pooling needs even H and W");
  cudaStream_t st = (cudaStream_t)stream;
  int lg8 = 0;
  if (dir == 0 && vec8(nch, cin_s, in_off, cout_s, out_off, in, out, &lg8) && v.voxels() < (1LL << 31)) {
    const int per_row = (v.W / 2) << lg8;
    const int rows = v.Nb * v.D * (v.H / 2);
    pool2_fwd_vec_kernel<<<dim3((unsigned)nblk(per_row, 256), (unsigned)std::min(rows, 65535)), 256, 0, st>>>(
        (const bf16*)in, cin_s, in_off, lg8, v, (bf16*)out, cout_s, out_off);
  } else if (dir == 0) {
    long long n = v.voxels() / 4 * nch;
    pool2_fwd_kernel<<<nblk(n, 256), 256, 0, st>>>((const bf16*)in, cin_s, in_off, nch, v, (bf16*)out, cout_s,
                                                   out_off);
  } else {
    long long n = v.voxels() * nch;
    pool2_bwd_kernel<<<nblk(n, 256), 256, 0, st>>>((const float*)in, cin_s, in_off, nch, v, (float*)out, cout_s,
                                                   out_off);
  }
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_up2(int dir, const void* in, int cin_s, int in_off, int nch, const int* coarse_vol, void* out,
                           int cout_s, int out_off, mrb_stream_t stream) {
  MRB_REQUIRE(in && out && coarse_vol, "null pointer");
  Vol v = mkvol(coarse_vol);
  cudaStream_t st = (cudaStream_t)stream;
  int lg8 = 0;
  if (dir == 0 && vec8(nch, cin_s, in_off, cout_s, out_off, in, out, &lg8) && v.voxels() * 4 < (1LL << 31)) {
    const int per_row = (2 * v.W) << lg8;
    const int rows = v.Nb * v.D * 2 * v.H;
    up2_fwd_vec_kernel<<<dim3((unsigned)nblk(per_row, 256), (unsigned)std::min(rows, 65535)), 256, 0, st>>>(
        (const bf16*)in, cin_s, in_off, lg8, v, (bf16*)out, cout_s, out_off);
  } else if (dir == 0) {
    long long n = v.voxels() * 4 * nch;
    up2_fwd_kernel<<<nblk(n, 256), 256, 0, st>>>((const bf16*)in, cin_s, in_off, nch, v, (bf16*)out, cout_s, out_off);
  } else {
    long long n = v.voxels() * nch;
    up2_bwd_kernel<<<nblk(n, 256), 256, 0, st>>>((const float*)in, cin_s, in_off, nch, v, (float*)out, cout_s,
                                                 out_off);
  }
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_pack(const void* z, const float* scale, const int* vol, void* x, int cx, mrb_stream_t stream) {
  MRB_REQUIRE(z && scale && vol && x && cx >= 2, "bad arguments");
  Vol v = mkvol(vol);
  if (cx % 8 == 0 && ((uintptr_t)x & 15) == 0 && (long long)v.H * v.W < (1LL << 31)) {
    const int frames = v.Nb * v.D;
    pack_vec_kernel<<<dim3((unsigned)nblk((long long)v.H * v.W, 256), (unsigned)std::min(frames, 65535)), 256, 0,
                      (cudaStream_t)stream>>>((const float2*)z, scale, v, (bf16*)x, cx);
  } else {
    pack_kernel<<<nblk(v.voxels() * cx, 256), 256, 0, (cudaStream_t)stream>>>((const float2*)z, scale, v, (bf16*)x,
                                                                             cx);
  }
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_unpack(const void* zin, const float* net, int cy, const float* scale, const int* vol, void* zout,
                              mrb_stream_t stream) {
  MRB_REQUIRE(zin && net && scale && vol && zout, "bad arguments");
  Vol v = mkvol(vol);
  unpack_kernel<<<nblk(v.voxels(), 256), 256, 0, (cudaStream_t)stream>>>((const float2*)zin, net, cy, scale, v,
                                                                         (float2*)zout);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_mse(const void* zin, const void* target, const float* net, int cy, const float* scale,
                           const int* vol, float* grad, double* loss, double* part, int64_t part_len,
                           mrb_stream_t stream) {
  MRB_REQUIRE(zin && target && net && scale && vol && grad && loss && part, "bad arguments");
  Vol v = mkvol(vol);
  int nb = nblk(v.voxels(), 256);
  MRB_REQUIRE(nb <= part_len, "loss partial buffer too small");
  cudaStream_t st = (cudaStream_t)stream;
  mse_kernel<<<nb, 256, 0, st>>>((const float2*)zin, (const float2*)target, net, cy, scale, v,
                                 1.f / (float)(v.voxels() * 2), grad, part);
  MRB_LAUNCH_CHECK();
  sum_double_kernel<<<1, 32, 0, st>>>(part, nb, loss);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                            float eps, int step, void* wb, mrb_stream_t stream) {
  MRB_REQUIRE(w && g && m && v && step >= 1, "bad arguments");
  float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps, bc1, bc2, (bf16*)wb);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_cnn_to_bf16(const float* a, int64_t n, void* b, mrb_stream_t stream) {
  MRB_REQUIRE(a && b, "null pointer");
  f32_to_bf16_kernel<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(a, n, (bf16*)b);
  MRB_LAUNCH_CHECK();
  return 0;
}
