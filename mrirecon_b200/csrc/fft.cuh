// Fused, zero-pruned oversampled 2D FFT passes (fft.cu) used by the NUFFT plan.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "mrb_common.cuh"

namespace mrb {

// true when compiled kernels cover this 2D geometry (G0, G1 in the length list)
bool fft2_supported(int S0, int S1, int G0, int G1);
// bytes of the band buffer T (nb, C, S0, G1) complex
size_t fft2_tmp_bytes(int S0, int G1, int C, int nb);
// device twiddle table of a length-G transform
int fft2_twiddles(DevBuf& tw, int G, const float2** out);

// skip: device flag, the kernels return at once when it is non-zero (may be null)
// The row passes see a frame as S0 rows of S1 samples (a 3D volume S0 x S1 x S2
// is S0*S1 rows of S2); rowfac (S0) holds each row's signed deapodisation
// (-1)^(row parity) prod 1/Phi over the leading dims, coldeap (S1) the last
// dim's 1/Phi; the last dim's sign (-1)^(i + G1/2 - S1/2) is applied here.
// image (nb, S0, S1) [or coil images (nb, C, S0, S1)] -> T (nb, C, S0, G1)
int fft2_forward_rows(const void* x, const float2* maps, const float* rowfac, const float* coldeap, float2* Tb,
                      const float2* tw1, int S0,
                      int S1, int G0, int G1, int C, int nb, int coil_images, const double* skip,
                      cudaStream_t st);
// forward != 0: T -> grid (nb, C, G0, G1); else grid -> T.  blocked (forward
// only): each coil-frame's grid in blocks of 2 x 8 cells, cell (n0, n1) at
// ((n0 / 2) * (G1 / 8) + n1 / 8) * 16 + (n0 % 2) * 8 + n1 % 8 (the 2D interp's
// layout; G0 even, G1 a multiple of 8)
int fft2_columns(int forward, const float2* in, float2* out, const float2* tw0, int S0, int S1, int G0, int G1, int C,
                 int nb, const double* skip, cudaStream_t st, int blocked = 0);
// Forward column pass whose output is coil-interleaved: in (nb, C, S0, G1)
// band rows -> out (nb, G0 * G1 cells, C), for C in {8, 16, 32} (the 3D x pass
// writing the interp's (cell, coil) grid copy directly)
bool fft2_columns_il_supported(int G0, int C);
int fft2_columns_il(const float2* Tb, float2* out, const float2* tw0, int S0, int G0, int G1, int C, int nb,
                    const double* skip, cudaStream_t st);
// Forward column pass of a 2D grid with a coil-quad output: in (nb, C, S0, G1)
// band rows -> out (nb, C / 4 quads, G0 * G1 cells, 4 coils), the same values
// as fft2_columns with each cell's coils in groups of four (32 bytes), for the
// interp's 128-bit gathers of a cell's coil pairs.  C % 4 == 0.
int fft2_columns_cg(const float2* Tb, float2* out, const float2* tw0, int S0, int S1, int G0, int G1, int C, int nb,
                    const double* skip, cudaStream_t st);
// Forward column pass fused with the KB interp (2D): the block of a coil and
// a strip of interp_strip_width(G0) grid columns transforms those columns and
// the next three (the support of a sample starting in the strip reaches three
// columns further; wrapped at G1) in shared memory and interpolates every
// sample of the strip for that coil straight from there.  The oversampled
// grid is never written.
struct ColInterp {
  const float* gx;           // (B, 2, K) grid coordinates
  const float* wfwd;         // (B, K) forward weights or null
  const int* strip_start;    // (B * nstrips + 1): per-frame strip lists
  const int* strip_entries;  // sample indices, by (frame, strip), acquisition order within
  float2* y;                 // (nb, C, K)
  long long K;
  int B, nb, nstrips;
  float scale;               // ortho scale times the sample-side sign
  KBPoly kb;
};
int interp_strip_width(int G0);
int fft2_columns_interp(const float2* Tb, const float2* tw0, int S0, int S1, int G0, int G1, int C, int nb,
                        const ColInterp& ci, const double* skip, cudaStream_t st);
// Toeplitz normal operator on the band, in place: T <- IFFT_G0(P[frame] * FFT_G0(T)) per
// column; P (B, G0, G1) real, frame = be / (nb / B) (0 when B == 1)
int fft2_toeplitz_columns(float2* Tb, const float* P, const float2* tw0, int S0, int S1, int G0, int G1, int C, int nb,
                          int B, const double* skip, cudaStream_t st);
// T -> image (nb, S0, S1), coil-combined with conj(maps), scaled
int fft2_adjoint_rows(const float2* Tb, const float2* maps, const float* rowfac, const float* coldeap, void* x,
                      const float2* tw1, int S0,
                      int S1, int G0, int G1, int C, int nb, float scale, const double* skip,
                      cudaStream_t st);

}  // namespace mrb
