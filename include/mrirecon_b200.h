/*
 * mrirecon_b200 — C ABI of the B200-native NCG/NUFFT hot path.
 *
 * Every entry point returns 0 on success and a non-zero MRB_E* code on
 * failure; mrb_last_error() returns a message for the calling thread.  All
 * pointers marked "dev" are CUDA device pointers; sizes are element counts.
 * Every call is asynchronous on the given stream (no host synchronisation)
 * unless stated otherwise, so a sequence of calls can be captured into a
 * CUDA graph once the plan's buffers exist (the first forward/adjoint call
 * for a new batch size allocates; issue it before capture).
 *
 * Complex data is interleaved float32 pairs (C99 float _Complex / torch
 * complex64), row-major, last image axis fastest.
 *
 * Each declaration names the reference interface it replaces
 * (graspcg = timodelgado/mrirecon, paths relative to that project).
 */
#ifndef MRIRECON_B200_H
#define MRIRECON_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* mrb_stream_t;   /* == cudaStream_t */
typedef struct mrb_plan mrb_plan;            /* opaque NUFFT plan */

enum {
  MRB_OK = 0,
  MRB_EINVAL = 1,     /* bad argument / shape */
  MRB_ECUDA = 2,      /* CUDA runtime error */
  MRB_ECUFFT = 3,     /* cuFFT error */
  MRB_ENOMEM = 4,     /* allocation failed */
  MRB_ESTATE = 5,     /* plan not ready (points or maps missing) */
  MRB_ERANGE = 6      /* size above a fixed limit */
};

enum { MRB_DCF_NONE = 0, MRB_DCF_BALANCED = 1, MRB_DCF_STANDARD = 2 };
enum { MRB_IDX_REFERENCE = 0, MRB_IDX_CORRECTED = 1 };

int mrb_version(void);
const char* mrb_last_error(void);

/* ------------------------------------------------------------------------
 * NUFFT plan (Kaiser-Bessel, oversampled grid, SENSE coils, B frames)
 * ---------------------------------------------------------------------- */

/* Create a plan for nd-dimensional images of shape S[0..nd) with C coils,
 * B trajectory frames of K samples each, kernel width W (even), grid
 * oversampling osf (grid G_d = ceil(osf*S_d), must be even), and ortho
 * scaling 1/sqrt(prod G) when norm_ortho != 0.
 * Replaces: TorchKbNUFFTAdapter.prepare  graspcg/nufft/backends/torchkb.py:98-144
 *           PTNUFFTAdapter.prepare       graspcg/nufft/backends/ptnufft.py:102-216 */
int mrb_plan_create(mrb_plan** plan, int nd, const int* S, int C, int B, int64_t K,
                    int W, double osf, int norm_ortho);
int mrb_plan_destroy(mrb_plan* plan);

/* Tuning knobs read by set_points / the operators (autotuner):
 * key 0 = spread tile edge (cells), key 1 = coils per spread work item,
 * key 2 = interp mode (0 acquisition order, 1 tile-sorted order). */
int mrb_plan_set_option(mrb_plan* plan, int key, int64_t value);

/* Trajectory (dev, (B, nd, K) float32 radians in [-pi, pi)): float32 grid
 * coordinates (reference arithmetic) and the per-tile sorted sample lists.
 * Replaces the per-frame index tables of ptnufft.py:145-201. */
int mrb_plan_set_points(mrb_plan* plan, const float* traj, mrb_stream_t stream);

/* Density compensation (dev, (B, K) float32, or NULL) and its policy.
 * Replaces: TorchKbNUFFTAdapter._weights  graspcg/nufft/backends/torchkb.py:185-199 */
int mrb_plan_set_dcf(mrb_plan* plan, const float* dcf, int mode, int apply_fwd, int apply_adj,
                     mrb_stream_t stream);

/* Coil sensitivities (dev, (C, *S) complex64); copied into the plan. */
int mrb_plan_set_maps(mrb_plan* plan, const void* maps, mrb_stream_t stream);

/* Forward: x (dev, (nb, 1, *S) complex64) -> y (dev, (nb, C, K)).
 * nb is B_eff; frame be uses trajectory frame be / (nb / B) (or 0 if B == 1).
 * Replaces: TorchKbNUFFTAdapter.A  graspcg/nufft/backends/torchkb.py:202-270 */
int mrb_nufft_forward(mrb_plan* plan, const void* x, void* y, int nb, mrb_stream_t stream);

/* Forward for per-coil images x (dev, (nb, C, *S)): maps are not applied
 * (the Cin == C branch of TorchKbNUFFTAdapter.A, torchkb.py:244-247). */
int mrb_nufft_forward_coils(mrb_plan* plan, const void* x, void* y, int nb, mrb_stream_t stream);

/* Adjoint: y (dev, (nb, C, K)) -> x (dev, (nb, 1, *S)), coil-combined.
 * Replaces: TorchKbNUFFTAdapter.AH  graspcg/nufft/backends/torchkb.py:272-323 */
int mrb_nufft_adjoint(mrb_plan* plan, const void* y, void* x, int nb, mrb_stream_t stream);

/* Plan facts for tests and the bench (host copies, synchronous):
 * out[0] = number of spread entries, out[1] = tiles per frame,
 * out[2] = touched grid cells summed over frames, out[3] = spread tile edge,
 * out[4] = coils per spread work item, out[5] = grid cells per frame. */
int mrb_plan_info(mrb_plan* plan, int64_t* out, int nout);

/* floor of the float32 grid coordinates the plan computed, (B, nd, K) int32
 * (dev out).  Bit-exact key of the production binning. */
int mrb_plan_cell_base(mrb_plan* plan, int32_t* out, mrb_stream_t stream);

/* Stand-alone grid index table for one frame of trajectory (dev (nd, K)
 * float32 radians) on grid G: (K, W^nd) int64 (dev out).
 * convention MRB_IDX_REFERENCE reproduces the reference's literal table
 * (ptnufft.py:151-171, 173-195: float32 offsets -W/2..W/2-1 added before
 * floor, flat index nx + G0*ny (+G0*G1*nz)); MRB_IDX_CORRECTED gives the
 * integer-node, row-major table the operators use. */
int mrb_grid_indices(const float* traj, int nd, const int* G, int64_t K, int W, int convention,
                     int64_t* idx, mrb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* MRIRECON_B200_H */
