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
/* Number of kernel launches this library has issued in the process (host
 * side; a launch recorded into a CUDA graph counts once, at capture). */
int64_t mrb_launch_count(void);
/* Device blocks of 1 MiB and more that destroyed plans released are cached
 * (per device, up to 8 GiB) for the next plans, so that building operators
 * repeatedly (a new trajectory per scan) avoids gigabyte cudaMalloc / cudaFree
 * calls of very variable cost.  This returns the cached blocks to the driver
 * (like torch.cuda.empty_cache); the cache is also emptied when an allocation
 * would otherwise fail.  No reference counterpart. */
int mrb_release_cached_memory(void);

/* ------------------------------------------------------------------------
 * Grouped launches: many independent problems, one launch per kernel step
 *
 * Between mrb_group_begin(n) and mrb_group_end(stream) the entry points of
 * this library record their kernel launches instead of issuing them, each
 * into the list of the problem last chosen with mrb_group_select(i).  Their
 * stream arguments are ignored; device pointers and scalars are taken at the
 * call (device memory a call allocates is allocated then).
 * mrb_group_end issues the records on `stream` in steps: each step launches
 * the next record of every problem whose next record runs the same kernel as
 * ONE grouped launch (a table of the problems' arguments in kernel parameter
 * space, every block finding its problem and its own block coordinates there),
 * so each problem computes bit for bit what its own launches compute, in the
 * order it made them.  Problems must not share device buffers they write.
 * Inside a stream capture the grouped launches become the graph's nodes.
 * Entry points whose kernels have no grouped form fail inside a recording
 * (MRB_ESTATE): the 2D NUFFT in the fused FFT mode, the NCG kernels, the TV
 * passes and graph passes have one; the cuFFT mode, the 3D block spreads,
 * the Toeplitz column pass, the dots and the preconditioner set-up do not.
 * One recording per process at a time.  mrb_group_cancel drops an open
 * recording; mrb_group_stats returns the records and launches of the last
 * mrb_group_end.
 * The reference solves one problem per CGSolver call
 * (graspcg/solvers/cg.py:162-246); this interface has no counterpart there. */
int mrb_group_begin(int nproblems);
int mrb_group_select(int problem);
int mrb_group_end(mrb_stream_t stream);
int mrb_group_cancel(void);
int mrb_group_stats(int64_t* records, int64_t* launches);

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
 * key 2 = interp mode: 0 one thread per sample for all coils, in acquisition
 *         order; 1 (default) 2D: one thread per (sample, coil pair); 3D (coil-
 *         interleaved grid): segments of 8 consecutive samples visited in the
 *         Morton order of their tile (samples and results stay in acquisition
 *         order); both give the same results as mode 0,
 * key 3 = samples per spread work item (heavy tiles are split),
 * key 4 = FFT mode: 0 dense cuFFT transform with separate pad / crop kernels,
 *         1 fused zero-pruned passes (2D: rows then columns; 3D: z rows, then
 *         y and x columns; grids whose sides all have compiled kernels; the
 *         default wherever available),
 * key 6 = spread kernel: 1 one block per work item, all coils of a group
 *         sharing the staged samples (2D tile 16, 3D tile 8; other tiles fall
 *         back to 0; the 3D default), 0 one warp per work item and coil group
 *         (the 2D default), 2 (2D, coil groups of up to 16) one warp per work
 *         item that first tabulates each staged sample's inside taps and then
 *         runs only those (faster from 6 coils per item on, slower at 4: the
 *         autotuner times both); all give identical grids,
 * key 7 = grid mask (fused FFT mode): 1 (default) the adjoint spread keeps its
 *         own grid, zeroed once per trajectory and batch size, and stores only
 *         the cell pairs inside some sample's support (per-frame bitmaps built by
 *         set_points); 0 the spread writes every cell of every tile,
 * key 8 = 2D fused mode: the forward column pass interpolates the samples of
 *         each column strip from shared memory and never writes the grid
 *         (1; set before set_points, which then builds the per-frame strip
 *         lists) or writes the grid for a separate interp pass (0, the
 *         default: 2% slower forward, but each kernel on its own); same samples,
 * key 5 = forward interp on a coil-interleaved grid (1; the 3D default) or on
 *         the coil-planar grid (0; the 2D default).  3D: a copy of the grid (written by the x
 *         column pass for 8/16/32 coils, else by a tiled transpose; one more
 *         grid-sized buffer), then 128-bit gathers of all coils of a cell.
 *         2D fused FFT mode with C % 4 == 0: the forward column pass writes
 *         the plan's grid itself in coil quads, (quad, cell, 4 coils) (blocks
 *         of 4 columns x 4 coils, 128-byte stores), and the interp gathers coil
 *         pairs with 128-bit loads; no extra buffer.  Same samples.  On the
 *         GRASP workload the interp gains 20 us and the column pass loses 46 us,
 *         so 2D keeps the planar grid by default,
 * key 9 = 2D fused mode with the pair-parallel interp on the coil-planar grid:
 *         the forward column pass stores each coil-frame's grid in blocks of
 *         2 x 8 cells, cell (n0, n1) at ((n0/2)(G1/8) + n1/8) 16 + (n0%2) 8 +
 *         n1%8 (1, the default; G1 a multiple of 8), or row-major (0).  A
 *         sample's 4 x 4 taps meet 2 to 6 128-byte lines instead of 4 to 8, and
 *         a warp's stores still fill whole lines.  Same samples; on the GRASP
 *         workload the interp falls from 107 to 82 us and the column pass
 *         gains 3 us,
 * key 10 = 2D: the per-warp spread and the pair-parallel interp read each
 *         sample's first nodes and signed kernel weights from a table that
 *         set_points builds with the coordinates (1, the default; 40 bytes per
 *         sample) or evaluate the kernel polynomials per call (0).  Same
 *         weights bit for bit. */
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

/* One stage of the operators, for timing and tuning: stage 0 = pre-FFT
 * (SENSE, deapodisation, zero-pad; x -> grid), 1 = forward FFT, 2 = interp
 * (grid -> y), 3 = spread (y -> grid), 4 = inverse FFT, 5 = post-IFFT (crop,
 * deapodisation, conj-maps coil sum; grid -> x).  The grid is the plan's.
 * In FFT mode 1 stage 0 also runs the row transforms (x -> band buffer),
 * 1 the column transforms (band -> grid), 4 the inverse column transforms
 * (grid -> band) and 5 the inverse row transforms with crop and coil sum.
 * With option key 8 on (2D), stage 1 given a non-null y runs the column
 * transforms fused with the interp (band -> y, no grid) and stage 2 is not
 * needed; given a null y it writes the grid as above. */
int mrb_nufft_stage(mrb_plan* plan, int stage, const void* x, void* y, int nb, mrb_stream_t stream);

/* Plan facts for tests and the bench (host copies, synchronous):
 * out[0] = number of spread entries, out[1] = tiles per frame,
 * out[2] = touched grid cells summed over frames, out[3] = spread tile edge,
 * out[4] = coils per spread work item, out[5] = grid cells per frame,
 * out[6] = FFT mode (option key 4), out[7] = 1 when the spread runs the
 * block-per-tile kernel (option key 6), out[8] = 1 when the forward column
 * pass interpolates (option key 8), out[9] = 1 when the sample lists match
 * the current tile and chunk options (no set_points needed). */
int mrb_plan_info(mrb_plan* plan, int64_t* out, int nout);

/* Toeplitz normal operator (no counterpart in the reference; its item
 * "Toeplitz A^H A embedding").  With t_b(D) = sum_k w_k exp(i w_k . D) the
 * sampling point-spread function of frame b (w the product of the forward and
 * adjoint DCF weights), A^H A x = s^2 sum_n x_n t_b(r_m - r_n) is a circular
 * convolution on the 2x grid.  psf (dev, (B, G0, G1) float32) is its real
 * transfer function FFT(circular t_b) * s^2 / (G0 G1), rolled by (G0/2, G1/2);
 * copied into the plan.  Needs FFT mode 1. */
int mrb_plan_set_toeplitz(mrb_plan* plan, const float* psf, mrb_stream_t stream);
/* out (dev, (nb, 1, *S)) = A^H A x through the Toeplitz transfer function:
 * SENSE + row FFTs, column FFT x P x inverse column FFT in shared memory,
 * inverse row FFTs + conj(S_c) coil sum.  No gridding. */
int mrb_nufft_normal(mrb_plan* plan, const void* x, void* out, int nb, mrb_stream_t stream);

/* Device flag (dev, one double, or NULL to clear) read by every operator
 * kernel launched from now on: when it is non-zero at run time the kernel
 * returns without work.  A solver points it at its own "done" flag so that
 * graph replays past convergence (and finished instances of a batch) cost no
 * gridding or FFT work; the dense cuFFT transform (FFT mode 0) still runs.
 * No counterpart in the reference (its loop stops on the host). */
int mrb_plan_set_skip_flag(mrb_plan* plan, const double* flag);

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

/* ------------------------------------------------------------------------
 * Scratch for the FP64 reductions.  Every reducing entry point below takes
 * a caller-owned device workspace `ws` of at least mrb_workspace_bytes()
 * bytes (block partials and a completion counter), ZERO-FILLED before its
 * first use (the library leaves the counter at zero after every call); calls
 * on one stream may share it, calls that may overlap on the GPU need their
 * own.
 * ---------------------------------------------------------------------- */
int mrb_workspace_bytes(int64_t* bytes);

/* out[j] = sum_i Re(conj(a_j[i]) * b_j[i]) / (diag_j ? diag_j[i % ndiag] : 1),
 * FP64, j < npairs <= 8, n complex64 elements each; deterministic.
 * Replaces: dot_real0 / dot_precond0  graspcg/numerics/utils.py:94-206
 *           dot_chunked               graspcg/ops/dot.py:5-71 */
int mrb_dots_f64(int64_t n, int npairs, const void* const* a, const void* const* b,
                 const float* const* diag, int64_t ndiag, double* out, void* ws, mrb_stream_t stream);

/* Same result as mrb_dots_f64 without a caller workspace and without any
 * allocation: the block partials live in a fixed device array of 75,776 bytes
 * (1184 blocks x 8 doubles) that every GPU loading this library keeps until
 * the process exits.  For callers that cannot allocate device memory where
 * they need the dots (inside a CUDA stream capture, in real-time loops where
 * cudaMalloc/cudaFree would synchronise the device, or when another allocator
 * owns all device memory).  npairs above 8 is rejected (MRB_ERANGE).  A call
 * outside a stream capture looks up the array's device address on the current
 * device (cudaGetSymbolAddress, so a cudaDeviceReset leaves nothing stale); a
 * call inside a capture reuses the address of the last call outside one, so
 * the first call on a device must come before any capture (else MRB_ESTATE).  All
 * calls share the one array, so calls that overlap on the GPU (other streams,
 * other host threads) race; serialise them.  No part of the array needs to
 * start at zero: every call overwrites each partial it reads.
 * This entry point has no counterpart in the reference. */
int mrb_dots_f64_noalloc(int64_t n, int npairs, const void* const* a, const void* const* b,
                         const float* const* diag, int64_t ndiag, double* out, mrb_stream_t stream);

/* k-space passes over n complex64 samples (t from t_dev if non-NULL, else t_host;
 * the pass is skipped when skip != NULL and *skip != 0):
 *   mode 0: out[0..2] = |r|^2, Re<r,Ad>, |Ad|^2 (FP64)
 *   mode 1: r = Ax + t*Ad - y (Ad may be NULL), out[0] = |r|^2
 *   mode 2: r += t*Ad
 * Replaces: _ker_residual_energy_  graspcg/ops/objective.py:31-45 */
int mrb_kspace_pass(int mode, int64_t n, void* r, const void* Ad, const void* Ax, const void* y,
                    const double* t_dev, double t_host, const double* skip, double* out, void* ws,
                    mrb_stream_t stream);

/* ------------------------------------------------------------------------
 * Regularisation: fused Huber-TV energy + gradient
 * ---------------------------------------------------------------------- */
typedef struct mrb_tv_term {
  int enabled;
  int isotropic;         /* l2 coupling across axes if non-zero */
  float weight;          /* lambda */
  float eps;             /* Huber knee */
  int naxes;             /* <= 4 */
  int axes[4];           /* axis ids of the (F, 1, *S) image: 0 = frame, 2.. = spatial */
  float axis_weights[4]; /* per-axis scale of the forward differences */
  int frame_period;      /* > 0: the frame axis holds independent series of this many
                            frames (no difference across series boundaries); 0: one series */
} mrb_tv_term;

/* At z = x + t*d (d may be NULL) for an image (F, 1, *S) complex64 with
 * nd spatial dims: g_out = g_base + t*g_dir - sum_T lambda_T div p_T
 * (g_base/g_dir/g_out may be NULL), and FP64 reductions into out[0..10]:
 *   out[0..3]  lambda_T * sum e_T for the enabled terms in order
 *   out[4] Re<g,d>  out[5] <g,g/D>  out[6] |z|^2  out[7] |d|^2
 *   out[8] <g_prev,g/D>  out[9] <g_prev,g_prev/D>  out[10] Re<d,g_prev>
 * The pass is skipped when skip != NULL and (*skip == 0 if skip_if_zero
 * else *skip != 0).
 * Replaces: TVND.energy_grad_fixed_axes  graspcg/regularization/tv_nd.py:54-88
 *           (stencils graspcg/ops/ndops.py:28-148), RegManager.energy_and_grad
 *           graspcg/regularization/manager.py:38-142 for one shard, and the
 *           reg/slope part of Objective.f_g_tensor graspcg/ops/objective.py:255-291 */
int mrb_tv_grad(int nd, const int* S, int F, const mrb_tv_term* terms, int nterms, const void* x,
                const void* d, const double* t_dev, double t_host, const void* g_base, const void* g_dir,
                void* g_out, const float* diag, int64_t ndiag, const void* g_prev, const double* skip,
                int skip_if_zero, double* out, void* ws, mrb_stream_t stream);

/* Sum of the TV energies at z = x + ts[j]*d for j < J <= 24 (dev ts),
 * out[j] (FP64); one pass over x and d.  Skipped when *skip != 0.
 * Replaces the per-trial regulariser evaluations of the Armijo loop
 * graspcg/numerics/line_search.py:57-72. */
int mrb_tv_multi(int nd, const int* S, int F, const mrb_tv_term* terms, int nterms, const void* x,
                 const void* d, const double* ts, int J, const double* skip, double* out, void* ws,
                 mrb_stream_t stream);

/* ------------------------------------------------------------------------
 * Device-resident NCG controller.  `slots` is a device array of
 * mrb_ncg_slot_count() doubles (t, ls_ok, done, reason, iter, f0, g0d, ...);
 * `cfg` is a DEVICE array of 10 doubles {c1, ls_beta, ls_max_iter (<= 23),
 * max_iter, tol_g, tol_step, stop_window, stop_tol, direction (0 FR, 1 PR+,
 * 2 DY), history rows}, read by the kernels (a captured graph sees edits).  Replaces CGSolver.run graspcg/solvers/cg.py:162-246,
 * _armijo graspcg/numerics/line_search.py:24-79 and the directions of
 * graspcg/numerics/directions.py:75-162 without host synchronisation.
 * ---------------------------------------------------------------------- */
int mrb_ncg_slot_count(int64_t* slots, int64_t* hist_cols);
int mrb_ncg_set_steps(double* ts, int J, double beta, mrb_stream_t stream);
int mrb_ncg_armijo_select(double* slots, const double* cfg, mrb_stream_t stream);
/* The same backtracking choice in two phases (no reference counterpart): phase
 * 1 tries steps j = 1 .. J1-1 from a tv_multi pass over J1 steps; phase 2 (after
 * a tv_multi pass over the remaining steps, skipped through slot 20 when phase
 * 1 decided) continues at j = J1.  Same accepted step as the single pass. */
int mrb_ncg_armijo_phase(double* slots, const double* cfg, int J1, int phase, mrb_stream_t stream);
int mrb_ncg_control(double* slots, double* hist, const double* cfg, int nterms, int have_ft,
                    mrb_stream_t stream);
int mrb_ncg_update(int64_t n, void* x, void* d, const void* g, void* gr, const void* gAd, void* g_prev,
                   const float* diag, int64_t ndiag, double* slots, void* ws, mrb_stream_t stream);
int mrb_ncg_steepest(int64_t n, void* d, const void* g, void* g_prev, const float* diag, int64_t ndiag,
                     double* out, void* ws, mrb_stream_t stream);
/* Residual energy after the accepted step when the k-space residual is not
 * kept (Toeplitz schedule): slot err += 2 t erd + t^2 edd (no reference
 * counterpart; the reference recomputes A x every iteration). */
int mrb_ncg_err_step(double* slots, mrb_stream_t stream);
/* Optional restart after mrb_ncg_update (no counterpart in the reference,
 * whose loop stops when the new direction is not a descent direction): if
 * Re<g, d> >= 0, d = -g/D, the slope slot becomes -<g, g/D> and slot 19
 * counts the restarts.  Returns at once on the device when no restart is due. */
int mrb_ncg_restart(int64_t n, void* d, const void* g, const float* diag, int64_t ndiag, double* slots,
                    mrb_stream_t stream);

/* Jacobi diagonal of the preconditioner (float32, F*P entries, the layout of
 * the image (F, 1, *S); P pixels per frame).
 * mrb_precond_init: diag = base + alpha * sum_c |maps_c|^2 per pixel (maps
 * (C, *S) complex64, or NULL for diag = base).  The reference initialises the
 * diagonal to ones (graspcg/solvers/cg.py:95: base 1, maps NULL) and exposes
 * alpha as TorchKbNUFFTAdapter.diag_AHA_scalar (graspcg/nufft/backends/torchkb.py:341-364).
 * mrb_tv_add_diag: diag += the terms' diagonal at x, as
 * RegManager.add_diag (graspcg/regularization/manager.py:145-218) adds it for
 * identity regularisers: a term with the frame axis adds its frame profile
 * 2 lambda w_0^2 deg(f) (TVND.majorizer_profile, tv_nd.py:187-214; deg 1 at
 * the ends of each series of frame_period frames, 2 inside) when
 * frame_profile != 0; any other term adds per axis
 * lambda w^2 / sqrt(|D_a x|^2 + eps^2), once on the first and last slice and
 * twice inside (TVND.add_diag, tv_nd.py:113-164). */
int mrb_precond_init(int64_t P, int F, int C, const void* maps, float alpha, float base, float* diag,
                     mrb_stream_t stream);
int mrb_tv_add_diag(int nd, const int* S, int F, const mrb_tv_term* terms, int nterms, const void* x,
                    int frame_profile, float* diag, mrb_stream_t stream);
/* diag[f*P + p] += v[f] (dev v, F values): a per-frame diagonal profile, e.g.
 * GraphLaplacian.add_diag's lambda*deg (graspcg/regularization/graph_laplacian.py:236-275). */
int mrb_diag_add_frames(int64_t P, int F, const float* v, float* diag, mrb_stream_t stream);

/* Graph Laplacian regulariser over the frame axis of an image (B, N) complex64
 * (B frames of N voxels), L (dev, B x B float32, row-major) the weighted
 * Laplacian sum_i lambda_i L_i (B <= 128):
 *   mode 0: z = x + t*d (d may be NULL), acc += L z (acc may be NULL),
 *           out[0] = 1/2 Re<z, L z>  (the energy)
 *   mode 1: acc += L d, out[0] = Re<x, L d>, out[1] = Re<d, L d>
 *   mode 2: as mode 1 for a non-symmetric L ("rw"): out[0] = Re<x, (L + L^T)/2 d>,
 *           the slope of the energy along d (acc still gets L d)
 * (t from t_dev if non-NULL, else t_host; skipped when skip != NULL and
 * *skip != 0; FP64 reductions).
 * Replaces: GraphLaplacian.energy_grad  graspcg/regularization/graph_laplacian.py:171-234
 *           (_apply_L :135-168, normalisations none / rw / sym folded into L) */
int mrb_graph_pass(int mode, int B, int64_t N, const float* L, const void* x, const void* d,
                   const double* t_dev, double t_host, void* acc, const double* skip, double* out, void* ws,
                   mrb_stream_t stream);
/* Quadratic-term bookkeeping of the fast NCG schedule (slots 21..23 hold the
 * graph energy q0 and, per iteration, q1 = Re<x, L d>, q2 = Re<d, L d>):
 * phase 0 err += 2 q0; phase 1 (unless done) err += 2 q0, erd += q1,
 * edd += q2; phase 2 (accepted step) q0 += t q1 + t^2 q2 / 2.
 * No reference counterpart (the reference re-evaluates every regulariser at
 * each trial step, graspcg/ops/objective.py:255-262). */
int mrb_ncg_quad_fold(double* slots, int phase, mrb_stream_t stream);

/* Frame mixing over the leading (frame) axis: out (rows_out, N) (+)= M in,
 * in (rows_in, N); rows <= 128; in and out must not alias.
 * mrb_frame_mix: complex64 data, M complex64 row-major (rows_out x rows_in),
 * or, with conj_transpose, M given as (rows_in x rows_out) and applied as M^H.
 * mrb_frame_mix_real: float32 data and M (transpose: M given as
 * rows_in x rows_out, applied as M^T).
 * Replaces: TemporalBasisOp.forward_apply / adjoint_apply / diag_push
 *           graspcg/regularization/mapping.py:112-236 (u = U V, g_V += U^H g_u,
 *           diag_V += |U|^T k_u) and the per-frame factors of ScaleOp :44-110. */
int mrb_frame_mix(int rows_out, int rows_in, int64_t N, const void* M, int conj_transpose, const void* in,
                  void* out, int accumulate, mrb_stream_t stream);
int mrb_frame_mix_real(int rows_out, int rows_in, int64_t N, const float* M, int transpose, const float* in,
                       float* out, int accumulate, mrb_stream_t stream);

/* ------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference).  Activations are
 * channels-last BF16 volumes (Nb, D, H, W, channels) with a channel stride
 * and a channel offset (concatenation is a channel offset); `vol` is a host
 * int[4] {Nb, D, H, W}.  Weights are BF16 [27][cin][coutp], tap = kd*9+kh*3+kw
 * over (t, y, x); coutp and channel counts are multiples of 32.
 * ---------------------------------------------------------------------- */
/* 3x3x3 zero-padded convolution on tensor cores (BF16 in, FP32 accumulate),
 * + bias, optional ReLU; writes BF16 (yb) and/or FP32 (yf, accumulated when
 * yf_acc).  The data gradient is this call with mrb_cnn_flip_weights. */
int mrb_cnn_conv3d_fwd(const void* x, int cx, int ci_off, int cin, const void* w, int coutp, int cout,
                       const float* bias, int relu, void* yb, int cyb, int yb_off, float* yf, int cyf,
                       int yf_off, int yf_acc, const int* vol, mrb_stream_t stream);
/* Weight (and bias) gradient: dw[27][cin][coutp] = sum over voxels of
 * x(shifted) * gz, split-K partials in `part` summed in a fixed order. */
int mrb_cnn_conv3d_wgrad(const void* x, int cx, int ci_off, int cin, const void* gz, int cg, int cg_off,
                         int coutp, float* dw, float* dbias, float* part, int64_t part_floats,
                         const int* vol, mrb_stream_t stream);
/* The same weight and bias gradient on the 5th-generation tensor cores
 * (tcgen05.mma, FP32 accumulators in tensor memory): x and gz are first
 * repacked channels-first into `scratch` (x as three copies shifted by -1, 0, +1
 * voxel along W, so that every TMA box starts at a W coordinate that is a
 * multiple of 32), then each CTA accumulates a group of taps over a range of
 * 32-voxel K steps; partial sums (also in `scratch`) are added in a fixed
 * order.  Needs cin and coutp multiples of 16, the smaller of them <= 256,
 * coutp dividing 256 and W a multiple of 64 (mrb_cnn_wgrad_tc_scratch_bytes
 * fails otherwise); scratch: 256-byte aligned, of the size that function
 * returns for (cin, coutp, vol). */
int mrb_cnn_wgrad_tc_scratch_bytes(int cin, int coutp, const int* vol, int64_t* bytes);
int mrb_cnn_conv3d_wgrad_tc(const void* x, int cx, int ci_off, int cin, const void* gz, int cg, int cg_off,
                            int coutp, float* dw, float* dbias, void* scratch, int64_t scratch_bytes,
                            const int* vol, mrb_stream_t stream);
/* Spatially flipped, transposed weights [27][coutp][cinp] for the data gradient. */
int mrb_cnn_flip_weights(const void* w, int cin, int coutp, void* wd, int cinp, mrb_stream_t stream);
/* gz = g * (act > 0) over nch channels (BF16 out, padded to nchp). */
int mrb_cnn_relu_bwd(const float* g, int cgs, int g_off, const void* act, int cas, int a_off, int nch,
                     int64_t voxels, void* gz, int czs, int z_off, int nchp, mrb_stream_t stream);
/* 2x2 mean pooling over (y, x) (dir 0) or its adjoint (dir 1). */
int mrb_cnn_pool2(int dir, const void* in, int cin_s, int in_off, int nch, const int* fine_vol, void* out,
                  int cout_s, int out_off, mrb_stream_t stream);
/* Nearest 2x upsampling over (y, x) (dir 0) or its adjoint (dir 1). */
int mrb_cnn_up2(int dir, const void* in, int cin_s, int in_off, int nch, const int* coarse_vol, void* out,
                int cout_s, int out_off, mrb_stream_t stream);
/* complex image series z (Nb, D, H, W) * scale[Nb] -> 2 real channels of x. */
int mrb_cnn_pack(const void* z, const float* scale, const int* vol, void* x, int cx, mrb_stream_t stream);
/* zout = zin + net[channels 0, 1] / scale (residual output). */
int mrb_cnn_unpack(const void* zin, const float* net, int cy, const float* scale, const int* vol, void* zout,
                   mrb_stream_t stream);
/* Mean squared error of the residual output against target, FP64 loss, FP32
 * gradient with respect to the network output. */
int mrb_cnn_mse(const void* zin, const void* target, const float* net, int cy, const float* scale,
                const int* vol, float* grad, double* loss, double* part, int64_t part_len,
                mrb_stream_t stream);
/* Adam on FP32 master weights; refreshes the BF16 copy wb when non-null. */
int mrb_cnn_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                 float eps, int step, void* wb, mrb_stream_t stream);
int mrb_cnn_to_bf16(const float* a, int64_t n, void* b, mrb_stream_t stream);
/* The same 3x3x3 convolution on the 5th-generation tensor cores: tcgen05.mma
 * with the FP32 accumulator in tensor memory, operands staged by TMA (the 27
 * taps are coordinate offsets of one 5-D tensor map; out-of-volume reads are
 * the zero padding).  Weights K-major, wk [27][N][cin]; flip != 0 reads tap
 * 26 - t (data gradient with the forward weights [27][cin][cout] read as
 * [27][N = cin][K = cout]).  Needs cin % 32 == 0, N % 16 == 0, N <= 256, and a
 * 128-voxel (H, W) patch: W % 128 == 0, or W dividing 128 with H a multiple of
 * 128 / W (mrb_cnn_tc_supported).  Dims are host values. */
int mrb_cnn_tc_supported(int cin, int ci_off, int cx, int N, int W, int H);
int mrb_cnn_conv3d_tc(const void* x, int cx, int ci_off, int cin, const void* wk, int flip, int N, int cout,
                      const float* bias, int relu, void* yb, int cyb, int yb_off, float* yf, int cyf, int yf_off,
                      int yf_acc, int Nb, int D, int H, int W, mrb_stream_t stream);
/* Reads and clears the timeout flag of the tensor-core convolution
 * (synchronous; 0 = every barrier wait completed). */
int mrb_cnn_tc_error(int* out);

#ifdef __cplusplus
}
#endif

#endif /* MRIRECON_B200_H */
