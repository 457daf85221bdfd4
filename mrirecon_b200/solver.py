"""Non-linear CG solver (reference ``CGSolver`` surface) on the B200 kernels.

Same constructor, ``run()``, ``result()`` and ``history()`` as
graspcg/solvers/cg.py:30-287 (``CGConfig`` fields included), for one GPU.
Two schedules compute the same iterates (up to floating-point rounding):

``schedule="reference"``  the reference's own sequence of operations
    (cg.py:162-246, line_search.py:24-203, objective.py:114-291): every
    iteration re-applies A to x and d, every line-search trial applies A^H to
    the trial residual; host reads one FP64 scalar block per trial.  Armijo
    or strong Wolfe.

``schedule="fast"`` (default, Armijo)  device-resident and host-sync free:
    the data term is quadratic in t, so with r = Ax - y and Ad = A d kept in
    HBM, ||r + t Ad||^2 and A^H(r + t Ad) = A^H r + t A^H Ad follow from FP64
    scalars and two image vectors.  One iteration is 1 forward + 1 adjoint
    NUFFT, one pass that evaluates the TV energy at all ls_max_iter+1 trial
    steps, an on-device Armijo selection (first t = beta^j that satisfies
    f(t) <= f(0) + c1 t f'(0), exactly the backtracking sequence), the fused
    gradient/statistics pass at the accepted t and one fused update pass.
    Iterations are captured in a CUDA graph and replayed.

``schedule="toeplitz"`` (Armijo)  the fast schedule with the normal operator
    A^H A applied through its Toeplitz transfer function on the 2x grid
    (``B200NUFFTAdapter.prepare_toeplitz``): A^H r and A^H A d live in image
    space (A^H r = A^H A x - A^H y, A^H y computed once by the gridded
    adjoint), Re<r, Ad> = Re<A^H r, d>, ||Ad||^2 = Re<A^H A d, d>, and ||r||^2
    follows its quadratic recurrence.  One iteration is one fused FFT pass and
    no gridding; the operator differs from the gridded A^H A by the KB
    approximation of the point-spread function (stated in the tests).

FP64 holds every objective value, dot product and line-search decision.
``stop_window`` > 0 adds the windowed relative-objective stop rule
(f_{k-W} - f_k) <= W * stop_tol * |f_k| on the accepted objectives.
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass
from typing import Dict, List, Optional

import torch

from . import _lib
from .regularization import RegManager, workspace
from .roles import Roles

# slot indices (must match csrc/ncg.cu)
S_T, S_LS_OK, S_DONE, S_REASON, S_ITER, S_F0, S_G0D, S_FT, S_GDT = range(9)
S_ERR, S_ERD, S_EDD, S_RHO_PREV, S_RHO_INIT, S_BETA = range(9, 15)
S_CUM_X, S_CUM_G, S_CUM_S, S_NTRIAL, S_NRESTART, S_NOMORE = range(15, 21)
S_GQ0, S_GQ1, S_GQ2 = range(21, 24)
# trial steps of the first energy pass (t = 0, 1, 1/2, ..., 1/64): on the GRASP workload
# the accepted steps are 2^-3 .. 2^-11, three quarters of them >= 2^-6, so the second
# pass runs in a quarter of the iterations (8 is also the largest pass the 64-register
# variant of tv_multi_kernel takes)
ARMIJO_J1 = 8
S_RED, S_EJ, S_G0D_NEXT = 24, 48, 80
MAX_TERMS = 4
REASONS = {0: "running", 1: "line-search failed", 2: "converged (tol_g/tol_step)",
           3: "relative objective change", 4: "max_iter"}
DIRS = {"fr": 0, "prplus": 1, "dy": 2}


@dataclass
class CGConfig:
    devices: object = None
    direction: str = "fr"
    ls_name: str = "armijo"
    c1: float = 1e-4
    c2: float = 0.9
    ls_beta: float = 0.5
    ls_max_iter: int = 20
    ls_zoom: bool = True
    max_iter: int = 50
    tol_g: float = 1e-4
    tol_step: float = 1e-9
    init_mode: str = "keep"
    backproj_xfactor: float = 1.0
    record_history: bool = True
    verbose: bool = False
    # B200 additions
    schedule: str = "fast"
    stop_window: int = 0
    stop_tol: float = 1e-4
    cuda_graph: bool = True
    iters_per_graph: int = 8
    # replace a non-descent direction by steepest descent instead of stopping
    # (not in the reference, whose loop ends on the line-search failure; fast schedule)
    restart: bool = False
    # > 0: the frame axis holds independent series of this many frames (a batch of
    # separate problems; temporal TV does not couple series)
    series_length: int = 0
    # diagonal D of d = beta d - g/D: "none" keeps D = 1 as the reference solve does
    # (graspcg/solvers/cg.py:95); "jacobi" sets D = alpha sum_c |S_c|^2 (alpha the
    # operator's diag_AHA_scalar) plus RegManager.add_diag at the starting image,
    # once per run.  The gradient-norm stop then reads sqrt(<g, g/D>).
    precond: str = "none"


class capture_graph:
    """Capture the launches of a block into a CUDA graph on a side stream.

    torch.cuda.graph also empties torch's device and pinned-host caches before
    every capture, so the next solve's allocations go back to cudaMalloc /
    cudaHostAlloc; that costs tens to hundreds of milliseconds at random when
    a solver (and its graph) is built per scan.  The solvers allocate nothing
    inside the captured region, so the caches can stay."""

    def __init__(self, graph: torch.cuda.CUDAGraph, device):
        self.graph = graph
        self.device = device
        self.stream = torch.cuda.Stream(device)

    def __enter__(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        self._ctx = torch.cuda.stream(self.stream)
        self._ctx.__enter__()
        self.graph.capture_begin()
        return self.graph

    def __exit__(self, *exc):
        try:
            self.graph.capture_end()
        finally:
            self._ctx.__exit__(*exc)
            torch.cuda.current_stream(self.device).wait_stream(self.stream)
        return False


class _Shard:
    def __init__(self, device):
        self.device = device


class SolverWorkspace:
    """Minimal one-shard workspace view (names of graspcg/compat/names.py:12-27)."""

    _ALIAS = {"x": "var", "g": "grad", "dx": "dir", "Ax_sh": "fwd_var_sh", "Ad_sh": "fwd_dir_sh",
              "r_sh": "resid_sh", "y": "data"}

    def __init__(self, bufs: Dict[str, torch.Tensor], roles: Roles, device):
        self._bufs = bufs
        self.plan = type("Plan", (), {"roles_image": roles})()
        self.primary_device = device
        self.num_shards = 1
        self.dtype_r = torch.float32

    def has(self, name):
        return self._ALIAS.get(name, name) in self._bufs

    def get(self, name, i=0):
        return self._bufs[self._ALIAS.get(name, name)]

    def bind(self, i, *names):
        return tuple(self.get(n, i) for n in names)

    def iter_shards(self):
        yield _Shard(self.primary_device), 0

    def list_bufs(self):
        return list(self._bufs)

    def concat(self, name):
        return self.get(name)


class CGSolver:
    def __init__(self, y: torch.Tensor, nufft_op, regm: RegManager, cfg: Optional[CGConfig] = None,
                 x0: Optional[torch.Tensor] = None):
        self.cfg = cfg or CGConfig()
        c = self.cfg
        if c.direction.lower() not in DIRS:
            raise ValueError(f"direction must be one of {list(DIRS)}")
        if c.ls_name not in ("armijo", "wolfe"):
            raise ValueError("ls_name must be 'armijo' or 'wolfe'")
        if c.schedule not in ("fast", "reference", "toeplitz"):
            raise ValueError("schedule must be 'fast', 'toeplitz' or 'reference'")
        if c.schedule != "reference" and c.ls_name != "armijo":
            raise ValueError("the fast schedules implement Armijo; use schedule='reference' for Wolfe")
        if c.schedule != "reference" and not (1 <= c.ls_max_iter <= 23):
            raise ValueError("the fast schedule evaluates at most 23 trial steps per pass")
        if c.precond not in ("none", "jacobi"):
            raise ValueError("precond must be 'none' or 'jacobi'")
        _lib.require_cuda(y, "y")
        self.lib = _lib.load()
        self.y = y.to(torch.complex64).contiguous()
        self.op = nufft_op
        self.regm = regm
        dev = y.device
        self.device = dev
        ishape = tuple(nufft_op.image_shape(y))
        roles = getattr(nufft_op, "roles_image", None)
        if not isinstance(roles, Roles):
            roles = Roles(1, 1, len(ishape) - 2)
        self.roles = roles
        self.nd = len(ishape) - 2
        self.S = tuple(int(s) for s in ishape[2:])
        self.F = int(ishape[0])
        self.terms = regm.terms(roles, c.series_length) if regm is not None else []
        # graph Laplacian terms over the frame axis: one weighted B x B matrix
        self._L = regm.graph_matrix(self.F, dev) if regm is not None and hasattr(regm, "graph_matrix") else None
        # the direction pass of a non-symmetric L ("rw") also forms L^T d for the energy slope
        self._gmode = 1 if self._L is None or bool(torch.equal(self._L, self._L.t())) else 2
        if self._gmode == 2 and c.schedule == "toeplitz":
            raise ValueError("the toeplitz schedule needs a symmetric graph Laplacian (normalize 'none' or 'sym')")
        self.nterms = len(self.terms)
        self._terms_arr = (_lib.TVTerm * max(1, self.nterms))(*self.terms)
        self._Sarr = (ct.c_int * 3)(*(list(self.S) + [1] * (3 - self.nd)))
        z = lambda shape: torch.zeros(shape, dtype=torch.complex64, device=dev)
        self.x = z(ishape) if x0 is None else x0.to(dev, torch.complex64).contiguous().clone()
        if c.init_mode == "zero":
            self.x.zero_()
        self.d, self.g = z(ishape), z(ishape)
        self.gr, self.gAd = z(ishape), z(ishape)
        self.g_prev = z(ishape) if c.direction.lower() in ("prplus", "dy") else None
        self.r, self.Ad = torch.empty_like(self.y), torch.empty_like(self.y)
        self.n_img, self.n_k = self.x.numel(), self.y.numel()
        self.D = torch.ones(ishape, dtype=torch.float32, device=dev) if c.precond == "jacobi" else None
        self._ndiag = self.n_img if self.D is not None else 0
        self.precond_alpha = None
        nslots, self.hist_cols = _lib.ncg_slot_count()
        self.s = torch.zeros(nslots, dtype=torch.float64, device=dev)
        self.hist = torch.zeros((max(1, c.max_iter), self.hist_cols), dtype=torch.float64, device=dev)
        self.ts = torch.zeros(24, dtype=torch.float64, device=dev)
        self.ws_buf = workspace(dev)
        # the first TV energy pass of each iteration needs only x and d: it runs on a
        # side stream (own reduction scratch) while the NUFFT chain runs
        self._side = torch.cuda.Stream(dev)
        self.ws_side = torch.zeros(_lib.workspace_bytes(), dtype=torch.uint8, device=dev)
        self.cfg_dev = torch.tensor([c.c1, c.ls_beta, c.ls_max_iter, c.max_iter, c.tol_g, c.tol_step,
                                     c.stop_window, c.stop_tol, DIRS[c.direction.lower()], c.max_iter],
                                    dtype=torch.float64, device=dev)
        self._toep = None
        if c.schedule == "toeplitz":
            backend = getattr(nufft_op, "backend", nufft_op)
            if not hasattr(backend, "AHA"):
                raise ValueError("the toeplitz schedule needs the B200 NUFFT backend")
            if not getattr(backend, "_toeplitz", False):
                backend.prepare_toeplitz()
            self._toep = backend
            self.ahy = z(ishape)
            self._dot_a = (ct.c_void_p * 2)(_lib.ptr(self.gr), _lib.ptr(self.gAd))
            self._dot_b = (ct.c_void_p * 2)(_lib.ptr(self.d), _lib.ptr(self.d))
            self._dot_w = (ct.c_void_p * 2)(None, None)
        bufs = {"var": self.x, "grad": self.g, "dir": self.d, "data": self.y, "fwd_dir_sh": self.Ad,
                "resid_sh": self.r}
        if self.D is not None:
            bufs["diag"] = self.D
        self.ws = SolverWorkspace(bufs, roles, dev)
        self.iter = 0
        self._graph = None
        self._host_hist: List[dict] = []
        self.n_forward = 0
        self.n_adjoint = 0
        # kernel launches of the library: issued eagerly, recorded per graph, graph replays
        self.launch_stats = {"eager": 0, "per_graph": 0, "replays": 0}

    def reset(self, x0: Optional[torch.Tensor] = None) -> "CGSolver":
        """Start a new solve from x0 (default zeros), keeping buffers and the captured graph."""
        if x0 is None:
            self.x.zero_()
        else:
            self.x.copy_(x0)
        self.d.zero_()
        self.iter = 0
        self._host_hist = []
        self.hist.zero_()
        self.s.zero_()
        return self

    # ----------------------------------------------------------------- helpers
    def _st(self):
        return _lib.stream_ptr(self.device)

    def _A(self, x, out):
        self.op.A(x, out=out)
        self.n_forward += 1

    def _AH(self, y, out):
        self.op.AH(y, out=out)
        self.n_adjoint += 1

    def _tv_grad(self, d, t_dev, t_host, g_base, g_dir, g_out, out, skip=None, skip_if_zero=0):
        _lib.check(self.lib.mrb_tv_grad(self.nd, self._Sarr, self.F, self._terms_arr, self.nterms,
                                        _lib.ptr(self.x), _lib.ptr(d), t_dev, float(t_host), _lib.ptr(g_base),
                                        _lib.ptr(g_dir), _lib.ptr(g_out), _lib.ptr(self.D), self._ndiag,
                                        _lib.ptr(self.g_prev), skip,
                                        skip_if_zero, out, _lib.ptr(self.ws_buf), self._st()), "tv_grad")

    def _slot(self, i):
        return self.s.data_ptr() + 8 * i

    def _graph_pass(self, mode, d, t_dev, t_host, acc, out, skip=None):
        """mrb_graph_pass on the current x (no-op without graph terms)."""
        if self._L is None:
            return
        _lib.check(self.lib.mrb_graph_pass(mode, self.F, self.n_img // self.F, _lib.ptr(self._L), _lib.ptr(self.x),
                                           _lib.ptr(d), t_dev, float(t_host), _lib.ptr(acc), skip, out,
                                           _lib.ptr(self.ws_buf), self._st()), "graph_pass")

    def _quad_fold(self, phase):
        if self._L is not None:
            _lib.check(self.lib.mrb_ncg_quad_fold(_lib.ptr(self.s), phase, self._st()), "quad_fold")

    def _backend(self):
        return getattr(self.op, "backend", self.op)

    @torch.no_grad()
    def build_preconditioner(self) -> Optional[torch.Tensor]:
        """Fill D for precond="jacobi" at the current x (no-op for "none")."""
        if self.D is None:
            return None
        backend = self._backend()
        maps = getattr(backend, "_maps", None)
        if self.precond_alpha is None:
            if not hasattr(backend, "diag_AHA_scalar") or maps is None:
                raise ValueError("precond='jacobi' needs an operator with diag_AHA_scalar and coil maps")
            self.precond_alpha = float(backend.diag_AHA_scalar())
        P = self.n_img // self.F
        _lib.check(self.lib.mrb_precond_init(P, self.F, int(maps.shape[0]), _lib.ptr(maps),
                                             float(self.precond_alpha), 0.0, _lib.ptr(self.D), self._st()),
                   "precond_init")
        if self.regm is not None:
            self.regm.add_diag(self.ws, self.cfg.series_length)
        return self.D

    # ------------------------------------------------------------- fast path
    def _prime_fast(self):
        self.build_preconditioner()
        st = self._st()
        self._A(self.x, self.Ad)                               # Ax (into the Ad buffer)
        _lib.check(self.lib.mrb_kspace_pass(1, self.n_k, _lib.ptr(self.r), None, _lib.ptr(self.Ad),
                                            _lib.ptr(self.y), None, 0.0, None, self._slot(S_ERR),
                                            _lib.ptr(self.ws_buf), st), "kspace_pass")
        if self._toep is not None:
            # A^H r = A^H A x - A^H y (Toeplitz normal operator, gridded A^H y)
            self._AH(self.y, self.ahy)
            self._toep.AHA(self.x, out=self.gr)
            self.gr.sub_(self.ahy)
        else:
            self._AH(self.r, self.gr)
        # graph terms: gr += L x, q0 = 1/2 <x, L x>, err += 2 q0
        self._graph_pass(0, None, None, 0.0, self.gr, self._slot(S_GQ0))
        self._quad_fold(0)
        self._tv_grad(None, None, 0.0, self.gr, None, self.g, self._slot(S_RED))
        _lib.check(self.lib.mrb_ncg_steepest(self.n_img, _lib.ptr(self.d), _lib.ptr(self.g), _lib.ptr(self.g_prev),
                                             _lib.ptr(self.D), self._ndiag, self._slot(S_G0D), _lib.ptr(self.ws_buf),
                                             st), "steepest")
        J = self.cfg.ls_max_iter + 1
        _lib.check(self.lib.mrb_ncg_set_steps(_lib.ptr(self.ts), J, float(self.cfg.ls_beta), st), "set_steps")
        for i, v in ((S_DONE, 0.0), (S_REASON, 0.0), (S_ITER, float(self.iter)), (S_RHO_INIT, 0.0),
                     (S_CUM_X, 0.0), (S_CUM_G, 0.0), (S_CUM_S, 0.0), (S_LS_OK, 0.0)):
            self.s[i] = v

    def _iteration_fast(self):
        st = self._st()
        lib, ws = self.lib, _lib.ptr(self.ws_buf)
        J = self.cfg.ls_max_iter + 1
        J1 = min(J, ARMIJO_J1)
        main = torch.cuda.current_stream(self.device)
        self._side.wait_stream(main)
        with torch.cuda.stream(self._side):
            _lib.check(lib.mrb_tv_multi(self.nd, self._Sarr, self.F, self._terms_arr, self.nterms,
                                        _lib.ptr(self.x), _lib.ptr(self.d), _lib.ptr(self.ts), J1,
                                        self._slot(S_DONE), self._slot(S_EJ), _lib.ptr(self.ws_side),
                                        _lib.stream_ptr(self.device)), "tv_multi")
        if self._toep is not None:
            self._toep.AHA(self.d, out=self.gAd)
            # graph terms join the normal operator before Re<gr, d>, Re<gAd, d>
            self._graph_pass(self._gmode, self.d, None, 0.0, self.gAd, self._slot(S_GQ1), skip=self._slot(S_DONE))
            _lib.check(lib.mrb_dots_f64(self.n_img, 2, self._dot_a, self._dot_b, self._dot_w, 0,
                                        self._slot(S_ERD), ws, st), "dots")
        else:
            self._A(self.d, self.Ad)
            _lib.check(lib.mrb_kspace_pass(0, self.n_k, _lib.ptr(self.r), _lib.ptr(self.Ad), None, None, None,
                                           0.0, self._slot(S_DONE), self._slot(S_ERR), ws, st), "kspace_pass")
            self._AH(self.Ad, self.gAd)
            # graph terms: gAd += L d, q1 = Re<x, L d>, q2 = Re<d, L d> folded into the data scalars
            self._graph_pass(self._gmode, self.d, None, 0.0, self.gAd, self._slot(S_GQ1), skip=self._slot(S_DONE))
            self._quad_fold(1)
        # Armijo in two phases: the TV energies of the first ARMIJO_J1 trial steps
        # (side stream, above), the rest only when none of those is accepted
        main.wait_stream(self._side)
        _lib.check(lib.mrb_ncg_armijo_phase(_lib.ptr(self.s), _lib.ptr(self.cfg_dev), J1, 1, st), "armijo 1")
        if J > J1:
            _lib.check(lib.mrb_tv_multi(self.nd, self._Sarr, self.F, self._terms_arr, self.nterms,
                                        _lib.ptr(self.x), _lib.ptr(self.d), _lib.ptr(self.ts) + 8 * J1, J - J1,
                                        self._slot(S_NOMORE), self._slot(S_EJ + J1), ws, st), "tv_multi 2")
            _lib.check(lib.mrb_ncg_armijo_phase(_lib.ptr(self.s), _lib.ptr(self.cfg_dev), J1, 2, st), "armijo 2")
        self._tv_grad(self.d, self._slot(S_T), 0.0, self.gr, self.gAd, self.g, self._slot(S_RED),
                      skip=self._slot(S_LS_OK), skip_if_zero=1)
        _lib.check(lib.mrb_ncg_control(_lib.ptr(self.s), _lib.ptr(self.hist), _lib.ptr(self.cfg_dev),
                                       self.nterms, 1, st), "ncg_control")
        _lib.check(lib.mrb_ncg_update(self.n_img, _lib.ptr(self.x), _lib.ptr(self.d), _lib.ptr(self.g),
                                      _lib.ptr(self.gr), _lib.ptr(self.gAd), _lib.ptr(self.g_prev),
                                      _lib.ptr(self.D), self._ndiag,
                                      _lib.ptr(self.s), ws, st), "ncg_update")
        if self.cfg.restart:
            _lib.check(lib.mrb_ncg_restart(self.n_img, _lib.ptr(self.d), _lib.ptr(self.g), _lib.ptr(self.D),
                                           self._ndiag,
                                           _lib.ptr(self.s), st), "ncg_restart")
        if self._toep is not None:
            _lib.check(lib.mrb_ncg_err_step(_lib.ptr(self.s), st), "err_step")
        else:
            _lib.check(lib.mrb_kspace_pass(2, self.n_k, _lib.ptr(self.r), _lib.ptr(self.Ad), None, None,
                                           self._slot(S_T), 0.0, self._slot(S_DONE), None, ws, st), "kspace_pass")
            self._quad_fold(2)

    def _plan(self):
        """The B200 NUFFT plan behind the operator (front-end or adapter), if any."""
        backend = getattr(self.op, "backend", self.op)
        return getattr(backend, "plan", None)

    def _skip_on_done(self, on: bool):
        plan = self._plan()
        if plan is not None and hasattr(plan, "set_skip_flag"):
            plan.set_skip_flag(self._slot(S_DONE) if on else None)

    def _run_fast(self, max_iter):
        try:
            self._run_fast_body(max_iter)
        finally:
            self._skip_on_done(False)

    def _fast_setup(self, max_iter) -> bool:
        """Size the history for max_iter; True when a captured graph is still valid."""
        self.cfg_dev[3] = float(max_iter)
        ok = True
        if self.hist.shape[0] < max_iter:
            self.hist = torch.zeros((max_iter, self.hist_cols), dtype=torch.float64, device=self.device)
            self._graph = None                      # the captured graph wrote the old history buffer
            ok = False
        self.cfg_dev[9] = float(self.hist.shape[0])
        return ok

    def _run_fast_body(self, max_iter):
        c = self.cfg
        self._fast_setup(max_iter)
        n0 = _lib.launch_count()
        self._prime_fast()
        # iterations past the stop (graph replays) skip the operator kernels
        self._skip_on_done(True)
        self._iteration_fast()                                # eager: warms every lazy allocation
        self.launch_stats["eager"] += _lib.launch_count() - n0
        done = lambda: bool(self.s[S_DONE].item())
        if done():
            return
        use_graph = c.cuda_graph
        if use_graph and self._graph is None:
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            n1 = _lib.launch_count()
            with capture_graph(g, self.device):
                for _ in range(max(1, c.iters_per_graph)):
                    self._iteration_fast()
            self.launch_stats["per_graph"] = _lib.launch_count() - n1
            self._graph = g
            # capture does not execute: nothing ran
        while not done():
            if use_graph:
                self._graph.replay()
                self.launch_stats["replays"] += 1
            else:
                n2 = _lib.launch_count()
                for _ in range(max(1, c.iters_per_graph)):
                    self._iteration_fast()
                self.launch_stats["eager"] += _lib.launch_count() - n2

    # -------------------------------------------------------- reference path
    def _fg(self, t: float, out: torch.Tensor):
        """f(t), f'(t) at x + t d; fills g (objective.py:184-291)."""
        st = self._st()
        _lib.check(self.lib.mrb_kspace_pass(1, self.n_k, _lib.ptr(self.r), _lib.ptr(self.Ad), _lib.ptr(self.Ax),
                                            _lib.ptr(self.y), None, float(t), None, out.data_ptr(),
                                            _lib.ptr(self.ws_buf), st), "kspace_pass")
        self._AH(self.r, self.gr)
        self._graph_pass(0, self.d, None, t, self.gr, out.data_ptr() + 8 * 20)
        self._tv_grad(self.d, None, t, self.gr, None, self.g, out.data_ptr() + 8 * 8)
        v = out.tolist()
        f = 0.5 * v[0] + sum(v[8:8 + self.nterms]) + (v[20] if self._L is not None else 0.0)
        return f, v[8 + MAX_TERMS], v

    def _armijo_ref(self, out):
        c = self.cfg
        self._A(self.x, self.Ax)
        self._A(self.d, self.Ad)
        f0, g0d, _ = self._fg(0.0, out)
        self._ls0 = (f0, g0d)
        if not (g0d < 0) or math.isnan(g0d) or math.isinf(g0d):
            return False, 0.0, f0, g0d, None
        t = 1.0
        f_t = g_t = float("nan")
        v = None
        for _ in range(c.ls_max_iter):
            f_t, g_t, v = self._fg(t, out)
            if f_t <= f0 + c.c1 * t * g0d:
                return True, t, f_t, g_t, v
            t *= c.ls_beta
        return False, t, f_t, g_t, v

    def _wolfe_ref(self, out):
        c = self.cfg
        self._A(self.x, self.Ax)
        self._A(self.d, self.Ad)
        f0, g0d, _ = self._fg(0.0, out)
        self._ls0 = (f0, g0d)
        if not (g0d < 0) or math.isnan(g0d) or math.isinf(g0d):
            return False, 0.0, f0, g0d, None
        t, t_prev, f_prev, g_prev = 1.0, 0.0, f0, g0d
        for i in range(c.ls_max_iter):
            f_t, g_t, v = self._fg(t, out)
            if (f_t > f0 + c.c1 * t * g0d) or (i > 0 and f_t >= f_prev):
                return self._zoom_ref(t_prev, f_prev, t, f0, g0d, out)
            if abs(g_t) <= c.c2 * abs(g0d):
                return True, t, f_t, g_t, v
            if g_t >= 0:
                return self._zoom_ref(t, f_t, t_prev, f0, g0d, out)
            t_prev, f_prev, g_prev = t, f_t, g_t
            t = min(2.0 * t, 1e6)
        return False, t_prev, f_prev, g_prev, None

    def _zoom_ref(self, t_lo, f_lo, t_hi, f0, g0d, out):
        c = self.cfg
        for _ in range(c.ls_max_iter):
            t_mid = 0.5 * (t_lo + t_hi)
            f_mid, g_mid, v = self._fg(t_mid, out)
            if (f_mid > f0 + c.c1 * t_mid * g0d) or (f_mid >= f_lo):
                t_hi = t_mid
            else:
                if abs(g_mid) <= c.c2 * abs(g0d):
                    return True, t_mid, f_mid, g_mid, v
                if g_mid * (t_hi - t_lo) >= 0:
                    t_hi = t_lo
                t_lo, f_lo = t_mid, f_mid
        f_lo, g_lo, v = self._fg(t_lo, out)
        return True, t_lo, f_lo, g_lo, v

    def _run_reference(self, max_iter):
        c = self.cfg
        st = self._st()
        n0 = _lib.launch_count()
        try:
            self._run_reference_body(max_iter, c, st)
        finally:
            self.launch_stats["eager"] += _lib.launch_count() - n0

    def _run_reference_body(self, max_iter, c, st):
        self.Ax = getattr(self, "Ax", None)
        if self.Ax is None:
            self.Ax = torch.empty_like(self.y)
        out = torch.zeros(24, dtype=torch.float64, device=self.device)
        self.build_preconditioner()
        # prime (cg.py:178-190): f_g(0) at x with d as it is, then d = -g/D
        self._A(self.x, self.Ax)
        self._A(self.d, self.Ad)
        self._fg(0.0, out)
        _lib.check(self.lib.mrb_ncg_steepest(self.n_img, _lib.ptr(self.d), _lib.ptr(self.g), _lib.ptr(self.g_prev),
                                             _lib.ptr(self.D), self._ndiag, self._slot(S_G0D), _lib.ptr(self.ws_buf),
                                             st), "steepest")
        rho_prev = None
        cum = {"x": 0.0, "g": 0.0, "s": 0.0}
        fa: List[float] = []
        ls = self._wolfe_ref if c.ls_name == "wolfe" else self._armijo_ref
        direction = c.direction.lower()
        for k in range(max_iter):
            self.iter = k
            ok, t, f_t, g_t, v = ls(out)
            if not ok:
                self.stop_reason = REASONS[1]
                break
            r0 = 8 + MAX_TERMS
            xn = math.sqrt(max(v[r0 + 2], 0.0))
            sn = math.sqrt(max(v[r0 + 3], 0.0))
            rho = v[r0 + 1]
            gn = math.sqrt(max(rho, 0.0))
            cum["x"] += xn
            cum["g"] += gn
            cum["s"] += sn
            f0, g0d = self._ls0
            if not fa:
                fa.append(f0)
            fa.append(f_t)
            self._host_hist.append(dict(iter=k, f=f0, gdot=g0d, gdot_at_step=g_t, step=t, xnorm=cum["x"],
                                        gnorm=cum["g"], stepnorm=cum["s"], xnorm_iter=xn, gnorm_iter=gn,
                                        stepnorm_iter=sn, f_accepted=f_t))
            done, reason = False, 0
            if gn <= (1.0 + xn) * c.tol_g and sn <= (1.0 + xn) * c.tol_step:
                done, reason = True, 2
            elif c.stop_window > 0 and len(fa) - 1 >= c.stop_window:
                fk, fw = fa[-1], fa[-1 - c.stop_window]
                if fw - fk <= c.stop_window * c.stop_tol * abs(fk):
                    done, reason = True, 3
            beta = 0.0
            if not done:
                if direction == "fr":
                    if rho_prev is None:
                        rho_prev = rho
                    beta = rho / max(rho_prev, 1e-20)
                    rho_prev = rho
                elif direction == "prplus":
                    beta = max((rho - v[r0 + 4]) / max(v[r0 + 5], 1e-20), 0.0)
                else:
                    beta = rho / max(v[r0 + 0] - v[r0 + 6], 1e-20)
            self.s[S_T] = t
            self.s[S_LS_OK] = 1.0
            self.s[S_DONE] = 1.0 if done else 0.0
            self.s[S_BETA] = beta
            _lib.check(self.lib.mrb_ncg_update(self.n_img, _lib.ptr(self.x), _lib.ptr(self.d), _lib.ptr(self.g),
                                               None, None, _lib.ptr(self.g_prev), _lib.ptr(self.D), self._ndiag,
                                               _lib.ptr(self.s),
                                               _lib.ptr(self.ws_buf), st), "ncg_update")
            if done:
                self.stop_reason = REASONS[reason]
                break
        else:
            self.stop_reason = REASONS[4]

    # ------------------------------------------------------------------- API
    @torch.no_grad()
    def run(self, max_iter: Optional[int] = None, tol_g: Optional[float] = None,
            tol_step: Optional[float] = None) -> "CGSolver":
        c = self.cfg
        if tol_g is not None:
            c.tol_g = float(tol_g)
        if tol_step is not None:
            c.tol_step = float(tol_step)
        self.cfg_dev[4] = float(c.tol_g)
        self.cfg_dev[5] = float(c.tol_step)
        max_iter = int(max_iter or c.max_iter)
        with torch.cuda.device(self.device):
            if c.schedule in ("fast", "toeplitz"):
                self._run_fast(max_iter)
                self.iter = int(self.s[S_ITER].item())
                self.stop_reason = REASONS[int(self.s[S_REASON].item())]
            else:
                self._run_reference(max_iter)
        return self

    @property
    def restarts(self) -> int:
        """Directions replaced by steepest descent in the last run (CGConfig.restart)."""
        return int(self.s[S_NRESTART].item())

    def launches(self) -> int:
        """Library kernel launches executed so far by this solver."""
        ls = self.launch_stats
        return ls["eager"] + ls["per_graph"] * ls["replays"]

    @torch.no_grad()
    def result(self) -> torch.Tensor:
        return self.x.detach()

    def history(self) -> List[dict]:
        if self.cfg.schedule == "reference":
            return list(self._host_hist)
        n = int(self.s[S_ITER].item())
        h = self.hist[:n].cpu().tolist()
        keys = ("f", "gdot", "gdot_at_step", "step", "xnorm", "gnorm", "stepnorm", "xnorm_iter", "gnorm_iter",
                "stepnorm_iter", "f_accepted")
        return [dict(iter=k, **{kk: row[i] for i, kk in enumerate(keys)}) for k, row in enumerate(h)]

    def objective(self) -> float:
        """0.5 ||A x - y||^2 + R(x) at the current x (FP64), recomputed from scratch."""
        out = torch.zeros(24, dtype=torch.float64, device=self.device)
        tmp = torch.empty_like(self.y)
        self._A(self.x, tmp)
        _lib.check(self.lib.mrb_kspace_pass(1, self.n_k, _lib.ptr(tmp), None, _lib.ptr(tmp), _lib.ptr(self.y),
                                            None, 0.0, None, out.data_ptr(), _lib.ptr(self.ws_buf), self._st()),
                   "kspace_pass")
        self.regularizer_energy_into(self.x, out)
        v = out.tolist()
        return 0.5 * v[0] + self.regularizer_energy_from(v)

    def regularizer_energy_into(self, x: torch.Tensor, out: torch.Tensor) -> None:
        """R(x) terms of image x into the FP64 device vector out (24 values; TV terms
        at 8 + i, the graph term at 20), on the device without a host read."""
        _lib.check(self.lib.mrb_tv_grad(self.nd, self._Sarr, self.F, self._terms_arr, self.nterms,
                                        _lib.ptr(x), None, None, 0.0, None, None, None, None, 0, None,
                                        None, 0, out.data_ptr() + 64, _lib.ptr(self.ws_buf), self._st()),
                   "tv_grad")
        if self._L is not None:
            _lib.check(self.lib.mrb_graph_pass(0, self.F, self.n_img // self.F, _lib.ptr(self._L), _lib.ptr(x),
                                               None, None, 0.0, None, None, out.data_ptr() + 8 * 20,
                                               _lib.ptr(self.ws_buf), self._st()), "graph_pass")

    def regularizer_energy_from(self, v: List[float]) -> float:
        """R from the values regularizer_energy_into wrote (read to the host as v)."""
        return sum(v[8:8 + self.nterms]) + (v[20] if self._L is not None else 0.0)
