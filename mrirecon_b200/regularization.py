"""Huber-TV regularisers on the fused sm_100a TV kernel.

Mirrors the reference's regulariser plug-in surface:
* ``TVParams`` / ``TVND``      graspcg/regularization/tv_nd.py:19-238
* ``RegContext`` / ``RegParams`` graspcg/regularization/base.py:12-84
* ``RegManager.energy_and_grad`` graspcg/regularization/manager.py:38-142
  (one shard: the temporal halo of manager.py:268-301 is the identity)
* ``RegManager.add_diag`` / ``TVND.add_diag`` manager.py:145-218, tv_nd.py:113-214
* ``GraphLapParams`` / ``GraphLaplacian`` graspcg/regularization/graph_laplacian.py:11-321

``TVND.energy_grad_fixed_axes(ctx, axes)`` adds its gradient into ``ctx.g``
in place and returns the energy as a 0-D FP64 device tensor, computed by
``mrb_tv_grad`` (one fused stencil pass; no torch elementwise chain).
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple, Union

import torch

from . import _lib
from .roles import Roles

AxesSpec = Union[str, Sequence[int], Tuple[int, ...]]


@dataclass(frozen=True)
class RegParams:
    weight: float = 0.0
    eps: float = 0.0
    axes: AxesSpec = "spatial"
    isotropic: bool = True


@dataclass(frozen=True)
class TVParams(RegParams):
    weight: float = 0.0
    eps: float = 1e-3
    axes: AxesSpec = "spatial"
    isotropic: bool = True
    axis_weights: Optional[Sequence[float]] = None


@dataclass(frozen=True)
class RegContext:
    x: torch.Tensor
    g: torch.Tensor
    diag: Optional[torch.Tensor]
    roles_image: Roles
    device: torch.device
    dtype_c: torch.dtype
    dtype_r: torch.dtype
    axes_resolver: Optional[object] = None
    arena: Optional[object] = None
    write_interior_slice: Optional[Tuple[slice, ...]] = None
    ws: Optional[object] = None
    shard_index: Optional[int] = None
    halo_map: Optional[dict] = None


def tv_term_struct(params: TVParams, axes: Sequence[int], frame_period: int = 0) -> _lib.TVTerm:
    if len(axes) > 4:
        raise ValueError("the fused TV kernel supports at most 4 axes per term")
    t = _lib.TVTerm()
    t.enabled = 1 if (params.weight != 0.0 and len(axes) > 0) else 0
    t.isotropic = 1 if params.isotropic else 0
    t.weight = float(params.weight)
    t.eps = float(params.eps)
    t.naxes = len(axes)
    aw = list(params.axis_weights) if params.axis_weights is not None else [1.0] * len(axes)
    if len(aw) != len(axes):
        raise ValueError("axis_weights must match len(axes).")
    for i, (a, w) in enumerate(zip(axes, aw)):
        t.axes[i] = int(a)
        t.axis_weights[i] = float(w)
    t.frame_period = int(frame_period)
    return t


def image_geometry(x: torch.Tensor, roles: Roles):
    """(nd, S, F) of an image (F, 1, *S) with roles (1, 1, nd)."""
    if int(roles.unlike) != 1 or int(roles.like) != 1 or x.ndim != roles.total() or int(x.shape[1]) != 1:
        raise ValueError("the B200 regularisers take images (B, 1, *S) with roles (1, 1, nd); "
                         f"got shape {tuple(x.shape)} and {roles}")
    nd = int(roles.nufft)
    return nd, tuple(int(s) for s in x.shape[2:]), int(x.shape[0])


def _whole_tensor(interior, shape) -> bool:
    """True when a write-interior slice tuple covers every index of `shape`: what
    graspcg's RegManager passes for a single shard (graspcg/regularization/
    manager.py:268-301 gives slice(0, B) on the frame axis when a temporal term
    asks for a halo but there is no neighbouring shard)."""
    if interior is None:
        return True
    for sl, n in zip(interior, shape):
        if not isinstance(sl, slice):
            return False
        start, stop, step = sl.indices(int(n))
        if (start, stop, step) != (0, int(n), 1):
            return False
    return True


class TVND:
    """N-D Huber TV (reference TVND contract), evaluated by the fused CUDA kernel."""

    Params = TVParams

    def __init__(self, name: str, params: TVParams):
        self.name = name
        self.params = params

    def _resolve_axes(self, ctx: RegContext) -> Tuple[int, ...]:
        if getattr(ctx, "axes_resolver", None) is not None:
            return tuple(int(a) for a in ctx.axes_resolver(self.params.axes))
        return ctx.roles_image.resolve_axes(self.params.axes)

    def energy_grad(self, ctx: RegContext) -> torch.Tensor:
        return self.energy_grad_fixed_axes(ctx, self._resolve_axes(ctx))

    @torch.no_grad()
    def energy_grad_fixed_axes(self, ctx: RegContext, axes: Tuple[int, ...]) -> torch.Tensor:
        if len(axes) == 0 or self.params.weight == 0.0:
            return torch.zeros((), device=ctx.device, dtype=torch.float64)
        x, g = ctx.x, ctx.g
        if not _whole_tensor(ctx.write_interior_slice, x.shape):
            raise NotImplementedError("halo-extended shards are not supported by the single-GPU B200 path")
        _lib.require_cuda(x, "x")
        if x.dtype != torch.complex64 or g.dtype != torch.complex64 or not x.is_contiguous() or not g.is_contiguous():
            raise ValueError("TVND (B200) needs contiguous complex64 x and g")
        nd, S, F = image_geometry(x, ctx.roles_image)
        term = tv_term_struct(self.params, axes)
        out = torch.zeros(16, dtype=torch.float64, device=x.device)
        ws = workspace(x.device)
        Sarr = (ct.c_int * 3)(*(list(S) + [1] * (3 - nd)))
        _lib.check(_lib.load().mrb_tv_grad(nd, Sarr, F, ct.byref(term), 1, _lib.ptr(x), None, None, 0.0,
                                           _lib.ptr(g), None, _lib.ptr(g), None, 0, None, None, 0,
                                           _lib.ptr(out), _lib.ptr(ws), _lib.stream_ptr(x.device)), "tv_grad")
        return out[0]

    def halo(self, roles: Roles):
        axes = roles.resolve_axes(self.params.axes)
        return {0: 1} if any(a == 0 for a in axes) else {}

    # -- diagonal preconditioner (graspcg/regularization/tv_nd.py:113-214) ----
    @torch.no_grad()
    def add_diag(self, ctx: RegContext) -> bool:
        """ctx.diag += lambda w_a^2 / sqrt(|D_a x|^2 + eps^2) per axis (once on the
        first and last slice, twice inside), on every axis of the term, the frame
        axis included (tv_nd.py:113-164); ``mrb_tv_add_diag`` with no frame profile."""
        if ctx.diag is None or self.params.weight == 0.0:
            return False
        axes = self._resolve_axes(ctx)
        if not axes:
            return False
        _add_diag_kernel(ctx.x, ctx.diag, ctx.roles_image, [tv_term_struct(self.params, axes)], frame_profile=0)
        return True

    def majorizer_diag(self, ctx: RegContext) -> torch.Tensor:
        """0-D k = 2 lambda sum_a w_a^2 (tv_nd.py:166-185; zero when the axis
        weights do not match the axes)."""
        axes = self._resolve_axes(ctx)
        k = 0.0
        if axes and self.params.weight != 0.0:
            aw = self.params.axis_weights
            if aw is None:
                k = 2.0 * self.params.weight * float(len(axes))
            elif len(aw) == len(axes):
                k = 2.0 * self.params.weight * sum(float(w) ** 2 for w in aw)
        return torch.tensor(k, device=ctx.device, dtype=ctx.dtype_r)

    def majorizer_profile(self, ctx: RegContext) -> Optional[List[Tuple[int, torch.Tensor]]]:
        """[(0, v)] with v = 2 lambda w_0^2 (1, 2, ..., 2, 1) over the frames when the
        term includes the frame axis, else None (tv_nd.py:187-214)."""
        axes = self._resolve_axes(ctx)
        if self.params.weight == 0.0 or 0 not in axes:
            return None
        w0 = 1.0
        if self.params.axis_weights is not None:
            if len(self.params.axis_weights) != len(axes):
                return None
            w0 = float(dict(zip(axes, self.params.axis_weights)).get(0, 1.0))
        B = int(ctx.x.shape[0])
        v = torch.ones(B, device=ctx.device, dtype=ctx.dtype_r)
        if B > 2:
            v[1:-1] = 2.0
        return [(0, v * (2.0 * self.params.weight * w0 * w0))]


def _frame_profile(D: torch.Tensor, v: torch.Tensor) -> None:
    """D[f, ...] += v[f] (mrb_diag_add_frames)."""
    F = int(D.shape[0])
    vv = v.detach().to(device=D.device, dtype=torch.float32).contiguous()
    _lib.check(_lib.load().mrb_diag_add_frames(D.numel() // F, F, _lib.ptr(vv), _lib.ptr(D),
                                               _lib.stream_ptr(D.device)), "diag_add_frames")


def _add_diag_kernel(x: torch.Tensor, D: torch.Tensor, roles: Roles, terms: Sequence[_lib.TVTerm],
                     frame_profile: int) -> None:
    _lib.require_cuda(x, "x")
    _lib.require_cuda(D, "diag")
    if x.dtype != torch.complex64 or not x.is_contiguous():
        raise ValueError("the diagonal pass needs a contiguous complex64 x")
    if D.dtype != torch.float32 or not D.is_contiguous() or D.numel() != x.numel():
        raise ValueError("diag must be a contiguous float32 tensor with one entry per voxel of x")
    nd, S, F = image_geometry(x, roles)
    Sarr = (ct.c_int * 3)(*(list(S) + [1] * (3 - nd)))
    arr = (_lib.TVTerm * max(1, len(terms)))(*terms)
    _lib.check(_lib.load().mrb_tv_add_diag(nd, Sarr, F, arr, len(terms), _lib.ptr(x), int(frame_profile),
                                           _lib.ptr(D), _lib.stream_ptr(x.device)), "tv_add_diag")


@dataclass(frozen=True)
class GraphLapParams(RegParams):   # graph_laplacian.py:11-20
    weight: float = 0.0
    normalize: str = "none"        # "none": L = D - W; "rw": I - D^-1 W; "sym": I - D^-1/2 W D^-1/2
    mm_chunk_cols: int = 65536     # accepted for interface parity; the kernel tiles 32 columns at a time


class GraphLaplacian:
    """Graph Laplacian over the frame axis (graspcg/regularization/graph_laplacian.py:22-321):
    E(x) = lambda/2 sum_p <x[:, p], L x[:, p]>, gradient lambda L x.

    W (B x B, dense or sparse COO) is symmetrised as (W + W^T)/2 with a zero
    diagonal and its degrees taken on the host (:45-80); the weighted Laplacian
    lambda L is built once per device as a dense B x B float32 matrix, and
    ``mrb_graph_pass`` applies it to all pixel columns in one pass.  The
    reference's "row" spelling fails there (its code tests "rw"); here it is an
    error at construction."""

    Params = GraphLapParams

    def __init__(self, name: str, W: torch.Tensor, params: GraphLapParams):
        self.name = name
        self.params = params
        norm = (params.normalize or "none").lower()
        if norm not in ("none", "rw", "sym"):
            raise ValueError("normalize must be 'none', 'rw' or 'sym'")
        Wc = W.detach().to("cpu")
        Wd = Wc.to_dense() if Wc.is_sparse else Wc
        Wd = (0.5 * (Wd + Wd.transpose(0, 1))).to(torch.float32).clone()
        Wd.fill_diagonal_(0.0)
        self._W_cpu = Wd
        self._deg_cpu = Wd.sum(dim=1).clamp_min(0.0)
        self._cache = {}

    @property
    def frames(self) -> int:
        return int(self._W_cpu.shape[0])

    def laplacian(self) -> torch.Tensor:
        """lambda L as a dense FP64 CPU matrix."""
        W = self._W_cpu.to(torch.float64)
        deg = self._deg_cpu.to(torch.float64)
        norm = (self.params.normalize or "none").lower()
        eye = torch.eye(W.shape[0], dtype=torch.float64)
        if norm == "none":
            L = torch.diag(deg) - W
        elif norm == "rw":
            L = eye - W / deg.clamp_min(1e-20).view(-1, 1)
        else:
            dmh = torch.rsqrt(deg.clamp_min(1e-20))
            L = eye - dmh.view(-1, 1) * W * dmh.view(1, -1)
            L = 0.5 * (L + L.t())      # exactly symmetric after rounding
        return float(self.params.weight) * L

    def matrix(self, device) -> torch.Tensor:
        device = torch.device(device)
        key = (device.type, device.index)
        m = self._cache.get(key)
        if m is None:
            m = self.laplacian().to(torch.float32).contiguous().to(device)
            self._cache[key] = m
        return m

    def halo(self, roles: Roles):
        return {}

    @torch.no_grad()
    def energy_grad(self, ctx: RegContext) -> torch.Tensor:
        """ctx.g += lambda L x; returns lambda/2 sum Re<x, L x> (0-D FP64) (:171-234)."""
        if self.params.weight == 0.0:
            return torch.zeros((), device=ctx.device, dtype=torch.float64)
        x, g = ctx.x, ctx.g
        _lib.require_cuda(x, "x")
        if x.dtype != torch.complex64 or not x.is_contiguous() or (g is not None and not g.is_contiguous()):
            raise ValueError("GraphLaplacian (B200) needs contiguous complex64 x and g")
        B = int(x.shape[0])
        if B != self.frames:
            raise ValueError(f"W is {self.frames} x {self.frames} but the image has {B} frames")
        out = torch.zeros(2, dtype=torch.float64, device=x.device)
        _lib.check(_lib.load().mrb_graph_pass(0, B, x.numel() // B, _lib.ptr(self.matrix(x.device)), _lib.ptr(x),
                                              None, None, 0.0, _lib.ptr(g), None, _lib.ptr(out),
                                              _lib.ptr(workspace(x.device)), _lib.stream_ptr(x.device)),
                   "graph_pass")
        return out[0]

    def energy_grad_fixed_axes(self, ctx: RegContext, axes=None) -> torch.Tensor:
        return self.energy_grad(ctx)

    def _profile(self) -> torch.Tensor:
        norm = (self.params.normalize or "none").lower()
        v = self._deg_cpu if norm == "none" else (self._deg_cpu > 0).to(torch.float32)
        return v * float(self.params.weight)

    @torch.no_grad()
    def add_diag(self, ctx: RegContext) -> bool:
        """ctx.diag += lambda deg (none) or lambda 1{deg > 0} (rw, sym) per frame (:236-275)."""
        if ctx.diag is None or self.params.weight == 0.0:
            return False
        D = ctx.diag
        _lib.require_cuda(D, "diag")
        if D.dtype != torch.float32 or not D.is_contiguous():
            raise ValueError("diag must be contiguous float32")
        B = int(D.shape[0])
        v = self._profile().to(D.device)
        _lib.check(_lib.load().mrb_diag_add_frames(D.numel() // B, B, _lib.ptr(v), _lib.ptr(D),
                                                   _lib.stream_ptr(D.device)), "diag_add_frames")
        return True

    def majorizer_diag(self, ctx: RegContext) -> torch.Tensor:
        return torch.zeros((), device=ctx.device, dtype=ctx.dtype_r)

    def majorizer_profile(self, ctx: RegContext):
        if self.params.weight == 0.0:
            return None
        return [(0, self._profile().to(device=ctx.device, dtype=ctx.dtype_r))]


_WS = {}


def workspace(device) -> torch.Tensor:
    """Per-device reduction scratch (allocated once, outside any graph capture)."""
    device = torch.device(device)
    key = (device.type, device.index)
    ws = _WS.get(key)
    if ws is None:
        ws = torch.zeros(_lib.workspace_bytes(), dtype=torch.uint8, device=device)   # counter starts at zero
        _WS[key] = ws
    return ws


class RegManager:
    """Regulariser orchestration for one shard (graspcg/regularization/manager.py:19-142)."""

    def __init__(self, regs: Sequence[TVND], *, compile_kernels: bool = False):
        self._regs: List[TVND] = list(regs)

    @property
    def regs(self) -> List[TVND]:
        return self._regs

    def terms(self, roles: Roles, series_length: int = 0) -> List[_lib.TVTerm]:
        """Kernel descriptors of the active TV terms.  series_length > 0 splits the
        frame axis into independent series (several problems solved in one batch)."""
        from .mapping import fused_tv
        out = []
        for r0 in self._regs:
            if isinstance(r0, GraphLaplacian):
                continue                      # applied by graph_matrix / mrb_graph_pass
            r = fused_tv(r0)
            if r is None or not isinstance(r.params, TVParams):
                raise TypeError(f"regulariser {r0.name!r} is neither a TV term (possibly behind an identity map) "
                                "nor a graph Laplacian: the fused solver cannot evaluate it")
            axes = roles.resolve_axes(r.params.axes)
            t = tv_term_struct(r.params, axes, series_length)
            if t.enabled:
                out.append(t)
        if len(out) > 4:
            raise ValueError("at most 4 active TV terms")
        return out

    def graph_matrix(self, frames: int, device) -> Optional[torch.Tensor]:
        """Sum of the GraphLaplacian terms' lambda L (frames x frames float32 on
        device), or None when there is none."""
        g = [r for r in self._regs if isinstance(r, GraphLaplacian) and r.params.weight != 0.0]
        if not g:
            return None
        for r in g:
            if r.frames != frames:
                raise ValueError(f"graph regulariser {r.name!r} is over {r.frames} frames, the image has {frames}")
        L = sum(r.laplacian() for r in g)
        return L.to(torch.float32).contiguous().to(device)

    @torch.no_grad()
    def add_diag(self, ws, series_length: int = 0) -> None:
        """ws "diag" += the regularisers' diagonal at ws "var" (manager.py:145-218,
        one shard).  TV terms: a term over the frame axis adds its frame profile
        (preference (1) of the reference), any other its lagged diffusivity
        (preference (2)), in one ``mrb_tv_add_diag`` pass.  Other regularisers,
        in the reference's order: frame profile, own add_diag (which may write a
        parameter diagonal even without an image one), scalar majorizer."""
        from .mapping import fused_tv
        roles = ws.plan.roles_image
        x = ws.get("var", 0)
        D = ws.get("diag", 0) if ws.has("diag") else None
        tv = [r for r in self._regs if isinstance(r, TVND)]
        terms = RegManager(tv).terms(roles, series_length) if tv else []
        if terms and D is not None:
            _add_diag_kernel(x, D, roles, terms, frame_profile=1)
        for r in self._regs:
            if isinstance(r, TVND):
                continue
            ctx = RegContext(x=x, g=None, diag=D, roles_image=roles, device=x.device, dtype_c=x.dtype,
                             dtype_r=torch.float32, ws=ws, shard_index=0)
            # (1) frame profile, (2) the regulariser's own add_diag, (3) its scalar majorizer
            prof_fn = getattr(r, "majorizer_profile", None)
            if D is not None and callable(prof_fn):
                prof = prof_fn(ctx)
                if prof:
                    for axis, v in prof:
                        if int(axis) != 0:
                            raise NotImplementedError("only frame-axis profiles are supported")
                        _frame_profile(D, v)
                    continue
            add = getattr(r, "add_diag", None)
            if callable(add):
                add(ctx)
                continue
            maj = getattr(r, "majorizer_diag", None)
            k = maj(ctx) if callable(maj) else None
            if k is not None and D is not None:
                if k.ndim == 0:
                    _frame_profile(D, torch.full((int(D.shape[0]),), float(k)))
                elif k.ndim == 1 and int(k.shape[0]) == int(D.shape[0]):
                    _frame_profile(D, k)

    @torch.no_grad()
    def energy_and_grad(self, ws) -> torch.Tensor:
        roles = ws.plan.roles_image
        x = ws.get("var", 0)
        g = ws.get("grad", 0)
        total = torch.zeros((), device=x.device, dtype=torch.float64)
        for r in self._regs:
            axes = roles.resolve_axes(getattr(r.params, "axes", "spatial"))
            ctx = RegContext(x=x, g=g, diag=None, roles_image=roles, device=x.device, dtype_c=x.dtype,
                             dtype_r=torch.float32, ws=ws, shard_index=0)
            total = total + r.energy_grad_fixed_axes(ctx, axes)
        return total
