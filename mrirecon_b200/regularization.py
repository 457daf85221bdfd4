"""Huber-TV regularisers on the fused sm_100a TV kernel.

Mirrors the reference's regulariser plug-in surface:
* ``TVParams`` / ``TVND``      graspcg/regularization/tv_nd.py:19-238
* ``RegContext`` / ``RegParams`` graspcg/regularization/base.py:12-84
* ``RegManager.energy_and_grad`` graspcg/regularization/manager.py:38-142
  (one shard: the temporal halo of manager.py:268-301 is the identity)

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
        interior = ctx.write_interior_slice
        if interior is not None and any(s != slice(None) for s in interior):
            raise NotImplementedError("halo-extended shards are not supported by the single-GPU B200 path")
        x, g = ctx.x, ctx.g
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
        out = []
        for r in self._regs:
            if not isinstance(r.params, TVParams):
                raise TypeError(f"regulariser {r.name!r} is not a TV term")
            axes = roles.resolve_axes(r.params.axes)
            t = tv_term_struct(r.params, axes, series_length)
            if t.enabled:
                out.append(t)
        if len(out) > 4:
            raise ValueError("at most 4 active TV terms")
        return out

    @torch.no_grad()
    def add_diag(self, ws, series_length: int = 0) -> None:
        """ws "diag" += the regularisers' diagonal at ws "var" (manager.py:145-218,
        one shard, identity regularisers): a term over the frame axis adds its frame
        profile (preference (1) of the reference), any other term its lagged
        diffusivity (preference (2)).  One ``mrb_tv_add_diag`` pass for all terms."""
        if not ws.has("diag"):
            return
        roles = ws.plan.roles_image
        terms = self.terms(roles, series_length)
        if terms:
            _add_diag_kernel(ws.get("var", 0), ws.get("diag", 0), roles, terms, frame_profile=1)

    @torch.no_grad()
    def energy_and_grad(self, ws) -> torch.Tensor:
        roles = ws.plan.roles_image
        x = ws.get("var", 0)
        g = ws.get("grad", 0)
        total = torch.zeros((), device=x.device, dtype=torch.float64)
        for r in self._regs:
            axes = roles.resolve_axes(r.params.axes)
            ctx = RegContext(x=x, g=g, diag=None, roles_image=roles, device=x.device, dtype_c=x.dtype,
                             dtype_r=torch.float32)
            total = total + r.energy_grad_fixed_axes(ctx, axes)
        return total
