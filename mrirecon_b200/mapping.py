"""Mapped regularisers: a regulariser evaluated on u = Op(x) (or on u built from
parameter buffers), with its gradient pushed back through the operator.

Mirrors graspcg/regularization/mapping.py and wrappers.py for one shard:

* ``IdentityOp``        mapping.py:31-42
* ``ScaleOp``           mapping.py:44-110 (per-frame factors 1/s from ``ws.scale``)
* ``TemporalBasisOp``   mapping.py:112-236 (u = U V, gradient into ``ws[grad_key]``)
* ``ComposeOp``         mapping.py:238-276
* ``LinOpAdapter``      mapping.py:278-294
* ``MappedRegularizer`` mapping.py:296-414
* ``Transformed``       wrappers.py:9-130 (operator-aware diagonal)

The frame-axis products (U V, U^H g_u, |U|^T k, diag(1/s) z) run in
``mrb_frame_mix`` / ``mrb_frame_mix_real``: one pass over the parameter or
image columns with the small matrix in shared memory.  Shards with a halo are
not supported (one GPU); the interior slice is the whole frame axis.
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence, Tuple

import torch

from . import _lib
from .regularization import RegContext, TVND
from .roles import Roles


def _mix(M: torch.Tensor, inp: torch.Tensor, out: torch.Tensor, conj_t: bool = False, accumulate: bool = False):
    """out (R_out, ...) (+)= M inp over the leading axis (complex64), M (R_out, R_in)
    or, with conj_t, M (R_in, R_out) applied as M^H."""
    _lib.require_cuda(inp, "input")
    Ri, Ro = int(inp.shape[0]), int(out.shape[0])
    N = inp.numel() // Ri
    if out.numel() // Ro != N or not inp.is_contiguous() or not out.is_contiguous():
        raise ValueError("frame mix: contiguous (rows, ...) tensors with equal trailing sizes")
    Mc = M.to(device=inp.device, dtype=torch.complex64).contiguous()
    if tuple(Mc.shape) != ((Ri, Ro) if conj_t else (Ro, Ri)):
        raise ValueError(f"frame mix: matrix {tuple(Mc.shape)} does not match {Ro} x {Ri} rows")
    _lib.check(_lib.load().mrb_frame_mix(Ro, Ri, N, _lib.ptr(Mc), int(conj_t), _lib.ptr(inp), _lib.ptr(out),
                                         int(accumulate), _lib.stream_ptr(inp.device)), "frame_mix")
    return out


def _mix_real(M: torch.Tensor, inp: torch.Tensor, out: torch.Tensor, transpose: bool = False,
              accumulate: bool = False):
    """Real counterpart of _mix (float32 data and matrix; transpose applies M^T)."""
    _lib.require_cuda(inp, "input")
    Ri, Ro = int(inp.shape[0]), int(out.shape[0])
    N = inp.numel() // Ri
    if out.numel() // Ro != N or not inp.is_contiguous() or not out.is_contiguous():
        raise ValueError("frame mix: contiguous (rows, ...) tensors with equal trailing sizes")
    if inp.dtype != torch.float32 or out.dtype != torch.float32:
        raise ValueError("frame mix (real): float32 data")
    Mr = M.to(device=inp.device, dtype=torch.float32).contiguous()
    _lib.check(_lib.load().mrb_frame_mix_real(Ro, Ri, N, _lib.ptr(Mr), int(transpose), _lib.ptr(inp), _lib.ptr(out),
                                              int(accumulate), _lib.stream_ptr(inp.device)), "frame_mix_real")
    return out


def _add_profile(D: torch.Tensor, v: torch.Tensor) -> None:
    """D[f, ...] += v[f] (mrb_diag_add_frames)."""
    F = int(D.shape[0])
    vv = v.to(device=D.device, dtype=torch.float32).contiguous()
    _lib.check(_lib.load().mrb_diag_add_frames(D.numel() // F, F, _lib.ptr(vv), _lib.ptr(D),
                                               _lib.stream_ptr(D.device)), "diag_add_frames")


def _whole(interior, ndim):
    if interior is not None and any(s != slice(None) for s in interior):
        raise NotImplementedError("halo-extended shards are not supported by the single-GPU B200 path")
    return (slice(None),) * ndim


# ------------------------------------------------------------------ operators
class IdentityOp:
    def forward_apply(self, z_ext, ctx, interior):
        return z_ext

    def adjoint_apply(self, grad_u_int, ctx, interior):
        return grad_u_int

    def halo_extra(self, roles: Roles) -> Dict[int, int]:
        return {}

    def roles_for_output(self, roles: Roles) -> Roles:
        return roles

    def diag_push(self, k_u_int, ctx, interior):
        return k_u_int

    def diag_push_profile(self, axis, v1d, ctx, interior):
        return (axis, v1d)


class ScaleOp:
    """u = (1/s) x per frame, 1/s from ``ws.scale.inv_for_shard(shard, anchor)``;
    the identity when the workspace has no scale."""

    @staticmethod
    def _inv(ctx, anchor):
        ws, i = getattr(ctx, "ws", None), getattr(ctx, "shard_index", None)
        if ws is None or i is None or not hasattr(ws, "scale") or ws.scale is None:
            return None
        inv = ws.scale.inv_for_shard(ws.shard_for_index(i), anchor=anchor)
        return inv.reshape(int(inv.shape[0])).detach().to("cpu", torch.float32)   # F host values

    def forward_apply(self, z_ext, ctx, interior):
        _whole(interior, z_ext.ndim)
        inv = self._inv(ctx, z_ext)
        if inv is None:
            return z_ext
        return _mix(torch.diag(inv), z_ext.contiguous(), torch.empty_like(z_ext))

    def adjoint_apply(self, grad_u_int, ctx, interior):
        inv = self._inv(ctx, grad_u_int)
        if inv is None:
            return grad_u_int
        return _mix(torch.diag(inv), grad_u_int.contiguous(), torch.empty_like(grad_u_int))

    def halo_extra(self, roles):
        return {}

    def roles_for_output(self, roles):
        return roles

    def diag_push(self, k_u_int, ctx, interior):
        inv = self._inv(ctx, k_u_int)
        if inv is None:
            return k_u_int
        k = k_u_int.to(torch.float32).contiguous()
        return _mix_real(torch.diag(inv * inv), k, torch.empty_like(k))

    def diag_push_profile(self, axis, v1d, ctx, interior):
        if axis != 0:
            return (axis, v1d)
        inv = self._inv(ctx, ctx.x)
        if inv is None:
            return (axis, v1d)
        return (axis, v1d.detach().to("cpu", torch.float32) * inv * inv)


@dataclass
class TemporalBasisOp:
    """Parameter-space operator u = U V (U (B, K), V = ws[param_key] (K, ...));
    the adjoint adds U^H g_u into ws[grad_key] and returns zeros for x."""
    U: torch.Tensor
    param_key: str = "V"
    grad_key: str = "g_V"
    diag_key: str = "diag_V"

    def _U(self, B, device):
        if int(self.U.shape[0]) < B:
            raise ValueError(f"U has {int(self.U.shape[0])} rows, the image {B} frames")
        return self.U[:B].to(device=device)

    def forward_apply(self, z_ext, ctx, interior):
        assert ctx.ws is not None and ctx.shard_index is not None, "TemporalBasisOp requires ws/shard_index"
        _whole(interior, z_ext.ndim)
        V = ctx.ws.get(self.param_key, ctx.shard_index)
        B = int(ctx.ws.get("var", ctx.shard_index).shape[0])
        u = torch.empty((B,) + tuple(V.shape[1:]), dtype=torch.complex64, device=V.device)
        return _mix(self._U(B, V.device), V.to(torch.complex64).contiguous(), u)

    def adjoint_apply(self, grad_u_int, ctx, interior):
        assert ctx.ws is not None and ctx.shard_index is not None
        ws, i = ctx.ws, ctx.shard_index
        gV = ws.get(self.grad_key, i)
        B = int(ws.get("var", i).shape[0])
        if gV.dtype != torch.complex64 or not gV.is_contiguous():
            raise ValueError("the parameter gradient buffer must be contiguous complex64")
        _mix(self._U(B, gV.device), grad_u_int.contiguous(), gV, conj_t=True, accumulate=True)
        return torch.zeros_like(ctx.x)

    def halo_extra(self, roles):
        return {}

    def roles_for_output(self, roles):
        return roles

    def diag_push(self, k_u_int, ctx, interior):
        """diag_V[k, p] += sum_t |U_tk|^2 k_u[t, p]; terminal (returns None)."""
        ws, i = ctx.ws, ctx.shard_index
        try:
            V = ws.get(self.param_key, i)
            Dp = ws.get(self.diag_key, i)
        except Exception:
            return None
        B = int(ws.get("var", i).shape[0])
        U2 = self.U[:B].detach().to("cpu").abs().to(torch.float32) ** 2   # (B, K), host
        k = k_u_int.to(device=V.device, dtype=torch.float32).reshape(B, -1).contiguous()
        _mix_real(U2, k, Dp, transpose=True, accumulate=True)
        return None

    def diag_push_profile(self, axis, v1d, ctx, interior):
        if axis != 0:
            return None
        ws, i = ctx.ws, ctx.shard_index
        try:
            V = ws.get(self.param_key, i)
            Dp = ws.get(self.diag_key, i)
        except Exception:
            return None
        B = int(ws.get("var", i).shape[0])
        U2 = self.U[:B].detach().to("cpu").abs().to(torch.float64) ** 2
        DV = U2.transpose(0, 1) @ v1d.detach().to("cpu", torch.float64).reshape(B)   # (K,): K x B host flops
        _add_profile(Dp, DV)
        return None


class ComposeOp:
    """Forward left to right, adjoint and diagonal pushes right to left."""

    def __init__(self, ops: Sequence[Any]):
        self.ops: List[Any] = list(ops)

    def forward_apply(self, z_ext, ctx, interior):
        u = z_ext
        for op in self.ops:
            u = op.forward_apply(u, ctx, interior)
        return u

    def adjoint_apply(self, grad_u_int, ctx, interior):
        g = grad_u_int
        for op in reversed(self.ops):
            g = op.adjoint_apply(g, ctx, interior)
        return g

    def halo_extra(self, roles):
        merged: Dict[int, int] = {}
        for op in self.ops:
            for ax, k in op.halo_extra(roles).items():
                merged[ax] = max(merged.get(ax, 0), int(k))
        return merged

    def roles_for_output(self, roles):
        for op in self.ops:
            roles = op.roles_for_output(roles)
        return roles

    def diag_push(self, k_u_int, ctx, interior):
        km = k_u_int
        for op in reversed(self.ops):
            km = op.diag_push(km, ctx, interior)
            if km is None:
                return None
        return km

    def diag_push_profile(self, axis, v1d, ctx, interior):
        pair = (axis, v1d)
        for op in reversed(self.ops):
            if pair is None:
                return None
            pair = op.diag_push_profile(pair[0], pair[1], ctx, interior)
        return pair


class LinOpAdapter:
    """Adapt an object with fwd(x) / adj(y) to the operator interface."""

    def __init__(self, linop):
        self.linop = linop

    def forward_apply(self, z_ext, ctx, interior):
        return self.linop.fwd(z_ext)

    def adjoint_apply(self, grad_u_int, ctx, interior):
        return self.linop.adj(grad_u_int)

    def halo_extra(self, roles):
        return {}

    def roles_for_output(self, roles):
        return roles


# -------------------------------------------------------------- regularisers
def _sub_ctx(ctx: RegContext, u: torch.Tensor, g_u: torch.Tensor, roles_u: Roles) -> RegContext:
    return RegContext(x=u, g=g_u, diag=None, roles_image=roles_u, device=u.device, dtype_c=ctx.dtype_c,
                      dtype_r=ctx.dtype_r, axes_resolver=ctx.axes_resolver, arena=ctx.arena,
                      write_interior_slice=None, ws=ctx.ws, shard_index=ctx.shard_index, halo_map=ctx.halo_map)


def _axes_on_u(inner, ctx: RegContext, roles_u: Roles) -> Tuple[int, ...]:
    spec = getattr(getattr(inner, "params", None), "axes", "spatial")
    if ctx.axes_resolver is not None:
        try:
            return tuple(int(a) for a in ctx.axes_resolver(spec))
        except Exception:
            pass
    return roles_u.resolve_axes(spec)


@dataclass
class MappedRegularizer:
    """``inner`` evaluated on u = op(x); its gradient goes back through the op
    (into ctx.g for field operators, into parameter buffers for parameter ones)."""
    name: str
    inner: Any
    op: Any

    @property
    def params(self):
        return getattr(self.inner, "params", None)

    @params.setter
    def params(self, v):
        setattr(self.inner, "params", v)

    def halo(self, roles: Roles):
        out: Dict[int, int] = {}
        for h in (getattr(self.inner, "halo", lambda r: {})(roles) or {}, self.op.halo_extra(roles) or {}):
            for ax, k in h.items():
                out[ax] = max(out.get(ax, 0), int(k))
        return out

    @torch.no_grad()
    def energy_grad_fixed_axes(self, ctx: RegContext, axes: Tuple[int, ...]) -> torch.Tensor:
        interior = _whole(ctx.write_interior_slice, ctx.x.ndim)
        roles_u = self.op.roles_for_output(ctx.roles_image)
        u = self.op.forward_apply(ctx.x, ctx, interior).contiguous()
        g_u = torch.zeros_like(u, dtype=ctx.dtype_c)
        sub = _sub_ctx(ctx, u, g_u, roles_u)
        if hasattr(self.inner, "energy_grad_fixed_axes"):
            E = self.inner.energy_grad_fixed_axes(sub, axes)
        else:
            E = self.inner.energy_grad(sub)
        g_prev = self.op.adjoint_apply(g_u, ctx, interior)
        if g_prev is not None and ctx.g is not None:
            ctx.g.add_(g_prev)
        return E

    def energy_grad(self, ctx: RegContext) -> torch.Tensor:
        roles_u = self.op.roles_for_output(ctx.roles_image)
        return self.energy_grad_fixed_axes(ctx, _axes_on_u(self.inner, ctx, roles_u))


@dataclass
class Transformed:
    """Regulariser ``base`` behind an operator (unified op, or fwd/adj object),
    with the operator-aware diagonal of wrappers.py:43-110."""
    base: Any
    op: Any
    name: str
    params: Any = None
    _mr: MappedRegularizer = field(init=False)

    def __post_init__(self):
        op_u = self.op if (hasattr(self.op, "forward_apply") and hasattr(self.op, "adjoint_apply")) \
            else LinOpAdapter(self.op)
        self._mr = MappedRegularizer(name=self.name, inner=self.base, op=op_u)
        if self.params is None:
            self.params = getattr(self.base, "params", None)

    def halo(self, roles):
        try:
            return self._mr.halo(roles)
        except Exception:
            return {}

    def energy_grad(self, ctx: RegContext) -> torch.Tensor:
        return self._mr.energy_grad(ctx)

    def energy_grad_fixed_axes(self, ctx: RegContext, axes) -> torch.Tensor:
        return self._mr.energy_grad_fixed_axes(ctx, axes)

    @torch.no_grad()
    def add_diag(self, ctx: RegContext) -> None:
        """(A) the base's frame profile pushed through the op into ctx.diag; then
        (B) the base's scalar majorizer k on u pushed through the op (into ctx.diag
        for field operators, into the parameter diagonal for parameter ones); an
        identity op without majorizer falls back to base.add_diag."""
        try:
            op = self._mr.op
            interior = _whole(ctx.write_interior_slice, ctx.x.ndim)
            roles_u = op.roles_for_output(ctx.roles_image)
            u = op.forward_apply(ctx.x, ctx, interior)
            sub = _sub_ctx(ctx, u, torch.zeros_like(u, dtype=ctx.dtype_c), roles_u)
            if ctx.diag is not None:
                prof_fn = getattr(self.base, "majorizer_profile", None)
                prof = prof_fn(sub) if callable(prof_fn) else None
                if prof:
                    axis, v1d = prof[0]
                    pushed = op.diag_push_profile(axis, v1d, ctx, interior) \
                        if hasattr(op, "diag_push_profile") else None
                    if pushed is not None:
                        axis2, v2 = pushed
                        if int(axis2) != 0:
                            raise NotImplementedError("only frame-axis profiles are supported")
                        _add_profile(ctx.diag, v2)
                        return
            try:
                k = self.base.majorizer_diag(sub)
            except Exception:
                k = None
            if k is None:
                if isinstance(op, IdentityOp):
                    self.base.add_diag(ctx)
                return
            k_int = torch.ones_like(u.real, dtype=sub.dtype_r) * k.to(device=u.device, dtype=sub.dtype_r)
            pushed = op.diag_push(k_int, ctx, interior) if hasattr(op, "diag_push") else None
            if pushed is not None and ctx.diag is not None:
                ctx.diag.add_(pushed.to(ctx.diag.dtype))
        except Exception as e:   # the reference keeps the diagonal optional (warns and skips)
            warnings.warn(f"Failed to add diag for transformed regularizer {self.name}: {e}")

    def majorizer_diag(self, ctx):
        try:
            return self.base.majorizer_diag(ctx)
        except Exception:
            return None


def fused_tv(reg) -> Optional[TVND]:
    """The TVND the fused solver can evaluate in place of ``reg`` (a TVND, or a
    TVND behind an identity map, or behind a ScaleOp when the solver's workspace
    has no scale), else None."""
    if isinstance(reg, TVND):
        return reg
    mr = reg._mr if isinstance(reg, Transformed) else reg
    if isinstance(mr, MappedRegularizer) and isinstance(mr.inner, TVND):
        ops = mr.op.ops if isinstance(mr.op, ComposeOp) else [mr.op]
        if all(isinstance(o, (IdentityOp, ScaleOp)) for o in ops):
            return mr.inner
    return None
