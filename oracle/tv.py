"""Huber-TV energy/gradient restatement (CPU; TEST INFRASTRUCTURE ONLY).

Restates graspcg/regularization/tv_nd.py:54-88 (TVND.energy_grad_fixed_axes)
with the stencils of graspcg/ops/ndops.py:

* forward difference, last slice zero            ndops.py:28-42
* backward difference, first slice = p[0]        ndops.py:45-59
* iso energy  sqrt(sum_i |g_i|^2 + eps^2) - eps  ndops.py:66-81
* aniso energy sum_i (sqrt(|g_i|^2+eps^2) - eps) ndops.py:84-98
* flux g_i / max(sqrt(.), 1e-12)                 ndops.py:101-110, 121-135
* grad += -lambda * sum_i bwd_diff(p_i)          tv_nd.py:70-86
  (axis weights scale the forward differences only, as in tv_nd.py:59-70)
* energy E = lambda * sum(e)                     tv_nd.py:87

Works on the whole image tensor (one shard, so the temporal halo of
manager.py:268-301 is the identity).
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import torch


def fwd_diff(x: torch.Tensor, dim: int) -> torch.Tensor:
    out = torch.roll(x, shifts=-1, dims=dim) - x
    idx = [slice(None)] * out.ndim
    idx[dim] = -1
    out[tuple(idx)] = 0
    return out


def bwd_diff(y: torch.Tensor, dim: int) -> torch.Tensor:
    out = y - torch.roll(y, shifts=1, dims=dim)
    idx = [slice(None)] * out.ndim
    idx[dim] = 0
    out[tuple(idx)] = y[tuple(idx)]
    return out


def _abs2(g: torch.Tensor) -> torch.Tensor:
    return g.real * g.real + g.imag * g.imag if g.is_complex() else g * g


def tv_energy_grad(x: torch.Tensor, axes: Sequence[int], weight: float, eps: float = 1e-3,
                   isotropic: bool = True, axis_weights: Optional[Sequence[float]] = None
                   ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Return (E, grad) with E = lambda * sum e(x) and grad = -lambda * div p."""
    rdt = x.real.dtype
    if len(axes) == 0 or weight == 0.0:
        return torch.zeros((), dtype=rdt), torch.zeros_like(x)
    aw = list(axis_weights) if axis_weights is not None else [1.0] * len(axes)
    if len(aw) != len(axes):
        raise ValueError("axis_weights must match len(axes).")
    grads = [float(wi) * fwd_diff(x, ax) for wi, ax in zip(aw, axes)]
    eps_t = torch.tensor(eps, dtype=rdt)
    if isotropic:
        ss = sum(_abs2(g) for g in grads)
        den = torch.sqrt(ss + eps_t * eps_t)
        e = den - eps_t
        dcl = den.clamp_min(1e-12)
        flux = [g / dcl for g in grads]
    else:
        e = sum(torch.sqrt(_abs2(g) + eps_t * eps_t) - eps_t for g in grads)
        flux = [g / torch.sqrt(_abs2(g) + eps_t * eps_t).clamp_min(1e-12) for g in grads]
    div = sum(bwd_diff(p, ax) for p, ax in zip(flux, axes))
    return (e * weight).sum(), -weight * div


# --- diagonal preconditioner -------------------------------------------------
def tv_add_diag(D: torch.Tensor, x: torch.Tensor, axes: Sequence[int], weight: float, eps: float = 1e-3,
                axis_weights: Optional[Sequence[float]] = None, frame_profile: bool = True,
                frame_period: int = 0) -> None:
    """D += the term's diagonal at x, in place (FP64 when D is FP64).

    frame_profile and the term covers the frame axis 0: D += 2 lambda w_0^2 deg(f)
    with deg 1 at both ends of each series and 2 inside
    (TVND.majorizer_profile, graspcg/regularization/tv_nd.py:187-214, as
    RegManager.add_diag prefers it, manager.py:176-191).  Otherwise, per axis:
    s = lambda w_a^2 / sqrt(|fwd_diff(x)|^2 + eps^2), D += s on the first and
    last slice along the axis and 2 s inside (TVND.add_diag, tv_nd.py:113-164).
    frame_period > 0 splits the frames into independent series of that length.
    """
    if weight == 0.0 or len(axes) == 0:
        return
    aw = list(axis_weights) if axis_weights is not None else [1.0] * len(axes)
    F = int(x.shape[0])
    P = frame_period if frame_period > 0 else F
    if frame_profile and 0 in axes:
        w0 = float(aw[list(axes).index(0)])
        fl = torch.arange(F) % P
        deg = torch.where((fl > 0) & (fl < P - 1), 2.0, 1.0) if P > 2 else torch.ones(F)
        D += (2.0 * weight * w0 * w0 * deg.to(D.dtype)).view(-1, *([1] * (D.ndim - 1)))
        return
    xs = x.to(torch.complex128)
    for ax, wa in zip(axes, aw):
        if ax == 0 and P != F:
            parts = [fwd_diff(xs[i:i + P], 0) for i in range(0, F, P)]
            gi = torch.cat(parts, 0)
        else:
            gi = fwd_diff(xs, ax)
        s = weight * float(wa) ** 2 / torch.sqrt(_abs2(gi) + eps * eps)
        n = int(x.shape[ax]) if ax != 0 else P
        pos = torch.arange(int(x.shape[ax])) % n
        mult = torch.where((pos > 0) & (pos < n - 1), 2.0, 1.0).to(torch.float64) if n >= 3 else \
            torch.ones(int(x.shape[ax]), dtype=torch.float64)
        shape = [1] * x.ndim
        shape[ax] = -1
        D += (s * mult.view(shape)).to(D.dtype)


def sense_diag(maps: torch.Tensor, alpha: float, F: int, base: float = 0.0) -> torch.Tensor:
    """base + alpha sum_c |S_c|^2 per pixel, repeated over F frames, shape (F, 1, *S)
    (FP64): the data part of the Jacobi diagonal, alpha the A^H A gain of
    TorchKbNUFFTAdapter.diag_AHA_scalar (graspcg/nufft/backends/torchkb.py:341-364)."""
    m = maps.to(torch.complex128)
    sos = (m.real ** 2 + m.imag ** 2).sum(0)
    return (base + alpha * sos).unsqueeze(0).unsqueeze(0).expand(F, 1, *sos.shape).clone()
