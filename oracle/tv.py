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
