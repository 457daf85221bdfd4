"""Graph-Laplacian regulariser restatement (CPU, FP64; TEST INFRASTRUCTURE ONLY).

Restates graspcg/regularization/graph_laplacian.py:

* W symmetrised (W + W^T)/2, diagonal zeroed       :45-67 (dense and sparse)
* degree deg_t = sum_s W_ts, clamped at 0           :69-80
* L = D - W ("none"), I - D^-1 W ("rw"),
  I - D^-1/2 W D^-1/2 ("sym"), deg clamped at 1e-20  :103-168
* E = lambda/2 sum_p Re<x[:, p], L x[:, p]>, grad = lambda L x   :171-234
* diagonal: lambda deg ("none") or lambda 1{deg > 0}            :236-321
"""
from __future__ import annotations

from dataclasses import dataclass

import torch


def laplacian(W: torch.Tensor, normalize: str = "none") -> torch.Tensor:
    Wd = W.to_dense() if W.is_sparse else W
    Wd = (0.5 * (Wd + Wd.transpose(0, 1))).to(torch.float64).clone()
    Wd.fill_diagonal_(0.0)
    deg = Wd.sum(dim=1).clamp_min(0.0)
    eye = torch.eye(Wd.shape[0], dtype=torch.float64)
    if normalize == "none":
        return torch.diag(deg) - Wd
    if normalize == "rw":
        return eye - Wd / deg.clamp_min(1e-20).view(-1, 1)
    if normalize == "sym":
        dmh = 1.0 / torch.sqrt(deg.clamp_min(1e-20))
        return eye - dmh.view(-1, 1) * Wd * dmh.view(1, -1)
    raise ValueError(normalize)


def degree_profile(W: torch.Tensor, normalize: str, weight: float) -> torch.Tensor:
    Wd = W.to_dense() if W.is_sparse else W
    Wd = (0.5 * (Wd + Wd.transpose(0, 1))).to(torch.float64).clone()
    Wd.fill_diagonal_(0.0)
    deg = Wd.sum(dim=1).clamp_min(0.0)
    v = deg if normalize == "none" else (deg > 0).to(torch.float64)
    return weight * v


def graph_energy_grad(x: torch.Tensor, L: torch.Tensor, weight: float = 1.0):
    """(E, grad) for an image (B, ...) with the frame axis first."""
    B = x.shape[0]
    X = x.reshape(B, -1).to(torch.complex128)
    Y = L.to(torch.complex128) @ X
    E = 0.5 * weight * (X.conj() * Y).real.sum()
    return E, (weight * Y).reshape(x.shape).to(x.dtype)


@dataclass
class GraphSpec:
    """A graph term for the NCG oracle: E = weight/2 <x, L x> over frames."""
    L: torch.Tensor
    weight: float = 1.0
