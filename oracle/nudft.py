"""FP64 direct NUDFT and its true adjoint (TEST INFRASTRUCTURE ONLY).

``nudft_forward`` restates the reference's ground truth ``_nudft_A``
(graspcg/tests/test_nufft_precision_gt.py:48-89): centred coordinates
r in [-S/2, S/2) (``_coords_centered`` :48-53), E = exp(-i w.r), SENSE maps
per coil, optional sqrt(dcf) after.

``nudft_adjoint`` is the exact adjoint conj(E)^T of that forward.  The
reference's ``_nudft_AH`` (:91-121) computes ``Y_LK @ E_conj`` with E_conj of
shape (R, K) used as if it were (K, R); it only runs when K == R and then is
not the adjoint, so it is not restated.
"""
from __future__ import annotations

import torch


def coords_centered(spatial):
    axes = [torch.arange(S, dtype=torch.float64) - (S // 2) for S in spatial]
    mesh = torch.meshgrid(*axes, indexing="ij")
    return torch.stack([m.reshape(-1) for m in mesh], dim=1)          # (R, nd)


def nudft_matrix(spatial, traj_b):
    omega = torch.as_tensor(traj_b).to(torch.float64).transpose(0, 1)  # (K, nd)
    return torch.exp(-1j * (omega @ coords_centered(spatial).T))        # (K, R)


def nudft_forward(maps, x, traj_b, dcf_b=None):
    """x (L,1,*S), maps (C,*S), traj_b (nd,K) radians -> (L,C,K) complex128."""
    maps = maps.to(torch.complex128)
    x = x.to(torch.complex128)
    L, C = x.shape[0], maps.shape[0]
    spatial = tuple(maps.shape[1:])
    E = nudft_matrix(spatial, traj_b)
    X = x.reshape(L, -1)
    M = maps.reshape(C, -1)
    y = torch.stack([(X * M[c].unsqueeze(0)) @ E.T for c in range(C)], dim=1)
    if dcf_b is not None:
        # sqrt taken in the dcf's own dtype, as the reference does (:87-88)
        y = y * torch.sqrt(torch.as_tensor(dcf_b).clamp_min(0)).to(y.dtype)
    return y


def nudft_adjoint(maps, y, traj_b, dcf_b=None):
    """True adjoint of nudft_forward: y (L,C,K) -> (L,1,*S) complex128."""
    maps = maps.to(torch.complex128)
    y = y.to(torch.complex128)
    L, C, K = y.shape
    spatial = tuple(maps.shape[1:])
    E = nudft_matrix(spatial, traj_b)                                     # (K, R)
    if dcf_b is not None:
        y = y * torch.sqrt(torch.as_tensor(dcf_b).clamp_min(0)).to(y.dtype)
    M = maps.reshape(C, -1)
    x = torch.zeros((L, M.shape[1]), dtype=torch.complex128)
    for c in range(C):
        x += (y[:, c, :] @ E.conj()) * M[c].conj().unsqueeze(0)
    return x.reshape((L, 1) + spatial)
