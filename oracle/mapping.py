"""Temporal-basis mapping restatement (CPU, FP64; TEST INFRASTRUCTURE ONLY).

Restates graspcg/regularization/mapping.py:112-236 (TemporalBasisOp) for one
shard: u = U V over the frame axis (:133-152), g_V += U^H g_u (:154-172),
diag_V[k, p] += sum_t |U_tk|^2 k_u[t, p] (:178-206) and the frame-profile push
DV_k = sum_t |U_tk|^2 v_t broadcast over the parameter columns (:207-236).
"""
from __future__ import annotations

import torch


def basis_forward(U: torch.Tensor, V: torch.Tensor) -> torch.Tensor:
    K = V.shape[0]
    u = U.to(torch.complex128) @ V.reshape(K, -1).to(torch.complex128)
    return u.reshape((U.shape[0],) + tuple(V.shape[1:]))


def basis_adjoint(U: torch.Tensor, g_u: torch.Tensor) -> torch.Tensor:
    B = g_u.shape[0]
    gV = U.to(torch.complex128).conj().transpose(0, 1) @ g_u.reshape(B, -1).to(torch.complex128)
    return gV.reshape((U.shape[1],) + tuple(g_u.shape[1:]))


def basis_diag_push(U: torch.Tensor, k_u: torch.Tensor) -> torch.Tensor:
    B = k_u.shape[0]
    U2 = U.to(torch.complex128).abs() ** 2
    DV = U2.transpose(0, 1) @ k_u.reshape(B, -1).to(torch.float64)
    return DV.reshape((U.shape[1],) + tuple(k_u.shape[1:]))


def basis_profile_push(U: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    U2 = U.to(torch.complex128).abs() ** 2
    return U2.transpose(0, 1) @ v.to(torch.float64)
