"""Sampling density compensation estimated on the GPU.

The fixed-point iteration of Pipe and Menon (Magn. Reson. Med. 41:179, 1999),

    w  <-  w / (G G^H w),

with G the plan's own Kaiser-Bessel interpolation (grid -> samples) and G^H its
spread (samples -> grid), both run by this package's gridding kernels on the
oversampled grid without the FFT.  At the fixed point G G^H w = 1: the spread
of the weighted samples is flat wherever the trajectory reaches.  The reference
takes density compensation as an input (graspcg/nufft/backends/torchkb.py:
185-199); this estimator has no counterpart there.  The weights are in the
units of the unnormalised kernel (peak 1); pass them as ``dcf`` to the adapter
or the front-end (``dcf_mode`` "balanced" or "standard").
"""
from __future__ import annotations

from typing import Sequence

import torch


def estimate_dcf(traj: torch.Tensor, im_shape: Sequence[int], iters: int = 20, kwidth: int = 4,
                 osf: float = 2.0) -> torch.Tensor:
    """traj (B, nd, K) or (nd, K) float32 radians in [-pi, pi) on a CUDA device,
    im_shape the image size (nd ints).  Returns (B, K) float32 weights."""
    from .nufft import KBPlan, OPT_FFT_MODE
    if traj.ndim == 2:
        traj = traj.unsqueeze(0)
    if traj.ndim != 3 or int(traj.shape[1]) != len(im_shape):
        raise ValueError("traj must be (B, nd, K) with nd = len(im_shape)")
    if not traj.is_cuda:
        raise ValueError("traj must be on a CUDA device")
    dev = traj.device
    B, _, K = (int(s) for s in traj.shape)
    S = tuple(int(s) for s in im_shape)
    plan = KBPlan(S, 1, B, K, W=kwidth, osf=osf, ortho=False, device=dev)
    plan.set_option(OPT_FFT_MODE, 0)     # the spread and the interp share one plain grid
    plan.set_points(traj.to(torch.float32).contiguous())
    plan.set_maps(torch.ones((1,) + S, dtype=torch.complex64, device=dev))
    w = torch.ones((B, 1, K), dtype=torch.complex64, device=dev)
    c = torch.empty_like(w)
    tiny = torch.finfo(torch.float32).tiny
    for _ in range(int(iters)):
        plan.stage("spread", None, w, B)      # grid = G^H w
        plan.stage("interp", None, c, B)      # c = G grid
        w = (w.real / c.real.clamp_min(tiny)).to(torch.complex64)
    return w.real.reshape(B, K).contiguous()
