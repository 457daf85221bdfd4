"""FP32 CPU restatement of the warm-start network (TEST INFRASTRUCTURE ONLY).

Same architecture, weight layout and loss as ``mrirecon_b200.warmstart``, built
from torch.nn.functional so that torch.autograd gives the reference gradients
the GPU kernels are checked against.  Activations are (Nb, C, D, H, W) here;
weights are stored as in the kernels, [27][cin][cout] with tap = kd*9 + kh*3 + kw.

Architecture (3 levels, 32 base channels, 3x3x3 convolutions over (t, y, x)):
  c1 2->32, c2 32->32 (B1); pool; c3 32->64, c4 64->64 (B2); pool; c5 64->128;
  up; c6 [up(c5), B2] 192->64; up; c7 [up(c6), B1] 96->32; c8 32->2 (linear);
  output = input + c8.  ReLU after c1..c7, pooling = 2x2 mean over (y, x),
  up = nearest 2x over (y, x).
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import torch
import torch.nn.functional as Fn

# name, cin (real), cout (real)
LAYERS: List[Tuple[str, int, int]] = [("c1", 2, 32), ("c2", 32, 32), ("c3", 32, 64), ("c4", 64, 64),
                                      ("c5", 64, 128), ("c6", 192, 64), ("c7", 96, 32), ("c8", 32, 2)]


def conv(x: torch.Tensor, w27: torch.Tensor, b: torch.Tensor, relu: bool) -> torch.Tensor:
    """x (Nb, cin, D, H, W); w27 [27][cin][cout] -> torch weight (cout, cin, 3, 3, 3)."""
    cin, cout = w27.shape[1], w27.shape[2]
    w = w27.permute(2, 1, 0).reshape(cout, cin, 3, 3, 3)
    y = Fn.conv3d(x, w, b, padding=1)
    return Fn.relu(y) if relu else y


def pool(x):
    return Fn.avg_pool3d(x, kernel_size=(1, 2, 2))


def up(x):
    return x.repeat_interleave(2, dim=3).repeat_interleave(2, dim=4)


def forward(x2: torch.Tensor, P: Dict[str, Tuple[torch.Tensor, torch.Tensor]], x_res=None) -> torch.Tensor:
    """x2 (Nb, 2, D, H, W) -> network output (Nb, 2, D, H, W); the residual adds
    x_res (default x2)."""
    a1 = conv(x2, *P["c1"], True)
    b1 = conv(a1, *P["c2"], True)
    a2 = conv(pool(b1), *P["c3"], True)
    b2 = conv(a2, *P["c4"], True)
    a3 = conv(pool(b2), *P["c5"], True)
    c2 = conv(torch.cat([up(a3), b2], 1), *P["c6"], True)
    c1 = conv(torch.cat([up(c2), b1], 1), *P["c7"], True)
    return (x2 if x_res is None else x_res) + conv(c1, *P["c8"], False)


def loss(x2: torch.Tensor, t2: torch.Tensor, P, x_res=None) -> torch.Tensor:
    """Mean squared error over all real values."""
    return ((forward(x2, P, x_res) - t2) ** 2).mean()
