"""TEST INFRASTRUCTURE (checker only, never on the product path): the Pipe-Menon
density compensation iteration w <- w / (G G^H w) restated on the CPU in FP64
with the oracle's own Kaiser-Bessel tables (oracle/kb.py), for the parity test
of mrirecon_b200.dcf.estimate_dcf.  G is the gridding interpolation without the
FFT; the reference has no estimator (it takes DCF as an input,
graspcg/nufft/backends/torchkb.py:185-199), so this restates the published
algorithm (Pipe and Menon, Magn. Reson. Med. 41:179, 1999)."""
import numpy as np
import torch

from .kb import KBNufft


def pipe_menon(traj: torch.Tensor, im_shape, iters: int = 20) -> torch.Tensor:
    """traj (B, nd, K) radians; returns (B, K) float64 weights."""
    if traj.ndim == 2:
        traj = traj.unsqueeze(0)
    S = tuple(int(s) for s in im_shape)
    k = KBNufft(torch.ones((1,) + S, dtype=torch.complex128), traj, None, norm="none")
    gtot = int(np.prod(k.G))
    out = []
    for b in range(k.B):
        idx, wt = k.idx[b], k.w[b].to(torch.float64)           # (K, W^nd)
        w = torch.ones(k.K, dtype=torch.float64)
        for _ in range(int(iters)):
            grid = torch.zeros(gtot, dtype=torch.float64)
            grid.index_add_(0, idx.reshape(-1), (wt * w[:, None]).reshape(-1))
            c = (grid[idx] * wt).sum(-1)
            w = w / c.clamp_min(1e-300)
        out.append(w)
    return torch.stack(out)
