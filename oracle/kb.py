"""Kaiser-Bessel gridding restatement (CPU; TEST INFRASTRUCTURE ONLY).

Follows the reference's pure-torch KB gridder for the arithmetic that fixes the
grid indices and weights, and the torchkb adapter for SENSE/DCF semantics:

* grid size            graspcg/nufft/backends/ptnufft.py:71-72   (ceil(osf*S))
* KB shape parameter   graspcg/nufft/backends/ptnufft.py:125     (Beatty 2005)
* KB weight formula    graspcg/nufft/backends/ptnufft.py:79-90   (clamped arg)
* float32 coordinates  graspcg/nufft/backends/ptnufft.py:151-153 (u = w/2pi+0.5;
                       gx = clamp(u*G, 0, G-1e-6), all float32)
* literal ptnufft
  index tables         graspcg/nufft/backends/ptnufft.py:155-171, 176-195
* SENSE / DCF / coil   graspcg/nufft/backends/torchkb.py:185-199, 202-323
  combine, B_eff       graspcg/nufft/backends/torchkb.py:151-183

Conventions that the reference gets wrong (ptnufft is not a working NUFFT: its
flat index is transposed, it measures distances to cell centres n+0.5, it has
no fftshift and its deapodisation is numerically broken) are restated in their
corrected form, which is what the CUDA path implements:

* integer-node distances d = gx - n, n = floor(gx) + o, o in [-W/2+1, W/2];
* row-major flat index (last image axis fastest);
* image pixel i sits at grid node i + G/2 - S//2 (centred coordinate i - S//2);
* ifftshift -> FFT -> fftshift, forward FFT unnormalised, adjoint = its exact
  adjoint (unnormalised inverse), optional ortho scale 1/sqrt(prod G);
* analytic KB deapodisation (closed-form Fourier transform of the truncated
  KB window, Jackson et al. 1991 / Beatty et al. 2005).
"""
from __future__ import annotations

import math
from typing import Optional, Sequence, Tuple

import numpy as np
import torch

TWO_PI_F32 = np.float32(2.0 * math.pi)


# ----------------------------------------------------------------------------
# scalar parameters
# ----------------------------------------------------------------------------

def grid_shape(spatial: Sequence[int], osf: float = 2.0) -> Tuple[int, ...]:
    """Oversampled grid per dim (ptnufft.py:71-72)."""
    return tuple(int(math.ceil(osf * s)) for s in spatial)


def kb_beta(W: int = 4, osf: float = 2.0) -> float:
    """KB shape parameter (ptnufft.py:125)."""
    return math.pi * math.sqrt(((W / float(osf)) * (float(osf) - 0.5)) ** 2 - 0.8)


def i0(x):
    """Modified Bessel I0 in float64 via torch.special.i0."""
    return torch.special.i0(torch.as_tensor(x, dtype=torch.float64))


def kb_weight(d: torch.Tensor, beta: float, W: int = 4) -> torch.Tensor:
    """phi(d) = I0(beta*sqrt(max(0, 1-(2|d|/W)^2))) / I0(beta)  (ptnufft.py:79-90), float64."""
    d = torch.as_tensor(d, dtype=torch.float64)
    arg = (1.0 - (2.0 * d.abs() / float(W)) ** 2).clamp_min(0.0)
    return torch.special.i0(beta * torch.sqrt(arg)) / i0(beta)


def deapod_1d(S: int, G: int, W: int, beta: float) -> torch.Tensor:
    """Closed-form FT of the truncated KB window at the image's centred coords.

    Phi(nu) = W/I0(beta) * sinh(sqrt(beta^2-(pi W nu)^2)) / sqrt(beta^2-(pi W nu)^2),
    nu = (i - S//2)/G.  Returns Phi (float64, shape (S,)); the operator divides
    the image by it.
    """
    r = torch.arange(S, dtype=torch.float64) - (S // 2)
    a = beta * beta - (math.pi * W * r / G) ** 2
    out = torch.empty_like(a)
    pos = a > 0
    sa = torch.sqrt(a[pos])
    out[pos] = torch.sinh(sa) / sa
    neg = a < 0
    sn = torch.sqrt(-a[neg])
    out[neg] = torch.sin(sn) / sn
    out[a == 0] = 1.0
    return out * (W / float(i0(beta)))


# ----------------------------------------------------------------------------
# binning (float32 arithmetic identical to the reference)
# ----------------------------------------------------------------------------

def grid_coords_f32(traj_nd_k, G: Sequence[int]) -> np.ndarray:
    """Float32 grid coordinates gx_d for one frame, (nd, K).

    Same operation sequence as ptnufft.py:151-153 on CPU torch:
    u = w / float32(2pi) + 0.5 ; gx = u * G ; clamp(gx, 0, float32(G - 1e-6)).
    """
    c = np.asarray(traj_nd_k, dtype=np.float32)
    out = np.empty_like(c)
    for d in range(c.shape[0]):
        u = c[d] / TWO_PI_F32 + np.float32(0.5)
        gx = u * np.float32(G[d])
        out[d] = np.minimum(np.maximum(gx, np.float32(0.0)), np.float32(G[d] - 1e-6))
    return out


def ptnufft_indices(traj_nd_k, G: Sequence[int], W: int = 4) -> np.ndarray:
    """The reference's literal (K, W^nd) int64 index table (ptnufft.py:155-171/176-195).

    Offsets -W//2 .. -W//2+W-1 added in float32 before floor, remainder G,
    flat index nx + G0*ny (+ G0*G1*nz).
    """
    gx = grid_coords_f32(traj_nd_k, G)
    nd = gx.shape[0]
    r = W // 2
    offs = np.arange(-r, -r + W).astype(np.float32)
    n = [np.mod(np.floor(gx[d][:, None] + offs[None, :]).astype(np.int64), G[d]) for d in range(nd)]
    K = gx.shape[1]
    if nd == 2:
        idx = n[0][:, :, None] + G[0] * n[1][:, None, :]
    else:
        idx = (n[0][:, :, None, None] + G[0] * n[1][:, None, :, None]
               + (G[0] * G[1]) * n[2][:, None, None, :])
    return idx.reshape(K, W ** nd)


def node_offsets(W: int) -> np.ndarray:
    if W % 2:
        raise ValueError("kernel width must be even")
    return np.arange(-W // 2 + 1, W // 2 + 1, dtype=np.int64)


def cell_base(traj_nd_k, G: Sequence[int]) -> np.ndarray:
    """floor(gx) per dim (int64, (nd, K)): the production binning key."""
    return np.floor(grid_coords_f32(traj_nd_k, G)).astype(np.int64)


def cell_indices(traj_nd_k, G: Sequence[int], W: int = 4):
    """Corrected-convention table: flat row-major node index and float64 weights.

    Returns (idx (K, W^nd) int64, w (K, W^nd) float64, sign (K, W^nd) int8)
    where sign = (-1)^(sum of node coordinates) is what the CUDA path folds in
    for the fftshift; the oracle itself does not use it.
    """
    gx = grid_coords_f32(traj_nd_k, G)
    nd, K = gx.shape
    base = np.floor(gx).astype(np.int64)
    o = node_offsets(W)
    beta = kb_beta(W, 2.0)
    ns, ws = [], []
    for d in range(nd):
        n = base[d][:, None] + o[None, :]                   # (K, W) unwrapped
        dist = gx[d].astype(np.float64)[:, None] - n.astype(np.float64)
        ws.append(dist)
        ns.append(np.mod(n, G[d]))
    return gx, ns, ws


class KBNufft:
    """Corrected KB NUFFT with SENSE, DCF and B_eff semantics of the torchkb adapter.

    maps (C, *S) complex; traj (B, nd, K) radians (float32 arithmetic for the
    grid coordinates); dcf (B, K) / (K,) / None.
    A : x (B_eff, 1, *S) -> y (B_eff, C, K)
    AH: y (B_eff, C, K)   -> x (B_eff, 1, *S)
    """

    def __init__(self, maps: torch.Tensor, traj: torch.Tensor, dcf: Optional[torch.Tensor] = None, *,
                 W: int = 4, osf: float = 2.0, dtype: torch.dtype = torch.complex128,
                 dcf_mode: str = "balanced", apply_dcf_in_fwd: bool = False,
                 apply_dcf_in_adj: bool = True, norm: str = "ortho"):
        self.dtype = dtype
        self.rdt = torch.float64 if dtype == torch.complex128 else torch.float32
        self.maps = maps.detach().to("cpu", dtype)
        self.C = int(maps.shape[0])
        self.S = tuple(int(s) for s in maps.shape[1:])
        self.nd = len(self.S)
        self.G = grid_shape(self.S, osf)
        if any(g % 2 for g in self.G):
            raise ValueError("oversampled grid must be even in every dim")
        self.W = int(W)
        self.beta = kb_beta(W, osf)
        traj = torch.as_tensor(traj).detach().to("cpu", torch.float32)
        if traj.ndim == 2:
            traj = traj.unsqueeze(0)
        self.B, _, self.K = (int(s) for s in traj.shape)
        self.traj = traj
        self.dcf_mode = dcf_mode
        self.apply_dcf_in_fwd = apply_dcf_in_fwd
        self.apply_dcf_in_adj = apply_dcf_in_adj
        if dcf is not None:
            d = torch.as_tensor(dcf).detach().to("cpu", torch.float64)
            if d.ndim == 1:
                d = d.view(1, -1)
            if int(d.shape[0]) == 1:
                d = d.expand(self.B, -1)
            self.dcf = d.contiguous()
        else:
            self.dcf = None
        self.scale = 1.0 / math.sqrt(float(np.prod(self.G))) if norm == "ortho" else 1.0
        # per-frame tables
        self.idx, self.w = [], []
        W_ = self.W
        for b in range(self.B):
            gx, ns, dists = cell_indices(traj[b].numpy(), self.G, W_)
            wd = [kb_weight(torch.from_numpy(dd), self.beta, W_) for dd in dists]   # (K, W) float64
            nt = [torch.from_numpy(n) for n in ns]
            if self.nd == 2:
                idx = nt[0][:, :, None] * self.G[1] + nt[1][:, None, :]
                w = wd[0][:, :, None] * wd[1][:, None, :]
            else:
                idx = ((nt[0][:, :, None, None] * self.G[1] + nt[1][:, None, :, None]) * self.G[2]
                       + nt[2][:, None, None, :])
                w = wd[0][:, :, None, None] * wd[1][:, None, :, None] * wd[2][:, None, None, :]
            self.idx.append(idx.reshape(self.K, -1))
            self.w.append(w.reshape(self.K, -1).to(self.rdt))
        dap = [deapod_1d(S, G, W_, self.beta) for S, G in zip(self.S, self.G)]
        inv = 1.0 / dap[0]
        for d in range(1, self.nd):
            inv = inv.unsqueeze(-1) * (1.0 / dap[d]).view(*([1] * d), -1)
        self.invdeap = inv.to(self.rdt)
        self.place = tuple(slice(G // 2 - S // 2, G // 2 - S // 2 + S) for S, G in zip(self.S, self.G))
        self.sdims = tuple(range(1, 1 + self.nd))

    # --- helpers -------------------------------------------------------------
    def frame_of(self, Bx: int):
        if Bx == self.B:
            return lambda be: be
        if self.B == 1:
            return lambda be: 0
        if Bx % self.B == 0:
            r = Bx // self.B
            return lambda be: be // r
        raise ValueError(f"omega batch {self.B} incompatible with requested {Bx}")

    def dcf_weight(self, b: int, direction: str) -> Optional[torch.Tensor]:
        if self.dcf is None:
            return None
        d = self.dcf[b]
        if self.dcf_mode == "balanced":
            return torch.sqrt(d.clamp_min(0))
        if self.dcf_mode == "standard":
            if (direction == "A" and self.apply_dcf_in_fwd) or (direction == "AH" and self.apply_dcf_in_adj):
                return d
        return None

    # --- operators -----------------------------------------------------------
    def A(self, x: torch.Tensor) -> torch.Tensor:
        x = x.to("cpu", self.dtype)
        Bx = int(x.shape[0])
        fr = self.frame_of(Bx)
        y = torch.empty((Bx, self.C, self.K), dtype=self.dtype)
        for be in range(Bx):
            b = fr(be)
            img = x[be, 0] * self.invdeap * self.maps                  # (C, *S)
            g = torch.zeros((self.C,) + self.G, dtype=self.dtype)
            g[(slice(None),) + self.place] = img
            g = torch.fft.fftshift(torch.fft.fftn(torch.fft.ifftshift(g, dim=self.sdims), dim=self.sdims),
                                   dim=self.sdims).reshape(self.C, -1)
            yb = (g[:, self.idx[b]] * self.w[b].to(self.dtype)).sum(-1) * self.scale
            dw = self.dcf_weight(b, "A")
            if dw is not None:
                yb = yb * dw.to(self.dtype)
            y[be] = yb
        return y

    def AH(self, y: torch.Tensor) -> torch.Tensor:
        y = y.to("cpu", self.dtype)
        Bx = int(y.shape[0])
        fr = self.frame_of(Bx)
        x = torch.empty((Bx, 1) + self.S, dtype=self.dtype)
        n_cells = int(np.prod(self.G))
        for be in range(Bx):
            b = fr(be)
            yb = y[be]
            dw = self.dcf_weight(b, "AH")
            if dw is not None:
                yb = yb * dw.to(self.dtype)
            g = torch.zeros((self.C, n_cells), dtype=self.dtype)
            idx, w = self.idx[b], self.w[b].to(self.dtype)
            for m in range(idx.shape[1]):
                g.index_add_(1, idx[:, m], yb * w[:, m])
            g = g.view((self.C,) + self.G)
            g = torch.fft.fftshift(torch.fft.ifftn(torch.fft.ifftshift(g, dim=self.sdims), dim=self.sdims,
                                                   norm="forward"), dim=self.sdims)
            img = g[(slice(None),) + self.place] * self.invdeap * self.maps.conj()
            x[be, 0] = img.sum(0) * self.scale
        return x
