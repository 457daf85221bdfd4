"""Seeded synthetic workloads (the reference ships no data generators).

* ``ellipse_phantom``   random ellipses: centres U[-0.6,0.6], semi-axes
  U[0.1,0.4], angle U[0,pi), intensity U[0.1,1], phase U[0,2pi)
* ``dynamic_phantom``   the same ellipses, each scaled over frames by a
  gamma-variate enhancement curve (GRASP-style DCE series)
* ``ellipsoid_phantom`` 3D analogue
* ``coil_maps``         Gaussian sensitivities centred on a circle (2D) or a
  sphere-ish ring (3D) of radius 0.7
* ``golden_angle_radial`` 2D radial spokes at 111.246 deg increments,
  continuous across frames, readout k in [-pi, pi) step 2pi/n_read
* ``golden_means_koosh`` 3D radial spokes from the 2D golden means
  (phi1, phi2 = 0.4656, 0.6823)
* ``add_noise``          complex Gaussian noise of std sigma per component

All run on the CPU with a torch.Generator (input generation, not the hot path)
and return CPU tensors; callers move them to the device.
"""
from __future__ import annotations

import math
from typing import Optional, Tuple

import torch

GOLDEN_ANGLE_DEG = 111.246117975
GOLDEN_MEANS_3D = (0.4656, 0.6823)


def _grid2(N: int):
    yy, xx = torch.meshgrid(torch.linspace(-1, 1, N, dtype=torch.float64),
                            torch.linspace(-1, 1, N, dtype=torch.float64), indexing="ij")
    return xx, yy


def ellipse_params(n: int, seed: int):
    g = torch.Generator().manual_seed(seed)
    out = []
    for _ in range(n):
        cx, cy, a, b, th, v, ph = (float(t) for t in torch.rand(7, generator=g, dtype=torch.float64))
        out.append(dict(cx=0.6 * (2 * cx - 1), cy=0.6 * (2 * cy - 1), a=0.1 + 0.3 * a, b=0.1 + 0.3 * b,
                        th=th * math.pi, v=0.1 + 0.9 * v, ph=2 * math.pi * ph))
    return out


def ellipse_masks(N: int, params):
    xx, yy = _grid2(N)
    masks = []
    for p in params:
        c, s = math.cos(p["th"]), math.sin(p["th"])
        xr = (xx - p["cx"]) * c + (yy - p["cy"]) * s
        yr = -(xx - p["cx"]) * s + (yy - p["cy"]) * c
        masks.append(((xr / p["a"]) ** 2 + (yr / p["b"]) ** 2 <= 1.0))
    return masks


def ellipse_phantom(N: int, n_ellipses: int = 10, seed: int = 0) -> torch.Tensor:
    """(N, N) complex64."""
    params = ellipse_params(n_ellipses, seed)
    img = torch.zeros((N, N), dtype=torch.complex128)
    for p, m in zip(params, ellipse_masks(N, params)):
        img[m] += p["v"] * complex(math.cos(p["ph"]), math.sin(p["ph"]))
    return img.to(torch.complex64)


def gamma_variate(n_frames: int, t0: float, tmax: float, alpha: float = 3.0) -> torch.Tensor:
    """Normalised gamma-variate curve (peak 1 at tmax) sampled on frames 0..n-1, zero before t0."""
    t = torch.arange(n_frames, dtype=torch.float64)
    tt = ((t - t0) / max(tmax - t0, 1e-6)).clamp_min(0.0)
    c = tt ** alpha * torch.exp(alpha * (1.0 - tt))
    return c


def dynamic_phantom(N: int, n_frames: int, n_ellipses: int = 10, seed: int = 0,
                    enhancement: float = 1.0) -> torch.Tensor:
    """(F, N, N) complex64: baseline ellipses, each with its own gamma-variate enhancement."""
    params = ellipse_params(n_ellipses, seed)
    g = torch.Generator().manual_seed(seed + 1000)
    imgs = torch.zeros((n_frames, N, N), dtype=torch.complex128)
    for p, m in zip(params, ellipse_masks(N, params)):
        t0 = float(torch.rand(1, generator=g)) * 0.3 * n_frames
        tm = t0 + 2.0 + float(torch.rand(1, generator=g)) * 0.4 * n_frames
        amp = enhancement * float(torch.rand(1, generator=g))
        curve = 1.0 + amp * gamma_variate(n_frames, t0, tm)
        val = p["v"] * complex(math.cos(p["ph"]), math.sin(p["ph"]))
        imgs[:, m] += (curve * val).view(-1, 1).to(torch.complex128)
    return imgs.to(torch.complex64)


def ellipsoid_phantom(N: int, n_ellipsoids: int = 10, seed: int = 0) -> torch.Tensor:
    """(N, N, N) complex64 random axis-aligned-then-rotated-in-plane ellipsoids."""
    g = torch.Generator().manual_seed(seed)
    ax = torch.linspace(-1, 1, N, dtype=torch.float64)
    zz, yy, xx = torch.meshgrid(ax, ax, ax, indexing="ij")
    img = torch.zeros((N, N, N), dtype=torch.complex128)
    for _ in range(n_ellipsoids):
        r = torch.rand(9, generator=g, dtype=torch.float64)
        c = 0.5 * (2 * r[:3] - 1)
        s = 0.1 + 0.3 * r[3:6]
        th = float(r[6]) * math.pi
        v = 0.1 + 0.9 * float(r[7])
        ph = 2 * math.pi * float(r[8])
        xr = (xx - c[0]) * math.cos(th) + (yy - c[1]) * math.sin(th)
        yr = -(xx - c[0]) * math.sin(th) + (yy - c[1]) * math.cos(th)
        m = (xr / s[0]) ** 2 + (yr / s[1]) ** 2 + ((zz - c[2]) / s[2]) ** 2 <= 1.0
        img[m] += v * complex(math.cos(ph), math.sin(ph))
    return img.to(torch.complex64)


def coil_maps(N: int, n_coils: int, ndim: int = 2, radius: float = 0.7, width: float = 0.5) -> torch.Tensor:
    """(C, *[N]*ndim) complex64 Gaussian maps centred on a circle (a ring at z=0 and +-0.5 in 3D),
    with a small linear phase per coil so that maps are genuinely complex."""
    maps = []
    if ndim == 2:
        xx, yy = _grid2(N)
        for c in range(n_coils):
            t = 2 * math.pi * c / n_coils
            mag = torch.exp(-((xx - radius * math.cos(t)) ** 2 + (yy - radius * math.sin(t)) ** 2) / width)
            phase = 0.5 * (xx * math.cos(t) + yy * math.sin(t))
            maps.append(mag * torch.exp(1j * phase))
    else:
        ax = torch.linspace(-1, 1, N, dtype=torch.float64)
        zz, yy, xx = torch.meshgrid(ax, ax, ax, indexing="ij")
        for c in range(n_coils):
            t = 2 * math.pi * c / n_coils
            z0 = (-0.5, 0.0, 0.5)[c % 3] if n_coils > 4 else 0.0
            mag = torch.exp(-((xx - radius * math.cos(t)) ** 2 + (yy - radius * math.sin(t)) ** 2
                              + (zz - z0) ** 2) / width)
            phase = 0.5 * (xx * math.cos(t) + yy * math.sin(t))
            maps.append(mag * torch.exp(1j * phase))
    return torch.stack(maps).to(torch.complex64)


def golden_angle_radial(n_spokes: int, n_read: int, first_spoke: int = 0) -> torch.Tensor:
    """(2, n_spokes*n_read) float32 radians; spoke s has angle (first_spoke+s)*111.246 deg."""
    ang = (torch.arange(n_spokes, dtype=torch.float64) + first_spoke) * math.radians(GOLDEN_ANGLE_DEG)
    kr = (torch.arange(n_read, dtype=torch.float64) - n_read // 2) * (2 * math.pi / n_read)
    kx = kr.view(1, -1) * torch.cos(ang).view(-1, 1)
    ky = kr.view(1, -1) * torch.sin(ang).view(-1, 1)
    return torch.stack([kx.reshape(-1), ky.reshape(-1)]).to(torch.float32)


def grasp_trajectory(n_frames: int, spokes_per_frame: int, n_read: int) -> torch.Tensor:
    """(F, 2, spokes*n_read): frame f uses the continuous golden-angle spokes f*spf ... f*spf+spf-1."""
    return torch.stack([golden_angle_radial(spokes_per_frame, n_read, f * spokes_per_frame)
                        for f in range(n_frames)])


def golden_means_koosh(n_spokes: int, n_read: int) -> torch.Tensor:
    """(3, n_spokes*n_read) float32 radians, 3D radial (koosh-ball) spokes."""
    p1, p2 = GOLDEN_MEANS_3D
    i = torch.arange(n_spokes, dtype=torch.float64)
    kz = (i * p1) % 1.0 * 2 - 1
    az = 2 * math.pi * ((i * p2) % 1.0)
    st = torch.sqrt((1 - kz ** 2).clamp_min(0))
    dirs = torch.stack([st * torch.cos(az), st * torch.sin(az), kz], 1)          # (S, 3)
    kr = (torch.arange(n_read, dtype=torch.float64) - n_read // 2) * (2 * math.pi / n_read)
    pts = dirs.unsqueeze(1) * kr.view(1, -1, 1)                                      # (S, R, 3)
    return pts.reshape(-1, 3).T.contiguous().to(torch.float32)


def add_noise(y: torch.Tensor, sigma: float, seed: int = 0) -> torch.Tensor:
    g = torch.Generator().manual_seed(seed)
    n = torch.randn(y.shape, generator=g, dtype=torch.float32) + 1j * torch.randn(y.shape, generator=g,
                                                                                   dtype=torch.float32)
    return y + (sigma * n).to(y.device, y.dtype)


def random_traj(B: int, nd: int, K: int, seed: int = 0) -> torch.Tensor:
    g = torch.Generator().manual_seed(seed)
    return (torch.rand((B, nd, K), generator=g) * 2 * math.pi - math.pi).to(torch.float32)
