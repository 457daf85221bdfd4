"""Seeded synthetic reconstruction problems shared by the bench and the warm-start tools.

``grasp``      256x256 complex64, 12 coils, 34 frames x 21 golden-angle spokes x
               512 samples, gamma-variate dynamic ellipse phantom, complex
               Gaussian k-space noise sigma 1e-3, spatial TV 1e-3 + temporal TV
               5e-3 (eps 1e-3).
``radial128``  128x128, 8 coils, one frame of 64 spokes x 256 samples, spatial TV 1e-3.
"""
from __future__ import annotations

import torch

WORKLOADS = {
    "grasp": dict(name="grasp_256x256_34fr_12coil_21spk_512ro", N=256, C=12, F=34, spf=21, nread=512,
                  lam_s=1e-3, lam_t=5e-3, eps=1e-3, sigma=1e-3),
    "radial128": dict(name="radial_128x128_1fr_8coil_64spk_256ro", N=128, C=8, F=1, spf=64, nread=256,
                      lam_s=1e-3, lam_t=0.0, eps=1e-3, sigma=0.0),
}
STOP_WINDOW, STOP_TOL = 10, 1e-4


def make_inputs(w):
    """(x_true (F,1,N,N), maps (C,N,N), traj (F,2,K)) on the CPU."""
    from . import phantoms
    N, C, F = w["N"], w["C"], w["F"]
    x_true = phantoms.dynamic_phantom(N, F, seed=0).unsqueeze(1)
    maps = phantoms.coil_maps(N, C)
    traj = phantoms.grasp_trajectory(F, w["spf"], w["nread"])
    return x_true, maps, traj


def axis_spec():
    from .layout import AxisSpec
    return AxisSpec(image_labels=("B", "coil", "X", "Y"), kspace_labels=("B", "coil", "K"),
                    image_fft_labels=("X", "Y"), coil_label="coil")


def regs(w):
    from .regularization import RegManager, TVND, TVParams
    r = [TVND("tv_spatial", TVParams(weight=w["lam_s"], eps=w["eps"], axes="spatial"))]
    if w["lam_t"] > 0:
        r.append(TVND("tv_temporal", TVParams(weight=w["lam_t"], eps=w["eps"], axes="temporal")))
    return RegManager(r)


def solver_cfg(max_iter=3000):
    from .solver import CGConfig
    return CGConfig(direction="fr", ls_name="armijo", max_iter=max_iter, stop_window=STOP_WINDOW,
                    stop_tol=STOP_TOL, schedule="fast", cuda_graph=True, iters_per_graph=8)


def build(w, device, autotune: bool = False):
    """Operator, noisy data and ground truth of workload `w` on `device`."""
    from . import phantoms
    from .nufft import NUFFT, NUFFTConfig
    dev = torch.device(device)
    x_true, maps, traj = make_inputs(w)
    op = NUFFT(maps.to(dev), traj.to(dev), None, axis=axis_spec(),
               config=NUFFTConfig(ndim=2, traj_units="rad", autotune=autotune), device=dev)
    y = op.A(x_true.to(dev))
    if w["sigma"] > 0:
        y = phantoms.add_noise(y, w["sigma"], seed=1)
    return op, y, x_true, maps, traj


# 16 independent 2D radial recons of uneven size (spatial TV only)
BATCHED = dict(name="batched16_uneven_2d_radial", n=16, sizes=(96, 128, 192, 256, 320), spokes=(32, 200),
               coils=(4, 16), lam_s=1e-3, eps=1e-3, sigma=0.0, seed=7)


def batched_instances(device, spec=BATCHED, autotune: bool = True):
    """Seeded instances: matrix size from spec['sizes'], spokes and coils uniform in
    their ranges, 2N samples per spoke, 10-ellipse phantom, Gaussian coil maps.
    Returns a list of dicts (N, C, spokes, x_true, y, op, regm) on `device`."""
    from . import phantoms
    from .nufft import NUFFT, NUFFTConfig
    from .regularization import RegManager, TVND, TVParams
    dev = torch.device(device)
    g = torch.Generator().manual_seed(spec["seed"])
    out = []
    for i in range(spec["n"]):
        N = spec["sizes"][int(torch.randint(len(spec["sizes"]), (1,), generator=g))]
        spokes = int(torch.randint(spec["spokes"][0], spec["spokes"][1] + 1, (1,), generator=g))
        C = int(torch.randint(spec["coils"][0], spec["coils"][1] + 1, (1,), generator=g))
        x = phantoms.ellipse_phantom(N, seed=1000 * spec["seed"] + i).reshape(1, 1, N, N).to(dev)
        maps = phantoms.coil_maps(N, C).to(dev)
        traj = phantoms.golden_angle_radial(spokes, 2 * N).unsqueeze(0).to(dev)
        op = NUFFT(maps, traj, None, axis=axis_spec(),
                   config=NUFFTConfig(ndim=2, traj_units="rad", autotune=autotune), device=dev)
        y = op.A(x)
        if spec["sigma"] > 0:
            y = phantoms.add_noise(y, spec["sigma"], seed=spec["seed"] + i)
        regm = RegManager([TVND("tv_spatial", TVParams(weight=spec["lam_s"], eps=spec["eps"], axes="spatial"))])
        out.append(dict(N=N, C=C, spokes=spokes, x_true=x, y=y, op=op, regm=regm))
    return out
