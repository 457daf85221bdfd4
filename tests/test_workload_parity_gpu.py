"""Parity at the sizes the benchmarks run, not only at toy sizes.

* GRASP operator (256x256, 34 frames, 12 coils, 21 x 512 golden-angle samples
  per frame) with the plan options the bench uses (autotuned spread tile,
  chunk and kernel; centre tiles split into many chunks): A and A^H against
  the oracle's FP64 Kaiser-Bessel gridding, rel-L2 <= 1e-5, adjoint ratio
  within 1e-5.
* The 128x128 single-frame workload (8 coils, 64 x 256 golden-angle samples,
  spatial TV 1e-3): 20 FR/Armijo iterations of both solver schedules against
  the reference CGSolver run in ``ncg_radial128.npz`` (made by
  ``make_golden.py`` from the reference itself): identical accepted steps,
  objective history rel <= 1e-4, final image rel-L2 <= 1e-3.
* The batched workload's size classes: one operator per matrix size in
  {96, 128, 192, 256, 320} with 2N samples per spoke, 320x320 at 16 coils,
  autotuned like the batch: A and A^H against the FP64 oracle, rel-L2 <= 1e-5.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel
from oracle import kb as okb
from mrirecon_b200 import phantoms
from mrirecon_b200.nufft import B200NUFFTAdapter, NUFFT, NUFFTConfig
from mrirecon_b200.regularization import RegManager, TVND, TVParams
from mrirecon_b200.solver import CGConfig, CGSolver
from mrirecon_b200.workloads import WORKLOADS, axis_spec, make_inputs

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _rand_c(shape, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                         torch.randn(shape, generator=g, dtype=torch.float64))


def _check_operator(op, maps, traj, x, seed):
    """A(x) and A^H(y) of `op` (front-end NUFFT) against the FP64 oracle."""
    dev = torch.device("cuda")
    orc = okb.KBNufft(maps.to(torch.complex128), traj, None, dtype=torch.complex128, norm="ortho")
    C, K = int(maps.shape[0]), int(traj.shape[-1])
    y = _rand_c((x.shape[0], C, K), seed)
    yg = op.A(x.to(dev, torch.complex64)).cpu()
    xg = op.AH(y.to(dev, torch.complex64)).cpu()
    ya = orc.A(x.to(torch.complex128))
    assert rel(yg, ya) < TOL, f"forward rel {rel(yg, ya):.3e}"
    del ya
    xa = orc.AH(y)
    assert rel(xg, xa) < TOL, f"adjoint rel {rel(xg, xa):.3e}"
    lhs = torch.vdot(yg.to(torch.complex128).reshape(-1), y.reshape(-1))
    rhs = torch.vdot(x.to(torch.complex128).reshape(-1), xg.to(torch.complex128).reshape(-1))
    assert abs(complex(lhs / rhs) - 1) < 1e-5


def test_grasp_operator_vs_fp64_oracle(cuda):
    w = WORKLOADS["grasp"]
    x_true, maps, traj = make_inputs(w)
    op = NUFFT(maps.to(cuda), traj.to(cuda), None, axis=axis_spec(),
               config=NUFFTConfig(ndim=2, traj_units="rad", autotune=True), device=cuda)
    assert op.backend.plan.info()["fft_mode"] == 1       # the bench's fused FFT passes
    # the phantom plus a little white noise, so that high frequencies are tested too
    x = x_true.to(torch.complex128) + 0.05 * _rand_c(x_true.shape, 21)
    _check_operator(op, maps, traj, x, 22)


def _radial128_solver(schedule, **kw):
    g = golden("ncg_radial128.npz")
    w = WORKLOADS["radial128"]
    _, maps, traj = make_inputs(w)
    dev = torch.device("cuda")
    ad = B200NUFFTAdapter(ndim=2)
    ad.prepare(tuple(maps.shape), traj.to(dev), None, maps.to(dev), torch.complex64, dev)
    regm = RegManager([TVND("s", TVParams(weight=w["lam_s"], eps=w["eps"], axes="spatial"))])
    cfg = CGConfig(direction="fr", ls_name="armijo", max_iter=len(g["f"]), tol_g=0.0, tol_step=0.0,
                   schedule=schedule, **kw)
    return g, CGSolver(torch.from_numpy(g["y"]).to(dev), ad, regm, cfg)


@pytest.mark.parametrize("schedule,graph", [("reference", False), ("fast", False), ("fast", True)])
def test_radial128_20_iterations_vs_reference_cgsolver(cuda, schedule, graph):
    g, s = _radial128_solver(schedule, cuda_graph=graph)
    s.run()
    h = s.history()
    assert len(h) == len(g["f"]) == 20
    np.testing.assert_array_equal([r["step"] for r in h], g["step"])
    np.testing.assert_allclose([r["f"] for r in h], g["f"], rtol=1e-4)
    np.testing.assert_allclose([r["xnorm"] for r in h], g["xnorm"], rtol=1e-4)
    assert rel(s.result(), torch.from_numpy(g["x"])) < 1e-3


@pytest.mark.parametrize("N,C,spokes", [(96, 15, 108), (128, 11, 192), (192, 12, 116), (256, 16, 178),
                                        (320, 16, 51)])
def test_batched_size_classes_vs_fp64_oracle(cuda, N, C, spokes):
    maps = phantoms.coil_maps(N, C)
    traj = phantoms.golden_angle_radial(spokes, 2 * N).unsqueeze(0)
    op = NUFFT(maps.to(cuda), traj.to(cuda), None, axis=axis_spec(),
               config=NUFFTConfig(ndim=2, traj_units="rad", autotune=True), device=cuda)
    x = phantoms.ellipse_phantom(N, seed=N).reshape(1, 1, N, N).to(torch.complex128)
    x = x + 0.05 * _rand_c(x.shape, N)
    _check_operator(op, maps, traj, x, N + 1)
