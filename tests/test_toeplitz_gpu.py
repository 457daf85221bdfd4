"""Toeplitz normal operator A^H A (transfer function on the 2x grid) and the
``schedule="toeplitz"`` NCG: parity against the gridded operator, the FP64
NUDFT normal operator (the physics truth) and the gridded solve.

Stated tolerances: the Toeplitz A^H A differs from the gridded A^H(A x) and
from the exact NUDFT normal operator by the KB approximation (W=4, osf=2):
rel-L2 <= 3e-3; it is Hermitian to FP32 rounding (1e-5)."""
import pytest
import torch

from conftest import rel
from oracle.nudft import nudft_forward, nudft_adjoint
from mrirecon_b200 import phantoms
from mrirecon_b200.nufft import B200NUFFTAdapter
from mrirecon_b200.regularization import RegManager, TVND, TVParams
from mrirecon_b200.solver import CGConfig, CGSolver

pytestmark = pytest.mark.gpu


def _adapter(maps, traj, dev, dcf=None, **kw):
    ad = B200NUFFTAdapter(ndim=2, **kw)
    ad.prepare(tuple(maps.shape), traj.to(dev), None if dcf is None else dcf.to(dev), maps.to(dev), torch.complex64,
               torch.device(dev))
    return ad


@pytest.mark.parametrize("S,C,B,kw", [((32, 32), 3, 2, {}), ((48, 40), 2, 3, {}),
                                      ((32, 32), 2, 2, {"dcf": True}), ((32, 32), 3, 2, {"psf": "kb"})])
def test_normal_operator_parity(cuda, S, C, B, kw):
    """psf="exact" (default): the Toeplitz A^H A is the FP64 NUDFT normal
    operator to FP32 rounding (1e-5) and within the KB error of the gridded
    A^H(A x) (3e-3); psf="kb" is within 3e-3 of both."""
    maps = phantoms.coil_maps(max(S), C)[:, :S[0], :S[1]].contiguous().to(torch.complex64)
    traj = torch.stack([phantoms.golden_angle_radial(15, 2 * max(S), 15 * b) for b in range(B)])
    dcf = None
    if kw.get("dcf"):
        dcf = torch.linalg.vector_norm(traj, dim=1) / 3.2 + 0.01
    ad = _adapter(maps, traj, cuda, dcf)
    mode = kw.get("psf", "exact")
    ad.prepare_toeplitz(mode)
    g = torch.Generator().manual_seed(5)
    x = torch.randn((B, 1) + S, generator=g, dtype=torch.complex64).to(cuda)
    z = torch.randn((B, 1) + S, generator=g, dtype=torch.complex64).to(cuda)
    t = ad.AHA(x)
    grid = ad.AH(ad.A(x))
    assert rel(t, grid) < 3e-3
    # exact FP64 normal operator (ortho scale 1/sqrt(prod G); DCF weights w on the data)
    s2 = 1.0 / (4 * S[0] * S[1])
    m64 = maps.to(torch.complex128)
    w = None if dcf is None else dcf.to(torch.float64)
    ex = []
    for b in range(B):
        yb = nudft_forward(m64, x[b:b + 1].cpu().to(torch.complex128), traj[b])
        if w is not None:
            yb = yb * w[b]
        ex.append(nudft_adjoint(m64, yb, traj[b], None))
    ex = torch.cat(ex) * s2
    assert rel(t, ex) < (1e-5 if mode == "exact" else 3e-3)
    # Hermitian
    lhs = torch.vdot(z.reshape(-1), t.reshape(-1))
    rhs = torch.vdot(ad.AHA(z).reshape(-1), x.reshape(-1))
    assert abs(complex(lhs / rhs) - 1) < 1e-5


def test_toeplitz_schedule_matches_gridded_solve(cuda):
    """2D+t GRASP-like problem: the Toeplitz schedule reaches the windowed
    tolerance; its result, scored with the gridded operator, has an objective
    within 2% of the gridded solve's and an image within 2e-2.  The two solves
    minimise different data terms (the exact NUDFT normal operator against the
    KB-gridded one, which also generated the data); at convergence the data term
    is a small difference of large numbers, so the KB error of ~6e-4 on ||A x||^2
    shows up as percent-level objective differences."""
    N, C, F = 64, 4, 6
    x_true = phantoms.dynamic_phantom(N, F, seed=2).unsqueeze(1)
    maps = phantoms.coil_maps(N, C)
    traj = phantoms.grasp_trajectory(F, 13, 2 * N)
    ad = _adapter(maps, traj, cuda)
    y = phantoms.add_noise(ad.A(x_true.to(cuda)), 1e-3, seed=3)
    regm = RegManager([TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial")),
                       TVND("t", TVParams(weight=5e-3, eps=1e-3, axes="temporal"))])
    cfg = dict(max_iter=400, stop_window=10, stop_tol=1e-4, restart=True)
    sg = CGSolver(y, ad, regm, CGConfig(**cfg)).run()
    st = CGSolver(y, ad, regm, CGConfig(schedule="toeplitz", **cfg)).run()
    assert st.stop_reason.startswith("relative") and sg.stop_reason.startswith("relative")
    fg, ft = sg.objective(), st.objective()
    assert abs(ft - fg) <= 2e-2 * abs(fg)
    assert rel(st.result(), sg.result()) < 2e-2
    # the accepted objectives decrease, and the device recurrence for ||r||^2
    # reproduces the Toeplitz-model objective 0.5 (x^H T x - 2 Re<x, A^H y> + ||y||^2)
    # + TV(x) evaluated directly at the result (TV = gridded objective - gridded data term)
    fs = [h["f"] for h in st.history()]
    assert all(b <= a * (1 + 1e-6) for a, b in zip(fs, fs[1:]))
    x = st.result()
    d = lambda a, b: float(torch.vdot(a.reshape(-1), b.reshape(-1)).real.double())
    data_t = 0.5 * (d(x, ad.AHA(x)) - 2.0 * d(x, ad.AH(y)) + d(y, y))
    r = ad.A(x) - y
    f_t = data_t + (ft - 0.5 * d(r, r))
    assert abs(st.history()[-1]["f_accepted"] - f_t) <= 1e-3 * abs(f_t)
