"""Inputs that must fail cleanly: an error status or a stopped solve, never a
GPU fault or a hang.

* Zero-length or negative sizes are refused by the C ABI's argument checks
  before any CUDA call (so these run on the CPU), and by the adapter.
* Non-finite data: a NaN in y makes the objective and the first slope
  non-finite; the line search refuses it (as graspcg's Armijo does,
  graspcg/numerics/line_search.py:40-45), so the solve stops at iteration 0
  with the line-search reason and the image stays finite.
* A non-adjoint operator pair (A^H replaced by -A^H, so -g is an ascent
  direction): the first slope is positive, the line search refuses it and the
  solve stops at iteration 0.
"""
import ctypes

import pytest
import torch

from mrirecon_b200 import phantoms


def test_zero_and_negative_sizes_refused_without_gpu():
    from mrirecon_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    S = (ctypes.c_int * 2)(32, 32)
    assert lib.mrb_plan_create(ctypes.byref(h), 2, S, 2, 1, 0, 4, 2.0, 1) == 1          # K = 0
    assert "must be positive" in _lib.last_error()
    assert lib.mrb_plan_create(ctypes.byref(h), 2, S, 2, 0, 100, 4, 2.0, 1) == 1        # B = 0
    P = (ctypes.c_void_p * 1)(0)
    out = ctypes.c_double(0.0)
    assert lib.mrb_dots_f64(-1, 1, P, P, None, 0, ctypes.byref(out), None, None) == 1   # negative n
    assert lib.mrb_dots_f64(4, 0, P, P, None, 0, ctypes.byref(out), None, None) == 1    # no pairs
    assert lib.mrb_dots_f64_noalloc(4, 0, P, P, None, 0, ctypes.byref(out), None) == 6  # MRB_ERANGE


@pytest.mark.gpu
def test_adapter_rejects_empty_trajectory(cuda):
    from mrirecon_b200.nufft import B200NUFFTAdapter
    ad = B200NUFFTAdapter(ndim=2)
    maps = phantoms.coil_maps(16, 2).to(cuda)
    with pytest.raises((ValueError, RuntimeError)):
        ad.prepare((2, 16, 16), torch.zeros((1, 2, 0), device=cuda), None, maps, torch.complex64, cuda)


def _problem(cuda, N=32, C=3, F=2):
    from mrirecon_b200.nufft import B200NUFFTAdapter
    maps = phantoms.coil_maps(N, C)
    traj = phantoms.grasp_trajectory(F, 5, 2 * N)
    ad = B200NUFFTAdapter(ndim=2)
    ad.prepare((C, N, N), traj.to(cuda), None, maps.to(cuda), torch.complex64, cuda)
    y = ad.A(phantoms.dynamic_phantom(N, F, seed=2).unsqueeze(1).to(cuda))
    return ad, y


def _solver(op, y, schedule):
    from mrirecon_b200.regularization import RegManager, TVND, TVParams
    from mrirecon_b200.solver import CGConfig, CGSolver
    regm = RegManager([TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial"))])
    return CGSolver(y, op, regm, CGConfig(max_iter=20, tol_g=0.0, tol_step=0.0, schedule=schedule))


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", ["reference", "fast"])
def test_nan_in_data_stops_at_first_line_search(cuda, schedule):
    ad, y = _problem(cuda)
    y[0, 1, 7] = float("nan")
    s = _solver(ad, y, schedule).run()
    assert s.iter == 0 and s.stop_reason.startswith("line-search")
    assert torch.isfinite(torch.view_as_real(s.result())).all()


class _NegatedAdjoint:
    """A forward/adjoint pair that is not adjoint: A^H is replaced by -A^H."""

    def __init__(self, ad):
        self.ad = ad

    def __getattr__(self, name):
        return getattr(self.ad, name)

    def A(self, x, out=None):
        return self.ad.A(x, out=out)

    def AH(self, y, out=None):
        r = self.ad.AH(y, out=out)
        r.neg_()
        return r


@pytest.mark.gpu
def test_non_adjoint_pair_stops_at_first_line_search(cuda):
    ad, y = _problem(cuda)
    s = _solver(_NegatedAdjoint(ad), y, "reference").run()
    assert s.iter == 0 and s.stop_reason.startswith("line-search")
    assert torch.equal(s.result(), torch.zeros_like(s.result()))
