"""graspcg's own front-end and solver driving this library: the drop-in, executed.

graspcg is imported from an installed copy of the reference: the directory in
the environment variable MRB_GRASPCG_PATH, else ``baseline/_ref`` beside this
repository.  The tests skip, saying so, when neither holds an importable
graspcg.

The B200 backend is registered in-process exactly as INTEGRATION.md tells a
graspcg maintainer to do it, without editing any reference file:

1. a module ``graspcg.nufft.backends.b200`` that re-exports
   ``B200NUFFTAdapter``;
2. in ``graspcg/nufft/api.py`` a ``'b200'`` branch beside ``'torchkb'`` in
   ``NUFFT.__init__``'s backend selection (api.py:111-143), and the fold-path
   tests of ``A`` and ``AH`` (api.py:195, 248) extended from ``== 'torchkb'``
   to ``in ('torchkb', 'b200')``.

Step 2 is applied to api.py's source text in memory (each anchor must match
exactly once) and the patched module stands in for ``graspcg.nufft.api`` for
the duration of a test.  Two environment workarounds that change no
arithmetic: TorchDynamo is disabled (graspcg wraps small kernels in
torch.compile) and, without a GPU, ``DeviceArena`` gets no pinned memory.

The CPU test runs the same registration with an adapter around the oracle's
KB operator, so the plumbing is checked here; the GPU tests run the real
adapter: graspcg's front-end against this package's, and graspcg's CGSolver
(with this package's TVND in graspcg's RegManager) against this package's
CGSolver.
"""
import importlib
import os
import sys
import types

import numpy as np
import pytest
import torch

from conftest import ROOT, rel

ANCHOR_BRANCH = "        elif self.cfg.backend == 'cufi':\n"
B200_BRANCH = """        elif self.cfg.backend == 'b200':
            from .backends.b200 import B200NUFFTAdapter
            be = B200NUFFTAdapter(ndim=ndim)
            be.traj_units = self.cfg.traj_units
            be.apply_dcf_in_fwd = self.cfg.apply_dcf_in_fwd
            be.apply_dcf_in_adj = self.cfg.apply_dcf_in_adj
            be.dcf_mode = self.cfg.dcf_mode
            self._backend = be
            like_prod = int(maps.shape[0])

"""
ANCHOR_FOLD_A = "        if self.cfg.backend == 'torchkb':\n            # TorchKb canonical out view"
ANCHOR_FOLD_AH = "        if self.cfg.backend == 'torchkb':\n            # Canonical input view"


def _graspcg_path():
    p = os.environ.get("MRB_GRASPCG_PATH") or os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isfile(os.path.join(p, "graspcg", "nufft", "api.py")):
        pytest.skip(f"graspcg is not installed at {p} (set MRB_GRASPCG_PATH to an installed copy)")
    return p


def _patched_api_source(src):
    for anchor in (ANCHOR_BRANCH, ANCHOR_FOLD_A, ANCHOR_FOLD_AH):
        assert src.count(anchor) == 1, f"api.py anchor not found exactly once: {anchor!r}"
    src = src.replace(ANCHOR_BRANCH, B200_BRANCH + ANCHOR_BRANCH)
    for anchor in (ANCHOR_FOLD_A, ANCHOR_FOLD_AH):
        src = src.replace(anchor, anchor.replace("== 'torchkb'", "in ('torchkb', 'b200')"))
    return src


@pytest.fixture
def graspcg_b200(monkeypatch):
    """graspcg with the b200 backend registered; yields a namespace of its modules.
    `ns.register(cls)` sets the adapter class the b200 module re-exports."""
    path = _graspcg_path()
    monkeypatch.syspath_prepend(path)
    monkeypatch.setattr(torch._dynamo.config, "disable", True)
    api0 = importlib.import_module("graspcg.nufft.api")
    assert os.path.dirname(os.path.dirname(os.path.dirname(api0.__file__))) == os.path.abspath(path)
    import graspcg.workspace.unified_arena as ua
    if not torch.cuda.is_available():
        orig = ua.DeviceArena.__init__

        def _init(self, *a, **k):
            k["pin_memory"] = False
            orig(self, *a, **k)
        monkeypatch.setattr(ua.DeviceArena, "__init__", _init)
    b200_mod = types.ModuleType("graspcg.nufft.backends.b200")
    monkeypatch.setitem(sys.modules, "graspcg.nufft.backends.b200", b200_mod)
    src = _patched_api_source(open(api0.__file__).read())
    api = types.ModuleType("graspcg.nufft.api")
    api.__file__ = api0.__file__
    api.__package__ = "graspcg.nufft"
    monkeypatch.setitem(sys.modules, "graspcg.nufft.api", api)
    exec(compile(src, api0.__file__, "exec"), api.__dict__)

    ns = types.SimpleNamespace(api=api)
    ns.register = lambda cls: setattr(b200_mod, "B200NUFFTAdapter", cls)
    from graspcg.core.roles import Roles
    from graspcg.nufft.layout import AxisSpec
    from graspcg.regularization.manager import RegManager
    from graspcg.regularization.tv_nd import TVND, TVParams
    from graspcg.solvers.cg import CGConfig, CGSolver
    ns.Roles, ns.AxisSpec, ns.RegManager, ns.CGConfig, ns.CGSolver = Roles, AxisSpec, RegManager, CGConfig, CGSolver
    ns.TVND, ns.TVParams = TVND, TVParams
    yield ns


def _axis(ns):
    return ns.AxisSpec(image=("B", "coil", "X", "Y"), kspace=("B", "coil", "K"), image_fft=("X", "Y"),
                       coil="coil")


def _problem(N=48, F=5, C=4, spf=7, nread=96):
    from mrirecon_b200 import phantoms
    maps = phantoms.coil_maps(N, C)
    traj = phantoms.grasp_trajectory(F, spf, nread)
    xt = phantoms.dynamic_phantom(N, F, seed=5).unsqueeze(1)
    return maps, traj, xt


class OracleAdapter:
    """The torchkb adapter surface around the oracle's FP32 KB operator (CPU),
    standing in for the B200 adapter in the CPU plumbing test."""

    backend_name = "oracle"

    def __init__(self, ndim):
        self.ndim = ndim
        self.traj_units, self.dcf_mode = "rad", "balanced"
        self.apply_dcf_in_fwd, self.apply_dcf_in_adj = False, True

    def prepare(self, im_shape, traj, dcf, maps, dtype=torch.complex64, device=None, like_prod=1):
        from oracle.kb import KBNufft
        self.kb = KBNufft(maps, traj, dcf, dtype=torch.complex64, norm="ortho")
        self.K = int(traj.shape[-1])

    def k_per_frame(self):
        return self.K

    def A(self, x, out=None):
        r = self.kb.A(x).to(x.dtype)
        return r if out is None else out.copy_(r)

    def AH(self, y, out=None):
        r = self.kb.AH(y).to(y.dtype)
        return r if out is None else out.copy_(r)


def test_registration_plumbing_cpu(graspcg_b200):
    """graspcg's front-end builds the registered adapter for backend 'b200' and
    takes its fold path; graspcg's CGSolver runs on it and matches the oracle's
    restatement of the same solve step for step."""
    ns = graspcg_b200
    ns.register(OracleAdapter)
    # (a sparse sampling: graspcg stops at its first line-search failure, which
    # the FR direction's first beta = 1 causes early on densely sampled data)
    maps, traj, xt = _problem(N=32, F=3, C=3, spf=5, nread=64)
    op = ns.api.NUFFT(maps, traj, None, axis=_axis(ns),
                      config=ns.api.NUFFTConfig(ndim=2, backend="b200", traj_units="rad"))
    assert isinstance(op._backend, OracleAdapter)
    y = op.A(xt)
    assert y.shape == (3, 3, 5 * 64)
    assert rel(y, op._backend.A(xt)) == 0.0
    op.roles_image = ns.Roles(1, 1, 2)
    regm = ns.RegManager([ns.TVND("s", ns.TVParams(weight=1e-3, eps=1e-3, axes=(2, 3)))], compile_kernels=False)
    s = ns.CGSolver(y, op, regm, ns.CGConfig(devices="cpu", max_iter=5, tol_g=0.0, tol_step=0.0))
    s.run()
    from oracle.ncg import NCGConfig, NCGOracle, TVSpec
    o = NCGOracle(op._backend.A, op._backend.AH, y, torch.zeros_like(xt), [TVSpec((2, 3), 1e-3)],
                  NCGConfig(max_iter=5, tol_g=0.0, tol_step=0.0)).run()
    fs = [r["f"] for r in s.history()]
    assert len(fs) == len(o.hist) == 5
    np.testing.assert_allclose(fs, [h["f"] for h in o.hist], rtol=1e-5)


@pytest.mark.gpu
def test_graspcg_frontend_on_b200(cuda, graspcg_b200):
    """graspcg's NUFFT(backend='b200') gives exactly this package's adapter
    results (same kernels, through graspcg's views) and the FP64 oracle's
    within 1e-5."""
    from oracle import kb as okb
    from mrirecon_b200.nufft import B200NUFFTAdapter
    ns = graspcg_b200
    ns.register(B200NUFFTAdapter)
    maps, traj, xt = _problem()
    op = ns.api.NUFFT(maps.to(cuda), traj.to(cuda), None, axis=_axis(ns),
                      config=ns.api.NUFFTConfig(ndim=2, backend="b200", traj_units="rad"))
    assert isinstance(op._backend, B200NUFFTAdapter)
    ad = B200NUFFTAdapter(ndim=2)
    ad.prepare(tuple(maps.shape), traj.to(cuda), None, maps.to(cuda), torch.complex64, cuda)
    x = xt.to(cuda)
    y = op.A(x)
    assert torch.equal(y, ad.A(x))
    xh = op.AH(y)
    assert torch.equal(xh, ad.AH(y))
    orc = okb.KBNufft(maps.to(torch.complex128), traj, None, dtype=torch.complex128)
    assert rel(y, orc.A(xt)) < 1e-5
    assert rel(xh, orc.AH(y.cpu())) < 1e-5


@pytest.mark.gpu
def test_graspcg_cgsolver_on_b200_operator(cuda, graspcg_b200):
    """graspcg's CGSolver (FR, Armijo) on graspcg's front-end with the b200
    backend and this package's TVND terms in graspcg's RegManager: 10
    iterations equal this package's CGSolver (reference schedule) on the same
    problem, objective history rel <= 1e-4, same accepted steps, image <= 1e-3."""
    from mrirecon_b200 import phantoms
    from mrirecon_b200.nufft import B200NUFFTAdapter
    from mrirecon_b200.regularization import RegManager, TVND, TVParams
    from mrirecon_b200.solver import CGConfig, CGSolver
    ns = graspcg_b200
    ns.register(B200NUFFTAdapter)
    maps, traj, xt = _problem()
    op = ns.api.NUFFT(maps.to(cuda), traj.to(cuda), None, axis=_axis(ns),
                      config=ns.api.NUFFTConfig(ndim=2, backend="b200", traj_units="rad"))
    op.roles_image = ns.Roles(1, 1, 2)      # (B, 1, X, Y) images: the coil slot counts
    y = phantoms.add_noise(op.A(xt.to(cuda)), 1e-3, seed=1)

    def tv_terms():
        return [TVND("s", TVParams(weight=1e-3, eps=1e-3, axes=(2, 3))),
                TVND("t", TVParams(weight=5e-3, eps=1e-3, axes=(0,)))]

    ref = ns.CGSolver(y, op, ns.RegManager(tv_terms(), compile_kernels=False),
                      ns.CGConfig(devices="cuda", max_iter=10, tol_g=0.0, tol_step=0.0))
    ref.run()
    ad = B200NUFFTAdapter(ndim=2)
    ad.prepare(tuple(maps.shape), traj.to(cuda), None, maps.to(cuda), torch.complex64, cuda)
    mine = CGSolver(y, ad, RegManager(tv_terms()),
                    CGConfig(max_iter=10, tol_g=0.0, tol_step=0.0, schedule="reference"))
    mine.run()
    hr, hm = ref.history(), mine.history()
    assert len(hr) == len(hm) == 10
    np.testing.assert_array_equal([r["step"] for r in hm], [r["step"] for r in hr])
    np.testing.assert_allclose([r["f"] for r in hm], [r["f"] for r in hr], rtol=1e-4)
    assert rel(mine.result(), ref.result()) < 1e-3
