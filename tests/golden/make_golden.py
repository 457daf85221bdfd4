"""Generate the golden fixtures in this folder from the reference itself.

Run where the reference package is importable: its path is the first argument
or, without one, the environment variable MRB_REFERENCE_PATH (there is no
default).  The reference is pure Python; it is
imported with two environment workarounds that change no arithmetic:
``DeviceArena`` is created without pinned host memory (no CUDA driver) and
TorchDynamo is disabled (no Inductor toolchain).

    python tests/golden/make_golden.py /path/to/reference [fixture ...]

(fixture names: ptnufft_idx nudft_a tv ncg_small ncg_radial128; all by default)

Writes:
  ptnufft_idx.npz  PTNUFFTAdapter.prepare index tables (the reference's literal
                   integer grid indices) for 2D/3D trajectories incl. edge values
  nudft_a.npz      the reference's _nudft_A ground truth on a small case
  tv.npz           TVND energy/gradient (iso, aniso, axis weights, temporal)
  ncg_small.npz    CGSolver histories and iterates on a small 2D+t problem,
                   driven by the oracle's KB operator (oracle.kb.KBNufft)
  ncg_radial128.npz  CGSolver (FR, Armijo) for 20 iterations on the 128x128,
                   8-coil, 64-spoke x 256-sample golden-angle workload with
                   spatial TV 1e-3, driven by the same KB operator: data,
                   history and final image
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _import_reference(path):
    os.environ["TORCHDYNAMO_DISABLE"] = "1"
    sys.path.insert(0, path)
    import graspcg.workspace.unified_arena as ua
    orig = ua.DeviceArena.__init__

    def _init(self, *a, **k):
        k["pin_memory"] = False
        orig(self, *a, **k)
    ua.DeviceArena.__init__ = _init


def edge_traj(B, nd, K, seed):
    """Random radians in [-pi, pi) plus edge values: -pi, pi-eps, 0, -0, values
    that land on integer grid nodes and just below them."""
    g = torch.Generator().manual_seed(seed)
    t = torch.rand((B, nd, K), generator=g) * (2 * math.pi) - math.pi
    edges = torch.tensor([-math.pi, math.pi - 1e-7, 0.0, -0.0, 1e-8, -1e-8, math.pi / 2, -math.pi / 2,
                          3.0, -3.0, 1e-3, -1e-3], dtype=torch.float32)
    t[:, :, :edges.numel()] = edges.view(1, 1, -1)
    # integer grid nodes for grids of 64, 80 and 48 cells and just below them
    for j, G in enumerate((64, 80, 48)[: max(1, (K - 16) // 128)]):
        n = torch.randint(0, G, (B, nd, 64), generator=g).float()
        on = ((n / G - 0.5) * (2 * math.pi)).float()
        below = torch.nextafter(on, torch.full_like(on, -10.0))
        s = 16 + j * 128
        t[:, :, s:s + 64] = on
        t[:, :, s + 64:s + 128] = below
    return t.float().contiguous()


def make_ptnufft_idx():
    from graspcg.nufft.backends.ptnufft import PTNUFFTAdapter
    out = {}
    cases = [("2d_32", (32, 32), 1500), ("2d_24x40", (24, 40), 1500), ("3d_12x10x8", (12, 10, 8), 500)]
    for name, S, K in cases:
        nd = len(S)
        traj = edge_traj(2, nd, K, seed=len(name) + nd)
        ad = PTNUFFTAdapter(ndim=nd)
        ad.prepare((1,) + S, traj, None, torch.ones((1,) + S, dtype=torch.complex64),
                   torch.complex64, torch.device("cpu"))
        out[f"{name}_traj"] = traj.numpy()
        out[f"{name}_grid"] = np.array(ad._grid_shape, dtype=np.int64)
        out[f"{name}_idx"] = np.stack([i.numpy() for i in ad._idx_B]).astype(np.int32)
        out[f"{name}_beta"] = np.float64(ad._beta)
    np.savez_compressed(os.path.join(HERE, "ptnufft_idx.npz"), **out)


def make_nudft():
    from graspcg.tests.test_nufft_precision_gt import _nudft_A
    g = torch.Generator().manual_seed(7)
    S, C, K, L = (16, 20), 2, 300, 2
    maps = (torch.randn((C,) + S, generator=g, dtype=torch.float64)
            + 1j * torch.randn((C,) + S, generator=g, dtype=torch.float64)) / math.sqrt(C)
    x = (torch.randn((L, 1) + S, generator=g, dtype=torch.float64)
         + 1j * torch.randn((L, 1) + S, generator=g, dtype=torch.float64))
    traj = (torch.rand((2, K), generator=g) * 2 * math.pi - math.pi).float()
    dcf = torch.rand((K,), generator=g) + 0.1
    y = _nudft_A(maps, x, traj, dcf)
    np.savez_compressed(os.path.join(HERE, "nudft_a.npz"), maps=maps.numpy(), x=x.numpy(),
                        traj=traj.numpy(), dcf=dcf.numpy(), y=y.numpy())


def make_tv():
    from graspcg.core.roles import Roles
    from graspcg.regularization.base import RegContext
    from graspcg.regularization.tv_nd import TVND, TVParams
    g = torch.Generator().manual_seed(11)
    out = {}
    x = (torch.randn((5, 1, 12, 10), generator=g) + 1j * torch.randn((5, 1, 12, 10), generator=g))
    x[:, :, 3:6, 2:7] += 3.0       # step edges
    cases = {
        "iso_sp": dict(weight=1e-3, eps=1e-3, axes=(2, 3), isotropic=True),
        "aniso_sp": dict(weight=2e-3, eps=1e-2, axes=(2, 3), isotropic=False),
        "aw_sp": dict(weight=1e-3, eps=1e-3, axes=(2, 3), isotropic=True, axis_weights=(2.0, 0.5)),
        "temporal": dict(weight=5e-3, eps=1e-3, axes="temporal", isotropic=True),
        "iso_3ax": dict(weight=3e-3, eps=1e-3, axes=(0, 2, 3), isotropic=True),
    }
    roles = Roles(1, 1, 2)
    for dt_name, dt in (("c64", torch.complex64), ("c128", torch.complex128)):
        xd = x.to(dt)
        out[f"x_{dt_name}"] = xd.numpy()
        for name, p in cases.items():
            reg = TVND(name, TVParams(**p))
            axes = roles.resolve_axes(p["axes"])
            gbuf = torch.zeros_like(xd)
            ctx = RegContext(x=xd, g=gbuf, diag=None, roles_image=roles, device=xd.device,
                             dtype_c=xd.dtype, dtype_r=xd.real.dtype)
            E = reg.energy_grad_fixed_axes(ctx, axes)
            out[f"{name}_{dt_name}_E"] = np.float64(E.item())
            out[f"{name}_{dt_name}_g"] = gbuf.numpy()
            out[f"{name}_axes"] = np.array(axes, dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "tv.npz"), **out)


def ncg_problem():
    """Small 2D+t problem: 3 frames of 24x24, 3 coils, 600 samples per frame."""
    g = torch.Generator().manual_seed(0)
    N, C, B, K = 24, 3, 3, 600
    maps = ((torch.randn((C, N, N), generator=g) + 1j * torch.randn((C, N, N), generator=g)) / 2).to(torch.complex64)
    traj = (torch.rand((B, 2, K), generator=g) * 2 * math.pi - math.pi).float()
    xt = (torch.randn((B, 1, N, N), generator=g) + 1j * torch.randn((B, 1, N, N), generator=g)).to(torch.complex64)
    noise = (torch.randn((B, C, K), generator=g) + 1j * torch.randn((B, C, K), generator=g)).to(torch.complex64)
    return maps, traj, xt, noise


def kb_operator(maps, traj):
    """The oracle's FP32 KB operator (ortho) with the operator surface the
    reference CGSolver consumes, and Roles(1, 1, 2) for (B, 1, X, Y) images."""
    sys.path.insert(0, REPO)
    from oracle.kb import KBNufft
    from graspcg.core.roles import Roles
    kb = KBNufft(maps, traj, None, dtype=torch.complex64, norm="ortho")

    class Op:
        roles_image = Roles(1, 1, 2)
        roles_kspace = Roles(1, 1, 1)

        def image_shape(self, y):
            return (y.shape[0], 1) + kb.S

        def A(self, x, out=None):
            r = kb.A(x).to(x.dtype)
            return r if out is None else out.copy_(r)

        def AH(self, y, out=None):
            r = kb.AH(y).to(y.dtype)
            return r if out is None else out.copy_(r)

    return Op()


HIST_KEYS = ("f", "gdot", "gdot_at_step", "step", "xnorm", "gnorm", "stepnorm")


def make_ncg():
    from graspcg.solvers.cg import CGSolver, CGConfig
    from graspcg.regularization.manager import RegManager
    from graspcg.regularization.tv_nd import TVND, TVParams

    maps, traj, xt, noise = ncg_problem()
    op = kb_operator(maps, traj)
    y = op.A(xt) + 0.01 * noise
    out = dict(maps=maps.numpy(), traj=traj.numpy(), xt=xt.numpy(), y=y.numpy())
    runs = {
        "fr_armijo": dict(direction="fr", ls_name="armijo", max_iter=12),
        "prplus_armijo": dict(direction="prplus", ls_name="armijo", max_iter=8),
        "dy_armijo": dict(direction="dy", ls_name="armijo", max_iter=8),
        "fr_wolfe": dict(direction="fr", ls_name="wolfe", max_iter=6),
    }
    keys = HIST_KEYS
    for name, kw in runs.items():
        regm = RegManager([TVND("s", TVParams(weight=1e-3, eps=1e-3, axes=(2, 3))),
                           TVND("t", TVParams(weight=5e-3, eps=1e-3, axes="temporal"))],
                          compile_kernels=False)
        s = CGSolver(y=y, nufft_op=op, regm=regm,
                     cfg=CGConfig(devices="cpu", tol_g=0.0, tol_step=0.0, **kw))
        s.run()
        h = s.history()
        for k in keys:
            out[f"{name}_{k}"] = np.array([r[k] for r in h], dtype=np.float64)
        out[f"{name}_x"] = s.result().numpy()
    np.savez_compressed(os.path.join(HERE, "ncg_small.npz"), **out)


def make_ncg_radial128():
    """The reference CGSolver on the single-frame 128x128 golden-angle workload
    (8 coils, 64 spokes x 256 samples, spatial TV 1e-3, no noise), 20 FR/Armijo
    iterations from x = 0."""
    sys.path.insert(0, REPO)
    from mrirecon_b200.workloads import WORKLOADS, make_inputs
    from graspcg.solvers.cg import CGSolver, CGConfig
    from graspcg.regularization.manager import RegManager
    from graspcg.regularization.tv_nd import TVND, TVParams
    w = WORKLOADS["radial128"]
    xt, maps, traj = make_inputs(w)
    op = kb_operator(maps, traj)
    y = op.A(xt)
    regm = RegManager([TVND("s", TVParams(weight=w["lam_s"], eps=w["eps"], axes=(2, 3)))],
                      compile_kernels=False)
    s = CGSolver(y=y, nufft_op=op, regm=regm,
                 cfg=CGConfig(devices="cpu", direction="fr", ls_name="armijo", max_iter=20, tol_g=0.0,
                              tol_step=0.0))
    s.run()
    h = s.history()
    out = dict(y=y.numpy(), x=s.result().numpy())
    for k in HIST_KEYS:
        out[k] = np.array([r[k] for r in h], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "ncg_radial128.npz"), **out)


FIXTURES = {"ptnufft_idx": make_ptnufft_idx, "nudft_a": make_nudft, "tv": make_tv, "ncg_small": make_ncg,
            "ncg_radial128": make_ncg_radial128}

if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MRB_REFERENCE_PATH")
    if not ref:
        sys.exit("usage: make_golden.py /path/to/reference [fixture ...] (or set MRB_REFERENCE_PATH)")
    _import_reference(ref)
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    for name in (sys.argv[2:] or list(FIXTURES)):
        FIXTURES[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
