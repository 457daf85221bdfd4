"""The CPU oracle pinned against the reference's own outputs (golden fixtures)."""
import math

import numpy as np
import pytest
import torch

from conftest import golden, rel
from oracle import kb as okb
from oracle.nudft import nudft_forward, nudft_adjoint
from oracle.tv import tv_energy_grad
from oracle.ncg import NCGOracle, NCGConfig, TVSpec


@pytest.mark.parametrize("case", ["2d_32", "2d_24x40", "3d_12x10x8"])
def test_ptnufft_indices_bit_exact(case):
    g = golden("ptnufft_idx.npz")
    traj, G, idx = g[f"{case}_traj"], tuple(int(v) for v in g[f"{case}_grid"]), g[f"{case}_idx"]
    for b in range(traj.shape[0]):
        mine = okb.ptnufft_indices(traj[b], G, 4)
        assert np.array_equal(mine.astype(np.int64), idx[b].astype(np.int64))


def test_beta_matches_reference():
    g = golden("ptnufft_idx.npz")
    assert okb.kb_beta(4, 2.0) == pytest.approx(float(g["2d_32_beta"]), rel=0, abs=1e-12)


def test_nudft_forward_matches_reference_ground_truth():
    g = golden("nudft_a.npz")
    maps, x = torch.from_numpy(g["maps"]), torch.from_numpy(g["x"])
    traj, dcf = torch.from_numpy(g["traj"]), torch.from_numpy(g["dcf"])
    y = nudft_forward(maps, x, traj, dcf)
    assert rel(y, torch.from_numpy(g["y"])) < 1e-13


def test_nudft_adjoint_is_true_adjoint():
    g = golden("nudft_a.npz")
    maps, x = torch.from_numpy(g["maps"]), torch.from_numpy(g["x"])
    traj, dcf = torch.from_numpy(g["traj"]), torch.from_numpy(g["dcf"])
    y = nudft_forward(maps, x, traj, dcf)
    yy = torch.randn_like(y)
    lhs = torch.vdot(y.reshape(-1), yy.reshape(-1))
    rhs = torch.vdot(x.reshape(-1), nudft_adjoint(maps, yy, traj, dcf).reshape(-1))
    assert abs(lhs / rhs - 1) < 1e-12


@pytest.mark.parametrize("S", [(16, 20), (15, 17)])
def test_kb_oracle_vs_nudft(S):
    torch.manual_seed(0)
    C, K = 2, 700
    maps = torch.randn((C,) + S, dtype=torch.complex128)
    traj = (torch.rand(1, 2, K) * 2 * math.pi - math.pi)
    x = torch.randn((1, 1) + S, dtype=torch.complex128)
    op = okb.KBNufft(maps, traj, None, norm="none")
    assert rel(op.A(x), nudft_forward(maps, x, traj[0])) < 1.5e-3
    yy = torch.randn((1, C, K), dtype=torch.complex128)
    assert rel(op.AH(yy), nudft_adjoint(maps, yy, traj[0])) < 1.5e-3
    lhs = torch.vdot(op.A(x).reshape(-1), yy.reshape(-1))
    rhs = torch.vdot(x.reshape(-1), op.AH(yy).reshape(-1))
    assert abs(lhs / rhs - 1) < 1e-12


@pytest.mark.parametrize("name", ["iso_sp", "aniso_sp", "aw_sp", "temporal", "iso_3ax"])
@pytest.mark.parametrize("dt", ["c64", "c128"])
def test_tv_oracle_matches_reference(name, dt):
    g = golden("tv.npz")
    x = torch.from_numpy(g[f"x_{dt}"])
    axes = tuple(int(a) for a in g[f"{name}_axes"])
    p = dict(iso_sp=(1e-3, 1e-3, True, None), aniso_sp=(2e-3, 1e-2, False, None),
             aw_sp=(1e-3, 1e-3, True, (2.0, 0.5)), temporal=(5e-3, 1e-3, True, None),
             iso_3ax=(3e-3, 1e-3, True, None))[name]
    E, gr = tv_energy_grad(x, axes, p[0], p[1], p[2], p[3])
    tol = 1e-5 if dt == "c64" else 1e-12
    assert abs(float(E) - float(g[f"{name}_{dt}_E"])) <= tol * abs(float(g[f"{name}_{dt}_E"]))
    assert rel(gr, torch.from_numpy(g[f"{name}_{dt}_g"])) < tol


@pytest.mark.parametrize("run,direction,ls,iters", [("fr_armijo", "fr", "armijo", 12),
                                                     ("prplus_armijo", "prplus", "armijo", 8),
                                                     ("dy_armijo", "dy", "armijo", 8),
                                                     ("fr_wolfe", "fr", "wolfe", 6)])
def test_ncg_oracle_reproduces_reference_history(run, direction, ls, iters):
    g = golden("ncg_small.npz")
    maps, traj = torch.from_numpy(g["maps"]), torch.from_numpy(g["traj"])
    y = torch.from_numpy(g["y"])
    k = okb.KBNufft(maps, traj, None, dtype=torch.complex64, norm="ortho")
    o = NCGOracle(lambda x: k.A(x).to(torch.complex64), lambda v: k.AH(v).to(torch.complex64), y,
                  torch.zeros((y.shape[0], 1) + tuple(maps.shape[1:]), dtype=torch.complex64),
                  [TVSpec((2, 3), 1e-3), TVSpec((0,), 5e-3)],
                  NCGConfig(direction=direction, ls_name=ls, max_iter=iters, tol_g=0.0, tol_step=0.0))
    o.run()
    f_ref = g[f"{run}_f"]
    assert len(o.hist) == len(f_ref)
    np.testing.assert_allclose([h["f"] for h in o.hist], f_ref, rtol=2e-5)
    np.testing.assert_array_equal([h["step"] for h in o.hist], g[f"{run}_step"])
    np.testing.assert_allclose([h["xnorm"] for h in o.hist], g[f"{run}_xnorm"], rtol=1e-4)
    assert rel(o.x, torch.from_numpy(g[f"{run}_x"])) < 1e-4


def test_pipe_menon_oracle_flattens_radial_density():
    """Oracle of the density-compensation estimator: after the iterations the
    spread of the weighted samples is flat (G G^H w = 1 at the samples) and the
    weights of a radial trajectory grow with |k| (fewer samples per area
    farther out)."""
    import numpy as np
    from oracle.dcf import pipe_menon
    from oracle.kb import KBNufft
    from mrirecon_b200 import phantoms
    N = 32
    traj = phantoms.golden_angle_radial(24, 2 * N).unsqueeze(0)
    w = pipe_menon(traj, (N, N), iters=30)[0]
    k = KBNufft(torch.ones((1, N, N), dtype=torch.complex128), traj, None, norm="none")
    idx, wt = k.idx[0], k.w[0].to(torch.float64)
    grid = torch.zeros(int(np.prod(k.G)), dtype=torch.float64)
    grid.index_add_(0, idx.reshape(-1), (wt * w[:, None]).reshape(-1))
    c = (grid[idx] * wt).sum(-1)
    assert float((c - 1).abs().median()) < 0.05
    # averaged over the spokes (golden-angle gaps vary), the weight is linear in |k|
    spokes, nread = 48, 2 * N
    traj = phantoms.golden_angle_radial(spokes, nread).unsqueeze(0)
    prof = pipe_menon(traj, (N, N), iters=30)[0].reshape(spokes, nread).mean(0)
    kr = torch.linalg.vector_norm(traj[0].to(torch.float64), dim=0).reshape(spokes, nread)[0]
    mid = (kr > 0.3) & (kr < 2.5)
    assert np.corrcoef(kr[mid].numpy(), prof[mid].numpy())[0, 1] > 0.99


# --- Jacobi diagonal (RegManager.add_diag, manager.py:145-218) ------------------
def _diag_loops(x, axes, lam, eps, aw, frame_profile, period=0):
    """Per-voxel loops over the formula of tv_nd.py:113-164 / :187-214."""
    F, _, H, W = x.shape
    P = period or F
    out = np.zeros((F, 1, H, W))
    xs = x.numpy().astype(np.complex128)
    size = {0: P, 1: 1, 2: H, 3: W}
    for f in range(F):
        for i in range(H):
            for j in range(W):
                acc = 0.0
                if frame_profile and 0 in axes:
                    w0 = aw[list(axes).index(0)]
                    fl = f % P
                    acc += 2 * lam * w0 * w0 * (2.0 if (P > 2 and 0 < fl < P - 1) else 1.0)
                else:
                    for a, w in zip(axes, aw):
                        c = {0: f % P, 1: 0, 2: i, 3: j}[a]
                        n = size[a]
                        nb = {0: (f + 1, 0, i, j), 2: (f, 0, i + 1, j), 3: (f, 0, i, j + 1)}.get(a)
                        dv = xs[nb] - xs[f, 0, i, j] if c < n - 1 else 0.0
                        s = lam * w * w / math.sqrt(abs(dv) ** 2 + eps * eps)
                        acc += 2 * s if (n >= 3 and 0 < c < n - 1) else s
                out[f, 0, i, j] = acc
    return out


@pytest.mark.parametrize("axes,aw,profile,period", [((2, 3), (1.0, 1.0), True, 0), ((2, 3), (2.0, 0.5), True, 0),
                                                    ((0,), (1.0,), True, 0), ((0,), (1.5,), False, 0),
                                                    ((0,), (1.0,), False, 3), ((0, 2, 3), (1.0, 1.0, 1.0), True, 3)])
def test_diag_oracle_matches_loops(axes, aw, profile, period):
    from oracle.tv import tv_add_diag
    g = torch.Generator().manual_seed(3)
    x = torch.complex(torch.randn(6, 1, 4, 5, generator=g), torch.randn(6, 1, 4, 5, generator=g)) * 0.01
    D = torch.zeros(6, 1, 4, 5, dtype=torch.float64)
    tv_add_diag(D, x, axes, 2e-3, 1e-3, aw, frame_profile=profile, frame_period=period)
    np.testing.assert_allclose(D.numpy(), _diag_loops(x, axes, 2e-3, 1e-3, aw, profile, period), rtol=1e-12)


def test_diag_oracle_reference_expectations():
    """The reference's own add_diag expectations: the temporal profile of
    test_reg_diag_mapped.py:122-134 (frames 5: (1,2,2,2,1) * 2 lambda) and the
    identity case of test_regularization_ns.py:168-178 (the diagonal grows)."""
    from oracle.tv import tv_add_diag
    D = torch.zeros(5, 1, 2, 2, dtype=torch.float64)
    tv_add_diag(D, torch.zeros(5, 1, 2, 2, dtype=torch.complex64), (0,), 1e-3, 1e-3)
    np.testing.assert_allclose(D.mean(dim=(1, 2, 3)).numpy(), np.array([1, 2, 2, 2, 1]) * 2e-3, atol=1e-12)
    x = torch.randn(4, 1, 8, 8, dtype=torch.complex64, generator=torch.Generator().manual_seed(0)) * 0.01
    D = torch.zeros(4, 1, 8, 8, dtype=torch.float64)
    before = D.clone()
    tv_add_diag(D, x, (2, 3), 1.0, 1e-3)
    assert torch.all(D > before)


def test_majorizer_host_logic():
    """TVND.majorizer_diag / majorizer_profile (tv_nd.py:166-214): host arithmetic."""
    from mrirecon_b200.regularization import RegContext, TVND, TVParams
    from mrirecon_b200.roles import Roles
    roles = Roles(1, 1, 2)
    x = torch.zeros(5, 1, 2, 2, dtype=torch.complex64)
    ctx = RegContext(x=x, g=x, diag=None, roles_image=roles, device=x.device, dtype_c=x.dtype,
                     dtype_r=torch.float32)
    sp = TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial"))
    assert abs(float(sp.majorizer_diag(ctx)) - 2 * 1e-3 * 2) < 1e-9
    assert sp.majorizer_profile(ctx) is None
    aw = TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial", axis_weights=(2.0, 0.5)))
    assert abs(float(aw.majorizer_diag(ctx)) - 2 * 1e-3 * 4.25) < 1e-9
    tm = TVND("t", TVParams(weight=1e-3, eps=1e-3, axes="temporal"))
    (ax, v), = tm.majorizer_profile(ctx)
    assert ax == 0
    np.testing.assert_allclose(v.numpy(), np.array([1, 2, 2, 2, 1]) * 2e-3, rtol=1e-6)


# --- graph Laplacian (graph_laplacian.py:22-321) --------------------------------
def test_graph_oracle_degree_profile_reference_case():
    """Chain graph over 5 frames, weight 2: diagonal (1,2,2,2,1) * 2
    (the expectation of the reference's test_regularization_ns.py:206-235)."""
    from oracle.graph import degree_profile
    W = torch.zeros(5, 5)
    for t in range(4):
        W[t, t + 1] = W[t + 1, t] = 1.0
    np.testing.assert_allclose(degree_profile(W, "none", 2.0).numpy(), [2, 4, 4, 4, 2])
    np.testing.assert_allclose(degree_profile(W, "sym", 2.0).numpy(), [2, 2, 2, 2, 2])


@pytest.mark.parametrize("norm", ["none", "rw", "sym"])
def test_graph_oracle_gradient_matches_finite_difference(norm):
    """Directional derivative of the energy against central differences (the
    reference's test_regularization_ns.py:238-280 checks the sym case the same way)."""
    from oracle.graph import graph_energy_grad, laplacian
    g = torch.Generator().manual_seed(4)
    W = torch.rand(6, 6, generator=g, dtype=torch.float64)
    L = laplacian(W, norm)
    if norm == "rw":   # I - D^-1 W is not symmetric: the energy's gradient is (L + L^T)/2 x
        L = 0.5 * (L + L.T)
    x = torch.randn(6, 1, 4, 4, dtype=torch.complex128, generator=g) * 0.05
    d = torch.randn(6, 1, 4, 4, dtype=torch.complex128, generator=g) * 0.1
    _, gr = graph_energy_grad(x, L, 1e-3)
    h = 1e-5
    fd = (graph_energy_grad(x + h * d, L, 1e-3)[0] - graph_energy_grad(x - h * d, L, 1e-3)[0]) / (2 * h)
    an = (gr.conj() * d).real.sum()
    assert abs(float(an - fd)) <= 1e-9 * max(1.0, abs(float(an)))


def test_graph_laplacian_host_matrix_matches_oracle():
    """GraphLaplacian's dense lambda L (host arithmetic) equals the oracle's for
    dense and sparse W and all three normalisations."""
    from oracle.graph import laplacian
    from mrirecon_b200.regularization import GraphLaplacian, GraphLapParams
    g = torch.Generator().manual_seed(5)
    W = torch.rand(7, 7, generator=g)
    W[3, :] = 0
    W[:, 3] = 0                      # an isolated frame
    for norm in ("none", "rw", "sym"):
        for Win in (W, W.to_sparse()):
            r = GraphLaplacian("g", Win, GraphLapParams(weight=0.5, normalize=norm))
            np.testing.assert_allclose(r.laplacian().numpy(), 0.5 * laplacian(W, norm).numpy(), rtol=1e-6,
                                       atol=1e-7)
    with pytest.raises(ValueError):
        GraphLaplacian("g", W, GraphLapParams(weight=0.5, normalize="row"))


def test_basis_push_oracle_reference_expectations():
    """The reference's temporal-basis push (test_reg_diag_mapped.py:93-122):
    |U|^2 = [[1,0,0],[0,4,0]], k = 2 lambda * 2 axes: diag_V = (k, 4k, 0)."""
    from oracle.mapping import basis_diag_push, basis_profile_push
    U = torch.tensor([[1.0, 0.0, 0.0], [0.0, 2.0, 0.0]])
    k = 2.0 * 1e-3 * 2.0
    DV = basis_diag_push(U, torch.full((2, 1, 3, 2), k, dtype=torch.float64))
    np.testing.assert_allclose(DV[:, 0, 0, 0].numpy(), [k, 4 * k, 0.0], atol=1e-15)
    np.testing.assert_allclose(basis_profile_push(U, torch.tensor([1.0, 1.0])).numpy(), [1.0, 4.0, 0.0])


def test_fused_solver_term_classification():
    """Host logic: which regularisers the fused solver evaluates as TV terms
    (a TVND, bare or behind identity / scale maps), which as graph terms, and
    which it refuses (parameter-space mappings)."""
    from mrirecon_b200.mapping import (ComposeOp, IdentityOp, MappedRegularizer, ScaleOp, TemporalBasisOp,
                                       Transformed, fused_tv)
    from mrirecon_b200.regularization import GraphLaplacian, GraphLapParams, RegManager, TVND, TVParams
    from mrirecon_b200.roles import Roles
    tv = TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial"))
    assert fused_tv(tv) is tv
    assert fused_tv(MappedRegularizer("m", tv, IdentityOp())) is tv
    assert fused_tv(Transformed(tv, ScaleOp(), "t")) is tv
    assert fused_tv(MappedRegularizer("c", tv, ComposeOp([IdentityOp(), ScaleOp()]))) is tv
    basis = MappedRegularizer("p", tv, TemporalBasisOp(U=torch.randn(4, 2)))
    assert fused_tv(basis) is None
    gl = GraphLaplacian("g", torch.ones(4, 4), GraphLapParams(weight=1.0))
    roles = Roles(1, 1, 2)
    terms = RegManager([tv, gl, Transformed(tv, IdentityOp(), "t")]).terms(roles)
    assert len(terms) == 2 and all(t.naxes == 2 for t in terms)
    with pytest.raises(TypeError):
        RegManager([basis]).terms(roles)
    Lg = gl.laplacian().numpy()          # W = ones, diagonal removed: deg 3, L = 3 I - (J - I) = 4 I - J
    np.testing.assert_allclose(Lg, 4 * np.eye(4) - np.ones((4, 4)), atol=1e-12)
