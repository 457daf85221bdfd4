"""Mapped regularisers and the frame-mixing kernels on the GPU against the
FP64 oracle and the reference's own test expectations.

Tolerances: frame mixes rel <= 1e-5 (FP32 FMAs against FP64); mapped TV
energies/gradients rel <= 1e-5; diagonal pushes rel <= 1e-6.
"""
import numpy as np
import pytest
import torch

from conftest import rel
from oracle.mapping import basis_adjoint, basis_diag_push, basis_forward
from oracle.tv import tv_energy_grad
from mrirecon_b200 import _lib
from mrirecon_b200.mapping import (ComposeOp, IdentityOp, MappedRegularizer, ScaleOp, TemporalBasisOp, Transformed,
                                   _mix, _mix_real)
from mrirecon_b200.regularization import RegManager, TVND, TVParams
from mrirecon_b200.roles import Roles

pytestmark = pytest.mark.gpu


class _Shard:
    b_start = 0


class _Scale:
    def __init__(self, inv):
        self.inv = float(inv)

    def inv_for_shard(self, shard, anchor):
        return torch.full((anchor.shape[0],) + (1,) * (anchor.ndim - 1), self.inv, device=anchor.device)


class _WS:
    def __init__(self, **bufs):
        self._b = dict(bufs)
        self.plan = type("Plan", (), {"roles_image": Roles(1, 1, 2)})()
        self.scale = bufs.pop("scale", None)
        self._b.pop("scale", None)

    def has(self, k):
        return k in self._b

    def get(self, k, i=0):
        return self._b[k]

    def shard_for_index(self, i):
        return _Shard()


def _c(shape, seed, scale=1.0):
    g = torch.Generator().manual_seed(seed)
    return torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g)) * scale


@pytest.mark.parametrize("Ro,Ri", [(34, 4), (4, 34), (128, 128), (1, 1)])
def test_frame_mix_vs_oracle(cuda, Ro, Ri):
    M = _c((Ro, Ri), 1)
    x = _c((Ri, 1, 10, 13), 2)
    o = _c((Ro, 1, 10, 13), 3)
    out = o.to(cuda)
    _mix(M, x.to(cuda), out, accumulate=True)
    ref = o.to(torch.complex128) + (M.to(torch.complex128) @ x.reshape(Ri, -1).to(torch.complex128)).reshape(o.shape)
    assert rel(out.cpu(), ref) < 1e-5
    # M^H applied from M stored (Ri, Ro)
    Mt = _c((Ri, Ro), 4)
    out2 = torch.empty((Ro, 1, 10, 13), dtype=torch.complex64, device=cuda)
    _mix(Mt, x.to(cuda), out2, conj_t=True)
    ref2 = (Mt.to(torch.complex128).conj().T @ x.reshape(Ri, -1).to(torch.complex128)).reshape(out2.shape)
    assert rel(out2.cpu(), ref2) < 1e-5
    # real data, transposed matrix
    R = torch.rand(Ri, Ro)
    k = torch.rand(Ri, 1, 10, 13)
    outr = torch.zeros(Ro, 1, 10, 13, device=cuda)
    _mix_real(R, k.to(cuda), outr, transpose=True)
    refr = (R.double().T @ k.reshape(Ri, -1).double()).reshape(outr.shape)
    assert rel(outr.cpu().double(), refr) < 1e-5


def test_mapped_temporal_basis_updates_gV_not_var(cuda):
    """The reference's test_regularization_ns.py:123-148 on one shard, with the
    values checked: E = TV(U V), g_V = U^H grad TV(U V), g(var) untouched."""
    T, K = 6, 3
    U = torch.randn(T, K, generator=torch.Generator().manual_seed(0))
    V = _c((K, 1, 8, 8), 5, 0.1)
    x = torch.zeros((T, 1, 8, 8), dtype=torch.complex64, device=cuda)
    g = torch.zeros_like(x)
    gV = torch.zeros((K, 1, 8, 8), dtype=torch.complex64, device=cuda)
    ws = _WS(var=x, grad=g, V=V.to(cuda), g_V=gV)
    tv = TVND("tv_sp", TVParams(weight=0.5, eps=1e-3, axes="spatial", isotropic=True))
    regm = RegManager([MappedRegularizer(name="tv_UV", inner=tv, op=TemporalBasisOp(U=U))])
    E = float(regm.energy_and_grad(ws))
    assert torch.count_nonzero(g) == 0
    u = basis_forward(U, V)
    Eo, gu = tv_energy_grad(u, (2, 3), 0.5, 1e-3)
    assert abs(E - float(Eo)) <= 1e-5 * abs(float(Eo))
    assert rel(gV.cpu(), basis_adjoint(U, gu)) < 1e-5


def test_transformed_diag_pushes_reference_expectations(cuda):
    """test_reg_diag_mapped.py:72-122: a ScaleOp (1/s = 2.5) pushes
    k (2.5)^2 into the image diagonal; a TemporalBasisOp with |U|^2 =
    [[1,0,0],[0,4,0]] pushes (k, 4k, 0) into diag_V, k = 2 lambda * 2."""
    k = 2.0 * 1e-3 * 2.0
    x = torch.zeros((2, 1, 4, 4), dtype=torch.complex64, device=cuda)
    D = torch.zeros((2, 1, 4, 4), device=cuda)
    reg = TVND(name="tv", params=TVParams(weight=1e-3, eps=1e-3, axes="spatial"))
    ws = _WS(var=x, diag=D, scale=_Scale(2.5))
    RegManager([Transformed(base=reg, op=ScaleOp(), name="tv_scaled", params=reg.params)]).add_diag(ws)
    assert torch.allclose(D.cpu(), torch.full((2, 1, 4, 4), k * 2.5 ** 2), atol=1e-7, rtol=0)
    U = torch.tensor([[1.0, 0.0, 0.0], [0.0, 2.0, 0.0]])
    x = torch.zeros((2, 1, 3, 2), dtype=torch.complex64, device=cuda)
    V = torch.zeros((3, 1, 3, 2), dtype=torch.complex64, device=cuda)
    dV = torch.zeros((3, 1, 3, 2), device=cuda)
    ws = _WS(var=x, V=V, diag_V=dV)
    op = TemporalBasisOp(U=U, param_key="V", grad_key="g_V", diag_key="diag_V")
    RegManager([Transformed(base=reg, op=op, name="tv_on_UV", params=reg.params)]).add_diag(ws)
    exp = basis_diag_push(U, torch.full((2, 1, 3, 2), k, dtype=torch.float64))
    assert torch.allclose(dV.cpu().double(), exp, atol=1e-9, rtol=0)
    assert torch.allclose(dV[:, 0, 0, 0].cpu(), torch.tensor([k, 4 * k, 0.0]), atol=1e-7, rtol=0)


def test_diag_identity_vs_mapped(cuda):
    """test_regularization_ns.py:167-193: identity TV raises the image
    diagonal everywhere; a MappedRegularizer over a TemporalBasisOp leaves it."""
    B = 4
    x = _c((B, 1, 8, 8), 6, 0.01).to(cuda)
    D = torch.zeros((B, 1, 8, 8), device=cuda)
    RegManager([TVND("tv_id", TVParams(weight=1.0, eps=1e-3, axes="spatial"))]).add_diag(_WS(var=x, diag=D))
    assert bool((D > 0).all())
    D2 = torch.zeros_like(D)
    V = _c((2, 1, 8, 8), 7, 0.01).to(cuda)
    reg = MappedRegularizer("tv_UV", TVND("tv_map", TVParams(weight=1.0, eps=1e-3, axes="spatial")),
                            TemporalBasisOp(U=torch.randn(B, 2)))
    RegManager([reg]).add_diag(_WS(var=x, diag=D2, V=V, g_V=torch.zeros_like(V)))
    assert torch.count_nonzero(D2) == 0


def test_identity_mapped_tv_in_solver_equals_plain_tv(cuda):
    """A TV term behind IdentityOp / ScaleOp (no scale) / their composition is
    fused like the bare TV term: identical solver history."""
    from mrirecon_b200 import phantoms
    from mrirecon_b200.nufft import B200NUFFTAdapter
    from mrirecon_b200.solver import CGConfig, CGSolver
    N, F, C = 32, 4, 3
    maps = phantoms.coil_maps(N, C)
    traj = phantoms.grasp_trajectory(F, 7, 64)
    ad = B200NUFFTAdapter(ndim=2)
    ad.prepare((C, N, N), traj.to(cuda), None, maps.to(cuda), torch.complex64, cuda)
    y = phantoms.add_noise(ad.A(phantoms.dynamic_phantom(N, F, seed=5).unsqueeze(1).to(cuda)), 1e-3, seed=1)
    tv = lambda: TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial"))
    cfg = lambda: CGConfig(max_iter=10, tol_g=0.0, tol_step=0.0)
    ref = CGSolver(y, ad, RegManager([tv()]), cfg()).run()
    for reg in (MappedRegularizer("m", tv(), IdentityOp()), Transformed(tv(), ScaleOp(), "t"),
                MappedRegularizer("c", tv(), ComposeOp([IdentityOp(), ScaleOp()]))):
        s = CGSolver(y, ad, RegManager([reg]), cfg()).run()
        assert [h["f"] for h in s.history()] == [h["f"] for h in ref.history()]
    with pytest.raises(TypeError):
        CGSolver(y, ad, RegManager([MappedRegularizer("p", tv(), TemporalBasisOp(U=torch.randn(F, 2)))]), cfg())
