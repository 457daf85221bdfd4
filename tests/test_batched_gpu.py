"""Batched uneven solves (one CUDA graph, one branch per instance) and the
plan skip flag the batch relies on."""
import pytest
import torch

from conftest import rel
from mrirecon_b200 import phantoms
from mrirecon_b200.batched import BatchedSolver
from mrirecon_b200.nufft import NUFFT, NUFFTConfig
from mrirecon_b200.regularization import RegManager, TVND, TVParams
from mrirecon_b200.solver import CGConfig, CGSolver
from mrirecon_b200.workloads import axis_spec

pytestmark = pytest.mark.gpu


def _instances(dev, sizes, coils, spokes):
    out = []
    for i, (N, C, sp) in enumerate(zip(sizes, coils, spokes)):
        x = phantoms.ellipse_phantom(N, seed=50 + i).reshape(1, 1, N, N).to(dev)
        maps = phantoms.coil_maps(N, C).to(dev)
        traj = phantoms.golden_angle_radial(sp, 2 * N).unsqueeze(0).to(dev)
        op = NUFFT(maps, traj, None, axis=axis_spec(), config=NUFFTConfig(ndim=2, traj_units="rad"), device=dev)
        y = op.A(x)
        regm = RegManager([TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial"))])
        out.append((y, op, regm))
    return out


def _cfg(**kw):
    d = dict(max_iter=300, stop_window=10, stop_tol=1e-4, cuda_graph=True, iters_per_graph=8)
    d.update(kw)
    return CGConfig(**d)


@pytest.mark.parametrize("graph", [True, False])
def test_batched_equals_separate_solves(cuda, graph):
    """Every instance of the batch follows exactly its own solve: same iterates,
    same iteration count, bit for bit, whether the batch runs as one graph or eagerly."""
    probs = _instances(cuda, sizes=(48, 32, 80, 40), coils=(3, 2, 4, 5), spokes=(20, 9, 31, 14))
    bs = BatchedSolver(probs, _cfg(cuda_graph=graph)).run()
    its = bs.iterations()
    assert len(set(its)) > 1, "instances should stop at different iterations"
    for (y, op, regm), x_b, it in zip(probs, bs.results(), its):
        s = CGSolver(y, op, regm, _cfg()).run()
        assert s.iter == it
        assert torch.equal(s.result(), x_b)
    # a second run from the reset state repeats the first
    first = [x.clone() for x in bs.results()]
    bs.reset().run()
    assert bs.iterations() == its
    assert all(torch.equal(a, b) for a, b in zip(first, bs.results()))
    if graph:
        assert bs.launch_stats["replays"] > 0


def test_skip_flag_leaves_outputs(cuda):
    """A set skip flag makes the operator kernels return without writing."""
    probs = _instances(cuda, sizes=(32,), coils=(2,), spokes=(12,))
    y, op, _ = probs[0]
    plan = op.backend.plan
    flag = torch.ones(1, dtype=torch.float64, device=cuda)
    x = torch.randn((1, 1, 32, 32), dtype=torch.complex64, device=cuda)
    out = torch.full_like(y, 7.0)
    plan.set_skip_flag(flag.data_ptr())
    op.A(x, out=out)
    xa = torch.full_like(x, 3.0)
    op.AH(y, out=xa)
    torch.cuda.synchronize()
    assert bool((out == 7.0).all()) and bool((xa == 3.0).all())
    flag.zero_()
    op.A(x, out=out)
    ref = torch.empty_like(out)
    plan.set_skip_flag(None)
    op.A(x, out=ref)
    assert rel(out, ref) == 0.0


def test_batched_graph_and_jacobi_equal_separate_solves(cuda):
    """Multi-frame instances with a spatial TV and a frame-chain graph Laplacian,
    solved with the Jacobi diagonal: the batch (one graph, a branch per instance)
    follows each instance's own solve bit for bit."""
    from mrirecon_b200.regularization import GraphLaplacian, GraphLapParams
    probs = []
    for i, (N, F, C, spf) in enumerate(((32, 4, 3, 7), (48, 6, 2, 9), (40, 5, 4, 5))):
        maps = phantoms.coil_maps(N, C).to(cuda)
        traj = phantoms.grasp_trajectory(F, spf, 2 * N).to(cuda)
        op = NUFFT(maps, traj, None, axis=axis_spec(), config=NUFFTConfig(ndim=2, traj_units="rad"), device=cuda)
        y = op.A(phantoms.dynamic_phantom(N, F, seed=60 + i).unsqueeze(1).to(cuda))
        W = torch.zeros(F, F)
        for t in range(F - 1):
            W[t, t + 1] = W[t + 1, t] = 1.0
        regm = RegManager([TVND("s", TVParams(weight=1e-3, eps=1e-3, axes="spatial")),
                           GraphLaplacian("g", W, GraphLapParams(weight=5e-3, normalize="none"))])
        probs.append((y, op, regm))
    bs = BatchedSolver(probs, _cfg(precond="jacobi", max_iter=120)).run()
    for (y, op, regm), x_b, it in zip(probs, bs.results(), bs.iterations()):
        s = CGSolver(y, op, regm, _cfg(precond="jacobi", max_iter=120)).run()
        assert s.iter == it
        assert torch.equal(s.result(), x_b)
