"""Batched uneven solves (grouped launches over all instances, or one graph
branch per instance) and the plan skip flag the batch relies on."""
import ctypes

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


@pytest.mark.parametrize("grouped", [True, False])
@pytest.mark.parametrize("graph", [True, False])
def test_batched_equals_separate_solves(cuda, graph, grouped):
    """Every instance of the batch follows exactly its own solve: same iterates,
    same iteration count, bit for bit, whether the batch runs as grouped launches
    or one branch per instance, as one graph or eagerly."""
    probs = _instances(cuda, sizes=(48, 32, 80, 40), coils=(3, 2, 4, 5), spokes=(20, 9, 31, 14))
    bs = BatchedSolver(probs, _cfg(cuda_graph=graph), grouped=grouped).run()
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


def test_grouped_launches_cover_all_instances(cuda):
    """Grouped mode issues one launch per kernel step for the instances that
    share the kernel's compile-time shape: 6 instances in two size classes
    (FFT lengths 64 and 96) need far fewer launches per iteration than one
    branch per instance, and every instance ends bit for bit where its own
    solve ends."""
    probs = _instances(cuda, sizes=(32, 48, 32, 48, 32, 48), coils=(2, 3, 4, 2, 3, 4),
                       spokes=(9, 14, 11, 17, 10, 13))
    g = BatchedSolver(probs, _cfg(iters_per_graph=1), grouped=True)
    b = BatchedSolver(probs, _cfg(iters_per_graph=1), grouped=False)
    g.run()
    b.run()
    rec, launches = g.group_stats()
    assert rec > 0 and launches > 0
    assert launches * 2 <= rec, (rec, launches)
    assert g.launch_stats["per_graph"] * 2 <= b.launch_stats["per_graph"], (g.launch_stats, b.launch_stats)
    assert g.iterations() == b.iterations()
    for (y, op, regm), x_g, x_b, it in zip(probs, g.results(), b.results(), g.iterations()):
        s = CGSolver(y, op, regm, _cfg(iters_per_graph=1)).run()
        assert s.iter == it
        assert torch.equal(s.result(), x_b)
        assert torch.equal(s.result(), x_g)


def test_grouped_operator_equals_plain_calls(cuda):
    """Forward and adjoint NUFFT of three plans of one size class (each stage
    in one grouped launch: rows, columns, interp; spread, reduction, inverse
    columns and rows) equal the plain per-plan calls bit for bit."""
    from mrirecon_b200 import _lib
    lib = _lib.load()
    probs = _instances(cuda, sizes=(40, 40, 40), coils=(3, 4, 2), spokes=(15, 11, 19))
    ops = [op for _, op, _ in probs]
    g = torch.Generator(device="cpu").manual_seed(5)
    xs = [torch.randn((1, 1, 40, 40), dtype=torch.complex64, generator=g).to(cuda) for _ in ops]
    ys = [torch.randn(tuple(y.shape), dtype=torch.complex64, generator=g).to(cuda) for y, _, _ in probs]
    plain_f = [op.A(x) for op, x in zip(ops, xs)]
    plain_a = [op.AH(y) for op, y in zip(ops, ys)]
    grp_f = [torch.full_like(f, float("nan")) for f in plain_f]
    grp_a = [torch.full_like(a, float("nan")) for a in plain_a]
    assert lib.mrb_group_begin(len(ops)) == 0
    try:
        for i, op in enumerate(ops):
            assert lib.mrb_group_select(i) == 0
            op.A(xs[i], out=grp_f[i])
            op.AH(ys[i], out=grp_a[i])
    except BaseException:
        lib.mrb_group_cancel()
        raise
    _lib.check(lib.mrb_group_end(_lib.stream_ptr(cuda)), "group_end")
    rec, launches = ctypes.c_int64(0), ctypes.c_int64(0)
    _lib.check(lib.mrb_group_stats(ctypes.byref(rec), ctypes.byref(launches)), "group_stats")
    torch.cuda.synchronize()
    # plans without split tiles skip the reduction: nearly every step serves all three
    assert launches.value * 2 <= rec.value, (rec.value, launches.value)
    for a, b in zip(grp_f + grp_a, plain_f + plain_a):
        assert torch.equal(a, b)


def test_recording_rejects_kernels_without_grouped_form(cuda):
    """An entry point whose kernel has no grouped form fails inside a recording
    (its launch would otherwise run ahead of the recorded ones); the recording
    can then be cancelled and the library used as before."""
    from mrirecon_b200 import _lib
    lib = _lib.load()
    N, C = 16, 2
    maps = torch.ones((C, N, N), dtype=torch.complex64, device=cuda)
    D = torch.zeros(N * N, dtype=torch.float32, device=cuda)
    assert lib.mrb_group_begin(1) == 0
    try:
        rc = lib.mrb_precond_init(N * N, 1, C, _lib.ptr(maps), 1.0, 0.0, _lib.ptr(D), _lib.stream_ptr(cuda))
        assert rc == 5 and "grouped form" in _lib.last_error()
    finally:
        lib.mrb_group_cancel()
    torch.cuda.synchronize()
    _lib.check(lib.mrb_precond_init(N * N, 1, C, _lib.ptr(maps), 1.0, 0.0, _lib.ptr(D), _lib.stream_ptr(cuda)),
               "precond_init")
    torch.cuda.synchronize()
    assert torch.allclose(D, torch.full_like(D, 2.0))
