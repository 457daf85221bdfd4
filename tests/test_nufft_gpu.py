"""NUFFT parity on the GPU: CUDA path (through the C ABI) vs the CPU oracle.

Tolerances: bin/cell indices bit-exact; forward/adjoint rel-L2 <= 1e-5 against
the oracle's FP64 KB gridding with the same conventions (the stated target);
KB approximation error vs the FP64 NUDFT <= 2e-3 (W=4, osf=2 gives ~6e-4).
"""
import math

import numpy as np
import pytest
import torch

from conftest import golden, rel
from oracle import kb as okb
from oracle.nudft import nudft_forward, nudft_adjoint
from mrirecon_b200 import phantoms
from mrirecon_b200.nufft import B200NUFFTAdapter, grid_indices, NUFFT, NUFFTConfig
from mrirecon_b200.layout import AxisSpec

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _rand_c(shape, seed, dtype=torch.complex128):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, generator=g, dtype=torch.float64)
            + 1j * torch.randn(shape, generator=g, dtype=torch.float64)).to(dtype)


def _adapter(maps, traj, dcf=None, dev="cuda", **kw):
    ad = B200NUFFTAdapter(ndim=maps.ndim - 1, **kw)
    ad.prepare(tuple(maps.shape), traj.to(dev), None if dcf is None else dcf.to(dev),
               maps.to(dev, torch.complex64), torch.complex64, torch.device(dev))
    return ad


@pytest.mark.parametrize("case", ["2d_32", "2d_24x40", "3d_12x10x8"])
def test_reference_grid_indices_bit_exact(cuda, case):
    g = golden("ptnufft_idx.npz")
    traj, G, idx = g[f"{case}_traj"], tuple(int(v) for v in g[f"{case}_grid"]), g[f"{case}_idx"]
    for b in range(traj.shape[0]):
        mine = grid_indices(torch.from_numpy(traj[b]).to(cuda), G, 4, "reference").cpu().numpy()
        assert np.array_equal(mine, idx[b].astype(np.int64))


@pytest.mark.parametrize("S,K", [((32, 32), 1500), ((24, 40), 1500), ((12, 10, 8), 500)])
def test_corrected_indices_and_cell_base_bit_exact(cuda, S, K):
    g = golden("ptnufft_idx.npz")
    key = {2: "2d_32", 3: "3d_12x10x8"}[len(S)]
    traj = torch.from_numpy(g[f"{key}_traj"])[:, :, :K]
    G = okb.grid_shape(S, 2.0)
    # stand-alone table
    for b in range(traj.shape[0]):
        mine = grid_indices(traj[b].to(cuda), G, 4, "corrected").cpu().numpy()
        o = okb.KBNufft(torch.ones((1,) + S, dtype=torch.complex128), traj[b:b + 1], None)
        assert np.array_equal(mine, o.idx[0].numpy())
    # the plan's binning key
    ad = _adapter(torch.ones((1,) + S, dtype=torch.complex64), traj)
    base = ad.plan.cell_base().cpu().numpy()
    for b in range(traj.shape[0]):
        assert np.array_equal(base[b], okb.cell_base(traj[b].numpy(), G).astype(np.int32))


def _check_pair(maps, traj, dcf=None, nb=None, seed=1, **kw):
    dev = "cuda"
    B, nd, K = traj.shape
    nb = nb or B
    S = tuple(maps.shape[1:])
    C = maps.shape[0]
    ad = _adapter(maps, traj, dcf, **kw)
    orc = okb.KBNufft(maps.to(torch.complex128), traj, dcf, dtype=torch.complex128,
                      dcf_mode=kw.get("dcf_mode", "balanced"), apply_dcf_in_fwd=kw.get("apply_dcf_in_fwd", False),
                      apply_dcf_in_adj=kw.get("apply_dcf_in_adj", True), norm=kw.get("norm", "ortho"))
    x = _rand_c((nb, 1) + S, seed)
    y = _rand_c((nb, C, K), seed + 1)
    yg = ad.A(x.to(dev, torch.complex64))
    xg = ad.AH(y.to(dev, torch.complex64))
    ya, xa = orc.A(x), orc.AH(y)
    assert rel(yg, ya) < TOL, f"forward rel {rel(yg, ya):.3e}"
    assert rel(xg, xa) < TOL, f"adjoint rel {rel(xg, xa):.3e}"
    if kw.get("dcf_mode", "balanced") != "standard":      # standard DCF is one-sided: not an adjoint pair
        lhs = torch.vdot(yg.cpu().to(torch.complex128).reshape(-1), y.reshape(-1))
        rhs = torch.vdot(x.reshape(-1), xg.cpu().to(torch.complex128).reshape(-1))
        assert abs(complex(lhs / rhs) - 1) < 1e-5
    return ad


@pytest.mark.parametrize("S", [(32, 32), (24, 40), (31, 33), (64, 48), (33, 35), (17, 9)])
def test_forward_adjoint_vs_oracle_2d(cuda, S):
    C = 3
    maps = _rand_c((C,) + S, 5, torch.complex64)
    traj = phantoms.random_traj(2, 2, 1200, seed=3)
    _check_pair(maps, traj)


def test_radial_edges_and_wrap(cuda):
    """Golden-angle spokes hit k = -pi exactly (wraps to the far grid edge)."""
    maps = phantoms.coil_maps(48, 4).to(torch.complex64)
    traj = torch.stack([phantoms.golden_angle_radial(9, 96, 9 * f) for f in range(3)])
    _check_pair(maps, traj)


@pytest.mark.parametrize("mode,fwd,adj", [("balanced", False, True), ("standard", True, False),
                                          ("standard", False, True), ("none", False, True)])
def test_dcf_modes(cuda, mode, fwd, adj):
    maps = _rand_c((2, 20, 20), 8, torch.complex64)
    traj = phantoms.random_traj(2, 2, 500, seed=9)
    dcf = torch.rand(2, 500, generator=torch.Generator().manual_seed(2)) + 0.1
    _check_pair(maps, traj, dcf, dcf_mode=mode, apply_dcf_in_fwd=fwd, apply_dcf_in_adj=adj)


@pytest.mark.parametrize("chunk", [None, 16])
def test_beff_repeat_interleave(cuda, chunk):
    """B_eff = 2*B uses trajectory frame be // 2 (torchkb _expand_omega)."""
    maps = _rand_c((2, 16, 16), 4, torch.complex64)
    traj = phantoms.random_traj(2, 2, 400, seed=4)
    _check_pair(maps, traj, nb=4, chunk=chunk)


def test_single_frame_expanded(cuda):
    """B = 1 trajectory applied to B_eff = 3 images (the expand branch)."""
    maps = _rand_c((2, 20, 20), 14, torch.complex64)
    traj = phantoms.golden_angle_radial(24, 40).unsqueeze(0)
    _check_pair(maps, traj, nb=3, chunk=16)


def test_unnormalised(cuda):
    maps = _rand_c((2, 16, 18), 6, torch.complex64)
    traj = phantoms.random_traj(1, 2, 400, seed=6)
    _check_pair(maps, traj, norm="none")


@pytest.mark.parametrize("tile,cpi,chunk", [(8, 1, None), (16, 2, 16), (32, 3, 64), (4, 4, None), (16, 4, 100000)])
def test_tiling_options_identical(cuda, tile, cpi, chunk):
    """Every tile / coil-group / chunk choice gives the same grid (up to the
    summation order of split tiles), deterministically."""
    maps = phantoms.coil_maps(64, 5).to(torch.complex64)
    traj = phantoms.grasp_trajectory(2, 13, 128)
    y = _rand_c((2, 5, traj.shape[-1]), 3, torch.complex64).to(cuda)
    ref = _adapter(maps, traj).AH(y)
    ad = _adapter(maps, traj, tile=tile, coils_per_item=cpi, chunk=chunk)
    out = ad.AH(y)
    assert rel(out, ref) < 1e-6
    out2 = ad.AH(y)
    assert torch.equal(out, out2)


@pytest.mark.parametrize("chunk", [None, 16])
def test_3d_vs_oracle(cuda, chunk):
    S = (12, 10, 8)
    maps = _rand_c((2,) + S, 12, torch.complex64)
    traj = phantoms.random_traj(2, 3, 700, seed=13)
    _check_pair(maps, traj, chunk=chunk)


def test_3d_radial_koosh(cuda):
    """Golden-means koosh-ball spokes: every spoke crosses the centre tile, which
    is split into many chunks."""
    S = (24, 24, 24)
    maps = phantoms.coil_maps(24, 3, ndim=3).to(torch.complex64)
    traj = phantoms.golden_means_koosh(300, 48).unsqueeze(0)
    _check_pair(maps, traj, chunk=32)


def test_vs_nudft_fixture(cuda):
    """KB approximation error against the reference's _nudft_A ground truth."""
    g = golden("nudft_a.npz")
    maps, x = torch.from_numpy(g["maps"]), torch.from_numpy(g["x"])
    traj, dcf = torch.from_numpy(g["traj"]), torch.from_numpy(g["dcf"])
    ad = _adapter(maps.to(torch.complex64), traj.unsqueeze(0), dcf.unsqueeze(0), norm="none")
    y = ad.A(x.to(cuda, torch.complex64))
    assert rel(y, torch.from_numpy(g["y"])) < 2e-3
    yy = _rand_c(tuple(y.shape), 3)
    xa = ad.AH(yy.to(cuda, torch.complex64))
    xt = nudft_adjoint(maps, yy, traj, dcf)
    assert rel(xa, xt) < 2e-3


def test_front_end_layouts(cuda):
    """User layout (B, L, coil, X, Y) / (B, L, coil, K) through the NUFFT front-end."""
    B, L, C, S, K = 2, 2, 3, (20, 24), 300
    maps = _rand_c((C,) + S, 21, torch.complex64)
    traj = phantoms.random_traj(B, 2, K, seed=22)
    axis = AxisSpec(image_labels=("B", "L", "coil", "X", "Y"), kspace_labels=("B", "L", "coil", "K"),
                    image_fft_labels=("X", "Y"), coil_label="coil")
    op = NUFFT(maps.to(cuda), traj.to(cuda), None, axis=axis,
               config=NUFFTConfig(ndim=2, traj_units="rad"), device=cuda)
    assert op.roles_image.resolve_axes("spatial") == (3, 4)
    x = _rand_c((B, L, 1) + S, 23, torch.complex64).to(cuda)
    y = torch.empty((B, L, C, K), dtype=torch.complex64, device=cuda)
    op.A(x, out=y)
    orc = okb.KBNufft(maps, traj, None, dtype=torch.complex128)
    ya = orc.A(x.cpu().reshape(B * L, 1, *S)).reshape(B, L, C, K)
    assert rel(y, ya) < TOL
    xh = torch.empty_like(x)
    op.AH(y, out=xh)
    xa = orc.AH(y.cpu().reshape(B * L, C, K).to(torch.complex128)).reshape(B, L, 1, *S)
    assert rel(xh, xa) < TOL
    # permuted user layout (coil first in k-space)
    axis2 = AxisSpec(image=("B", "X", "Y"), kspace=("coil", "B", "K"), image_fft=("X", "Y"), coil="coil")
    op2 = NUFFT(maps.to(cuda), traj.to(cuda), None, axis=axis2, config=NUFFTConfig(ndim=2, traj_units="rad"))
    x2 = x[:, 0, 0]
    y2 = op2.A(x2)
    assert tuple(y2.shape) == (C, B, K)
    assert rel(y2.permute(1, 0, 2), orc.A(x2.cpu().unsqueeze(1))) < TOL


def test_errors_are_raised(cuda):
    maps = _rand_c((2, 16, 16), 1, torch.complex64)
    traj = phantoms.random_traj(2, 2, 100, seed=1)
    ad = _adapter(maps, traj)
    with pytest.raises(ValueError):
        ad.A(torch.zeros((3, 1, 16, 16), dtype=torch.complex64, device=cuda))   # B mismatch
    with pytest.raises(ValueError):
        ad.AH(torch.zeros((2, 3, 100), dtype=torch.complex64, device=cuda))      # coil mismatch
    with pytest.raises(ValueError):
        ad.A(torch.zeros((2, 1, 16, 16), dtype=torch.complex64, device=cuda),
             out=torch.zeros((2, 2, 99), dtype=torch.complex64, device=cuda))
    with pytest.raises(RuntimeError):
        ad.A(torch.zeros((2, 1, 16, 16), dtype=torch.complex64))                 # CPU tensor


def test_coil_images_forward(cuda):
    """Cin == C: per-coil images, maps not applied (torchkb.py:244-247)."""
    C, S = 3, (16, 20)
    maps = _rand_c((C,) + S, 31, torch.complex64)
    traj = phantoms.random_traj(1, 2, 300, seed=32)
    ad = _adapter(maps, traj)
    xc = _rand_c((1, C) + S, 33)
    y = ad.A(xc.to(cuda, torch.complex64))
    orc = okb.KBNufft(torch.ones((1,) + S, dtype=torch.complex128), traj, None)
    ya = torch.cat([orc.A(xc[:, c:c + 1]) for c in range(C)], dim=1)
    assert rel(y, ya) < TOL


def test_autotuner_picks_a_timed_candidate(cuda, tmp_path, monkeypatch):
    """The autotuner times the spread candidates on the plan's trajectory, keeps
    the fastest, caches it per size class, and the tuned plan still matches the oracle."""
    monkeypatch.setenv("MRB_TUNE_CACHE", str(tmp_path / "tune.json"))
    maps = phantoms.coil_maps(48, 4).to(torch.complex64)
    traj = phantoms.grasp_trajectory(3, 9, 96)
    ad = _check_pair(maps, traj, autotune=True)
    assert ad.tuned is not None and not ad.tuned.get("cached")
    best = ad.tuned
    assert best["ms"] == min(t["ms"] for t in best["tried"])
    info = ad.plan.info()
    assert (info["tile"], info["coils_per_item"]) == (best["tile"], best["cpi"])
    ad2 = _check_pair(maps, traj, autotune=True)
    assert ad2.tuned.get("cached") and ad2.tuned["tile"] == best["tile"]


@pytest.mark.parametrize("S,C,nb", [((128, 128), 12, 3), ((96, 80), 4, 2), ((160, 192), 3, 2), ((20, 20), 5, 2)])
def test_fused_fft_matches_cufft(cuda, S, C, nb):
    """The fused zero-pruned row/column FFT passes (default for 2D grids with
    compiled lengths, radices 8/4/2/3/5) agree with the dense cuFFT path."""
    maps = _rand_c((C,) + S, 41, torch.complex64)
    traj = phantoms.random_traj(nb, 2, 900, seed=42)
    fused = _adapter(maps, traj)
    dense = _adapter(maps, traj, fft_mode=0)
    assert fused.plan.info()["fft_mode"] == 1 and dense.plan.info()["fft_mode"] == 0
    x = _rand_c((nb, 1) + S, 43, torch.complex64).to(cuda)
    y = _rand_c((nb, C, 900), 44, torch.complex64).to(cuda)
    assert rel(fused.A(x), dense.A(x)) < 2e-6
    assert rel(fused.AH(y), dense.AH(y)) < 2e-6
    xc = _rand_c((nb, C) + S, 45, torch.complex64).to(cuda)
    yf = torch.empty_like(y)
    yd = torch.empty_like(y)
    _lib_forward_coils(fused, xc, yf, nb)
    _lib_forward_coils(dense, xc, yd, nb)
    assert rel(yf, yd) < 2e-6


def _lib_forward_coils(ad, xc, y, nb):
    from mrirecon_b200 import _lib
    _lib.check(_lib.load().mrb_nufft_forward_coils(ad.plan.h, _lib.ptr(xc), _lib.ptr(y), nb,
                                                   _lib.stream_ptr(xc.device)), "forward_coils")


def test_fft_mode_selection(cuda):
    """Fused FFT by default where kernels exist; cuFFT for other 2D sizes and 3D;
    asking for the fused mode where it does not exist is an error."""
    traj2 = phantoms.random_traj(1, 2, 100, seed=1)
    assert _adapter(_rand_c((2, 32, 40), 1, torch.complex64), traj2).plan.info()["fft_mode"] == 1
    assert _adapter(_rand_c((2, 31, 33), 1, torch.complex64), traj2).plan.info()["fft_mode"] == 0
    traj3 = phantoms.random_traj(1, 3, 100, seed=1)
    ad3 = _adapter(_rand_c((2, 8, 8, 8), 1, torch.complex64), traj3)
    assert ad3.plan.info()["fft_mode"] == 0
    with pytest.raises(RuntimeError):
        _adapter(_rand_c((2, 8, 8, 8), 1, torch.complex64), traj3, fft_mode=1)
    with pytest.raises(RuntimeError):
        _adapter(_rand_c((2, 31, 33), 1, torch.complex64), traj2, fft_mode=1)


@pytest.mark.parametrize("C,nb", [(4, 2), (3, 2), (2, 1)])
def test_3d_interleaved_interp_identical(cuda, C, nb):
    """The 3D forward interp on the coil-interleaved grid copy (128-bit gathers
    for even C, 64-bit for odd C) sums in the planar kernel's order: the
    samples are bit-identical."""
    S = (16, 12, 10)
    maps = _rand_c((C,) + S, 21, torch.complex64)
    traj = phantoms.random_traj(2 if nb == 2 else 1, 3, 900, seed=17)
    x = _rand_c((nb, 1) + S, 5, torch.complex64).to(cuda)
    y1 = _adapter(maps, traj, interleave=1).A(x)
    y0 = _adapter(maps, traj, interleave=0).A(x)
    assert torch.equal(y0, y1)
    # acquisition visiting order instead of the Morton segment order
    ad = _adapter(maps, traj, interleave=1)
    ad.plan.set_option(2, 0)
    assert torch.equal(ad.A(x), y1)


@pytest.mark.parametrize("C,chunk", [(20, None), (5, 16), (1, 64)])
def test_3d_block_spread_vs_oracle(cuda, C, chunk):
    """The block-per-tile 3D spread (tile 8) with two coil groups (C = 20:
    16 + 4), an odd coil count and a single coil, with and without split tiles."""
    S = (12, 10, 8)
    maps = _rand_c((C,) + S, 31, torch.complex64)
    traj = phantoms.random_traj(2, 3, 700, seed=19)
    _check_pair(maps, traj, chunk=chunk)


def test_3d_block_spread_matches_warp_kernel(cuda):
    """Tile 8 (block kernel) and tile 4 (per-warp kernel) give the same grid up
    to the summation order of split tiles; the block kernel is deterministic."""
    S = (24, 24, 24)
    maps = phantoms.coil_maps(24, 6, ndim=3).to(torch.complex64)
    traj = phantoms.golden_means_koosh(200, 48).unsqueeze(0)
    y = _rand_c((1, 6, traj.shape[-1]), 3, torch.complex64).to(cuda)
    ref = _adapter(maps, traj, tile=4, coils_per_item=2).AH(y)
    ad = _adapter(maps, traj, tile=8, chunk=100000)
    out = ad.AH(y)
    assert rel(out, ref) < 1e-6
    assert torch.equal(out, ad.AH(y))


@pytest.mark.parametrize("C,cpi,chunk,nb", [(16, 16, None, 1), (16, 16, 64, 2), (12, 16, None, 2), (20, 16, 128, 1),
                                            (5, 8, None, 1), (8, 8, 32, 2), (16, 8, None, 1)])
def test_3d_shared_staging_spread_identical(cuda, C, cpi, chunk, nb):
    """The 3D spread with shared staging and tap tables (option key 6 = 2; one
    block of 16 warps serves two coil groups of 8 when the coils per item exceed
    8, swapped pair slots on odd cells) gives the block kernel's grid bit for bit:
    partial second groups, split tiles, several coil groups per tile."""
    S = (16, 12, 20)
    maps = _rand_c((C,) + S, 41, torch.complex64)
    traj = phantoms.golden_means_koosh(120, 32).unsqueeze(0)
    y = _rand_c((nb, C, traj.shape[-1]), 42, torch.complex64).to(cuda)
    ad = _adapter(maps, traj, tile=8, chunk=chunk, coils_per_item=cpi)
    ad.plan.set_option(6, 1)
    x1 = ad.AH(y)
    ad.plan.set_option(6, 2)
    assert ad.plan.info()["block_spread"] == 1
    assert torch.equal(ad.AH(y), x1)


@pytest.mark.parametrize("C,chunk,nb", [(12, None, 2), (12, 16, 2), (3, 32, 1), (7, None, 2), (20, 64, 2)])
def test_2d_block_spread_identical_to_warp_kernel(cuda, C, chunk, nb):
    """The block-per-tile 2D spread (tile 16: 2, 4 or 8 coil pairs per lane
    group, two coil groups at C = 20) sums every (cell, coil) in the per-warp
    kernel's order: same grid bit for bit, split tiles included."""
    maps = _rand_c((C, 40, 36), 51, torch.complex64)
    traj = phantoms.grasp_trajectory(nb, 11, 96)
    y = _rand_c((nb, C, traj.shape[-1]), 52, torch.complex64).to(cuda)
    blk = _adapter(maps, traj, tile=16, chunk=chunk, spread_kernel=1, coils_per_item=16)
    warp = _adapter(maps, traj, tile=16, chunk=chunk, spread_kernel=0)
    assert blk.plan.info()["block_spread"] == 1 and warp.plan.info()["block_spread"] == 0
    assert torch.equal(blk.AH(y), warp.AH(y))


@pytest.mark.parametrize("S,C,nb,B", [((64, 64), 5, 2, 2), ((48, 40), 3, 4, 2), ((40, 40), 4, 3, 1)])
def test_grid_mask_identical(cuda, S, C, nb, B):
    """Fused FFT mode: restricting the column passes and the spread write-out to
    the touched cells (per-frame bitmaps, frame = be // (nb // B)) gives the same
    forward and adjoint results bit for bit, including after the unmasked
    passes have left other values in the grid."""
    maps = _rand_c((C,) + S, 61, torch.complex64)
    traj = phantoms.grasp_trajectory(B, 7, 2 * S[0])
    K = traj.shape[-1]
    x = _rand_c((nb, 1) + S, 62, torch.complex64).to(cuda)
    y = _rand_c((nb, C, K), 63, torch.complex64).to(cuda)
    ad = _adapter(maps, traj)
    assert ad.plan.info()["fft_mode"] == 1
    ad.plan.set_option(7, 0)
    ya, xa = ad.A(x), ad.AH(y)
    ad.plan.set_option(7, 1)
    assert torch.equal(ad.A(x), ya) and torch.equal(ad.AH(y), xa)
    ad.plan.set_option(7, 0)
    assert torch.equal(ad.A(x), ya) and torch.equal(ad.AH(y), xa)
    if B > 1 and nb > B:
        # a smaller batch maps the grid slots to other trajectory frames
        ad.plan.set_option(7, 0)
        xb = ad.AH(y[:B])
        ad.plan.set_option(7, 1)
        ad.AH(y)
        assert torch.equal(ad.AH(y[:B]), xb)


@pytest.mark.parametrize("C,nb,B", [(12, 2, 2), (5, 4, 2), (1, 1, 1), (3, 3, 1)])
def test_2d_pair_parallel_interp_identical(cuda, C, nb, B):
    """2D interp with one thread per (sample, coil pair) (mode 1, the default) sums
    in the per-sample kernel's order: identical samples, odd coil counts included."""
    maps = _rand_c((C, 40, 48), 71, torch.complex64)
    traj = phantoms.random_traj(B, 2, 1000, seed=72)
    x = _rand_c((nb, 1, 40, 48), 73, torch.complex64).to(cuda)
    for fft_mode in (1, 0):
        ad = _adapter(maps, traj, fft_mode=fft_mode)
        y1 = ad.A(x)
        ad.plan.set_option(2, 0)
        assert torch.equal(ad.A(x), y1)


@pytest.mark.parametrize("S,C,nb,B", [((40, 48), 12, 2, 2), ((40, 48), 5, 3, 1), ((320, 160), 3, 1, 1),
                                      ((48, 40), 1, 4, 2), ((384, 40), 2, 2, 2)])
def test_2d_blocked_grid_identical(cuda, S, C, nb, B):
    """Fused 2D mode: the forward column pass storing each coil-frame's grid in
    2 x 8 cell blocks (option key 9 = 1, the default) and the pair-parallel
    interp reading it give the samples of the row-major grid bit for bit
    (grid sides 80 ... 768; column blocks of 16, 12 and 10 columns, the last
    two starting off an 8-column boundary)."""
    maps = _rand_c((C,) + S, 77, torch.complex64)
    traj = phantoms.random_traj(B, 2, 1000, seed=78)
    x = _rand_c((nb, 1) + S, 79, torch.complex64).to(cuda)
    ad = _adapter(maps, traj)
    assert ad.plan.info()["fft_mode"] == 1
    y1 = ad.A(x)
    ad.plan.set_option(9, 0)
    y0 = ad.A(x)
    assert torch.equal(y0, y1)
    ad.plan.set_option(9, 1)
    assert torch.equal(ad.A(x), y1)
    assert torch.equal(ad.AH(y1), ad.AH(y0))


@pytest.mark.parametrize("fft_mode,C,nb,B", [(1, 12, 2, 2), (1, 3, 3, 1), (0, 4, 2, 2), (1, 1, 1, 1)])
def test_2d_tap_table_identical(cuda, fft_mode, C, nb, B):
    """2D spread and interp reading the per-sample tap table built by set_points
    (option key 10 = 1, the default) give the grids and samples of the inline
    kernel evaluation bit for bit, with and without adjoint density weights."""
    maps = _rand_c((C, 40, 48), 80, torch.complex64)
    traj = phantoms.random_traj(B, 2, 1000, seed=81)
    dcf = torch.rand(B, 1000, generator=torch.Generator().manual_seed(82)) + 0.5
    x = _rand_c((nb, 1, 40, 48), 83, torch.complex64).to(cuda)
    for w in (None, dcf):
        ad = _adapter(maps, traj, dcf=w, fft_mode=fft_mode)
        y1 = ad.A(x)
        x1 = ad.AH(y1)
        ad.plan.set_option(10, 0)
        assert torch.equal(ad.A(x), y1)
        assert torch.equal(ad.AH(y1), x1)
        ad.plan.set_option(10, 1)
        assert torch.equal(ad.A(x), y1)


@pytest.mark.parametrize("S,C,nb,B", [((40, 48), 12, 2, 2), ((40, 48), 8, 3, 1), ((32, 32), 16, 1, 1),
                                      ((48, 40), 4, 4, 2), ((320, 160), 4, 1, 1), ((40, 48), 5, 2, 1)])
def test_2d_interleaved_grid_interp_identical(cuda, S, C, nb, B):
    """Fused 2D mode: the forward column pass writing the grid in coil quads
    (column groups with a tail at G0 = 640) and the interleaved interp (option
    key 5 = 1 with coil counts divisible by 4; C = 5 stays planar) give
    the samples of the planar column pass and pair-parallel interp bit for bit."""
    maps = _rand_c((C,) + S, 74, torch.complex64)
    traj = phantoms.random_traj(B, 2, 1000, seed=75)
    x = _rand_c((nb, 1) + S, 76, torch.complex64).to(cuda)
    ad = _adapter(maps, traj)
    assert ad.plan.info()["fft_mode"] == 1
    ad.plan.set_option(5, 1)
    y1 = ad.A(x)
    ad.plan.set_option(5, 0)
    assert torch.equal(ad.A(x), y1)
    ad.plan.set_option(5, 1)
    assert torch.equal(ad.A(x), y1)


@pytest.mark.parametrize("tile,cpi,chunk,fft_mode,mask", [(16, 6, None, 1, 1), (16, 12, 16, 1, 1), (8, 4, None, 1, 0),
                                                          (4, 3, 32, 1, 1), (32, 2, None, 1, 1), (16, 5, 64, 0, 1),
                                                          (16, 16, None, 1, 1)])
def test_2d_tap_table_spread_identical_to_earlier_kernel(cuda, tile, cpi, chunk, fft_mode, mask):
    """The per-warp 2D spread that tabulates each staged sample's inside taps
    (option key 6 = 2) gives the grid of the kernel that evaluates every tap per
    lane task (key 6 = 0) bit for bit: tiles 4 .. 32, odd coil groups, split
    tiles, the masked write-out and the dense FFT mode."""
    C = 12
    maps = _rand_c((C, 48, 40), 53, torch.complex64)
    traj = phantoms.grasp_trajectory(2, 11, 96)
    y = _rand_c((2, C, traj.shape[-1]), 54, torch.complex64).to(cuda)
    ad = _adapter(maps, traj, tile=tile, chunk=chunk, coils_per_item=cpi, fft_mode=fft_mode)
    ad.plan.set_option(7, mask)
    ad.plan.set_option(6, 0)
    x0 = ad.AH(y)
    ad.plan.set_option(6, 2)
    assert torch.equal(ad.AH(y), x0)
    ad.plan.set_option(6, 0)
    assert torch.equal(ad.AH(y), x0)


@pytest.mark.parametrize("S,C,nb,B", [((16, 20, 24), 3, 2, 1), ((24, 16, 32), 4, 2, 2), ((20, 20, 20), 1, 1, 1),
                                      ((16, 20, 24), 16, 2, 2), ((20, 16, 24), 8, 1, 1)])
def test_fused_fft_3d_matches_cufft(cuda, S, C, nb, B):
    """3D zero-pruned passes (z rows fused with SENSE/deapodisation, then y and x
    columns, and the reverse with crop and coil sum; the default where every
    grid side has compiled kernels) agree with the dense cuFFT path, forward
    from images and from coil images, and adjoint."""
    maps = _rand_c((C,) + S, 81, torch.complex64)
    traj = phantoms.random_traj(B, 3, 700, seed=82)
    fused = _adapter(maps, traj)
    dense = _adapter(maps, traj, fft_mode=0)
    assert fused.plan.info()["fft_mode"] == 1 and dense.plan.info()["fft_mode"] == 0
    x = _rand_c((nb, 1) + S, 83, torch.complex64).to(cuda)
    y = _rand_c((nb, C, 700), 84, torch.complex64).to(cuda)
    assert rel(fused.A(x), dense.A(x)) < 2e-6
    assert rel(fused.AH(y), dense.AH(y)) < 2e-6
    xc = _rand_c((nb, C) + S, 85, torch.complex64).to(cuda)
    yf = torch.empty_like(y)
    yd = torch.empty_like(y)
    _lib_forward_coils(fused, xc, yf, nb)
    _lib_forward_coils(dense, xc, yd, nb)
    assert rel(yf, yd) < 2e-6
    # with 8 / 16 / 32 coils the x pass writes the interp's (cell, coil) copy
    # itself; the planar interp reads the same values in the same order
    planar = _adapter(maps, traj, interleave=0)
    assert torch.equal(fused.A(x), planar.A(x))


@pytest.mark.parametrize("S,C,nb,B,dcf", [((256, 256), 4, 2, 2, False), ((40, 48), 3, 4, 2, True),
                                          ((64, 48), 1, 1, 1, False), ((24, 40), 5, 3, 1, True)])
def test_fused_column_interp_identical(cuda, S, C, nb, B, dcf):
    """2D fused mode: the forward column pass that interpolates each column
    strip's samples from shared memory (option key 8) gives the
    same samples bit for bit as the column pass that writes the grid followed
    by the interp kernel, including strips that wrap at the grid edge, the
    frame mapping of a repeated trajectory and forward DCF weights."""
    maps = _rand_c((C,) + S, 91, torch.complex64)
    traj = torch.stack([phantoms.golden_angle_radial(9, 2 * S[0], 9 * f) for f in range(B)])
    w = torch.rand(B, traj.shape[-1], generator=torch.Generator().manual_seed(92)) + 0.1 if dcf else None
    kw = dict(dcf_mode="standard", apply_dcf_in_fwd=True, apply_dcf_in_adj=False) if dcf else {}
    on = _adapter(maps, traj, w, col_interp=1, **kw)
    off = _adapter(maps, traj, w, **kw)
    assert on.plan.info()["col_interp"] == 1 and off.plan.info()["col_interp"] == 0
    x = _rand_c((nb, 1) + S, 93, torch.complex64).to(cuda)
    assert torch.equal(on.A(x), off.A(x))
    xc = _rand_c((nb, C) + S, 94, torch.complex64).to(cuda)
    y1 = torch.empty((nb, C, traj.shape[-1]), dtype=torch.complex64, device=cuda)
    y0 = torch.empty_like(y1)
    _lib_forward_coils(on, xc, y1, nb)
    _lib_forward_coils(off, xc, y0, nb)
    assert torch.equal(y1, y0)


def test_plan_memory_reuse_and_release(cuda):
    """Plans built one after another reuse the device blocks of destroyed plans
    (a block cache instead of cudaMalloc / cudaFree per plan); results stay
    identical, and mrb_release_cached_memory hands the cache back."""
    import gc
    from mrirecon_b200 import _lib
    maps = phantoms.coil_maps(64, 4).to(torch.complex64)
    traj = phantoms.grasp_trajectory(3, 9, 128)
    x = _rand_c((3, 1, 64, 64), 101, torch.complex64).to(cuda)
    y = _rand_c((3, 4, traj.shape[-1]), 102, torch.complex64).to(cuda)
    outs = []
    for rnd in range(3):
        ad = _adapter(maps, traj)
        outs.append((ad.A(x), ad.AH(y)))
        del ad
        gc.collect()
        if rnd == 1:
            assert _lib.load().mrb_release_cached_memory() == 0
    for ya, xa in outs[1:]:
        assert torch.equal(ya, outs[0][0]) and torch.equal(xa, outs[0][1])


@pytest.mark.parametrize("S,B,spokes", [((32, 32), 2, 24), ((20, 24), 1, 16), ((12, 10, 8), 1, 0)])
def test_estimate_dcf_vs_oracle(cuda, S, B, spokes):
    """Density compensation by the Pipe-Menon iteration on the GPU gridding
    (spread then interp on the plan's grid, no FFT) against the FP64 CPU
    restatement: relative L2 <= 1e-4 after 20 iterations (FP32 grid sums)."""
    from mrirecon_b200.dcf import estimate_dcf
    from oracle.dcf import pipe_menon
    if len(S) == 2:
        traj = torch.stack([phantoms.golden_angle_radial(spokes, 2 * max(S), spokes * f) for f in range(B)])
    else:
        traj = phantoms.random_traj(B, 3, 600, seed=111)
    w = estimate_dcf(traj.to(cuda), S, iters=20)
    wo = pipe_menon(traj, S, iters=20)
    assert rel(w, wo) < 1e-4
