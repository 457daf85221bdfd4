"""Roles and the layout grammar against their contract (CPU).

The expected values restate graspcg's ``Roles`` (graspcg/core/roles.py:37-65)
and layout planners (graspcg/nufft/layout.py:11-193).  Where an installed copy
of the reference is importable (MRB_GRASPCG_PATH or ``baseline/_ref``), the
same specs are also run through the reference classes and the results and
exception types compared.
"""
import importlib
import os

import pytest
import torch

from conftest import ROOT
from mrirecon_b200.layout import (AxisSpec, plan_image_layout, plan_image_layout_from_sizes,
                                  plan_kspace_layout, plan_kspace_layout_from_sizes, user_image_shape,
                                  user_kspace_shape)
from mrirecon_b200.roles import Roles

SPECS = ["temporal", "time", "unlike", "like", "spatial", "image", "nufft", "all", "none", "SPATIAL",
         (2, 3), [0, -1], (-1, -1, 2), ("temporal", 3), ["like", "spatial", 1], (), "bogus", ("x",),
         (7,), (-9,), 3, (1.5,), {"a": 1}]


def _outcome(fn):
    try:
        return ("ok", fn())
    except (KeyError, TypeError, IndexError, ValueError) as e:
        return ("raise", type(e))


def test_roles_resolve_expected():
    r = Roles(1, 1, 2)
    assert r.resolve_axes("spatial") == (2, 3)
    assert r.resolve_axes("temporal") == (0,)
    assert r.resolve_axes(("temporal", 3, -1, 0)) == (0, 3)
    assert r.resolve_axes("all") == (0, 1, 2, 3) and r.resolve_axes("none") == ()
    assert r.total() == r.ndim == 4 and r.spatial == (2, 3) and r.like_axes == (1,)
    assert Roles(2, 0, 3).resolve_axes(["like", "image"]) == (2, 3, 4)
    with pytest.raises(KeyError):
        r.resolve_axes("bogus")
    with pytest.raises(TypeError):
        r.resolve_axes(3)
    with pytest.raises(TypeError):
        r.resolve_axes((1.5,))
    with pytest.raises(IndexError):
        r.resolve_axes((4,))
    assert Roles(1, 1, 2) == Roles(1, 1, 2) and hash(Roles(1, 1, 2)) == hash(Roles(1, 1, 2))


def test_layout_expected():
    ax = AxisSpec(image=("B", "T", "coil", "X", "Y"), kspace=("B", "T", "coil", "K"), image_fft=("X", "Y"))
    assert ax.coil == "coil" and ax.kspace_fft == ("K",)
    assert AxisSpec(image_labels=("B", "X"), kspace_labels=("B", "K"), image_fft_labels=("X",),
                    coil_label="c").coil == "c"
    p = plan_image_layout(torch.zeros(2, 5, 1, 8, 6), ax)
    assert (p.B, p.like_labels, p.like_sizes, p.L_other, p.spatial) == (2, ("T",), (5,), 5, (8, 6))
    q = plan_kspace_layout(torch.zeros(2, 5, 4, 30), ax)
    assert (q.B, q.like_sizes, q.C, q.K) == (2, (5,), 4, 30)
    with pytest.raises(ValueError):
        plan_image_layout(torch.zeros(2, 5, 3, 8, 6), ax)
    with pytest.raises(ValueError):
        plan_image_layout(torch.zeros(2, 8, 6), ax)
    with pytest.raises(TypeError):
        AxisSpec(image=("B", "X"), kspace=("B", "K"))
    assert user_image_shape(ax, 2, (5,), (8, 6)) == (2, 5, 1, 8, 6)
    assert user_kspace_shape(ax, 2, (5,), 4, 30) == (2, 5, 4, 30)
    ax2 = AxisSpec(image=("B", "T", "E", "X"), kspace=("B", "T", "E", "coil", "K"), image_fft=("X",))
    assert plan_image_layout_from_sizes(1, (6,), (8,), ax2).like_sizes == (6, 1)
    assert plan_kspace_layout_from_sizes(1, (2, 3), 4, 9, ax2).L_other == 6
    with pytest.raises(ValueError):
        plan_image_layout_from_sizes(1, (2, 3, 4), (8,), ax2)


@pytest.fixture
def reference(monkeypatch):
    p = os.environ.get("MRB_GRASPCG_PATH") or os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isfile(os.path.join(p, "graspcg", "core", "roles.py")):
        pytest.skip(f"graspcg is not installed at {p}")
    monkeypatch.syspath_prepend(p)
    return importlib.import_module("graspcg.core.roles"), importlib.import_module("graspcg.nufft.layout")


@pytest.mark.parametrize("counts", [(1, 1, 2), (1, 0, 3), (2, 1, 2), (0, 0, 1)])
def test_roles_against_reference(reference, counts):
    ref_roles, _ = reference
    mine, ref = Roles(*counts), ref_roles.Roles(*counts)
    assert mine.token_map() == ref.token_map()
    for spec in SPECS:
        assert _outcome(lambda: mine.resolve_axes(spec)) == _outcome(lambda: ref.resolve_axes(spec)), spec


def test_layout_against_reference(reference):
    _, ref = reference
    kw = [dict(image=("B", "T", "coil", "X", "Y"), kspace=("B", "T", "coil", "K"), image_fft=("X", "Y")),
          dict(image_labels=("B", "coil", "X"), kspace_labels=("B", "coil", "K"), image_fft_labels=("X",),
               coil_label="coil"),
          dict(image=("T", "E", "X", "Y"), kspace=("T", "E", "c", "K"), image_fft=("X", "Y"), coil="c")]
    for k in kw:
        a, b = AxisSpec(**k), ref.AxisSpec(**k)
        for f in ("image", "kspace", "image_fft", "kspace_fft", "coil"):
            assert getattr(a, f) == getattr(b, f)
        for shape in [(2, 5, 1, 8, 6), (2, 5, 3, 8, 6), (3, 1, 7), (2, 3, 8, 6), (4, 4, 4, 4)]:
            x = torch.zeros(shape)
            if len(shape) != len(a.image):
                # the reference maps labels onto the leading dims of any tensor;
                # here a tensor whose rank differs from the labels is refused
                assert _outcome(lambda: plan_image_layout(x, a)) == ("raise", ValueError)
                continue
            pa = _outcome(lambda: plan_image_layout(x, a))
            pb = _outcome(lambda: ref.plan_image_layout(x, b))
            assert pa[0] == pb[0], (k, shape)
            if pa[0] == "ok":
                for f in ("B", "like_labels", "like_sizes", "L_other", "spatial"):
                    assert getattr(pa[1], f) == getattr(pb[1], f)
        for L in [(), (5,), (2, 3), (1, 2, 3)]:
            qa = _outcome(lambda: plan_kspace_layout_from_sizes(2, L, 4, 30, a))
            qb = _outcome(lambda: ref.plan_kspace_layout_from_sizes(2, L, 4, 30, b))
            assert qa[0] == qb[0] and (qa[0] != "ok" or (qa[1].like_sizes, qa[1].L_other) ==
                                       (qb[1].like_sizes, qb[1].L_other)), (k, L)
