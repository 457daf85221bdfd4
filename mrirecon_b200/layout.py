"""Axis grammar and layout planners of the NUFFT front-end.

The interface follows graspcg/nufft/layout.py:11-193 so that reference callers
construct axis specs and read plans unchanged: ``AxisSpec`` takes either the
``*_labels`` keyword names or the shorter legacy names (``image``, ``kspace``,
``image_fft``, ``kspace_fft``, ``coil``), the coil label defaults to 'coil' and
the k-space FFT labels to ('K',); a plan carries B, the "like" labels and
sizes (image or k-space labels that are neither 'B', the coil label nor an FFT
label) with their product, and the spatial sizes or the coil count and K.
Errors keep the reference's exception types: TypeError for a spec without its
three required label groups, ValueError for a tensor that does not fit.

Here an AxisSpec resolves its keywords through one alias table, and the
planners share one classification of labels into roles.
"""
from __future__ import annotations

from dataclasses import dataclass
import math
from typing import Dict, Sequence, Tuple

import torch

# (field, its legacy keyword)
_FIELDS = (("image_labels", "image"), ("kspace_labels", "kspace"), ("image_fft_labels", "image_fft"),
           ("kspace_fft_labels", "kspace_fft"), ("coil_label", "coil"))
_DEFAULTS = {"kspace_fft_labels": ("K",), "coil_label": "coil"}


@dataclass(frozen=True, init=False)
class AxisSpec:
    image_labels: Tuple[str, ...]
    kspace_labels: Tuple[str, ...]
    image_fft_labels: Tuple[str, ...]
    kspace_fft_labels: Tuple[str, ...]
    coil_label: str

    def __init__(self, **names):
        legacy_of = dict(_FIELDS)
        known = set(legacy_of) | set(legacy_of.values())
        unknown = sorted(set(names) - known)
        if unknown:
            raise TypeError(f"AxisSpec got unexpected keyword(s) {unknown}")
        for field, legacy in _FIELDS:
            v = names.get(field)
            if v is None:
                v = names.get(legacy)
            if v is None:
                v = _DEFAULTS.get(field)
            if v is None:
                raise TypeError(f"AxisSpec needs {field}= (or {legacy}=); the image, k-space and image FFT "
                                f"labels have no default")
            object.__setattr__(self, field, str(v) if field == "coil_label" else tuple(v))

    image = property(lambda self: self.image_labels)
    kspace = property(lambda self: self.kspace_labels)
    image_fft = property(lambda self: self.image_fft_labels)
    kspace_fft = property(lambda self: self.kspace_fft_labels)
    coil = property(lambda self: self.coil_label)


def _like(labels: Sequence[str], fft: Sequence[str], coil: str) -> Tuple[str, ...]:
    """Labels that are neither the batch 'B', the coil label nor an FFT label."""
    skip = set(fft) | {"B", coil}
    return tuple(l for l in labels if l not in skip)


def like_labels_image(axis: AxisSpec) -> Tuple[str, ...]:
    return _like(axis.image, axis.image_fft, axis.coil)


def like_labels_kspace(axis: AxisSpec) -> Tuple[str, ...]:
    return _like(axis.kspace, axis.kspace_fft, axis.coil)


@dataclass(frozen=True)
class ImageLayoutPlan:
    axis: AxisSpec
    B: int
    like_labels: Tuple[str, ...]
    like_sizes: Tuple[int, ...]
    L_other: int
    spatial: Tuple[int, ...]


@dataclass(frozen=True)
class KspaceLayoutPlan:
    axis: AxisSpec
    B: int
    like_labels: Tuple[str, ...]
    like_sizes: Tuple[int, ...]
    L_other: int
    C: int
    K: int


def _sizes_by_label(t: torch.Tensor, labels: Sequence[str], what: str) -> Dict[str, int]:
    if t.ndim != len(labels):
        raise ValueError(f"{what} tensor of shape {tuple(t.shape)} does not match the {len(labels)} labels "
                         f"{tuple(labels)}")
    return {l: int(n) for l, n in zip(labels, t.shape)}


def plan_image_layout(x_user: torch.Tensor, axis: AxisSpec) -> ImageLayoutPlan:
    size = _sizes_by_label(x_user, axis.image, "image")
    ncoil = size.get(axis.coil, 1)
    if ncoil != 1:
        raise ValueError(f"images are coil-combined: axis {axis.coil!r} has size {ncoil} instead of 1")
    like = like_labels_image(axis)
    ls = tuple(size[l] for l in like)
    return ImageLayoutPlan(axis, size.get("B", 1), like, ls, math.prod(ls), tuple(size[l] for l in axis.image_fft))


def plan_kspace_layout(y_user: torch.Tensor, axis: AxisSpec) -> KspaceLayoutPlan:
    size = _sizes_by_label(y_user, axis.kspace, "k-space")
    like = like_labels_kspace(axis)
    ls = tuple(size[l] for l in like)
    return KspaceLayoutPlan(axis, size.get("B", 1), like, ls, math.prod(ls), size[axis.coil],
                            size[axis.kspace_fft[0]])


def _like_sizes(like: Tuple[str, ...], L_sizes: Sequence[int]) -> Tuple[Tuple[int, ...], int]:
    """Sizes of the like labels from bare sizes: none, one per label, or a single
    product that goes to the first label (the others get 1)."""
    L_sizes = [int(v) for v in L_sizes]
    if not like:
        return (), 1
    if len(L_sizes) == len(like):
        return tuple(L_sizes), math.prod(L_sizes)
    if len(L_sizes) == 1:
        return (L_sizes[0],) + (1,) * (len(like) - 1), L_sizes[0]
    raise ValueError(f"{len(L_sizes)} like sizes given for the like labels {like}: give none, one, "
                     f"or {len(like)}")


def plan_image_layout_from_sizes(B, L_sizes, spatial, axis: AxisSpec) -> ImageLayoutPlan:
    like = like_labels_image(axis)
    ls, L = _like_sizes(like, L_sizes)
    return ImageLayoutPlan(axis, int(B), like, ls, L, tuple(int(s) for s in spatial))


def plan_kspace_layout_from_sizes(B, L_sizes, C, K, axis: AxisSpec) -> KspaceLayoutPlan:
    like = like_labels_kspace(axis)
    ls, L = _like_sizes(like, L_sizes)
    return KspaceLayoutPlan(axis, int(B), like, ls, L, int(C), int(K))


def user_kspace_shape(axis: AxisSpec, B, L_sizes, C, K) -> Tuple[int, ...]:
    plan = plan_kspace_layout_from_sizes(B, L_sizes, C, K, axis)
    size = dict(zip(plan.like_labels, plan.like_sizes))
    size.update({"B": plan.B, axis.coil: plan.C, axis.kspace_fft[0]: plan.K})
    return tuple(int(size[l]) for l in axis.kspace)


def user_image_shape(axis: AxisSpec, B, L_sizes, spatial) -> Tuple[int, ...]:
    plan = plan_image_layout_from_sizes(B, L_sizes, spatial, axis)
    size = dict(zip(plan.like_labels, plan.like_sizes))
    size.update(zip(axis.image_fft, plan.spatial))
    size.update({"B": plan.B, axis.coil: 1})
    return tuple(int(size[l]) for l in axis.image)
