"""Axis grammar and layout planners of the NUFFT front-end.

Same behaviour as graspcg/nufft/layout.py:11-193: ``AxisSpec`` accepts the new
(``image_labels``...) or legacy (``image``...) keyword names; the planners
infer B, the "like" labels/sizes (every image label that is not 'B', the coil
label or an FFT label) and the spatial / coil / K sizes from a tensor or from
bare sizes.  Images must be coil-combined (coil axis of size 1 if present).
"""
from __future__ import annotations

from dataclasses import dataclass
from functools import reduce
import operator
from typing import Dict, Sequence, Tuple

import torch


@dataclass(init=False)
class AxisSpec:
    image_labels: Tuple[str, ...]
    kspace_labels: Tuple[str, ...]
    image_fft_labels: Tuple[str, ...]
    kspace_fft_labels: Tuple[str, ...]
    coil_label: str

    def __init__(self, *, image_labels=None, kspace_labels=None, image_fft_labels=None, kspace_fft_labels=None,
                 coil_label=None, image=None, kspace=None, image_fft=None, kspace_fft=None, coil=None):
        image_labels = image_labels if image_labels is not None else image
        kspace_labels = kspace_labels if kspace_labels is not None else kspace
        image_fft_labels = image_fft_labels if image_fft_labels is not None else image_fft
        kspace_fft_labels = kspace_fft_labels if kspace_fft_labels is not None else kspace_fft
        if coil_label is None:
            coil_label = coil if coil is not None else "coil"
        if image_labels is None or kspace_labels is None or image_fft_labels is None:
            raise TypeError("AxisSpec requires image(_labels)=..., kspace(_labels)=..., image_fft(_labels)=...")
        if kspace_fft_labels is None:
            kspace_fft_labels = ("K",)
        object.__setattr__(self, "image_labels", tuple(image_labels))
        object.__setattr__(self, "kspace_labels", tuple(kspace_labels))
        object.__setattr__(self, "image_fft_labels", tuple(image_fft_labels))
        object.__setattr__(self, "kspace_fft_labels", tuple(kspace_fft_labels))
        object.__setattr__(self, "coil_label", str(coil_label))

    @property
    def image(self):
        return self.image_labels

    @property
    def kspace(self):
        return self.kspace_labels

    @property
    def image_fft(self):
        return self.image_fft_labels

    @property
    def kspace_fft(self):
        return self.kspace_fft_labels

    @property
    def coil(self):
        return self.coil_label


def _prod(seq: Sequence[int]) -> int:
    return int(reduce(operator.mul, seq, 1))


def like_labels_image(axis: AxisSpec) -> Tuple[str, ...]:
    return tuple(l for l in axis.image if l not in axis.image_fft and l != "B" and l != axis.coil)


def like_labels_kspace(axis: AxisSpec) -> Tuple[str, ...]:
    return tuple(l for l in axis.kspace if l not in axis.kspace_fft and l not in ("B", axis.coil))


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


def plan_image_layout(x_user: torch.Tensor, axis: AxisSpec) -> ImageLayoutPlan:
    if x_user.ndim != len(axis.image):
        raise ValueError(f"image tensor has {x_user.ndim} dims but the axis spec names {len(axis.image)}")
    sizes = {l: int(x_user.shape[i]) for i, l in enumerate(axis.image)}
    if axis.coil in sizes and sizes[axis.coil] != 1:
        raise ValueError("Image is expected coil-combined; axis.coil dim must be size 1 if present.")
    ll = like_labels_image(axis)
    ls = tuple(sizes[l] for l in ll)
    return ImageLayoutPlan(axis, sizes.get("B", 1), ll, ls, _prod(ls) if ll else 1,
                           tuple(sizes[l] for l in axis.image_fft))


def plan_kspace_layout(y_user: torch.Tensor, axis: AxisSpec) -> KspaceLayoutPlan:
    if y_user.ndim != len(axis.kspace):
        raise ValueError(f"k-space tensor has {y_user.ndim} dims but the axis spec names {len(axis.kspace)}")
    sizes = {l: int(y_user.shape[i]) for i, l in enumerate(axis.kspace)}
    ll = like_labels_kspace(axis)
    ls = tuple(sizes[l] for l in ll)
    return KspaceLayoutPlan(axis, sizes.get("B", 1), ll, ls, _prod(ls) if ll else 1, sizes[axis.coil],
                            sizes[axis.kspace_fft[0]])


def _like_from_sizes(like_labels, L_sizes):
    if len(like_labels) == 0:
        return tuple(), 1
    if len(L_sizes) == len(like_labels):
        ls = tuple(int(v) for v in L_sizes)
        return ls, _prod(ls)
    if len(L_sizes) == 1:
        pad = [1] * len(like_labels)
        pad[0] = int(L_sizes[0])
        return tuple(pad), int(L_sizes[0])
    raise ValueError("L_sizes length must be 0, 1, or match number of like labels.")


def plan_image_layout_from_sizes(B, L_sizes, spatial, axis: AxisSpec) -> ImageLayoutPlan:
    ll = like_labels_image(axis)
    ls, L = _like_from_sizes(ll, L_sizes)
    return ImageLayoutPlan(axis, int(B), ll, ls, int(L), tuple(int(s) for s in spatial))


def plan_kspace_layout_from_sizes(B, L_sizes, C, K, axis: AxisSpec) -> KspaceLayoutPlan:
    ll = like_labels_kspace(axis)
    ls, L = _like_from_sizes(ll, L_sizes)
    return KspaceLayoutPlan(axis, int(B), ll, ls, int(L), int(C), int(K))


def user_kspace_shape(axis: AxisSpec, B, L_sizes, C, K) -> Tuple[int, ...]:
    plan = plan_kspace_layout_from_sizes(B, L_sizes, C, K, axis)
    size: Dict[str, int] = {"B": plan.B, axis.coil: plan.C, axis.kspace_fft[0]: plan.K}
    size.update({l: int(s) for l, s in zip(plan.like_labels, plan.like_sizes)})
    return tuple(int(size[l]) for l in axis.kspace)


def user_image_shape(axis: AxisSpec, B, L_sizes, spatial) -> Tuple[int, ...]:
    plan = plan_image_layout_from_sizes(B, L_sizes, spatial, axis)
    size: Dict[str, int] = {"B": plan.B, axis.coil: 1}
    size.update({l: int(s) for l, s in zip(plan.like_labels, plan.like_sizes)})
    size.update({l: int(spatial[i]) for i, l in enumerate(axis.image_fft)})
    return tuple(int(size[l]) for l in axis.image)
