"""Axis roles of an image-like tensor: (unlike..., like..., nufft...).

Same contract as graspcg/core/roles.py:7-80 (``Roles(unlike, like, nufft)``
with the tokens "temporal"/"time"/"unlike", "like", "spatial"/"image"/"nufft",
"all", "none", explicit (negative allowed) indices, de-duplicated in order).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Sequence, Tuple, Union

AxesSpec = Union[str, Sequence[int], Tuple[int, ...]]


@dataclass(frozen=True)
class Roles:
    unlike: int
    like: int
    nufft: int

    def total(self) -> int:
        return int(self.unlike) + int(self.like) + int(self.nufft)

    @property
    def ndim(self) -> int:
        return self.total()

    def token_map(self) -> Dict[str, Tuple[int, ...]]:
        u, l, n = int(self.unlike), int(self.like), int(self.nufft)
        unlike = tuple(range(u))
        like = tuple(range(u, u + l))
        spatial = tuple(range(u + l, u + l + n))
        return {"temporal": unlike, "time": unlike, "unlike": unlike, "like": like,
                "spatial": spatial, "image": spatial, "nufft": spatial,
                "all": tuple(range(u + l + n)), "none": ()}

    def resolve_axes(self, spec: AxesSpec) -> Tuple[int, ...]:
        tm = self.token_map()
        total = self.total()
        if isinstance(spec, str):
            key = spec.lower()
            if key not in tm:
                raise KeyError(f"Unknown axes token '{spec}'.")
            return tm[key]
        if not isinstance(spec, (list, tuple)):
            raise TypeError(f"Bad axes spec type: {type(spec)}")
        out = []
        for s in spec:
            if isinstance(s, str):
                key = s.lower()
                if key not in tm:
                    raise KeyError(f"Unknown axes token '{s}'.")
                out.extend(tm[key])
            elif isinstance(s, int):
                ax = s if s >= 0 else total + s
                if ax < 0 or ax >= total:
                    raise IndexError(f"Axis {s} out of range for total dims {total}")
                out.append(ax)
            else:
                raise TypeError(f"Bad axes element type: {type(s)}")
        seen, uniq = set(), []
        for a in out:
            if a not in seen:
                seen.add(a)
                uniq.append(a)
        return tuple(uniq)

    @property
    def temporal(self) -> Tuple[int, ...]:
        return self.token_map()["temporal"]

    @property
    def like_axes(self) -> Tuple[int, ...]:
        return self.token_map()["like"]

    @property
    def spatial(self) -> Tuple[int, ...]:
        return self.token_map()["spatial"]
