"""Axis roles of an image-like tensor: (unlike..., like..., nufft...).

The contract of graspcg's ``Roles`` (graspcg/core/roles.py:7-80) is kept so
that reference code and this package exchange role objects freely: the
constructor ``Roles(unlike, like, nufft)``, the tokens ("temporal", "time" and
"unlike" name the leading group; "like"; "spatial", "image" and "nufft" name
the trailing group; "all"; "none"), explicit axis indices with negative values
counted from the end, the first-seen order with repeats dropped, and the
exception types (KeyError for an unknown token, TypeError for a spec or
element of the wrong type, IndexError for an axis outside the tensor).

Here the three groups are laid out once per object as contiguous index
ranges, and every token is an alias of one group (or of all of them), so a
spec resolves by table lookups only.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Iterable, Sequence, Tuple, Union

AxesSpec = Union[str, Sequence[int], Tuple[int, ...]]

# token -> the group(s) it names, in axis order
_TOKEN_GROUPS: Dict[str, Tuple[str, ...]] = {
    "unlike": ("unlike",), "temporal": ("unlike",), "time": ("unlike",),
    "like": ("like",),
    "nufft": ("nufft",), "spatial": ("nufft",), "image": ("nufft",),
    "all": ("unlike", "like", "nufft"),
    "none": (),
}


@dataclass(frozen=True)
class Roles:
    unlike: int
    like: int
    nufft: int

    def __post_init__(self):
        start, spans = 0, {}
        for group in ("unlike", "like", "nufft"):
            count = int(getattr(self, group))
            spans[group] = tuple(range(start, start + count))
            start += count
        table = {tok: sum((spans[g] for g in groups), ()) for tok, groups in _TOKEN_GROUPS.items()}
        object.__setattr__(self, "_table", table)
        object.__setattr__(self, "_n", start)

    def total(self) -> int:
        return self._n

    @property
    def ndim(self) -> int:
        return self._n

    def token_map(self) -> Dict[str, Tuple[int, ...]]:
        return dict(self._table)

    def _token(self, name: str) -> Tuple[int, ...]:
        hit = self._table.get(name.lower())
        if hit is None:
            raise KeyError(f"axes token {name!r} is not one of {sorted(self._table)}")
        return hit

    def _index(self, i: int) -> int:
        ax = i + self._n if i < 0 else i
        if not 0 <= ax < self._n:
            raise IndexError(f"axis {i} does not exist in a tensor of {self._n} axes")
        return ax

    def _items(self, spec: AxesSpec) -> Iterable[int]:
        if isinstance(spec, str):
            yield from self._token(spec)
            return
        if not isinstance(spec, (list, tuple)):
            raise TypeError(f"axes spec must be a token or a list/tuple of tokens and ints, not {type(spec).__name__}")
        for item in spec:
            if isinstance(item, str):
                yield from self._token(item)
            elif isinstance(item, int):
                yield self._index(item)
            else:
                raise TypeError(f"axes spec element must be a token or an int, not {type(item).__name__}")

    def resolve_axes(self, spec: AxesSpec) -> Tuple[int, ...]:
        return tuple(dict.fromkeys(self._items(spec)))

    @property
    def temporal(self) -> Tuple[int, ...]:
        return self._table["unlike"]

    @property
    def like_axes(self) -> Tuple[int, ...]:
        return self._table["like"]

    @property
    def spatial(self) -> Tuple[int, ...]:
        return self._table["nufft"]
