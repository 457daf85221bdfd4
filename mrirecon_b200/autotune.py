"""Spread tile / coil-group / chunk / kernel autotuner.

For a prepared plan it times the adjoint spread stage (the kernel whose speed
depends on the tiling; interp, pre/post and the FFT do not) for a list of
(tile edge, coils per work item, samples per chunk, kernel) candidates on the plan's
own trajectory, keeps the fastest and caches the choice per size class
(nd, image shape, frames, coils and samples per frame bucketed) and GPU name in a JSON
file (``$MRB_TUNE_CACHE`` or ``~/.cache/mrirecon_b200/spread_tune.json``).
All candidates compute the same grid (deterministically, up to the order in
which split tiles sum their partial tiles).
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, Iterable, Optional, Sequence, Tuple

import torch

# (tile edge, coils per work item, samples per chunk, kernel): kernel 1 is the
# block-per-tile spread (2D tile 16, 3D tile 8; coils per block = min(coils per
# item, 16)), kernel 0 the per-warp spread
CANDIDATES_2D: Tuple[Tuple[int, int, int, int], ...] = (
    (16, 16, 128, 1), (16, 16, 256, 1), (16, 16, 512, 1), (16, 16, 64, 1),
    (16, 4, 128, 0), (16, 6, 128, 0), (8, 4, 64, 0), (32, 2, 128, 0),
    (16, 6, 128, 2), (16, 12, 128, 2), (16, 4, 128, 2))
CANDIDATES_3D: Tuple[Tuple[int, int, int, int], ...] = (
    (8, 16, 4096, 1), (8, 8, 4096, 1), (8, 16, 1024, 1), (8, 8, 1024, 1), (8, 16, 16384, 1), (4, 4, 256, 0),
    (4, 8, 256, 0), (8, 16, 4096, 2), (8, 8, 4096, 2), (8, 16, 1024, 2))


def _cache_path() -> str:
    p = os.environ.get("MRB_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "mrirecon_b200", "spread_tune.json")


def size_class(plan) -> str:
    """Tuning key: GPU, image shape, frames, coils rounded up to a multiple of 4
    and samples per frame in half-octave buckets (plans in one class share a choice)."""
    name = torch.cuda.get_device_name(plan.device)
    cq = -(-int(plan.C) // 4) * 4
    kq = round(2.0 * math.log2(max(1, int(plan.K)))) / 2.0
    return f"{name}|nd{plan.nd}|S{'x'.join(map(str, plan.S))}|C{cq}|B{plan.B}|K2^{kq:g}"


def _load() -> Dict[str, dict]:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(d: Dict[str, dict]) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
    except Exception:
        pass


def time_spread(plan, y: torch.Tensor, nb: int, reps: int = 5) -> float:
    for _ in range(2):
        plan.stage("spread", None, y, nb)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(plan.device)
    a.record()
    for _ in range(reps):
        plan.stage("spread", None, y, nb)
    b.record()
    torch.cuda.synchronize(plan.device)
    return a.elapsed_time(b) / reps


def apply(plan, traj: torch.Tensor, tile: int, cpi: int, chunk: int, kernel: int = 1) -> None:
    from .nufft import OPT_CHUNK, OPT_COILS_PER_ITEM, OPT_SPREAD_KERNEL, OPT_TILE
    plan.set_option(OPT_TILE, tile)
    plan.set_option(OPT_COILS_PER_ITEM, cpi)
    plan.set_option(OPT_CHUNK, chunk)
    plan.set_option(OPT_SPREAD_KERNEL, kernel)
    if not plan.info()["points_ready"]:      # the lists depend on the tile and chunk only
        plan.set_points(traj)


def tune(plan, traj: torch.Tensor, candidates: Optional[Iterable[Tuple[int, ...]]] = None,
         reps: int = 5, use_cache: bool = True) -> dict:
    """Pick (tile, coils per item, chunk, kernel) for `plan`; leaves the plan set to it."""
    key = size_class(plan)
    cache = _load() if use_cache else {}
    if use_cache and key in cache and "kernel" in cache[key]:
        c = cache[key]
        apply(plan, traj, c["tile"], c["cpi"], c["chunk"], c["kernel"])
        return dict(c, cached=True)
    if candidates is None:
        candidates = CANDIDATES_2D if plan.nd == 2 else CANDIDATES_3D
    g = torch.Generator(device=plan.device).manual_seed(0)
    y = torch.randn((plan.B, plan.C, plan.K), dtype=torch.complex64, device=plan.device, generator=g)
    results = []
    for cand in candidates:
        tile, cpi, chunk = cand[:3]
        kernel = cand[3] if len(cand) > 3 else 0
        if tile < 4 or min(plan.G) < tile:
            continue
        try:
            apply(plan, traj, tile, min(cpi, plan.C), chunk, kernel)
            results.append((time_spread(plan, y, plan.B, reps), tile, min(cpi, plan.C), chunk, kernel))
        except RuntimeError:
            continue                     # e.g. shared memory above the per-block limit
    if not results:
        raise RuntimeError("no spread configuration could be timed")
    ms, tile, cpi, chunk, kernel = min(results)
    apply(plan, traj, tile, cpi, chunk, kernel)
    best = {"tile": tile, "cpi": cpi, "chunk": chunk, "kernel": kernel, "ms": ms,
            "tried": [{"tile": t, "cpi": c, "chunk": h, "kernel": kk, "ms": m} for m, t, c, h, kk in sorted(results)]}
    if use_cache:
        cache[key] = {k: best[k] for k in ("tile", "cpi", "chunk", "kernel", "ms")}
        _store(cache)
    return best
