"""Many independent reconstructions of uneven size solved together on one GPU.

Each instance keeps its own NUFFT plan (grid, band buffer, spread tile/bin
sizes autotuned per size class), its own NCG state, FP64 reduction scratch and
device-side controller, so every instance follows exactly the iterations it
would follow alone.  An instance that has met its stop rule sets its device
done flag; from then on its operator kernels return at once (plan skip flag)
and its controller and update kernels leave the state unchanged, so the solve
continues until the last instance stops.

Grouped mode (the default): one NCG iteration of every instance is recorded
through the library's launch recorder (mrb_group_begin / mrb_group_select /
mrb_group_end) and issued as grouped launches: each kernel step of the
iteration (row FFTs, column FFTs, interp, k-space pass, spread, split-tile
reduction, inverse passes, TV energies and gradient, Armijo, controller,
update, restart) is ONE launch over all instances, whose blocks find their
instance and its arguments in a table in kernel parameter space.  Instances
that differ in a kernel's compile-time shape (the FFT length of their size
class, the spread tile and variant) take one launch per shape.  With
split_by_shape (the default) the instances of one image shape form a partition
recorded on its own and replayed on its own stream, so that size classes do
not wait for one another at every kernel step.  `iters_per_graph` iterations
of these launches are captured in one CUDA graph.

Branch mode (grouped=False): the graph forks from the capture stream to one
stream per instance and joins back; every instance issues its own launches.
It serves the paths without grouped kernels (Toeplitz normal operator, cuFFT
mode, 3D block spreads).

Both modes are bit-identical to solving the instances one after another.
The reference solves one problem per CGSolver call (graspcg/solvers/cg.py:162-246);
this module has no counterpart there.
"""
from __future__ import annotations

import ctypes as ct
from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib
from .solver import CGConfig, CGSolver, REASONS, S_DONE, S_ITER, S_REASON, capture_graph


class BatchedSolver:
    """Solve `problems` = [(y, op, regm), ...] with one CGConfig, all in one graph."""

    def __init__(self, problems: Sequence[Tuple[torch.Tensor, object, object]], cfg: Optional[CGConfig] = None,
                 grouped: bool = True, split_by_shape: bool = True):
        if len(problems) == 0:
            raise ValueError("no problems")
        self.cfg = cfg or CGConfig()
        if self.cfg.schedule != "fast":
            raise ValueError("batched solves use the fast (device-controlled) schedule")
        self.solvers: List[CGSolver] = []
        for y, op, regm in problems:
            s = CGSolver(y, op, regm, CGConfig(**vars(self.cfg)))
            # private reduction scratch: instances run concurrently
            s.ws_buf = torch.zeros(_lib.workspace_bytes(), dtype=torch.uint8, device=s.device)
            self.solvers.append(s)
        self.device = self.solvers[0].device
        if any(s.device != self.device for s in self.solvers):
            raise ValueError("all instances must live on one device")
        self.grouped = bool(grouped)
        self.lib = _lib.load()
        self.streams = [torch.cuda.Stream(self.device) for _ in self.solvers]
        # grouped mode: instances of one image shape (one FFT size class) form a
        # partition whose grouped launches run on a stream of their own, so that
        # size classes do not wait for one another at every kernel step
        shapes: dict = {}
        for i, s in enumerate(self.solvers):
            key = tuple(s.x.shape) if split_by_shape else ()
            shapes.setdefault(key, []).append(i)
        self.partitions: List[List[int]] = list(shapes.values())
        self._stats = [0, 0]
        self.part_streams = [torch.cuda.Stream(self.device) for _ in self.partitions]
        self._graph = None
        self._done = torch.zeros(len(self.solvers), dtype=torch.float64, device=self.device)
        self.launch_stats = {"eager": 0, "per_graph": 0, "replays": 0}

    def reset(self, x0s: Optional[Sequence[torch.Tensor]] = None) -> "BatchedSolver":
        for i, s in enumerate(self.solvers):
            s.reset(None if x0s is None else x0s[i])
        return self

    def _fork(self, fn):
        main = torch.cuda.current_stream(self.device)
        for s, st in zip(self.solvers, self.streams):
            st.wait_stream(main)
            with torch.cuda.stream(st):
                fn(s)
        for st in self.streams:
            main.wait_stream(st)

    def _record(self, fn):
        """fn(s) for every instance, one recording per partition; each partition's
        recorded kernel launches are issued as grouped launches on its own stream,
        forked from and joined to the current stream."""
        lib = self.lib
        main = torch.cuda.current_stream(self.device)
        one = len(self.partitions) == 1
        self._stats = [0, 0]
        for part, st in zip(self.partitions, self.part_streams):
            if not one:
                st.wait_stream(main)
            _lib.check(lib.mrb_group_begin(len(part)), "group_begin")
            try:
                for k, i in enumerate(part):
                    _lib.check(lib.mrb_group_select(k), "group_select")
                    fn(self.solvers[i])
            except BaseException:
                lib.mrb_group_cancel()
                raise
            _lib.check(lib.mrb_group_end(_lib.stream_ptr(self.device) if one else st.cuda_stream), "group_end")
            r, l = ct.c_int64(0), ct.c_int64(0)
            _lib.check(lib.mrb_group_stats(ct.byref(r), ct.byref(l)), "group_stats")
            self._stats[0] += int(r.value)
            self._stats[1] += int(l.value)
        if not one:
            for st in self.part_streams:
                main.wait_stream(st)

    def _step(self, fn):
        """fn(s) for every instance: grouped launches or one stream per instance."""
        if self.grouped:
            self._record(fn)
        else:
            self._fork(fn)

    def group_stats(self) -> Tuple[int, int]:
        """(records, launches) of the last grouped step, summed over the partitions."""
        return tuple(getattr(self, "_stats", (0, 0)))

    def _all_done(self) -> bool:
        torch.stack([s.s[S_DONE] for s in self.solvers], out=self._done)
        return bool(self._done.min().item() != 0.0)

    @torch.no_grad()
    def run(self, max_iter: Optional[int] = None) -> "BatchedSolver":
        c = self.cfg
        max_iter = int(max_iter or c.max_iter)
        with torch.cuda.device(self.device):
            try:
                for s in self.solvers:
                    if not s._fast_setup(max_iter):
                        self._graph = None
                n0 = _lib.launch_count()

                def first(s):
                    s._prime_fast()
                    s._skip_on_done(True)
                self._fork(first)
                self._step(lambda s: s._iteration_fast())
                self.launch_stats["eager"] += _lib.launch_count() - n0
                if not self._all_done():
                    if c.cuda_graph and self._graph is None:
                        torch.cuda.synchronize(self.device)
                        g = torch.cuda.CUDAGraph()
                        n1 = _lib.launch_count()
                        with capture_graph(g, self.device):
                            for _ in range(max(1, c.iters_per_graph)):
                                self._step(lambda s: s._iteration_fast())
                        self.launch_stats["per_graph"] = _lib.launch_count() - n1
                        self._graph = g
                    while not self._all_done():
                        if c.cuda_graph:
                            self._graph.replay()
                            self.launch_stats["replays"] += 1
                        else:
                            n2 = _lib.launch_count()
                            for _ in range(max(1, c.iters_per_graph)):
                                self._step(lambda s: s._iteration_fast())
                            self.launch_stats["eager"] += _lib.launch_count() - n2
            finally:
                for s in self.solvers:
                    s._skip_on_done(False)
            for s in self.solvers:
                s.iter = int(s.s[S_ITER].item())
                s.stop_reason = REASONS[int(s.s[S_REASON].item())]
        return self

    def results(self) -> List[torch.Tensor]:
        return [s.result() for s in self.solvers]

    def iterations(self) -> List[int]:
        return [s.iter for s in self.solvers]

    def launches(self) -> int:
        ls = self.launch_stats
        return ls["eager"] + ls["per_graph"] * ls["replays"]
