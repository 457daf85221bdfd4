"""Many independent reconstructions of uneven size solved together on one GPU.

Each instance keeps its own NUFFT plan (grid, band buffer, spread tile/bin
sizes autotuned per size class), its own NCG state, FP64 reduction scratch and
device-side controller, so every instance follows exactly the iterations it
would follow alone.  One CUDA graph holds `iters_per_graph` NCG iterations of
every instance as parallel branches: the graph forks from the capture stream to
one stream per instance and joins back, so the GPU runs the instances' kernels
concurrently and one graph launch advances every solve.  An instance that has
met its stop rule sets its device done flag; from then on its operator kernels
return at once (plan skip flag) and its controller and update kernels leave the
state unchanged, so replays continue until the last instance stops.

The reference solves one problem per CGSolver call (graspcg/solvers/cg.py:162-246);
this module has no counterpart there.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib
from .solver import CGConfig, CGSolver, REASONS, S_DONE, S_ITER, S_REASON, capture_graph


class BatchedSolver:
    """Solve `problems` = [(y, op, regm), ...] with one CGConfig, all in one graph."""

    def __init__(self, problems: Sequence[Tuple[torch.Tensor, object, object]], cfg: Optional[CGConfig] = None):
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
        self.streams = [torch.cuda.Stream(self.device) for _ in self.solvers]
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
                    s._iteration_fast()
                self._fork(first)
                self.launch_stats["eager"] += _lib.launch_count() - n0
                if not self._all_done():
                    if c.cuda_graph and self._graph is None:
                        torch.cuda.synchronize(self.device)
                        g = torch.cuda.CUDAGraph()
                        n1 = _lib.launch_count()
                        with capture_graph(g, self.device):
                            def body(s):
                                for _ in range(max(1, c.iters_per_graph)):
                                    s._iteration_fast()
                            self._fork(body)
                        self.launch_stats["per_graph"] = _lib.launch_count() - n1
                        self._graph = g
                    while not self._all_done():
                        if c.cuda_graph:
                            self._graph.replay()
                            self.launch_stats["replays"] += 1
                        else:
                            n2 = _lib.launch_count()
                            self._fork(lambda s: [s._iteration_fast() for _ in range(max(1, c.iters_per_graph))])
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
