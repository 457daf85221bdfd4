#!/usr/bin/env python
"""Benchmark: GRASP-style 2D+t reconstruction, seconds to tolerance on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload grasp|radial128] [--no-cpu-baseline]

Workload (default ``grasp``): 256x256 complex64 images, 12 coils, 34 frames x
21 golden-angle spokes x 512 samples, ellipse phantom with gamma-variate
enhancement, complex Gaussian noise sigma=1e-3, spatial TV lambda=1e-3 +
temporal TV lambda=5e-3 (eps 1e-3), plain NCG (FR, Armijo, c1=1e-4, beta=0.5)
from x = 0 until the windowed relative objective change
(f_{k-10} - f_k) <= 10 * 1e-4 * |f_k| on the accepted objectives.  FP32
gridding/FFT/TV, FP64 reductions.  All inputs are seeded synthetic data.

One step = one reconstruction to tolerance with the inputs resident in HBM
(``value`` = mean seconds per step, lower is better): the learned warm start
(BF16 2D+t CNN on the density-compensated adjoint, packaged weights; the scaled
adjoint when the network's objective is not lower) followed by plain NCG to the
same tolerance.  ``plain_ncg`` reports plain NCG from x = 0 the same way, and
``warm_start.image_err_vs_plain`` the difference of the two results.  ``e2e`` repeats the step
through the public API from pinned host buffers (H2D of y, trajectory and
maps, operator preparation, solver, D2H of the image).  The working set
(~1 GB per solve, 855 MB oversampled grid) is far larger than L2, so no
explicit flush is needed between steps.

``--impl reference`` times the reference algorithm on the host CPU (the CPU
restatement of graspcg's CGSolver schedule with a CPU Kaiser-Bessel
operator, all host threads): one step = one NCG iteration of that schedule on
the same workload; seconds-to-tolerance = mean seconds per iteration x the
iteration count to tolerance of the same algorithm on the same inputs.

Multi-GPU (torchrun): every rank runs an independent replica of the workload
(the path does not shard); timings are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

from mrirecon_b200.warmstart import WarmStartCNN, tolerance_study, warm_start  # noqa: E402

METRIC = "GRASP recon s-to-tol (1e-4 rel obj): warm-start+NCG vs plain NCG; NUFFT GB/s"

from mrirecon_b200.workloads import (WORKLOADS, STOP_WINDOW, STOP_TOL, make_inputs, axis_spec,  # noqa: E402
                                     regs, solver_cfg)

# The CPU port of the reference solve run once to the windowed tolerance on a
# workload (tests/golden/make_port_history.py): its iteration count to
# tolerance and objective history.  One full run takes tens of minutes on the
# host, so the reference arm times a bounded sample of iterations, checks that
# the sample retraces the committed history, and scales by the committed count.
PORT_HISTORY = os.path.join(ROOT, "tests", "golden", "port_{}.npz")


def port_history(workload):
    import numpy as np
    path = PORT_HISTORY.format(workload)
    if not os.path.exists(path):
        return None
    d = np.load(path)
    return {"iters_to_tol": int(d["iters_to_tol"]), "stop": str(d["stop_reason"]), "f": d["f"].tolist(),
            "f_accepted": d["f_accepted"].tolist(), "s_per_iter": float(d["s_per_iter"]),
            "threads": int(d["threads"])}


def history_rel_diff(f_a, f_b):
    """Largest relative difference of two objective histories over their common length."""
    n = min(len(f_a), len(f_b))
    if n == 0:
        return None, 0
    return max(abs(a - b) / max(abs(b), 1e-300) for a, b in zip(f_a[:n], f_b[:n])), n


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of each
# stage's kernels on the grasp workload, from ncu captures of
# `python bench.py --nufft-only` (fft = the forward column pass storing the grid
# in 2 x 8 cell blocks, interp = the pair-parallel interp reading it, spread =
# spread_kernel storing whole 32-byte sectors that hold a touched cell into a
# grid whose other cells stay zero from a one-time fill, post = the inverse row
# pass; the small split-tile reduction is not included)
NCU_TRAFFIC = {"grasp": {"pre": 396.30e6, "fft": 1225.29e6, "interp": 344.36e6, "spread": 281.54e6,
                         "ifft": 1256.29e6, "post": 455.38e6}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="grasp", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-iters", type=int, default=1)
    ap.add_argument("--no-3d", action="store_true", help="skip the 3D koosh-ball NUFFT throughput block")
    ap.add_argument("--no-batched", action="store_true", help="skip the 16-instance uneven batch block")
    ap.add_argument("--no-toeplitz", action="store_true", help="skip the Toeplitz-schedule solve block")
    ap.add_argument("--no-jacobi", action="store_true", help="skip the Jacobi-preconditioned solve block")
    ap.add_argument("--no-tol-study", action="store_true",
                    help="skip the warm-start vs plain agreement study over stop tolerances")
    ap.add_argument("--nufft-only", action="store_true",
                    help="profiling case: prepare the workload's operator and run 3 forward/adjoint pairs")
    ap.add_argument("--ncg-only", type=int, default=0, metavar="K",
                    help="profiling case: K eager iterations of the workload's plain NCG solver between "
                         "cudaProfilerStart/Stop")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the 16-instance uneven batch block (grouped, branch and sequential solves)")
    ap.add_argument("--batched-profile", choices=["grouped", "branch"], default=None,
                    help="profiling case: one eager NCG iteration of the 16-instance batch (after 3 untimed "
                         "ones) between cudaProfilerStart/Stop")
    ap.add_argument("--plan-option", action="append", default=[], metavar="KEY=VALUE",
                    help="profiling cases: set a NUFFT plan option (mrb_plan_set_option key) before the runs")
    ap.add_argument("--koosh-only", type=int, default=0, metavar="N",
                    help="profiling case: the 3D koosh-ball operator scaled to an N^3 image (spokes x (N/160)^2, "
                         "samples per spoke x N/160, 16 coils), 3 forward/adjoint pairs")
    return ap.parse_args()


# ----------------------------------------------------------------------------
# clocks (nvidia-smi sampled during the timed region)
# ----------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [v.strip() for v in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------
# distributed plumbing (replicas)
# ----------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, ws, dev):
    if ws == 1:
        return v
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------
# algorithmic bytes (per launch) of the gridding kernels
# ----------------------------------------------------------------------------
def algorithmic_bytes(w, info):
    """Bytes each stage must move at least once (per call over all frames and coils).
    Fused FFT mode: the row passes write / read the (F, C, N, 2N) band buffer and
    the column passes read / write it and the full grid."""
    F, C, K, N = w["F"], w["C"], w["spf"] * w["nread"], w["N"]
    G2 = (2 * N) ** 2
    T = info["touched_cells"]                      # summed over frames
    N2 = N ** 2
    band = F * C * 8 * N * 2 * N
    ab = {"interp": C * (8 * T + 8 * K * F) + 4 * 2 * K * F,
          "spread": F * (C * (8 * K + 8 * G2) + 4 * 2 * K)}
    if info.get("fft_mode", 0) == 1:
        ab.update(pre=F * 8 * N2 + C * 8 * N2 + band, fft=band + F * C * 8 * G2,
                  ifft=F * C * 8 * G2 + band, post=band + C * 8 * N2 + F * 8 * N2)
    else:
        ab.update(pre=F * 8 * N2 + C * 8 * N2 + F * C * 8 * G2, fft=F * C * 16 * G2, ifft=F * C * 16 * G2,
                  post=F * C * 8 * N2 + C * 8 * N2 + F * 8 * N2)
    return ab


def time_stages(op, x, y, nb, reps=20):
    plan = op.backend.plan
    ev = lambda: torch.cuda.Event(enable_timing=True)
    out = {}
    # warm
    op.backend.A(x, out=y)
    op.backend.AH(y, out=x)
    torch.cuda.synchronize()
    for name, args in (("pre", (x, None)), ("fft", (None, None)), ("interp", (None, y)),
                       ("spread", (None, y)), ("ifft", (None, None)), ("post", (x, None))):
        a, b = ev(), ev()
        a.record()
        for _ in range(reps):
            plan.stage(name, args[0], args[1], nb)
        b.record()
        torch.cuda.synchronize()
        out[name] = a.elapsed_time(b) / reps
    for name, fn in (("A", lambda: op.backend.A(x, out=y)), ("AH", lambda: op.backend.AH(y, out=x))):
        a, b = ev(), ev()
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        out[name] = a.elapsed_time(b) / reps
    return out


# ----------------------------------------------------------------------------
# CPU: the reference schedule restated (oracle), bounded sample
# ----------------------------------------------------------------------------
def cpu_reference_sample(w, n_iter, warm_iter=0):
    """Seconds per NCG iteration of the reference schedule on the host CPU."""
    from oracle import kb as okb
    from oracle.ncg import NCGOracle, NCGConfig, TVSpec
    from mrirecon_b200 import phantoms
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    x_true, maps, traj = make_inputs(w)
    k = okb.KBNufft(maps, traj, None, dtype=torch.complex64, norm="ortho")
    y = k.A(x_true).to(torch.complex64)
    if w["sigma"] > 0:
        y = phantoms.add_noise(y, w["sigma"], seed=1)
    specs = [TVSpec((2, 3), w["lam_s"], w["eps"])]
    if w["lam_t"] > 0:
        specs.append(TVSpec((0,), w["lam_t"], w["eps"]))
    A = lambda v: k.A(v).to(torch.complex64)
    AH = lambda v: k.AH(v).to(torch.complex64)
    o = NCGOracle(A, AH, y, torch.zeros_like(x_true), specs, NCGConfig(max_iter=1))
    # prime (cg.py:178-190) untimed
    o.begin_linesearch()
    o.f_g(0.0)
    o.d = -(o.g / o.D)
    times, fs = [], []
    for it in range(warm_iter + n_iter):
        t0 = time.perf_counter()
        ok, t, f_t, g_t = o.armijo()
        if ok:
            o.x = o.x + o.d * t
            o.dir_update()
        dt = time.perf_counter() - t0
        fs.append(o._ls0[0])
        if it >= warm_iter:
            times.append(dt)
        if not ok:
            break
    return times, cores, fs


# ----------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------
def run_reference(args, w, ws, rank):
    if rank != 0:
        return 0
    times, cores, fs = cpu_reference_sample(w, args.steps, args.warmup)
    s_iter = sum(times) / max(1, len(times))
    port = port_history(args.workload)
    n_tol = port["iters_to_tol"] if port else None
    value = s_iter * n_tol if n_tol else None
    d, n = history_rel_diff(fs, port["f"]) if port else (None, 0)
    # the same port on another host's cores rounds its FP32 sums differently: the
    # histories agree to the 1e-4 objective bar the solver tests use, not bit for bit
    check = {"iterations_compared": n, "max_rel_diff": d, "retraces": d is not None and d <= 1e-4, "bar": 1e-4,
             "port_stop": port["stop"] if port else None}
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": s_iter * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded)",
            "config": {"workload": w["name"], "schedule": "reference (2 A + 1 A^H per trial per iteration)"},
            "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port",
                             "sample": f"{len(times)} NCG iterations (after {args.warmup} untimed) of the "
                                       f"reference schedule on the full workload; s-to-tol = s/iter x "
                                       f"{n_tol} iterations, the count the same port reached the windowed "
                                       f"tolerance in when run to it (tests/golden/port_{args.workload}.npz)"},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "s_per_iter": s_iter, "iters_to_tol": n_tol, "iters_to_tol_source": "CPU port run to tolerance",
            "port_history_check": check}
    print(json.dumps(line), flush=True)
    return 0


def set_plan_options(plan, traj, options):
    """KEY=VALUE strings -> mrb_plan_set_option; the sample lists are rebuilt if an option needs it."""
    for kv in options:
        k, v = kv.split("=")
        plan.set_option(int(k), int(v))
    if options and not plan.info()["points_ready"]:
        plan.set_points(traj)


def run_nufft_only(w, local, options=()):
    """Profiling case: the workload's operator, three A/A^H pairs, nothing else."""
    from mrirecon_b200.nufft import NUFFT, NUFFTConfig
    dev = torch.device("cuda", local)
    x_true, maps, traj = make_inputs(w)
    op = NUFFT(maps.to(dev), traj.to(dev), None, axis=axis_spec(), config=NUFFTConfig(ndim=2, traj_units="rad"),
               device=dev)
    set_plan_options(op.backend.plan, traj.to(dev), options)
    x = x_true.to(dev)
    y = op.A(x)
    for _ in range(3):
        op.A(x, out=y)
        op.AH(y, out=x)
    torch.cuda.synchronize()
    print(json.dumps({"nufft_only": w["name"], "plan": op.backend.plan.info()}))
    return 0


def run_ncg_only(w, n_iter, local):
    """Profiling case: the workload's plain NCG solver (fast schedule, eager
    launches), primed outside the profiled range; n_iter iterations between
    cudaProfilerStart and cudaProfilerStop (ncu --profile-from-start off)."""
    from mrirecon_b200 import phantoms
    from mrirecon_b200.nufft import NUFFT, NUFFTConfig
    from mrirecon_b200.solver import CGSolver
    dev = torch.device("cuda", local)
    x_true, maps, traj = make_inputs(w)
    op = NUFFT(maps.to(dev), traj.to(dev), None, axis=axis_spec(), config=NUFFTConfig(ndim=2, traj_units="rad"),
               device=dev)
    y = phantoms.add_noise(op.A(x_true.to(dev)), w["sigma"], seed=1) if w["sigma"] > 0 else op.A(x_true.to(dev))
    cfg = solver_cfg()
    cfg.cuda_graph = False
    s = CGSolver(y, op, regs(w), cfg)
    s._fast_setup(cfg.max_iter)
    s._prime_fast()
    s._iteration_fast()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(n_iter):
        s._iteration_fast()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"ncg_only": w["name"], "iterations": n_iter, "iter": int(s.s[4].item())}))
    return 0


def run_batched_profile(mode, local):
    """Profiling case: the 16-instance uneven batch (grouped launches or one
    stream per instance), primed and run for 3 eager iterations, then 10 timed
    iterations (CUDA events) and one iteration between cudaProfilerStart and
    cudaProfilerStop (ncu --profile-from-start off)."""
    from mrirecon_b200.batched import BatchedSolver
    from mrirecon_b200.workloads import batched_instances
    dev = torch.device("cuda", local)
    inst = batched_instances(dev)
    cfg = solver_cfg()
    cfg.restart = True
    cfg.cuda_graph = False
    bs = BatchedSolver([(p["y"], p["op"], p["regm"]) for p in inst], cfg, grouped=(mode == "grouped"))
    for s in bs.solvers:
        s._fast_setup(cfg.max_iter)

    def first(s):
        s._prime_fast()
        s._skip_on_done(True)
    bs._fork(first)
    step = lambda: bs._step(lambda s: s._iteration_fast())
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = _lib_launches()
    a.record()
    for _ in range(10):
        step()
    b.record()
    torch.cuda.synchronize()
    launches = (_lib_launches() - n0) / 10
    torch.cuda.profiler.start()
    step()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"batched_profile": mode, "eager_ms_per_iteration": a.elapsed_time(b) / 10,
                      "launches_per_iteration": launches}))
    return 0


def _lib_launches():
    from mrirecon_b200 import _lib
    return _lib.launch_count()


KOOSH = dict(name="koosh3d_160cube_16coil_20000spk_256ro", N=160, C=16, spokes=20000, nread=256)


def koosh_operator(dev, N=160):
    """The koosh-ball operator, image, maps and trajectory; N < 160 scales the
    case down at the same angular and radial sample density."""
    from mrirecon_b200 import phantoms
    from mrirecon_b200.layout import AxisSpec
    from mrirecon_b200.nufft import NUFFT, NUFFTConfig
    k = KOOSH
    C = k["C"]
    spokes = int(round(k["spokes"] * (N / k["N"]) ** 2))
    nread = 2 * int(round(k["nread"] * N / k["N"] / 2))
    x = phantoms.ellipsoid_phantom(N, seed=0).reshape(1, 1, N, N, N).to(dev, torch.complex64)
    maps = phantoms.coil_maps(N, C, ndim=3).to(dev)
    traj = phantoms.golden_means_koosh(spokes, nread).unsqueeze(0).to(dev)
    axis = AxisSpec(image_labels=("B", "coil", "X", "Y", "Z"), kspace_labels=("B", "coil", "K"),
                    image_fft_labels=("X", "Y", "Z"), coil_label="coil")
    op = NUFFT(maps, traj, None, axis=axis, config=NUFFTConfig(ndim=3, traj_units="rad"), device=dev)
    return op, x, maps, traj


def run_koosh_only(N, local):
    """Profiling case: the (scaled) koosh-ball operator, three A/A^H pairs."""
    dev = torch.device("cuda", local)
    op, x, maps, traj = koosh_operator(dev, N)
    y = op.A(x)
    for _ in range(3):
        op.A(x, out=y)
        op.AH(y, out=x)
    torch.cuda.synchronize()
    print(json.dumps({"koosh_only": N, "samples": int(traj.shape[-1]), "plan": op.backend.plan.info()}))
    return 0


def koosh3d_throughput(dev, reps=10):
    """3D radial koosh-ball NUFFT (160^3, 16 coils, 20,000 golden-means spokes x 256
    samples, grid 320^3): per-stage device times, algorithmic GB/s and fraction of
    the measured HBM peak, A / A^H times."""
    k = KOOSH
    N, C = k["N"], k["C"]
    op, x, maps, traj = koosh_operator(dev, N)
    y = op.A(x)
    st = time_stages(op, x.clone(), torch.empty_like(y), 1, reps=reps)
    info = op.backend.plan.info()
    K = k["spokes"] * k["nread"]
    Gc = (2 * N) ** 3
    T = info["touched_cells"]
    N3 = N ** 3
    ab = {"interp": C * (8 * T + 8 * K) + 12 * K, "spread": C * (8 * K + 8 * Gc) + 12 * K}
    if info.get("fft_mode", 0) == 1:
        # zero-pruned passes: z rows -> band1 (C, N, N, 2N), y columns -> band2
        # (C, N, 2N, 2N), x columns -> grid; the adjoint in reverse
        b1, b2 = C * 8 * N * N * 2 * N, C * 8 * N * 4 * N * N
        ab.update(pre=8 * N3 + C * 8 * N3 + b1, fft=b1 + 2 * b2 + C * 8 * Gc, ifft=C * 8 * Gc + 2 * b2 + b1,
                  post=b1 + C * 8 * N3 + 8 * N3)
        fft = "fused zero-pruned z / y / x passes (320^3 grid, 16 coils)"
    else:
        ab.update(pre=8 * N3 + C * 8 * N3 + C * 8 * Gc, fft=C * 16 * Gc, ifft=C * 16 * Gc,
                  post=C * 8 * N3 + C * 8 * N3 + 8 * N3)
        fft = "cuFFT dense 320^3 (C2C, batch 16)"
    gbs = {n: ab[n] / (st[n] * 1e-3) / 1e9 for n in ab}
    del op, y, maps, traj, x
    torch.cuda.empty_cache()
    return {"workload": k["name"], "nufft_ms": st, "nufft_gbs": gbs, "touched_cells": T,
            "samples": K, "grid_cells": Gc, "fft": fft}


def batched_throughput(dev, steps=3):
    """16 uneven independent 2D radial recons to tolerance, device seconds per
    batch: grouped launches (one launch per kernel step over all instances of a
    kernel shape, captured in one CUDA graph), one graph branch per instance,
    and the same solves run one after another (each with its own graph)."""
    from mrirecon_b200.batched import BatchedSolver
    from mrirecon_b200.solver import CGSolver
    from mrirecon_b200.workloads import BATCHED, batched_instances
    inst = batched_instances(dev)
    cfg = solver_cfg()
    # densely sampled instances overshoot on the first Armijo step and the first
    # FR update (beta = 1) then gives a non-descent direction: restart instead of stopping
    cfg.restart = True
    probs = [(p["y"], p["op"], p["regm"]) for p in inst]
    bs = BatchedSolver(probs, cfg, grouped=True)
    br = BatchedSolver(probs, cfg, grouped=False)
    seq = [CGSolver(p["y"], p["op"], p["regm"], cfg) for p in inst]
    bs.reset().run()
    br.reset().run()
    for s in seq:
        s.reset().run()
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(solver):
        torch.cuda.synchronize()
        a, b = ev(), ev()
        l0 = solver.launches()
        a.record()
        for _ in range(steps):
            solver.reset().run()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1e3 / steps, (solver.launches() - l0) // steps

    t_b, launches = timed(bs)
    t_r, launches_r = timed(br)
    a, b = ev(), ev()
    a.record()
    for _ in range(steps):
        for s in seq:
            s.reset().run()
    b.record()
    torch.cuda.synchronize()
    t_s = a.elapsed_time(b) / 1e3 / steps
    same = all(torch.equal(x, s.result()) for x, s in zip(bs.results(), seq))
    same_r = all(torch.equal(x, s.result()) for x, s in zip(br.results(), seq))
    return {"workload": BATCHED["name"], "batched_graph_s": t_b, "sequential_s": t_s, "speedup": t_s / t_b,
            "mode": "grouped launches (one per kernel step over the instances of an image shape; shapes on their own "
                    "streams), one CUDA graph",
            "gpu_launches_per_batch": launches, "identical_to_sequential": bool(same),
            "branch_graph_s": t_r, "branch_gpu_launches_per_batch": launches_r,
            "branch_identical_to_sequential": bool(same_r),
            "solver": "plain NCG FR+Armijo (fast schedule) with restart on non-descent",
            "instances": [{"N": p["N"], "coils": p["C"], "spokes": p["spokes"], "iters": s.iter,
                           "restarts": s.restarts, "stop": s.stop_reason} for p, s in zip(inst, bs.solvers)]}


def cpu_leg_parity(w, op, y, f_hist_plain, iters_plain, port):
    """Parity at the headline shape, computed on the host beside the CPU baseline
    (outside every timed region): the GPU operator against the oracle's FP64
    Kaiser-Bessel gridding (A of the phantom, A^H of the measured data, rel-L2,
    and the adjoint ratio <A x, y> / <x, A^H y>), and the GPU plain NCG
    objective history against the CPU port's history to tolerance."""
    from oracle import kb as okb
    x_true, maps, traj = make_inputs(w)
    orc = okb.KBNufft(maps.to(torch.complex128), traj, None, dtype=torch.complex128, norm="ortho")
    x64 = x_true.to(torch.complex128)
    y64 = y.cpu().to(torch.complex128)
    yg = op.A(x_true.to(y.device)).cpu().to(torch.complex128)
    xg = op.AH(y).cpu().to(torch.complex128)
    rel = lambda u, v: float(torch.linalg.vector_norm(u - v) / torch.linalg.vector_norm(v))
    fwd = rel(yg, orc.A(x64))
    adj = rel(xg, orc.AH(y64))
    ratio = complex(torch.vdot(yg.reshape(-1), y64.reshape(-1)) / torch.vdot(x64.reshape(-1), xg.reshape(-1)))
    out = {"operator_vs_fp64_oracle": {"forward_rel_l2": fwd, "adjoint_rel_l2": adj,
                                       "adjoint_ratio_err": abs(ratio - 1), "bar": 1e-5}}
    if port:
        d20, _ = history_rel_diff(f_hist_plain[:20], port["f"][:20])
        dall, nall = history_rel_diff(f_hist_plain, port["f"])
        out["plain_ncg_vs_cpu_port"] = {"first_20_max_rel_diff": d20, "all_common_max_rel_diff": dall,
                                        "common_iterations": nall, "gpu_iters_to_tol": iters_plain,
                                        "port_iters_to_tol": port["iters_to_tol"],
                                        "port_final_f": port["f_accepted"][-1] if port["f_accepted"] else None}
    return out


def solve_once(solver, cnn):
    """One reconstruction to tolerance: plain NCG from x = 0, or the learned
    warm start (with its fallback to the scaled adjoint) followed by NCG."""
    if cnn is None:
        solver.reset().run()
    else:
        warm_start(solver, cnn)
        solver.run()


def time_solves(solver, cnn, steps, ws, dev, local):
    """K solves with the inputs resident, device time (max over ranks) per solve."""
    from mrirecon_b200 import _lib
    l_lib, l_sol, l_eager = _lib.launch_count(), solver.launches(), solver.launch_stats["eager"]
    barrier(ws)
    torch.cuda.synchronize()
    iters = []
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            solve_once(solver, cnn)
            iters.append(solver.iter)
        e1.record()
        torch.cuda.synchronize()
    barrier(ws)
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3, ws, dev) / steps
    # eager launches (solver, warm start, network) + graph replays of the solver
    replayed = (solver.launches() - l_sol) - (solver.launch_stats["eager"] - l_eager)
    launches = (_lib.launch_count() - l_lib) + replayed
    return {"value": t, "iters_to_tol": iters[-1], "ms_per_iter": t * 1e3 / max(1, iters[-1]),
            "gpu_launches": launches // steps * steps, "clocks": clk.summary()}


def e2e_solves(y, traj, maps, regm, cfgN, cnn, steps, ws, dev, warmup=1):
    """The same solve through the public API from pinned host buffers: H2D of the
    data, trajectory and maps, operator preparation, (warm start,) NCG, D2H.
    `warmup` untimed steps first; each timed step bracketed by its own CUDA events."""
    import gc
    from mrirecon_b200.nufft import NUFFT
    from mrirecon_b200.solver import CGSolver
    y_h = y.cpu().pin_memory()
    tr_h = traj.pin_memory()
    mp_h = maps.pin_memory()
    x_pin = None

    def one():
        nonlocal x_pin
        y_d = y_h.to(dev, non_blocking=True)
        tr_d = tr_h.to(dev, non_blocking=True)
        mp_d = mp_h.to(dev, non_blocking=True)
        op2 = NUFFT(mp_d, tr_d, None, axis=axis_spec(), config=cfgN, device=dev)
        s2 = CGSolver(y_d, op2, regm, solver_cfg())
        if cnn is not None:
            warm_start(s2, cnn)
        s2.run()
        x = s2.result()
        if x_pin is None:
            x_pin = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
        x_pin.copy_(x, non_blocking=True)   # D2H into a pinned host buffer, waited for by the caller
        return x_pin

    for _ in range(max(1, warmup)):
        one()
        gc.collect()
    barrier(ws)
    torch.cuda.synchronize()
    per_step = []
    for _ in range(steps):
        # the previous step's operator and solver are released before the clock starts
        gc.collect()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        x_h = one()
        b.record()
        torch.cuda.synchronize()
        per_step.append(a.elapsed_time(b) / 1e3)
    barrier(ws)
    e2e = max_over_ranks(sum(per_step), ws, dev) / steps
    return e2e, y_h.numel() * 8 + tr_h.numel() * 4 + mp_h.numel() * 8, x_h.numel() * 8, per_step


def toeplitz_solve(op, y, regm, x_ref, f_ref, steps=3):
    """Plain NCG with the Toeplitz normal operator on the same problem: device
    seconds per solve (transfer-function set-up timed separately), iterations,
    image error and objective (gridded operator) against the gridded solve."""
    from mrirecon_b200.solver import CGSolver
    ev = lambda: torch.cuda.Event(enable_timing=True)
    a, b = ev(), ev()
    torch.cuda.synchronize()
    a.record()
    op.backend.prepare_toeplitz()
    b.record()
    torch.cuda.synchronize()
    t_setup = a.elapsed_time(b) / 1e3
    cfg = solver_cfg()
    cfg.schedule = "toeplitz"
    s = CGSolver(y, op, regm, cfg)
    s.reset().run()
    a, b = ev(), ev()
    a.record()
    for _ in range(steps):
        s.reset().run()
    b.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3 / steps
    xr = s.result()
    err = float(torch.linalg.vector_norm(xr - x_ref) / torch.linalg.vector_norm(x_ref))
    f = s.objective()
    return {"s_to_tol": t, "psf_setup_s": t_setup, "iters_to_tol": s.iter, "ms_per_iter": t * 1e3 / max(1, s.iter),
            "image_err_vs_gridded_plain": err, "objective_gridded": f,
            "objective_rel_diff_vs_gridded_plain": (f - f_ref) / abs(f_ref), "stop": s.stop_reason}


def jacobi_solve(op, y, regm, x_ref, f_ref, steps=3):
    """Plain NCG with the Jacobi diagonal (precond="jacobi": alpha sum|S|^2 plus the
    regularisers' add_diag at the zero start) on the same problem and stop rule:
    device seconds per solve including the diagonal set-up, iterations, image
    error and objective against the unpreconditioned solve."""
    from mrirecon_b200.solver import CGSolver
    cfg = solver_cfg()
    cfg.precond = "jacobi"
    s = CGSolver(y, op, regm, cfg)
    s.reset().run()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    a, b = ev(), ev()
    torch.cuda.synchronize()
    a.record()
    for _ in range(steps):
        s.reset().run()
    b.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3 / steps
    xr = s.result()
    err = float(torch.linalg.vector_norm(xr - x_ref) / torch.linalg.vector_norm(x_ref))
    f = s.objective()
    # the two solves stop at different objectives: also the first iteration at
    # which the preconditioned solve reaches the plain solve's final objective
    fa = [h["f_accepted"] for h in s.history()]
    k_ref = next((k + 1 for k, v in enumerate(fa) if v <= f_ref), None)
    ms_it = t * 1e3 / max(1, s.iter)
    return {"s_to_tol": t, "iters_to_tol": s.iter, "ms_per_iter": ms_it,
            "image_err_vs_plain": err, "objective": f, "objective_rel_diff_vs_plain": (f - f_ref) / abs(f_ref),
            "iters_to_plain_objective": k_ref,
            "s_to_plain_objective_est": None if k_ref is None else k_ref * ms_it / 1e3, "stop": s.stop_reason}


def run_b200(args, w, ws, rank, local):
    from mrirecon_b200 import _lib, phantoms
    from mrirecon_b200.nufft import NUFFT, NUFFTConfig
    from mrirecon_b200.solver import CGSolver
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    x_true, maps, traj = make_inputs(w)
    cfgN = NUFFTConfig(ndim=2, traj_units="rad", autotune=True)
    op = NUFFT(maps.to(dev), traj.to(dev), None, axis=axis_spec(), config=cfgN, device=dev)
    y = op.A(x_true.to(dev))
    if w["sigma"] > 0:
        y = phantoms.add_noise(y, w["sigma"], seed=1)
    regm = regs(w)
    solver = CGSolver(y, op, regm, solver_cfg())
    cnn = WarmStartCNN.pretrained(dev)
    for _ in range(max(args.warmup, 1)):
        solve_once(solver, None)
        solve_once(solver, cnn)
    # ---- timed: K solves with inputs resident, plain NCG then warm-start + NCG ----
    plain = time_solves(solver, None, args.steps, ws, dev, local)
    x_plain = solver.result().clone()
    f_plain = solver.objective()
    f_hist_plain = [h["f"] for h in solver.history()]
    warm = time_solves(solver, cnn, args.steps, ws, dev, local)
    x_warm = solver.result().clone()
    f_warm = solver.objective()
    warm["image_err_vs_plain"] = float(torch.linalg.vector_norm(x_warm - x_plain) / torch.linalg.vector_norm(x_plain))
    warm["objective"], plain["objective"] = f_warm, f_plain
    xt = x_true.to(dev).reshape(x_plain.shape)
    plain["image_err_vs_truth"] = float(torch.linalg.vector_norm(x_plain - xt) / torch.linalg.vector_norm(xt))
    warm["image_err_vs_truth"] = float(torch.linalg.vector_norm(x_warm - xt) / torch.linalg.vector_norm(xt))
    value = warm["value"]
    clocks = warm.pop("clocks")
    plain_clocks = plain.pop("clocks")
    launches = warm.pop("gpu_launches")
    plain["gpu_launches"] = plain.pop("gpu_launches")
    iters = warm["iters_to_tol"]
    # ---- e2e through the public API from pinned host buffers ----
    p_e2e, _, _, p_steps = e2e_solves(y, traj, maps, regm, cfgN, None, args.steps, ws, dev, args.warmup)
    plain["e2e"] = {"value": p_e2e, "unit": "s", "per_step": p_steps}
    e2e, h2d, d2h, e2e_steps = e2e_solves(y, traj, maps, regm, cfgN, cnn, args.steps, ws, dev, args.warmup)
    # ---- NUFFT stage timings and roofline ----
    xs = torch.zeros((w["F"], 1, w["N"], w["N"]), dtype=torch.complex64, device=dev)
    ys = torch.empty_like(y)
    stages = time_stages(op, xs, ys, w["F"])
    info = op.backend.plan.info()
    ab = algorithmic_bytes(w, info)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    gbs = {k: ab[k] / (stages[k] * 1e-3) / 1e9 for k in ("pre", "fft", "interp", "spread", "ifft", "post")}
    own = ("pre", "fft", "interp", "spread", "ifft", "post") if info.get("fft_mode", 0) == 1 else \
        ("pre", "interp", "spread", "post")
    mine = {k: stages[k] for k in own}
    dom = max(mine, key=mine.get)
    kname = {"pre": "fwd_rows_kernel", "fft": "fwd_cols_kernel", "interp": "interp2p_kernel",
             "spread": "spread_kernel", "ifft": "adj_cols_kernel", "post": "adj_rows_kernel"}
    if info.get("fft_mode", 0) != 1:
        kname.update(pre="pre_fft_kernel", post="post_ifft_kernel")
    roof = {"kernel": kname[dom], "stage": dom, "bound": "hbm", "achieved": gbs[dom], "peak": hbm, "unit": "GB/s",
            "frac": gbs[dom] / hbm, "peak_source": peak_src,
            "traffic": NCU_TRAFFIC.get(args.workload, {}).get(dom) if info.get("fft_mode", 0) == 1 else None,
            "algorithmic_bytes_per_launch": ab[dom], "launch_ms": stages[dom]}
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded)",
            "config": {"workload": w["name"], "global_batch": ws, "frames": w["F"], "coils": w["C"],
                       "samples_per_frame": w["spf"] * w["nread"],
                       "solver": "learned warm start (BF16 2D+t CNN, fallback to the scaled adjoint) + plain NCG "
                                 "FR+Armijo (fast schedule, gridded operator)",
                       "stop": f"windowed rel obj change W={STOP_WINDOW} tol={STOP_TOL}",
                       "l2": "working set > L2 (no flush)", "parallelism": f"replicas x{ws}"},
            "iters_to_tol": iters, "ms_per_iter": value * 1e3 / max(1, iters),
            "warm_start": warm, "plain_ncg": plain, "plain_clocks": plain_clocks,
            "nufft_ms": stages, "nufft_gbs": gbs, "nufft_frac_of_peak": {k: v / hbm for k, v in gbs.items()},
            "fft_mode": "fused zero-pruned row/column passes" if info.get("fft_mode", 0) == 1 else "cuFFT",
            "roofline": roof, "spread_tuning": op.backend.tuned,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "per_step": e2e_steps},
            "gpu_launches": launches, "clocks": clocks}
    if not args.no_jacobi:
        line["jacobi"] = jacobi_solve(op, y, regm, x_plain, f_plain)
    if not args.no_toeplitz:
        line["toeplitz"] = toeplitz_solve(op, y, regm, x_plain, f_plain)
    if not args.no_batched:
        line["batched16"] = batched_throughput(dev)
    if not args.no_3d:
        k3 = koosh3d_throughput(dev)
        k3["frac_of_peak"] = {n: v / hbm for n, v in k3["nufft_gbs"].items()}
        line["koosh3d"] = k3
    if not args.no_tol_study:
        line["tolerance_study"] = tolerance_study(cnn, workload=args.workload, device=dev)
        from mrirecon_b200.warmstart import training_step_time
        line["warmstart_training_step"] = training_step_time(dev)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        times, cores, _ = cpu_reference_sample(w, args.cpu_sample_iters, 0)
        s_iter = sum(times) / max(1, len(times))
        port = port_history(args.workload)
        n_tol = port["iters_to_tol"] if port else plain["iters_to_tol"]
        src = (f"the count the same port reached the windowed tolerance in when run to it "
               f"(tests/golden/port_{args.workload}.npz)") if port else "the count of plain NCG on the GPU"
        line["cpu_baseline"] = {"value": s_iter * n_tol, "unit": "s", "cores": cores, "kind": "port",
                                "sample": f"{len(times)} NCG iteration(s) of the reference schedule on the full "
                                          f"workload ({s_iter:.2f} s/iter); s-to-tol = s/iter x {n_tol} "
                                          f"iterations, {src} (the reference has no learned start)",
                                "s_per_iter": s_iter, "iters_to_tol": n_tol}
        line["parity"] = cpu_leg_parity(w, op, y, f_hist_plain, plain["iters_to_tol"], port)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    w = WORKLOADS[args.workload]
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            return run_reference(args, w, ws, rank)
        if args.nufft_only:
            return run_nufft_only(w, local, args.plan_option)
        if args.koosh_only:
            return run_koosh_only(args.koosh_only, local)
        if args.ncg_only:
            return run_ncg_only(w, args.ncg_only, local)
        if args.batched_profile:
            return run_batched_profile(args.batched_profile, local)
        if args.batched_only:
            print(json.dumps({"batched16": batched_throughput(torch.device("cuda", local))}))
            return 0
        return run_b200(args, w, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
