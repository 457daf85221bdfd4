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
(``value`` = mean seconds per step, lower is better).  ``e2e`` repeats the step
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

METRIC = "GRASP recon s-to-tol (1e-4 rel obj): warm-start+NCG vs plain NCG; NUFFT GB/s"

WORKLOADS = {
    "grasp": dict(name="grasp_256x256_34fr_12coil_21spk_512ro", N=256, C=12, F=34, spf=21, nread=512,
                  lam_s=1e-3, lam_t=5e-3, eps=1e-3, sigma=1e-3),
    "radial128": dict(name="radial_128x128_1fr_8coil_64spk_256ro", N=128, C=8, F=1, spf=64, nread=256,
                      lam_s=1e-3, lam_t=0.0, eps=1e-3, sigma=0.0),
}
STOP_WINDOW, STOP_TOL = 10, 1e-4
# iterations to tolerance of plain NCG on the default workload (measured on
# B200 by this script's b200 arm; the reference arm multiplies its measured
# seconds per iteration by it)
ITERS_TO_TOL = {"grasp": 252, "radial128": None}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="grasp", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-iters", type=int, default=1)
    ap.add_argument("--nufft-only", action="store_true",
                    help="profiling case: prepare the workload's operator and run 3 forward/adjoint pairs")
    return ap.parse_args()


# ----------------------------------------------------------------------------
# inputs
# ----------------------------------------------------------------------------
def make_inputs(w):
    from mrirecon_b200 import phantoms
    N, C, F = w["N"], w["C"], w["F"]
    x_true = phantoms.dynamic_phantom(N, F, seed=0).unsqueeze(1)          # (F,1,N,N)
    maps = phantoms.coil_maps(N, C)
    traj = phantoms.grasp_trajectory(F, w["spf"], w["nread"])             # (F,2,K)
    return x_true, maps, traj


def axis_spec():
    from mrirecon_b200.layout import AxisSpec
    return AxisSpec(image_labels=("B", "coil", "X", "Y"), kspace_labels=("B", "coil", "K"),
                    image_fft_labels=("X", "Y"), coil_label="coil")


def regs(w):
    from mrirecon_b200.regularization import RegManager, TVND, TVParams
    r = [TVND("tv_spatial", TVParams(weight=w["lam_s"], eps=w["eps"], axes="spatial"))]
    if w["lam_t"] > 0:
        r.append(TVND("tv_temporal", TVParams(weight=w["lam_t"], eps=w["eps"], axes="temporal")))
    return RegManager(r)


def solver_cfg(max_iter=3000):
    from mrirecon_b200.solver import CGConfig
    return CGConfig(direction="fr", ls_name="armijo", max_iter=max_iter, stop_window=STOP_WINDOW,
                    stop_tol=STOP_TOL, schedule="fast", cuda_graph=True, iters_per_graph=8)


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
    F, C, K = w["F"], w["C"], w["spf"] * w["nread"]
    G2 = (2 * w["N"]) ** 2
    T = info["touched_cells"]                      # summed over frames
    N2 = w["N"] ** 2
    return {
        "interp": C * (8 * T + 8 * K * F) + 4 * 2 * K * F,
        "spread": F * (C * (8 * K + 8 * G2) + 4 * 2 * K),
        "pre": F * 8 * N2 + C * 8 * N2 + F * C * 8 * G2,
        "post": F * C * 8 * N2 + C * 8 * N2 + F * 8 * N2,
    }


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
    times = []
    for it in range(warm_iter + n_iter):
        t0 = time.perf_counter()
        ok, t, f_t, g_t = o.armijo()
        if ok:
            o.x = o.x + o.d * t
            o.dir_update()
        dt = time.perf_counter() - t0
        if it >= warm_iter:
            times.append(dt)
        if not ok:
            break
    return times, cores


# ----------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------
def run_reference(args, w, ws, rank):
    if rank != 0:
        return 0
    times, cores = cpu_reference_sample(w, args.steps, args.warmup)
    s_iter = sum(times) / max(1, len(times))
    n_tol = ITERS_TO_TOL.get(args.workload)
    value = s_iter * n_tol if n_tol else None
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": s_iter * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded)",
            "config": {"workload": w["name"], "schedule": "reference (2 A + 1 A^H per trial per iteration)"},
            "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port",
                             "sample": f"{len(times)} NCG iterations (after {args.warmup} untimed) of the "
                                       f"reference schedule on the full workload; s-to-tol = s/iter x "
                                       f"{n_tol} iterations to tolerance"},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "s_per_iter": s_iter, "iters_to_tol": n_tol}
    print(json.dumps(line), flush=True)
    return 0


def run_nufft_only(w, local):
    """Profiling case: the workload's operator, three A/A^H pairs, nothing else."""
    from mrirecon_b200.nufft import NUFFT, NUFFTConfig
    dev = torch.device("cuda", local)
    x_true, maps, traj = make_inputs(w)
    op = NUFFT(maps.to(dev), traj.to(dev), None, axis=axis_spec(), config=NUFFTConfig(ndim=2, traj_units="rad"),
               device=dev)
    x = x_true.to(dev)
    y = op.A(x)
    for _ in range(3):
        op.A(x, out=y)
        op.AH(y, out=x)
    torch.cuda.synchronize()
    print(json.dumps({"nufft_only": w["name"], "plan": op.backend.plan.info()}))
    return 0


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
    for _ in range(max(args.warmup, 1)):
        solver.reset().run()
    iters = solver.iter
    # ---- timed: K solves with inputs resident ----
    l0 = solver.launches()
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        iters_list = []
        for _ in range(args.steps):
            solver.reset().run()
            iters_list.append(solver.iter)
        e1.record()
        torch.cuda.synchronize()
    barrier(ws)
    t_dev = e0.elapsed_time(e1) / 1e3
    launches = solver.launches() - l0
    t_max = max_over_ranks(t_dev, ws, dev)
    value = t_max / args.steps
    clocks = clk.summary()
    hist = solver.history()
    f_final = hist[-1]["f_accepted"] if hist else None
    # ---- e2e through the public API from pinned host buffers ----
    y_h = y.cpu().pin_memory()
    tr_h = traj.pin_memory()
    mp_h = maps.pin_memory()
    barrier(ws)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        y_d = y_h.to(dev, non_blocking=True)
        tr_d = tr_h.to(dev, non_blocking=True)
        mp_d = mp_h.to(dev, non_blocking=True)
        op2 = NUFFT(mp_d, tr_d, None, axis=axis_spec(), config=cfgN, device=dev)
        s2 = CGSolver(y_d, op2, regm, solver_cfg())
        s2.run()
        x_h = s2.result().to("cpu")
    b.record()
    torch.cuda.synchronize()
    barrier(ws)
    e2e = max_over_ranks(a.elapsed_time(b) / 1e3, ws, dev) / args.steps
    h2d = y_h.numel() * 8 + tr_h.numel() * 4 + mp_h.numel() * 8
    d2h = x_h.numel() * 8
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
    gbs = {k: ab[k] / (stages[k] * 1e-3) / 1e9 for k in ("interp", "spread", "pre", "post")}
    mine = {k: stages[k] for k in ("pre", "interp", "spread", "post")}
    dom = max(mine, key=mine.get)
    roof = {"kernel": f"{dom}_kernel", "bound": "hbm", "achieved": gbs[dom], "peak": hbm, "unit": "GB/s",
            "frac": gbs[dom] / hbm, "peak_source": peak_src, "traffic": None,
            "algorithmic_bytes_per_launch": ab[dom], "launch_ms": stages[dom]}
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded)",
            "config": {"workload": w["name"], "global_batch": ws, "frames": w["F"], "coils": w["C"],
                       "samples_per_frame": w["spf"] * w["nread"], "solver": "plain NCG FR+Armijo (fast schedule)",
                       "stop": f"windowed rel obj change W={STOP_WINDOW} tol={STOP_TOL}",
                       "l2": "working set > L2 (no flush)", "parallelism": f"replicas x{ws}"},
            "iters_to_tol": iters, "ms_per_iter": value * 1e3 / max(1, iters), "f_final": f_final,
            "nufft_ms": stages, "nufft_gbs": gbs, "roofline": roof, "spread_tuning": op.backend.tuned,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches, "clocks": clocks}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        times, cores = cpu_reference_sample(w, args.cpu_sample_iters, 0)
        s_iter = sum(times) / max(1, len(times))
        line["cpu_baseline"] = {"value": s_iter * iters, "unit": "s", "cores": cores, "kind": "port",
                                "sample": f"{len(times)} NCG iteration(s) of the reference schedule on the full "
                                          f"workload ({s_iter:.2f} s/iter); s-to-tol = s/iter x {iters} "
                                          f"iterations of the same algorithm", "s_per_iter": s_iter}
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
            return run_nufft_only(w, local)
        return run_b200(args, w, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
