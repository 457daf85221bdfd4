"""Run the CPU port of the reference solve to tolerance on a workload and keep its history.

    python tests/golden/make_port_history.py [grasp|radial128] [max_iter]

The port is ``oracle.ncg.NCGOracle`` (graspcg's CGSolver schedule restated:
FR + Armijo, c1 = 1e-4, t0 = 1, x0.5, <= 20 trials, diag = ones) on the FP32
Kaiser-Bessel operator ``oracle.kb.KBNufft`` (ortho scaling) and the
workload's TV terms, from x = 0, stopped by the windowed relative objective
change (W = 10, tol = 1e-4) that the GPU solver uses.  This is the same
computation that ``bench.py --impl reference`` times per iteration; one full
run takes tens of minutes on a CPU, so its iteration count to tolerance and
its objective history are committed here instead of being re-run by every
bench:

  port_<workload>.npz  f (f(x_k) at the start of each iteration), f_accepted,
                       step, gdot, iters_to_tol, stop_reason, s_per_iter,
                       threads, per-frame |x| of the result
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)


def port_solver(w, max_iter):
    from mrirecon_b200 import phantoms
    from mrirecon_b200.workloads import make_inputs, STOP_WINDOW, STOP_TOL
    from oracle import kb as okb
    from oracle.ncg import NCGConfig, NCGOracle, TVSpec
    x_true, maps, traj = make_inputs(w)
    k = okb.KBNufft(maps, traj, None, dtype=torch.complex64, norm="ortho")
    y = k.A(x_true).to(torch.complex64)
    if w["sigma"] > 0:
        y = phantoms.add_noise(y, w["sigma"], seed=1)
    specs = [TVSpec((2, 3), w["lam_s"], w["eps"])]
    if w["lam_t"] > 0:
        specs.append(TVSpec((0,), w["lam_t"], w["eps"]))
    cfg = NCGConfig(max_iter=max_iter, tol_g=0.0, tol_step=0.0, stop_window=STOP_WINDOW, stop_tol=STOP_TOL)
    A = lambda v: k.A(v).to(torch.complex64)
    AH = lambda v: k.AH(v).to(torch.complex64)
    return NCGOracle(A, AH, y, torch.zeros_like(x_true), specs, cfg)


def main():
    from mrirecon_b200.workloads import WORKLOADS
    name = sys.argv[1] if len(sys.argv) > 1 else "grasp"
    max_iter = int(sys.argv[2]) if len(sys.argv) > 2 else 600
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    o = port_solver(WORKLOADS[name], max_iter)
    t0 = time.perf_counter()
    o.run(log=lambda k, f: print(f"iteration {k}: f {f:.8e} ({time.perf_counter() - t0:.0f} s)", flush=True))
    dt = time.perf_counter() - t0
    h = o.hist
    out = {k: np.array([r[k] for r in h], dtype=np.float64) for k in ("f", "f_accepted", "step", "gdot")}
    out["iters_to_tol"] = np.int64(len(h))
    out["stop_reason"] = np.array(o.stop_reason)
    out["s_per_iter"] = np.float64(dt / max(1, len(h)))
    out["threads"] = np.int64(threads)
    out["frame_norms"] = o.x.reshape(o.x.shape[0], -1).abs().pow(2).sum(1).sqrt().double().numpy()
    np.savez_compressed(os.path.join(HERE, f"port_{name}.npz"), **out)
    print(f"{name}: {len(h)} iterations ({o.stop_reason}), {dt:.0f} s, final f {out['f_accepted'][-1]:.6e}")


if __name__ == "__main__":
    main()
