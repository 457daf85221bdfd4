"""Non-linear CG restatement, reference schedule (CPU; TEST INFRASTRUCTURE ONLY).

One shard, diag preconditioner = ones (the reference never fills it) unless a
diagonal D is given (then d = beta d - g/D and every rho is <g, g/D>), policy a
no-op.  Follows:

* CGSolver.run                 graspcg/solvers/cg.py:162-246
    prime: begin_linesearch, f_g(0), d = -g/D, dir.init_state  (:178-190)
    loop: line search; stop on failure (:197-202); x += t d (:205-207);
    stats (:210-222); converged (:233-235); dir.update (:238-244)
* Armijo / strong Wolfe        graspcg/numerics/line_search.py:24-203
* FR / PR+ / DY directions     graspcg/numerics/directions.py:75-162
    (FR seeds rho_prev with the current rho on its first update, so the first
     FR beta is 1: directions.py:146-156)
* Objective.f_g_tensor         graspcg/ops/objective.py:184-291
    r = Ax + t Ad - y; f = 0.5||r||^2 + R(x + t d); g = A^H r + grad R
* optional restart (NCGConfig.restart, not in the reference): a direction
    with Re<g, d> >= 0 after the update becomes -g/D
* converged                    graspcg/solvers/utils.py:40-43
* history                      graspcg/solvers/utils.py:64-87; the reference
    adds xnorm/gnorm/stepnorm into live StatsBoard slots that are never reset,
    so its history reports running sums of them: reproduced here.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import torch

from .graph import GraphSpec, graph_energy_grad
from .tv import tv_energy_grad


@dataclass
class TVSpec:
    axes: Sequence[int]
    weight: float
    eps: float = 1e-3
    isotropic: bool = True
    axis_weights: Optional[Sequence[float]] = None


@dataclass
class NCGConfig:
    direction: str = "fr"
    ls_name: str = "armijo"
    c1: float = 1e-4
    c2: float = 0.9
    ls_beta: float = 0.5
    ls_max_iter: int = 20
    max_iter: int = 50
    tol_g: float = 1e-4
    tol_step: float = 1e-9
    restart: bool = False   # not in the reference: non-descent direction -> -g/D
    # not in the reference: windowed relative objective change on the accepted
    # objectives fa = [f(x_0), f(x_1), ...]: stop after iteration k when
    # fa[k+1-W] - fa[k+1] <= W * stop_tol * |fa[k+1]| (W = stop_window > 0)
    stop_window: int = 0
    stop_tol: float = 1e-4


def _rdot(a, b):
    return torch.vdot(a.reshape(-1), b.reshape(-1)).real


class NCGOracle:
    """x, y are CPU tensors; A/AH map between them; regs are TVSpec."""

    def __init__(self, A: Callable, AH: Callable, y: torch.Tensor, x0: torch.Tensor,
                 regs: Sequence[TVSpec], cfg: Optional[NCGConfig] = None, D: Optional[torch.Tensor] = None):
        self.Aop, self.AHop = A, AH
        self.cfg = cfg or NCGConfig()
        self.y = y
        self.x = x0.clone()
        self.d = torch.zeros_like(x0)
        self.g = torch.zeros_like(x0)
        # preconditioner diagonal: ones as in the reference solve, or a given D
        self.D = torch.ones(x0.shape, dtype=x0.real.dtype) if D is None else D.to(x0.real.dtype).reshape(x0.shape)
        self.regs = list(regs)
        self.Ax = None
        self.Ad = None
        self.rho_prev = None
        self.g_prev = None
        self.hist: List[Dict[str, float]] = []
        self.n_A = 0
        self.n_AH = 0
        self.n_restart = 0
        self._cum = {"xnorm": 0.0, "gnorm": 0.0, "stepnorm": 0.0}

    # --- objective -----------------------------------------------------------
    def begin_linesearch(self):
        self.Ax = self.Aop(self.x)
        self.Ad = self.Aop(self.d)
        self.n_A += 2

    def f_g(self, t: float):
        r = self.Ad * t + self.Ax - self.y
        f_data = 0.5 * _rdot(r, r)
        g = self.AHop(r)
        self.n_AH += 1
        xt = self.x + self.d * t
        f_reg = torch.zeros((), dtype=f_data.dtype)
        for s in self.regs:
            if isinstance(s, GraphSpec):
                E, gr = graph_energy_grad(xt, s.L, s.weight)
                E = E.to(f_data.dtype)
            else:
                E, gr = tv_energy_grad(xt, s.axes, s.weight, s.eps, s.isotropic, s.axis_weights)
            f_reg = f_reg + E
            g = g + gr
        self.g = g
        return float(f_data + f_reg), float(_rdot(g, self.d))

    # --- line searches -------------------------------------------------------
    def armijo(self):
        c = self.cfg
        self.begin_linesearch()
        t = 1.0
        f0, g0d = self.f_g(0.0)
        self._ls0 = (f0, g0d)
        if not (g0d < 0) or math.isnan(g0d) or math.isinf(g0d):
            return False, 0.0, f0, g0d
        f_t = g_t = float("nan")
        for _ in range(c.ls_max_iter):
            f_t, g_t = self.f_g(t)
            if f_t <= f0 + c.c1 * t * g0d:
                return True, t, f_t, g_t
            t *= c.ls_beta
        return False, t, f_t, g_t

    def wolfe(self):
        c = self.cfg
        self.begin_linesearch()
        t = 1.0
        f0, g0d = self.f_g(0.0)
        self._ls0 = (f0, g0d)
        if not (g0d < 0) or math.isnan(g0d) or math.isinf(g0d):
            return False, 0.0, f0, g0d
        t_prev, f_prev, g_prev = 0.0, f0, g0d
        for i in range(c.ls_max_iter):
            f_t, g_t = self.f_g(t)
            if (f_t > f0 + c.c1 * t * g0d) or (i > 0 and f_t >= f_prev):
                return self._zoom(t_prev, f_prev, t, f0, g0d)
            if abs(g_t) <= c.c2 * abs(g0d):
                return True, t, f_t, g_t
            if g_t >= 0:
                return self._zoom(t, f_t, t_prev, f0, g0d)
            t_prev, f_prev, g_prev = t, f_t, g_t
            t = min(2.0 * t, 1e6)
        return False, t_prev, f_prev, g_prev

    def _zoom(self, t_lo, f_lo, t_hi, f0, g0d):
        c = self.cfg
        for _ in range(c.ls_max_iter):
            t_mid = 0.5 * (t_lo + t_hi)
            f_mid, g_mid = self.f_g(t_mid)
            if (f_mid > f0 + c.c1 * t_mid * g0d) or (f_mid >= f_lo):
                t_hi = t_mid
            else:
                if abs(g_mid) <= c.c2 * abs(g0d):
                    return True, t_mid, f_mid, g_mid
                if g_mid * (t_hi - t_lo) >= 0:
                    t_hi = t_lo
                t_lo, f_lo = t_mid, f_mid
        f_lo, g_lo = self.f_g(t_lo)
        return True, t_lo, f_lo, g_lo

    # --- directions ------------------------------------------------------------
    def _pdot(self, a, b):
        return float(_rdot(a, b / self.D))

    def dir_init(self):
        if self.cfg.direction in ("prplus", "dy"):
            self.g_prev = self.g.clone()

    def dir_update(self):
        name = self.cfg.direction
        if name == "fr":
            if self.rho_prev is None:
                self.rho_prev = self._pdot(self.g, self.g)
            rho = self._pdot(self.g, self.g)
            beta = rho / max(self.rho_prev, 1e-20)
            self.rho_prev = rho
        elif name == "prplus":
            num = self._pdot(self.g, self.g) - self._pdot(self.g_prev, self.g)
            den = self._pdot(self.g_prev, self.g_prev)
            beta = max(num / max(den, 1e-20), 0.0)
        elif name == "dy":
            num = self._pdot(self.g, self.g)
            den = float(_rdot(self.d, self.g)) - float(_rdot(self.d, self.g_prev))
            beta = num / max(den, 1e-20)
        else:
            raise ValueError(name)
        self.d = self.d * beta - self.g / self.D
        if self.cfg.restart and not (float(_rdot(self.g, self.d)) < 0.0):
            self.d = -(self.g / self.D)
            self.n_restart += 1
        if name in ("prplus", "dy"):
            self.g_prev = self.g.clone()
        return beta

    # --- driver ----------------------------------------------------------------
    def run(self, max_iter: Optional[int] = None, stop: Optional[Callable[[List[float]], bool]] = None,
            log: Optional[Callable[[int, float], None]] = None):
        c = self.cfg
        self.stop_reason = "max_iter"
        fa: List[float] = []
        max_iter = int(max_iter or c.max_iter)
        self.begin_linesearch()
        self.f_g(0.0)
        self.d = -(self.g / self.D)
        self.dir_init()
        ls = self.wolfe if c.ls_name == "wolfe" else self.armijo
        for k in range(max_iter):
            ok, t, f_t, g_t = ls()
            if not ok:
                self.stop_reason = "line search failed"
                break
            self.x = self.x + self.d * t
            xn = math.sqrt(max(float(_rdot(self.x, self.x)), 0.0))
            sn = math.sqrt(max(float(_rdot(self.d, self.d)), 0.0))
            gn = math.sqrt(max(self._pdot(self.g, self.g), 0.0))
            for kk, v in (("xnorm", xn), ("stepnorm", sn), ("gnorm", gn)):
                self._cum[kk] += v
            f0, g0d = self._ls0
            if not fa:
                fa.append(f0)
            fa.append(f_t)
            self.hist.append(dict(iter=k, f=f0, gdot=g0d, gdot_at_step=g_t, step=t,
                                  xnorm=self._cum["xnorm"], gnorm=self._cum["gnorm"],
                                  stepnorm=self._cum["stepnorm"],
                                  xnorm_iter=xn, gnorm_iter=gn, stepnorm_iter=sn, f_accepted=f_t))
            if log is not None:
                log(k, f_t)
            if gn <= (1.0 + xn) * c.tol_g and sn <= (1.0 + xn) * c.tol_step:
                self.stop_reason = "converged"
                break
            W = c.stop_window
            if W > 0 and len(fa) - 1 >= W and fa[-1 - W] - fa[-1] <= W * c.stop_tol * abs(fa[-1]):
                self.stop_reason = "relative objective change"
                break
            if stop is not None and stop([h["f"] for h in self.hist]):
                self.stop_reason = "callback"
                break
            self.dir_update()
        return self
