"""B200 NUFFT backend and the user-facing front-end.

``B200NUFFTAdapter`` has the adapter surface of the reference's torchkb
backend (graspcg/nufft/backends/torchkb.py:9-364): ``prepare``, ``A``,
``AH`` (out=-first, shapes (B_eff, Cin, *S) / (B_eff, L, Cin, *S) and
(B_eff, C, K) / (B_eff, L, C, K)), ``k_per_frame``, ``diag_AHA_profile``,
``diag_AHA_scalar`` and the attributes ``traj_units``, ``dcf_mode``,
``apply_dcf_in_fwd`` / ``apply_dcf_in_adj``.  The arithmetic runs in the
hand-written sm_100a kernels of ``libmrirecon_b200.so``; there is no CPU path.

``NUFFT`` mirrors the reference front-end graspcg/nufft/api.py:52-376 (axis
labelled user layouts folded to canonical views, out= writes in place) with
``NUFFTConfig(backend='b200')``.  Two differences, both fixes:
* ``roles_image`` counts the image's size-1 coil slot as a like axis, so that
  the "spatial" token resolves to the FFT axes (api.py:159-161 leaves the coil
  slot out and "spatial" then names (coil, X));
* ``norm`` (default 'ortho') scales A and AH by 1/sqrt(prod G), which the
  Armijo line search needs to find a step from t = 1 in 20 halvings.
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass, field
from typing import Literal, Optional, Sequence, Tuple

import torch

from . import _lib
from .layout import (AxisSpec, plan_image_layout, plan_kspace_layout, plan_image_layout_from_sizes,
                     plan_kspace_layout_from_sizes, user_image_shape, user_kspace_shape)
from .roles import Roles

OPT_TILE, OPT_COILS_PER_ITEM, OPT_INTERP_MODE, OPT_CHUNK, OPT_FFT_MODE, OPT_INTERLEAVE, OPT_SPREAD_KERNEL, \
    OPT_GRID_MASK, OPT_COL_INTERP, OPT_GRID_BLOCKS, OPT_TAP_TABLE = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10
FFT_CUFFT, FFT_FUSED = 0, 1
_DCF_MODES = {"none": 0, "balanced": 1, "standard": 2}


class KBPlan:
    """Owner of one ``mrb_plan`` (trajectory tables, maps, grid, cuFFT plans)."""

    def __init__(self, S: Sequence[int], C: int, B: int, K: int, *, W: int = 4, osf: float = 2.0,
                 ortho: bool = True, device=None):
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.S = tuple(int(s) for s in S)
        self.nd = len(self.S)
        self.C, self.B, self.K = int(C), int(B), int(K)
        h = ct.c_void_p()
        arr = (ct.c_int * 3)(*(list(self.S) + [1] * (3 - self.nd)))
        with torch.cuda.device(self.device):
            _lib.check(self.lib.mrb_plan_create(ct.byref(h), self.nd, arr, self.C, self.B, self.K, int(W),
                                                float(osf), 1 if ortho else 0), "plan_create")
        self.h = h
        self.G = tuple(int(math.ceil(osf * s)) for s in self.S)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                self.lib.mrb_plan_destroy(h)
            except Exception:
                pass
            self.h = None

    def set_option(self, key: int, value: int) -> None:
        _lib.check(self.lib.mrb_plan_set_option(self.h, int(key), int(value)), "plan_set_option")

    def set_points(self, traj: torch.Tensor) -> None:
        _lib.require_cuda(traj, "traj")
        traj = traj.to(torch.float32).contiguous()
        if tuple(traj.shape) != (self.B, self.nd, self.K):
            raise ValueError(f"traj must be {(self.B, self.nd, self.K)}, got {tuple(traj.shape)}")
        with torch.cuda.device(self.device):
            _lib.check(self.lib.mrb_plan_set_points(self.h, _lib.ptr(traj), _lib.stream_ptr()), "plan_set_points")
        self._traj = traj

    def set_dcf(self, dcf: Optional[torch.Tensor], mode: str, apply_fwd: bool, apply_adj: bool) -> None:
        if dcf is not None:
            _lib.require_cuda(dcf, "dcf")
            dcf = dcf.to(torch.float32).contiguous()
            if tuple(dcf.shape) != (self.B, self.K):
                raise ValueError(f"dcf must be {(self.B, self.K)}")
        with torch.cuda.device(self.device):
            _lib.check(self.lib.mrb_plan_set_dcf(self.h, _lib.ptr(dcf), _DCF_MODES[mode], int(apply_fwd),
                                                 int(apply_adj), _lib.stream_ptr()), "plan_set_dcf")
        self._dcf = dcf

    def set_maps(self, maps: torch.Tensor) -> None:
        _lib.require_cuda(maps, "maps")
        maps = maps.to(torch.complex64).contiguous()
        if tuple(maps.shape) != (self.C,) + self.S:
            raise ValueError(f"maps must be {(self.C,) + self.S}")
        with torch.cuda.device(self.device):
            _lib.check(self.lib.mrb_plan_set_maps(self.h, _lib.ptr(maps), _lib.stream_ptr()), "plan_set_maps")

    def forward(self, x: torch.Tensor, y: torch.Tensor, nb: int, coil_images: bool = False) -> None:
        fn = self.lib.mrb_nufft_forward_coils if coil_images else self.lib.mrb_nufft_forward
        _lib.check(fn(self.h, _lib.ptr(x), _lib.ptr(y), int(nb), _lib.stream_ptr(x.device)), "nufft_forward")

    def adjoint(self, y: torch.Tensor, x: torch.Tensor, nb: int) -> None:
        _lib.check(self.lib.mrb_nufft_adjoint(self.h, _lib.ptr(y), _lib.ptr(x), int(nb), _lib.stream_ptr(y.device)),
                   "nufft_adjoint")

    STAGES = {"pre": 0, "fft": 1, "interp": 2, "spread": 3, "ifft": 4, "post": 5}

    def stage(self, name: str, x: Optional[torch.Tensor], y: Optional[torch.Tensor], nb: int) -> None:
        """Run one stage of the operators on the plan's grid (timing / tuning)."""
        _lib.check(self.lib.mrb_nufft_stage(self.h, self.STAGES[name], _lib.ptr(x), _lib.ptr(y), int(nb),
                                            _lib.stream_ptr(self.device)), "nufft_stage")

    def set_toeplitz(self, psf: torch.Tensor) -> None:
        """Transfer function (B, G0, G1) float32 of the Toeplitz normal operator (copied)."""
        _lib.require_cuda(psf, "psf")
        if psf.dtype != torch.float32 or not psf.is_contiguous():
            raise ValueError("psf must be contiguous float32")
        _lib.check(self.lib.mrb_plan_set_toeplitz(self.h, _lib.ptr(psf), _lib.stream_ptr(self.device)),
                   "plan_set_toeplitz")

    def normal(self, x: torch.Tensor, out: torch.Tensor, nb: int) -> None:
        """out = A^H A x through the Toeplitz transfer function (no gridding)."""
        _lib.check(self.lib.mrb_nufft_normal(self.h, _lib.ptr(x), _lib.ptr(out), int(nb),
                                             _lib.stream_ptr(self.device)), "nufft_normal")

    def set_skip_flag(self, ptr: Optional[int]) -> None:
        """Device address of a double that, when non-zero, makes the operator
        kernels launched from now on return at once (None clears it)."""
        _lib.check(self.lib.mrb_plan_set_skip_flag(self.h, ptr), "plan_set_skip_flag")

    def info(self) -> dict:
        out = (ct.c_int64 * 10)()
        _lib.check(self.lib.mrb_plan_info(self.h, out, 10), "plan_info")
        keys = ("entries", "tiles_per_frame", "touched_cells", "tile", "coils_per_item", "grid_cells", "fft_mode",
                "block_spread", "col_interp", "points_ready")
        return {k: int(v) for k, v in zip(keys, out)}

    def cell_base(self) -> torch.Tensor:
        out = torch.empty((self.B, self.nd, self.K), dtype=torch.int32, device=self.device)
        _lib.check(self.lib.mrb_plan_cell_base(self.h, _lib.ptr(out), _lib.stream_ptr(self.device)), "cell_base")
        return out


def grid_indices(traj_nd_k: torch.Tensor, G: Sequence[int], W: int = 4, convention: str = "reference") -> torch.Tensor:
    """(K, W^nd) int64 grid index table for one frame, computed on the GPU.

    convention 'reference' reproduces graspcg/nufft/backends/ptnufft.py:151-195
    bit for bit; 'corrected' is the integer-node row-major table of the operators.
    """
    lib = _lib.load()
    _lib.require_cuda(traj_nd_k, "traj")
    t = traj_nd_k.to(torch.float32).contiguous()
    nd, K = int(t.shape[0]), int(t.shape[1])
    out = torch.empty((K, W ** nd), dtype=torch.int64, device=t.device)
    arr = (ct.c_int * 3)(*(list(G) + [1] * (3 - nd)))
    conv = {"reference": 0, "corrected": 1}[convention]
    _lib.check(lib.mrb_grid_indices(_lib.ptr(t), nd, arr, K, int(W), conv, _lib.ptr(out),
                                    _lib.stream_ptr(t.device)), "grid_indices")
    return out


def _to_BndK(traj: torch.Tensor, ndim: int) -> torch.Tensor:
    """Normalise to (B, nd, K) (graspcg/nufft/backends/torchkb.py:65-85)."""
    if traj.ndim == 2:
        t = traj
        if int(t.shape[0]) != ndim and int(t.shape[1]) == ndim:
            t = t.transpose(0, 1).contiguous()
        if int(t.shape[0]) != ndim:
            raise ValueError(f"traj has wrong nd; expected {ndim}")
        return t.unsqueeze(0)
    if traj.ndim == 3:
        if int(traj.shape[1]) == ndim:
            return traj
        if int(traj.shape[2]) == ndim:
            return traj.transpose(1, 2).contiguous()
        raise ValueError("traj must be (B,nd,K) or (B,K,nd)")
    raise ValueError("traj must have 2 or 3 dims")


@dataclass
class B200NUFFTAdapter:
    """Drop-in NUFFT backend adapter (torchkb adapter surface) on the B200 kernels."""

    ndim: int
    backend_name: str = "b200"
    traj_units: Literal["rad", "norm"] = "rad"
    dcf_mode: Literal["balanced", "standard", "none"] = "balanced"
    apply_dcf_in_fwd: bool = False
    apply_dcf_in_adj: bool = True
    kwidth: int = 4
    osf: float = 2.0
    norm: Literal["ortho", "none"] = "ortho"
    tile: Optional[int] = None
    coils_per_item: Optional[int] = None
    chunk: Optional[int] = None
    fft_mode: Optional[int] = None
    interleave: Optional[int] = None   # interp on a coil-interleaved grid (default 1; 2D: fused FFT mode)
    spread_kernel: Optional[int] = None  # 1 block per tile (default), 0 warp per tile and coil group
    col_interp: Optional[int] = None     # 2D fused mode: interp inside the forward column pass (default 0)
    autotune: bool = False
    tuned: Optional[dict] = None

    _im_shape: Optional[Tuple[int, ...]] = None
    _maps: Optional[torch.Tensor] = None
    _traj_BndK: Optional[torch.Tensor] = None
    _dcf_BK: Optional[torch.Tensor] = None
    _K: int = 0
    _dev: Optional[torch.device] = None
    _dtype: torch.dtype = torch.complex64
    _plan: Optional[KBPlan] = None
    _alpha_scalar: Optional[float] = None

    # -- prepare ---------------------------------------------------------------
    def scale_traj(self, traj: torch.Tensor) -> torch.Tensor:
        t = _to_BndK(traj, self.ndim).to(torch.float32)
        if self.traj_units == "rad":
            return t
        if self.traj_units == "norm":
            return (2.0 * math.pi) * t
        raise ValueError("traj_units must be 'rad' or 'norm'")

    def prepare(self, im_shape, traj, dcf, maps, dtype, device, like_prod: int = 1) -> None:
        if self.ndim not in (2, 3):
            raise ValueError("B200NUFFTAdapter supports ndim in {2,3}")
        device = torch.device(device)
        if device.type != "cuda":
            raise RuntimeError("B200NUFFTAdapter runs on CUDA devices only (no CPU fallback)")
        if dtype != torch.complex64:
            raise ValueError("B200NUFFTAdapter computes in complex64 (FP32 gridding and FFT)")
        self._im_shape = tuple(int(s) for s in im_shape)
        C = self._im_shape[0]
        S = self._im_shape[1:]
        if len(S) != self.ndim:
            raise ValueError(f"im_shape {im_shape} does not match ndim={self.ndim}")
        self._dev, self._dtype = device, dtype
        self._maps = maps.to(device=device, dtype=dtype).contiguous()
        self._traj_BndK = self.scale_traj(traj).to(device).contiguous()
        B, _, K = (int(s) for s in self._traj_BndK.shape)
        self._K = K
        if dcf is None:
            self._dcf_BK = None
        else:
            d = dcf
            if d.ndim == 1:
                d = d.view(1, -1)
            if d.ndim != 2:
                raise ValueError("dcf must be (B,K) or (K)")
            d = d.to(device=device, dtype=torch.float32).contiguous()
            if int(d.shape[-1]) != K:
                raise ValueError("dcf must have K samples")
            if int(d.shape[0]) == 1 and B > 1:
                d = d.expand(B, -1).contiguous()
            if int(d.shape[0]) != B:
                raise ValueError(f"dcf batch {int(d.shape[0])} does not match trajectory batch {B}")
            self._dcf_BK = d
        with torch.cuda.device(device):
            plan = KBPlan(S, C, B, K, W=self.kwidth, osf=self.osf, ortho=(self.norm == "ortho"), device=device)
            if self.tile is not None:
                plan.set_option(OPT_TILE, self.tile)
            if self.coils_per_item is not None:
                plan.set_option(OPT_COILS_PER_ITEM, self.coils_per_item)
            if self.chunk is not None:
                plan.set_option(OPT_CHUNK, self.chunk)
            if self.fft_mode is not None:
                plan.set_option(OPT_FFT_MODE, self.fft_mode)
            if self.interleave is not None:
                plan.set_option(OPT_INTERLEAVE, self.interleave)
            if self.spread_kernel is not None:
                plan.set_option(OPT_SPREAD_KERNEL, self.spread_kernel)
            if self.col_interp is not None:
                plan.set_option(OPT_COL_INTERP, self.col_interp)
            plan.set_points(self._traj_BndK)
            plan.set_dcf(self._dcf_BK, self.dcf_mode, self.apply_dcf_in_fwd, self.apply_dcf_in_adj)
            plan.set_maps(self._maps)
            if self.autotune:
                from .autotune import tune
                self.tuned = tune(plan, self._traj_BndK)
        self._plan = plan
        self._alpha_scalar = None

    def k_per_frame(self) -> int:
        return int(self._K)

    # -- Toeplitz normal operator ----------------------------------------------
    @torch.no_grad()
    def prepare_toeplitz(self, psf: str = "exact") -> torch.Tensor:
        """Compute and install the Toeplitz transfer function of A^H A.

        t_b(D) = sum_k w_k exp(i w_k . D) (w = forward x adjoint DCF weights) on
        the lags D = i - G/2 of a G0 x G1 image.  psf="exact": the exponential
        separates, t_b = E0^T diag(w) E1 with E_d[k, i] = exp(i w_dk (i - G_d/2)),
        one FP64 matrix product per frame (exact to rounding, so the Toeplitz
        A^H A is the NUDFT normal operator and positive semi-definite);
        psf="kb": the adjoint NUFFT of w onto the G0 x G1 image (a second,
        unnormalised plan, its own KB gridding).  Placed circularly (lag -G/2 set
        to zero, never used by the linear convolution of an S image), its FFT is
        real.  Scaled by s^2 / (G0 G1) (s the ortho factor) and rolled by G/2 for
        the row passes' (-1)^n signs.  Needs a 2D plan in the fused FFT mode with
        G >= 2 S - 1 (osf >= 2).  Returns the transfer function."""
        if self.ndim != 2:
            raise ValueError("the Toeplitz normal operator is 2D")
        plan = self._plan
        if plan.info()["fft_mode"] != FFT_FUSED:
            raise RuntimeError("the Toeplitz normal operator needs the fused FFT mode")
        S = self._im_shape[1:]
        G = tuple(int(math.ceil(self.osf * s)) for s in S)
        if any(g < 2 * s - 1 for g, s in zip(G, S)):
            raise ValueError("the Toeplitz embedding needs a grid of at least 2S-1 (osf >= 2)")
        B, K = int(self._traj_BndK.shape[0]), int(self._K)
        dev = self._dev
        w = torch.ones((B, K), dtype=torch.float32, device=dev)
        if self._dcf_BK is not None and self.dcf_mode != "none":
            d = self._dcf_BK
            if self.dcf_mode == "balanced":
                w = d.clamp_min(0)
            else:
                w = d ** (int(self.apply_dcf_in_fwd) + int(self.apply_dcf_in_adj))
        if psf == "exact":
            t = torch.empty((B,) + G, dtype=torch.complex128, device=dev)
            lag = [torch.arange(g, dtype=torch.float64, device=dev) - g // 2 for g in G]
            for b in range(B):
                om = self._traj_BndK[b].to(torch.float64)                      # (2, K)
                e0 = torch.polar(torch.ones(1, dtype=torch.float64, device=dev), om[0][:, None] * lag[0][None, :])
                e1 = torch.polar(torch.ones(1, dtype=torch.float64, device=dev), om[1][:, None] * lag[1][None, :])
                t[b] = e0.transpose(0, 1) @ (w[b].to(torch.float64)[:, None] * e1)
        elif psf == "kb":
            psf_op = B200NUFFTAdapter(ndim=2, dcf_mode="none", kwidth=self.kwidth, osf=self.osf, norm="none")
            psf_op.prepare((1,) + G, self._traj_BndK, None, torch.ones((1,) + G, dtype=torch.complex64, device=dev),
                           torch.complex64, dev)
            t = psf_op.AH(w.to(torch.complex64).reshape(B, 1, K)).reshape(B, *G)
            del psf_op
        else:
            raise ValueError("psf must be 'exact' or 'kb'")
        c = torch.roll(t, shifts=(G[0] // 2, G[1] // 2), dims=(1, 2))
        c[:, G[0] // 2, :] = 0
        c[:, :, G[1] // 2] = 0
        P = torch.fft.fft2(c.to(torch.complex128)).real
        s2 = 1.0 / (G[0] * G[1]) if self.norm == "ortho" else 1.0
        P = torch.roll(P * (s2 / (G[0] * G[1])), shifts=(G[0] // 2, G[1] // 2), dims=(1, 2))
        P = P.to(torch.float32).contiguous()
        plan.set_toeplitz(P)
        self._toeplitz = True
        return P

    def AHA(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """A^H A x by the Toeplitz transfer function (prepare_toeplitz first)."""
        if not getattr(self, "_toeplitz", False):
            raise RuntimeError("call prepare_toeplitz() first")
        if x.dtype != torch.complex64 or not x.is_contiguous():
            raise ValueError("x must be contiguous complex64")
        nb = int(x.shape[0])
        if out is None:
            out = torch.empty_like(x)
        self._plan.normal(x, out, nb)
        return out

    # operator conveniences so the adapter can drive the solver directly
    @property
    def roles_image(self) -> Roles:
        return Roles(unlike=1, like=1, nufft=self.ndim)

    @property
    def roles_kspace(self) -> Roles:
        return Roles(unlike=1, like=1, nufft=1)

    def image_shape(self, y: torch.Tensor) -> Tuple[int, ...]:
        return (int(y.shape[0]), 1) + tuple(self._im_shape[1:])

    @property
    def plan(self) -> KBPlan:
        if self._plan is None:
            raise RuntimeError("call prepare() first")
        return self._plan

    def _check_batch(self, Bx: int) -> None:
        B = int(self._traj_BndK.shape[0])
        if not (Bx == B or B == 1 or Bx % B == 0):
            raise ValueError(f"omega batch {B} incompatible with requested {Bx}. "
                             "Prepare with matching B or fold like->batch only when Bx is a multiple of B.")

    # -- operators -----------------------------------------------------------
    @torch.no_grad()
    def A(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        plan = self.plan
        _lib.require_cuda(x, "x")
        C = int(self._im_shape[0])
        S = tuple(self._im_shape[1:])
        K = self._K
        Bx = int(x.shape[0])
        if x.ndim == 2 + self.ndim:
            L, Cin = 1, int(x.shape[1])
            need = (Bx, C, K)
        elif x.ndim == 3 + self.ndim:
            L, Cin = int(x.shape[1]), int(x.shape[2])
            need = (Bx, L, C, K)
        else:
            raise ValueError(f"x must be (B,C,*S) or (B,L,C,*S); got shape {tuple(x.shape)} for ndim={self.ndim}")
        if Cin not in (1, C):
            raise ValueError(f"image coil slot must be 1 or {C}; got {Cin}")
        if tuple(x.shape[-self.ndim:]) != S:
            raise ValueError(f"image spatial shape {tuple(x.shape[-self.ndim:])} does not match maps {S}")
        self._check_batch(Bx)
        if out is not None and tuple(out.shape) != need:
            raise ValueError(f"out has shape {tuple(out.shape)} but expected {need}")
        nb = Bx * L
        xc = x.to(torch.complex64).contiguous()
        direct = out is not None and out.is_contiguous() and out.dtype == torch.complex64
        y = out if direct else torch.empty(need, dtype=torch.complex64, device=x.device)
        plan.forward(xc, y, nb, coil_images=(Cin == C and C > 1))
        if out is not None and not direct:
            out.copy_(y)
            return out
        return y

    @torch.no_grad()
    def AH(self, y: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        plan = self.plan
        _lib.require_cuda(y, "y")
        Cm = int(self._im_shape[0])
        S = tuple(self._im_shape[1:])
        Bx = int(y.shape[0])
        if y.ndim == 3:
            L, C = 1, int(y.shape[1])
            need = (Bx, 1) + S
        elif y.ndim == 4:
            L, C = int(y.shape[1]), int(y.shape[2])
            need = (Bx, L, 1) + S
        else:
            raise ValueError("y must be (B,C,K) or (B,L,C,K)")
        if C != Cm:
            raise ValueError(f"y coil dim {C} must equal maps C {Cm}")
        if int(y.shape[-1]) != self._K:
            raise ValueError(f"y has {int(y.shape[-1])} samples per frame, plan has {self._K}")
        self._check_batch(Bx)
        if out is not None and tuple(out.shape) != need:
            raise ValueError(f"out has shape {tuple(out.shape)} but expected {need}")
        yc = y.to(torch.complex64).contiguous()
        direct = out is not None and out.is_contiguous() and out.dtype == torch.complex64
        x = out if direct else torch.empty(need, dtype=torch.complex64, device=y.device)
        plan.adjoint(yc, x, Bx * L)
        if out is not None and not direct:
            out.copy_(x)
            return out
        return x

    # -- calibration (graspcg/nufft/backends/torchkb.py:328-364) --------------
    @torch.no_grad()
    def diag_AHA_profile(self) -> torch.Tensor:
        B = int(self._traj_BndK.shape[0])
        if self._dcf_BK is None:
            return torch.full((B,), float(self._K), device=self._dev, dtype=torch.float32)
        return self._dcf_BK.sum(dim=1).to(torch.float32)

    @torch.no_grad()
    def diag_AHA_scalar(self) -> float:
        if self._alpha_scalar is not None:
            return float(self._alpha_scalar)
        S = tuple(self._im_shape[1:])
        ctr = tuple(s // 2 for s in S)
        B = int(self._traj_BndK.shape[0])
        x0 = torch.zeros((B, 1) + S, device=self._dev, dtype=self._dtype)
        x0[(0, 0) + ctr] = 1.0
        z = self.AH(self.A(x0))
        zc = float(z[(0, 0) + ctr].real.item())
        sos = float((self._maps.abs() ** 2).sum(dim=0)[ctr].clamp_min(1e-20).item())
        self._alpha_scalar = zc / sos
        return self._alpha_scalar


@dataclass(frozen=True)
class NUFFTConfig:
    """Front-end configuration (graspcg/nufft/api.py:30-47) for the B200 backend."""
    ndim: Literal[2, 3]
    backend: Literal["b200"] = "b200"
    traj_units: Literal["norm", "rad"] = "norm"
    dcf_mode: Literal["standard", "balanced", "none"] = "balanced"
    apply_dcf_in_fwd: bool = False
    apply_dcf_in_adj: bool = True
    kwidth: int = 4
    osf: float = 2.0
    norm: Literal["ortho", "none"] = "ortho"
    autotune: bool = False


class NUFFT:
    """Axis-labelled NUFFT front-end (graspcg/nufft/api.py:52-376), B200 backend."""

    def __init__(self, maps: torch.Tensor, traj: torch.Tensor, dcf: Optional[torch.Tensor], *, axis: AxisSpec,
                 config: NUFFTConfig, dtype: torch.dtype = torch.complex64, device: Optional[torch.device] = None):
        if maps.ndim not in (3, 4):
            raise ValueError("maps must be (C,X,Y) or (C,X,Y,Z)")
        ndim = 2 if maps.ndim == 3 else 3
        if config.ndim != ndim:
            raise ValueError(f"config.ndim={config.ndim} must match maps dimensionality {ndim}")
        if config.backend != "b200":
            raise ValueError("backend must be 'b200'")
        self.maps, self.traj0, self.dcf0 = maps, traj, dcf
        self.axis, self.cfg, self.dtype = axis, config, dtype
        self.device = torch.device(device) if device is not None else maps.device
        self._traj_BndK = _to_BndK(traj, ndim).to(self.device, dtype=torch.float32).contiguous()
        if dcf is None:
            self._dcf_BK = None
        else:
            d = dcf.view(1, -1) if dcf.ndim == 1 else dcf
            if d.ndim != 2:
                raise ValueError("dcf must be (B,K) or (K)")
            self._dcf_BK = d.to(self.device, dtype=torch.float32).contiguous()
        be = B200NUFFTAdapter(ndim=ndim, traj_units=config.traj_units, dcf_mode=config.dcf_mode,
                              apply_dcf_in_fwd=config.apply_dcf_in_fwd, apply_dcf_in_adj=config.apply_dcf_in_adj,
                              kwidth=config.kwidth, osf=config.osf, norm=config.norm, autotune=config.autotune)
        self._backend = be
        im_shape = (int(maps.shape[0]),) + tuple(int(s) for s in maps.shape[1:])
        be.prepare(im_shape, self._traj_BndK, self._dcf_BK, maps.to(self.device, dtype=dtype).contiguous(),
                   dtype=dtype, device=self.device, like_prod=int(maps.shape[0]))
        like_img = tuple(l for l in axis.image if l not in axis.image_fft and l not in ("B", axis.coil))
        like_ks = tuple(l for l in axis.kspace if l not in axis.kspace_fft and l not in ("B", axis.coil))
        coil_slot = 1 if axis.coil in axis.image else 0
        self.roles_image = Roles(unlike=1, like=len(like_img) + coil_slot, nufft=len(axis.image_fft))
        self.roles_kspace = Roles(unlike=1, like=len(like_ks), nufft=1)

    @property
    def backend(self) -> B200NUFFTAdapter:
        return self._backend

    def k_per_frame(self) -> int:
        return self._backend.k_per_frame()

    def image_shape(self, y_user: torch.Tensor) -> Tuple[int, ...]:
        B = int(self._traj_BndK.shape[0])
        return (B, 1) + tuple(int(s) for s in self.maps.shape[1:])

    def domain_shape(self) -> Tuple[int, ...]:
        return (1, 1) + tuple(int(s) for s in self.maps.shape[1:])

    def _kspace_view(self, y_user, B, L_sizes, C, K):
        plan = plan_kspace_layout_from_sizes(B, L_sizes, C, K, self.axis)
        dims = ("B",) + tuple(plan.like_labels) + (self.axis.coil, self.axis.kspace_fft[0])
        mp = {l: i for i, l in enumerate(self.axis.kspace)}
        return y_user.permute(*[mp[l] for l in dims]).reshape(B * max(1, plan.L_other), C, K)

    def _image_view(self, x_user, img_plan):
        dims = ["B"] + list(img_plan.like_labels) + [self.axis.coil] + list(self.axis.image_fft)
        mp = {l: i for i, l in enumerate(self.axis.image)}
        perm = [mp[l] for l in dims if l in mp]
        xp = x_user.permute(*perm)
        return xp.reshape(int(img_plan.B) * max(1, int(img_plan.L_other)), 1, *img_plan.spatial)

    @torch.no_grad()
    def A(self, x_user: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        ip = plan_image_layout(x_user, self.axis)
        C, K = int(self.maps.shape[0]), self.k_per_frame()
        shape = user_kspace_shape(self.axis, ip.B, ip.like_sizes, C, K)
        if out is None:
            y_user = torch.empty(shape, device=self.device, dtype=x_user.dtype)
        else:
            if tuple(out.shape) != tuple(shape):
                raise ValueError(f"out has shape {tuple(out.shape)} but expected {tuple(shape)}")
            y_user = out
        y_view = self._kspace_view(y_user, ip.B, ip.like_sizes, C, K)
        x_view = self._image_view(x_user, ip)
        res = self._backend.A(x_view, out=y_view)
        if res.data_ptr() != y_view.data_ptr() or not _same_view(res, y_view):
            y_view.copy_(res)
        return y_user

    @torch.no_grad()
    def AH(self, y_user: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        kp = plan_kspace_layout(y_user, self.axis)
        spatial = tuple(int(s) for s in self.maps.shape[1:])
        C = int(self.maps.shape[0])
        shape = user_image_shape(self.axis, kp.B, kp.like_sizes, spatial)
        if out is None:
            x_user = torch.empty(shape, device=self.device, dtype=y_user.dtype)
        else:
            if tuple(out.shape) != tuple(shape):
                raise ValueError(f"out has shape {tuple(out.shape)} but expected {tuple(shape)}")
            x_user = out
        y_view = self._kspace_view(y_user, kp.B, kp.like_sizes, C, kp.K)
        ip = plan_image_layout_from_sizes(kp.B, kp.like_sizes, spatial, self.axis)
        x_view = self._image_view(x_user, ip)
        res = self._backend.AH(y_view, out=x_view)
        if res.data_ptr() != x_view.data_ptr() or not _same_view(res, x_view):
            x_view.copy_(res)
        return x_user


def _same_view(a: torch.Tensor, b: torch.Tensor) -> bool:
    return a.shape == b.shape and a.stride() == b.stride() and a.data_ptr() == b.data_ptr()


NSNUFFT = NUFFT
