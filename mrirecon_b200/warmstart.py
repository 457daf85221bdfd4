"""Learned warm start for GRASP-style NCG: a BF16 2D+t residual CNN.

The network (3 levels, 32 base channels, 3x3x3 convolutions over (t, y, x),
U-Net skips, output = input + net(input)) maps a normalised adjoint
reconstruction -- the density-compensated adjoint A^H(w y) with the radial
ramp w ~ |k| (``ramp_adjoint``), whose point-spread function is far narrower
than that of A^H y -- to an estimate of the converged NCG reconstruction.  It is
trained on pairs (adjoint recon -> converged NCG recon) that the solver of
this package generates on seeded synthetic phantoms, with the project's own
CUDA kernels (``csrc/cnn.cu``): BF16 tensor-core implicit-GEMM convolution
forward / data gradient / weight gradient, FP32 accumulation and FP32 master
weights updated by Adam.  NCG always runs after it to the same objective
tolerance, and it is only used when its objective is below the adjoint
start's (``warm_start``).  The reference has no learned component.

Layers (kernel channel counts; the input is padded to 32 channels, the last
layer's 2 outputs to 32):
  c1 2->32, c2 32->32 = B1; pool; c3 32->64, c4 64->64 = B2; pool; c5 64->128;
  up; c6 [up(c5), B2] 192->64; up; c7 [up(c6), B1] 96->32; c8 32->2.
"""
from __future__ import annotations

import ctypes as ct
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import _lib

# name, kernel cin (padded), real cin, coutp (padded), real cout, relu
LAYERS: List[Tuple[str, int, int, int, int, bool]] = [
    ("c1", 32, 2, 32, 32, True), ("c2", 32, 32, 32, 32, True), ("c3", 32, 32, 64, 64, True),
    ("c4", 64, 64, 64, 64, True), ("c5", 64, 64, 128, 128, True), ("c6", 192, 192, 64, 64, True),
    ("c7", 96, 96, 32, 32, True), ("c8", 32, 32, 32, 2, False)]
XC = 32          # channels of the packed input tensor

# Weights trained for the GRASP acquisition (256^2, 12 coils, 21 golden-angle
# spokes x 512 samples per frame) by
#   python -m mrirecon_b200.warmstart --out mrirecon_b200/weights/warmstart_grasp256.npz \
#       --series 2000 --per-solve 25 --epochs 12
# (2,000 seeded 8-frame series, pairs from this package's NCG, ~13 GPU-minutes on one B200).
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warmstart_grasp256.npz")

_SIGS = {
    "mrb_cnn_conv3d_fwd": [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p,
                           ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_int,
                           ct.c_void_p, ct.c_void_p],
    "mrb_cnn_conv3d_wgrad": [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_int,
                             ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p],
    "mrb_cnn_flip_weights": [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p],
    "mrb_cnn_relu_bwd": [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int64,
                         ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p],
    "mrb_cnn_pool2": [ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int,
                      ct.c_int, ct.c_void_p],
    "mrb_cnn_up2": [ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int,
                    ct.c_void_p],
    "mrb_cnn_pack": [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p],
    "mrb_cnn_unpack": [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p],
    "mrb_cnn_mse": [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                    ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_void_p],
    "mrb_cnn_adam": [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_float, ct.c_float,
                     ct.c_float, ct.c_float, ct.c_int, ct.c_void_p, ct.c_void_p],
    "mrb_cnn_to_bf16": [ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p],
    "mrb_cnn_tc_supported": [ct.c_int] * 6,
    "mrb_cnn_conv3d_tc": [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_int,
                          ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int,
                          ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p],
    "mrb_cnn_tc_error": [ct.c_void_p],
    "mrb_cnn_wgrad_tc_scratch_bytes": [ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p],
    "mrb_cnn_conv3d_wgrad_tc": [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int,
                                ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_void_p,
                                ct.c_void_p],
}


def _lib_cnn():
    lib = _lib.load()
    if not getattr(lib, "_cnn_sigs", False):
        for n, args in _SIGS.items():
            f = getattr(lib, n)
            f.restype = ct.c_int
            f.argtypes = args
        lib._cnn_sigs = True
    return lib


def _p(t):
    return _lib.ptr(t)


def _vol(Nb, D, H, W):
    return (ct.c_int * 4)(Nb, D, H, W)


class WarmStartCNN:
    """Weights, Adam state and activation buffers of the warm-start network."""

    def __init__(self, device="cuda", seed: int = 0):
        self.device = torch.device(device)
        self.lib = _lib_cnn()
        g = torch.Generator().manual_seed(seed)
        self.w32: Dict[str, torch.Tensor] = {}
        self.b32: Dict[str, torch.Tensor] = {}
        for name, cinp, cin, coutp, cout, relu in LAYERS:
            w = torch.zeros((27, cinp, coutp), dtype=torch.float32)
            std = math.sqrt(2.0 / (27 * cin)) * (0.1 if name == "c8" else 1.0)
            w[:, :cin, :cout] = torch.randn((27, cin, cout), generator=g) * std
            self.w32[name] = w.to(self.device)
            self.b32[name] = torch.zeros(coutp, dtype=torch.float32, device=self.device)
        self.step = 0
        self.m = {k: torch.zeros_like(v) for k, v in self._params()}
        self.v = {k: torch.zeros_like(v) for k, v in self._params()}
        self._bufs: Dict[tuple, dict] = {}
        # convolutions run on tcgen05 (tensor memory) where the shape allows,
        # on the warp-level mma.sync kernel otherwise
        self.use_tc = True
        # weight gradients on tcgen05 too (mrb_cnn_conv3d_wgrad_tc) where the shape allows
        self.use_tc_wgrad = True
        self.refresh()

    # -------------------------------------------------------------- parameters
    def _params(self):
        for name, *_ in LAYERS:
            yield "w:" + name, self.w32[name]
            yield "b:" + name, self.b32[name]

    def refresh(self):
        """BF16 weights for the forward pass, their K-major copy for the tensor-core
        convolution and flipped BF16 weights for the data gradient."""
        st = _lib.stream_ptr(self.device)
        self.wb, self.wd, self.wk = {}, {}, {}
        for name, cinp, cin, coutp, cout, relu in LAYERS:
            wb = torch.empty((27, cinp, coutp), dtype=torch.bfloat16, device=self.device)
            _lib.check(self.lib.mrb_cnn_to_bf16(_p(self.w32[name]), wb.numel(), _p(wb), st), "to_bf16")
            self.wb[name] = wb
            self.wk[name] = wb.permute(0, 2, 1).contiguous()
            wd = torch.empty((27, coutp, cinp), dtype=torch.bfloat16, device=self.device)
            _lib.check(self.lib.mrb_cnn_flip_weights(_p(wb), cinp, coutp, _p(wd), cinp, st), "flip")
            self.wd[name] = wd

    def state_dict(self):
        return {k: v.detach().cpu().numpy() for k, v in self._params()}

    def load_state_dict(self, d):
        for name, *_ in LAYERS:
            self.w32[name].copy_(torch.as_tensor(np.asarray(d["w:" + name])))
            self.b32[name].copy_(torch.as_tensor(np.asarray(d["b:" + name])))
        self.refresh()

    def save(self, path):
        np.savez_compressed(path, **self.state_dict())

    def load(self, path):
        self.load_state_dict(np.load(path))
        return self

    @classmethod
    def pretrained(cls, device="cuda", path: str = DEFAULT_WEIGHTS) -> "WarmStartCNN":
        """The network with the packaged GRASP weights."""
        return cls(device).load(path)

    # ------------------------------------------------------------------ buffers
    def _buffers(self, Nb, D, H, W, train: bool):
        key = (Nb, D, H, W, train)
        b = self._bufs.get(key)
        if b is not None:
            return b
        if H % 4 or W % 4:
            raise ValueError("the warm-start network needs H and W divisible by 4")
        dev = self.device
        bf = lambda *s: torch.zeros(s, dtype=torch.bfloat16, device=dev)
        f32 = lambda *s: torch.zeros(s, dtype=torch.float32, device=dev)
        V1, V2, V3 = Nb * D * H * W, Nb * D * (H // 2) * (W // 2), Nb * D * (H // 4) * (W // 4)
        b = dict(X0=bf(V1, XC), A1=bf(V1, 32), CAT1=bf(V1, 96), P1=bf(V2, 32), A2=bf(V2, 64), CAT2=bf(V2, 192),
                 P2=bf(V3, 64), A3=bf(V3, 128), C2=bf(V2, 64), C1=bf(V1, 32), O=f32(V1, 32),
                 scale=f32(Nb), loss=torch.zeros(1, dtype=torch.float64, device=dev))
        if train:
            b.update(gO=f32(V1, 32), gC1=f32(V1, 32), gCAT1=f32(V1, 96), gC2=f32(V2, 64), gCAT2=f32(V2, 192),
                     gA3=f32(V3, 128), gP2=f32(V3, 64), gA2=f32(V2, 64), gP1=f32(V2, 32), gA1=f32(V1, 32),
                     gz32=bf(V1, 32), gz64=bf(V2, 64), gz128=bf(V3, 128), gz32h=bf(V2, 32),
                     lpart=torch.zeros((V1 + 255) // 256, dtype=torch.float64, device=dev))
            self.dw = {n: torch.zeros_like(self.w32[n]) for n, *_ in LAYERS}
            self.db = {n: torch.zeros_like(self.b32[n]) for n, *_ in LAYERS}
            wmax = max(27 * cinp * coutp for _, cinp, _, coutp, _, _ in LAYERS)
            b["wpart"] = torch.zeros(wmax * 64, dtype=torch.float32, device=dev)
        self._bufs[key] = b
        return b

    # ----------------------------------------------------------------- forward
    def _conv(self, name, x, cx, xoff, vol, yb=None, cyb=0, ybo=0, yf=None, cyf=0, yfo=0, acc=0, weights=None,
              cin=None, coutp=None, cout=None, relu=None, bias=True, dgrad=False):
        _, cinp, _, coutp_l, cout_l, relu_l = next(l for l in LAYERS if l[0] == name)
        k = cinp if cin is None else cin
        n = coutp_l if coutp is None else coutp
        co = cout_l if cout is None else cout
        Nb, D, H, W = (int(v) for v in vol)
        if self.use_tc and self.lib.mrb_cnn_tc_supported(k, xoff, cx, n, W, H) and (yb is None or (cyb % 8 == 0 and ybo % 8 == 0)):
            # K-major weights: forward [27][N = cout][K = cin]; data gradient: the
            # forward weights [27][cin][cout] read as [27][N = cin][K = cout], taps flipped
            wk = self.wb[name] if dgrad else self.wk[name]
            _lib.check(self.lib.mrb_cnn_conv3d_tc(
                _p(x), cx, xoff, k, _p(wk), 1 if dgrad else 0, n, co, _p(self.b32[name]) if bias else None,
                int(relu_l if relu is None else relu), _p(yb), cyb, ybo, _p(yf), cyf, yfo, acc, Nb, D, H, W,
                _lib.stream_ptr(self.device)), f"conv {name}")
            return
        w = self.wb[name] if weights is None else weights
        _lib.check(self.lib.mrb_cnn_conv3d_fwd(
            _p(x), cx, xoff, cinp if cin is None else cin, _p(w), coutp_l if coutp is None else coutp,
            cout_l if cout is None else cout, _p(self.b32[name]) if bias else None,
            int(relu_l if relu is None else relu), _p(yb), cyb, ybo, _p(yf), cyf, yfo, acc, vol,
            _lib.stream_ptr(self.device)), f"conv {name}")

    def forward(self, z: torch.Tensor, train: bool = False) -> dict:
        """z (Nb, D, H, W) complex64 (normalised by the per-series scale) -> buffers with O."""
        Nb, D, H, W = (int(s) for s in z.shape)
        b = self._buffers(Nb, D, H, W, train)
        st = _lib.stream_ptr(self.device)
        L = self.lib
        v1, v2, v3 = _vol(Nb, D, H, W), _vol(Nb, D, H // 2, W // 2), _vol(Nb, D, H // 4, W // 4)
        _lib.check(L.mrb_cnn_pack(_p(z), _p(b["scale"]), v1, _p(b["X0"]), XC, st), "pack")
        self._conv("c1", b["X0"], XC, 0, v1, yb=b["A1"], cyb=32)
        self._conv("c2", b["A1"], 32, 0, v1, yb=b["CAT1"], cyb=96, ybo=64)
        _lib.check(L.mrb_cnn_pool2(0, _p(b["CAT1"]), 96, 64, 32, v1, _p(b["P1"]), 32, 0, st), "pool1")
        self._conv("c3", b["P1"], 32, 0, v2, yb=b["A2"], cyb=64)
        self._conv("c4", b["A2"], 64, 0, v2, yb=b["CAT2"], cyb=192, ybo=128)
        _lib.check(L.mrb_cnn_pool2(0, _p(b["CAT2"]), 192, 128, 64, v2, _p(b["P2"]), 64, 0, st), "pool2")
        self._conv("c5", b["P2"], 64, 0, v3, yb=b["A3"], cyb=128)
        _lib.check(L.mrb_cnn_up2(0, _p(b["A3"]), 128, 0, 128, v3, _p(b["CAT2"]), 192, 0, st), "up2")
        self._conv("c6", b["CAT2"], 192, 0, v2, yb=b["C2"], cyb=64)
        _lib.check(L.mrb_cnn_up2(0, _p(b["C2"]), 64, 0, 64, v2, _p(b["CAT1"]), 96, 0, st), "up1")
        self._conv("c7", b["CAT1"], 96, 0, v1, yb=b["C1"], cyb=32)
        self._conv("c8", b["C1"], 32, 0, v1, yf=b["O"], cyf=32)
        b["vols"] = (v1, v2, v3)
        b["shape"] = (Nb, D, H, W)
        return b

    def set_scale(self, z: torch.Tensor) -> torch.Tensor:
        """Per-series scale 1 / max|z| (written into the buffers used by forward)."""
        Nb, D, H, W = (int(s) for s in z.shape)
        s = 1.0 / z.reshape(Nb, -1).abs().amax(dim=1).clamp_min(1e-20)
        for train in (False, True):
            key = (Nb, D, H, W, train)
            if key in self._bufs:
                self._bufs[key]["scale"].copy_(s)
        return s

    @torch.no_grad()
    def infer(self, z: torch.Tensor) -> torch.Tensor:
        """Warm start for adjoint reconstructions z (Nb, D, H, W) complex64."""
        z = z.to(torch.complex64).contiguous()
        b = self._buffers(*(int(s) for s in z.shape), False)
        self.set_scale(z)
        self.forward(z, False)
        out = torch.empty_like(z)
        _lib.check(self.lib.mrb_cnn_unpack(_p(z), _p(b["O"]), 32, _p(b["scale"]), b["vols"][0], _p(out),
                                           _lib.stream_ptr(self.device)), "unpack")
        return out

    # ---------------------------------------------------------------- training
    def _wgrad(self, name, x, cx, xoff, gz, cg, goff, vol, b):
        _, cinp, _, coutp, _, _ = next(l for l in LAYERS if l[0] == name)
        if self.use_tc and self.use_tc_wgrad:
            # tcgen05 weight gradient where the shape allows (scratch shared by all
            # layers of a batch shape, sized for the largest)
            nbytes = ct.c_int64(0)
            if self.lib.mrb_cnn_wgrad_tc_scratch_bytes(cinp, coutp, vol, ct.byref(nbytes)) == 0:
                sc = b.get("wtc")
                if sc is None or sc.numel() < nbytes.value:
                    sc = b["wtc"] = torch.empty(nbytes.value, dtype=torch.uint8, device=self.device)
                _lib.check(self.lib.mrb_cnn_conv3d_wgrad_tc(_p(x), cx, xoff, cinp, _p(gz), cg, goff, coutp,
                                                            _p(self.dw[name]), _p(self.db[name]), _p(sc), sc.numel(),
                                                            vol, _lib.stream_ptr(self.device)), f"wgrad tc {name}")
                return
        _lib.check(self.lib.mrb_cnn_conv3d_wgrad(_p(x), cx, xoff, cinp, _p(gz), cg, goff, coutp, _p(self.dw[name]),
                                                 _p(self.db[name]), _p(b["wpart"]), b["wpart"].numel(), vol,
                                                 _lib.stream_ptr(self.device)), f"wgrad {name}")

    def _dgrad(self, name, gz, cg, vol, gout, cgo, goff, acc=0):
        _, cinp, _, coutp, _, _ = next(l for l in LAYERS if l[0] == name)
        self._conv(name, gz, cg, 0, vol, yf=gout, cyf=cgo, yfo=goff, acc=acc, weights=self.wd[name],
                   cin=coutp, coutp=cinp, cout=cinp, relu=False, bias=False, dgrad=True)

    def _relu_bwd(self, g, cgs, goff, act, cas, aoff, nch, V, gz, czs):
        _lib.check(self.lib.mrb_cnn_relu_bwd(_p(g), cgs, goff, _p(act), cas, aoff, nch, V, _p(gz), czs, 0, czs,
                                             _lib.stream_ptr(self.device)), "relu_bwd")

    def loss_and_grad(self, z: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        """Forward + backward on one batch; leaves dW/db in self.dw/self.db; returns the loss (device)."""
        Nb, D, H, W = (int(s) for s in z.shape)
        b = self._buffers(Nb, D, H, W, True)
        self.set_scale(z)
        self.forward(z, True)
        L, st = self.lib, _lib.stream_ptr(self.device)
        v1, v2, v3 = b["vols"]
        V1, V2, V3 = Nb * D * H * W, Nb * D * (H // 2) * (W // 2), Nb * D * (H // 4) * (W // 4)
        _lib.check(L.mrb_cnn_mse(_p(z), _p(target), _p(b["O"]), 32, _p(b["scale"]), v1, _p(b["gO"]), _p(b["loss"]),
                                 _p(b["lpart"]), b["lpart"].numel(), st), "mse")
        # c8 (linear)
        self._relu_bwd(b["gO"], 32, 0, None, 0, 0, 32, V1, b["gz32"], 32)
        self._wgrad("c8", b["C1"], 32, 0, b["gz32"], 32, 0, v1, b)
        self._dgrad("c8", b["gz32"], 32, v1, b["gC1"], 32, 0)
        # c7
        self._relu_bwd(b["gC1"], 32, 0, b["C1"], 32, 0, 32, V1, b["gz32"], 32)
        self._wgrad("c7", b["CAT1"], 96, 0, b["gz32"], 32, 0, v1, b)
        self._dgrad("c7", b["gz32"], 32, v1, b["gCAT1"], 96, 0)
        # up1 -> C2, c6
        _lib.check(L.mrb_cnn_up2(1, _p(b["gCAT1"]), 96, 0, 64, v2, _p(b["gC2"]), 64, 0, st), "up1 bwd")
        self._relu_bwd(b["gC2"], 64, 0, b["C2"], 64, 0, 64, V2, b["gz64"], 64)
        self._wgrad("c6", b["CAT2"], 192, 0, b["gz64"], 64, 0, v2, b)
        self._dgrad("c6", b["gz64"], 64, v2, b["gCAT2"], 192, 0)
        # up2 -> A3, c5
        _lib.check(L.mrb_cnn_up2(1, _p(b["gCAT2"]), 192, 0, 128, v3, _p(b["gA3"]), 128, 0, st), "up2 bwd")
        self._relu_bwd(b["gA3"], 128, 0, b["A3"], 128, 0, 128, V3, b["gz128"], 128)
        self._wgrad("c5", b["P2"], 64, 0, b["gz128"], 128, 0, v3, b)
        self._dgrad("c5", b["gz128"], 128, v3, b["gP2"], 64, 0)
        # pool2 -> B2 (accumulate into the skip gradient), c4
        _lib.check(L.mrb_cnn_pool2(1, _p(b["gP2"]), 64, 0, 64, v2, _p(b["gCAT2"]), 192, 128, st), "pool2 bwd")
        self._relu_bwd(b["gCAT2"], 192, 128, b["CAT2"], 192, 128, 64, V2, b["gz64"], 64)
        self._wgrad("c4", b["A2"], 64, 0, b["gz64"], 64, 0, v2, b)
        self._dgrad("c4", b["gz64"], 64, v2, b["gA2"], 64, 0)
        # c3
        self._relu_bwd(b["gA2"], 64, 0, b["A2"], 64, 0, 64, V2, b["gz64"], 64)
        self._wgrad("c3", b["P1"], 32, 0, b["gz64"], 64, 0, v2, b)
        self._dgrad("c3", b["gz64"], 64, v2, b["gP1"], 32, 0)
        # pool1 -> B1, c2
        _lib.check(L.mrb_cnn_pool2(1, _p(b["gP1"]), 32, 0, 32, v1, _p(b["gCAT1"]), 96, 64, st), "pool1 bwd")
        self._relu_bwd(b["gCAT1"], 96, 64, b["CAT1"], 96, 64, 32, V1, b["gz32"], 32)
        self._wgrad("c2", b["A1"], 32, 0, b["gz32"], 32, 0, v1, b)
        self._dgrad("c2", b["gz32"], 32, v1, b["gA1"], 32, 0)
        # c1
        self._relu_bwd(b["gA1"], 32, 0, b["A1"], 32, 0, 32, V1, b["gz32"], 32)
        self._wgrad("c1", b["X0"], XC, 0, b["gz32"], 32, 0, v1, b)
        return b["loss"]

    def adam_step(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.step += 1
        st = _lib.stream_ptr(self.device)
        for name, *_ in LAYERS:
            for kind, p, gr in (("w:", self.w32[name], self.dw[name]), ("b:", self.b32[name], self.db[name])):
                _lib.check(self.lib.mrb_cnn_adam(_p(p), _p(gr), _p(self.m[kind + name]), _p(self.v[kind + name]),
                                                 p.numel(), lr, b1, b2, eps, self.step, None, st), "adam")
        self.refresh()

    def train(self, inputs: torch.Tensor, targets: torch.Tensor, epochs: int = 5, batch: int = 4,
              lr: float = 1e-3, seed: int = 0, log=None) -> List[float]:
        """inputs / targets (S, D, H, W) complex64 on the device; returns the mean loss per epoch."""
        g = torch.Generator().manual_seed(seed)
        S = int(inputs.shape[0])
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(S, generator=g)
            tot = torch.zeros((), dtype=torch.float64, device=self.device)
            nb = 0
            for i in range(0, S - batch + 1, batch):
                idx = perm[i:i + batch].to(self.device)
                l = self.loss_and_grad(inputs[idx].contiguous(), targets[idx].contiguous())
                tot += l[0]
                nb += 1
                self.adam_step(lr)
            hist.append(float(tot) / max(1, nb))
            if log:
                log(f"epoch {ep}: loss {hist[-1]:.4e}")
        return hist


# ---------------------------------------------------------------------------
# training pairs and the warm-start solve
# ---------------------------------------------------------------------------
@dataclass
class PairSpec:
    """Training series: the GRASP workload's acquisition (256^2, 12 coils, 21
    golden-angle spokes x 512 samples per frame) over `frames` frames."""
    N: int = 256
    frames: int = 8
    coils: int = 12
    spokes: int = 21
    nread: int = 512
    lam_s: float = 1e-3
    lam_t: float = 5e-3
    eps: float = 1e-3
    sigma: float = 1e-3
    stop_tol: float = 5e-5
    max_iter: int = 800


def make_pairs(n_series: int, spec: PairSpec = PairSpec(), seed0: int = 1000, per_solve: int = 50,
               device="cuda", log=None):
    """(adjoint recon, converged NCG recon) pairs, (n_series, F, N, N) complex64 on the device.

    Series s has phantom seed seed0 + s and golden-angle spokes that continue
    across series; `per_solve` series are solved together in one NCG run whose
    temporal TV does not couple series (the objective is separable, so each
    series converges to its own minimiser)."""
    from . import phantoms
    from .nufft import B200NUFFTAdapter
    from .regularization import RegManager, TVND, TVParams
    from .solver import CGSolver, CGConfig
    dev = torch.device(device)
    F, N, C = spec.frames, spec.N, spec.coils
    maps = phantoms.coil_maps(N, C).to(dev)
    xs_adj, xs_ref = [], []
    for s0 in range(0, n_series, per_solve):
        P = min(per_solve, n_series - s0)
        traj = torch.stack([phantoms.golden_angle_radial(spec.spokes, spec.nread, ((s0 + p) * F + f) * spec.spokes)
                            for p in range(P) for f in range(F)]).to(dev)
        xt = torch.cat([phantoms.dynamic_phantom(N, F, seed=seed0 + s0 + p) for p in range(P)]).unsqueeze(1)
        ad = B200NUFFTAdapter(ndim=2)
        ad.prepare((C, N, N), traj, None, maps, torch.complex64, dev)
        y = ad.A(xt.to(dev))
        if spec.sigma > 0:
            y = phantoms.add_noise(y, spec.sigma, seed=seed0 + s0)
        regm = RegManager([TVND("s", TVParams(weight=spec.lam_s, eps=spec.eps, axes="spatial")),
                           TVND("t", TVParams(weight=spec.lam_t, eps=spec.eps, axes="temporal"))])
        cfg = CGConfig(max_iter=spec.max_iter, stop_window=10, stop_tol=spec.stop_tol, series_length=F)
        sol = CGSolver(y, ad, regm, cfg)
        sol.run()
        xs_ref.append(sol.result().reshape(P, F, N, N).clone())
        xs_adj.append(ramp_adjoint(ad, y).reshape(P, F, N, N))
        del ad._ramp_adapter
        if log:
            log(f"pairs {s0 + P}/{n_series}: {sol.iter} iterations ({sol.stop_reason})")
    return torch.cat(xs_adj), torch.cat(xs_ref)


def ramp_adjoint(op, y: torch.Tensor) -> torch.Tensor:
    """The network input: the density-compensated adjoint A^H(w * y) (gridding
    reconstruction) with the radial ramp w = max(|k|, pi / (2 max S)) / pi.
    `op` is a B200 NUFFT front-end or adapter and y is in its canonical
    (B, C, K) layout; the ramp weights are computed once and cached on the adapter."""
    from .nufft import B200NUFFTAdapter
    ad = getattr(op, "backend", op)
    C, K = int(ad._im_shape[0]), int(ad._K)
    w = getattr(ad, "_ramp_w", None)
    if w is None:
        S = ad._im_shape[1:]
        kr = torch.linalg.vector_norm(ad._traj_BndK, dim=1)
        w = (kr.clamp_min(math.pi / (2.0 * max(S))) / math.pi).to(torch.float32)
        ad._ramp_w = w
    yy = y.reshape(-1, C, K)
    if ad._dcf_BK is None or ad.dcf_mode == "none" or not ad.apply_dcf_in_adj:
        # the operator's own adjoint applied to the ramp-weighted samples (frame
        # be of a B_eff batch uses trajectory frame be // (nb / B))
        nb, B = int(yy.shape[0]), int(w.shape[0])
        wb = w if B in (1, nb) else w.repeat_interleave(nb // B, dim=0)
        return ad.AH((yy * wb[:, None, :]).contiguous())
    # an operator with its own adjoint weights: a second plan with the ramp alone
    r = getattr(ad, "_ramp_adapter", None)
    if r is None:
        r = B200NUFFTAdapter(ndim=ad.ndim, dcf_mode="standard", apply_dcf_in_fwd=False, apply_dcf_in_adj=True,
                             kwidth=ad.kwidth, osf=ad.osf, norm=ad.norm)
        r.prepare(ad._im_shape, ad._traj_BndK, w, ad._maps, torch.complex64, ad._dev)
        ad._ramp_adapter = r
    return r.AH(yy)


def _ls_scaled(op, y, x):
    """x times its least-squares data-consistency factor argmin_a ||a A x - y||
    (the sums in FP64 on the device, as warm_start forms them)."""
    from .regularization import workspace
    Ax = op.A(x)
    s = _dots_f64([(Ax, Ax), (Ax, y)], workspace(x.device))
    return (x * (s[1] / s[0].clamp_min(1e-30)).to(torch.float32)).to(torch.complex64)


def network_start(op, y, cnn: WarmStartCNN, image_shape) -> torch.Tensor:
    """The network's image for data y (LS-scaled), shaped like the solver's image."""
    return _ls_scaled(op, y, _network_image(op, y, cnn, image_shape))


def warm_start(solver, cnn: WarmStartCNN) -> dict:
    """Initial image for `solver` from the network, with the fallback rule:
    the network output is used only if its objective is below that of the
    adjoint start (the adjoint recon A^H y scaled by its least-squares factor).

    Both starts are scaled by their least-squares data-consistency factors
    a = Re<Ax, y> / ||Ax||^2, whose data terms follow from the same sums:
    0.5 ||a A x - y||^2 = 0.5 (||y||^2 - Re<Ax, y>^2 / ||Ax||^2).  The sums (FP64
    on the device) and the regularisers' energies at the scaled starts are read
    to the host once."""
    op = solver.op
    y = solver.y
    x_adj = op.AH(y)
    x_cnn = _network_image(op, y, cnn, x_adj.shape)
    ax_adj, ax_cnn = op.A(x_adj), op.A(x_cnn)
    s = _dots_f64([(ax_adj, ax_adj), (ax_adj, y), (ax_cnn, ax_cnn), (ax_cnn, y), (y, y)], solver.ws_buf)
    # the factors stay on the device: x * (num / den)
    a = torch.stack([s[1] / s[0].clamp_min(1e-30), s[3] / s[2].clamp_min(1e-30)]).to(torch.float32)
    x_adj = (x_adj * a[0]).to(torch.complex64)
    x_net = (x_cnn * a[1]).to(torch.complex64)
    e_adj = torch.zeros(24, dtype=torch.float64, device=y.device)
    e_net = torch.zeros(24, dtype=torch.float64, device=y.device)
    solver.regularizer_energy_into(x_adj, e_adj)
    solver.regularizer_energy_into(x_net, e_net)
    v = torch.cat([s, e_adj, e_net]).tolist()
    den_a, num_a, den_n, num_n, yy = v[:5]
    f_adj = 0.5 * max(yy - num_a * num_a / max(den_a, 1e-30), 0.0) + solver.regularizer_energy_from(v[5:29])
    f_net = 0.5 * max(yy - num_n * num_n / max(den_n, 1e-30), 0.0) + solver.regularizer_energy_from(v[29:53])
    use = f_net < f_adj
    solver.reset(x_net if use else x_adj)
    return {"used_network": bool(use), "f_network": f_net, "f_adjoint": f_adj}


def _dots_f64(pairs, ws) -> torch.Tensor:
    """Re<a_j, b_j> for (a_j, b_j) in pairs (complex64, equal lengths), FP64 on the
    device; ws is a reduction workspace of the library."""
    n = int(pairs[0][0].numel())
    A = (ct.c_void_p * len(pairs))(*[_p(a) for a, _ in pairs])
    B = (ct.c_void_p * len(pairs))(*[_p(b) for _, b in pairs])
    out = torch.empty(len(pairs), dtype=torch.float64, device=pairs[0][0].device)
    _lib.check(_lib.load().mrb_dots_f64(n, len(pairs), A, B, None, 0, _p(out), _p(ws), _lib.stream_ptr(out.device)),
               "dots_f64")
    return out


def _network_image(op, y, cnn: WarmStartCNN, image_shape) -> torch.Tensor:
    """The network's image for data y (not yet scaled), shaped like the solver's image."""
    z = ramp_adjoint(op, y)
    F = int(z.shape[0])
    S = tuple(int(s) for s in z.shape[2:])
    return cnn.infer(z.to(torch.complex64).reshape((1, F) + S)).reshape(image_shape)


def evaluate(cnn: "WarmStartCNN", workload: str = "grasp", device="cuda", reps: int = 1) -> dict:
    """Warm-start + NCG against plain NCG (from x = 0) on a seeded workload, both to
    the same windowed objective tolerance on the same GPU.  Times are device
    seconds per solve (CUDA events); the warm-started time includes the adjoint,
    the network, its least-squares scaling and the fallback test."""
    from .solver import CGSolver
    from .workloads import WORKLOADS, build, regs, solver_cfg
    w = WORKLOADS[workload]
    dev = torch.device(device)
    op, y, x_true, _, _ = build(w, dev)
    solver = CGSolver(y, op, regs(w), solver_cfg())
    solver.reset().run()
    warm_start(solver, cnn)
    solver.run()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    a, b = ev(), ev()
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        solver.reset().run()
    b.record()
    torch.cuda.synchronize()
    t_plain = a.elapsed_time(b) / 1e3 / reps
    it_plain = solver.iter
    x_plain = solver.result().clone()
    f_plain = solver.objective()
    a, b = ev(), ev()
    a.record()
    for _ in range(reps):
        info = warm_start(solver, cnn)
        solver.run()
    b.record()
    torch.cuda.synchronize()
    t_warm = a.elapsed_time(b) / 1e3 / reps
    x_warm = solver.result()
    xt = x_true.to(dev).reshape(x_plain.shape)
    rel = lambda u, v: float(torch.linalg.vector_norm(u - v) / torch.linalg.vector_norm(v))
    x_net = network_start(op, y, cnn, x_plain.shape)
    x_adj = _ls_scaled(op, y, op.AH(y))
    return {"workload": w["name"], "plain_s": t_plain, "plain_iters": it_plain, "f_plain": f_plain,
            "warm_s": t_warm, "warm_iters": solver.iter, "f_warm": solver.objective(),
            "err_vs_plain": rel(x_warm, x_plain), "plain_err_vs_truth": rel(x_plain, xt),
            "warm_err_vs_truth": rel(x_warm, xt), "network_start_err_vs_plain": rel(x_net, x_plain),
            "adjoint_start_err_vs_plain": rel(x_adj, x_plain), **info}


def training_step_time(device="cuda", batch: int = 2, frames: int = 8, N: int = 256, reps: int = 5) -> dict:
    """Device milliseconds of one training step (forward, backward, Adam) of the
    network on random series of the training shape (batch x frames x N x N), with
    the weight gradients on tcgen05 and on the mma.sync kernel."""
    dev = torch.device(device)
    net = WarmStartCNN(dev, seed=0)
    g = torch.Generator(device=dev).manual_seed(1)
    z = torch.randn((batch, frames, N, N), dtype=torch.complex64, device=dev, generator=g)
    t = z + 0.1 * torch.randn((batch, frames, N, N), dtype=torch.complex64, device=dev, generator=g)
    out = {"shape": [batch, frames, N, N]}
    for tc in (True, False):
        net.use_tc_wgrad = tc
        net.loss_and_grad(z, t)
        net.adam_step(lr=1e-5)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record()
        for _ in range(reps):
            net.loss_and_grad(z, t)
            net.adam_step(lr=1e-5)
        b.record()
        torch.cuda.synchronize(dev)
        out["step_ms_tc_wgrad" if tc else "step_ms_mma_wgrad"] = a.elapsed_time(b) / reps
    return out


def tolerance_study(cnn: "WarmStartCNN", tols=(1e-4, 3e-5, 1e-5, 3e-6, 1e-6), star_tol: float = 1e-8,
                    star_max_iter: int = 12000, workload: str = "grasp", device="cuda") -> dict:
    """How close the warm-started and the plain solve land at each windowed
    tolerance, measured against a tightly converged minimiser x*.

    x* is NCG from the learned warm start run to the windowed tolerance
    `star_tol` (in practice to its first line-search failure, where FP32 rounding
    leaves no step that lowers the objective, or `star_max_iter` iterations); the
    warm start lands at a lower objective there than the zero start does, so it
    is the closer estimate of the minimiser.  For every tol in
    `tols`, both solves run to that tolerance on the same GPU (device seconds of
    one solve after an untimed one that captures the graphs); each row reports
    their times, iterations, the image difference of the two results
    (rel-L2 against the plain one) and each result's rel-L2 distance to x*.
    `first_tol_within_1e-3` is the loosest tolerance at which the two results
    differ by at most 1e-3."""
    from .solver import CGSolver
    from .workloads import WORKLOADS, build, regs, solver_cfg
    w = WORKLOADS[workload]
    dev = torch.device(device)
    op, y, x_true, _, _ = build(w, dev)
    regm = regs(w)
    rel = lambda u, v: float(torch.linalg.vector_norm(u - v) / torch.linalg.vector_norm(v))
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def solver_at(tol, max_iter):
        cfg = solver_cfg(max_iter)
        cfg.stop_tol = tol
        return CGSolver(y, op, regm, cfg)

    def timed(fn):
        fn()                                   # graph capture, allocations
        a, b = ev(), ev()
        torch.cuda.synchronize()
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1e3

    star = solver_at(star_tol, star_max_iter)

    def star_solve():
        warm_start(star, cnn)
        star.run()
    t_star = timed(star_solve)
    x_star = star.result().clone()
    out = {"workload": w["name"], "x_star": {"start": "learned warm start", "stop_tol": star_tol,
                                              "iters": star.iter, "stop": star.stop_reason,
                                              "objective": star.objective(), "s": t_star,
                                              "err_vs_truth": rel(x_star, x_true.to(dev).reshape(x_star.shape))},
           "rows": []}
    del star
    for tol in tols:
        s = solver_at(tol, star_max_iter)
        t_plain = timed(lambda: s.reset().run())
        it_plain, x_plain, f_plain = s.iter, s.result().clone(), s.objective()

        def warm():
            warm_start(s, cnn)
            s.run()
        t_warm = timed(warm)
        x_warm = s.result()
        out["rows"].append({"stop_tol": tol, "plain_s": t_plain, "plain_iters": it_plain, "warm_s": t_warm,
                            "warm_iters": s.iter, "f_plain": f_plain, "f_warm": s.objective(),
                            "err_vs_plain": rel(x_warm, x_plain), "plain_err_vs_star": rel(x_plain, x_star),
                            "warm_err_vs_star": rel(x_warm, x_star)})
        del s
    ok = [r for r in out["rows"] if r["err_vs_plain"] <= 1e-3]
    out["first_tol_within_1e-3"] = ok[0]["stop_tol"] if ok else None
    return out


def main(argv=None):
    """Generate training pairs, train, save:  python -m mrirecon_b200.warmstart --out w.npz
    Evaluate saved weights on the GRASP workload:  python -m mrirecon_b200.warmstart --eval w.npz"""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--eval", default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--series", type=int, default=2000)
    ap.add_argument("--per-solve", type=int, default=25)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=2)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--frames", type=int, default=8)
    ap.add_argument("--init", default=None, help="start training from these weights (fine-tuning)")
    a = ap.parse_args(argv)
    if a.eval:
        net = WarmStartCNN("cuda", seed=0)
        net.load(a.eval)
        print(json.dumps(evaluate(net)), flush=True)
        return
    if not a.out:
        ap.error("--out or --eval is required")
    t0 = time.time()
    spec = PairSpec(frames=a.frames)
    xa, xr = make_pairs(a.series, spec, per_solve=a.per_solve, log=lambda m: print(m, flush=True))
    print(f"pairs: {time.time() - t0:.1f} s", flush=True)
    net = WarmStartCNN("cuda", seed=0)
    if a.init:
        net.load(a.init)
    t1 = time.time()
    hist = net.train(xa, xr, epochs=a.epochs, batch=a.batch, lr=a.lr, log=lambda m: print(m, flush=True))
    print(f"training: {time.time() - t1:.1f} s, loss per epoch {hist}", flush=True)
    net.save(a.out)
    print(json.dumps(evaluate(net)), flush=True)


if __name__ == "__main__":
    main()
