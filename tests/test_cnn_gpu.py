"""Warm-start network kernels vs FP32/FP64 CPU references.

Tolerances: single-layer conv forward / data gradient / weight gradient on
BF16-valued inputs rel-L2 <= 1e-5 (products of BF16 values are exact in FP32,
only FP32 accumulation differs from the FP64 reference); whole network
(BF16 activations between layers) loss rel <= 2e-2 and per-layer weight
gradients rel-L2 <= 6e-2 against torch.autograd in FP32 on the same weights.
"""
import ctypes as ct

import numpy as np
import pytest
import torch
import torch.nn.functional as Fn

from conftest import rel
from oracle import cnn as ocnn

pytestmark = pytest.mark.gpu


def _bf(t):
    return t.to(torch.bfloat16)


def _torch_w(w27):
    cin, cout = w27.shape[1], w27.shape[2]
    return w27.permute(2, 1, 0).reshape(cout, cin, 3, 3, 3)


@pytest.mark.parametrize("cin,cout,vol", [(32, 32, (2, 3, 8, 8)), (64, 128, (1, 4, 6, 10)), (192, 64, (1, 2, 4, 4))])
def test_conv_fwd_dgrad_wgrad_exact(cuda, cin, cout, vol):
    from mrirecon_b200 import _lib
    from mrirecon_b200.warmstart import _lib_cnn, _vol
    L = _lib_cnn()
    st = _lib.stream_ptr()
    g = torch.Generator().manual_seed(cin + cout)
    Nb, D, H, W = vol
    V = Nb * D * H * W
    x = _bf(torch.randn((V, cin), generator=g))
    w = _bf(torch.randn((27, cin, cout), generator=g) * 0.1)
    bias = torch.randn(cout, generator=g)
    gy = _bf(torch.randn((V, cout), generator=g))
    xc, wc, bc, gyc = x.to(cuda), w.to(cuda), bias.to(cuda), gy.to(cuda)
    y = torch.zeros((V, cout), dtype=torch.float32, device=cuda)
    _lib.check(L.mrb_cnn_conv3d_fwd(xc.data_ptr(), cin, 0, cin, wc.data_ptr(), cout, cout, bc.data_ptr(), 0, None, 0,
                                    0, y.data_ptr(), cout, 0, 0, _vol(*vol), st), "fwd")
    # FP64 reference on the same BF16 values
    x5 = x.double().reshape(Nb, D, H, W, cin).permute(0, 4, 1, 2, 3).requires_grad_(True)
    w5 = _torch_w(w.double()).requires_grad_(True)
    y5 = Fn.conv3d(x5, w5, bias.double(), padding=1)
    yref = y5.permute(0, 2, 3, 4, 1).reshape(V, cout)
    assert rel(y, yref) < 1e-5
    y5.backward(gy.double().reshape(Nb, D, H, W, cout).permute(0, 4, 1, 2, 3))
    # weight gradient
    dw = torch.zeros((27, cin, cout), dtype=torch.float32, device=cuda)
    db = torch.zeros(cout, dtype=torch.float32, device=cuda)
    part = torch.zeros(27 * cin * cout * 8, dtype=torch.float32, device=cuda)
    _lib.check(L.mrb_cnn_conv3d_wgrad(xc.data_ptr(), cin, 0, cin, gyc.data_ptr(), cout, 0, cout, dw.data_ptr(),
                                      db.data_ptr(), part.data_ptr(), part.numel(), _vol(*vol), st), "wgrad")
    dw_ref = w5.grad.reshape(cout, cin, 27).permute(2, 1, 0)
    assert rel(dw, dw_ref) < 1e-5
    assert rel(db, gy.double().sum(0)) < 1e-5
    # data gradient = forward conv with flipped, transposed weights
    wd = torch.empty((27, cout, cin), dtype=torch.bfloat16, device=cuda)
    _lib.check(L.mrb_cnn_flip_weights(wc.data_ptr(), cin, cout, wd.data_ptr(), cin, st), "flip")
    dx = torch.zeros((V, cin), dtype=torch.float32, device=cuda)
    _lib.check(L.mrb_cnn_conv3d_fwd(gyc.data_ptr(), cout, 0, cout, wd.data_ptr(), cin, cin, None, 0, None, 0, 0,
                                    dx.data_ptr(), cin, 0, 0, _vol(*vol), st), "dgrad")
    assert rel(dx, x5.grad.permute(0, 2, 3, 4, 1).reshape(V, cin)) < 1e-5


def _wgrad_tc(L, xc, cx, ci_off, cin, gyc, cg, cout, vol, dw, db):
    import ctypes as ct
    from mrirecon_b200 import _lib
    from mrirecon_b200.warmstart import _vol
    nbytes = ct.c_int64(0)
    _lib.check(L.mrb_cnn_wgrad_tc_scratch_bytes(cin, cout, _vol(*vol), ct.byref(nbytes)), "scratch size")
    scratch = torch.empty(nbytes.value, dtype=torch.uint8, device=xc.device)
    _lib.check(L.mrb_cnn_conv3d_wgrad_tc(xc.data_ptr(), cx, ci_off, cin, gyc.data_ptr(), cg, 0, cout, dw.data_ptr(),
                                         db.data_ptr(), scratch.data_ptr(), scratch.numel(), _vol(*vol),
                                         _lib.stream_ptr()), "wgrad tc")
    err = ct.c_int(0)
    _lib.check(L.mrb_cnn_tc_error(ct.byref(err)), "tc error")
    assert err.value == 0


@pytest.mark.parametrize("cin,cout,vol", [(32, 32, (2, 3, 8, 64)), (64, 128, (1, 4, 6, 64)),
                                          (192, 64, (1, 2, 4, 128)), (96, 32, (2, 3, 5, 64)),
                                          (64, 64, (1, 3, 4, 256))])
def test_conv_wgrad_tensor_cores_exact(cuda, cin, cout, vol):
    """Weight and bias gradient on tcgen05 (x on the M side when cin > cout, two
    M tiles at cin = 192, gz on the M side otherwise) against FP64 autograd on
    the same BF16 values and against the mma.sync kernel; the input is read at a
    channel offset inside a wider tensor."""
    from mrirecon_b200 import _lib
    from mrirecon_b200.warmstart import _lib_cnn, _vol
    L = _lib_cnn()
    st = _lib.stream_ptr()
    g = torch.Generator().manual_seed(7 * cin + cout)
    Nb, D, H, W = vol
    V = Nb * D * H * W
    cx, ci_off = cin + 32, 16
    xw = _bf(torch.randn((V, cx), generator=g))
    x = xw[:, ci_off:ci_off + cin]
    gy = _bf(torch.randn((V, cout), generator=g))
    x5 = x.double().reshape(Nb, D, H, W, cin).permute(0, 4, 1, 2, 3)
    w5 = torch.zeros((cout, cin, 3, 3, 3), dtype=torch.float64, requires_grad=True)
    y5 = Fn.conv3d(x5, w5, padding=1)
    y5.backward(gy.double().reshape(Nb, D, H, W, cout).permute(0, 4, 1, 2, 3))
    dw_ref = w5.grad.reshape(cout, cin, 27).permute(2, 1, 0)
    xc, gyc = xw.contiguous().to(cuda), gy.to(cuda)
    dw = torch.full((27, cin, cout), float("nan"), dtype=torch.float32, device=cuda)
    db = torch.full((cout,), float("nan"), dtype=torch.float32, device=cuda)
    for _ in range(2):                      # the scratch holds no state between calls
        _wgrad_tc(L, xc, cx, ci_off, cin, gyc, cout, cout, vol, dw, db)
        assert rel(dw, dw_ref) < 1e-5
        assert rel(db, gy.double().sum(0)) < 1e-5
    dw2 = torch.zeros_like(dw)
    part = torch.zeros(27 * cin * cout * 8, dtype=torch.float32, device=cuda)
    _lib.check(L.mrb_cnn_conv3d_wgrad(xc.data_ptr(), cx, ci_off, cin, gyc.data_ptr(), cout, 0, cout, dw2.data_ptr(),
                                      None, part.data_ptr(), part.numel(), _vol(*vol), st), "wgrad")
    assert rel(dw, dw2) < 1e-5


def test_network_loss_and_gradients_vs_autograd(cuda):
    from mrirecon_b200.warmstart import WarmStartCNN, LAYERS
    torch.manual_seed(0)
    net = WarmStartCNN(cuda, seed=3)
    # non-trivial last layer so every layer gets a gradient
    net.w32["c8"].mul_(10.0)
    net.refresh()
    Nb, D, H, W = 2, 3, 8, 12
    z = (torch.randn(Nb, D, H, W) + 1j * torch.randn(Nb, D, H, W)).to(torch.complex64)
    t = (torch.randn(Nb, D, H, W) + 1j * torch.randn(Nb, D, H, W)).to(torch.complex64)
    loss = float(net.loss_and_grad(z.to(cuda), t.to(cuda))[0])
    s = 1.0 / z.reshape(Nb, -1).abs().amax(1)
    zs = z * s.view(-1, 1, 1, 1)
    ts = t * s.view(-1, 1, 1, 1)
    x2 = torch.stack([zs.real, zs.imag], 1).float()
    t2 = torch.stack([ts.real, ts.imag], 1).float()
    P = {}
    for name, cinp, cin, coutp, cout, relu in LAYERS:
        w = net.wb[name].float().cpu()[:, :cin, :cout].clone().requires_grad_(True)
        b = net.b32[name].cpu()[:cout].clone().requires_grad_(True)
        P[name] = (w, b)
    lo = ocnn.loss(x2.to(torch.bfloat16).float(), t2, P, x_res=x2)
    lo.backward()
    assert abs(loss - float(lo)) <= 2e-2 * float(lo)
    for name, cinp, cin, coutp, cout, relu in LAYERS:
        gw = net.dw[name].cpu()[:, :cin, :cout]
        assert rel(gw, P[name][0].grad) < 6e-2, name
        assert rel(net.db[name].cpu()[:cout], P[name][1].grad) < 6e-2, name


def test_training_reduces_loss(cuda):
    from mrirecon_b200.warmstart import WarmStartCNN
    g = torch.Generator().manual_seed(0)
    S, D, H, W = 8, 4, 16, 16
    tgt = (torch.randn(S, D, H, W, generator=g) + 1j * torch.randn(S, D, H, W, generator=g)).to(torch.complex64)
    # inputs: blurred, scaled targets (a learnable map)
    inp = 0.5 * (tgt + torch.roll(tgt, 1, dims=2))
    net = WarmStartCNN(cuda, seed=1)
    hist = net.train(inp.to(cuda), tgt.to(cuda), epochs=12, batch=2, lr=2e-3)
    assert hist[-1] < 0.6 * hist[0]


@pytest.mark.parametrize("cin,cout,vol,ci_off", [(32, 32, (1, 3, 4, 32), 0), (64, 128, (2, 2, 2, 64), 32),
                                                 (192, 64, (1, 2, 1, 128), 0), (96, 32, (1, 3, 2, 64), 32)])
def test_conv_tcgen05_fwd_dgrad_exact(cuda, cin, cout, vol, ci_off):
    """tcgen05 / TMEM convolution (TMA-staged, zero padding by out-of-volume
    coordinates) against the FP64 reference on BF16 values: forward (FP32 and
    BF16-at-offset outputs) and the data gradient through the flipped-tap read
    of the forward weights; the barrier-timeout flag stays clear."""
    from mrirecon_b200 import _lib
    from mrirecon_b200.warmstart import _lib_cnn
    L = _lib_cnn()
    st = _lib.stream_ptr()
    Nb, D, H, W = vol
    assert L.mrb_cnn_tc_supported(cin, ci_off, cin + ci_off, cout, W, H)
    g = torch.Generator().manual_seed(7 * cin + cout)
    V = Nb * D * H * W
    cx = cin + ci_off
    xfull = _bf(torch.randn((V, cx), generator=g))
    x = xfull[:, ci_off:]
    w = _bf(torch.randn((27, cin, cout), generator=g) * 0.1)
    bias = torch.randn(cout, generator=g)
    gy = _bf(torch.randn((V, cout), generator=g))
    xc, bc, gyc = xfull.to(cuda), bias.to(cuda), gy.to(cuda)
    wk = w.permute(0, 2, 1).contiguous().to(cuda)          # [27][cout][cin], K-major
    y = torch.zeros((V, cout), dtype=torch.float32, device=cuda)
    yb = torch.zeros((V, cout + 32), dtype=torch.bfloat16, device=cuda)
    _lib.check(L.mrb_cnn_conv3d_tc(xc.data_ptr(), cx, ci_off, cin, wk.data_ptr(), 0, cout, cout, bc.data_ptr(), 0,
                                   yb.data_ptr(), cout + 32, 32, y.data_ptr(), cout, 0, 0, Nb, D, H, W, st), "tc fwd")
    x5 = x.double().reshape(Nb, D, H, W, cin).permute(0, 4, 1, 2, 3).requires_grad_(True)
    w5 = _torch_w(w.double())
    y5 = Fn.conv3d(x5, w5, bias.double(), padding=1)
    yref = y5.permute(0, 2, 3, 4, 1).reshape(V, cout)
    assert rel(y, yref) < 1e-5
    assert rel(yb[:, 32:].float(), yref) < 1e-2          # BF16 rounding of the output
    assert float(yb[:, :32].float().abs().max()) == 0.0   # channels before the offset untouched
    y5.backward(gy.double().reshape(Nb, D, H, W, cout).permute(0, 4, 1, 2, 3))
    wc = w.to(cuda)                                       # [27][cin][cout] read as [27][N = cin][K = cout]
    dx = torch.zeros((V, cin), dtype=torch.float32, device=cuda)
    _lib.check(L.mrb_cnn_conv3d_tc(gyc.data_ptr(), cout, 0, cout, wc.data_ptr(), 1, cin, cin, None, 0, None, 0, 0,
                                   dx.data_ptr(), cin, 0, 0, Nb, D, H, W, st), "tc dgrad")
    assert rel(dx, x5.grad.permute(0, 2, 3, 4, 1).reshape(V, cin)) < 1e-5
    err = ct.c_int(-1)
    _lib.check(L.mrb_cnn_tc_error(ct.byref(err)), "tc error flag")
    assert err.value == 0


def test_network_tcgen05_equals_mma_sync_path(cuda):
    """The network's inference and gradients agree on the tcgen05 and the
    mma.sync convolution paths (same BF16 operands, FP32 accumulation order
    differs)."""
    from mrirecon_b200.warmstart import WarmStartCNN
    net = WarmStartCNN(cuda, seed=5)
    net.w32["c8"].mul_(10.0)
    net.refresh()
    g = torch.Generator().manual_seed(2)
    z = (torch.randn((1, 4, 64, 64), generator=g) + 1j * torch.randn((1, 4, 64, 64), generator=g)).to(
        torch.complex64).to(cuda)
    tgt = (z * 0.5).contiguous()
    outs, losses, grads = [], [], []
    for tc in (True, False):
        net.use_tc = tc
        outs.append(net.infer(z).clone())
        losses.append(float(net.loss_and_grad(z, tgt)[0]))
        grads.append({k: v.clone() for k, v in net.dw.items()})
    assert rel(outs[0], outs[1]) < 1e-3
    assert abs(losses[0] - losses[1]) <= 1e-3 * abs(losses[1])
    for k in grads[0]:
        assert rel(grads[0][k], grads[1][k]) < 2e-2, k
