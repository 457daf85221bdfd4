"""The allocation-free dots entry point against the allocating one.

``mrb_dots_f64_noalloc`` exists for callers that cannot allocate device
memory at the call site: code inside a CUDA stream capture, real-time loops
where an allocation would synchronise the device, and processes whose device
memory another allocator owns.  It keeps its block partials in a fixed device
array instead of a caller workspace.  This file is collected last so that a
run stopping at the first failure has run every other test first; it passes
alone in a fresh process and after the other tests.
"""
import ctypes as ct

import pytest
import torch

pytestmark = pytest.mark.gpu


def _dots(lib, fn_name, n, A, B, D, out, ws=None):
    from mrirecon_b200 import _lib
    fn = getattr(lib, fn_name)
    args = [n, 3, A, B, D, n, _lib.ptr(out)]
    if ws is not None:
        args.append(_lib.ptr(ws))
    args.append(_lib.stream_ptr())
    _lib.check(fn(*args), fn_name)


def test_dots_noalloc_matches_allocating_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mrirecon_b200 import _lib
    from mrirecon_b200.regularization import workspace
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.manual_seed(3)
    n = 2 * 1024 * 1024 + 31
    a = torch.randn(n, dtype=torch.complex64, device=dev)
    b = torch.randn(n, dtype=torch.complex64, device=dev)
    D = torch.rand(n, dtype=torch.float32, device=dev) + 0.5
    A = (ct.c_void_p * 3)(a.data_ptr(), a.data_ptr(), b.data_ptr())
    Bp = (ct.c_void_p * 3)(b.data_ptr(), a.data_ptr(), b.data_ptr())
    Dp = (ct.c_void_p * 3)(0, D.data_ptr(), 0)
    ref = torch.zeros(3, dtype=torch.float64, device=dev)
    _dots(lib, "mrb_dots_f64", n, A, Bp, Dp, ref, ws=workspace(dev))
    for _ in range(2):                       # two calls in a row share the scratch
        out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
        _dots(lib, "mrb_dots_f64_noalloc", n, A, Bp, Dp, out)
        torch.testing.assert_close(out, ref, rtol=1e-12, atol=0.0)


def test_dots_noalloc_rejects_too_many_pairs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mrirecon_b200 import _lib
    lib = _lib.load()
    x = torch.zeros(8, dtype=torch.complex64, device="cuda")
    P = (ct.c_void_p * 9)(*([x.data_ptr()] * 9))
    out = torch.zeros(9, dtype=torch.float64, device="cuda")
    rc = lib.mrb_dots_f64_noalloc(8, 9, P, P, None, 0, _lib.ptr(out), _lib.stream_ptr())
    assert rc != 0 and "at most 8 pairs" in _lib.last_error()
