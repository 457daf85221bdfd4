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


def _dots(lib, fn_name, n, npairs, A, B, D, out, ws=None):
    from mrirecon_b200 import _lib
    fn = getattr(lib, fn_name)
    args = [n, npairs, A, B, D, n, _lib.ptr(out)]
    if ws is not None:
        args.append(_lib.ptr(ws))
    args.append(_lib.stream_ptr())
    _lib.check(fn(*args), fn_name)


def _operands(n, npairs, dev):
    """npairs (a_j, b_j, diag_j) triples (every third pair preconditioned), the
    FP64 CPU sums and the sums of |term| that scale the tolerance: the device
    rounds each FP32 term on its own, possibly with a fused multiply-add, so
    terms agree to a few FP32 ulps, not bit for bit."""
    g = torch.Generator(device="cpu").manual_seed(100 + npairs)
    a = [torch.randn(n, dtype=torch.complex64, generator=g) for _ in range(npairs)]
    b = [torch.randn(n, dtype=torch.complex64, generator=g) for _ in range(npairs)]
    d = [torch.rand(n, dtype=torch.float32, generator=g) + 0.5 if j % 3 == 1 else None for j in range(npairs)]
    want, scale = [], []
    for aj, bj, dj in zip(a, b, d):
        r = aj.real.double() * bj.real.double() + aj.imag.double() * bj.imag.double()
        if dj is not None:
            r = r / dj.double()
        want.append(r.sum().item())
        scale.append(r.abs().sum().item())
    a = [t.to(dev) for t in a]
    b = [t.to(dev) for t in b]
    d = [t.to(dev) if t is not None else None for t in d]
    A = (ct.c_void_p * npairs)(*[t.data_ptr() for t in a])
    B = (ct.c_void_p * npairs)(*[t.data_ptr() for t in b])
    D = (ct.c_void_p * npairs)(*[t.data_ptr() if t is not None else 0 for t in d])
    return (a, b, d), A, B, D, torch.tensor(want, dtype=torch.float64), torch.tensor(scale, dtype=torch.float64)


@pytest.mark.parametrize("npairs", [1, 3, 5, 7, 8])
def test_dots_noalloc_matches_allocating_entry_point(npairs):
    """Two calls in a row share the scratch; both equal the allocating entry
    point bit for bit, and that one the FP64 CPU sums to 1e-6 of the sum of
    |terms|.  npairs 5..8 run the 8-wide kernel whose unused slots hold no
    operands."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mrirecon_b200 import _lib
    from mrirecon_b200.regularization import workspace
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n = 2 * 1024 * 1024 + 31
    keep, A, Bp, Dp, want, scale = _operands(n, npairs, dev)
    ref = torch.zeros(npairs, dtype=torch.float64, device=dev)
    _dots(lib, "mrb_dots_f64", n, npairs, A, Bp, Dp, ref, ws=workspace(dev))
    assert torch.all((ref.cpu() - want).abs() <= 1e-6 * scale), (ref.cpu(), want)
    for _ in range(2):
        out = torch.full((npairs,), float("nan"), dtype=torch.float64, device=dev)
        _dots(lib, "mrb_dots_f64_noalloc", n, npairs, A, Bp, Dp, out)
        torch.testing.assert_close(out, ref, rtol=0.0, atol=0.0)


def test_dots_noalloc_inside_a_captured_graph():
    """After one call outside a capture, the entry point records into a CUDA
    graph without allocating: the replay equals the eager result and torch's
    allocator holds no more memory than before the capture."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mrirecon_b200 import _lib
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n = 1 << 20
    keep, A, Bp, Dp, want, scale = _operands(n, 3, dev)
    eager = torch.zeros(3, dtype=torch.float64, device=dev)
    _dots(lib, "mrb_dots_f64_noalloc", n, 3, A, Bp, Dp, eager)
    out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    side = torch.cuda.Stream(dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        graph.capture_begin()
        # (torch itself allocates a little state at capture_begin; measure around the call)
        before = torch.cuda.memory_allocated(dev)
        _dots(lib, "mrb_dots_f64_noalloc", n, 3, A, Bp, Dp, out)
        after = torch.cuda.memory_allocated(dev)
        graph.capture_end()
    assert after == before
    graph.replay()
    torch.cuda.synchronize()
    torch.testing.assert_close(out, eager, rtol=0.0, atol=0.0)
    del graph


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
