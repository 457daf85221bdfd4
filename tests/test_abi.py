"""The C-ABI library loads and exports every symbol the public header declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT


def _header_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(mrb_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_header_symbols():
    from mrirecon_b200 import _lib
    lib = _lib.load()
    missing = [n for n in _header_symbols() if not hasattr(lib, n)]
    assert not missing, f"symbols declared in include/ but not exported: {missing}"
    assert lib.mrb_version() >= 1


def test_binding_covers_header():
    from mrirecon_b200 import _lib
    hdr = set(_header_symbols())
    assert set(_lib.exported_symbols()) <= hdr | {"mrb_last_error", "mrb_version"}


def test_plan_create_rejects_bad_shapes_without_gpu():
    """Argument checks run on the host before any CUDA call."""
    from mrirecon_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    S = (ctypes.c_int * 3)(32, 32, 1)
    assert lib.mrb_plan_create(ctypes.byref(h), 4, S, 2, 1, 100, 4, 2.0, 1) != 0
    assert "nd must be 2 or 3" in _lib.last_error()
    assert lib.mrb_plan_create(ctypes.byref(h), 2, S, 2, 1, 100, 5, 2.0, 1) != 0
    assert lib.mrb_plan_create(ctypes.byref(h), 2, S, 0, 1, 100, 4, 2.0, 1) != 0


def test_group_recorder_state_without_gpu():
    """The launch recorder's host-side state machine: one recording at a time,
    problems selected in range, end/cancel only on an open recording; an empty
    recording ends without issuing anything."""
    from mrirecon_b200 import _lib
    lib = _lib.load()
    lib.mrb_group_cancel()
    assert lib.mrb_group_begin(0) != 0 and "nproblems" in _lib.last_error()
    assert lib.mrb_group_select(0) != 0 and "no recording" in _lib.last_error()
    assert lib.mrb_group_end(None) != 0 and "no recording" in _lib.last_error()
    assert lib.mrb_group_begin(3) == 0
    assert lib.mrb_group_begin(2) != 0 and "already open" in _lib.last_error()
    assert lib.mrb_group_select(2) == 0
    assert lib.mrb_group_select(3) != 0 and "outside" in _lib.last_error()
    assert lib.mrb_group_end(None) == 0           # nothing recorded: nothing issued
    rec, launches = ctypes.c_int64(-1), ctypes.c_int64(-1)
    assert lib.mrb_group_stats(ctypes.byref(rec), ctypes.byref(launches)) == 0
    assert rec.value == 0 and launches.value == 0
    assert lib.mrb_group_begin(1) == 0
    assert lib.mrb_group_cancel() == 0
    assert lib.mrb_group_end(None) != 0           # cancelled: closed
