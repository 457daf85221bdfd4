"""ctypes binding of the in-tree CUDA library ``libmrirecon_b200.so``.

The product path has no fallback: if the library is missing or CUDA is not
usable, every operator raises.  Device pointers and the current torch CUDA
stream are passed straight to the C ABI declared in
``include/mrirecon_b200.h``.
"""
from __future__ import annotations

import ctypes as ct
import os
import threading

import torch

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libmrirecon_b200.so")

_lib = None
_lock = threading.Lock()

c_int64_p = ct.POINTER(ct.c_int64)
c_int_p = ct.POINTER(ct.c_int)
c_double_p = ct.POINTER(ct.c_double)


class TVTerm(ct.Structure):
    """Mirror of ``mrb_tv_term``."""
    _fields_ = [
        ("enabled", ct.c_int),
        ("isotropic", ct.c_int),
        ("weight", ct.c_float),
        ("eps", ct.c_float),
        ("naxes", ct.c_int),
        ("axes", ct.c_int * 4),
        ("axis_weights", ct.c_float * 4),
        ("frame_period", ct.c_int),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "mrb_version": (ct.c_int, []),
    "mrb_last_error": (ct.c_char_p, []),
    "mrb_launch_count": (ct.c_int64, []),
    "mrb_release_cached_memory": (ct.c_int, []),
    "mrb_group_begin": (ct.c_int, [ct.c_int]),
    "mrb_group_select": (ct.c_int, [ct.c_int]),
    "mrb_group_end": (ct.c_int, [ct.c_void_p]),
    "mrb_group_cancel": (ct.c_int, []),
    "mrb_group_stats": (ct.c_int, [c_int64_p, c_int64_p]),
    "mrb_nufft_stage": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]),
    "mrb_plan_create": (ct.c_int, [ct.POINTER(ct.c_void_p), ct.c_int, c_int_p, ct.c_int, ct.c_int, ct.c_int64,
                                   ct.c_int, ct.c_double, ct.c_int]),
    "mrb_plan_destroy": (ct.c_int, [ct.c_void_p]),
    "mrb_plan_set_option": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int64]),
    "mrb_plan_set_points": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_plan_set_dcf": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p]),
    "mrb_plan_set_maps": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_nufft_forward": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]),
    "mrb_nufft_forward_coils": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]),
    "mrb_nufft_adjoint": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]),
    "mrb_plan_info": (ct.c_int, [ct.c_void_p, c_int64_p, ct.c_int]),
    "mrb_plan_set_skip_flag": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    "mrb_plan_set_toeplitz": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_nufft_normal": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]),
    "mrb_plan_cell_base": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_grid_indices": (ct.c_int, [ct.c_void_p, ct.c_int, c_int_p, ct.c_int64, ct.c_int, ct.c_int, ct.c_void_p,
                                    ct.c_void_p]),
    "mrb_workspace_bytes": (ct.c_int, [c_int64_p]),
    "mrb_dots_f64": (ct.c_int, [ct.c_int64, ct.c_int, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_void_p),
                                ct.POINTER(ct.c_void_p), ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_dots_f64_noalloc": (ct.c_int, [ct.c_int64, ct.c_int, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_void_p),
                                        ct.POINTER(ct.c_void_p), ct.c_int64, ct.c_void_p, ct.c_void_p]),
    "mrb_kspace_pass": (ct.c_int, [ct.c_int, ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                   ct.c_void_p, ct.c_double, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_tv_grad": (ct.c_int, [ct.c_int, c_int_p, ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p,
                               ct.c_void_p, ct.c_double, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                               ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p,
                               ct.c_void_p]),
    "mrb_tv_multi": (ct.c_int, [ct.c_int, c_int_p, ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p,
                                ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_ncg_slot_count": (ct.c_int, [c_int64_p, c_int64_p]),
    "mrb_ncg_set_steps": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double, ct.c_void_p]),
    "mrb_ncg_armijo_select": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_ncg_armijo_phase": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p]),
    "mrb_ncg_control": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p]),
    "mrb_ncg_update": (ct.c_int, [ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                  ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_ncg_steepest": (ct.c_int, [ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64,
                                    ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_ncg_err_step": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    "mrb_ncg_restart": (ct.c_int, [ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_void_p,
                                   ct.c_void_p]),
    "mrb_precond_init": (ct.c_int, [ct.c_int64, ct.c_int, ct.c_int, ct.c_void_p, ct.c_float, ct.c_float,
                                    ct.c_void_p, ct.c_void_p]),
    "mrb_tv_add_diag": (ct.c_int, [ct.c_int, c_int_p, ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int,
                                   ct.c_void_p, ct.c_void_p]),
    "mrb_diag_add_frames": (ct.c_int, [ct.c_int64, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "mrb_graph_pass": (ct.c_int, [ct.c_int, ct.c_int, ct.c_int64, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                  ct.c_void_p, ct.c_double, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                  ct.c_void_p]),
    "mrb_ncg_quad_fold": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_void_p]),
    "mrb_frame_mix": (ct.c_int, [ct.c_int, ct.c_int, ct.c_int64, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p,
                                 ct.c_int, ct.c_void_p]),
    "mrb_frame_mix_real": (ct.c_int, [ct.c_int, ct.c_int, ct.c_int64, ct.c_void_p, ct.c_int, ct.c_void_p,
                                      ct.c_void_p, ct.c_int, ct.c_void_p]),
}


def exported_symbols():
    """Names the binding expects the library to export."""
    return list(_SIGS)


def load(path: str = LIB_PATH):
    """Load the library (once).  Raises RuntimeError when it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with `python -m mrirecon_b200.build` "
                "(there is no CPU fallback for the B200 path)")
        lib = ct.CDLL(path, mode=ct.RTLD_GLOBAL)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    m = load().mrb_last_error()
    return m.decode() if m else ""


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        raise RuntimeError(f"mrirecon_b200 {what} failed (code {rc}): {last_error()}")


def stream_ptr(device=None) -> int:
    return int(torch.cuda.current_stream(device).cuda_stream)


def launch_count() -> int:
    """Kernel launches issued by the library so far (graph captures count once)."""
    return int(load().mrb_launch_count())


def workspace_bytes() -> int:
    v = ct.c_int64()
    check(load().mrb_workspace_bytes(ct.byref(v)), "workspace_bytes")
    return int(v.value)


def ncg_slot_count():
    a, b = ct.c_int64(), ct.c_int64()
    check(load().mrb_ncg_slot_count(ct.byref(a), ct.byref(b)), "ncg_slot_count")
    return int(a.value), int(b.value)


def ptr(t) -> int:
    if t is None:
        return 0
    return int(t.data_ptr())


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise RuntimeError(f"{name} must be a CUDA tensor (the B200 path has no CPU fallback)")
