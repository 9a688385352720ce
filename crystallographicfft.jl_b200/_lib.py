"""ctypes binding of libcfft_b200.so (the C ABI in include/cfft_b200.h).

The library is loaded from the package directory.  There is no fallback: if the
shared library is missing or cannot be loaded, importing the package raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcfft_b200.so")

c_int = ctypes.c_int
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p


class CFFTDesc(ctypes.Structure):
    _fields_ = [
        ("dim", c_int),
        ("N", c_int * 3),
        ("n_ops", c_int),
        ("R", c_int32_p),
        ("t", c_int32_p),
        ("lattice", ctypes.c_double * 9),
        ("ds", ctypes.c_double),
        ("precision", c_int),
        ("max_batch", c_int),
        ("path", c_int),
    ]


class CFFTInfo(ctypes.Structure):
    _fields_ = [
        ("N", c_int * 3), ("L", c_int * 3), ("M", c_int * 3), ("H", c_int * 3),
        ("n_spec", c_int), ("n_ops", c_int), ("n_rep", c_int), ("centering", c_int),
        ("centered", c_int), ("n_channels", c_int), ("n_orbits", c_int), ("n_rem_ops", c_int),
        ("precision", c_int), ("max_batch", c_int), ("P", c_int), ("workspace_bytes", ctypes.c_int64),
        ("exec_path", c_int), ("chunk", c_int), ("lanes", c_int),
    ]


class CFFTTuning(ctypes.Structure):
    _fields_ = [("chunk_bytes", ctypes.c_int64), ("lanes", c_int), ("zr_slots", c_int), ("wide", c_int),
                ("tma", c_int), ("cluster", c_int)]


STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "not commensurate", 4: "unsupported",
    5: "timeout", 6: "allocation failed", 7: "parity class not reachable",
}


class CFFTError(RuntimeError):
    """Raised for any non-zero cfft_status; `.status` holds the code."""

    def __init__(self, status, message):
        super().__init__(f"cfft status {status} ({STATUS.get(status, '?')}): {message}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libcfft_b200.so not built at {LIB_PATH}; run crystallographicfft.jl_b200/build.py")
    lib = ctypes.CDLL(LIB_PATH)
    sig = {
        "cfft_get_ops": (c_int, [c_int, c_int, c_int_p, c_int, c_int_p, c_int32_p, c_int32_p]),
        "cfft_list_groups": (c_int, [c_int, c_int_p, c_int]),
        "cfft_find_optimal_shift": (c_int, [c_int, c_int_p, c_int, c_int32_p, c_int32_p, c_double_p, c_int32_p]),
        "cfft_count_special_positions": (c_int, [c_int, c_int_p, c_int, c_int32_p, c_int32_p]),
        "cfft_auto_L": (c_int, [c_int, c_int, c_int32_p, c_int32_p, c_int_p]),
        "cfft_detect_centering": (c_int, [c_int, c_int_p, c_int, c_int32_p, c_int32_p]),
        "cfft_spectral_asu": (c_int, [c_int, c_int_p, c_int, c_int32_p, c_int32_p, c_int, c_int_p, c_int32_p, c_int32_p]),
        "cfft_plan_create": (c_int, [ctypes.POINTER(CFFTDesc), ctypes.POINTER(c_void_p)]),
        "cfft_plan_create_host": (c_int, [ctypes.POINTER(CFFTDesc), ctypes.POINTER(c_void_p)]),
        "cfft_plan_create_tuned": (c_int, [ctypes.POINTER(CFFTDesc), ctypes.POINTER(CFFTTuning),
                                           ctypes.POINTER(c_void_p)]),
        "cfft_plan_destroy": (c_int, [c_void_p]),
        "cfft_plan_info": (c_int, [c_void_p, ctypes.POINTER(CFFTInfo)]),
        "cfft_plan_spectral_asu": (c_int, [c_void_p, c_int32_p, c_int32_p]),
        "cfft_plan_q_tables": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_double), c_int32_p]),
        "cfft_block_plan_create": (c_int, [c_int, c_int32_p, c_int, ctypes.POINTER(c_void_p)]),
        "cfft_block_plan_destroy": (c_int, [c_void_p]),
        "cfft_block_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "cfft_block_backward": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "cfft_calc_asu": (c_int, [c_int, ctypes.POINTER(c_int), c_int, c_int32_p, c_int32_p, c_int,
                                  ctypes.POINTER(c_int), c_int32_p, c_int32_p, c_int32_p]),
        "cfft_fractal_tree": (c_int, [c_int, ctypes.POINTER(c_int), c_int, c_int32_p, c_int32_p, c_int, c_int,
                                      ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_int32_p]),
        "cfft_subgrid_spectrum": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "cfft_plan_rep_ops": (c_int, [c_void_p, c_int32_p, c_int32_p]),
        "cfft_plan_backward_tables": (c_int, [c_void_p, c_int32_p, c_int32_p, c_int32_p]),
        "cfft_plan_kernel": (c_int, [c_void_p, c_double_p]),
        "cfft_update_kernel": (c_int, [c_void_p, ctypes.c_double, c_double_p]),
        "cfft_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "cfft_backward": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "cfft_forward_plans": (c_int, [c_int, ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p),
                                       ctypes.POINTER(c_void_p), ctypes.POINTER(c_int), c_void_p]),
        "cfft_backward_plans": (c_int, [c_int, ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p),
                                        ctypes.POINTER(c_void_p), ctypes.POINTER(c_int), c_void_p]),
        "cfft_scft_step": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
        "cfft_step_diffusion": (c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_double, c_int, c_int, c_void_p]),
        "cfft_fullgrid_to_subgrid": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "cfft_subgrid_to_fullgrid": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "cfft_forward_host": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
        "cfft_backward_host": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
        "cfft_scft_step_host": (c_int, [c_void_p, c_void_p, c_int]),
        "cfft_profile_roundtrip": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                           ctypes.POINTER(ctypes.c_float), c_int_p]),
        "cfft_forward_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "cfft_plan_device_status": (c_int, [c_void_p, c_int]),
        "cfft_wait_selftest": (c_int, [c_void_p, ctypes.c_ulonglong, c_void_p]),
        "cfft_status_string": (ctypes.c_char_p, [c_int]),
        "cfft_last_error": (ctypes.c_char_p, []),
        "cfft_version": (c_int, []),
        "cfft_launch_count": (ctypes.c_int64, [c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()


def check(status):
    if status != 0:
        raise CFFTError(status, LIB.cfft_last_error().decode(errors="replace"))
    return status
