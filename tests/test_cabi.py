"""The C-ABI library loads without a GPU and exports every symbol include/cfft_b200.h
declares; host-only entry points return the documented status codes."""
import ctypes
import os
import re

import pytest

from conftest import PKG_DIR, ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "cfft_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cfft_[A-Za-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(cf):
    lib = ctypes.CDLL(os.path.join(PKG_DIR, "libcfft_b200.so"))
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings(cf):
    lib = cf.LIB
    for code in range(8):
        assert lib.cfft_status_string(code)
    assert lib.cfft_version() >= 100


def test_invalid_arguments(cf):
    lib = cf.LIB
    assert lib.cfft_plan_create(None, None) == 1
    n = ctypes.c_int(0)
    N = (ctypes.c_int * 3)(16, 16, 16)
    assert lib.cfft_get_ops(999, 3, N, 0, ctypes.byref(n), None, None) == 4
    assert lib.cfft_get_ops(229, 4, N, 0, ctypes.byref(n), None, None) == 1
    assert lib.cfft_forward(None, None, None, 1, None) == 1
    assert b"null" in lib.cfft_last_error() or lib.cfft_last_error()


def test_fractal_tree_invalid_arguments(cf):
    import numpy as np

    lib = cf.LIB
    N = (ctypes.c_int * 3)(8, 8, 8)
    R = np.eye(3, dtype=np.int32).ravel()
    t = np.zeros(3, dtype=np.int32)
    Rp = R.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    tp = t.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    n, inner = ctypes.c_int(-1), ctypes.c_int(-1)
    assert lib.cfft_fractal_tree(3, N, 1, Rp, tp, 0, 0, None, ctypes.byref(inner), None) == 1
    assert lib.cfft_fractal_tree(4, N, 1, Rp, tp, 0, 0, ctypes.byref(n), ctypes.byref(inner), None) == 1
    assert lib.cfft_fractal_tree(3, N, 0, Rp, tp, 0, 0, ctypes.byref(n), ctypes.byref(inner), None) == 1
    assert lib.cfft_fractal_tree(3, N, 1, Rp, tp, 7, 0, ctypes.byref(n), ctypes.byref(inner), None) == 1
    assert lib.cfft_fractal_tree(3, N, 1, Rp, tp, 0, 0, ctypes.byref(n), ctypes.byref(inner), None) == 0
    assert n.value == 1 and inner.value == 0  # P1: the root is the only leaf
    out = np.zeros(10, dtype=np.int32)
    op = out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    assert lib.cfft_fractal_tree(3, N, 1, Rp, tp, 0, 0, ctypes.byref(n), ctypes.byref(inner), op) == 1  # cap 0
    assert lib.cfft_fractal_tree(3, N, 1, Rp, tp, 0, 1, ctypes.byref(n), ctypes.byref(inner), op) == 0
    assert list(out) == [8, 8, 8, 1, 1, 1, 0, 0, 0, 0]


def test_plan_array_entry_points_validate_and_report(cf):
    # cfft_forward_plans / cfft_backward_plans: argument checks, and the first failing
    # plan's status with its index (host-only plans have no device state)
    import numpy as np

    lib = cf.LIB
    N = (16, 16, 16)
    _, ops_s = cf.find_optimal_shift(cf.get_ops(229, 3, N), N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plans = [cf.KRFFTPlan(spec, ops_s, precision=4, device=False) for _ in range(2)]
    hs = (ctypes.c_void_p * 2)(*[p.handle.value for p in plans])
    bufs = (ctypes.c_void_p * 2)(None, None)
    batch = (ctypes.c_int * 2)(1, 1)
    for fn in (lib.cfft_forward_plans, lib.cfft_backward_plans):
        assert fn(0, hs, bufs, bufs, batch, None) == 1
        assert fn(2, None, bufs, bufs, batch, None) == 1
        assert fn(2, hs, bufs, bufs, None, None) == 1
        assert fn(2, hs, bufs, bufs, batch, None) == 1
        assert lib.cfft_last_error().startswith(b"plan 0: ")
    for p in plans:
        p.close()


def test_plan_array_python_wrappers_reach_the_library(cf, monkeypatch):
    # forward_plans / backward_plans build their argument arrays and output tensors and
    # call the library; with host-only plans (and the CUDA-tensor check lifted for CPU
    # tensors) the call reaches cfft_forward_plans and returns plan 0's error
    import torch

    monkeypatch.setattr(cf.KRFFTPlan, "_check_tensor", lambda self, x, kind: None)
    monkeypatch.setattr(cf.KRFFTPlan, "_stream", staticmethod(lambda: ctypes.c_void_p(None)))
    plans, fields = [], []
    for sg, n, prec, B in ((229, 16, 4, 3), (47, 16, 8, 1)):
        N = (n, n, n)
        _, ops_s = cf.find_optimal_shift(cf.get_ops(sg, 3, N), N)
        spec = cf.calc_spectral_asu(ops_s, 3, N)
        p = cf.KRFFTPlan(spec, ops_s, precision=prec, device=False)
        plans.append(p)
        dt = torch.float32 if prec == 4 else torch.float64
        fields.append(torch.zeros(((B,) if B > 1 else ()) + tuple(reversed(p.M)), dtype=dt))
    with pytest.raises(cf.CFFTError) as e:
        cf.forward_plans(plans, fields)
    assert "plan 0: " in str(e.value)
    spectra = [torch.zeros((3, plans[0].n_spec), dtype=torch.complex64), torch.zeros(plans[1].n_spec, dtype=torch.complex128)]
    with pytest.raises(cf.CFFTError) as e:
        cf.backward_plans(plans, spectra)
    assert "plan 0: " in str(e.value)
    with pytest.raises(cf.CFFTError):
        cf.forward_plans(plans, fields[:1])
    for p in plans:
        p.close()
