"""Checks of the persistent bulk-copy (TMA) plane kernels, run by tests/test_gpu_tma.py in
a child process with CFFT_TMA=all (the switch is read once per process).  Exits non-zero
on the first failure.

- Im-3m 128^3 FP32, B = 64: both plane stages on the bulk-copy kernels (cfft_info
  exec_path bits 3 and 4); every field's forward spectrum against FP64 truth and the
  round trip (FP32 max relative error <= 1e-5, test/runtests.jl:199-216).
- Ia-3d 96^3 FP32 diffusion step (the forward kernel with interaction factors, channel
  edge 24): step_diffusion! (src/diffusion_solver.jl:254-267) against the FP64 oracle.
- Bounded waits: cfft_wait_selftest waits for bytes that no copy delivers, so its wait
  runs out and records CFFT_ERR_TIMEOUT in the plan's status; later execute calls report
  it until it is cleared, and the context stays usable.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import torch  # noqa: E402

from conftest import load_package, oracle_group, rel_err  # noqa: E402
from oracle import krfft_oracle as O  # noqa: E402

cf = load_package()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _dev(f0):
    return torch.tensor(np.ascontiguousarray(np.asarray(f0).transpose(2, 1, 0)), dtype=torch.float32, device="cuda:0")


def _host(t):
    return t.detach().cpu().numpy().astype(np.float64).transpose(2, 1, 0)


def headline_batch():
    N = (128, 128, 128)
    _, ops_s, oops = oracle_group(cf, O, 229, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    ospec = O.calc_spectral_asu(oops, 3, N)
    bases, truths = [], []
    for k in range(3):
        u = O.make_symmetric(oops, N, seed=900 + k)
        bases.append(O.pack_stride(u, [2, 2, 2]))
        truths.append(O.spectrum_on_asu(u, ospec))
    bases, truths = np.stack(bases), np.stack(truths)
    B = 64
    plan = cf.KRFFTPlan(spec, ops_s, precision=4, max_batch=B)
    assert plan.info.exec_path & 8 and plan.info.exec_path & 16, plan.info.exec_path
    coef = np.random.default_rng(3).standard_normal((B, 3))
    f0 = np.einsum("bk,kxyz->bxyz", coef, bases)
    x = torch.tensor(np.ascontiguousarray(f0.transpose(0, 3, 2, 1)), dtype=torch.float32, device="cuda:0")
    F = plan.forward(x)
    back = plan.backward(F)
    torch.cuda.synchronize()
    truth = coef @ truths
    fe = np.max(np.abs(F.cpu().numpy() - truth), axis=1) / np.max(np.abs(truth), axis=1)
    be = torch.max(torch.abs(back - x)).item() / torch.max(torch.abs(x)).item()
    print(f"bulk-copy planes, Im-3m 128^3 B={B}: forward max rel err {fe.max():.3e}, round trip {be:.3e}")
    assert fe.max() <= 1e-5 and be <= 1e-5
    plan.close()


def step_ia3d96():
    N = (96, 96, 96)
    _, ops_s, oops = oracle_group(cf, O, 230, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    lat = np.eye(3) * 3.8
    plan = cf.KRFFTPlan(spec, ops_s, precision=4, max_batch=1, ds=0.02, lattice=lat)
    assert plan.H == (24, 24, 24) and plan.info.exec_path & 8
    u = O.make_symmetric(oops, N, seed=8)
    f0 = O.pack_stride(u, plan.L)
    w = 0.3 * O.pack_stride(O.make_symmetric(oops, N, seed=9), plan.L)
    q = _dev(f0)
    plan.step_diffusion(q, _dev(w), 0.02, n_steps=2)
    oplan = O.plan_m2_scft_ops(oops, N, 0.02, lat)
    ref = f0
    for _ in range(2):
        ref = O.step_diffusion(lambda v: O.execute_m2_scft(oplan, v), ref, w, 0.02)
    err = rel_err(_host(q), ref)
    print(f"bulk-copy forward with interaction factors, Ia-3d 96^3 step: rel err {err:.3e}")
    assert err < 1e-5
    plan.close()


def timeout_selftest():
    N = (64, 64, 64)
    _, ops_s, oops = oracle_group(cf, O, 229, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.KRFFTPlan(spec, ops_s, precision=4, max_batch=1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert cf.LIB.cfft_plan_device_status(plan.handle, 0) == 0
    cf._lib.check(cf.LIB.cfft_wait_selftest(plan.handle, 2_000_000, stream))  # 2 ms limit
    torch.cuda.synchronize()
    assert cf.LIB.cfft_plan_device_status(plan.handle, 0) == 5
    u = O.make_symmetric(oops, N, seed=3)
    x = _dev(O.pack_stride(u, plan.L))
    F = torch.empty((1, plan.n_spec), dtype=torch.complex64, device="cuda:0")
    assert cf.LIB.cfft_forward(plan.handle, _ptr(x), _ptr(F), 1, stream) == 5  # reported, nothing launched
    assert cf.LIB.cfft_plan_device_status(plan.handle, 1) == 5                 # read and clear
    assert cf.LIB.cfft_plan_device_status(plan.handle, 0) == 0
    F = plan.forward(x)
    truth = O.spectrum_on_asu(u, O.calc_spectral_asu(oops, 3, N))
    assert rel_err(F.cpu().numpy().reshape(-1), truth) < 1e-5
    print("bounded wait: timeout recorded, reported, cleared; context usable")
    plan.close()


if __name__ == "__main__":
    for fn in (headline_batch, step_ia3d96, timeout_selftest):
        fn()
    print("TMA_CASES_OK")
