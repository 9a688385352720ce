"""The persistent bulk-copy (TMA) plane kernels and their bounded waits.

- Im-3m 128^3 FP32 plans run both plane stages on them (cfft_info.exec_path bits 3, 4);
  the headline parity of that path is tests/test_gpu_headline.py.
- The forward variant with interaction factors serves the Ia-3d 96^3 FP32 diffusion
  step (channel edge 24): step_diffusion! (src/diffusion_solver.jl:254-267) against the
  FP64 oracle.
- Every wait on a copy is bounded: a wait that runs out records CFFT_ERR_TIMEOUT in the
  plan's status word, and later execute calls report it until it is cleared.  The test
  makes a wait run out without any fault: cfft_wait_selftest waits for bytes that no
  copy delivers.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _dev(f0, dtype=torch.float32):
    return torch.tensor(np.ascontiguousarray(np.asarray(f0).transpose(2, 1, 0)), dtype=dtype, device="cuda:0")


def _host(t):
    return t.detach().cpu().numpy().astype(np.float64).transpose(2, 1, 0)


def test_headline_plan_uses_bulk_copy_planes(cf, prep):
    N = (128, 128, 128)
    p = prep(229, N, seed=5)
    plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=2)
    assert plan.info.exec_path & 8  # forward stage (the backward one is opt-in: CFFT_TMA=all)
    plan.close()


def test_step_diffusion_ia3d96_fp32_vs_oracle(cf, O, prep):
    # the E-fused forward plane kernel (channel edge 24) inside the contour step
    N = (96, 96, 96)
    p = prep(230, N, seed=8)
    plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=1, ds=0.02, lattice=np.eye(3) * 3.8)
    assert plan.H == (24, 24, 24) and plan.info.exec_path & 8
    f0 = O.pack_stride(p["u"], plan.L)
    w = 0.3 * O.pack_stride(O.make_symmetric(p["oops"], N, seed=9), plan.L)
    q = _dev(f0)
    plan.step_diffusion(q, _dev(w), 0.02, n_steps=2)
    oplan = O.plan_m2_scft_ops(p["oops"], N, 0.02, np.eye(3) * 3.8)
    ref = f0
    for _ in range(2):
        ref = O.step_diffusion(lambda x: O.execute_m2_scft(oplan, x), ref, w, 0.02)
    assert rel_err(_host(q), ref) < 1e-5
    plan.close()


def test_bounded_wait_timeout_reported(cf, O, prep):
    N = (64, 64, 64)
    p = prep(229, N, seed=3)
    plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert cf.LIB.cfft_plan_device_status(plan.handle, 0) == 0
    cf._lib.check(cf.LIB.cfft_wait_selftest(plan.handle, 2_000_000, stream))  # 2 ms limit
    torch.cuda.synchronize()
    assert cf.LIB.cfft_plan_device_status(plan.handle, 0) == 5
    x = _dev(O.pack_stride(p["u"], plan.L))
    F = torch.empty((1, plan.n_spec), dtype=torch.complex64, device="cuda:0")
    assert cf.LIB.cfft_forward(plan.handle, _ptr(x), _ptr(F), 1, stream) == 5  # reported, nothing launched
    assert cf.LIB.cfft_plan_device_status(plan.handle, 1) == 5                 # read and clear
    assert cf.LIB.cfft_plan_device_status(plan.handle, 0) == 0
    F = plan.forward(x)                                                         # the context is usable
    truth = O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N))
    assert rel_err(F.cpu().numpy().reshape(-1), truth) < 1e-5
    plan.close()
