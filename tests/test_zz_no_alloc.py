"""The allocation-free forward entry point (cfft_forward_noalloc).

It serves callers that may not allocate device memory: its scratch and tables live
in a static device array inside the library, so it runs from a host-only plan
(cfft_plan_create_host) with caller-owned input and output buffers.  This file is
collected last so that a run stopping at the first failure has run everything else.
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


@pytest.mark.parametrize("sg,N,precision,batch", [(229, (128, 128, 128), 4, 3), (47, (32, 32, 32), 8, 2),
                                                   (230, (48, 48, 48), 4, 2)])
def test_noalloc_matches_forward_twice(cf, O, prep, sg, N, precision, batch):
    p = prep(sg, N, seed=3)
    ref_plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=precision, max_batch=batch)
    host_plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=precision, max_batch=1, device=False)
    dev = torch.device("cuda:0")
    rdt = torch.float32 if precision == 4 else torch.float64
    cdt = torch.complex64 if precision == 4 else torch.complex128
    tol = 1e-5 if precision == 4 else 1e-12
    shape = (batch,) + tuple(reversed(ref_plan.M))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):  # two calls in a row: the shared static scratch is reused
        g = torch.Generator(device=dev).manual_seed(100 + call)
        f0 = torch.randn(shape, generator=g, device=dev, dtype=rdt)
        want = ref_plan.forward(f0)
        got = torch.full((batch, ref_plan.n_spec), float("nan"), dtype=cdt, device=dev)
        cf._lib.check(cf.LIB.cfft_forward_noalloc(host_plan.handle, _ptr(f0), _ptr(got), batch, stream))
        torch.cuda.synchronize()
        assert rel_err(got.cpu().numpy(), want.cpu().numpy()) < tol
    ref_plan.close()
    host_plan.close()


def test_noalloc_rejects_oversize(cf):
    # Im-3m 256^3 FP64 on the plain stride-2 path: one field needs 128^3 complex
    # doubles (32 MiB) of workspace plus tables, more than the static scratch.
    N = (256, 256, 256)
    _, ops_s = cf.find_optimal_shift(cf.get_ops(229, 3, N), N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.KRFFTPlan(spec, ops_s, precision=8, path=cf.PATH_M2, device=False)
    dummy = torch.zeros(16, device="cuda:0")
    st = cf.LIB.cfft_forward_noalloc(plan.handle, _ptr(dummy), _ptr(dummy), 1, None)
    assert st == 4
    assert b"static scratch holds" in cf.LIB.cfft_last_error()
    plan.close()
