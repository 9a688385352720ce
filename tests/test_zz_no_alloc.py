"""The allocation-free forward entry point (cfft_forward_noalloc).

It serves callers that may not allocate device memory: its scratch and tables live
in a static device array inside the library, so it runs from a host-only plan
(cfft_plan_create_host) with caller-owned input and output buffers.  This file is
collected last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err, oracle_shifted_ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


# Im-3m 128^3 FP32 needs 8 MiB of workspace per field, so 3 fields fit the 32 MiB
# array: a batch of 7 runs as chunks of 3 + 3 + 1 (the offsets of later chunks).
@pytest.mark.parametrize("sg,N,precision,batch", [(229, (128, 128, 128), 4, 3), (229, (128, 128, 128), 4, 7),
                                                   (47, (32, 32, 32), 8, 2), (230, (48, 48, 48), 4, 2)])
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


def test_noalloc_vs_oracle_spectrum(cf, O, prep):
    # Symmetric Im-3m 128^3 fields (seeded combinations of two oracle fields), FP32,
    # 7 fields = 3 chunks of the static array: every field's spectrum against the
    # FP64 truth on the spectral ASU (test/runtests.jl:199-216), on two calls in a row.
    N = (128, 128, 128)
    ps = [prep(229, N, seed=s) for s in (21, 22)]
    ospec = O.calc_spectral_asu(ps[0]["oops"], 3, N)
    bases = np.stack([O.pack_stride(p["u"], [2, 2, 2]) for p in ps])
    truths = np.stack([O.spectrum_on_asu(p["u"], ospec) for p in ps])
    host_plan = cf.KRFFTPlan(ps[0]["spec"], ps[0]["ops_s"], precision=4, max_batch=1, device=False)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        coef = np.random.default_rng(40 + call).standard_normal((7, 2))
        f0 = np.einsum("bk,kxyz->bxyz", coef, bases)
        x = torch.tensor(np.ascontiguousarray(f0.transpose(0, 3, 2, 1)), dtype=torch.float32, device="cuda:0")
        got = torch.full((7, host_plan.n_spec), float("nan"), dtype=torch.complex64, device="cuda:0")
        cf._lib.check(cf.LIB.cfft_forward_noalloc(host_plan.handle, _ptr(x), _ptr(got), 7, stream))
        torch.cuda.synchronize()
        truth = coef @ truths
        err = np.max(np.abs(got.cpu().numpy() - truth), axis=1) / np.max(np.abs(truth), axis=1)
        assert err.max() <= 1e-5, (call, err)
    host_plan.close()


def test_noalloc_rejects_oversize(cf):
    # Im-3m 256^3 FP64 on the plain stride-2 path: one field needs 128^3 complex
    # doubles (32 MiB) of workspace plus tables, more than the static scratch.
    N = (256, 256, 256)
    ops_s = oracle_shifted_ops(cf, 229, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.KRFFTPlan(spec, ops_s, precision=8, path=cf.PATH_M2, device=False)
    dummy = torch.zeros(16, device="cuda:0")
    st = cf.LIB.cfft_forward_noalloc(plan.handle, _ptr(dummy), _ptr(dummy), 1, None)
    assert st == 4
    assert b"static scratch holds" in cf.LIB.cfft_last_error()
    plan.close()
