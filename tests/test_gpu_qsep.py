"""Separable Q-multiply of the M2Q step for Pmmm-like plans (_is_pmmm_like,
_build_separable_data, _q_multiply_separable!, src/q_fused_krfft.jl:431-534,606-667):
twiddle -> WHT8 -> K -> /8 instead of the 8-tap Q-row gather.

It must agree with the generic Q path (CFFT_QSEP=0, read at plan creation) and with the
FP64 oracle's Q-matrix step and the full-grid truth (test/runtests.jl:317-402 bars:
1e-10 against the full grid, 1e-12 against the oracle), and it must not be taken by
groups whose representatives carry fractional (glide/screw) translations
(src/q_fused_krfft.jl:426-429).  Groups: Pmmm, Pm-3m, P4/mmm, Pm-3 and Im-3m."""
import os

import numpy as np
import pytest

from conftest import q_plan, rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DS = 0.05
LAT = np.diag([1.0, 1.3, 0.8])


def to_dev(f0, precision):
    dt = torch.float64 if precision == 8 else torch.float32
    return torch.tensor(np.ascontiguousarray(np.asarray(f0).transpose(2, 1, 0)), dtype=dt, device="cuda:0")


def from_dev(t):
    return t.detach().cpu().numpy().astype(np.float64).transpose(2, 1, 0)


def _generic(cf, p, precision, **kw):
    os.environ["CFFT_QSEP"] = "0"
    try:
        return q_plan(cf, p, cf.PATH_M2Q, DS, LAT, precision=precision, **kw)
    finally:
        del os.environ["CFFT_QSEP"]


@pytest.mark.parametrize("sg", [47, 221, 123, 200, 229])
def test_separable_matches_generic_oracle_and_fullgrid(cf, O, prep, sg):
    N = (32, 32, 32)
    p = prep(sg, N)
    sep = q_plan(cf, p, cf.PATH_M2Q, DS, LAT, precision=8)
    gen = _generic(cf, p, 8)
    assert sep.info.exec_path & 64 and not gen.info.exec_path & 64
    f0 = O.pack_stride(p["u"], sep.L)
    a, b = to_dev(f0, 8), to_dev(f0, 8)
    sep.scft_step(a)
    gen.scft_step(b)
    got = from_dev(a)
    assert np.max(np.abs(got - from_dev(b))) < 1e-13
    oplan = O.plan_m2_q_ops(p["oops"], N, DS, LAT)
    assert np.max(np.abs(got - O.execute_m2_q(oplan, f0))) < 1e-12
    assert np.max(np.abs(got - O.fullgrid_reference(p["u"], N, DS, LAT, sep.L))) < 1e-10
    sep.close()
    gen.close()


def test_separable_fp32_batched_pmmm64(cf, O, prep):
    N = (64, 64, 64)
    p = prep(47, N, seed=4)
    plan = q_plan(cf, p, cf.PATH_M2Q, DS, LAT, precision=4, max_batch=3)
    assert plan.info.exec_path & 64
    f0 = O.pack_stride(p["u"], plan.L)
    x = torch.stack([to_dev(f0, 4), to_dev(0.5 * f0, 4), to_dev(-f0, 4)])
    plan.scft_step(x)
    want = O.execute_m2_q(O.plan_m2_q_ops(p["oops"], N, DS, LAT), f0)
    for i, s in enumerate([1.0, 0.5, -1.0]):
        assert rel_err(from_dev(x[i]), s * want) < 1e-5
    plan.close()


@pytest.mark.parametrize("sg", [70, 230])
def test_nonsymmorphic_use_generic(cf, prep, sg):
    # Fddd, Ia-3d: fractional (glide / screw) translations in the representatives.  (Im-3m's
    # representatives are the eight diagonal operations with translations 0 or -1, so it
    # is Pmmm-like and takes the separable path, as _is_pmmm_like decides.)
    p = prep(sg, (32, 32, 32))
    plan = q_plan(cf, p, cf.PATH_M2Q, DS, np.eye(3), precision=8)
    assert not plan.info.exec_path & 64
    plan.close()


def test_separable_update_kernel(cf, O, prep):
    # update_m2_kernel! (src/q_fused_krfft.jl:1036-1052): the 1-D kernel factors follow
    p = prep(47, (32, 32, 32))
    plan = q_plan(cf, p, cf.PATH_M2Q, DS, LAT, precision=8)
    plan.update_kernel(0.11, LAT)
    fresh = q_plan(cf, p, cf.PATH_M2Q, 0.11, LAT, precision=8)
    f0 = O.pack_stride(p["u"], plan.L)
    a, b = to_dev(f0, 8), to_dev(f0, 8)
    plan.scft_step(a)
    fresh.scft_step(b)
    assert torch.max(torch.abs(a - b)).item() < 1e-14
    plan.close()
    fresh.close()
