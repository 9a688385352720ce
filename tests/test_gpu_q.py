"""Q-matrix diffusion step on the device: M2+Q (execute_m2_q!) and M7
(execute_m7_scft!) against the FP64 oracle and the full-grid truth, mirroring
test/runtests.jl:220-287 (M2Q vs full grid 1e-10, M7 vs M2Q 1e-12)."""
import numpy as np
import pytest

from conftest import q_plan, rel_err, oracle_shifted_ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

N16 = (16, 16, 16)
LAT = np.eye(3)
DS = 0.05


def to_dev(f0, precision):
    dt = torch.float64 if precision == 8 else torch.float32
    return torch.tensor(np.asarray(f0).ravel(order="F"), dtype=dt, device="cuda:0").view(*reversed(f0.shape))


def from_dev(t, M):
    return t.detach().cpu().numpy().astype(np.float64).ravel().reshape(M, order="F")


@pytest.mark.parametrize("sg", [47, 225, 229, 221, 227, 230, 63])
def test_m2q_vs_oracle_and_fullgrid(cf, O, prep, sg):
    p = prep(sg, N16)
    plan = q_plan(cf, p, cf.PATH_M2Q, DS, LAT)
    oplan = O.plan_m2_q_ops(p["oops"], N16, DS, LAT)
    f0 = O.pack_stride(p["u"], plan.L)
    q = to_dev(f0, 8)
    cf.execute_m2_q(plan, q)
    got = from_dev(q, plan.M)
    assert np.max(np.abs(got - O.execute_m2_q(oplan, f0))) < 1e-12
    assert np.max(np.abs(got - O.fullgrid_reference(p["u"], N16, DS, LAT, plan.L))) < 1e-10
    plan.close()


@pytest.mark.parametrize("sg", [225, 229, 227, 230, 63])
def test_m7_vs_m2q_and_oracle(cf, O, prep, sg):
    p = prep(sg, N16)
    m7 = q_plan(cf, p, cf.PATH_M7, DS, LAT)
    assert m7.centered
    oplan = O.plan_m2_q_ops(p["oops"], N16, DS, LAT)
    fold = O.plan_centering_fold(m7.centering, m7.M)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    q = to_dev(f0, 8)
    cf.execute_m7_scft(m7, q)
    got = from_dev(q, m7.M)
    assert np.max(np.abs(got - O.execute_m7_scft(oplan, fold, f0))) < 1e-12
    assert np.max(np.abs(got - O.execute_m2_q(oplan, f0))) < 1e-12
    m7.close()


def test_q_step_fp32_batched_64(cf, O, prep):
    # Im-3m 64^3 (M7: H = 16) and Pm-3m 64^3 (M2Q: H = 32), FP32, three fields per call
    for sg, path in ((229, cf.PATH_M7), (221, cf.PATH_M2Q)):
        N = (64, 64, 64)
        p = prep(sg, N, seed=5)
        plan = q_plan(cf, p, path, DS, LAT, precision=4, max_batch=3)
        oplan = O.plan_m2_q_ops(p["oops"], N, DS, LAT)
        f0 = O.pack_stride(p["u"], plan.L)
        fields = [f0, 0.5 * f0, -f0]
        batch = torch.stack([to_dev(f, 4) for f in fields])
        plan.scft_step(batch)
        want = O.execute_m2_q(oplan, f0)
        for i, s in enumerate([1.0, 0.5, -1.0]):
            assert rel_err(from_dev(batch[i], plan.M), s * want) < 1e-5
        plan.close()


def test_q_update_kernel_equals_fresh_plan(cf, O, prep):
    p = prep(229, N16)
    plan = q_plan(cf, p, cf.PATH_M2Q, DS, LAT)
    plan.update_kernel(0.10, LAT)
    fresh = q_plan(cf, p, cf.PATH_M2Q, 0.10, LAT)
    f0 = O.pack_stride(p["u"], plan.L)
    a, b = to_dev(f0, 8), to_dev(f0, 8)
    plan.scft_step(a)
    fresh.scft_step(b)
    assert torch.max(torch.abs(a - b)).item() < 1e-14
    plan.close()
    fresh.close()


def test_q_step_diffusion_vs_oracle(cf, O, prep):
    # step_diffusion! (src/diffusion_solver.jl:254-267) with the Q-fused operator
    p = prep(225, N16)
    plan = q_plan(cf, p, cf.PATH_M7, DS, LAT)
    oplan = O.plan_m2_q_ops(p["oops"], N16, DS, LAT)
    f0 = O.pack_stride(p["u"], plan.L)
    w = O.pack_stride(O.make_symmetric(p["oops"], N16, seed=99), plan.L)
    q = to_dev(f0, 8)
    plan.step_diffusion(q, to_dev(w, 8), 0.02, n_steps=3)
    ref = f0
    for _ in range(3):
        ref = O.step_diffusion(lambda x: O.execute_m2_q(oplan, x), ref, w, 0.02)
    assert np.max(np.abs(from_dev(q, plan.M) - ref)) < 1e-12
    plan.close()


@pytest.mark.parametrize("sg,n", [(47, 16), (47, 32), (123, 16)])
def test_qfused_solver_vs_fullgrid(cf, O, sg, n):
    # test/test_diffusion_solver.jl:52-135: f0 after the operator vs full-grid FFT -> K -> IFFT
    from conftest import to_oracle_ops

    N = (n, n, n)
    solver = cf.plan_diffusion(N, LAT, sg, 3, 0.1, method=":qfused")
    plan = solver.plan
    ops_s = oracle_shifted_ops(cf, sg, N)
    u = O.make_symmetric(to_oracle_ops(O, ops_s), N, seed=2)
    f0 = O.pack_stride(u, plan.L)
    q = to_dev(f0, 8)
    cf.apply_diffusion_operator(solver, q)
    want = O.fullgrid_reference(u, N, 0.1, LAT, plan.L)
    assert np.max(np.abs(from_dev(q, plan.M) - want)) < 1e-10
    plan.close()
