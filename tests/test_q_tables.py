"""Q-matrix tables of the M2Q / M7 plans (plan_m2_q, _build_q_matrices!,
src/q_fused_krfft.jl:83-169,182-413) from host-only plans, against the oracle:
gather indices bit-exact, Q first row within 1e-12."""
import numpy as np
import pytest

from conftest import q_plan

N16 = (16, 16, 16)
LAT = np.eye(3)


@pytest.mark.parametrize("sg", [47, 225, 229, 221, 227, 230, 63, 139])
def test_q_tables_match_oracle(cf, O, prep, sg):
    p = prep(sg, N16)
    plan = q_plan(cf, p, cf.PATH_M2Q, 0.05, LAT, device=False)
    Q, gather = plan.q_tables()
    oplan = O.plan_m2_q_ops(p["oops"], N16, 0.05, LAT)
    assert tuple(plan.L) == tuple(oplan.L)
    assert np.array_equal(gather, oplan.gather_idx)
    assert np.max(np.abs(Q - oplan.Q_first_row)) < 1e-12
    plan.close()


def test_q_tables_follow_update_kernel(cf, O, prep):
    # update_m2_kernel! (src/q_fused_krfft.jl:1036-1052) rebuilds Q for the new ds
    p = prep(229, N16)
    lat = np.array([[1.2, 0.0, 0.0], [0.0, 1.2, 0.0], [0.0, 0.0, 1.2]])
    plan = q_plan(cf, p, cf.PATH_M2Q, 0.05, lat, device=False)
    plan.update_kernel(0.11, lat)
    Q, _ = plan.q_tables()
    assert np.max(np.abs(Q - O.plan_m2_q_ops(p["oops"], N16, 0.11, lat).Q_first_row)) < 1e-12
    plan.close()


def test_m7_refuses_p_lattice(cf):
    # plan_m7_scft: "M7 SCFT requires centered lattice (I/F/C/A)" (src/q_fused_krfft.jl:834-838)
    with pytest.raises(cf.CFFTError):
        cf.plan_m7_scft(N16, 221, 3, 0.05, LAT, device=False)


def test_q_tables_refused_on_other_paths(cf, prep):
    p = prep(229, N16)
    plan = cf.KRFFTPlan(p["spec"], p["ops_s"], device=False)
    with pytest.raises(cf.CFFTError):
        plan.q_tables()
    plan.close()
