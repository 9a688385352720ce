"""The plan-array entry points (cfft_forward_plans / cfft_backward_plans; no reference
counterpart): one library call over plans of different groups, grids and precisions
gives what each plan's own forward and backward give."""
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


def test_plan_array_calls_match_single_plan_calls(cf, prep):
    # cfft_forward_plans / cfft_backward_plans (one library call over an array of plans of
    # different groups, grids and precisions) against the plans' own forward / backward
    cases = [(229, (32, 32, 32), 4, 3), (47, (16, 16, 16), 8, 2), (230, (48, 48, 48), 4, 1)]
    plans, fields = [], []
    g = torch.Generator(device="cuda").manual_seed(5)
    for sg, N, prec, B in cases:
        p = prep(sg, N, seed=7)
        plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=prec, max_batch=B)
        dt = torch.float32 if prec == 4 else torch.float64
        shape = ((B,) if B > 1 else ()) + tuple(reversed(plan.M))
        plans.append(plan)
        fields.append(torch.randn(shape, generator=g, device="cuda", dtype=dt))
    Fs = cf.forward_plans(plans, fields)
    backs = cf.backward_plans(plans, Fs)
    for plan, x, F, b, (_, _, prec, _) in zip(plans, fields, Fs, backs, cases):
        tol = 1e-6 if prec == 4 else 1e-14
        assert rel_err(F.cpu().numpy(), plan.forward(x).cpu().numpy()) <= tol
        assert rel_err(b.cpu().numpy(), plan.backward(F).cpu().numpy()) <= tol
    for plan in plans:
        plan.close()
