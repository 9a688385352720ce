"""Mixed batches: the autotuner's execution choices and the one-graph multi-plan runner
(crystallographicfft.jl_b200/batch.py; no reference counterpart).

- Every execution choice the autotuner may pick computes the same transform: tuned
  plans against the default plan (FP32, max relative error 1e-5) and the forward
  against the FP64 oracle's full-FFT truth.
- autotune_plan caches its choice: the second call returns the cached entry.
- MultiPlanStep replays the work of plans of different groups and grid edges as one CUDA
  graph; replays reproduce the direct run exactly.
"""
import json

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


@pytest.mark.parametrize("tuning", [dict(lanes=1), dict(lanes=3, chunk_bytes=4 << 20), dict(zr_slots=2),
                                    dict(wide=0), dict(tma=3), dict(cluster=8), dict(cluster=16)])
def test_tuned_plans_agree(cf, O, prep, tuning):
    N = (64, 64, 64)
    p = prep(229, N, seed=12)
    ref = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=20)
    try:
        plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=20, tuning=tuning)
    except cf.CFFTError:
        pytest.skip(f"{tuning} does not apply to this plan on this device")
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn((20,) + tuple(reversed(plan.M)), generator=g, device="cuda")
    Fa, Fb = ref.forward(x), plan.forward(x)
    assert rel_err(Fb.cpu().numpy(), Fa.cpu().numpy()) < 1e-5
    # x is not symmetric: the backward returns its symmetric part, the same for both plans
    assert rel_err(plan.backward(Fb).cpu().numpy(), ref.backward(Fa).cpu().numpy()) < 1e-5
    f0 = O.pack_stride(p["u"], plan.L)
    one = torch.tensor(np.ascontiguousarray(f0.transpose(2, 1, 0)), dtype=torch.float32, device="cuda")
    truth = O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N))
    F1 = plan.forward(one)  # a single field: spectrum (n_spec,), backward (M3, M2, M1)
    assert rel_err(F1.cpu().numpy(), truth) < 1e-5
    assert rel_err(plan.backward(F1).cpu().numpy(), f0.transpose(2, 1, 0)) < 1e-5
    ref.close()
    plan.close()


def test_autotune_caches(cf, prep, tmp_path):
    p = prep(221, (32, 32, 32))
    cache = tmp_path / "tune.json"
    knobs = (("lanes", (1, 2)), ("zr_slots", (2, 4)))
    tu, ms = cf.autotune_plan(p["spec"], p["ops_s"], precision=4, batch=4, op="fwdbwd", reps=2, cache_path=str(cache),
                              knobs=knobs)
    assert ms > 0 and set(tu) == set(cf.KRFFTPlan.TUNING_DEFAULTS)
    assert len(json.load(open(cache))) == 1
    tu2, ms2 = cf.autotune_plan(p["spec"], p["ops_s"], precision=4, batch=4, op="fwdbwd", reps=2,
                                cache_path=str(cache), knobs=knobs)
    assert tu2 == tu and ms2 == ms
    plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=4, tuning=tu)
    plan.close()


def test_multiplan_graph_replay(cf, prep):
    jobs, outs = [], []
    for sg, n, count in ((229, 32, 3), (230, 48, 2), (221, 64, 1)):
        N = (n, n, n)
        p = prep(sg, N)
        plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=count, ds=0.01)
        g = torch.Generator(device="cuda").manual_seed(n)
        q = torch.randn((count,) + tuple(reversed(plan.M)), generator=g, device="cuda")
        w = 0.1 * torch.randn_like(q)
        F = torch.empty((count, plan.n_spec), dtype=torch.complex64, device="cuda")
        qc = torch.empty_like(q)

        def run(plan=plan, q=q, w=w, F=F, qc=qc):
            plan.forward(q, out=F)
            plan.backward(F, out=qc)
            plan.step_diffusion(qc, w, 0.01, 6)

        jobs.append(run)
        outs.append((plan, qc, F))
    for r in jobs:  # direct reference run
        r()
    torch.cuda.synchronize()
    want = [(qc.clone(), F.clone()) for _, qc, F in outs]
    step = cf.MultiPlanStep(jobs)
    for _ in range(3):  # direct run + capture, then two replays
        for _, qc, F in outs:
            qc.zero_()
            F.zero_()
        step()
        torch.cuda.synchronize()
        for (_, qc, F), (wq, wF) in zip(outs, want):
            assert torch.equal(qc, wq) and torch.equal(F, wF)
    assert step.graph is not None and step.kernels_per_run > 0
    for plan, _, _ in outs:
        plan.close()


def test_autotune_path_picks_a_working_decomposition(cf, O, prep, tmp_path):
    # Im-3m 32^3: the centring fold, the plain stride-2 path and the Q-matrix steps all
    # apply; whichever the tuner keeps must give the default plan's spectra and steps.
    N = (32, 32, 32)
    p = prep(229, N, seed=4)
    path, tu, ms = cf.autotune_path(p["spec"], p["ops_s"], N=N, precision=4, batch=4, op="mixed", n_steps=6,
                                    ds=0.01, reps=2, cache_path=str(tmp_path / "t.json"),
                                    knobs=(("lanes", (1, 2)),))
    assert path in cf.batch.PATHS and ms > 0
    ref = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=4, ds=0.01)
    plan = cf.KRFFTPlan(p["spec"], p["ops_s"], precision=4, max_batch=4, ds=0.01, path=path, tuning=tu)
    f0 = O.pack_stride(p["u"], plan.L)
    x = torch.tensor(np.ascontiguousarray(f0.transpose(2, 1, 0)), dtype=torch.float32, device="cuda")
    x = x[None].repeat(4, 1, 1, 1).contiguous()
    assert rel_err(plan.forward(x).cpu().numpy(), ref.forward(x).cpu().numpy()) < 1e-5
    w = 0.1 * x
    qa, qb = x.clone(), x.clone()
    ref.step_diffusion(qa, w, 0.01, 6)
    plan.step_diffusion(qb, w, 0.01, 6)
    assert rel_err(qb.cpu().numpy(), qa.cpu().numpy()) < 1e-5
    ref.close()
    plan.close()
