"""What the trained warm-start network gains over the plain start (no reference
counterpart).

The shipped weights (crystallographicfft.jl_b200/data/sno_warmstart.npy) were trained
on the GPU by crystallographicfft.jl_b200/train_warmstart.py on 64^3 solutions of the
library's SCFT driver.  Here, for the Ia-3d gyroid at 96^3 (f = 0.4, chiN = 20, the
network predicting on the 96^3 grid it was not trained on) and for draws (chiN, f)
outside the training set at 64^3, the solve to a residual of 1e-6 from the network's
prediction must take at most half the time of the solve from the seeded plain start,
and reach the same free energy (|dF| <= 1e-7).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "crystallographicfft.jl_b200", "data", "sno_warmstart.npy")


def _compare(cf, sg, n, chiN, f, reps=2, plain=None):
    from crystallographicfft_b200 import warmstart as ws

    gg = ws.GroupGrid(sg, n)
    plan = cf.KRFFTPlan(gg.spec, gg.ops, N=gg.N, precision=4, max_batch=32)
    model = cf.SpectralNeuralOperator()
    model.load(WEIGHTS)
    ctx = model.bind(plan, sg, gg.shift, 1)
    plain0 = torch.tensor(gg.plain_start(f, chiN, plan.L), dtype=torch.float32, device="cuda")
    best_p, best_l, a, b = None, None, None, None
    for _ in range(reps):
        a = ws.time_to_tol(gg, chiN, f, plain0, warm=False, plain=plain and getattr(ws, plain))
        b = ws.time_to_tol(gg, chiN, f, None, warm=True, predict=lambda: ctx.predict([(chiN, f)])[0])
        best_p = a["seconds"] if best_p is None else min(best_p, a["seconds"])
        best_l = b["seconds"] if best_l is None else min(best_l, b["seconds"])
    for o in (ctx, model, plan):
        o.close()
    return best_p, best_l, a, b


def test_gyroid_96_learned_start_twice_as_fast(cf):
    plain_s, learned_s, a, b = _compare(cf, 230, 96, 20.0, 0.4)
    assert a["converged"] and b["converged"]
    assert a["F"] < 0.99 * 20.0 * 0.4 * 0.6  # ordered, below the disordered melt's F
    assert abs(a["F"] - b["F"]) <= 1e-7, (a["F"], b["F"])
    assert learned_s <= 0.5 * plain_s, (plain_s, learned_s, a, b)


# Draws outside the training set.  The plain start runs the training data's schedule (200
# simple-mixing iterations), which reaches the same structure as the data.
@pytest.mark.parametrize("sg,chiN,f", [(230, 17.3, 0.36), (229, 24.1, 0.33), (230, 26.5, 0.44)])
def test_held_out_draws_64(cf, sg, chiN, f):
    plain_s, learned_s, a, b = _compare(cf, sg, 64, chiN, f, plain="PLAIN_DATA")
    assert a["converged"] and b["converged"]
    assert abs(a["F"] - b["F"]) <= 1e-7, (a["F"], b["F"])
    assert learned_s <= 0.5 * plain_s, (plain_s, learned_s, a, b)


def test_prediction_is_grid_independent(cf):
    # The network's inputs are functions of physical position and its spectral weights are
    # indexed by Miller index, so its predictions on 64^3 (the training grid) and 96^3 are
    # samples of one field: their low-order Fourier coefficients, with each grid's origin
    # shift removed, agree (to the discretisation of the pointwise nonlinearity).
    from crystallographicfft_b200 import warmstart as ws

    coeffs = []
    for n in (64, 96):
        gg = ws.GroupGrid(230, n)
        plan = cf.KRFFTPlan(gg.spec, gg.ops, N=gg.N, precision=4, max_batch=32)
        model = cf.SpectralNeuralOperator()
        model.load(WEIGHTS)
        ctx = model.bind(plan, 230, gg.shift, 1)
        w = ctx.predict([(20.0, 0.4)])[0]
        F = plan.forward(w.contiguous()).cpu().numpy()  # (2, n_spec): w_A, w_B
        idx = np.asarray(gg.spec.idx)
        hc = np.where(idx >= n - n // 2, idx - n, idx)
        low = {}
        for i, h in enumerate(hc):
            if np.dot(h, h) <= 12:
                phase = np.exp(-2j * np.pi * np.dot(h, np.asarray(gg.shift)))
                low[tuple(int(v) for v in h)] = F[0, i] * phase / n ** 3
        coeffs.append(low)
        for o in (ctx, model, plan):
            o.close()
    common = sorted(set(coeffs[0]) & set(coeffs[1]))
    assert len(common) >= 3
    a = np.array([coeffs[0][h] for h in common])
    b = np.array([coeffs[1][h] for h in common])
    assert np.max(np.abs(a - b)) <= 2e-2 * np.max(np.abs(a)), (common, a, b)
