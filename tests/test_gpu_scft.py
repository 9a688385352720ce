"""The device SCFT driver (cfft_scft_*) against the FP64 SCFT oracle (oracle/scft_oracle.py).

The reference stops at the contour step (step_diffusion!, src/diffusion_solver.jl:254-282;
execute_m2_scft!, src/q_fused_krfft.jl:989-1026); the driver's propagators are batches of
that step.  AB diblock, f = 0.4, chiN = 20, Ns = 100, Ia-3d (No. 230), cubic cell
3.8 b sqrt(N) (= 3.8 sqrt(6) Rg), seeded Gaussian-filtered symmetric start.
Tolerances: FP64 evaluation within 1e-10 of the oracle; converged free energies within
|dF| <= 1e-7 (FP64); the FP32 driver's converged free energy within 5e-6 (about 1e-6
relative, FP32 precision) of the FP64 one.
"""
import numpy as np
import pytest

from oracle import scft_oracle as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

F_A, CHIN, NS = 0.4, 20.0, 100
CELL = 3.8 * np.sqrt(6.0)


def _setup(cf, prep, n, precision, seed=0, **kw):
    N = (n, n, n)
    p = prep(230, N)
    plan = cf.KRFFTPlan(p["spec"], p["ops_s"], N=N, ds=1.0 / NS, lattice=np.eye(3) * CELL, precision=precision,
                        max_batch=2)
    solver = cf.SCFTSolver(plan, F_A, CHIN, NS, **kw)
    orc = S.SCFTOracle(p["oops"], N, F_A, CHIN, NS, np.eye(3) * CELL)
    wA, wB = S.initial_fields(p["oops"], N, plan.L, F_A, CHIN, seed=seed)
    dt = torch.float64 if precision == 8 else torch.float32
    w = torch.tensor(np.stack([wA.transpose(2, 1, 0), wB.transpose(2, 1, 0)]), dtype=dt, device="cuda:0").contiguous()
    return plan, solver, orc, wA, wB, w


def _np(t):
    return t.cpu().numpy().astype(np.float64).transpose(0, 3, 2, 1)


def test_scft_evaluate_matches_oracle(cf, prep):
    plan, solver, orc, wA, wB, w = _setup(cf, prep, 32, 8)
    got = solver.evaluate(w)
    want = orc.evaluate(wA, wB)
    assert abs(got["Q"] - want["Q"]) / want["Q"] < 1e-10
    assert abs(got["F"] - want["F"]) < 1e-10 and abs(got["err"] - want["err"]) < 1e-10
    phi, d = _np(got["phi"]), _np(got["d"])
    assert np.max(np.abs(phi[0] - want["phiA"])) < 1e-10 and np.max(np.abs(phi[1] - want["phiB"])) < 1e-10
    assert np.max(np.abs(d[0] - want["dA"])) < 1e-9 and np.max(np.abs(d[1] - want["dB"])) < 1e-9
    solver.close()
    plan.close()


def test_scft_solve_matches_oracle_fp64(cf, prep):
    plan, solver, orc, wA, wB, w = _setup(cf, prep, 32, 8, tol=1e-7, max_iter=300)
    st = solver.solve(w)
    _, _, ev, it = orc.solve(wA, wB, tol=1e-7, max_iter=300)
    print(f"FP64 32^3: device F={st['F']:.12f} err={st['err']:.2e} it={st['iterations']}; "
          f"oracle F={ev['F']:.12f} err={ev['err']:.2e} it={it}")
    assert st["converged"] and st["err"] < 1e-7
    assert abs(st["F"] - ev["F"]) <= 1e-7
    phi = _np(solver.densities())
    assert np.max(np.abs(phi[0] - ev["phiA"])) < 1e-5
    assert np.max(np.abs(phi[0] + phi[1] - 1.0)) < 1e-6
    solver.close()
    plan.close()


def test_scft_solve_fp32(cf, prep):
    # FP32 fields and propagators, FP64 reductions: the converged free energy against the
    # FP64 oracle's
    plan, solver, orc, wA, wB, w = _setup(cf, prep, 32, 4, tol=1e-6, max_iter=300)
    st = solver.solve(w)
    _, _, ev, it = orc.solve(wA, wB, tol=1e-8, max_iter=400)
    print(f"FP32 32^3: device F={st['F']:.10f} err={st['err']:.2e} it={st['iterations']} conv={st['converged']}; "
          f"oracle F={ev['F']:.10f}")
    assert st["err"] < 1e-5
    assert abs(st["F"] - ev["F"]) <= 5e-6
    solver.close()
    plan.close()
