"""The SCFT oracle (oracle/scft_oracle.py) against textbook invariants, on CPU.

The reference has no SCFT driver (it stops at step_diffusion!,
src/diffusion_solver.jl:254-282), so the oracle is checked against exact results:
the homogeneous melt (uniform fields: phi_A = f, Q = exp(-(f w_A + (1 - f) w_B)),
F = chiN f (1 - f) at the disordered saddle point), incompressibility and a converged
microphase on a small Ia-3d grid.
"""
import numpy as np
import pytest

from oracle import krfft_oracle as O, scft_oracle as S

N = (16, 16, 16)
CELL = 3.8 * np.sqrt(6.0)


@pytest.fixture(scope="module")
def ia3d():
    _, oops = O.find_optimal_shift(O.get_ops(230, 3, N), N)
    return oops


def test_simpson_weights():
    assert np.allclose(S.simpson_weights(4) * 3, [1, 4, 2, 4, 1])
    assert np.allclose(S.simpson_weights(3), [0.5, 1, 1, 0.5])
    x = np.linspace(0, 1, 41)
    assert abs(np.sum(S.simpson_weights(40) * x ** 3) / 40 - 0.25) < 1e-12


def test_homogeneous_melt_exact(ia3d):
    f, chiN, Ns = 0.4, 20.0, 100
    sc = S.SCFTOracle(ia3d, N, f, chiN, Ns, np.eye(3) * CELL)
    M = tuple(n // 2 for n in N)
    wA, wB = np.full(M, 3.0), np.full(M, -1.5)
    ev = sc.evaluate(wA, wB)
    assert abs(ev["Q"] - np.exp(-(f * 3.0 + (1 - f) * -1.5))) < 1e-12
    assert np.max(np.abs(ev["phiA"] - f)) < 1e-12 and np.max(np.abs(ev["phiB"] - (1 - f))) < 1e-12
    # the disordered saddle point: w_A = chiN (1 - f), w_B = chiN f
    ev = sc.evaluate(np.full(M, chiN * (1 - f)), np.full(M, chiN * f))
    assert ev["err"] < 1e-13 and abs(ev["F"] - chiN * f * (1 - f)) < 1e-12


def test_oracle_converges_to_microphase(ia3d):
    f, chiN = 0.4, 20.0
    sc = S.SCFTOracle(ia3d, N, f, chiN, 100, np.eye(3) * CELL)
    wA, wB = S.initial_fields(ia3d, N, [2, 2, 2], f, chiN, seed=0)
    wA, wB, ev, it = sc.solve(wA, wB, tol=1e-8, max_iter=400)
    assert ev["err"] < 1e-8
    assert np.max(np.abs(ev["phiA"] + ev["phiB"] - 1)) < 1e-6   # incompressible at the saddle point
    assert ev["F"] < chiN * f * (1 - f)                          # below the disordered melt
    assert abs(ev["F"] - ev["F_mf"]) < 1e-7                      # Hamiltonian = mean-field F at the saddle
    assert np.ptp(ev["phiA"]) > 0.5                              # microphase separated
