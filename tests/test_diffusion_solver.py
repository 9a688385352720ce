"""Diffusion-solver helpers (src/matrix_q.jl, src/diffusion_solver.jl:20-80,165-252),
mirroring test/test_matrix_q.jl and test/test_diffusion_solver.jl:6-50 on the host."""
import numpy as np


def test_gradient_term_and_matrix_q(cf):
    # test/test_matrix_q.jl:8-56: P1 4^3, cubic box L = 10, ds = 0.01
    N, L = (4, 4, 4), 10.0
    spec = cf.calc_spectral_asu(1, 3, N)
    kern = cf.calc_gradient_term(N, 0.01, np.eye(3) * L)
    want = np.exp(-(2 * np.pi / L) ** 2 * 0.01)
    assert np.isclose(kern([1, 0, 0]), want)
    Q = cf.calc_matrix_q(spec, kern)
    assert Q.shape == (64, 64)
    i100 = next(i for i in range(64) if cf.get_k_vector(spec, i) == [1, 0, 0])
    assert np.isclose(Q[i100, i100], want) and Q[0, 1] == 0.0
    # p2mm 8^2 (test/test_matrix_q.jl:58-77)
    spec2 = cf.calc_spectral_asu(6, 2, (8, 8))
    Q2 = cf.calc_matrix_q(spec2, cf.calc_gradient_term((8, 8), 0.1, np.eye(2)))
    assert Q2.shape == (spec2.n_spec, spec2.n_spec) and np.all((Q2.diag >= 0) & (Q2.diag <= 1 + 1e-10))


def test_matrix_method_refused(cf):
    # the dense :matrix solver (src/diffusion_solver.jl:20-80) is not part of the device path
    import pytest

    with pytest.raises(cf.CFFTError):
        cf.plan_diffusion((8, 8), np.eye(2), 6, 2, 0.1, method=":matrix")
