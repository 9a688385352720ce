"""The reference's variant plans (recursive, sparse, selective, G0-ASU, general G0-ASU,
G0-ASU backward, fractal v1-v3, staged Pm-3m) through their reference names on the
device path, with the reference's own checks: test/runtests.jl:129-166,403-433,
test/test_selective_g0.jl, test/test_general_g0_asu.jl, test/test_g0_asu.jl,
test/test_g0_asu_backward.jl, test/test_fractal_krfft.jl,
test/test_staged_pm3m.jl (spectra against the full FFT of the same field)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

N16 = (16, 16, 16)


def _truth(O, p, N):
    return O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N))


def test_selective_pm3m(cf, O, prep):
    # runtests.jl:129-141: relative error < 1e-12
    p = prep(221, N16)
    plan = cf.plan_krfft_selective(p["spec"], p["ops_s"])
    F = cf.execute_selective_krfft(plan, p["spec"], p["u"])
    assert rel_err(F, _truth(O, p, N16)) < 1e-12
    plan.close()


@pytest.mark.parametrize("sg", [225, 227, 230])
def test_g0asu_vs_fft(cf, O, prep, sg):
    # runtests.jl:143-156,403-433: absolute error < 1e-10
    p = prep(sg, N16)
    plan = cf.plan_krfft_g0asu(p["spec"], p["ops_s"])
    F = cf.execute_g0asu_krfft(plan, p["spec"], p["u"])
    assert np.max(np.abs(F - _truth(O, p, N16))) < 1e-10
    plan.close()


def test_g0asu_backward_roundtrip_im3m(cf, O, prep):
    # runtests.jl:158-166: full grid back within 1e-10
    p = prep(229, N16)
    fplan = cf.plan_krfft_g0asu(p["spec"], p["ops_s"])
    F = cf.execute_g0asu_krfft(fplan, p["spec"], p["u"])
    bplan = cf.plan_krfft_g0asu_backward(p["spec"], p["ops_s"])
    u_out = np.zeros(N16)
    cf.execute_g0asu_ikrfft(bplan, p["spec"], F.copy(), u_out)
    assert np.max(np.abs(p["u"] - u_out)) < 1e-10
    fplan.close()
    bplan.close()


@pytest.mark.parametrize("sg", [221, 225])
def test_sparse_matches_selective(cf, prep, sg):
    # test_selective_g0.jl:70-81
    p = prep(sg, N16)
    a = cf.plan_krfft_sparse(p["spec"], p["ops_s"])
    b = cf.plan_krfft_selective(p["spec"], p["ops_s"])
    Fa = cf.execute_sparse_krfft(a, p["spec"], p["u"])
    Fb = cf.execute_selective_krfft(b, p["spec"], p["u"])
    assert np.max(np.abs(Fa - Fb)) < 1e-10
    a.close()
    b.close()


@pytest.mark.parametrize("sg", [221, 229, 47, 70, 63])
def test_general_g0asu_and_recursive(cf, O, prep, sg):
    # test_general_g0_asu.jl:60-105 (< 1e-9); recursive P3c forward
    p = prep(sg, N16)
    truth = _truth(O, p, N16)
    g = cf.plan_krfft_g0asu_general(p["spec"], p["ops_s"])
    assert rel_err(cf.execute_general_g0asu_krfft(g, p["spec"], p["u"]), truth) < 1e-9
    r = cf.plan_krfft_recursive(p["spec"], p["ops_s"])
    assert rel_err(cf.execute_recursive_krfft(r, p["spec"], p["u"]), truth) < 1e-9
    g.close()
    r.close()


@pytest.mark.parametrize("sg", [47, 221, 225, 229, 227, 230])
def test_fractal_v1_v2_v3(cf, O, prep, sg):
    # test_fractal_krfft.jl (< 1e-10 against the full FFT)
    p = prep(sg, N16)
    truth = _truth(O, p, N16)
    for make, run in ((cf.plan_fractal_krfft, cf.execute_fractal_krfft),
                      (cf.plan_fractal_krfft_v2, cf.execute_fractal_krfft_v2),
                      (cf.plan_fractal_krfft_v3, cf.execute_fractal_krfft_v3)):
        plan = make(p["spec"], p["ops_s"])
        assert np.max(np.abs(run(plan, p["u"]) - truth)) < 1e-10
        plan.close()


def test_variant_on_device_tensors(cf, O, prep):
    # CUDA tensors in and out (full grid (N3, N2, N1), x fastest)
    p = prep(229, N16)
    plan = cf.plan_krfft_g0asu(p["spec"], p["ops_s"])
    u = torch.tensor(p["u"].ravel(order="F"), dtype=torch.float64, device="cuda:0").view(*reversed(N16))
    F = cf.execute_g0asu_krfft(plan, p["spec"], u)
    assert F.is_cuda and np.max(np.abs(F.cpu().numpy() - _truth(O, p, N16))) < 1e-10
    plan.close()


@pytest.mark.parametrize("n", [32, 64])
def test_staged_pm3m(cf, O, n):
    # test_staged_pm3m.jl: F000 vs fft(f000), lookup_full_spectrum vs fft(u), vs G0-ASU
    from conftest import to_oracle_ops

    N = (n, n, n)
    fp = cf.plan_staged_pm3m_full(N)
    u = O.make_symmetric(to_oracle_ops(O, fp.ops_shifted), N, seed=21)
    F000 = cf.execute_staged_full(fp, u)
    assert F000.shape == (n // 2,) * 3
    assert np.max(np.abs(F000 - np.fft.fftn(u[::2, ::2, ::2]))) < 1e-10
    Fu = np.fft.fftn(u)
    rng = np.random.default_rng(0)
    for _ in range(50):
        h = rng.integers(0, n, 3)
        assert abs(cf.lookup_full_spectrum(fp, F000, *h) - Fu[h[0], h[1], h[2]]) < 1e-10
    g = cf.plan_krfft_g0asu(fp.spec, fp.ops_shifted)
    Fg = cf.execute_g0asu_krfft(g, fp.spec, u)
    idx = fp.plan.spectral_asu()[0]
    staged = np.array([cf.lookup_full_spectrum(fp, F000, *h) for h in idx])
    assert np.max(np.abs(staged - Fg)) < 1e-10
    fp.close()
    g.close()
