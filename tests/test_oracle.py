"""The FP64 oracle pinned the way the reference pins itself: against full-grid FFTs
(numpy's pocketfft in place of FFTW) and the reference tests' integer pins.
Mirrors test/runtests.jl, test/test_centering_fold.jl, test/test_centered_backward.jl,
test/test_centered_scft.jl, test/test_m2_scft.jl, test/test_q_fused.jl,
test/test_centering_prefold.jl and test/test_spectral_indexing.jl."""
import numpy as np
import pytest

from conftest import rel_err, to_oracle_ops

N16 = (16, 16, 16)
LAT = np.eye(3)
DS = 0.05


def test_shift_p2mm(cf, O):
    # test/runtests.jl:43-50
    N = (8, 8)
    ops = O.get_ops(6, 2, N)
    shift, _ = O.find_optimal_shift(ops, N)
    assert np.allclose(shift, [0.5 / 8, 0.5 / 8])
    ok, _ = O.check_shift_invariance(ops, shift, N)
    assert ok


def test_centering_classification(cf, O):
    # test/test_centering_prefold.jl:47-54
    N = N16
    expect = {1: "P", 221: "P", 229: "I", 225: "F", 70: "F", 35: "C", 139: "I", 69: "F"}
    for sg, c in expect.items():
        assert O.detect_centering_type(O.get_ops(sg, 3, N), N) == c


def test_strip_centering_counts(cf, O):
    # test/test_centering_prefold.jl:58-75
    N = N16
    sub, Ns = O.strip_centering(O.get_ops(229, 3, N), "I", N)
    assert Ns == (8, 8, 8) and len(sub) == 48
    sub, Ns = O.strip_centering(O.get_ops(225, 3, N), "F", N)
    assert Ns == (8, 8, 8) and len(sub) == 48
    _, Ns = O.strip_centering(O.get_ops(35, 3, N), "C", N)
    assert Ns == (8, 8, 16)


def test_fold_plan_metadata(O):
    # test/test_centering_fold.jl:32-54
    p = O.plan_centering_fold("F", (32, 32, 32))
    assert p.n_channels == 2 and p.H == (16, 16, 16) and p.offsets == [(0, 0, 0), (1, 1, 1)]
    p = O.plan_centering_fold("I", (32, 32, 32))
    assert p.n_channels == 4 and p.offsets == [(0, 0, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)]
    p = O.plan_centering_fold("C", (32, 32, 32))
    assert p.n_channels == 4 and p.H == (16, 16, 16)


def test_spectral_completeness(cf, O):
    # test/test_spectral_indexing.jl:40-70
    spec = O.calc_spectral_asu(O.get_ops(1, 2, (4, 4)), 2, (4, 4))
    assert spec.n_spec == 16 and spec.mult.sum() == 16
    spec = O.calc_spectral_asu(O.get_ops(6, 2, (16, 16)), 2, (16, 16))
    assert spec.mult.sum() == 256
    gamma = [i for i in range(spec.n_spec) if O.get_k_vector(spec, i) == [0, 0]]
    assert len(gamma) == 1 and spec.mult[gamma[0]] == 1


def test_frequency_aliasing(O):
    # test/test_spectral_indexing.jl:74-99
    s4 = O.SpectralIndexing(np.arange(4)[:, None], np.ones(4), [], (4,))
    assert [O.get_k_vector(s4, i) for i in range(4)] == [[0], [1], [-2], [-1]]
    s5 = O.SpectralIndexing(np.arange(5)[:, None], np.ones(5), [], (5,))
    assert [O.get_k_vector(s5, i) for i in range(5)] == [[0], [1], [2], [-2], [-1]]


def test_auto_L_pins(prep, O):
    # test/runtests.jl:224 (Pmmm L = (2,2,2)); :394 (P2/m anisotropic); test/test_auto_L.jl
    # prints L for a list of groups and asserts nothing
    assert O.auto_L(prep(47, N16)["oops"]) == [2, 2, 2]
    assert O.auto_L(prep(10, N16)["oops"]) != [2, 2, 2]


def test_orbit_coverage_pmmm(prep, O):
    # test/runtests.jl:51-66 (Pmmm 8^3: 64 orbits, disjoint, covering)
    p = prep(47, (8, 8, 8))
    assert O.count_special_positions_fast((8, 8, 8), p["oops"]) == 0


def test_fold_fft_vs_direct(prep, O):
    # test/runtests.jl:173-190, test/test_centering_fold.jl:57-87
    for sg, cent in [(229, "I"), (70, "F"), (225, "F"), (63, "C")]:
        p = prep(sg, N16)
        f0 = O.pack_stride(p["u"], [2, 2, 2])
        fp = O.plan_centering_fold(cent, f0.shape)
        G0 = O.assemble_G0(fp, O.fft_channels(O.centering_fold(fp, f0)))
        assert np.max(np.abs(G0 - np.fft.fftn(f0))) < 1e-10


def test_fold_unfold_identity(prep, O):
    # test/runtests.jl:258-270, test/test_m7_scft.jl:34-126 (1e-12)
    p = prep(229, N16)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    fp = O.plan_centering_fold("I", f0.shape)
    back = O.centering_unfold(fp, O.ifft_channels(O.fft_channels(O.centering_fold(fp, f0))))
    assert np.max(np.abs(back - f0)) < 1e-12


@pytest.mark.parametrize("sg", [221, 225, 227, 229, 230, 47, 63, 70, 72, 10])
def test_forward_vs_fft(prep, O, sg):
    # test/runtests.jl:199-216 and :436-476, test/test_krfft_fftw.jl:82-221,
    # test/test_krfft_general.jl:13-160 (centred / M2 forward vs fft(u) on the ASU)
    p = prep(sg, N16)
    spec_o = O.calc_spectral_asu(p["oops"], 3, N16)
    plan = O.plan_krfft_centered(spec_o, p["oops"])
    F = O.execute_centered_krfft(plan, p["u"]) if isinstance(plan, O.CenteredPlan) else O.execute_krfft(plan, p["u"])
    assert np.max(np.abs(F - O.spectrum_on_asu(p["u"], spec_o))) < 1e-8


@pytest.mark.parametrize("sg", [225, 229, 70, 72, 230, 227])
def test_centered_backward_roundtrip(prep, O, sg):
    # test/runtests.jl:290-306, test/test_centered_backward.jl:31-70 (1e-10)
    p = prep(sg, N16)
    spec_o = O.calc_spectral_asu(p["oops"], 3, N16)
    fwd = O.plan_krfft_centered(spec_o, p["oops"])
    bwd = O.plan_centered_ikrfft(spec_o, p["oops"], fwd)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    F = O.fft_reconstruct_centered(fwd, f0)
    assert np.max(np.abs(O.execute_centered_ikrfft(bwd, F) - f0)) < 1e-10
    # spectral consistency fwd∘bwd∘fwd (test/test_centered_backward.jl:74-104)
    F2 = O.fft_reconstruct_centered(fwd, O.execute_centered_ikrfft(bwd, F))
    assert np.max(np.abs(F2 - F)) < 1e-9


@pytest.mark.parametrize("sg", [229, 70, 225, 227, 230, 63])
def test_centered_scft_vs_fullgrid(prep, O, sg):
    # test/runtests.jl:309-320, test/test_centered_scft.jl:57-87 (1e-12)
    p = prep(sg, N16)
    spec_o = O.calc_spectral_asu(p["oops"], 3, N16)
    plan = O.plan_centered_scft(spec_o, p["oops"], N16, DS, LAT)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    out = O.execute_centered_scft(plan, f0)
    ref = O.fullgrid_reference(p["u"], N16, DS, LAT, [2, 2, 2])
    assert np.max(np.abs(out - ref)) < 1e-12


def test_centered_scft_identity_kernel(prep, O):
    # test/test_centered_scft.jl:126-153: Δs = 0 gives the identity
    p = prep(229, N16)
    spec_o = O.calc_spectral_asu(p["oops"], 3, N16)
    plan = O.plan_centered_scft(spec_o, p["oops"], N16, 0.0, LAT)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    assert np.max(np.abs(O.execute_centered_scft(plan, f0) - f0)) < 1e-12


@pytest.mark.parametrize("sg", [221, 225, 227, 230, 10, 47])
def test_m2_scft_vs_fullgrid(prep, O, sg):
    # test/runtests.jl:323-402 (1e-10)
    p = prep(sg, N16)
    plan = O.plan_m2_scft_ops(p["oops"], N16, DS, LAT)
    L = O.auto_L(p["oops"])
    f0 = O.pack_stride(p["u"], L)
    ref = O.fullgrid_reference(p["u"], N16, DS, LAT, L)
    assert np.max(np.abs(O.execute_m2_scft(plan, f0) - ref)) < 1e-10


def test_update_kernel_matches_fresh_plan(prep, O):
    # test/runtests.jl:347-365, test/test_centered_scft.jl:155-182
    p = prep(221, N16)
    plan = O.plan_m2_scft_ops(p["oops"], N16, 0.05, LAT)
    f0 = O.pack_stride(p["u"], O.auto_L(p["oops"]))
    a05 = O.execute_m2_scft(plan, f0)
    plan.K = O.kernel_spec(plan.spec, N16, 0.10, LAT)
    a10 = O.execute_m2_scft(plan, f0)
    b10 = O.execute_m2_scft(O.plan_m2_scft_ops(p["oops"], N16, 0.10, LAT), f0)
    assert np.max(np.abs(a10 - b10)) < 1e-14
    assert np.max(np.abs(a05 - a10)) > 1e-4


@pytest.mark.parametrize("sg", [47, 225])
def test_m2q_vs_fullgrid(prep, O, sg):
    # test/runtests.jl:220-254 (1e-10)
    p = prep(sg, N16)
    plan = O.plan_m2_q_ops(p["oops"], N16, DS, LAT)
    f0 = O.pack_stride(p["u"], plan.L)
    ref = O.fullgrid_reference(p["u"], N16, DS, LAT, plan.L)
    assert np.max(np.abs(O.execute_m2_q(plan, f0) - ref)) < 1e-10


def test_m7_vs_m2q(prep, O):
    # test/runtests.jl:273-287, test/test_m7_scft.jl:131-162 (1e-12)
    p = prep(225, N16)
    plan = O.plan_m2_q_ops(p["oops"], N16, DS, LAT)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    fold = O.plan_centering_fold("F", f0.shape)
    assert np.max(np.abs(O.execute_m7_scft(plan, fold, f0) - O.execute_m2_q(plan, f0))) < 1e-12


def test_fill_map_roundtrip(prep, O):
    # test/test_q_fused.jl:175-197
    p = prep(229, N16)
    L = O.auto_L(p["oops"])
    M = tuple(n // l for n, l in zip(N16, L))
    fm = O.build_fill_map(p["oops"], L, M, N16)
    f0 = O.pack_stride(p["u"], L)
    assert np.max(np.abs(O.subgrid_to_fullgrid(f0, fm, N16) - p["u"])) < 1e-12


def test_m2_backward_first_row_is_alias_mean(prep, O):
    # The per-fiber LU of _build_inv_recon_table! (src/krfft.jl:997-1068) yields the
    # first row of B^-1 = (1/d, ..., 1/d): the aliasing identity the device path uses.
    for sg in (47, 229, 230, 10):
        p = prep(sg, N16)
        spec_o = O.calc_spectral_asu(p["oops"], 3, N16)
        b = O.plan_m2_backward(spec_o, p["oops"])
        lut_s, lut_w, lut_c = O.build_spectral_reverse_lookup(spec_o, p["oops"])
        keep = b.inv_spec >= 0
        assert keep.any()
        # inv_w = x_a * sym_phase with |sym_phase| = 1  =>  |inv_w| = 1/d
        assert np.allclose(np.abs(b.inv_w[keep]), 1.0 / b.d, atol=1e-12)


@pytest.mark.parametrize("sg", [47, 123, 136, 221, 10, 2, 230, 70, 69, 139, 227])
def test_m2_backward_roundtrip(prep, O, sg):
    # test/test_m2_backward.jl:69-156: plan_krfft + fft_reconstruct!, then
    # execute_m2_backward!, recovers the symmetric field's subgrid (max error < 1e-10),
    # for the P groups and the centred groups the reference lists (N = 16 here)
    p = prep(sg, N16)
    spec_o = O.calc_spectral_asu(p["oops"], 3, N16)
    fwd = O.plan_krfft(spec_o, p["oops"])
    bwd = O.plan_m2_backward(spec_o, p["oops"])
    f0 = O.pack_stride(p["u"], O.auto_L(p["oops"]))
    back = O.execute_m2_backward(bwd, O.fft_reconstruct(fwd, f0))
    assert np.max(np.abs(np.real(back).reshape(f0.shape, order="F") - f0)) < 1e-10


def test_oracle_forward_and_roundtrip_all_groups(O):
    # The oracle's own transforms for every space group at 12^3 (its table's operations,
    # shifted by find_optimal_shift): the forward against numpy's full FFT on the spectral
    # ASU (test/runtests.jl:199-216) and the backward round trip to the subgrid
    # (test/test_m2_backward.jl, test/test_centered_backward.jl), each < 1e-9
    N = (12, 12, 12)
    bad = []
    for sg in range(1, 231):
        oops = O.find_optimal_shift(O.get_ops(sg, 3, N), N)[1]
        spec = O.calc_spectral_asu(oops, 3, N)
        u = O.make_symmetric(oops, N, seed=sg)
        fwd = O.plan_krfft_centered(spec, oops)
        if isinstance(fwd, O.CenteredPlan):
            F = O.execute_centered_krfft(fwd, u)
            f0 = O.pack_stride(u, [2, 2, 2])
            back = O.execute_centered_ikrfft(O.plan_centered_ikrfft(spec, oops, fwd), F)
        else:
            F = O.execute_krfft(fwd, u)
            f0 = O.pack_stride(u, O.auto_L(oops))
            back = np.real(O.execute_m2_backward(O.plan_m2_backward(spec, oops), F)).reshape(f0.shape, order="F")
        if np.max(np.abs(F - O.spectrum_on_asu(u, spec))) > 1e-9 or np.max(np.abs(back - f0)) > 1e-9:
            bad.append(sg)
    assert not bad, bad
