"""Host plan layer (C++ via the C ABI) against the oracle: integer tables must be
bit-exact (shift, shifted ops, spectral ASU points / multiplicities / order, L,
centring, representative ops), backward lookup tables must match the oracle's
M2 inverse table, and the generated space-group tables must agree with the
reference's Crystalline-derived mirror/glide table (tests/golden/mirror_table.json)."""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import to_oracle_ops

GROUPS = [1, 2, 10, 16, 25, 35, 47, 62, 63, 69, 70, 71, 72, 74, 75, 99, 123, 136, 139, 200, 221, 223, 224, 225,
          227, 229, 230]

EXPECTED_ORDER = {1: 1, 2: 2, 10: 4, 47: 8, 63: 16, 70: 32, 72: 16, 139: 32, 221: 48, 225: 192, 227: 192,
                  229: 96, 230: 96, 166: 36, 191: 24}


def test_group_orders(cf):
    for sg, n in EXPECTED_ORDER.items():
        N = (12, 12, 12)
        assert len(cf.get_ops(sg, 3, N)) == n


def test_all_table_groups_close(cf):
    assert len(cf.available_groups(3)) >= 130
    for sg in cf.available_groups(3):
        ops = cf.get_ops(sg, 3, (12, 12, 12))
        assert ops[0].R == (1, 0, 0, 0, 1, 0, 0, 0, 1) and ops[0].t == (0, 0, 0)
    for sg in cf.available_groups(2):
        ops = cf.get_ops(sg, 2, (12, 12))
        assert ops[0].R == (1, 0, 0, 1)


def test_not_commensurate(cf):
    with pytest.raises(cf.CFFTError) as e:
        cf.get_ops(227, 3, (10, 10, 10))  # 1/4 translations on a 10-point grid
    assert e.value.status == 3


def test_mirror_table_fixture(cf):
    table = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mirror_table.json")))
    for sg in cf.available_groups(3):
        ops = cf.get_ops(sg, 3, (12, 12, 12))
        e = table[str(sg)]
        cv = {tuple(Fraction(v, 12) for v in op.t) for op in ops
              if np.array_equal(op.Rm, np.eye(3, dtype=int)) and any(op.t)}
        assert cv == {tuple(Fraction(x) for x in v) for v in e["centering_vecs"]}, sg
        for n, tr in zip(e["normals"], e["translations"]):
            found = None
            for op in ops:
                R = op.Rm
                if not np.array_equal(R @ R, np.eye(3, dtype=int)) or round(np.linalg.det(R)) != -1:
                    continue
                A = R + np.eye(3, dtype=int)
                m = np.cross(A[0], A[1])
                if not m.any():
                    m = np.cross(A[0], A[2])
                if not m.any():
                    m = np.cross(A[1], A[2])
                if m.any() and not np.cross(m, np.array(n)).any():
                    found = op
                    break
            assert found is not None, (sg, n)
            assert tuple(Fraction(v, 12) % 1 for v in found.t) == tuple(Fraction(x) % 1 for x in tr), (sg, n)


@pytest.mark.parametrize("sg", GROUPS)
def test_plan_geometry_bit_exact(cf, O, sg):
    N = (16, 16, 16)
    ops = cf.get_ops(sg, 3, N)
    shift, ops_s = cf.find_optimal_shift(ops, N)
    oshift, oops_s = O.find_optimal_shift(to_oracle_ops(O, ops), N)
    assert np.array_equal(shift, oshift)
    assert [(a.R, a.t) for a in ops_s] == [(b.R, b.t) for b in oops_s]
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    ospec = O.calc_spectral_asu(oops_s, 3, N)
    assert np.array_equal(spec.idx, ospec.idx) and np.array_equal(spec.mult, ospec.mult)
    assert cf.auto_L(ops_s) == O.auto_L(oops_s)
    assert cf.detect_centering_type(ops_s, N) == O.detect_centering_type(oops_s, N)
    assert cf.count_special_positions((12, 12, 12), ops_s[:]) >= 0


@pytest.mark.parametrize("sg,N", [(229, (16, 16, 16)), (47, (16, 16, 16)), (230, (16, 16, 16)), (10, (16, 16, 16)),
                                  (225, (16, 16, 16)), (70, (16, 16, 16)), (221, (24, 24, 24)), (229, (24, 24, 24))])
def test_plan_tables_vs_oracle(cf, O, sg, N):
    ops = cf.get_ops(sg, 3, N)
    _, ops_s = cf.find_optimal_shift(ops, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.KRFFTPlan(spec, ops_s, ds=0.05, precision=8, device=False)
    oops = to_oracle_ops(O, ops_s)
    ospec = O.calc_spectral_asu(oops, 3, N)
    idx, mult = plan.spectral_asu()
    assert np.array_equal(idx, ospec.idx) and np.array_equal(mult, ospec.mult)
    L = O.auto_L(oops)
    assert plan.L == L and plan.M == tuple(n // l for n, l in zip(N, L))
    rep = plan.rep_ops()
    orep = O.select_rep_ops(oops, L, N)
    assert [(a.R, a.t) for a in rep] == [(b.R, b.t) for b in orep]
    # centring-fold metadata (plan_krfft_centered / plan_centering_fold)
    ofwd = O.plan_krfft_centered(ospec, oops)
    assert plan.centered == isinstance(ofwd, O.CenteredPlan)
    if plan.centered:
        assert plan.n_channels == ofwd.fold.n_channels and plan.H == ofwd.fold.H
    # backward lookup: per orbit representative and alias, the signed spectral index
    # and the phase must reproduce the oracle's M2 inverse table entry (weight / (1/d)).
    reps, s_tab, p_tab = plan.backward_tables()
    ob = O.plan_m2_backward(ospec, oops)
    d = ob.d
    P = plan.info.P
    for o, q in enumerate(reps):
        for a in range(d):
            s = int(s_tab[o, a])
            if s == 0:
                assert ob.inv_spec[a, q] < 0
                continue
            assert ob.inv_spec[a, q] == abs(s) - 1
            assert bool(ob.inv_conj[a, q]) == (s < 0)
            w = np.exp(2j * np.pi * p_tab[o, a] / P) / d
            assert abs(w - ob.inv_w[a, q]) < 1e-12
    # diffusion kernel K
    assert np.allclose(plan.kernel(), O.kernel_spec(ospec, N, 0.05, np.eye(3)), rtol=0, atol=1e-15)
    plan.close()


def test_orbit_representatives_cover_grid(cf, O):
    """Orbit representatives under the even-translation operations partition the
    alive channel positions exactly once (the device expansion writes each once)."""
    for sg in (229, 225, 47, 230):
        N = (16, 16, 16)
        _, ops_s = cf.find_optimal_shift(cf.get_ops(sg, 3, N), N)
        spec = cf.calc_spectral_asu(ops_s, 3, N)
        plan = cf.KRFFTPlan(spec, ops_s, device=False)
        reps, _, _ = plan.backward_tables()
        assert len(np.unique(reps)) == len(reps)
        assert plan.info.n_orbits == len(reps) > 0
        plan.close()


def test_plan_errors(cf):
    N = (16, 16, 16)
    _, ops_s = cf.find_optimal_shift(cf.get_ops(229, 3, N), N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    with pytest.raises(cf.CFFTError):
        cf.KRFFTPlan(spec, ops_s, precision=3, device=False)
    with pytest.raises(cf.CFFTError):
        cf.KRFFTPlan(spec, ops_s, max_batch=0, device=False)
    plan = cf.KRFFTPlan(spec, ops_s, device=False)
    with pytest.raises(cf.CFFTError) as e:
        plan.forward(np.zeros(plan.M))  # host-only plan has no device state
    assert e.value.status == 1
    plan.close()


def test_mirror_adaptation_table_matches_reference(cf):
    # MIRROR_ADAPTATION_TABLE (src/mirror_table.jl) recomputed from the operation table,
    # field by field against the reference's table (tests/golden/mirror_table.json)
    table = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mirror_table.json")))
    for sg in cf.available_groups(3):
        want, got = table[str(sg)], cf.get_mirror_adaptation(sg)
        assert got.n_mirrors == want["n_mirrors"], sg
        assert got.normals == want["normals"], sg
        assert [[x % 1 for x in t] for t in got.translations] == \
            [[Fraction(x) % 1 for x in t] for t in want["translations"]], sg
        assert got.centering == want["centering"], sg
        assert sorted(map(tuple, got.centering_vecs)) == sorted(tuple(Fraction(x) for x in v) for v in want["centering_vecs"]), sg
        for k in ("all_axial", "det_T", "mirror_reduction", "centering_multiplier", "effective_reduction", "has_glide"):
            assert getattr(got, k) == want[k], (sg, k)
        assert cf.needs_dct_path(sg) == (want["has_glide"] and want["n_mirrors"] >= 1)
        assert cf.needs_basis_change(sg) == (not want["all_axial"])


# ITA crystal classes by space-group number range -> point-group order
_CLASSES = [(1, 1, 1), (2, 2, 2), (3, 9, 2), (10, 15, 4), (16, 46, 4), (47, 74, 8), (75, 82, 4), (83, 122, 8),
            (123, 142, 16), (143, 146, 3), (147, 161, 6), (162, 167, 12), (168, 174, 6), (175, 190, 12),
            (191, 194, 24), (195, 199, 12), (200, 220, 24), (221, 230, 48)]


def test_all_230_groups_orders(cf):
    # get_ops (src/symmetry_ops.jl:51-53) covers every space group, as Crystalline.jl does:
    # distinct rotation parts = the crystal class order, pure translations = the centring
    assert cf.available_groups(3) == list(range(1, 231))
    table = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mirror_table.json")))
    for sg in range(1, 231):
        ops = cf.get_ops(sg, 3, (12, 12, 12))
        pg = next(o for lo, hi, o in _CLASSES if lo <= sg <= hi)
        assert len({op.R for op in ops}) == pg, sg
        n_cent = 1 + len(table[str(sg)]["centering_vecs"])
        assert len(ops) == pg * n_cent, sg


def test_all_17_plane_groups(cf):
    # plane groups 1-17: point-group order per crystal class, centring (c) doubles it
    pg = {1: 1, 2: 2, 3: 2, 4: 2, 5: 2, 6: 4, 7: 4, 8: 4, 9: 4, 10: 4, 11: 8, 12: 8,
          13: 3, 14: 6, 15: 6, 16: 6, 17: 12}
    assert cf.available_groups(2) == list(range(1, 18))
    for sg, order in pg.items():
        ops = cf.get_ops(sg, 2, (12, 12))
        assert len({op.R for op in ops}) == order, sg
        assert len(ops) == order * (2 if sg in (5, 9) else 1), sg


def test_spectral_asu_all_groups_vs_oracle(cf, O):
    # calc_spectral_asu (src/spectral_indexing.jl:22-176) for every space group and
    # plane group on the oracle's own operations: representatives and multiplicities
    # bit-exact.  The library walks each orbit once with the group's distinct rotations.
    for dim, groups, N in ((3, range(1, 231), (24, 24, 24)), (2, range(1, 18), (24, 24))):
        for sg in groups:
            oops = O.get_ops(sg, dim, N)
            _, oops_s = O.find_optimal_shift(oops, N)
            spec = cf.calc_spectral_asu([cf.SymOp(op.R, op.t) for op in oops_s], dim, N)
            ospec = O.calc_spectral_asu(oops_s, dim, N)
            assert np.array_equal(spec.idx, ospec.idx), (dim, sg)
            assert np.array_equal(spec.mult, ospec.mult), (dim, sg)


def test_spectral_asu_large_grids_vs_oracle(cf, O):
    # the sizes of the bench and SCFT workloads: Im-3m 128^3, Ia-3d 96^3, Fd-3m 64^3
    for sg, n in ((229, 128), (230, 96), (227, 64)):
        N = (n, n, n)
        oops = O.get_ops(sg, 3, N)
        _, oops_s = O.find_optimal_shift(oops, N)
        spec = cf.calc_spectral_asu([cf.SymOp(op.R, op.t) for op in oops_s], 3, N)
        ospec = O.calc_spectral_asu(oops_s, 3, N)
        assert np.array_equal(spec.idx, ospec.idx) and np.array_equal(spec.mult, ospec.mult), sg


def test_spectral_asu_open_operation_list(cf):
    # An operation list that is not closed ({I, 4-fold about z} without its powers) keeps
    # the reference's closure walk, so its orbits are those of the cyclic group it
    # generates; with t = 0 no point is extinct either way.
    I = ((1, 0, 0), (0, 1, 0), (0, 0, 1))
    R4 = ((0, -1, 0), (1, 0, 0), (0, 0, 1))
    R2 = ((-1, 0, 0), (0, -1, 0), (0, 0, 1))
    R4i = ((0, 1, 0), (-1, 0, 0), (0, 0, 1))
    N = (12, 12, 6)
    t0 = (0, 0, 0)
    open_list = cf.calc_spectral_asu([cf.SymOp(I, t0), cf.SymOp(R4, t0)], 3, N)
    group = cf.calc_spectral_asu([cf.SymOp(R, t0) for R in (I, R4, R2, R4i)], 3, N)
    assert np.array_equal(open_list.idx, group.idx) and np.array_equal(open_list.mult, group.mult)
    assert int(np.sum(group.mult)) == 12 * 12 * 6


def test_optimal_L_module(cf, O):
    # src/optimal_L.jl: the examples its docstrings give that its code reproduces
    assert cf.optimal_L_phase1(47, 3, (16, 16, 16)) == ([2, 2, 2], 1, 8)
    assert cf.optimal_L_phase1(25, 3, (16, 16, 16)) == ([2, 2, 1], 1, 4)
    assert cf.optimal_L(75, 3) == (4, 4, 2)
    assert cf.optimal_L(47, 3) == (2, 2, 2)  # the code's result; its docstring's (4,4,4) predates the b-shift
    assert cf.group_order(230) == 96
    assert cf.recommended_N(75, (30, 30, 30)) == (32, 32, 30)
    # optimal_L_phase1's L is auto_L's (src/krfft.jl:225-279) for every group, with one
    # active subgrid, and every grid recommended_N returns is a multiple of optimal_L
    N = (24, 24, 24)
    for sg in range(1, 231):
        _, oops = O.find_optimal_shift(O.get_ops(sg, 3, N), N)
        L, n_active, n_reach = cf.optimal_L_phase1([cf.SymOp(op.R, op.t) for op in oops])
        assert L == O.auto_L(oops) and n_active == 1 and n_reach == int(np.prod(L)), sg
        assert cf.group_order(sg) == len(oops)
        Lo = cf.optimal_L(sg)
        assert all(n % l == 0 and n >= 25 for n, l in zip(cf.recommended_N(sg, (25, 25, 25)), Lo))
        assert cf.optimal_L_isotropic(sg) % 2 == 0 or cf.optimal_L_isotropic(sg) % 3 == 0


def test_detect_centering_three_way(cf):
    # detect_centering (src/recursive_blocks.jl:368-403) tells F and I apart and calls
    # every other lattice P; detect_centering_type (src/symmetry_ops.jl:133-179) names all
    N = (24, 24, 24)
    for sg in range(1, 231):
        ops = cf.get_ops(sg, 3, N)
        full = cf.detect_centering_type(ops, N)
        want = full if full in ("F", "I") else "P"
        assert cf.detect_centering(ops, N) == want, (sg, full)


def test_centering_enum_and_convert_op(cf):
    # CenteringType (src/symmetry_ops.jl:122-131) compares with detect_centering_type's
    # result; convert_op (src/symmetry_ops.jl:38-49) scales fractional translations
    N = (16, 16, 16)
    assert cf.detect_centering_type(cf.get_ops(229, 3, N), N) == cf.CentI
    assert cf.detect_centering_type(cf.get_ops(225, 3, N), N) == cf.CentF
    assert cf.detect_centering_type(cf.get_ops(47, 3, N), N) == cf.CentP
    assert [c.value for c in cf.CenteringType] == ["P", "C", "A", "I", "F"]
    op = cf.convert_op(((0, -1, 0), (1, 0, 0), (0, 0, 1)), (0.5, 0.0, 0.25), N)
    assert op == cf.SymOp((0, -1, 0, 1, 0, 0, 0, 0, 1), (8, 0, 4))
    with pytest.raises(cf.CFFTError):
        cf.convert_op(np.eye(3), (1 / 3, 0, 0), N)
    # every operation of the table is convert_op of its own fractional form
    for sg in (2, 70, 167, 227, 230):
        for o in cf.get_ops(sg, 3, (24, 24, 24)):
            assert cf.convert_op(o.Rm, [v / 24 for v in o.t], (24, 24, 24)) == o


def test_backward_tables_all_groups_vs_oracle(cf, O):
    # The plan's backward lookup (_build_spectral_reverse_lookup / _build_inv_recon_table!,
    # src/krfft.jl:997-1255) for every space group at 12^3: per orbit representative and
    # alias, the signed spectral index and the phase of the oracle's M2 inverse table.
    # The library answers each lookup from the orbit minima of k and -k with the
    # reference's first-writer order; the oracle builds the reference's dense table.
    N = (12, 12, 12)
    for sg in range(1, 231):
        oops = O.find_optimal_shift(O.get_ops(sg, 3, N), N)[1]
        ops_s = [cf.SymOp(op.R, op.t) for op in oops]
        spec = cf.calc_spectral_asu(ops_s, 3, N)
        plan = cf.KRFFTPlan(spec, ops_s, precision=8, device=False)
        reps, s_tab, p_tab = plan.backward_tables()
        ospec = O.calc_spectral_asu(oops, 3, N)
        ob = O.plan_m2_backward(ospec, oops)
        P = plan.info.P
        for o, q in enumerate(reps):
            for a in range(ob.d):
                s = int(s_tab[o, a])
                if s == 0:
                    assert ob.inv_spec[a, q] < 0, (sg, o, a)
                    continue
                assert ob.inv_spec[a, q] == abs(s) - 1 and bool(ob.inv_conj[a, q]) == (s < 0), (sg, o, a)
                assert abs(np.exp(2j * np.pi * p_tab[o, a] / P) / ob.d - ob.inv_w[a, q]) < 1e-12, (sg, o, a)
        plan.close()


@pytest.mark.parametrize("sg,n", [(229, 128), (230, 96), (47, 64), (221, 64), (227, 64)])
def test_backward_tables_bench_sizes_vs_oracle(cf, O, sg, n):
    # the backward tables the device path uses at the bench and SCFT sizes (Im-3m 128^3,
    # Ia-3d 96^3, Pmmm / Pm-3m / Fd-3m 64^3), entry by entry against the oracle's dense
    # M2 inverse table
    N = (n, n, n)
    oops = O.find_optimal_shift(O.get_ops(sg, 3, N), N)[1]
    ops_s = [cf.SymOp(op.R, op.t) for op in oops]
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.KRFFTPlan(spec, ops_s, precision=4, device=False)
    reps, s_tab, p_tab = plan.backward_tables()
    ob = O.plan_m2_backward(O.calc_spectral_asu(oops, 3, N), oops)
    reps = np.asarray(reps)
    s = np.asarray(s_tab)
    os_, oc, ow = ob.inv_spec[:, reps].T, ob.inv_conj[:, reps].T, ob.inv_w[:, reps].T
    assert np.all(os_[s == 0] < 0)
    pres = s != 0
    assert np.array_equal(os_[pres], np.abs(s[pres]) - 1)
    assert np.array_equal(oc[pres].astype(bool), s[pres] < 0)
    w = np.exp(2j * np.pi * np.asarray(p_tab) / plan.info.P) / ob.d
    assert np.max(np.abs(w[pres] - ow[pres])) < 1e-12
    plan.close()


def test_concurrent_plan_builds_match_serial(cf):
    # Plans built from several host threads at once (as the warm-start data solves do)
    # get the same tables as serial builds: the planner's per-thread ASU cache and its own
    # worker threads do not mix results between callers.
    import threading

    cases = [(229, 32), (230, 48), (221, 32), (227, 32), (47, 32), (225, 32)]

    def tables(sg, n):
        N = (n, n, n)
        _, ops_s = cf.find_optimal_shift(cf.get_ops(sg, 3, N), N)
        spec = cf.calc_spectral_asu(ops_s, 3, N)
        p = cf.KRFFTPlan(spec, ops_s, precision=4, device=False)
        r = (np.asarray(spec.idx).copy(), *[np.asarray(x).copy() for x in p.backward_tables()])
        p.close()
        return r

    serial = [tables(*c) for c in cases]
    for _ in range(2):
        res = [None] * len(cases)
        ths = [threading.Thread(target=lambda i=i: res.__setitem__(i, tables(*cases[i]))) for i in range(len(cases))]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        for got, want in zip(res, serial):
            assert all(np.array_equal(a, b) for a, b in zip(got, want))


def test_plan_centering_fold_metadata(cf, O):
    # plan_centering_fold (src/centering_fold.jl:60-104): test/test_centering_fold.jl:32-54
    # pins the channel counts; offsets, twiddles and signs against the oracle's fold
    for c, n_ch in (("F", 2), ("I", 4), ("C", 4), ("A", 4)):
        M = (32, 24, 16)
        p = cf.plan_centering_fold(c, M)
        o = O.plan_centering_fold(c, M)
        assert p.n_channels == n_ch == o.n_channels and p.H == o.H == (16, 12, 8)
        assert p.offsets == o.offsets
        for k, off in enumerate(p.offsets):
            t = p.twiddle_1d[k]
            full = t[0][:, None, None] * t[1][None, :, None] * t[2][None, None, :]
            assert np.allclose(full, O._fold_twiddle(o, off), atol=1e-15)
            assert p.sign_table[k] == tuple((-1) ** (off[0] * (i & 1) + off[1] * ((i >> 1) & 1) + off[2] * ((i >> 2) & 1))
                                            for i in range(8))
    assert cf.plan_centering_fold(cf.CentI, (8, 8, 8)).n_channels == 4
    with pytest.raises(cf.CFFTError):
        cf.plan_centering_fold("P", (8, 8, 8))
    with pytest.raises(cf.CFFTError):
        cf.plan_centering_fold("I", (8, 7, 8))


def test_planner_on_random_subgroups_vs_oracle(cf, O):
    # Closed groups outside the standard tables: subgroups generated by two operations of
    # a random space group (seeded), shifted and planned; spectral ASU and backward tables
    # against the oracle's (its dense first-writer table) at 12^3.
    import random

    rng = random.Random(7)
    N = (12, 12, 12)
    ident = O.SymOp((1, 0, 0, 0, 1, 0, 0, 0, 1), (0, 0, 0))

    def compose(a, b):
        Ra, Rb = np.array(a.R).reshape(3, 3), np.array(b.R).reshape(3, 3)
        t = (Ra @ np.array(b.t) + np.array(a.t)) % 12
        return O.SymOp(tuple(int(v) for v in (Ra @ Rb).ravel()), tuple(int(v) for v in t))

    def closure(gens):
        grp, frontier = {(ident.R, ident.t): ident}, [ident]
        while frontier:
            nxt = []
            for a in frontier:
                for b in gens:
                    c = compose(a, b)
                    if (c.R, c.t) not in grp:
                        grp[(c.R, c.t)] = c
                        nxt.append(c)
            frontier = nxt
        return sorted(grp.values(), key=lambda o: (o.R != ident.R, o.R, o.t))

    checked = 0
    for _ in range(40):
        full = O.get_ops(rng.randint(1, 230), 3, N)
        ops = closure(rng.sample(full, min(2, len(full))))
        _, oops = O.find_optimal_shift(ops, N)
        ops_s = [cf.SymOp(op.R, op.t) for op in oops]
        spec = cf.calc_spectral_asu(ops_s, 3, N)
        ospec = O.calc_spectral_asu(oops, 3, N)
        assert np.array_equal(spec.idx, ospec.idx) and np.array_equal(spec.mult, ospec.mult)
        try:
            plan = cf.KRFFTPlan(spec, ops_s, precision=8, device=False)
        except cf.CFFTError:
            continue  # e.g. no representative for some parity class at this grid
        reps, s_tab, p_tab = plan.backward_tables()
        ob = O.plan_m2_backward(ospec, oops)
        reps, s = np.asarray(reps), np.asarray(s_tab)
        os_, oc, ow = ob.inv_spec[:, reps].T, ob.inv_conj[:, reps].T, ob.inv_w[:, reps].T
        assert np.all(os_[s == 0] < 0)
        pres = s != 0
        assert np.array_equal(os_[pres], np.abs(s[pres]) - 1) and np.array_equal(oc[pres].astype(bool), s[pres] < 0)
        w = np.exp(2j * np.pi * np.asarray(p_tab) / plan.info.P) / ob.d
        assert np.max(np.abs(w[pres] - ow[pres]), initial=0.0) < 1e-12
        plan.close()
        checked += 1
    assert checked >= 30
