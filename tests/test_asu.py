"""Real-space ASU, block packing and interleaved orbits (module ASU, src/asu.jl,
src/pack_asu.jl) against the oracle and the reference's own checks (test/runtests.jl:
40-78, test/test_asu.jl, test/test_packing.jl, test/test_interleaved_orbits.jl)."""
import numpy as np
import pytest

from conftest import to_oracle_ops, oracle_shifted_ops


@pytest.mark.parametrize("sg,dim,N", [(6, 2, (8, 8)), (47, 3, (8, 8, 8)), (221, 3, (8, 8, 8)), (229, 3, (8, 8, 8)),
                                      (225, 3, (8, 8, 8)), (230, 3, (8, 8, 8)), (10, 3, (8, 8, 8)),
                                      (63, 3, (8, 8, 8)), (75, 3, (8, 8, 8)), (194, 3, (6, 6, 6)), (1, 3, (4, 4, 4))])
def test_calc_asu_matches_oracle_and_covers_grid(cf, O, sg, dim, N):
    pts, shift = cf.calc_asu(sg, dim, N)
    ops_s = oracle_shifted_ops(cf, sg, N)
    want = O.calc_asu_points(N, to_oracle_ops(O, ops_s))
    assert [(tuple(p.idx), tuple(p.depth), p.multiplicity) for p in pts] == want
    cover = set()
    for p in pts:  # disjoint orbits covering the whole grid (test/test_asu.jl:40-66)
        orb = cf.compute_full_orbit(p.idx, ops_s, N)
        assert not (cover & orb)
        cover |= orb
    assert len(cover) == int(np.prod(N))


def test_reference_asu_sizes(cf):
    # test/runtests.jl:51-66
    assert len(cf.calc_asu(6, 2, (8, 8))[0]) == 16
    pts, shift = cf.calc_asu(47, 3, (8, 8, 8))
    assert len(pts) == 64
    assert np.allclose(cf.calc_asu(6, 2, (8, 8))[1], (0.5 / 8, 0.5 / 8))


@pytest.mark.parametrize("sg,dim,N", [(6, 2, (8, 8)), (7, 2, (8, 8)), (47, 3, (8, 8, 8)), (229, 3, (16, 16, 16))])
def test_pack_asu_covers_points(cf, sg, dim, N):
    # test/runtests.jl:69-78, test/test_packing.jl: every ASU point in exactly one block
    pts, shift = cf.calc_asu(sg, dim, N)
    c = cf.pack_asu(pts, N, shift=shift)
    seen = []
    for eff, blocks in c.dim_blocks.items():
        for b in blocks:
            assert sum(len(r) > 1 for r in b.range) == eff
            seen += [pt for pt in __import__("itertools").product(*b.range)]
    assert sorted(seen) == sorted(tuple(p.idx) for p in pts)


def test_interleaved_orbits_reference_cases(cf):
    # test/test_interleaved_orbits.jl
    N = (16, 16, 16)
    o = cf.analyze_interleaved_orbits(N, [cf.SymOp((1, 0, 0, 0, 1, 0, 0, 0, 1), (0, 0, 0))], L=(2, 2, 2))
    assert len(o) == 8 and all(x.multiplicity == 1 for x in o)
    o = cf.analyze_interleaved_orbits(N, cf.get_ops(75, 3, N), L=(2, 2, 2))
    assert len(o) == 6 and sum(x.multiplicity for x in o) == 8
    assert len([x for x in o if x.multiplicity == 2]) == 2
    o = cf.analyze_interleaved_orbits(N, cf.get_ops(47, 3, N), L=(2, 2, 2))
    assert len(o) == 8 and all(x.multiplicity == 1 for x in o)
    assert len(cf.analyze_interleaved_orbits(N, cf.get_ops(99, 3, N), L=(2, 2, 2))) <= 6


def test_pack_asu_interleaved_gamma0(cf, O):
    N = (16, 16, 16)
    ops_s = oracle_shifted_ops(cf, 229, N)
    u = O.make_symmetric(to_oracle_ops(O, ops_s), N, seed=4)
    c = cf.pack_asu_interleaved(u, N, ops_s, L=(2, 2, 2))
    (b,) = c.dim_blocks[3]
    assert np.array_equal(b.data, u[::2, ::2, ::2]) and b.orbit is None
    c = cf.pack_asu_interleaved(u, N, ops_s, L=(2, 2, 2), asu_only=False)
    assert sum(len(b.orbit.members) for b in c.dim_blocks[3]) == 8


def test_calc_asu_and_special_positions_all_groups(cf, O):
    # calc_asu (src/asu.jl:216-324) and _count_special_positions_fast (src/asu.jl:372-438)
    # for every space group and plane group on the oracle's shifted operations, and at
    # the unshifted ones (special positions on the grid): bit-exact against the oracle.
    # The library walks each orbit once when the operations are closed on the grid.
    # 8^3 for every group whose translations are in quarters and halves, 6^3 for the
    # trigonal and hexagonal ones (thirds and sixths)
    for dim, groups in ((3, range(1, 231)), (2, range(1, 18))):
        for sg in groups:
            n = 6 if (dim == 3 and 143 <= sg <= 194) or (dim == 2 and sg >= 13) else 8
            N = (n,) * dim
            oops = O.get_ops(sg, dim, N)
            _, oops_s = O.find_optimal_shift(oops, N)
            for ops in (oops, oops_s):
                lib_ops = [cf.SymOp(op.R, op.t) for op in ops]
                assert cf.count_special_positions(N, lib_ops) == O.count_special_positions_fast(N, ops), (dim, sg)
            pts = cf.calc_asu(N, [cf.SymOp(op.R, op.t) for op in oops_s])
            want = O.calc_asu_points(N, oops_s)
            assert [(tuple(p.idx), tuple(p.depth), p.multiplicity) for p in pts] == want, (dim, sg)


def test_calc_asu_large_grid(cf, O):
    # Im-3m 24^3: the orbits' sizes add up to the grid and match the oracle
    N = (24, 24, 24)
    oops_s = O.find_optimal_shift(O.get_ops(229, 3, N), N)[1]
    pts = cf.calc_asu(N, [cf.SymOp(op.R, op.t) for op in oops_s])
    assert sum(p.multiplicity for p in pts) == 24 ** 3
    assert [(tuple(p.idx), tuple(p.depth), p.multiplicity) for p in pts] == O.calc_asu_points(N, oops_s)


def test_pack_asu_interleaved_mode_b_cases(cf):
    # test/test_packing_mode_b.jl: P4 at L = 2 packs 6 orbit subgrids, each u[range] with
    # stride 2 starting at its representative; Pmmm packs 8 independent subgrids that
    # cover the grid.  That file calls the default, but the reference's source keeps
    # only the Gamma_0 orbit by default (asu_only = true, src/pack_asu.jl:113-143), so the
    # counts it asserts are those of asu_only = false.
    N = (16, 16, 16)
    u = np.random.default_rng(0).standard_normal(N) + 1j * np.random.default_rng(1).standard_normal(N)
    c = cf.pack_asu_interleaved(u, N, cf.get_ops(75, 3, N), L=(2, 2, 2), asu_only=False)
    blocks = c.dim_blocks[3]
    assert len(blocks) == 6
    for b in blocks:
        assert b.orbit is not None
        assert np.array_equal(b.data, u[tuple(slice(r.start, None, r.step) for r in b.range)])
        assert [r.start for r in b.range] == list(b.orbit.representative)
        assert all(r.step == 2 for r in b.range)
    c = cf.pack_asu_interleaved(u, N, cf.get_ops(47, 3, N), L=(2, 2, 2), asu_only=False)
    blocks = c.dim_blocks[3]
    assert len(blocks) == 8 and all(b.orbit.multiplicity == 1 for b in blocks)
    assert sum(b.data.size for b in blocks) == 16 ** 3
    assert len(cf.pack_asu_interleaved(u, N, cf.get_ops(75, 3, N), L=(2, 2, 2)).dim_blocks[3]) == 1
