"""The recursive parity tree of the fractal KRFFT plans (build_recursive_tree,
src/fractal_krfft.jl:300-636) and what the reference's own output pins with it.

tests/golden/tree_survey_64.json holds the survey the reference wrote at N = 64^3
(test/debug_tree_output.log, from test/debug_tree.jl): for 163 space groups, |G|, the
centring class, and the tree's reduction ratio N^3 / (total leaf volume).  The ratio
depends on every operation's translation, so reproducing it pins the operation tables
(the oracle's Hall-symbol table and the library's ITA-generator table) to the
reference's Crystalline-derived operations.  The survey was written by the reference
version whose tree took child translations from the half-grid-shifted operations and
had no centring split (its centring column is a prediction); the oracle's tree
reproduces that construction with two switches, and follows the current source by
default.
"""
import json
import os

import numpy as np
import pytest

from oracle import fractal_tree as FT

N64 = (64, 64, 64)
LABEL = {1: "P", 2: "I/C/A", 4: "F"}


def _survey():
    return json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tree_survey_64.json")))["groups"]


def _check(ops, row):
    r, _ = FT.reduction_ratio(N64, ops, child_shifted_t=True, centering_split=False)
    ci = FT.centering_index(ops, N64)
    return (len(ops), LABEL.get(ci), round(r, 1), round(r * ci, 1)) == (
        row["G"], row["centering"], row["ratio"], row["ratio_x_cent"])


def test_survey_fixture_covers_163_groups():
    rows = _survey()
    assert len(rows) == 163
    assert sorted(int(s) for s in rows) == list(range(16, 143)) + list(range(195, 231))


def test_oracle_operations_reproduce_reference_survey(O):
    bad = [sg for sg, row in _survey().items() if not _check(O.get_ops(int(sg), 3, N64), row)]
    assert not bad, bad


def test_library_operations_reproduce_reference_survey(cf, O):
    bad = []
    for sg, row in _survey().items():
        ops = [O.SymOp(op.R, op.t) for op in cf.get_ops(int(sg), 3, N64)]
        if not _check(ops, row):
            bad.append(sg)
    assert not bad, bad


def test_reference_tree_assertions(O):
    # test/test_fractal_krfft.jl:69-80: P1 is not decomposed
    ident = O.SymOp((1, 0, 0, 0, 1, 0, 0, 0, 1), (0, 0, 0))
    root = FT.build_recursive_tree((8, 8, 8), [ident])
    assert root.is_leaf and root.subgrid_N == (8, 8, 8)
    assert len(FT.collect_leaves(root)) == 1
    # every leaf is a distinct stride-scale subgrid inside the grid
    for sg in (47, 136, 200, 221, 225, 229):
        leaves = FT.collect_leaves(FT.build_recursive_tree((16, 16, 16), O.get_ops(sg, 3, (16, 16, 16))))
        assert len({(l.scale, l.offset) for l in leaves}) == len(leaves)
        for l in leaves:
            assert all(o < s for o, s in zip(l.offset, l.scale))
            assert all(n * s == 16 for n, s in zip(l.subgrid_N, l.scale))


def _oracle_leaves(O, N, ops, **kw):
    return [(l.subgrid_N, l.scale, l.offset) for l in FT.collect_leaves(FT.build_recursive_tree(N, ops, **kw))]


def _oracle_inner(node):
    return 0 if node.is_leaf else 1 + sum(_oracle_inner(c) for c in node.children)


def _lib_leaves(cf, N, ops, flags):
    arr, _, inner = cf.fractal_tree([cf.SymOp(op.R, op.t) for op in ops], N, flags=flags)
    return [tuple(tuple(int(v) for v in a[k]) for k in range(3)) for a in arr], inner


@pytest.mark.parametrize("sg", [2, 16, 20, 22, 47, 70, 123, 136, 141, 195, 196, 200, 216, 221, 225, 227, 229, 230])
def test_library_tree_equals_oracle(cf, O, sg):
    # the library's plan-layer tree, leaf by leaf (grid, stride, offset, in collect_leaves
    # order), for the current source and for the survey's construction, on the unshifted
    # and the shifted operations
    N = (32, 32, 32)
    ops = O.get_ops(sg, 3, N)
    for o in (ops, O.find_optimal_shift(ops, N)[1]):
        for flags, kw in ((0, {}), (3, dict(child_shifted_t=True, centering_split=False))):
            got, inner = _lib_leaves(cf, N, o, flags)
            assert got == _oracle_leaves(O, N, o, **kw), (sg, flags)
            assert inner == _oracle_inner(FT.build_recursive_tree(N, o, **kw)), (sg, flags)


def test_library_tree_reproduces_reference_survey(cf, O):
    bad = []
    for sg, row in _survey().items():
        lib_ops = cf.get_ops(int(sg), 3, N64)
        arr, _, _ = cf.fractal_tree(lib_ops, N64, flags=3)
        ratio = 64 ** 3 / float(sum(int(a[0][0]) * int(a[0][1]) * int(a[0][2]) for a in arr))
        if round(ratio, 1) != row["ratio"]:
            bad.append(sg)
    assert not bad, bad


def test_fractal_plan_tree(cf, O):
    # FractalCFFTPlan's n_leaves / n_inner (src/fractal_krfft.jl:104-114) on the plan; the
    # P1 tree is a single leaf (test/test_fractal_krfft.jl:69-80)
    N = (16, 16, 16)
    ops = O.get_ops(221, 3, N)
    lib_ops = [cf.SymOp(op.R, op.t) for op in ops]
    tree = cf.build_recursive_tree(N, lib_ops)
    assert [(l.subgrid_N, l.scale, l.offset) for l in cf.collect_leaves(tree)] == _oracle_leaves(O, N, ops)
    assert tree.fft_points() == sum(int(np.prod(l[0])) for l in _oracle_leaves(O, N, ops))
    ident = [cf.SymOp(((1, 0, 0), (0, 1, 0), (0, 0, 1)), (0, 0, 0))]
    p1 = cf.calc_asu_tree((8, 8, 8), ident)
    assert p1.n_leaves == 1 and p1.n_inner == 0 and p1.leaves[0].subgrid_N == (8, 8, 8)


def test_fractal_variant_plans_hold_the_tree(cf, O):
    # plan_fractal_krfft / _v2 / _v3 carry the tree of the operations they were given
    # (host-only plans: the tables, not the device path)
    N = (16, 16, 16)
    oops = O.get_ops(221, 3, N)  # unshifted, as test/test_fractal_krfft.jl passes them
    ops_s = [cf.SymOp(op.R, op.t) for op in oops]
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    want = _oracle_leaves(O, N, oops)
    inner = _oracle_inner(FT.build_recursive_tree(N, oops))
    for make in (cf.plan_fractal_krfft, cf.plan_fractal_krfft_v2, cf.plan_fractal_krfft_v3):
        plan = make(spec, ops_s, device=False)
        assert plan.n_leaves == len(want) and plan.n_inner == inner
        assert [(l.subgrid_N, l.scale, l.offset) for l in plan.tree.leaves] == want
        plan.close()
    plan = cf.plan_krfft_g0asu(spec, ops_s, device=False)
    assert not hasattr(plan, "tree")
    plan.close()


def _oracle_depths(node, d=0):
    return [d] if node.is_leaf else [x for c in node.children for x in _oracle_depths(c, d + 1)]


def test_tree_summary_and_half_grid_shift(cf, O):
    # tree_summary (src/fractal_krfft.jl:653-667) and shift_ops_half_grid
    # (src/fractal_krfft.jl:262-283), against the oracle
    N = (16, 16, 16)
    for sg in (47, 136, 200, 221, 229):
        oops = O.get_ops(sg, 3, N)
        lib = [cf.SymOp(op.R, op.t) for op in oops]
        root = FT.build_recursive_tree(N, oops)
        s = cf.tree_summary(cf.build_recursive_tree(N, lib))
        assert s == dict(n_gp_leaves=len(FT.collect_leaves(root)), n_sp_nodes=_oracle_inner(root),
                         max_depth=max(_oracle_depths(root)))
        sh = cf.shift_ops_half_grid(lib, N)
        want = FT._shift_half(FT._ops_int(oops, 3), N, 3)
        assert [tuple(op.t) for op in sh] == [tuple(v % n for v, n in zip(t, N)) for _, t in want]
        assert [op.R for op in sh] == [op.R for op in lib]
    hexa = [cf.SymOp(op.R, op.t) for op in O.get_ops(168, 3, (12, 12, 12))]
    with pytest.raises(cf.CFFTError):
        cf.shift_ops_half_grid(hexa, (12, 12, 12))
