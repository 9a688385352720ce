"""The oracle's own space-group operations (oracle/hall_groups.py, Hall symbols) and the
library's table (csrc/spacegroups.cpp, ITA generators) are two independent encodings.

- The oracle's table is pinned on its own to the ITA group orders and to the
  reference's Crystalline-derived mirror/centring table (src/mirror_table.jl:14-285,
  extracted to tests/golden/mirror_table.json).
- The library's table must then equal it, operation set by operation set, for all 230
  space groups and 17 plane groups (get_ops, src/symmetry_ops.jl:38-53).
"""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle import hall_groups as HG

# ITA crystal classes by space-group number range -> point-group order
_CLASSES = [(1, 1, 1), (2, 2, 2), (3, 9, 2), (10, 15, 4), (16, 46, 4), (47, 74, 8), (75, 82, 4), (83, 122, 8),
            (123, 142, 16), (143, 146, 3), (147, 161, 6), (162, 167, 12), (168, 174, 6), (175, 190, 12),
            (191, 194, 24), (195, 199, 12), (200, 220, 24), (221, 230, 48)]
_CENT_MULT = {"P": 1, "A": 2, "B": 2, "C": 2, "I": 2, "R": 3, "F": 4}
_PLANE_ORDERS = {1: 1, 2: 2, 3: 2, 4: 2, 5: 4, 6: 4, 7: 4, 8: 4, 9: 8, 10: 4, 11: 8, 12: 8, 13: 3, 14: 6, 15: 6,
                 16: 6, 17: 12}


def _point_order(sg):
    return next(o for a, b, o in _CLASSES if a <= sg <= b)


def _table():
    return json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mirror_table.json")))


def test_hall_groups_have_ita_orders():
    for sg, sym in HG.HALL_3D.items():
        ops = HG.fractional_ops(sg, 3)
        lat = sym.lstrip("-")[0]
        rots = {tuple(R.ravel()) for R, _ in ops}
        assert len(rots) == _point_order(sg), sg
        assert len(ops) == _point_order(sg) * _CENT_MULT[lat], sg
    for sg in HG.HALL_2D:
        assert len(HG.fractional_ops(sg, 2)) == _PLANE_ORDERS[sg], sg


def _mirror_normal(R):
    """Normal of a mirror/glide (R^2 = I, det R = -1), or None."""
    if not np.array_equal(R @ R, np.eye(3, dtype=int)) or round(np.linalg.det(R)) != -1:
        return None
    A = R + np.eye(3, dtype=int)
    for i, j in ((0, 1), (0, 2), (1, 2)):
        m = np.cross(A[i], A[j])
        if m.any():
            return m
    return None


def test_hall_groups_match_reference_mirror_table():
    table = _table()
    assert len(table) == 230
    for sg in range(1, 231):
        e = table[str(sg)]
        ops = HG.fractional_ops(sg, 3)
        cv = {t for R, t in ops if np.array_equal(R, np.eye(3, dtype=int)) and any(t)}
        assert cv == {tuple(Fraction(x) for x in v) for v in e["centering_vecs"]}, sg
        mirrors = [(m, t) for R, t in ops for m in [_mirror_normal(R)] if m is not None]
        assert len({tuple(np.sign(m[np.flatnonzero(m)[0]]) * m) for m, _ in mirrors}) >= e["n_mirrors"], sg
        for n, tr in zip(e["normals"], e["translations"]):
            want = tuple(Fraction(x) % 1 for x in tr)
            got = {t for m, t in mirrors if not np.cross(m, np.array(n)).any()}
            assert want in got, (sg, n, want, got)


def test_oracle_get_ops_grid_units(O):
    ops = O.get_ops(227, 3, (16, 16, 16))
    assert len(ops) == 192 and all(0 <= v < 16 for op in ops for v in op.t)
    with pytest.raises(ValueError):
        O.get_ops(227, 3, (10, 10, 10))  # quarter translations on a 10-point grid


def test_library_table_equals_oracle_table(cf):
    for dim, groups in ((3, range(1, 231)), (2, range(1, 18))):
        N = (12,) * dim
        for sg in groups:
            lib = {(op.R, tuple(Fraction(v, 12) % 1 for v in op.t)) for op in cf.get_ops(sg, dim, N)}
            ora = {(tuple(int(x) for x in R.ravel()), tuple(v % 1 for v in t)) for R, t in HG.fractional_ops(sg, dim)}
            assert lib == ora, (dim, sg)


@pytest.mark.parametrize("sg", [47, 70, 221, 227, 229, 230, 166, 194])
def test_library_shift_and_tables_on_oracle_ops(cf, O, sg):
    # The library's planner fed the oracle's operations agrees with the oracle's planner.
    N = (24, 24, 24)
    oops = O.get_ops(sg, 3, N)
    shift_o, oops_s = O.find_optimal_shift(oops, N)
    shift_l, ops_s = cf.find_optimal_shift([cf.SymOp(op.R, op.t) for op in oops], N)
    assert np.allclose(shift_o, shift_l)
    assert [op.t for op in ops_s] == [op.t for op in oops_s]
    spec_o = O.calc_spectral_asu(oops_s, 3, N)
    spec_l = cf.calc_spectral_asu(ops_s, 3, N)
    assert np.array_equal(spec_o.idx, spec_l.idx) and np.array_equal(spec_o.mult, spec_l.mult)
