"""The FP64 oracle of the warm-start network (oracle/sno_oracle.py) on the CPU:
its analytic gradients against central finite differences, the symmetry of its input
features and outputs, and the class table of the retained modes."""
import numpy as np
import pytest

from oracle import krfft_oracle as O
from oracle import sno_oracle as S


def _setup(sg, N, seed=0):
    ops = O.get_ops(sg, 3, N)
    shift, ops_s = O.find_optimal_shift(ops, N)
    a = np.stack([S.features(sg, N, 20.0, 0.4, ops, shift), S.features(sg, N, 14.0, 0.33, ops, shift)])
    return ops_s, a


def test_class_table():
    assert S.N_CLASS == 364
    assert S.mode_class(np.array([0, 0, 0])) == 0
    assert S.mode_class(np.array([3, -5, 1])) == S.mode_class(np.array([-1, 5, -3]))
    assert S.mode_class(np.array([12, 0, 0])) == -1


@pytest.mark.parametrize("sg", [229, 230, 221])
def test_features_and_output_symmetric(sg):
    N = (8, 8, 8)
    ops_s, a = _setup(sg, N)
    out, _ = S.SNO(S.init_params(1)).forward(a)
    X = O._all_coords(N)
    Nv = np.asarray(N)[:, None]
    for op in ops_s:
        y = O._lin_cm(np.mod(op.Rm @ X + op.tv[:, None], Nv), N)
        for fld in (a[0, 7], a[1, 15], out[0, 0], out[1, 1]):
            v = fld.ravel(order="F")
            assert np.max(np.abs(v[y] - v)) < 1e-12


def test_gradients_finite_differences():
    N = (8, 8, 8)
    _, a = _setup(221, N)
    p = S.init_params(1)
    tgt = np.random.default_rng(0).standard_normal((2, 2) + N) * 0.1
    net = S.SNO(p)
    out, c = net.forward(a)
    g = net.backward(out, tgt, c)
    for k, ix in [("lift_W", (2, 9)), ("W0", (11, 18)), ("b2", (12,)), ("S1", (0, 3, 4)), ("S3", (1, 0, 31)),
                  ("p1_W", (8, 17)), ("p2_b", (0,)), ("W3", (5, 7))]:
        eps = 1e-6
        vals = []
        for sgn in (1, -1):
            pp = {kk: v.copy() for kk, v in p.items()}
            pp[k][ix] += sgn * eps
            n2 = S.SNO(pp)
            vals.append(n2.loss(n2.forward(a)[0], tgt))
        fd = (vals[0] - vals[1]) / (2 * eps)
        assert abs(fd - g[k][ix]) <= 1e-6 * max(abs(fd), 1e-3), (k, ix, fd, g[k][ix])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0])
    r = S.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and abs(r[3] + 3.140625) < 1e-12 and r[4] == 0.0
