"""Plan-time symmetry and index geometry: the host-side mirror of the reference's
SymmetryOps / ASU / SpectralIndexing modules (src/symmetry_ops.jl, src/asu.jl,
src/spectral_indexing.jl) and auto_L (src/krfft.jl:225-279).

The arithmetic runs in libcfft_b200's C++ plan layer; this module only marshals
arrays.  Operations are integer Seitz pairs in grid units, x' = R x + t (mod N).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import LIB, CFFTError, check

CENTERING_NAMES = {0: "P", 1: "C", 2: "A", 3: "I", 4: "F"}


@dataclass(frozen=True)
class SymOp:
    """SymOp{D} (src/symmetry_ops.jl:17-20)."""

    R: tuple  # row-major D*D
    t: tuple  # D

    @property
    def dim(self) -> int:
        return len(self.t)

    @property
    def Rm(self) -> np.ndarray:
        return np.asarray(self.R, dtype=np.int64).reshape(self.dim, self.dim)

    @property
    def tv(self) -> np.ndarray:
        return np.asarray(self.t, dtype=np.int64)


def _pack(ops):
    """Pack D-dimensional ops into the C ABI's 3-D slots (R33 = 1, t3 = 0 for D = 2)."""
    n = len(ops)
    R = np.zeros((n, 3, 3), dtype=np.int32)
    t = np.zeros((n, 3), dtype=np.int32)
    for k, op in enumerate(ops):
        D = op.dim
        R[k, :D, :D] = op.Rm
        for d in range(D, 3):
            R[k, d, d] = 1
        t[k, :D] = op.tv
    return R, t


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _Nc(N, dim):
    arr = (ctypes.c_int * 3)(*(list(N) + [1] * (3 - len(N))))
    return arr


def get_ops(sg_num: int, dim: int, N) -> list:
    """get_ops (src/symmetry_ops.jl:51-53): ITA operations in grid units."""
    Nc = _Nc(N, dim)
    n = ctypes.c_int(0)
    check(LIB.cfft_get_ops(sg_num, dim, Nc, 0, ctypes.byref(n), None, None))
    R = np.zeros((n.value, 9), dtype=np.int32)
    t = np.zeros((n.value, 3), dtype=np.int32)
    check(LIB.cfft_get_ops(sg_num, dim, Nc, n.value, ctypes.byref(n), _ptr(R), _ptr(t)))
    out = []
    for k in range(n.value):
        Rk = R[k].reshape(3, 3)[:dim, :dim]
        out.append(SymOp(tuple(int(v) for v in Rk.ravel()), tuple(int(v) for v in t[k, :dim])))
    return out


def available_groups(dim: int = 3) -> list:
    n = LIB.cfft_list_groups(dim, None, 0)
    buf = (ctypes.c_int * n)()
    LIB.cfft_list_groups(dim, buf, n)
    return list(buf)


def apply_op(op: SymOp, x, N):
    """apply_op (src/symmetry_ops.jl:75-78)."""
    return tuple(int(v) for v in np.mod(op.Rm @ np.asarray(x) + op.tv, np.asarray(N)))


def check_shift_invariance(ops, shift, N):
    """check_shift_invariance (src/symmetry_ops.jl:81-94)."""
    s = np.asarray(shift, dtype=np.float64)
    deltas = []
    for op in ops:
        df = (op.Rm.astype(np.float64) @ s - s) * np.asarray(N, dtype=np.float64)
        di = np.rint(df)
        if not np.all(np.abs(df - di) <= 1e-5):
            return False, []
        deltas.append(di.astype(np.int64))
    return True, deltas


def dual_ops(ops):
    """dual_ops (src/symmetry_ops.jl:103-112)."""
    out = []
    for op in ops:
        Rinv = np.rint(np.linalg.inv(op.Rm.astype(np.float64))).astype(np.int64)
        out.append(SymOp(tuple(int(v) for v in Rinv.T.ravel()), tuple([0] * op.dim)))
    return out


def find_optimal_shift(ops, N):
    """find_optimal_shift (src/asu.jl:281-347) -> (shift, shifted_ops)."""
    dim = ops[0].dim
    R, t = _pack(ops)
    shift = np.zeros(3, dtype=np.float64)
    ts = np.zeros_like(t)
    check(LIB.cfft_find_optimal_shift(dim, _Nc(N, dim), len(ops), _ptr(R), _ptr(t),
                                      shift.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(ts)))
    shifted = [SymOp(op.R, tuple(int(v) for v in ts[k, :dim])) for k, op in enumerate(ops)]
    return shift[:dim], shifted


def fractal_tree(ops, N, *, flags=0):
    """build_recursive_tree + collect_leaves (src/fractal_krfft.jl:300-636) in the
    library's plan layer.  Returns (leaves, depths, n_inner): leaves is an int32 array
    (n_leaves, 3, dim) of [grid size, stride, offset] per leaf in collect_leaves order,
    depths the leaves' depths below the root.
    flags: 0 = the current source; 1 = child translations from the half-grid-shifted
    operations, 2 = no centring split (3 = both, the construction of the reference's
    tree survey)."""
    dim = ops[0].dim
    R, t = _pack(ops)
    Nc = _Nc(N, dim)
    n, inner = ctypes.c_int(0), ctypes.c_int(0)
    check(LIB.cfft_fractal_tree(dim, Nc, len(ops), _ptr(R), _ptr(t), int(flags), 0, ctypes.byref(n),
                                ctypes.byref(inner), None))
    out = np.zeros((n.value, 10), dtype=np.int32)
    check(LIB.cfft_fractal_tree(dim, Nc, len(ops), _ptr(R), _ptr(t), int(flags), n.value, ctypes.byref(n),
                                ctypes.byref(inner), _ptr(out)))
    return out[:, :9].reshape(n.value, 3, 3)[:, :, :dim], out[:, 9].copy(), int(inner.value)


def shift_ops_half_grid(ops, N):
    """shift_ops_half_grid (src/fractal_krfft.jl:262-283): the operations with the grid
    origin moved by half a grid step, t' = t + (I - R) b mod N with b = 1/2 in every
    dimension.  The fractal plans of the reference expect fields symmetric under these.
    Raises when a translation becomes fractional (e.g. hexagonal rotations), which the
    grid-unit operations here cannot hold."""
    out = []
    for op in ops:
        D, R = op.dim, op.Rm
        t2 = [2 * int(op.t[d]) + sum((1 if d == j else 0) - int(R[d, j]) for j in range(D)) for d in range(D)]
        if any(v % 2 for v in t2):
            raise CFFTError(1, "shift_ops_half_grid: a shifted translation is not on the grid")
        out.append(SymOp(op.R, tuple((v // 2) % N[d] for d, v in enumerate(t2))))
    return out


def count_special_positions(N, ops) -> int:
    """_count_special_positions_fast (src/asu.jl:372-438)."""
    dim = ops[0].dim
    R, t = _pack(ops)
    return int(LIB.cfft_count_special_positions(dim, _Nc(N, dim), len(ops), _ptr(R), _ptr(t)))


def auto_L(ops_shifted):
    """auto_L (src/krfft.jl:225-279)."""
    dim = ops_shifted[0].dim
    R, t = _pack(ops_shifted)
    L = (ctypes.c_int * 3)()
    check(LIB.cfft_auto_L(dim, len(ops_shifted), _ptr(R), _ptr(t), L))
    return [int(v) for v in L][:dim]


class CenteringType(str, __import__("enum").Enum):
    """CenteringType (src/symmetry_ops.jl:122-131): the lattice centrings as the values
    detect_centering_type returns, so that detect_centering_type(ops, N) == CentI."""

    CentP = "P"
    CentC = "C"
    CentA = "A"
    CentI = "I"
    CentF = "F"


CentP, CentC, CentA, CentI, CentF = (CenteringType.CentP, CenteringType.CentC, CenteringType.CentA,
                                     CenteringType.CentI, CenteringType.CentF)


def convert_op(R, t_frac, N) -> SymOp:
    """convert_op (src/symmetry_ops.jl:38-49) for an operation given by its rotation and
    fractional translation: the translation in grid units, round(t_frac * N), which must
    lie within 1e-5 of a whole number of grid steps."""
    D = len(N)
    Rm = np.asarray(R, dtype=np.float64).reshape(D, D)
    tg = np.asarray(t_frac, dtype=np.float64) * np.asarray(N, dtype=np.float64)
    ti = np.rint(tg)
    if not np.allclose(tg, ti, rtol=0.0, atol=1e-5):
        raise CFFTError(1, f"convert_op: symmetry operation not commensurate with grid {tuple(N)}")
    return SymOp(tuple(int(v) for v in np.rint(Rm).ravel()), tuple(int(v) for v in ti))


def detect_centering_type(ops, N) -> str:
    """detect_centering_type (src/symmetry_ops.jl:133-179): 'P', 'C', 'A', 'I' or 'F'."""
    dim = ops[0].dim
    R, t = _pack(ops)
    c = LIB.cfft_detect_centering(dim, _Nc(N, dim), len(ops), _ptr(R), _ptr(t))
    if c < 0:
        check(1)
    return CENTERING_NAMES[c]


def strip_centering(ops, centering: str, N):
    """strip_centering (src/symmetry_ops.jl:192-222)."""
    D = len(N)
    if centering in ("I", "F"):
        halve = [True] * D
    elif centering == "C":
        halve = [d < 2 for d in range(D)]
    elif centering == "A":
        halve = [d >= 1 for d in range(D)]
    else:
        halve = [False] * D
    Nsub = tuple(N[d] // 2 if halve[d] else N[d] for d in range(D))
    seen, out = set(), []
    for op in ops:
        ts = tuple(int(op.t[d] % Nsub[d]) for d in range(D))
        if (op.R, ts) not in seen:
            seen.add((op.R, ts))
            out.append(SymOp(op.R, ts))
    return out, Nsub


@dataclass
class SpectralIndexing:
    """SpectralIndexing (src/spectral_indexing.jl:9-13): sorted orbit representatives."""

    idx: np.ndarray   # (n_spec, D) 0-based frequency indices
    mult: np.ndarray  # (n_spec,)
    ops: list         # the direct operations the ASU was built from
    N: tuple

    @property
    def n_spec(self) -> int:
        return int(self.idx.shape[0])


def calc_spectral_asu(ops_or_sg, dim: int, N) -> SpectralIndexing:
    """calc_spectral_asu (src/spectral_indexing.jl:22-176, 184-187)."""
    ops = get_ops(ops_or_sg, dim, N) if isinstance(ops_or_sg, (int, np.integer)) else list(ops_or_sg)
    R, t = _pack(ops)
    n = ctypes.c_int(0)
    Nc = _Nc(N, dim)
    check(LIB.cfft_spectral_asu(dim, Nc, len(ops), _ptr(R), _ptr(t), 0, ctypes.byref(n), None, None))
    idx = np.zeros((n.value, 3), dtype=np.int32)
    mult = np.zeros(n.value, dtype=np.int32)
    check(LIB.cfft_spectral_asu(dim, Nc, len(ops), _ptr(R), _ptr(t), n.value, ctypes.byref(n), _ptr(idx), _ptr(mult)))
    return SpectralIndexing(idx[:, :dim].astype(np.int64), mult.astype(np.int64), ops, tuple(N))


def get_k_vector(spec: SpectralIndexing, i: int):
    """get_k_vector (src/spectral_indexing.jl:195-238) for the 0-based point i: frequency
    v >= N - N div 2 maps to v - N, i.e. [-N/2, N/2) for even N (the reference's code maps
    N/2 to -N/2, whatever its docstring says)."""
    if i < 0 or i >= spec.n_spec:
        raise IndexError(f"Index {i} out of bounds for SpectralIndexing with {spec.n_spec} points")
    out = []
    for d, n in enumerate(spec.N):
        v = int(spec.idx[i, d])
        out.append(v - n if v >= n - n // 2 else v)
    return out


# ---------------------------------------------------------------------------
# Mirror / glide adaptation data (src/mirror_table.jl:14-285)
# ---------------------------------------------------------------------------


@dataclass
class MirrorAdaptationEntry:
    """MirrorAdaptationEntry (src/mirror_table.jl:14-26), computed from the operation table:
    up to three mutually orthogonal mirror/glide planes, the centring and the reduction
    factors of a DCT-style mirror adaptation."""

    n_mirrors: int
    normals: list          # integer plane normals (null vector of R + I)
    translations: list     # fractional (Fraction) translation of the first op per normal
    centering: str         # P, I, F, C, A, B, R
    centering_vecs: list   # fractional centring translations
    all_axial: bool
    det_T: int
    mirror_reduction: int
    centering_multiplier: int
    effective_reduction: int
    has_glide: bool


def _mirror_normal(R):
    """Null vector of R + I (the -1 eigenvector) from cross products of its rows, as a
    primitive integer vector with the sign the cross product gives."""
    A = R + np.eye(3, dtype=np.int64)
    for a, b in ((0, 1), (0, 2), (1, 2)):
        n = np.cross(A[a], A[b])
        if n.any():
            g = int(np.gcd.reduce(np.abs(n)))
            return n // g
    return None


def _centering_class(vecs):
    from fractions import Fraction

    half, zero = Fraction(1, 2), Fraction(0)
    if not vecs:
        return "P"
    fset = {(zero, half, half), (half, zero, half), (half, half, zero)}
    if len(vecs) >= 3 and fset <= set(vecs):
        return "F"
    if (half, half, half) in vecs:
        return "I"
    for v in vecs:
        if sorted(v) == [zero, half, half]:
            return "C" if v[2] == 0 else ("B" if v[1] == 0 else "A")
    if (Fraction(2, 3), Fraction(1, 3), Fraction(1, 3)) in vecs or (Fraction(1, 3), Fraction(2, 3), Fraction(2, 3)) in vecs:
        return "R"
    return "other"


def get_mirror_adaptation(sg: int) -> MirrorAdaptationEntry:
    """get_mirror_adaptation (src/mirror_table.jl:265) from this library's operation table:
    mirror/glide operations are those with R^2 = I and det R = -1; planes with parallel
    normals keep the first operation in listing order; the kept set is the orthogonal
    triple (else pair, else single) preferring axial normals, as the table's generator
    chooses it."""
    from fractions import Fraction

    N = (12, 12, 12)  # every ITA translation is a multiple of 1/12
    ops = get_ops(sg, 3, N)
    eye = np.eye(3, dtype=np.int64)
    frac = lambda t: tuple(Fraction(int(v) % 12, 12) for v in t)
    cvecs = [frac(op.t) for op in ops if np.array_equal(op.Rm, eye) and any(v % 12 for v in op.t)]
    cent = _centering_class(cvecs)
    mirrors = []
    for op in ops:
        R = op.Rm
        if not np.array_equal(R @ R, eye) or round(np.linalg.det(R)) != -1:
            continue
        n = _mirror_normal(R)
        if n is None or any(not np.cross(n, m[0]).any() for m in mirrors):
            continue
        mirrors.append((n, frac(op.t)))
    score = lambda m: int(np.sum(m[0] == 0))
    best, best_score = [], -1
    for i in range(len(mirrors)):
        for j in range(i + 1, len(mirrors)):
            if np.dot(mirrors[i][0], mirrors[j][0]) != 0:
                continue
            for k in range(j + 1, len(mirrors)):
                if np.dot(mirrors[i][0], mirrors[k][0]) == 0 and np.dot(mirrors[j][0], mirrors[k][0]) == 0:
                    s = score(mirrors[i]) + score(mirrors[j]) + score(mirrors[k])
                    if s > best_score or len(best) < 3:
                        best, best_score = [mirrors[i], mirrors[j], mirrors[k]], s
            if len(best) < 2:
                best, best_score = [mirrors[i], mirrors[j]], score(mirrors[i]) + score(mirrors[j])
        if not best:
            best, best_score = [mirrors[i]], score(mirrors[i])
    normals = [m[0] for m in best]
    all_axial = all(int(np.count_nonzero(n)) == 1 for n in normals)
    # The reference's table carries det_T = 1 in every entry, non-axial normals included,
    # so the effective reduction is mirror_reduction x centring multiplier throughout.
    det_T = 1
    nm = len(best)
    mult = {"F": 4, "I": 2, "C": 2, "A": 2, "B": 2}.get(cent, 1)  # R keeps 1, as the table has it
    return MirrorAdaptationEntry(
        n_mirrors=nm, normals=[[int(v) for v in n] for n in normals], translations=[list(m[1]) for m in best],
        centering=cent, centering_vecs=[list(v) for v in cvecs], all_axial=all_axial, det_T=int(det_T),
        mirror_reduction=2 ** nm, centering_multiplier=mult, effective_reduction=(2 ** nm) * mult // int(det_T),
        has_glide=any(any(x != 0 for x in m[1]) for m in best))


class _MirrorTable(dict):
    """MIRROR_ADAPTATION_TABLE (src/mirror_table.jl:28-259): entries computed on first use."""

    def __missing__(self, sg):
        e = get_mirror_adaptation(int(sg))
        self[sg] = e
        return e


MIRROR_ADAPTATION_TABLE = _MirrorTable()


def needs_dct_path(sg: int) -> bool:
    """needs_dct_path (src/mirror_table.jl:267-278): glide planes auto_L cannot use."""
    e = MIRROR_ADAPTATION_TABLE[sg]
    return e.has_glide and e.n_mirrors >= 1


def needs_basis_change(sg: int) -> bool:
    """needs_basis_change (src/mirror_table.jl:280-285)."""
    return not MIRROR_ADAPTATION_TABLE[sg].all_axial


# ----------------------------------------------------------------------------------
# Choice of the decomposition factor and of the grid (src/optimal_L.jl)
# ----------------------------------------------------------------------------------

_GRID_FOR_TABLES = 24  # every group's translations are whole grid steps at 24 per edge


def _reach(ops, L):
    return {tuple(int(op.t[d]) % L[d] for d in range(len(L))) for op in ops}


def optimal_L_phase1(*args):
    """optimal_L_phase1(ops_shifted) or optimal_L_phase1(sg, dim, N)
    (src/optimal_L.jl:59-104,106-110) -> (L, n_active, n_reachable): L_d = 2 where some
    shifted operation has an odd translation, the subgrids reachable from subgrid 0 are
    {t mod L}, and when they do not cover all prod(L) subgrids L is reduced to the
    largest set of dimensions whose subgrids are all reachable."""
    if len(args) == 3:
        sg, dim, N = args
        _, ops = find_optimal_shift(get_ops(sg, dim, N), N)
    else:
        (ops,) = args
    dim = ops[0].dim
    L = [2 if any(int(op.t[d]) % 2 == 1 for op in ops) else 1 for d in range(dim)]
    n_sub = int(np.prod(L))
    if n_sub == 1:
        return L, 1, 1
    n_reach = len(_reach(ops, L))
    n_active = n_sub // n_reach
    if n_active > 1:  # _optimize_L_for_coverage (src/optimal_L.jl:117-166)
        best, best_prod, best_active, best_reach = [1] * dim, 1, 1, 1
        for mask in range(2 ** dim):
            Lt = [2 if (mask >> d) & 1 and L[d] == 2 else 1 for d in range(dim)]
            ns = int(np.prod(Lt))
            if ns == 1:
                continue
            nr = len(_reach(ops, Lt))
            na = ns // nr
            if na == 1 and (ns > best_prod // max(best_active, 1) or best_active > 1):
                best, best_prod, best_active, best_reach = Lt, ns, 1, nr
        return best, best_active, best_reach
    return L, n_active, n_reach


def _point_rotations(sg, D):
    seen, out = set(), []
    for op in get_ops(sg, D, (_GRID_FOR_TABLES,) * D):
        if op.R not in seen:
            seen.add(op.R)
            out.append(op.Rm)
    return out


def _rotation_order(R):
    Rn = R.copy()
    for n in range(1, 13):
        if np.array_equal(Rn, np.eye(len(R), dtype=R.dtype)):
            return n
        Rn = Rn @ R
    return 1


def optimal_L(sg, D=3):
    """optimal_L (src/optimal_L.jl:194-206): per axis, the lcm of the orders of the
    rotations that move it (2 for a flipped axis of an improper operation), at least 2."""
    import math

    cycles = [[] for _ in range(D)]
    for R in _point_rotations(sg, D):
        if np.array_equal(R, np.eye(D, dtype=R.dtype)):
            continue
        order = _rotation_order(R)
        for d in range(D):
            moved = R[d, d] != 1 or any(R[d, i] != 0 or R[i, d] != 0 for i in range(D) if i != d)
            if moved:
                cycles[d].append(order)
        if round(np.linalg.det(R)) < 0:
            for d in range(D):
                if R[d, d] == -1:
                    cycles[d].append(2)
    return tuple(max(math.lcm(*c), 2) if c else 2 for c in cycles)


def optimal_L_isotropic(sg, D=3):
    """optimal_L_isotropic (src/optimal_L.jl:215-228): the lcm of all rotation orders
    (2 for improper operations), at least 2."""
    import math

    cycles = set()
    for R in _point_rotations(sg, D):
        if np.array_equal(R, np.eye(D, dtype=R.dtype)):
            continue
        cycles.add(_rotation_order(R))
        if round(np.linalg.det(R)) < 0:
            cycles.add(2)
    return max(math.lcm(*cycles), 2) if cycles else 2


def recommended_N(sg, target_N):
    """recommended_N (src/optimal_L.jl:236-246): each edge rounded up to a multiple of
    optimal_L."""
    L = optimal_L(sg, len(target_N))
    return tuple(L[d] * -(-int(target_N[d]) // L[d]) for d in range(len(target_N)))


def group_order(sg, D=3):
    """group_order (src/optimal_L.jl:258-261): |G| with every centring translation."""
    return len(get_ops(sg, D, (_GRID_FOR_TABLES,) * D))


def detect_centering(ops, N):
    """detect_centering (src/recursive_blocks.jl:368-403): 'F' with at least three pure
    translations, one of them a face vector (two halves and a zero); 'I' with a body
    vector (1/2, 1/2, 1/2); 'P' otherwise (C, A and R centrings included)."""
    D = len(N)
    n_cent, body, face = 0, False, False
    for op in ops:
        if not np.array_equal(op.Rm, np.eye(D, dtype=np.int64)) or all(abs(int(v)) < 0.1 for v in op.t):
            continue
        n_cent += 1
        frac = [int(op.t[d]) / N[d] for d in range(D)]
        if all(abs(f - 0.5) < 0.01 for f in frac):
            body = True
        n_half = sum(abs(f - 0.5) < 0.01 for f in frac)
        n_zero = sum(abs(f) < 0.01 for f in frac)
        if n_half == 2 and n_zero == 1:
            face = True
    if face and n_cent >= 3:
        return "F"
    if body and n_cent >= 1:
        return "I"
    return "P"
