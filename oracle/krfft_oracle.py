"""FP64 CPU oracle for the KRFFT / SCFT-diffusion hot path.

TEST INFRASTRUCTURE ONLY.  This module restates, in numpy, the algorithms of
CrystallographicFFT.jl that the B200 library replaces, so that tests, the smoke
check and the CPU-baseline leg of bench.py can check the CUDA path against an
independent implementation.  Nothing in the product imports it.

Parity status: the reference (Julia + FFTW + Crystalline.jl) cannot run in this
environment, so the oracle is pinned (a) against full-grid numpy FFTs exactly as
the reference's own tests pin the reference against FFTW (test/runtests.jl,
test/test_centering_fold.jl, test/test_centered_*.jl, test/test_m2_*.jl,
test/test_q_fused.jl), and (b) against the integer pins those tests hold
(ASU sizes, centering classes, fold metadata, stripped op counts, auto-L).
Its space-group operations come from its own Hall-symbol table (hall_groups.py),
pinned to the reference's Crystalline-derived mirror/centring table
(src/mirror_table.jl, tests/golden/mirror_table.json), to the ITA group orders, and
to the reference's own recursive-tree survey output (test/debug_tree_output.log,
tests/golden/tree_survey_64.json, reproduced through fractal_tree.py for its 163
groups); nothing here loads the library under test.

Layout conventions follow the reference: grids are indexed [x, y, z] with x
fastest in memory (Julia column-major == numpy order='F'); the oracle stores
arrays as numpy arrays of shape (N1, N2, N3) and converts with order='F' when a
flat buffer is needed.  Spectral-ASU vectors are in the reference's sorted
(h1, h2, h3) lexicographic order.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Symmetry operations (src/symmetry_ops.jl)
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class SymOp:
    """Seitz operation in grid units: x' = R x + t (mod N) (src/symmetry_ops.jl:17-20)."""

    R: tuple
    t: tuple

    @property
    def Rm(self):
        return np.array(self.R, dtype=np.int64).reshape(len(self.t), len(self.t))

    @property
    def tv(self):
        return np.array(self.t, dtype=np.int64)


def get_ops(sg, dim, N):
    """get_ops (src/symmetry_ops.jl:51-53) with convert_op (:38-46), from the oracle's own
    Hall-symbol table (oracle/hall_groups.py), independent of the library's table."""
    from . import hall_groups

    return hall_groups.get_ops(sg, dim, tuple(N), SymOp)


def make_op(R, t):
    R = np.asarray(R, dtype=np.int64)
    return SymOp(tuple(int(v) for v in R.ravel()), tuple(int(v) for v in np.asarray(t).ravel()))


def apply_op(op, x, N):
    """apply_op (src/symmetry_ops.jl:61-78)."""
    return tuple(int(v) for v in np.mod(op.Rm @ np.asarray(x) + op.tv, np.asarray(N)))


def check_shift_invariance(ops, shift, N):
    """check_shift_invariance (src/symmetry_ops.jl:81-94)."""
    shift = np.asarray(shift, dtype=np.float64)
    Nv = np.asarray(N, dtype=np.float64)
    deltas = []
    for op in ops:
        df = (op.Rm.astype(np.float64) @ shift - shift) * Nv
        di = np.rint(df)
        if not np.all(np.abs(df - di) <= 1e-5):
            return False, []
        deltas.append(di.astype(np.int64))
    return True, deltas


def dual_ops(ops):
    """dual_ops (src/symmetry_ops.jl:103-112): R* = (R^-1)^T."""
    out = []
    for op in ops:
        Rinv = np.rint(np.linalg.inv(op.Rm.astype(np.float64))).astype(np.int64)
        out.append(make_op(Rinv.T, np.zeros(len(op.t), dtype=np.int64)))
    return out


CENT_P, CENT_C, CENT_A, CENT_I, CENT_F = "P", "C", "A", "I", "F"


def detect_centering_type(ops, N):
    """detect_centering_type (src/symmetry_ops.jl:133-179)."""
    D = len(N)
    pure = []
    for op in ops:
        if not np.array_equal(op.Rm, np.eye(D, dtype=np.int64)):
            continue
        if all(abs(op.t[d]) < 0.1 for d in range(D)):
            continue
        pure.append(tuple(abs(abs(op.t[d]) / N[d] - 0.5) < 0.01 for d in range(D)))
    if not pure or D < 3:
        return CENT_P
    has_xyz = any(all(t) for t in pure)
    has_0yz = any((not t[0]) and t[1] and t[2] for t in pure)
    has_x0z = any(t[0] and (not t[1]) and t[2] for t in pure)
    has_xy0 = any(t[0] and t[1] and (not t[2]) for t in pure)
    if has_0yz + has_x0z + has_xy0 >= 2:
        return CENT_F
    if has_xyz:
        return CENT_I
    if has_xy0:
        return CENT_C
    if has_0yz:
        return CENT_A
    if has_x0z:
        return CENT_A
    return CENT_P


def strip_centering(ops, centering, N):
    """strip_centering (src/symmetry_ops.jl:192-222)."""
    D = len(N)
    if centering in (CENT_I, CENT_F):
        halve = [True] * D
    elif centering == CENT_C:
        halve = [d < 2 for d in range(D)]
    elif centering == CENT_A:
        halve = [d >= 1 for d in range(D)]
    else:
        halve = [False] * D
    Nsub = tuple(N[d] // 2 if halve[d] else N[d] for d in range(D))
    seen, out = set(), []
    for op in ops:
        tsub = tuple(int(np.mod(op.t[d], Nsub[d])) for d in range(D))
        key = (op.R, tsub)
        if key not in seen:
            seen.add(key)
            out.append(SymOp(op.R, tsub))
    return out, Nsub


# ---------------------------------------------------------------------------
# Magic shift (src/asu.jl:281-438)
# ---------------------------------------------------------------------------


def _lin_cm(coords, N):
    """Column-major linear index of integer coords (shape (D, n))."""
    lin = np.zeros(coords.shape[1], dtype=np.int64)
    stride = 1
    for d in range(len(N)):
        lin += coords[d] * stride
        stride *= N[d]
    return lin


def _all_coords(N):
    grids = np.meshgrid(*[np.arange(n, dtype=np.int64) for n in N], indexing="ij")
    return np.stack([g.ravel(order="F") for g in grids])  # column-major enumeration


def count_special_positions_fast(N, ops):
    """_count_special_positions_fast (src/asu.jl:372-438): orbits shorter than |ops|.

    The operations form a group, so every orbit is the set of images of its
    smallest member; the orbit size is the number of points sharing that smallest
    image index.
    """
    X = _all_coords(N)
    Nv = np.asarray(N, dtype=np.int64)[:, None]
    rep = np.arange(X.shape[1], dtype=np.int64)
    for op in ops:
        img = _lin_cm(np.mod(op.Rm @ X + op.tv[:, None], Nv), N)
        np.minimum(rep, img, out=rep)
    sizes = np.bincount(rep, minlength=X.shape[1])
    reps = np.unique(rep)
    return int(np.count_nonzero(sizes[reps] < len(ops)))


def _rescale_ops(ops, N_from, N_to):
    """_rescale_ops (src/asu.jl:355-363): t * N_to ÷ N_from with truncating division."""
    def tdiv(a, b):
        q = abs(a) // abs(b)
        return q if (a >= 0) == (b > 0) else -q

    return [SymOp(op.R, tuple(tdiv(op.t[d] * N_to[d], N_from[d]) for d in range(len(N_to)))) for op in ops]


def _odd_product(ops, D):
    p = 1
    for d in range(D):
        p *= 2 if any(op.t[d] % 2 == 1 for op in ops) else 1
    return p


def find_optimal_shift(ops, N):
    """find_optimal_shift (src/asu.jl:281-347): returns (shift, shifted_ops)."""
    D = len(N)
    Np = tuple([12] * D)
    proxy = _rescale_ops(ops, N, Np)
    cands = [np.zeros(D), np.full(D, 0.5), np.full(D, 1.0 / 3.0), np.full(D, 0.25)]
    best_frac, min_sp = cands[0], None
    for frac in cands:
        shift = frac / np.asarray(Np)
        ok, deltas = check_shift_invariance(proxy, shift, Np)
        if not ok:
            continue
        cur = [SymOp(op.R, tuple(int(v) for v in op.tv + deltas[i])) for i, op in enumerate(proxy)]
        sp = count_special_positions_fast(Np, cur)
        if min_sp is None or sp < min_sp:
            min_sp, best_frac = sp, frac
        if min_sp == 0:
            break
    shift = best_frac / np.asarray(N, dtype=np.float64)
    ok, deltas = check_shift_invariance(ops, shift, N)
    if ok:
        best = [SymOp(op.R, tuple(int(v) for v in op.tv + deltas[i])) for i, op in enumerate(ops)]
    else:
        shift = np.zeros(D)
        best = list(ops)
    half = np.full(D, 0.5) / np.asarray(N, dtype=np.float64)
    okh, dh = check_shift_invariance(ops, half, N)
    if okh:
        oh = [SymOp(op.R, tuple(int(v) for v in op.tv + dh[i])) for i, op in enumerate(ops)]
        if _odd_product(oh, D) > _odd_product(best, D):
            shift, best = half, oh
    return shift, best


# ---------------------------------------------------------------------------
# Spectral ASU (src/spectral_indexing.jl)
# ---------------------------------------------------------------------------


@dataclass
class SpectralIndexing:
    idx: np.ndarray        # (n_spec, D) 0-based representatives
    mult: np.ndarray       # (n_spec,)
    ops: list              # dual ops
    N: tuple

    @property
    def n_spec(self):
        return self.idx.shape[0]


def calc_spectral_asu(direct_ops, dim, N):
    """calc_spectral_asu (src/spectral_indexing.jl:22-176)."""
    D = len(N)
    rec = dual_ops(direct_ops)
    X = _all_coords(N)
    Nv = np.asarray(N, dtype=np.int64)[:, None]
    rep = np.arange(X.shape[1], dtype=np.int64)
    for op in rec:
        np.minimum(rep, _lin_cm(np.mod(op.Rm @ X, Nv), N), out=rep)
    mult = np.bincount(rep, minlength=X.shape[1])
    reps = np.unique(rep)
    K = X[:, reps]                                      # (D, n_orbits)
    stab = np.zeros(reps.size, dtype=np.complex128)
    for g, op in enumerate(rec):
        is_stab = np.all(np.mod(op.Rm @ K - K, Nv) == 0, axis=0)
        phase = np.zeros(reps.size)
        for d in range(D):
            phase += K[d] * direct_ops[g].t[d] / N[d]
        stab += np.where(is_stab, np.exp(-2j * np.pi * phase), 0.0)
    keep = np.abs(stab) > 1e-5
    K, m = K[:, keep], mult[reps[keep]]
    order = np.lexsort(tuple(K[d] for d in reversed(range(D))))
    return SpectralIndexing(K[:, order].T.copy(), m[order].copy(), rec, tuple(N))


def get_k_vector(spec, i):
    """get_k_vector (src/spectral_indexing.jl:195-238), 0-based i: wrap to (-N/2, N/2]."""
    out = []
    for d, n in enumerate(spec.N):
        v = int(spec.idx[i, d])
        out.append(v - n if v >= n - n // 2 else v)
    return out


def k_vectors(spec):
    idx = spec.idx.astype(np.int64)
    Nv = np.asarray(spec.N, dtype=np.int64)
    return np.where(idx >= Nv - Nv // 2, idx - Nv, idx)


# ---------------------------------------------------------------------------
# Stride-L selection (src/krfft.jl:225-279, 958-987)
# ---------------------------------------------------------------------------


def auto_L(ops):
    """auto_L (src/krfft.jl:225-279)."""
    D = len(ops[0].t)
    Lmax = [1] * D
    for op in ops:
        for d in range(D):
            if op.t[d] % 2 == 1:
                Lmax[d] = 2
    n = int(np.prod(Lmax))
    if n <= 1:
        return Lmax
    reach = {tuple(op.t[d] % Lmax[d] for d in range(D)) for op in ops}
    if len(reach) == n:
        return Lmax
    best = [1] * D
    for mask in range(1, 2 ** D):
        Lt = [2 if ((mask >> d) & 1 and Lmax[d] == 2) else 1 for d in range(D)]
        ns = int(np.prod(Lt))
        r = {tuple(op.t[d] % Lt[d] for d in range(D)) for op in ops}
        if len(r) == ns and ns > int(np.prod(best)):
            best = Lt
    return best


def _parity_classes(L):
    """Iterators.product order (first axis fastest)."""
    D = len(L)
    out = []
    for flat in range(int(np.prod(L))):
        x, r = [], flat
        for d in range(D):
            x.append(r % L[d])
            r //= L[d]
        out.append(tuple(x))
    return out


def select_rep_ops(ops, L, N):
    """_select_rep_ops (src/krfft.jl:958-987)."""
    D = len(L)
    reps, qual = {}, {}
    for op in ops:
        x0 = tuple(op.t[d] % L[d] for d in range(D))
        R = op.Rm
        diag = all(R[i, j] == 0 for i in range(D) for j in range(D) if i != j)
        simple = all(op.t[d] % N[d] in (0, N[d] - 1) for d in range(D))
        q = (2 if simple else 1) if diag else 0
        if x0 not in reps or q > qual[x0]:
            reps[x0], qual[x0] = op, q
    out = []
    for x0 in _parity_classes(L):
        if x0 not in reps:
            raise ValueError(f"Subgrid x0={x0} not reachable")
        out.append(reps[x0])
    return out


# ---------------------------------------------------------------------------
# Forward M2 KRFFT (src/krfft.jl:301-621)
# ---------------------------------------------------------------------------


@dataclass
class GeneralPlan:
    spec: SpectralIndexing
    L: list
    M: tuple
    N: tuple
    rep_ops: list
    recon_idx: np.ndarray      # (d, n_spec) 0-based column-major M-grid index
    recon_w: np.ndarray        # (d, n_spec) complex weights
    phase_factors: list = field(default_factory=list)


def plan_krfft(spec, ops_shifted):
    """plan_krfft(spec, ops) auto-L variant (src/krfft.jl:301-389)."""
    N = spec.N
    D = len(N)
    L = auto_L(ops_shifted)
    M = tuple(N[d] // L[d] for d in range(D))
    if any(L[d] * M[d] != N[d] for d in range(D)):
        raise ValueError("Grid size not divisible by auto L")
    rep = select_rep_ops(ops_shifted, L, N)
    hv = k_vectors(spec).T  # (D, n_spec)
    d = len(rep)
    idx = np.zeros((d, spec.n_spec), dtype=np.int64)
    w = np.zeros((d, spec.n_spec), dtype=np.complex128)
    Mv = np.asarray(M, dtype=np.int64)[:, None]
    for g, op in enumerate(rep):
        phase = np.zeros(spec.n_spec)
        for dd in range(D):
            phase += hv[dd] * op.t[dd] / N[dd]
        w[g] = np.exp(-1j * 2 * np.pi * phase)
        idx[g] = _lin_cm(np.mod(op.Rm.T @ hv, Mv), M)
    all_diag = all(np.count_nonzero(op.Rm - np.diag(np.diag(op.Rm))) == 0 for op in rep)
    simple_t = all(all(op.t[dd] in (0, -1) or op.t[dd] % N[dd] in (0, N[dd] - 1) for dd in range(D)) for op in rep)
    pf = []
    if all_diag and simple_t:
        pf = [np.exp(2j * np.pi * np.arange(M[dd]) / N[dd]) for dd in range(D)]
    return GeneralPlan(spec, L, M, N, rep, idx, w, pf)


def fast_reconstruct(plan, Y):
    """fast_reconstruct! (src/krfft.jl:461-545): Pmmm separable or table path."""
    Yf = np.asarray(Y).ravel(order="F")
    D = len(plan.M)
    if (D == 3 and len(plan.rep_ops) == 8 and len(plan.phase_factors) == 3
            and plan.spec.n_spec == int(np.prod(plan.M))):
        return _fast_reconstruct_pmmm(plan, np.asarray(Y).reshape(plan.M, order="F"))
    return np.einsum("gs,gs->s", plan.recon_w, Yf[plan.recon_idx])


def _fast_reconstruct_pmmm(plan, Y):
    """_fast_reconstruct_pmmm! (src/krfft.jl:475-526), row-major h order."""
    M1, M2, M3 = plan.M
    p1, p2, p3 = plan.phase_factors
    i = np.arange(M1)[:, None, None]
    j = np.arange(M2)[None, :, None]
    k = np.arange(M3)[None, None, :]
    fi, fj, fk = np.mod(M1 - i, M1), np.mod(M2 - j, M2), np.mod(M3 - k, M3)
    w1, w2, w3 = p1[:, None, None], p2[None, :, None], p3[None, None, :]
    sum_p = Y[i, j, k] + w1 * Y[fi, j, k] + w2 * Y[i, fj, k] + w1 * w2 * Y[fi, fj, k]
    sum_m = Y[i, j, fk] + w1 * Y[fi, j, fk] + w2 * Y[i, fj, fk] + w1 * w2 * Y[fi, fj, fk]
    out = sum_p + w3 * sum_m
    return out.reshape(-1)  # C order == h1 outermost, h3 innermost


def pack_stride(u, L):
    """pack_stride! / pack_stride_real! / fullgrid_to_subgrid! (src/krfft.jl:571-600,
    src/centering_fold.jl:375-380, src/q_fused_krfft.jl:698-719)."""
    sl = tuple(slice(0, None, l) for l in L)
    return np.array(u[sl], dtype=np.float64)


def fft_reconstruct(plan, f0):
    """fft_reconstruct! (src/krfft.jl:554-562): FFT of the M-grid then reconstruct."""
    Y = np.fft.fftn(np.asarray(f0, dtype=np.complex128).reshape(plan.M, order="F") if np.ndim(f0) == 1 else f0)
    return fast_reconstruct(plan, Y)


def execute_krfft(plan, u):
    """execute_krfft! (src/krfft.jl:608-621)."""
    return fft_reconstruct(plan, pack_stride(u, plan.L))


# ---------------------------------------------------------------------------
# Backward M2 (src/krfft.jl:997-1311)
# ---------------------------------------------------------------------------


def build_spectral_reverse_lookup(spec, ops_shifted):
    """_build_spectral_reverse_lookup (src/krfft.jl:1183-1255).

    Returns dense arrays over the full grid (column-major linear index):
    spec index (-1 = absent), symmetry phase, conjugation flag.  First writer wins,
    in the reference's iteration order.
    """
    N = spec.N
    D = len(N)
    Nv = np.asarray(N, dtype=np.int64)
    H = spec.idx.T.astype(np.int64)  # (D, n)
    n = spec.n_spec
    keys, sidx, ph, cj = [], [], [], []
    sr = np.arange(n)
    zero = np.zeros(n)
    keys.append(_lin_cm(H, N)); sidx.append(sr); ph.append(zero); cj.append(np.zeros(n, bool))
    for op in ops_shifted:
        hr = np.mod(op.Rm.T @ H, Nv[:, None])
        phase = np.zeros(n)
        for d in range(D):
            phase += H[d] * op.t[d] / N[d]
        keys.append(_lin_cm(hr, N)); sidx.append(sr); ph.append(phase); cj.append(np.zeros(n, bool))
        keys.append(_lin_cm(np.mod(-hr, Nv[:, None]), N)); sidx.append(sr); ph.append(-phase); cj.append(np.ones(n, bool))
    keys.append(_lin_cm(np.mod(-H, Nv[:, None]), N)); sidx.append(sr); ph.append(zero); cj.append(np.ones(n, bool))
    # interleave in the reference order: for each s, [identity, (rot, neg) per op..., neg_asu]
    K = np.stack(keys, axis=1).ravel()
    S = np.stack(sidx, axis=1).ravel()
    PH = np.stack(ph, axis=1).ravel()
    CJ = np.stack(cj, axis=1).ravel()
    _, first = np.unique(K, return_index=True)
    total = int(np.prod(N))
    lut_s = np.full(total, -1, dtype=np.int64)
    lut_w = np.zeros(total, dtype=np.complex128)
    lut_c = np.zeros(total, dtype=bool)
    lut_s[K[first]] = S[first]
    lut_w[K[first]] = np.exp(2j * np.pi * PH[first])
    lut_c[K[first]] = CJ[first]
    return lut_s, lut_w, lut_c


@dataclass
class M2BackwardPlan:
    L: list
    M: tuple
    N: tuple
    d: int
    inv_spec: np.ndarray   # (d, M_vol), -1 = zero entry
    inv_w: np.ndarray      # (d, M_vol)
    inv_conj: np.ndarray   # (d, M_vol)
    n_spec: int


def plan_m2_backward(spec, ops_shifted):
    """plan_m2_backward (src/krfft.jl:1101-1170) with the per-fiber LU of
    _build_inv_recon_table! (src/krfft.jl:997-1068)."""
    N = spec.N
    D = len(N)
    L = auto_L(ops_shifted)
    M = tuple(N[d] // L[d] for d in range(D))
    rep = select_rep_ops(ops_shifted, L, N)
    d = len(rep)
    lut_s, lut_w, lut_c = build_spectral_reverse_lookup(spec, ops_shifted)
    alphas = _parity_classes(L)
    Q = _all_coords(M)  # (D, M_vol)
    Mvol = Q.shape[1]
    Nv = np.asarray(N, dtype=np.int64)[:, None]
    hs = [Q + np.asarray([M[dd] * a[dd] for dd in range(D)], dtype=np.int64)[:, None] for a in alphas]
    B = np.empty((Mvol, d, d), dtype=np.complex128)
    for a in range(d):
        for b, op in enumerate(rep):
            phase = np.zeros(Mvol)
            for dd in range(D):
                phase += hs[a][dd] * op.t[dd] / N[dd]
            B[:, a, b] = np.exp(-2j * np.pi * phase)
    e1 = np.zeros((Mvol, d), dtype=np.complex128)
    e1[:, 0] = 1.0
    x = np.linalg.solve(np.transpose(B, (0, 2, 1)), e1[..., None])[..., 0]  # B^T x = e1
    inv_spec = np.full((d, Mvol), -1, dtype=np.int64)
    inv_w = np.zeros((d, Mvol), dtype=np.complex128)
    inv_c = np.zeros((d, Mvol), dtype=bool)
    for a in range(d):
        key = _lin_cm(np.mod(hs[a], Nv), N)
        s = lut_s[key]
        found = s >= 0
        inv_spec[a] = np.where(found, s, -1)
        inv_w[a] = np.where(found, x[:, a] * lut_w[key], 0.0)
        inv_c[a] = found & lut_c[key]
    return M2BackwardPlan(L, M, N, d, inv_spec, inv_w, inv_c, spec.n_spec)


def inv_reconstruct_m2(bplan, F):
    """_inv_reconstruct_m2! (src/krfft.jl:1285-1311)."""
    F = np.asarray(F, dtype=np.complex128)
    vals = np.where(bplan.inv_spec >= 0, F[np.maximum(bplan.inv_spec, 0)], 0.0)
    vals = np.where(bplan.inv_conj, np.conj(vals), vals)
    return np.sum(bplan.inv_w * vals, axis=0)


def execute_m2_backward(bplan, F):
    """execute_m2_backward! (src/krfft.jl:1269-1277): returns the complex f0 (M-grid)."""
    Y = inv_reconstruct_m2(bplan, F).reshape(bplan.M, order="F")
    return np.fft.ifftn(Y)


# ---------------------------------------------------------------------------
# Centering fold (src/centering_fold.jl:41-580)
# ---------------------------------------------------------------------------


def alive_offsets(centering):
    """_alive_offsets (src/centering_fold.jl:111-127)."""
    return {
        CENT_I: [(0, 0, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
        CENT_F: [(0, 0, 0), (1, 1, 1)],
        CENT_C: [(0, 0, 0), (1, 1, 0), (0, 0, 1), (1, 1, 1)],
        CENT_A: [(0, 0, 0), (0, 1, 1), (1, 0, 0), (1, 1, 1)],
    }[centering]


@dataclass
class FoldPlan:
    centering: str
    M: tuple
    H: tuple
    n_channels: int
    offsets: list


def plan_centering_fold(centering, M):
    """plan_centering_fold (src/centering_fold.jl:60-104)."""
    if not all(m % 2 == 0 for m in M):
        raise ValueError("Subgrid dimensions must be even for centering fold")
    offs = alive_offsets(centering)
    return FoldPlan(centering, tuple(M), tuple(m // 2 for m in M), len(offs), offs)


def _fold_twiddle(fp, off):
    H, M = fp.H, fp.M
    t = [np.exp(-2j * np.pi * off[d] * np.arange(H[d]) / M[d]) for d in range(3)]
    return t[0][:, None, None] * t[1][None, :, None] * t[2][None, None, :]


def centering_fold(fp, f0):
    """centering_fold! (src/centering_fold.jl:140-257): returns n_ch channels (H grid)."""
    H1, H2, H3 = fp.H
    f0 = np.asarray(f0, dtype=np.float64)
    v = {}
    for ex, ey, ez in itertools.product((0, 1), repeat=3):
        v[(ex, ey, ez)] = f0[ex * H1:(ex + 1) * H1, ey * H2:(ey + 1) * H2, ez * H3:(ez + 1) * H3]
    chans = []
    for off in fp.offsets:
        g = sum(((-1) ** (off[0] * e[0] + off[1] * e[1] + off[2] * e[2])) * v[e] for e in v)
        chans.append(g * _fold_twiddle(fp, off))
    return chans


def fft_channels(chans):
    """fft_channels! (src/centering_fold.jl:264-268)."""
    return [np.fft.fftn(c) for c in chans]


def assemble_G0(fp, chan_fft):
    """assemble_G0! (src/centering_fold.jl:277-296)."""
    G0 = np.zeros(fp.M, dtype=np.complex128)
    for off, c in zip(fp.offsets, chan_fft):
        G0[off[0]::2, off[1]::2, off[2]::2] = c
    return G0


def disassemble_G0(fp, G0):
    """disassemble_G0! (src/centering_fold.jl:454-469)."""
    return [np.array(G0[off[0]::2, off[1]::2, off[2]::2]) for off in fp.offsets]


def ifft_channels(chan_fft):
    """ifft_channels! (src/centering_fold.jl:442-446)."""
    return [np.fft.ifftn(c) for c in chan_fft]


def centering_unfold(fp, chans):
    """centering_unfold! (src/centering_fold.jl:481-580): inverse WHT/8 after the
    conjugate twiddle, keeping the real part."""
    H1, H2, H3 = fp.H
    coeff = {}
    for off, c in zip(fp.offsets, chans):
        coeff[off] = np.real(c * np.conj(_fold_twiddle(fp, off)))
    f0 = np.zeros(fp.M, dtype=np.float64)
    for e in itertools.product((0, 1), repeat=3):
        acc = np.zeros(fp.H)
        for off, g in coeff.items():
            acc += ((-1) ** (off[0] * e[0] + off[1] * e[1] + off[2] * e[2])) * g
        f0[e[0] * H1:(e[0] + 1) * H1, e[1] * H2:(e[1] + 1) * H2, e[2] * H3:(e[2] + 1) * H3] = acc / 8.0
    return f0


@dataclass
class CenteredPlan:
    krfft: GeneralPlan
    fold: FoldPlan


def plan_krfft_centered(spec, ops_shifted, centering="auto"):
    """plan_krfft_centered (src/centering_fold.jl:328-367): falls back to plan_krfft."""
    N = spec.N
    cent = detect_centering_type(ops_shifted, N) if centering == "auto" else centering
    L = auto_L(ops_shifted)
    if cent == CENT_P or any(l != 2 for l in L) or len(N) != 3:
        return plan_krfft(spec, ops_shifted)
    M = tuple(n // 2 for n in N)
    if any(m % 2 for m in M):
        return plan_krfft(spec, ops_shifted)
    return CenteredPlan(plan_krfft(spec, ops_shifted), plan_centering_fold(cent, M))


def fft_reconstruct_centered(plan, f0):
    """fft_reconstruct_centered! (src/centering_fold.jl:421-431)."""
    ch = fft_channels(centering_fold(plan.fold, f0))
    return fast_reconstruct(plan.krfft, assemble_G0(plan.fold, ch))


def execute_centered_krfft(plan, u):
    """execute_centered_krfft! (src/centering_fold.jl:392-413)."""
    return fft_reconstruct_centered(plan, pack_stride(u, [2, 2, 2]))


@dataclass
class CenteredBackwardPlan:
    fold: FoldPlan
    M: tuple
    offsets: np.ndarray        # CSR row pointers (n_orbits + 1)
    spec_idx: np.ndarray       # signed 1-based (negative = conjugate)
    weight: np.ndarray
    orbit_rep: np.ndarray      # 0-based column-major positions
    member_oid: np.ndarray     # per position
    member_phase: np.ndarray   # per position
    n_spec: int


def plan_centered_ikrfft(spec, ops_shifted, fwd):
    """plan_centered_ikrfft (src/centering_fold.jl:630-731): M2 inverse table, orbit BFS
    under the even-translation operations, CSR at orbit representatives."""
    M = fwd.krfft.M
    m2 = plan_m2_backward(spec, ops_shifted)
    rem = [(op.Rm, op.tv // 2) for op in ops_shifted if np.all(op.tv % 2 == 0)]
    Mvol = int(np.prod(M))
    oid = np.zeros(Mvol, dtype=np.int64)
    oph = np.zeros(Mvol, dtype=np.complex128)
    reps = []
    Mv = np.asarray(M, dtype=np.int64)
    for m in range(Mvol):
        if oid[m]:
            continue
        reps.append(m)
        o = len(reps)
        oid[m] = o
        oph[m] = 1.0
        queue = [m]
        while queue:
            cur = queue.pop(0)
            qv = np.array([cur % M[0], (cur // M[0]) % M[1], cur // (M[0] * M[1])], dtype=np.int64)
            for R, s in rem:
                rq = np.mod(R.T @ qv, Mv)
                rl = int(rq[0] + M[0] * rq[1] + M[0] * M[1] * rq[2])
                if oid[rl] == 0:
                    oid[rl] = o
                    oph[rl] = np.exp(2j * np.pi * float(np.sum(qv * s / Mv))) * oph[cur]
                    queue.append(rl)
    reps = np.asarray(reps, dtype=np.int64)
    offs = [0]
    sidx, wts = [], []
    for q in reps:
        for a in range(m2.d):
            w = m2.inv_w[a, q]
            if abs(w) > 1e-15:
                s = m2.inv_spec[a, q] + 1
                sidx.append(-s if m2.inv_conj[a, q] else s)
                wts.append(w)
        offs.append(len(sidx))
    return CenteredBackwardPlan(fwd.fold, M, np.asarray(offs), np.asarray(sidx, dtype=np.int64),
                                np.asarray(wts, dtype=np.complex128), reps, oid - 1, oph, spec.n_spec)


def inv_recon_orbit(bplan, F):
    """_inv_recon_orbit! (src/centering_fold.jl:782-813)."""
    F = np.asarray(F, dtype=np.complex128)
    s = bplan.spec_idx
    vals = np.where(s > 0, F[np.abs(s) - 1], np.conj(F[np.abs(s) - 1])) * bplan.weight
    rows = np.repeat(np.arange(len(bplan.orbit_rep)), np.diff(bplan.offsets))
    reps_val = np.bincount(rows, weights=vals.real, minlength=len(bplan.orbit_rep)) + \
        1j * np.bincount(rows, weights=vals.imag, minlength=len(bplan.orbit_rep))
    G0 = bplan.member_phase * reps_val[bplan.member_oid]
    return G0.reshape(bplan.M, order="F")


def execute_centered_ikrfft(bplan, F):
    """execute_centered_ikrfft! (src/centering_fold.jl:745-764): returns real f0."""
    G0 = inv_recon_orbit(bplan, F)
    return centering_unfold(bplan.fold, ifft_channels(disassemble_G0(bplan.fold, G0)))


# ---------------------------------------------------------------------------
# Diffusion kernel and SCFT plans
# ---------------------------------------------------------------------------


def kernel_spec(spec, N, ds, lattice):
    """K(h) = exp(-ds |2 pi A^-T h_c|^2) (src/centering_fold.jl:881-891)."""
    recip = 2 * np.pi * np.linalg.inv(np.asarray(lattice, dtype=np.float64)).T
    Nv = np.asarray(N, dtype=np.int64)
    hc = np.where(spec.idx >= Nv // 2, spec.idx - Nv, spec.idx).astype(np.float64)
    k = hc @ recip.T
    return np.exp(-np.sum(k * k, axis=1) * ds)


@dataclass
class CenteredSCFTPlan:
    fwd: CenteredPlan
    bwd: CenteredBackwardPlan
    K: np.ndarray


def plan_centered_scft(spec, ops_shifted, N, ds, lattice):
    """plan_centered_scft (src/centering_fold.jl:868-896)."""
    fwd = plan_krfft_centered(spec, ops_shifted)
    bwd = plan_centered_ikrfft(spec, ops_shifted, fwd)
    return CenteredSCFTPlan(fwd, bwd, kernel_spec(spec, N, ds, lattice))


def execute_centered_scft(plan, f0):
    """execute_centered_scft! (src/centering_fold.jl:908-931) (returns the new f0)."""
    F = fft_reconstruct_centered(plan.fwd, f0) * plan.K
    return execute_centered_ikrfft(plan.bwd, F)


def update_kernel(plan, spec, N, ds, lattice):
    """update_kernel! (src/centering_fold.jl:939-953)."""
    plan.K = kernel_spec(spec, N, ds, lattice)


@dataclass
class M2SCFTPlan:
    fwd: GeneralPlan
    bwd: M2BackwardPlan
    K: np.ndarray
    spec: SpectralIndexing


def plan_m2_scft_ops(ops_shifted, N, ds, lattice):
    """plan_m2_scft (src/q_fused_krfft.jl:948-978) given shifted operations."""
    spec = calc_spectral_asu(ops_shifted, len(N), N)
    return M2SCFTPlan(plan_krfft(spec, ops_shifted), plan_m2_backward(spec, ops_shifted),
                      kernel_spec(spec, N, ds, lattice), spec)


def execute_m2_scft(plan, f0):
    """execute_m2_scft! (src/q_fused_krfft.jl:989-1026)."""
    F = fft_reconstruct(plan.fwd, f0) * plan.K
    return np.real(execute_m2_backward(plan.bwd, F))


# ---------------------------------------------------------------------------
# Q-fused M2 / M7 (src/q_fused_krfft.jl:83-895) and grid conversion
# ---------------------------------------------------------------------------


@dataclass
class M2QPlan:
    L: tuple
    M: tuple
    N: tuple
    rep_ops: list
    Q_first_row: np.ndarray   # (d, M_vol)
    gather_idx: np.ndarray    # (d, M_vol) 0-based
    fill_map: np.ndarray      # (N_vol,) 0-based
    ops: list


def plan_m2_q_ops(ops_shifted, N, ds, lattice):
    """plan_m2_q (src/q_fused_krfft.jl:83-169) given shifted operations:
    Q(q) = B^-1 diag(K(h_a)) B, first row (src/q_fused_krfft.jl:182-413)."""
    D = len(N)
    L = auto_L(ops_shifted)
    M = tuple(N[d] // L[d] for d in range(D))
    rep = select_rep_ops(ops_shifted, L, N)
    d = len(rep)
    recip = 2 * np.pi * np.linalg.inv(np.asarray(lattice, dtype=np.float64)).T
    alphas = _parity_classes(L)
    Q = _all_coords(M)
    Mvol = Q.shape[1]
    Mv = np.asarray(M, dtype=np.int64)[:, None]
    Nv = np.asarray(N, dtype=np.int64)[:, None]
    B = np.empty((Mvol, d, d), dtype=np.complex128)
    Kv = np.empty((Mvol, d))
    for a, al in enumerate(alphas):
        h = Q + np.asarray([M[dd] * al[dd] for dd in range(D)], dtype=np.int64)[:, None]
        hc = np.where(h >= Nv // 2, h - Nv, h).astype(np.float64)
        k = recip @ hc
        Kv[:, a] = np.exp(-np.sum(k * k, axis=0) * ds)
        for b, op in enumerate(rep):
            phase = np.zeros(Mvol)
            for dd in range(D):
                phase += h[dd] * op.t[dd] / N[dd]
            B[:, a, b] = np.exp(-1j * 2 * np.pi * phase)
    KB = Kv[:, :, None] * B
    Qf = np.linalg.solve(B, KB)
    gather = np.stack([_lin_cm(np.mod(op.Rm.T @ Q, Mv), M) for op in rep])
    return M2QPlan(tuple(L), M, tuple(N), rep, Qf[:, 0, :].T.copy(), gather,
                   build_fill_map(ops_shifted, L, M, N), list(ops_shifted))


def execute_m2_q(plan, f0):
    """execute_m2_q! (src/q_fused_krfft.jl:553-576) via the generic Q path."""
    Y = np.fft.fftn(np.asarray(f0, dtype=np.complex128)).ravel(order="F")
    Yn = np.sum(plan.Q_first_row * Y[plan.gather_idx], axis=0)
    return np.real(np.fft.ifftn(Yn.reshape(plan.M, order="F")))


def execute_m7_scft(plan, fold, f0):
    """execute_m7_scft! (src/q_fused_krfft.jl:870-895): fold + channel FFTs + Q + unfold."""
    G0 = assemble_G0(fold, fft_channels(centering_fold(fold, f0))).ravel(order="F")
    Gn = np.sum(plan.Q_first_row * G0[plan.gather_idx], axis=0).reshape(plan.M, order="F")
    return centering_unfold(fold, ifft_channels(disassemble_G0(fold, Gn)))


def build_fill_map(ops_shifted, L, M, N):
    """_build_fill_map (src/q_fused_krfft.jl:733-783): first op landing on the subgrid."""
    X = _all_coords(N)
    Nv = np.asarray(N, dtype=np.int64)[:, None]
    Lv = np.asarray(L, dtype=np.int64)[:, None]
    out = np.full(X.shape[1], -1, dtype=np.int64)
    for op in ops_shifted:
        y = np.mod(op.Rm @ X + op.tv[:, None], Nv)
        on = np.all(y % Lv == 0, axis=0) & (out < 0)
        out[on] = _lin_cm(y[:, on] // Lv, M)
    if np.any(out < 0):
        raise ValueError("No symmetry operation maps a grid point to the subgrid")
    return out


def subgrid_to_fullgrid(f0, fill_map, N):
    """subgrid_to_fullgrid! (src/q_fused_krfft.jl:681-688)."""
    return np.asarray(f0).ravel(order="F")[fill_map].reshape(N, order="F")


def step_diffusion(apply_diffusion, u, w, dt):
    """step_diffusion! (src/diffusion_solver.jl:254-267) with interaction_step!
    (src/diffusion_solver.jl:270-282)."""
    u = u * np.exp(-w * dt / 2)
    u = apply_diffusion(u)
    return u * np.exp(-w * dt / 2)


# ---------------------------------------------------------------------------
# Test helpers (test/test_helpers.jl) with a numpy generator
# ---------------------------------------------------------------------------


def make_symmetric(ops, N, seed=42, rng=None):
    """make_symmetric (test/test_helpers.jl:11-29) with numpy's seeded normal draws."""
    rng = np.random.default_rng(seed) if rng is None else rng
    u = rng.standard_normal(N)
    X = _all_coords(N)
    Nv = np.asarray(N, dtype=np.int64)[:, None]
    us = np.zeros(int(np.prod(N)))
    uf = u.ravel(order="F")
    for op in ops:
        y = _lin_cm(np.mod(op.Rm @ X + op.tv[:, None], Nv), N)
        np.add.at(us, y, uf)
    return (us / len(ops)).reshape(N, order="F")


def fullgrid_reference(u, N, ds, lattice, L):
    """fullgrid_reference (test/test_helpers.jl:56-73): IFFT(K FFT(u)) on the stride-L subgrid."""
    F = np.fft.fftn(u)
    recip = 2 * np.pi * np.linalg.inv(np.asarray(lattice, dtype=np.float64)).T
    ax = [np.arange(n) for n in N]
    hc = [np.where(a >= n // 2, a - n, a).astype(np.float64) for a, n in zip(ax, N)]
    H = np.stack(np.meshgrid(*hc, indexing="ij"))
    k = np.tensordot(recip, H, axes=(1, 0))
    Kf = np.exp(-np.sum(k * k, axis=0) * ds)
    out = np.real(np.fft.ifftn(Kf * F))
    return pack_stride(out, L)


def spectrum_on_asu(u, spec):
    """Full-grid FFT sampled at the spectral-ASU points (the tests' truth)."""
    F = np.fft.fftn(u)
    idx = spec.idx
    return F[tuple(idx[:, d] for d in range(idx.shape[1]))]


# ---------------------------------------------------------------------------
# Real-space ASU (src/asu.jl:216-324), pure Python (small grids only)
# ---------------------------------------------------------------------------


def calc_asu_points(N, ops):
    """calc_asu(N, ops) (src/asu.jl:216-324): recursive even/odd splitting of the grid;
    returns sorted [(idx tuple, depth tuple, orbit size)]."""
    D = len(N)
    out = []
    stack = [(tuple(N), [(np.array(op.Rm), np.array(op.tv)) for op in ops], (1,) * D, (0,) * D, (0,) * D,
              (False,) * D)]

    def apply(R, t, x, n):
        return tuple(int(v) for v in np.mod(R @ np.asarray(x) + t, np.asarray(n)))

    while stack:
        n, cops, scale, offset, depth, gp = stack.pop()
        if any(v == 0 for v in n):
            continue
        if all(gp) or all(v <= 1 for v in n):
            seen = set()
            for p in itertools.product(*[range(v) for v in reversed(n)]):
                p = tuple(reversed(p))  # first axis fastest
                if p in seen:
                    continue
                orbit, work = {p}, [p]
                while work:
                    c = work.pop()
                    for R, t in cops:
                        y = apply(R, t, c, n)
                        if y not in orbit:
                            orbit.add(y)
                            work.append(y)
                rep = min(orbit)
                out.append((tuple(scale[d] * rep[d] + offset[d] for d in range(D)), depth, len(orbit)))
                seen |= orbit
            continue
        egp = list(gp)
        for d in range(D):
            if gp[d]:
                continue
            e, o = [0] * D, [0] * D
            o[d] = 1
            for R, t in cops:
                if apply(R, t, e, n)[d] % 2 != 0 or apply(R, t, o, n)[d] % 2 != 1:
                    egp[d] = True
                    break
        ranges = [range(1) if (egp[d] or n[d] <= 1) else range(2) for d in range(D)]
        for par in itertools.product(*reversed(ranges)):
            par = tuple(reversed(par))
            S = np.array([1 if egp[d] else 2 for d in range(D)])
            new, ok = [], True
            for R, t in cops:
                Rv = R * S[None, :]
                tv = R @ np.asarray(par) + t - np.asarray(par)
                if np.any(Rv % S[:, None] != 0) or np.any(tv % S != 0):
                    ok = False
                    break
                new.append((Rv // S[:, None], tv // S))
            if not ok:
                continue
            stack.append((tuple(n[d] if egp[d] else n[d] // 2 for d in range(D)), new,
                          tuple(scale[d] * S[d] for d in range(D)),
                          tuple(scale[d] * par[d] + offset[d] for d in range(D)),
                          tuple(depth[d] if egp[d] else depth[d] + (par[d] == 0) for d in range(D)),
                          tuple(egp[d] or par[d] == 1 for d in range(D))))
    return sorted(out)
