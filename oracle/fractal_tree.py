"""The recursive parity tree of the fractal KRFFT, restated for the oracle.

TEST INFRASTRUCTURE ONLY.  Integer restatement of build_recursive_tree and
collect_leaves (src/fractal_krfft.jl:133-620): each node splits the dimensions whose
parity every diagonal operation preserves into even and odd sectors, merges sectors
related by an operation of the half-grid-shifted group into one representative child,
and passes the child the operations that map its sector to itself, rewritten in the
child's coordinates; a node left with only centring translations splits into its alive
(non-extinct) sectors, each a leaf.  The leaves' volumes give the tree's reduction
ratio N^3 / sum(leaf volumes), which the reference's own survey output
(test/debug_tree_output.log, extracted to tests/golden/tree_survey_64.json) pins for
200 space groups at 64^3.
"""
from __future__ import annotations

import cmath
from dataclasses import dataclass, field


@dataclass
class Node:
    """A FractalNode (src/fractal_krfft.jl:32-98): grid size, stride and offset in the
    original grid, its operations (R, t) as integer tuples, and its children."""

    subgrid_N: tuple
    scale: tuple
    offset: tuple
    ops: list
    children: list = field(default_factory=list)
    is_leaf: bool = False
    split_dims: tuple = ()
    sector_rep_idx: list = field(default_factory=list)
    is_centering_split: bool = False


def _ops_int(ops, D):
    """Operations as (R rows, t) integer tuples (R given flat or nested)."""
    import numpy as np

    out = []
    for op in ops:
        R = np.asarray(op.R, dtype=np.int64).reshape(D, D)
        out.append((tuple(tuple(int(v) for v in row) for row in R), tuple(int(v) for v in op.t)))
    return out


def _is_identity(R, D):
    return all(R[i][j] == (1 if i == j else 0) for i in range(D) for j in range(D))


def _find_split_dims(diag_ops, N, D):
    """find_split_dims (src/fractal_krfft.jl:159-186)."""
    dims = []
    for d in range(D):
        if N[d] % 2 != 0 or N[d] <= 1:
            continue
        ok = True
        for R, t in diag_ops:
            if t[d] % 2 != 0 or (R[d][d] + t[d]) % 2 != 1:
                ok = False
                break
        if ok:
            dims.append(d)
    return dims


def _round_half_even_twice(x2):
    """round(x2 / 2) with ties to even (Julia's round(Int, x)), for an integer x2."""
    q, r = divmod(x2, 2)
    if r == 0:
        return q
    return q if q % 2 == 0 else q + 1


def _shift_half(ops, N, D):
    """shift_ops_half_grid (src/fractal_krfft.jl:262-283): t' = mod(t + (I - R) b, N)
    with b = 1/2, then rounded as the reference rounds it before every use
    (round(Int, t'), ties to even).  Returns (R, t') with t' integral."""
    out = []
    for R, t in ops:
        tn = []
        for d in range(D):
            x2 = 2 * t[d] + sum((1 if d == j else 0) - R[d][j] for j in range(D))  # 2 (t + (I - R) b)
            tn.append(_round_half_even_twice(x2 % (2 * N[d])))
        out.append((R, tuple(tn)))
    return out


def _half_shift_parity(ts, R, p, D):
    """Parities of R p + t' for a shifted translation t' (integral after rounding)."""
    return [(ts[d] + sum(R[d][j] * p[j] for j in range(D))) % 2 for d in range(D)]


def build_recursive_tree(N, ops, *, child_shifted_t=False, centering_split=True):
    """build_recursive_tree (src/fractal_krfft.jl:300-520) on grid-unit operations.

    The two switches give the construction of the reference version that wrote its
    survey log (test/debug_tree_output.log): child translations from the half-grid
    shifted operations (the form src/fractal_krfft.jl:430-437 names a double-shift bug)
    and no centring split (the log's centring column is a prediction).  The defaults
    follow the current source."""
    D = len(N)
    root = Node(tuple(N), (1,) * D, (0,) * D, _ops_int(ops, D))
    queue = [root]
    while queue:
        node = queue.pop()
        cN = node.subgrid_N
        if any(x == 0 for x in cN):
            node.is_leaf = True
            continue
        diag = [(R, t) for R, t in node.ops if all(R[i][j] == 0 for i in range(D) for j in range(D) if i != j)]
        if not any(not _is_identity(R, D) for R, _ in node.ops):
            cent = []
            for R, t in node.ops:
                if not _is_identity(R, D):
                    continue
                tm = tuple(t[d] % cN[d] for d in range(D))
                if any(tm):
                    cent.append(tm)
            if centering_split and cent and all(x >= 2 for x in cN):
                _centering_split(node, cent, cN, D)
                continue
            node.is_leaf = True
            continue
        split = _find_split_dims(diag, cN, D)
        if not split or all(x <= 1 for x in cN):
            node.is_leaf = True
            continue
        node.split_dims = tuple(split)
        nsec = 1 << len(split)
        parities = []
        for bits in range(nsec):
            p = [0] * D
            for k, d in enumerate(split):
                p[d] = (bits >> k) & 1
            parities.append(p)
        shifted = _shift_half(node.ops, cN, D)
        # find_sector_orbits (src/fractal_krfft.jl:203-250)
        index = {tuple(p): i for i, p in enumerate(parities)}
        orbit_rep = list(range(nsec))
        visited = [False] * nsec
        for i in range(nsec):
            if visited[i]:
                continue
            visited[i] = True
            for R, ts in shifted:
                img = _half_shift_parity(ts, R, parities[i], D)
                for d in range(D):
                    if d not in split:
                        img[d] = 0
                j = index.get(tuple(img))
                if j is not None and not visited[j]:
                    visited[j] = True
                    orbit_rep[j] = i
        S = [2 if d in split else 1 for d in range(D)]
        child_N = tuple(cN[d] // 2 if d in split else cN[d] for d in range(D))
        reps = sorted(set(orbit_rep))
        child_of = {r: c for c, r in enumerate(reps)}
        node.sector_rep_idx = [child_of[orbit_rep[s]] for s in range(nsec)]
        for ri in reps:
            p = parities[ri]
            new_ops, seen = [], set()
            for (R, t), (_, ts) in zip(node.ops, shifted):
                img = _half_shift_parity(ts, R, p, D)
                if any(img[d] != p[d] for d in split):
                    continue
                Rn, tn, valid = [[0] * D for _ in range(D)], [0] * D, True
                for i in range(D):
                    for j in range(D):
                        rv = R[i][j] * S[j]
                        if rv % S[i] != 0:
                            valid = False
                            break
                        Rn[i][j] = rv // S[i]
                    if not valid:
                        break
                    ti = ts[i] if child_shifted_t else t[i]
                    tv = ti - p[i] + sum(R[i][j] * p[j] for j in range(D))
                    if tv % S[i] != 0:
                        valid = False
                        break
                    tn[i] = tv // S[i]
                if valid:
                    key = (tuple(tuple(r) for r in Rn), tuple(tn))
                    if key not in seen:
                        seen.add(key)
                        new_ops.append(key)
            child = Node(child_N, tuple(node.scale[d] * S[d] for d in range(D)),
                         tuple(node.scale[d] * p[d] + node.offset[d] for d in range(D)), new_ops)
            node.children.append(child)
            queue.append(child)
    return root


def _centering_split(node, cent, cN, D):
    """_setup_centering_split! (src/fractal_krfft.jl:535-604): every even dimension
    splits, and each sector whose centring phase sum does not vanish is a leaf."""
    node.is_centering_split = True
    split = [d for d in range(D) if cN[d] >= 2 and cN[d] % 2 == 0]
    node.split_dims = tuple(split)
    nsec = 1 << len(split)
    parities = []
    for bits in range(nsec):
        p = [0] * D
        for k, d in enumerate(split):
            p[d] = (bits >> k) & 1
        parities.append(p)
    group = {(0,) * D}
    q = [(0,) * D]
    for t in cent:
        if t not in group:
            group.add(t)
            q.append(t)
    while q:
        g = q.pop()
        for t in cent:
            h = tuple((g[d] + t[d]) % cN[d] for d in range(D))
            if h not in group:
                group.add(h)
                q.append(h)
    S = [2 if d in split else 1 for d in range(D)]
    child_N = tuple(cN[d] // 2 if d in split else cN[d] for d in range(D))
    node.sector_rep_idx = [0] * nsec
    c = 0
    for s, p in enumerate(parities):
        z = sum(cmath.exp(-2j * cmath.pi * sum(p[d] * tau[d] / cN[d] for d in range(D))) for tau in group)
        if abs(z) < 0.5:
            continue
        c += 1
        node.sector_rep_idx[s] = c
        node.children.append(Node(child_N, tuple(node.scale[d] * S[d] for d in range(D)),
                                  tuple(node.scale[d] * p[d] + node.offset[d] for d in range(D)), [],
                                  is_leaf=True))


def collect_leaves(node):
    """collect_leaves (src/fractal_krfft.jl:622-636): depth first, children in order."""
    if node.is_leaf:
        return [node]
    out = []
    for ch in node.children:
        out += collect_leaves(ch)
    return out


def centering_index(ops, N):
    """The centring sublattice index of the survey (test/debug_tree.jl:13-31): the size of
    the group generated by the pure translations (R = I, t != 0) mod N."""
    D = len(N)
    cents = [t for R, t in _ops_int(ops, D) if _is_identity(R, D) and any(t)]
    group = {(0,) * D}
    q = [(0,) * D]
    while q:
        g = q.pop()
        for t in cents:
            h = tuple((g[d] + t[d]) % N[d] for d in range(D))
            if h not in group:
                group.add(h)
                q.append(h)
    return len(group)


def reduction_ratio(N, ops, **kw):
    """N^3 over the leaves' total volume (test/debug_tree.jl:42-54)."""
    leaves = collect_leaves(build_recursive_tree(N, ops, **kw))
    total = 0
    for leaf in leaves:
        v = 1
        for n in leaf.subgrid_N:
            v *= n
        total += v
    vol = 1
    for n in N:
        vol *= n
    return vol / total, len(leaves)
