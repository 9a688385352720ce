"""Real-space asymmetric unit, block packing and interleaved subgrid orbits
(module ASU, src/asu.jl:1-46,216-436 and src/pack_asu.jl).

calc_asu runs in the library's C++ plan layer (cfft_calc_asu); the packing and orbit
analysis are host bookkeeping over its output.  Block data are numpy arrays
(column-major index order, as Julia arrays) or, for pack_asu_interleaved of a CUDA
tensor, CUDA tensors.
"""
from __future__ import annotations

import ctypes
import itertools
from dataclasses import dataclass, field

import numpy as np

from . import symmetry as sym
from ._lib import LIB, check


@dataclass
class ASUPoint:
    """ASUPoint (src/asu.jl:24-28)."""

    idx: list
    depth: list
    multiplicity: int


@dataclass
class InterleavedOrbit:
    """InterleavedOrbit (src/asu.jl:16-22): an orbit of stride-L subgrids (coset shifts)."""

    representative: list
    members: list
    ops: list
    multiplicity: int


@dataclass
class ASUBlock:
    """ASUBlock (src/asu.jl:30-38): dense block of the ASU with its global 0-based ranges."""

    data: object
    range: list           # one python range (start, stop, step) per dimension, 0-based
    depth: list
    orbit: InterleavedOrbit | None = None


@dataclass
class CrystallographicASU:
    """CrystallographicASU (src/asu.jl:40-44): blocks grouped by effective dimension."""

    dim_blocks: dict = field(default_factory=dict)
    shift: tuple = ()


def calc_asu(*args):
    """calc_asu(sg_num, dim, N) -> (points, shift) with the magic shift (src/asu.jl:51-55),
    or calc_asu(N, ops) -> points for already shifted operations (src/asu.jl:216-324)."""
    if len(args) == 3:
        sg_num, dim, N = args
        ops = sym.get_ops(sg_num, dim, N)
        shift, ops_s = sym.find_optimal_shift(ops, N)
        return _calc_asu(tuple(N), ops_s), tuple(float(v) for v in shift)
    N, ops = args
    return _calc_asu(tuple(N), ops)


def _calc_asu(N, ops):
    dim = len(N)
    R, t = sym._pack(ops)
    Nc = (ctypes.c_int * 3)(*(list(N) + [1] * (3 - dim)))
    n = ctypes.c_int(0)
    check(LIB.cfft_calc_asu(dim, Nc, len(ops), sym._ptr(R), sym._ptr(t), 0, ctypes.byref(n), None, None, None))
    idx = np.zeros((n.value, 3), dtype=np.int32)
    depth = np.zeros((n.value, 3), dtype=np.int32)
    mult = np.zeros(n.value, dtype=np.int32)
    check(LIB.cfft_calc_asu(dim, Nc, len(ops), sym._ptr(R), sym._ptr(t), n.value, ctypes.byref(n), sym._ptr(idx),
                            sym._ptr(depth), sym._ptr(mult)))
    return [ASUPoint([int(v) for v in idx[k, :dim]], [int(v) for v in depth[k, :dim]], int(mult[k]))
            for k in range(n.value)]


def compute_full_orbit(idx, ops, N):
    """Full orbit of a grid point under the operations (test/test_helpers.jl)."""
    seen = {tuple(idx)}
    stack = [tuple(idx)]
    while stack:
        x = np.array(stack.pop())
        for op in ops:
            y = tuple(int(v) for v in sym.apply_op(op, x, N))
            if y not in seen:
                seen.add(y)
                stack.append(y)
    return seen


def pack_asu(points, N, dtype=np.float64, *, shift=None):
    """pack_asu (src/pack_asu.jl:6-94): points of equal depth are packed greedily into
    rectangular unit-stride blocks grown from the smallest remaining point, one
    dimension after the other; blocks are grouped by their effective dimension."""
    D = len(N)
    groups = {}
    for p in points:
        groups.setdefault(tuple(p.depth), []).append(p)
    blocks = []
    for depth in sorted(groups):
        pool = sorted(tuple(p.idx) for p in groups[depth])
        left = set(pool)
        for start in pool:
            if start not in left:
                continue
            lo, hi = list(start), list(start)
            for d in range(D):
                while True:
                    nxt = hi[d] + 1
                    face = [range(lo[k], hi[k] + 1) if k != d else range(nxt, nxt + 1) for k in range(D)]
                    if any(pt not in left for pt in itertools.product(*face)):
                        break
                    hi[d] = nxt
            rng = [range(lo[d], hi[d] + 1) for d in range(D)]
            for pt in itertools.product(*rng):
                left.discard(pt)
            blocks.append(ASUBlock(np.zeros(tuple(len(r) for r in rng), dtype=dtype), rng, list(depth)))
    out = CrystallographicASU({}, tuple(shift) if shift is not None else tuple(0.0 for _ in range(D)))
    for b in blocks:
        out.dim_blocks.setdefault(sum(len(r) > 1 for r in b.range), []).append(b)
    return out


def analyze_interleaved_orbits(N, ops, L=None):
    """analyze_interleaved_orbits (src/asu.jl:337-436): orbits of the coset shifts
    x in [0, L) under x -> (R x + t) mod L, with every operation mapping the
    representative onto each member."""
    D = len(N)
    L = tuple(L) if L is not None else (2,) * D
    Lv = np.asarray(L, dtype=np.int64)
    visited, orbits = set(), []
    coarse = [tuple(reversed(c)) for c in itertools.product(*[range(l) for l in reversed(L)])]  # first axis fastest
    for p in coarse:
        if p in visited:
            continue
        members, queue = {p}, [p]
        while queue:
            cur = np.array(queue.pop(0), dtype=np.int64)
            for op in ops:
                x = tuple(int(v) for v in np.mod(op.Rm @ cur + np.asarray(op.t), Lv))
                if x not in members:
                    members.add(x)
                    queue.append(x)
        final = sorted(members)
        pv = np.array(p, dtype=np.int64)
        op_lists = [[op for op in ops if tuple(int(v) for v in np.mod(op.Rm @ pv + np.asarray(op.t), Lv)) == m]
                    for m in final]
        orbits.append(InterleavedOrbit(list(p), [list(m) for m in final], op_lists, len(final)))
        visited |= members
    return orbits


def pack_asu_interleaved(u, N, ops, *, L=None, asu_only=True):
    """pack_asu_interleaved (src/pack_asu.jl:108-202): the stride-L subgrid of each orbit
    representative (only the Gamma_0 = (0, ..., 0) orbit with asu_only), as full-dimension
    blocks; CUDA tensors ((N3, N2, N1), x fastest) are sliced on the device."""
    D = len(N)
    orbits = analyze_interleaved_orbits(N, ops, L=L)
    L = tuple(L) if L is not None else (2,) * D
    if asu_only:
        orbits = [next((o for o in orbits if not any(o.representative)), orbits[0])]
    blocks = []
    for o in orbits:
        rng = [range(o.representative[d], N[d], L[d]) for d in range(D)]
        if hasattr(u, "is_cuda"):
            sl = tuple(slice(r.start, None, r.step) for r in reversed(rng))
            data = u[sl].contiguous()
        else:
            data = np.array(np.asarray(u)[tuple(slice(r.start, None, r.step) for r in rng)])
        blocks.append(ASUBlock(data, rng, [0] * D, None if asu_only else o))
    return CrystallographicASU({D: blocks}, tuple(0.0 for _ in range(D)))


class CFFTPlan:
    """CFFTPlan / plan_cfft (src/cfft_plan.jl:4-41): the real-space ASU packed into
    blocks, with one device block plan (cfft_block_plan) transforming all of them."""

    def __init__(self, N, sg_num, T=np.float64, *, dim=None):
        dim = len(N) if dim is None else dim
        points, shift = calc_asu(sg_num, dim, tuple(N))
        self.asu = pack_asu(points, tuple(N), T, shift=shift)
        self.N = tuple(N)
        self.precision = 4 if np.dtype(T) in (np.dtype(np.float32), np.dtype(np.complex64)) else 8
        self.order = [(d, i) for d in sorted(self.asu.dim_blocks) for i in range(len(self.asu.dim_blocks[d]))]
        shapes = [self.asu.dim_blocks[d][i].data.shape for d, i in self.order]
        dims = np.ones((len(shapes), 3), dtype=np.int32)
        for k, sh in enumerate(shapes):
            dims[k, :len(sh)] = sh
        self.shapes = shapes
        h = ctypes.c_void_p()
        check(LIB.cfft_block_plan_create(len(shapes), sym._ptr(dims), self.precision, ctypes.byref(h)))
        self._h = h

    def _run(self, y, x, inverse):
        import torch

        cdt = torch.complex64 if self.precision == 4 else torch.complex128
        blocks = [x.dim_blocks[d][i].data for d, i in self.order]
        on_dev = hasattr(blocks[0], "is_cuda")
        if on_dev:  # (n3, n2, n1) tensors: C order is the blocks' column-major order
            flat = torch.cat([b.reshape(-1).to(cdt) for b in blocks])
        else:
            flat = torch.as_tensor(np.concatenate([np.asarray(b).ravel(order="F") for b in blocks])).to(cdt).to("cuda")
        out = torch.empty_like(flat)
        fn = LIB.cfft_block_backward if inverse else LIB.cfft_block_forward
        check(fn(self._h, ctypes.c_void_p(flat.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        pos = 0
        host = None if on_dev else out.cpu().numpy()
        for (d, i), sh in zip(self.order, self.shapes):
            n = int(np.prod(sh))
            yb = y.dim_blocks[d][i]
            if on_dev:
                yb.data = out[pos:pos + n].view(tuple(reversed(sh)))
            else:
                yb.data = host[pos:pos + n].reshape(sh, order="F").copy()
            pos += n
        return y

    def close(self):
        if self._h:
            LIB.cfft_block_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan_cfft(N, sg_num, T=np.float64, ArrayType=None, *, dim=None):
    """plan_cfft (src/cfft_plan.jl:15-41)."""
    return CFFTPlan(N, sg_num, T, dim=dim)


def mul(y, plan, x):
    """mul!(y, ::CFFTPlan, x) (src/execution.jl:16-35): forward FFT of every block."""
    return plan._run(y, x, False)


def ldiv(y, plan, x):
    """ldiv!(y, ::CFFTPlan, x) (src/execution.jl:42-60): inverse FFT (1/n) of every block."""
    return plan._run(y, x, True)
