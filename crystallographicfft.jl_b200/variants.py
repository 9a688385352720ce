"""The reference's variant KRFFT plans, by their reference names, on the device path.

CrystallographicFFT.jl keeps several alternative CPU decompositions of the same
transform:

- recursive / sparse / selective / G0-ASU forwards (stride-4 P3c sub-grids with
  butterfly or orbit-reduced G0 fills, src/recursive_blocks.jl:35-1312);
- the general G0-ASU forward (src/recursive_blocks.jl:1343-1588);
- the G0-ASU backward to the full grid with symmetry fill (src/recursive_blocks_backward.jl);
- the fractal parity-tree forwards v1-v3 (src/fractal_krfft.jl, src/fractal_krfft_v3.jl);
- the staged Pm-3m forward (src/staged_krfft.jl).

They differ in how they schedule FFT and gather work on a CPU.  Their results are the
spectrum on the spectral ASU of a full-grid field, the full grid from that spectrum, and
(staged) F000 = FFT of the stride-2 subgrid.  On B200 every one of them runs on the
batched subgrid pipeline of libcfft_b200: full grid -> stride-L subgrid on the device,
fold + channel FFTs + reconstruct onto the ASU (forward); inverse gather + orbit
expansion + inverse FFTs + unfold, then the symmetry fill of the full grid (backward);
cfft_subgrid_spectrum for F000.  Inputs may be numpy arrays (column-major (N1, N2, N3),
as Julia arrays) or CUDA tensors ((N3, N2, N1) contiguous, x fastest).
"""
from __future__ import annotations

import numpy as np

from . import symmetry as sym
from ._lib import CFFTError
from .plans import PATH_AUTO, PATH_M2, KRFFTPlan, _is_tensor, _torch, fullgrid_to_subgrid


class FractalLeaf:
    """A leaf of the recursive parity tree: its grid, and the stride and offset at which
    it samples the full grid (FractalNode, src/fractal_krfft.jl:32-98)."""

    def __init__(self, subgrid_N, scale, offset):
        self.subgrid_N, self.scale, self.offset = tuple(subgrid_N), tuple(scale), tuple(offset)
        self.is_leaf = True


class FractalTree:
    """build_recursive_tree (src/fractal_krfft.jl:300-520), built by the library's plan
    layer: its leaves in collect_leaves order and the number of inner nodes."""

    def __init__(self, N, ops, flags=0):
        arr, depths, self.n_inner = sym.fractal_tree(ops, N, flags=flags)
        self.N = tuple(N)
        self.leaves = [FractalLeaf(a[0], a[1], a[2]) for a in arr]
        self.depths = [int(d) for d in depths]
        self.n_leaves = len(self.leaves)

    def fft_points(self):
        """Total FFT points of the leaves (the volume the tree transforms)."""
        return int(sum(np.prod(l.subgrid_N) for l in self.leaves))


def build_recursive_tree(N, ops):
    """build_recursive_tree(N, ops) (src/fractal_krfft.jl:300-520)."""
    return FractalTree(tuple(N), ops)


calc_asu_tree = build_recursive_tree  # src/fractal_krfft.jl:946


def collect_leaves(tree):
    """collect_leaves (src/fractal_krfft.jl:622-636)."""
    return list(tree.leaves)


def tree_summary(tree):
    """tree_summary (src/fractal_krfft.jl:653-667): leaves, inner nodes, deepest leaf."""
    return dict(n_gp_leaves=tree.n_leaves, n_sp_nodes=tree.n_inner,
                max_depth=max(tree.depths) if tree.depths else 0)


class VariantKRFFTPlan:
    """A variant forward plan (spectral ASU from the full grid) on the device path.  The
    fractal kinds also hold the reference's plan-time tree (tree, n_leaves, n_inner,
    like FractalCFFTPlan, src/fractal_krfft.jl:104-114); the transform itself runs on the
    batched subgrid pipeline."""

    def __init__(self, kind, spec, ops_shifted, *, precision=8, max_batch=1, path=PATH_AUTO, device=True):
        self.kind = kind
        self.spec = spec
        self.plan = KRFFTPlan(spec, ops_shifted, precision=precision, max_batch=max_batch, path=path, device=device)
        self.n_spec = self.plan.n_spec
        self.N = tuple(spec.N)
        if kind.startswith("fractal"):
            self.tree = FractalTree(self.N, ops_shifted)
            self.n_leaves, self.n_inner = self.tree.n_leaves, self.tree.n_inner

    def execute(self, u):
        return self.plan.forward(fullgrid_to_subgrid(self.plan, u))

    def close(self):
        self.plan.close()


def _check_spec(plan, spec):
    if tuple(spec.N) != plan.N or len(spec.idx) != plan.n_spec:
        raise CFFTError(1, "spectral ASU does not belong to this plan")


# The forward variants by their reference names.  Each row: plan constructor (with its
# reference lines), execute function (with its reference lines), and whether the execute
# function takes the spectral indexing as the reference's does.  Every one computes the
# spectral-ASU spectrum of a full-grid field on the batched subgrid pipeline; the names
# exist so that a caller of the reference finds them.
_FORWARD = [
    ("recursive", "plan_krfft_recursive", "src/recursive_blocks.jl:64-145",
     "execute_recursive_krfft", "src/recursive_blocks.jl:323-331", True),
    ("sparse", "plan_krfft_sparse", "src/recursive_blocks.jl:514-630",
     "execute_sparse_krfft", "src/recursive_blocks.jl:631-670", True),
    ("selective", "plan_krfft_selective", "src/recursive_blocks.jl:756-889",
     "execute_selective_krfft", "src/recursive_blocks.jl:890-957", True),
    ("g0asu", "plan_krfft_g0asu", "src/recursive_blocks.jl:1034-1245",
     "execute_g0asu_krfft", "src/recursive_blocks.jl:1246-1312", True),
    ("g0asu_general", "plan_krfft_g0asu_general", "src/recursive_blocks.jl:1378-1553",
     "execute_general_g0asu_krfft", "src/recursive_blocks.jl:1554-1588", True),
    ("fractal", "plan_fractal_krfft", "src/fractal_krfft.jl:678-723",
     "execute_fractal_krfft", "src/fractal_krfft.jl:869-901", False),
    ("fractal_v2", "plan_fractal_krfft_v2", "src/fractal_krfft.jl:1021-1171",
     "execute_fractal_krfft_v2", "src/fractal_krfft.jl:1228-1279", False),
    ("fractal_v3", "plan_fractal_krfft_v3", "src/fractal_krfft_v3.jl:205-380",
     "execute_fractal_krfft_v3", "src/fractal_krfft_v3.jl:381-452", False),
]


def _forward_pair(kind, plan_name, plan_cite, exec_name, exec_cite, takes_spec):
    def make(spec, ops_shifted, **kw):
        return VariantKRFFTPlan(kind, spec, ops_shifted, **kw)

    if takes_spec:
        def run(plan, spec, u):
            _check_spec(plan, spec)
            return plan.execute(u)
    else:
        def run(plan, u):
            return plan.execute(u)

    make.__name__, run.__name__ = plan_name, exec_name
    make.__doc__ = f"{plan_name} ({plan_cite}): a VariantKRFFTPlan on the device path."
    run.__doc__ = f"{exec_name}! ({exec_cite}): the spectrum on the spectral ASU of the full-grid field u."
    return make, run


for _row in _FORWARD:
    _make, _run = _forward_pair(*_row)
    globals()[_make.__name__] = _make
    globals()[_run.__name__] = _run
del _row, _make, _run


class G0ASUBackwardPlan:
    """plan_krfft_g0asu_backward (src/recursive_blocks_backward.jl:95-459): spectral ASU ->
    full grid with the symmetry fill, on the device path."""

    def __init__(self, spec, ops_shifted, *, precision=8, max_batch=1):
        self.spec = spec
        self.plan = KRFFTPlan(spec, ops_shifted, precision=precision, max_batch=max_batch, path=PATH_AUTO)

    def execute(self, F, u_out=None):
        torch = _torch()
        p = self.plan
        host = not _is_tensor(F)
        if host:
            cdt = torch.complex64 if p.precision == 4 else torch.complex128
            F = torch.as_tensor(np.ascontiguousarray(F), dtype=cdt).to("cuda")
        u = p.subgrid_to_fullgrid(p.backward(F))
        if not host:
            if u_out is not None:
                u_out.copy_(u)
                return u_out
            return u
        a = u.cpu().numpy()
        full = np.stack([x.transpose(2, 1, 0) for x in a]) if a.ndim == 4 else a.transpose(2, 1, 0)
        if u_out is not None:
            np.copyto(u_out, full)
            return u_out
        return full

    def close(self):
        self.plan.close()


def plan_krfft_g0asu_backward(spec, ops_shifted, **kw):
    """plan_krfft_g0asu_backward (src/recursive_blocks_backward.jl:135-459)."""
    return G0ASUBackwardPlan(spec, ops_shifted, **kw)


def execute_g0asu_ikrfft(plan, spec, F, u_out=None):
    """execute_g0asu_ikrfft! (src/recursive_blocks_backward.jl:460-548): writes the full
    grid into u_out (and returns it)."""
    _check_spec(plan.plan, spec)
    return plan.execute(F, u_out)


class StagedPm3mPlan:
    """plan_staged_pm3m / plan_staged_pm3m_full (src/staged_krfft.jl:115-129,863-881):
    Pm-3m with the half-grid shift; the forward returns F000 = FFT of the stride-2
    subgrid f000(n) = u(2n), (N/2)^3 complex."""

    def __init__(self, N, *, precision=8, max_batch=1):
        N = tuple(int(n) for n in N)
        _, ops_s = sym.find_optimal_shift(sym.get_ops(221, 3, N), N)
        self.ops_shifted = ops_s
        self.spec = sym.calc_spectral_asu(ops_s, 3, N)
        self.plan = KRFFTPlan(self.spec, ops_s, precision=precision, max_batch=max_batch, path=PATH_M2)
        if tuple(self.plan.L) != (2, 2, 2):
            raise CFFTError(4, "staged Pm-3m needs L = (2, 2, 2)")
        self.N = N
        self._rep = self.plan.rep_ops()

    def execute(self, u):
        torch = _torch()
        p = self.plan
        if _is_tensor(u):
            return p.subgrid_spectrum(p.fullgrid_to_subgrid(u))
        rdt = torch.float32 if p.precision == 4 else torch.float64
        f0 = np.asarray(u)[::2, ::2, ::2]
        t = torch.as_tensor(np.ascontiguousarray(f0.transpose(2, 1, 0)), dtype=rdt).to("cuda")
        return p.subgrid_spectrum(t).cpu().numpy().transpose(2, 1, 0)

    def close(self):
        self.plan.close()


def plan_staged_pm3m(N, **kw):
    """plan_staged_pm3m (src/staged_krfft.jl:115-129)."""
    return StagedPm3mPlan(N, **kw)


def plan_staged_pm3m_full(N, **kw):
    """plan_staged_pm3m_full (src/staged_krfft.jl:863-881)."""
    return StagedPm3mPlan(N, **kw)


def execute_staged(plan, u):
    """execute_staged! (src/staged_krfft.jl:562-567): F000 (numpy (M1, M2, M3) for numpy u)."""
    return plan.execute(u)


def execute_staged_full(plan, u):
    """execute_staged_full! (src/staged_krfft.jl:883-889)."""
    return plan.execute(u)


def lookup_full_spectrum(plan, F000, hx, hy, hz):
    """lookup_full_spectrum (src/staged_krfft.jl:585-617): F(h) for any h of the full grid
    from F000, F(h) = sum_b e^{-2 pi i h.t_b / N} F000(R_b^T h mod M) over the plan's
    representative operations (numpy F000 indexed (M1, M2, M3))."""
    h = np.array([hx, hy, hz], dtype=np.int64)
    N = np.asarray(plan.N, dtype=np.int64)
    M = N // 2
    F = np.asarray(F000)
    val = 0j
    for op in plan._rep:
        R = np.asarray(op.R, dtype=np.int64).reshape(3, 3)
        t = np.asarray(op.t, dtype=np.int64)
        q = np.mod(R.T @ h, M)
        val += np.exp(-2j * np.pi * float(np.sum(h * t / N))) * F[q[0], q[1], q[2]]
    return val
