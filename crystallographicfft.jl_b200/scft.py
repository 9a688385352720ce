"""SCFT driver for an AB diblock melt on a KRFFT plan (cfft_scft_*, include/cfft_b200.h).

The reference provides the contour step this runs on (step_diffusion!,
src/diffusion_solver.jl:254-282; execute_m2_scft!, src/q_fused_krfft.jl:989-1026) but no
SCFT driver; the iteration here is the textbook one, documented in csrc/scft.cu.  Fields
are [w_A | w_B] on the plan's stride-L subgrid, a contiguous (2, M3, M2, M1) CUDA tensor
in the plan's precision.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import symmetry as sym
from ._lib import LIB, CFFTError, check
from .plans import KRFFTPlan, _torch


class _Params(ctypes.Structure):
    _fields_ = [("f", ctypes.c_double), ("chiN", ctypes.c_double), ("Ns", ctypes.c_int), ("history", ctypes.c_int),
                ("tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("lam_simple", ctypes.c_double),
                ("lam_anderson", ctypes.c_double), ("anderson_start", ctypes.c_double), ("min_simple", ctypes.c_int)]


class _State(ctypes.Structure):
    _fields_ = [("Q", ctypes.c_double), ("F", ctypes.c_double), ("err", ctypes.c_double),
                ("iterations", ctypes.c_int), ("converged", ctypes.c_int)]


_SIGS = {
    "cfft_scft_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_Params), ctypes.POINTER(ctypes.c_void_p)]),
    "cfft_scft_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cfft_scft_evaluate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.POINTER(_State), ctypes.c_void_p]),
    "cfft_scft_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_State), ctypes.c_void_p]),
    "cfft_scft_densities": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
}
for _n, (_r, _a) in _SIGS.items():
    getattr(LIB, _n).restype = _r
    getattr(LIB, _n).argtypes = _a


def _state(s):
    return {"Q": s.Q, "F": s.F, "err": s.err, "iterations": s.iterations, "converged": bool(s.converged)}


class SCFTSolver:
    """Self-consistent field iteration of an incompressible AB diblock melt on `plan`
    (whose ds must be 1/Ns and max_batch at least 2): A-block fraction f, chiN, Ns
    contour steps, Anderson mixing over `history` iterates below `anderson_start` once
    `min_simple` simple-mixing iterations have run."""

    def __init__(self, plan, f, chiN, Ns, *, history=20, tol=1e-6, max_iter=1000, lam_simple=0.1,
                 lam_anderson=1.0, anderson_start=0.2, min_simple=0):
        self.plan = plan
        self.params = dict(f=f, chiN=chiN, Ns=Ns, history=history, tol=tol, max_iter=max_iter,
                           lam_simple=lam_simple, lam_anderson=lam_anderson, anderson_start=anderson_start,
                           min_simple=min_simple)
        p = _Params(**self.params)
        h = ctypes.c_void_p()
        check(LIB.cfft_scft_create(plan.handle, ctypes.byref(p), ctypes.byref(h)))
        self._h = h

    def _stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)

    def _check_field(self, w):
        torch = _torch()
        dt = torch.float64 if self.plan.precision == 8 else torch.float32
        M = self.plan.M
        if not (w.is_cuda and w.is_contiguous() and w.dtype == dt and w.numel() == 2 * int(np.prod(M))):
            raise CFFTError(1, f"w must be a contiguous CUDA {dt} tensor of 2 x {tuple(reversed(M))}")

    def evaluate(self, w):
        """Q, F, err, densities phi = [phi_A | phi_B] and residuals d of the fields w."""
        torch = _torch()
        self._check_field(w)
        phi, d = torch.empty_like(w), torch.empty_like(w)
        s = _State()
        check(LIB.cfft_scft_evaluate(self._h, ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(phi.data_ptr()),
                                     ctypes.c_void_p(d.data_ptr()), ctypes.byref(s), self._stream()))
        out = _state(s)
        out.update(phi=phi, d=d)
        return out

    def solve(self, w):
        """Iterates w (in place) to err < tol; returns the final state."""
        self._check_field(w)
        s = _State()
        check(LIB.cfft_scft_solve(self._h, ctypes.c_void_p(w.data_ptr()), ctypes.byref(s), self._stream()))
        return _state(s)

    def densities(self):
        torch = _torch()
        dt = torch.float64 if self.plan.precision == 8 else torch.float32
        phi = torch.empty((2,) + tuple(reversed(self.plan.M)), dtype=dt, device="cuda")
        check(LIB.cfft_scft_densities(self._h, ctypes.c_void_p(phi.data_ptr()), self._stream()))
        return phi

    def close(self):
        if getattr(self, "_h", None):
            LIB.cfft_scft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan_scft(sg, N, cell, *, f=0.4, chiN=20.0, Ns=100, precision=4, ops=None, path=0, tuning=None, **kw):
    """A plan for group `sg` on grid N with cubic cell edge `cell` (lattice = cell * I)
    and ds = 1/Ns, and its SCFTSolver.  `ops` (shifted operations) defaults to the
    library's table shifted by find_optimal_shift; `path` selects the plan's contour
    step (cfft_path: the spectral-ASU step by default, or the Q-matrix steps) and `tuning`
    its execution choices (cfft_tuning fields as a dict)."""
    N = tuple(N)
    if ops is None:
        _, ops = sym.find_optimal_shift(sym.get_ops(sg, len(N), N), N)
    spec = sym.calc_spectral_asu(ops, len(N), N)
    plan = KRFFTPlan(spec, ops, N=N, ds=1.0 / Ns, lattice=np.eye(3) * cell, precision=precision, max_batch=2,
                     path=path, tuning=tuning)
    return plan, SCFTSolver(plan, f, chiN, Ns, **kw)


def initial_fields(ops_shifted, N, L, f, chiN, *, seed=0, sigma=2.0, amplitude=1.0):
    """Seeded start (numpy, host): N(0, 1) noise on the full grid, Gaussian filter of
    width sigma grid points, averaged over the operations, standard deviation
    `amplitude`: w_A = chiN (1 - f) + eta, w_B = chiN f - eta on the stride-L subgrid.
    Returned as a (2, M3, M2, M1) float64 array in memory order."""
    N = tuple(N)
    rng = np.random.default_rng(seed)
    u = rng.standard_normal(N)  # indexed [x, y, z]
    K2 = sum(np.meshgrid(*[(2 * np.pi * np.fft.fftfreq(n)) ** 2 for n in N], indexing="ij"))
    u = np.real(np.fft.ifftn(np.fft.fftn(u) * np.exp(-0.5 * sigma ** 2 * K2)))
    idx = np.stack(np.meshgrid(*[np.arange(n) for n in N], indexing="ij")).reshape(3, -1)
    Nv = np.asarray(N)[:, None]
    acc = np.zeros(idx.shape[1])
    for op in ops_shifted:
        y = np.mod(op.Rm @ idx + op.tv[:, None], Nv)
        acc += u[y[0], y[1], y[2]]
    eta = (acc / len(ops_shifted)).reshape(N)
    eta -= eta.mean()
    eta *= amplitude / max(eta.std(), 1e-300)
    sub = eta[::L[0], ::L[1], ::L[2]].transpose(2, 1, 0)  # (M3, M2, M1) memory order
    return np.stack([chiN * (1.0 - f) + sub, chiN * f - sub])
