"""Plan objects and execute functions: the host-side mirror of the reference's
KRFFT / centred / M2 / SCFT / diffusion plan API (src/krfft.jl, src/centering_fold.jl,
src/q_fused_krfft.jl, src/diffusion_solver.jl), running on libcfft_b200.

Names follow the reference with the Julia `!` dropped (execute_centered_krfft! ->
execute_centered_krfft).  Unlike the reference, outputs never alias plan-owned
buffers: every execute call returns a fresh array/tensor or writes the caller's.

Array conventions
  * numpy inputs use the reference's indexing: a real field has shape (M1, M2, M3)
    (or (B, M1, M2, M3)); it is read x-fastest (Fortran order), exactly like a Julia
    Array.  Spectra are 1-D complex vectors (or (B, n_spec)) in spectral-ASU order.
    numpy calls go through the host-buffer C entry points (copies on the plan's stream).
  * torch CUDA tensors are device buffers in memory order: a field is a contiguous
    (M3, M2, M1) tensor (or (B, M3, M2, M1)), spectra (n_spec,) / (B, n_spec) complex.
    They run on torch's current stream without host synchronisation.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import symmetry as sym
from ._lib import LIB, CFFTDesc, CFFTError, CFFTInfo, CFFTTuning, check

PATH_AUTO, PATH_M2, PATH_CENTERED, PATH_M2Q, PATH_M7, PATH_FULLGRID = 0, 1, 2, 3, 4, 5
_REAL = {4: np.float32, 8: np.float64}
_CPLX = {4: np.complex64, 8: np.complex128}


def _torch():
    import torch  # device buffers and streams only

    return torch


def _is_tensor(x) -> bool:
    return type(x).__module__.startswith("torch")


class KRFFTPlan:
    """One device plan for a (group, grid, precision, batch): forward, backward and
    the SCFT diffusion step share it.  Mirrors GeneralCFFTPlan / CenteredKRFFTPlan /
    M2BackwardPlan / CenteredKRFFTBackwardPlan / CenteredSCFTPlan / M2SCFTPlan."""

    TUNING_DEFAULTS = dict(chunk_bytes=0, lanes=0, zr_slots=0, wide=-1, tma=-1, cluster=-1)

    def __init__(self, spec, ops_shifted, *, N=None, ds=0.0, lattice=None, precision=8, max_batch=1,
                 path=PATH_AUTO, device=True, tuning=None):
        N = tuple(spec.N if N is None else N)
        dim = len(N)
        self.spec = spec
        self.ops = list(ops_shifted)
        self.N = N
        self.dim = dim
        self.precision = int(precision)
        self.max_batch = int(max_batch)
        self.ds = float(ds)
        lat = np.eye(3) if lattice is None else np.asarray(lattice, dtype=np.float64)
        if lat.shape == (2, 2):
            l3 = np.eye(3)
            l3[:2, :2] = lat
            lat = l3
        self.lattice = lat
        R, t = sym._pack(self.ops)
        self._R, self._t = R, t  # keep alive for the call
        d = CFFTDesc()
        d.dim = dim
        for i in range(3):
            d.N[i] = N[i] if i < dim else 1
        d.n_ops = len(self.ops)
        d.R = R.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        d.t = t.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        for i, v in enumerate(lat.ravel(order="F")):
            d.lattice[i] = float(v)
        d.ds = self.ds
        d.precision = self.precision
        d.max_batch = self.max_batch
        d.path = int(path)
        h = ctypes.c_void_p()
        self.tuning = dict(self.TUNING_DEFAULTS, **(tuning or {}))
        if tuning and device:
            tu = CFFTTuning(**self.tuning)
            check(LIB.cfft_plan_create_tuned(ctypes.byref(d), ctypes.byref(tu), ctypes.byref(h)))
        else:
            create = LIB.cfft_plan_create if device else LIB.cfft_plan_create_host
            check(create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        info = CFFTInfo()
        check(LIB.cfft_plan_info(h, ctypes.byref(info)))
        self.info = info
        self.L = [info.L[i] for i in range(dim)]
        self.M = tuple(info.M[i] for i in range(dim))
        self.H = tuple(info.H[i] for i in range(dim))
        self.n_spec = info.n_spec
        self.centered = bool(info.centered)
        self.centering = sym.CENTERING_NAMES[info.centering]
        self.n_channels = info.n_channels
        if spec is not None and spec.n_spec != self.n_spec:
            raise CFFTError(1, "spectral ASU does not match the plan's operations")

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            LIB.cfft_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def mvol(self) -> int:
        return int(np.prod(self.M))

    # -- tables ---------------------------------------------------------------
    def q_tables(self):
        """Q-matrix first row (n_rep, Mvol) complex and gather indices (n_rep, Mvol), 0-based
        column-major subgrid positions, of an M2Q / M7 plan (_build_q_matrices!,
        src/q_fused_krfft.jl:182-413)."""
        d, mvol = self.info.n_rep, self.mvol
        q = np.zeros(2 * d * mvol, dtype=np.float64)
        gidx = np.zeros(d * mvol, dtype=np.int32)
        check(LIB.cfft_plan_q_tables(self._h, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), sym._ptr(gidx)))
        return (q[0::2] + 1j * q[1::2]).reshape(d, mvol), gidx.reshape(d, mvol)

    def spectral_asu(self):
        idx = np.zeros((self.n_spec, 3), dtype=np.int32)
        mult = np.zeros(self.n_spec, dtype=np.int32)
        check(LIB.cfft_plan_spectral_asu(self._h, sym._ptr(idx), sym._ptr(mult)))
        return idx[:, : self.dim].astype(np.int64), mult.astype(np.int64)

    def rep_ops(self):
        n = self.info.n_rep
        R = np.zeros((n, 9), dtype=np.int32)
        t = np.zeros((n, 3), dtype=np.int32)
        check(LIB.cfft_plan_rep_ops(self._h, sym._ptr(R), sym._ptr(t)))
        D = self.dim
        return [sym.SymOp(tuple(int(v) for v in R[k].reshape(3, 3)[:D, :D].ravel()), tuple(int(v) for v in t[k, :D]))
                for k in range(n)]

    def backward_tables(self):
        no, d = self.info.n_orbits, self.info.n_rep
        reps = np.zeros(no, dtype=np.int32)
        s = np.zeros(no * d, dtype=np.int32)
        p = np.zeros(no * d, dtype=np.int32)
        check(LIB.cfft_plan_backward_tables(self._h, sym._ptr(reps), sym._ptr(s), sym._ptr(p)))
        return reps, s.reshape(no, d), p.reshape(no, d)

    def kernel(self):
        K = np.zeros(self.n_spec, dtype=np.float64)
        check(LIB.cfft_plan_kernel(self._h, K.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return K

    def update_kernel(self, ds, lattice=None):
        self.ds = float(ds)
        lat_p = None
        if lattice is not None:
            lat = np.asarray(lattice, dtype=np.float64)
            if lat.shape == (2, 2):
                l3 = np.eye(3)
                l3[:2, :2] = lat
                lat = l3
            self.lattice = lat
            self._lat_buf = np.ascontiguousarray(lat.ravel(order="F"))
            lat_p = self._lat_buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        check(LIB.cfft_update_kernel(self._h, self.ds, lat_p))

    # -- array plumbing -------------------------------------------------------
    def _field_host(self, f):
        a = np.asarray(f, dtype=_REAL[self.precision])
        if a.shape == self.M:
            return np.ascontiguousarray(a.ravel(order="F")), 1, False
        if a.ndim == len(self.M) + 1 and a.shape[1:] == self.M:
            return np.ascontiguousarray(np.stack([x.ravel(order="F") for x in a])), a.shape[0], True
        raise CFFTError(1, f"field shape {a.shape} does not match subgrid {self.M}")

    def _unfield_host(self, flat, B, batched):
        f = flat.reshape(B, -1)
        out = np.stack([x.reshape(self.M, order="F") for x in f])
        return out if batched else out[0]

    def _batch_of(self, x, per):
        n = x.numel()
        if n % per:
            raise CFFTError(1, "buffer size is not a whole number of fields")
        return n // per

    @staticmethod
    def _stream():
        torch = _torch()
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _new_field_tensor(self, B, like):
        torch = _torch()
        dt = torch.float32 if self.precision == 4 else torch.float64
        shape = tuple(reversed(self.M))
        return torch.empty(((B,) + shape) if B > 1 else shape, dtype=dt, device=like.device)

    def _new_spec_tensor(self, B, like):
        torch = _torch()
        dt = torch.complex64 if self.precision == 4 else torch.complex128
        return torch.empty((B, self.n_spec) if B > 1 else (self.n_spec,), dtype=dt, device=like.device)

    def _check_tensor(self, x, kind):
        torch = _torch()
        if not x.is_cuda or not x.is_contiguous():
            raise CFFTError(1, "tensors must be contiguous CUDA tensors")
        want = {("r", 4): torch.float32, ("r", 8): torch.float64, ("c", 4): torch.complex64, ("c", 8): torch.complex128}
        if x.dtype != want[(kind, self.precision)]:
            raise CFFTError(1, f"tensor dtype {x.dtype} does not match plan precision {self.precision}")

    # -- execution ------------------------------------------------------------
    def forward(self, f0, out=None):
        """fft_reconstruct_centered! / fft_reconstruct!: subgrid f0 -> spectral ASU."""
        if _is_tensor(f0):
            self._check_tensor(f0, "r")
            B = self._batch_of(f0, self.mvol)
            F = self._new_spec_tensor(B, f0) if out is None else out
            self._check_tensor(F, "c")
            check(LIB.cfft_forward(self._h, ctypes.c_void_p(f0.data_ptr()), ctypes.c_void_p(F.data_ptr()), B, self._stream()))
            return F
        flat, B, batched = self._field_host(f0)
        F = np.empty((B, self.n_spec), dtype=_CPLX[self.precision])
        check(LIB.cfft_forward_host(self._h, flat.ctypes.data_as(ctypes.c_void_p), F.ctypes.data_as(ctypes.c_void_p), B))
        return F if batched else F[0]

    def backward(self, F, out=None):
        """ifft_unrecon_centered! / execute_m2_backward!: spectral ASU -> subgrid f0 (real)."""
        if _is_tensor(F):
            self._check_tensor(F, "c")
            B = self._batch_of(F, self.n_spec)
            f0 = self._new_field_tensor(B, F) if out is None else out
            self._check_tensor(f0, "r")
            check(LIB.cfft_backward(self._h, ctypes.c_void_p(F.data_ptr()), ctypes.c_void_p(f0.data_ptr()), B, self._stream()))
            return f0
        Fa = np.ascontiguousarray(np.asarray(F, dtype=_CPLX[self.precision]))
        batched = Fa.ndim == 2
        Fa = Fa.reshape(-1, self.n_spec)
        B = Fa.shape[0]
        flat = np.empty((B, self.mvol), dtype=_REAL[self.precision])
        check(LIB.cfft_backward_host(self._h, Fa.ctypes.data_as(ctypes.c_void_p), flat.ctypes.data_as(ctypes.c_void_p), B))
        return self._unfield_host(flat, B, batched)

    def scft_step(self, f0):
        """execute_centered_scft! / execute_m2_scft!: f0 <- IKRFFT(K . KRFFT(f0)).
        Tensors are updated in place; numpy input returns the new field."""
        if _is_tensor(f0):
            self._check_tensor(f0, "r")
            B = self._batch_of(f0, self.mvol)
            check(LIB.cfft_scft_step(self._h, ctypes.c_void_p(f0.data_ptr()), B, self._stream()))
            return f0
        flat, B, batched = self._field_host(f0)
        check(LIB.cfft_scft_step_host(self._h, flat.ctypes.data_as(ctypes.c_void_p), B))
        return self._unfield_host(flat, B, batched)

    def step_diffusion(self, q, w, dt, n_steps=1):
        """step_diffusion! repeated n_steps times (device tensors, in place on q)."""
        if not (_is_tensor(q) and _is_tensor(w)):
            raise CFFTError(1, "step_diffusion operates on CUDA tensors")
        self._check_tensor(q, "r")
        self._check_tensor(w, "r")
        B = self._batch_of(q, self.mvol)
        if w.numel() != q.numel():
            raise CFFTError(1, "w must have the layout of q")
        check(LIB.cfft_step_diffusion(self._h, ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                                      float(dt), int(n_steps), B, self._stream()))
        return q

    def fullgrid_to_subgrid(self, u, out=None):
        """fullgrid_to_subgrid! (src/q_fused_krfft.jl:698-719) on device tensors."""
        self._check_tensor(u, "r")
        nvol = int(np.prod(self.N))
        B = self._batch_of(u, nvol)
        f0 = self._new_field_tensor(B, u) if out is None else out
        check(LIB.cfft_fullgrid_to_subgrid(self._h, ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(f0.data_ptr()), B, self._stream()))
        return f0

    def subgrid_spectrum(self, f0, out=None):
        """G0 = FFT_M(f0) of each field on the whole subgrid, (B, M3, M2, M1) complex
        (cfft_subgrid_spectrum; the F000 of execute_staged!, the Y buffer of execute_m2_q!)."""
        torch = _torch()
        self._check_tensor(f0, "r")
        B = self._batch_of(f0, self.mvol)
        cdt = torch.complex64 if self.precision == 4 else torch.complex128
        shape = tuple(reversed(self.M))
        G0 = torch.empty(((B,) + shape) if B > 1 else shape, dtype=cdt, device=f0.device) if out is None else out
        self._check_tensor(G0, "c")
        check(LIB.cfft_subgrid_spectrum(self._h, ctypes.c_void_p(f0.data_ptr()), ctypes.c_void_p(G0.data_ptr()), B,
                                        self._stream()))
        return G0

    def subgrid_to_fullgrid(self, f0, out=None):
        """subgrid_to_fullgrid! (src/q_fused_krfft.jl:681-688) on device tensors."""
        torch = _torch()
        self._check_tensor(f0, "r")
        B = self._batch_of(f0, self.mvol)
        shape = tuple(reversed(self.N))
        u = torch.empty(((B,) + shape) if B > 1 else shape, dtype=f0.dtype, device=f0.device) if out is None else out
        check(LIB.cfft_subgrid_to_fullgrid(self._h, ctypes.c_void_p(f0.data_ptr()), ctypes.c_void_p(u.data_ptr()), B, self._stream()))
        return u


# ---------------------------------------------------------------------------
# Reference-named constructors and execute functions
# ---------------------------------------------------------------------------


# Alive parity offsets of the centring fold, in the reference's order (_alive_offsets,
# src/centering_fold.jl:111-127); the plane kernels fold the channels in this order.
_ALIVE_OFFSETS = {"I": [(0, 0, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)], "F": [(0, 0, 0), (1, 1, 1)],
                  "C": [(0, 0, 0), (1, 1, 0), (0, 0, 1), (1, 1, 1)], "A": [(0, 0, 0), (0, 1, 1), (1, 0, 0), (1, 1, 1)]}


@dataclass
class SubgridCenteringFoldPlan:
    """SubgridCenteringFoldPlan (src/centering_fold.jl:41-53): the fold's geometry.  The
    channel buffers and FFT plans of the reference have no counterpart: the fold, the
    channel FFTs and G0 assembly run fused in the library's plane kernels."""

    centering: str
    M: tuple
    H: tuple
    n_channels: int
    offsets: list       # alive parity offsets per channel
    twiddle_1d: list    # per channel, per dimension: e^{-2 pi i off_d n / M_d}, n < H_d
    sign_table: list    # per channel, 8 signs (-1)^{off . e}, e = (ex, ey, ez), ex fastest


def plan_centering_fold(centering, M):
    """plan_centering_fold (src/centering_fold.jl:60-104) for centring I, F, C or A (a
    string or a CenteringType) on a stride-2 subgrid M with even edges."""
    c = getattr(centering, "value", centering)
    if c not in _ALIVE_OFFSETS:
        raise CFFTError(1, f"Centering fold not applicable for {c}")
    M = tuple(int(m) for m in M)
    if any(m % 2 for m in M):
        raise CFFTError(1, "Subgrid dimensions must be even for centering fold")
    H = tuple(m // 2 for m in M)
    offs = _ALIVE_OFFSETS[c]
    tw = [tuple(np.ones(H[d], dtype=np.complex128) if o[d] == 0 else
                np.exp(-2j * np.pi * o[d] * np.arange(H[d]) / M[d]) for d in range(3)) for o in offs]
    signs = [tuple(1 - 2 * ((o[0] * (i & 1) + o[1] * ((i >> 1) & 1) + o[2] * ((i >> 2) & 1)) & 1) for i in range(8))
             for o in offs]
    return SubgridCenteringFoldPlan(c, M, H, len(offs), list(offs), tw, signs)


def _plan_array_call(fn, plans, ins, outs, in_kind, out_kind, per):
    n = len(plans)
    if n < 1 or len(ins) != n or len(outs) != n:
        raise CFFTError(1, "plans, inputs and outputs must be lists of the same non-zero length")
    batch = []
    for p, x, y in zip(plans, ins, outs):
        p._check_tensor(x, in_kind)
        p._check_tensor(y, out_kind)
        batch.append(p._batch_of(x, per(p)))
    hs = (ctypes.c_void_p * n)(*[p.handle.value for p in plans])
    xs = (ctypes.c_void_p * n)(*[x.data_ptr() for x in ins])
    ys = (ctypes.c_void_p * n)(*[y.data_ptr() for y in outs])
    bs = (ctypes.c_int * n)(*batch)
    check(fn(n, hs, xs, ys, bs, KRFFTPlan._stream()))
    return outs


def forward_plans(plans, fields, out=None):
    """The forward transforms of several plans in one library call (cfft_forward_plans):
    plans[i] on the CUDA tensor fields[i] (its subgrid batch), in list order on torch's
    current stream.  Returns the spectra (new tensors unless `out` is given)."""
    outs = list(out) if out is not None else [p._new_spec_tensor(p._batch_of(x, p.mvol), x)
                                              for p, x in zip(plans, fields)]
    return _plan_array_call(LIB.cfft_forward_plans, list(plans), list(fields), outs, "r", "c", lambda p: p.mvol)


def backward_plans(plans, spectra, out=None):
    """The backward transforms of several plans in one library call (cfft_backward_plans)."""
    outs = list(out) if out is not None else [p._new_field_tensor(p._batch_of(F, p.n_spec), F)
                                              for p, F in zip(plans, spectra)]
    return _plan_array_call(LIB.cfft_backward_plans, list(plans), list(spectra), outs, "c", "r", lambda p: p.n_spec)


def plan_krfft(spec, ops_shifted, *, precision=8, max_batch=1):
    """plan_krfft(spec, ops_shifted) auto-L variant (src/krfft.jl:301-389)."""
    return KRFFTPlan(spec, ops_shifted, precision=precision, max_batch=max_batch, path=PATH_M2)


def plan_m2_backward(spec, ops_shifted, *, precision=8, max_batch=1):
    """plan_m2_backward (src/krfft.jl:1101-1170)."""
    return KRFFTPlan(spec, ops_shifted, precision=precision, max_batch=max_batch, path=PATH_M2)


def plan_krfft_centered(spec, ops_shifted, *, centering="auto", precision=8, max_batch=1):
    """plan_krfft_centered (src/centering_fold.jl:328-367): centred fold when the
    group is centred with L = (2,2,2) and even M, else the plain M2 plan."""
    if centering not in ("auto", sym.detect_centering_type(ops_shifted, spec.N)):
        raise CFFTError(4, "explicit centring must match the operations")
    return KRFFTPlan(spec, ops_shifted, precision=precision, max_batch=max_batch, path=PATH_CENTERED)


def plan_centered_ikrfft(spec, ops_shifted, fwd):
    """plan_centered_ikrfft (src/centering_fold.jl:630-731): the forward plan already
    holds the backward orbit tables, so it is returned for the backward calls."""
    if spec.n_spec != fwd.n_spec:
        raise CFFTError(1, "spectral ASU does not match the forward plan")
    return fwd


def plan_centered_scft(spec, ops_shifted, N, ds, lattice, *, precision=8, max_batch=1):
    """plan_centered_scft (src/centering_fold.jl:868-896)."""
    return KRFFTPlan(spec, ops_shifted, N=N, ds=ds, lattice=lattice, precision=precision, max_batch=max_batch,
                     path=PATH_CENTERED)


def plan_m2_scft(N, sg_num, dim, ds, lattice, *, precision=8, max_batch=1):
    """plan_m2_scft (src/q_fused_krfft.jl:948-978)."""
    ops = sym.get_ops(sg_num, dim, N)
    _, ops_s = sym.find_optimal_shift(ops, N)
    spec = sym.calc_spectral_asu(ops_s, dim, N)
    return KRFFTPlan(spec, ops_s, N=N, ds=ds, lattice=lattice, precision=precision, max_batch=max_batch,
                     path=PATH_M2)


def plan_m2_q(N, sg_num, dim, ds, lattice, *, precision=8, max_batch=1, device=True):
    """plan_m2_q (src/q_fused_krfft.jl:83-169): the plain stride-L path whose SCFT step
    multiplies the subgrid spectrum by the first row of Q(q) = B^-1 diag(K) B."""
    ops = sym.get_ops(sg_num, dim, N)
    _, ops_s = sym.find_optimal_shift(ops, N)
    spec = sym.calc_spectral_asu(ops_s, dim, N)
    return KRFFTPlan(spec, ops_s, N=N, ds=ds, lattice=lattice, precision=precision, max_batch=max_batch,
                     path=PATH_M2Q, device=device)


def execute_m2_q(plan, f0):
    """execute_m2_q! (src/q_fused_krfft.jl:553-576): f0 <- real(IFFT(Q . FFT(f0)))."""
    return plan.scft_step(f0)


def plan_m7_scft(N, sg_num, dim, ds, lattice, *, precision=8, max_batch=1, device=True):
    """plan_m7_scft (src/q_fused_krfft.jl:822-850): centring fold + channel FFTs + Q-multiply
    + unfold.  Raises CFFTError for P lattices and odd subgrids, like the reference."""
    ops = sym.get_ops(sg_num, dim, N)
    _, ops_s = sym.find_optimal_shift(ops, N)
    spec = sym.calc_spectral_asu(ops_s, dim, N)
    return KRFFTPlan(spec, ops_s, N=N, ds=ds, lattice=lattice, precision=precision, max_batch=max_batch,
                     path=PATH_M7, device=device)


def execute_m7_scft(plan, f0):
    """execute_m7_scft! (src/q_fused_krfft.jl:870-895)."""
    return plan.scft_step(f0)


class CenteringPreFoldPlan:
    """CenteringPreFoldPlan / plan_centering_prefold (src/centering_prefold.jl:27-58): the
    channel definition of the prefold (parity classes kept, halved grid, shift offsets of
    the folded copies).  Host metadata only; the device prefold is plan_krfft_prefold."""

    def __init__(self, centering, N):
        N = tuple(int(n) for n in N)
        h = tuple(n // 2 for n in N)
        if centering == "I":
            self.N_sub, self.parities = h, [(0, 0, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)]
            self.shift_offsets = [(h[0], 0, 0), (0, h[1], 0), (0, 0, h[2])]
        elif centering == "F":
            self.N_sub, self.parities, self.shift_offsets = h, [(0, 0, 0), (1, 1, 1)], [(h[0], 0, 0)]
        elif centering == "C":
            self.N_sub, self.parities, self.shift_offsets = (h[0], h[1], N[2]), [(0, 0, 0), (1, 1, 0)], [(h[0], 0, 0)]
        elif centering == "A":
            self.N_sub, self.parities, self.shift_offsets = (N[0], h[1], h[2]), [(0, 0, 0), (0, 1, 1)], [(0, h[1], 0)]
        else:
            raise CFFTError(1, "CentP has no pre-fold")
        self.centering, self.N_full, self.n_channels = centering, N, len(self.parities)


def plan_centering_prefold(centering, N):
    """plan_centering_prefold (src/centering_prefold.jl:36-58)."""
    return CenteringPreFoldPlan(centering, N)


def plan_krfft_prefold(ops_shifted, N, *, precision=8, max_batch=1, ds=0.0, lattice=None, device=True):
    """The prefold CenteredKRFFTPlan (plan_krfft_centered(ops, N), src/centering_prefold.jl:
    175-205; that constructor shares its name and struct name with the fold plan in the
    reference): a full-grid plan whose forward folds the whole grid into the parity
    channels of (N/2)^3 and merges the channel spectra onto the spectral ASU.  Its
    backward returns the whole grid with the symmetry fill."""
    dim = len(N)
    spec = sym.calc_spectral_asu(ops_shifted, dim, N)
    return KRFFTPlan(spec, ops_shifted, N=N, ds=ds, lattice=np.eye(3) if lattice is None else lattice,
                     precision=precision, max_batch=max_batch, path=PATH_FULLGRID, device=device)


def execute_prefold_krfft(plan, u):
    """execute_centered_krfft!(::CenteredKRFFTPlan (prefold), u) (src/centering_prefold.jl:
    236-244): prefold + channel FFTs + _merge_channels! -> spectrum on the ASU."""
    return plan.forward(u)


def execute_krfft(plan, u):
    """execute_krfft! (src/krfft.jl:608-621): pack the stride-L subgrid of u, FFT, reconstruct."""
    return plan.forward(fullgrid_to_subgrid(plan, u))


def fft_reconstruct(plan, f0):
    """fft_reconstruct! (src/krfft.jl:554-562)."""
    return plan.forward(f0)


def execute_centered_krfft(plan, u):
    """execute_centered_krfft! (src/centering_fold.jl:392-413)."""
    return plan.forward(fullgrid_to_subgrid(plan, u))


def fft_reconstruct_centered(plan, f0):
    """fft_reconstruct_centered! (src/centering_fold.jl:421-431)."""
    return plan.forward(f0)


def execute_m2_backward(plan, F):
    """execute_m2_backward! (src/krfft.jl:1269-1277): returns the real subgrid field."""
    return plan.backward(F)


def execute_centered_ikrfft(plan, F, f0_out=None):
    """execute_centered_ikrfft! (src/centering_fold.jl:745-764)."""
    f0 = plan.backward(F, out=f0_out if _is_tensor(F) else None)
    if f0_out is not None and not _is_tensor(F):
        f0_out[...] = f0
        return f0_out
    return f0


def ifft_unrecon_centered(plan, F):
    """ifft_unrecon_centered! (src/centering_fold.jl:772-775)."""
    return plan.backward(F)


def execute_centered_scft(plan, f0):
    """execute_centered_scft! (src/centering_fold.jl:908-931)."""
    return plan.scft_step(f0)


def execute_m2_scft(plan, f0):
    """execute_m2_scft! (src/q_fused_krfft.jl:989-1026)."""
    return plan.scft_step(f0)


def update_kernel(plan, spec, N, ds_new, lattice):
    """update_kernel! (src/centering_fold.jl:939-953)."""
    plan.update_kernel(ds_new, lattice)


def update_m2_kernel(plan, N, sg_num, dim, ds_new, lattice):
    """update_m2_kernel! (src/q_fused_krfft.jl:1036-1052)."""
    plan.update_kernel(ds_new, lattice)


def fullgrid_to_subgrid(plan, u):
    """fullgrid_to_subgrid! (src/q_fused_krfft.jl:698-719)."""
    if _is_tensor(u):
        return plan.fullgrid_to_subgrid(u)
    a = np.asarray(u)
    sl = tuple(slice(0, None, l) for l in plan.L)
    return np.array(a[sl] if a.shape == tuple(plan.N) else a[(slice(None),) + sl])


def subgrid_to_fullgrid(plan, f0):
    """subgrid_to_fullgrid! (src/q_fused_krfft.jl:681-688)."""
    return plan.subgrid_to_fullgrid(f0)


class DiffusionSolver:
    """QFusedDiffusionSolver (src/diffusion_solver.jl:82-91) on the device plan: the
    stride-L subgrid field, the M2Q Q-matrix step (plan_m2_q) on the device."""

    def __init__(self, plan):
        self.plan = plan

    def apply_diffusion_operator(self, u):
        """apply_diffusion_operator! (src/diffusion_solver.jl:87-91)."""
        return self.plan.scft_step(u)

    def step(self, u, w, dt, n_steps=1):
        return self.plan.step_diffusion(u, w, dt, n_steps)


class Diagonal:
    """The diagonal Q of calc_matrix_q (a LinearAlgebra.Diagonal in the reference)."""

    def __init__(self, d):
        self.diag = np.asarray(d, dtype=np.float64)

    @property
    def shape(self):
        return (len(self.diag), len(self.diag))

    def __getitem__(self, ij):
        i, j = ij
        return self.diag[i] if i == j else 0.0

    def __matmul__(self, v):
        return self.diag[:, None] * v if np.ndim(v) == 2 else self.diag * v


def calc_gradient_term(N, ds, lattice):
    """calc_gradient_term (src/matrix_q.jl:18-48): k -> exp(-|B k|^2 ds) with the integer
    harmonic k and B = 2 pi inv(A)^T (no division by N)."""
    B = 2 * np.pi * np.linalg.inv(np.asarray(lattice, dtype=np.float64)).T

    def kernel(k):
        K = B @ np.asarray(k, dtype=np.float64)
        return float(np.exp(-np.dot(K, K) * ds))

    return kernel


def calc_matrix_q(indexing, kernel_func):
    """calc_matrix_q (src/matrix_q.jl:61-79): Q_ii = kernel(get_k_vector(i))."""
    return Diagonal([kernel_func(sym.get_k_vector(indexing, i)) for i in range(indexing.n_spec)])


def plan_diffusion(N, lattice, sg_num, dim, ds, *, method="qfused", precision=8, max_batch=1):
    """plan_diffusion (src/diffusion_solver.jl:165-252) on the device: :qfused, the M2Q
    subgrid solver.  The reference's :matrix branch (a dense real-ASU x spectral-ASU
    transform and its pseudo-inverse, src/diffusion_solver.jl:20-80) is a host-side
    dense solve outside the KRFFT path this library accelerates, and is refused, as is
    the :krfft branch: the legacy solver on the mode-B plan_krfft(real_asu, spec_asu,
    ops) of src/krfft.jl:119-389 (an FFT of every orbit block of a stride-2 packing,
    recombined by a sparse matrix and its adjoint, map_fft! / map_ifft!), whose scale the
    reference derived empirically (src/diffusion_solver.jl:93-160).  :qfused computes the
    same contour step on one subgrid."""
    method = str(method).lstrip(":")
    if method == "qfused":
        ops = sym.get_ops(sg_num, dim, N)
        _, ops_s = sym.find_optimal_shift(ops, N)
        spec = sym.calc_spectral_asu(ops_s, dim, N)
        return DiffusionSolver(KRFFTPlan(spec, ops_s, N=N, ds=ds, lattice=lattice, precision=precision,
                                         max_batch=max_batch, path=PATH_M2Q))
    raise CFFTError(4, f"method {method!r}: the device solver is :qfused (:matrix and :krfft are not built)")


def step_diffusion(solver, u, w, dt, n_steps=1):
    """step_diffusion! (src/diffusion_solver.jl:254-267): u <- e^{-w dt/2} D(e^{-w dt/2} u)."""
    return solver.step(u, w, dt, n_steps)


def apply_diffusion_operator(solver, u):
    """apply_diffusion_operator! (src/diffusion_solver.jl:66-91)."""
    return solver.apply_diffusion_operator(u)
