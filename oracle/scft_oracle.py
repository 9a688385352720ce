"""FP64 CPU oracle of the SCFT driver for an AB diblock melt (TEST INFRASTRUCTURE ONLY).

The reference stops at the contour step (step_diffusion!, src/diffusion_solver.jl:254-282;
execute_m2_scft!, src/q_fused_krfft.jl:989-1026); it has no SCFT driver.  This module is
the textbook self-consistent field iteration built on that step, restated in numpy so
the library's device driver (cfft_scft_*) can be checked against it:

- Gaussian chain, contour s in [0, 1] with Ns steps of ds = 1/Ns, the A block on
  s < f (NA = round(f Ns) steps) and the B block after it; lengths in units of Rg.
- Propagators: q(r, 0) = 1 and q_dagger(r, 1) = 1, each step
  q <- e^{-w ds/2} IFFT(e^{-k^2 ds} FFT(e^{-w ds/2} q)) on the stride-L subgrid (the
  M2 SCFT step of the oracle's KRFFT with K = exp(-ds |2 pi A^-T h|^2)).
- Q = <q(r, 1)> (mean over the subgrid, which equals the mean over the full grid for
  symmetric fields); phi_A = (1/Q) int_0^f q q_dagger ds and phi_B over [f, 1] by
  Simpson's rule (trapezoid when a block has an odd number of steps).
- Residuals of the incompressible melt (w_A = chiN phi_B + xi, w_B = chiN phi_A + xi,
  xi = (w_A + w_B - chiN) / 2):
  d_A = chiN (phi_B - 1/2) + (w_B - w_A)/2,  d_B = chiN (phi_A - 1/2) + (w_A - w_B)/2;
  error = sqrt(sum(d_A^2 + d_B^2) / sum(w_A^2 + w_B^2)).
- Free energy per chain: the field-theoretic Hamiltonian
  F = -ln Q + <(w_B - w_A)^2 / (4 chiN) - (w_A + w_B) / 2> + chiN / 4, equal at the saddle
  point to the mean-field -ln Q + <chiN phi_A phi_B - w_A phi_A - w_B phi_B> and stationary
  there (error second order in the residual); `F_mf` is the mean-field form.
- Mixing: simple mixing w += lam_s d for the first `min_simple` iterations and while the
  error is above `anderson_start`, then
  Anderson mixing (D. G. Anderson, J. ACM 12, 547 (1965); as used for SCFT by
  R. B. Thompson et al., J. Chem. Phys. 120, 31 (2004) and M. W. Matsen, Eur. Phys. J.
  E 30, 361 (2009)) over the last `history` iterations:
  U_mn = (d_k - d_{k-m}).(d_k - d_{k-n}), V_m = (d_k - d_{k-m}).d_k, U c = V,
  w_{k+1} = w_k + sum c_m (w_{k-m} - w_k) + lam (d_k + sum c_m (d_{k-m} - d_k)).
"""
from __future__ import annotations

import numpy as np

from . import krfft_oracle as O


def simpson_weights(n):
    """Weights of n + 1 equally spaced samples (Simpson for even n, trapezoid otherwise), times ds."""
    w = np.ones(n + 1)
    if n == 0:
        return np.zeros(1)
    if n % 2 == 0:
        w[1:-1:2] = 4.0
        w[2:-1:2] = 2.0
        return w / 3.0
    w[0] = w[-1] = 0.5
    return w


class SCFTOracle:
    def __init__(self, ops_shifted, N, f, chiN, Ns, lattice, history=20, lam_simple=0.1, lam_anderson=1.0,
                 anderson_start=0.2, min_simple=0):
        self.N, self.f, self.chiN, self.Ns = tuple(N), float(f), float(chiN), int(Ns)
        self.NA = int(round(self.f * self.Ns))
        self.ds = 1.0 / self.Ns
        self.plan = O.plan_m2_scft_ops(ops_shifted, self.N, self.ds, lattice)
        self.history, self.lam_s, self.lam_a, self.a_start = history, lam_simple, lam_anderson, anderson_start
        self.min_simple = int(min_simple)

    def _step(self, q, w):
        return O.step_diffusion(lambda x: O.execute_m2_scft(self.plan, x), q, w, self.ds)

    def propagators(self, wA, wB):
        """q[j] = q(r, j ds) and qd[j] = q_dagger(r, j ds), j = 0..Ns."""
        Ns, NA = self.Ns, self.NA
        q = [np.ones_like(wA)]
        for i in range(Ns):
            q.append(self._step(q[-1], wA if i < NA else wB))
        qd = [np.ones_like(wA)]
        for i in range(Ns):  # segment (Ns-1-i, Ns-i)
            qd.append(self._step(qd[-1], wA if Ns - 1 - i < NA else wB))
        return q, qd[::-1]

    def evaluate(self, wA, wB):
        """Q, phi_A, phi_B, residuals, error and free energy of the fields (wA, wB)."""
        q, qd = self.propagators(wA, wB)
        Ns, NA, ds, chiN = self.Ns, self.NA, self.ds, self.chiN
        Q = float(np.mean(q[Ns]))
        sa, sb = simpson_weights(NA), simpson_weights(Ns - NA)
        phiA = sum(sa[j] * q[j] * qd[j] for j in range(NA + 1)) * ds / Q
        phiB = sum(sb[j] * q[NA + j] * qd[NA + j] for j in range(Ns - NA + 1)) * ds / Q
        dA = chiN * (phiB - 0.5) + 0.5 * (wB - wA)
        dB = chiN * (phiA - 0.5) + 0.5 * (wA - wB)
        err = float(np.sqrt((np.sum(dA ** 2) + np.sum(dB ** 2)) / (np.sum(wA ** 2) + np.sum(wB ** 2))))
        F_mf = -np.log(Q) + float(np.mean(chiN * phiA * phiB - wA * phiA - wB * phiB))
        F = -np.log(Q) + float(np.mean((wB - wA) ** 2 / (4.0 * chiN) - 0.5 * (wA + wB))) + 0.25 * chiN
        return dict(Q=Q, phiA=phiA, phiB=phiB, dA=dA, dB=dB, err=err, F=F, F_mf=F_mf)

    def solve(self, wA, wB, tol=1e-6, max_iter=2000, callback=None):
        """Iterate from (wA, wB) until error < tol.  Returns (wA, wB, last evaluation, iterations)."""
        W, D = [], []
        w = np.concatenate([wA.ravel(), wB.ravel()])
        shape, n = wA.shape, wA.size
        for it in range(max_iter):
            ev = self.evaluate(w[:n].reshape(shape), w[n:].reshape(shape))
            if callback:
                callback(it, ev)
            if ev["err"] < tol:
                return w[:n].reshape(shape), w[n:].reshape(shape), ev, it
            d = np.concatenate([ev["dA"].ravel(), ev["dB"].ravel()])
            if ev["err"] > self.a_start or it < self.min_simple:
                W.clear()
                D.clear()
                w = w + self.lam_s * d
                continue
            W.append(w.copy())
            D.append(d)
            if len(W) > self.history + 1:
                W.pop(0)
                D.pop(0)
            m = len(W) - 1
            Wn, Dn = w.copy(), d.copy()
            if m > 0:
                dk = D[-1]
                dd = [dk - D[-1 - i] for i in range(1, m + 1)]
                U = np.array([[a @ b for b in dd] for a in dd])
                V = np.array([a @ dk for a in dd])
                c = np.linalg.solve(U, V)
                for i in range(1, m + 1):
                    Wn += c[i - 1] * (W[-1 - i] - W[-1])
                    Dn += c[i - 1] * (D[-1 - i] - D[-1])
            w = Wn + self.lam_a * Dn
        ev = self.evaluate(w[:n].reshape(shape), w[n:].reshape(shape))
        return w[:n].reshape(shape), w[n:].reshape(shape), ev, max_iter


def initial_fields(oops, N, L, f, chiN, seed=0, sigma=2.0, amplitude=1.0):
    """Seeded start: i.i.d. N(0, 1) on the full grid, Gaussian filter of width sigma grid
    points (in Fourier space), averaged over the group, scaled to standard deviation
    `amplitude`; w_A = chiN (1 - f) + eta, w_B = chiN f - eta on the stride-L subgrid."""
    rng = np.random.default_rng(seed)
    u = rng.standard_normal(N)
    k = [np.fft.fftfreq(n) for n in N]
    K2 = sum(np.meshgrid(*[(2 * np.pi * kk) ** 2 for kk in k], indexing="ij"))
    u = np.real(np.fft.ifftn(np.fft.fftn(u) * np.exp(-0.5 * sigma ** 2 * K2)))
    eta = _symmetrize(oops, u, N)
    eta = eta - eta.mean()
    eta *= amplitude / max(eta.std(), 1e-300)
    sub = O.pack_stride(eta, L)
    return chiN * (1.0 - f) + sub, chiN * f - sub


def _symmetrize(oops, u, N):
    """Average of u over the operations: (1/|G|) sum_g u(g x)."""
    X = O._all_coords(N)
    Nv = np.asarray(N, dtype=np.int64)[:, None]
    flat = u.ravel(order="F")
    acc = np.zeros(flat.size)
    for op in oops:
        acc += flat[O._lin_cm(np.mod(op.Rm @ X + op.tv[:, None], Nv), N)]
    return (acc / len(oops)).reshape(N, order="F")
