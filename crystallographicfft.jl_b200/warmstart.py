"""Training data, training loop and evaluation of the learned SCFT warm start (no
reference counterpart).

- `GroupGrid`: a group on a grid with its seeded plain start (Gaussian-filtered noise
  symmetrised over the group, the same noise for every (chiN, f)).
- `generate`: converged fields of draws (chiN, f) from the plain start, solved on
  several host threads: the training and held-out sets (`generate_sharded` splits the
  draws over the GPUs of a process group and gathers the results).
- `train`: Adam over shuffled mini-batches of one group at a time (contexts of one
  model bound to each group's plan), cosine learning-rate decay; optionally data
  parallel over the ranks of a process group (one gradient all-reduce per step).
- `time_to_tol`: FP32 iterations to a switch residual, then FP64 to the tolerance,
  from the plain start (simple mixing first, `PLAIN`) or from a prediction (Anderson
  mixing from the first iteration, `WARM`), timed with CUDA events.

Fields are [w_A | w_B] (2, M3, M2, M1) on each plan's subgrid.
"""
from __future__ import annotations

import time

import numpy as np

from . import sno
from . import symmetry as sym
from ._lib import CFFTError
from .plans import _torch
from .scft import initial_fields, plan_scft
from .sno import GROUP_SLOTS, SpectralNeuralOperator

CELL = 3.8 * np.sqrt(6.0)  # cubic cell edge in units of Rg (3.8 b sqrt(N))
# Mixing schedules: from the plain start, simple mixing first lets the ordered structure grow
# out of the unstable modes (Anderson mixing from a near-uniform start converges to the
# disordered state); a prediction starts with Anderson mixing.
PLAIN = dict(min_simple=100, lam_simple=0.1, anderson_start=0.2)       # timed plain start
PLAIN_DATA = dict(min_simple=200, lam_simple=0.1, anderson_start=0.2)  # training-data solves
WARM = dict(min_simple=0, lam_simple=0.1, anderson_start=0.3)          # from a prediction


class GroupGrid:
    """Group and grid of a family of solves: shifted operations, the seeded plain start
    (the same noise for every (chiN, f), so the plain start picks the same structure
    across draws), and SCFT plans per solve."""

    def __init__(self, sg, n, Ns=100, cell=CELL, seed=0):
        self.sg, self.N, self.Ns, self.cell = sg, (n, n, n), Ns, cell
        self.shift, self.ops = sym.find_optimal_shift(sym.get_ops(sg, 3, self.N), self.N)
        self.spec = sym.calc_spectral_asu(self.ops, 3, self.N)
        self.seed = seed
        self._noise = {}

    def solver(self, f, chiN, precision, tol, schedule, max_iter=3000, history=20):
        return plan_scft(self.sg, self.N, self.cell, f=f, chiN=chiN, Ns=self.Ns, precision=precision, ops=self.ops,
                         tol=tol, max_iter=max_iter, history=history, **schedule)

    def plain_start(self, f, chiN, L):
        """[w_A | w_B] = (chiN (1 - f) + eta, chiN f - eta), eta the seeded filtered noise."""
        key = tuple(L)
        if key not in self._noise:
            self._noise[key] = initial_fields(self.ops, self.N, L, 0.0, 0.0, seed=self.seed, sigma=2.0,
                                              amplitude=1.0)[0]
        eta = self._noise[key]
        return np.stack([chiN * (1.0 - f) + eta, chiN * f - eta])


def generate(gg, draws, tol=1e-4, schedule=None, max_iter=1000, threads=8, log=None):
    """Converged FP32 fields of every (chiN, f) in draws from the plain start: a float32
    CUDA tensor (len(draws), 2, M3, M2, M1), the final states and the solve times.  The
    solves run on `threads` host threads, each with its own CUDA stream and plans (the
    SCFT driver synchronises once per iteration, so one solve leaves the GPU mostly idle)."""
    import threading

    torch = _torch()
    schedule = schedule or PLAIN_DATA
    n = len(draws)
    probe, _ = gg.solver(0.4, 20.0, 4, tol, schedule)
    L, M = probe.L, probe.M
    probe.close()
    gg.plain_start(0.4, 20.0, L)  # noise computed once, before the threads start
    out = torch.empty((n, 2) + tuple(reversed(M)), dtype=torch.float32, device="cuda")
    states, times = [None] * n, [0.0] * n
    errors = []

    def work(indices):
        st = torch.cuda.Stream()
        try:
            with torch.cuda.stream(st):
                for i in indices:
                    chiN, f = float(draws[i][0]), float(draws[i][1])
                    plan, sol = gg.solver(f, chiN, 4, tol, schedule, max_iter=max_iter)
                    w = torch.tensor(gg.plain_start(f, chiN, L), dtype=torch.float32, device="cuda").contiguous()
                    t0 = time.time()
                    try:
                        states[i] = sol.solve(w)
                    except CFFTError as e:  # a diverged solve is reported, not fatal
                        states[i] = dict(Q=float("nan"), F=float("nan"), err=float("inf"), iterations=-1,
                                         converged=False, error=str(e))
                    times[i] = time.time() - t0
                    out[i].copy_(w)
                    sol.close()
                    plan.close()
            st.synchronize()
        except Exception as e:  # reported after the join
            errors.append(e)

    parts = [list(range(k, n, threads)) for k in range(threads)]
    ths = [threading.Thread(target=work, args=(p,)) for p in parts if p]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    if errors:
        raise errors[0]
    torch.cuda.synchronize()
    if log:
        conv = sum(1 for s in states if s["converged"])
        log(f"group {gg.sg} {gg.N[0]}^3: {n} draws, {conv} converged, mean {np.mean([s['iterations'] for s in states]):.0f}"
            f" iterations, {np.sum(times):.1f} s of solves")
    return out, states, times


def gather_rows(local, extra, n, dist):
    """Reassemble rows computed round-robin over the ranks (rank r holds rows r, r + world,
    ...): `local` is this rank's tensor of rows and `extra` a list of per-row Python
    objects.  Returns the n rows in order and the n objects, on every rank."""
    torch = _torch()
    world, rank = dist.get_world_size(), dist.get_rank()
    n_max = (n + world - 1) // world
    pad = torch.zeros((n_max,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad)
    objs = [None] * world
    dist.all_gather_object(objs, list(extra))
    out = torch.empty((n,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    rows = [None] * n
    for r in range(world):
        idx = list(range(r, n, world))
        if idx:
            out[torch.as_tensor(idx, device=local.device)] = bufs[r][: len(idx)]
        for j, i in enumerate(idx):
            rows[i] = objs[r][j]
    return out, rows


def generate_sharded(gg, draws_, dist, **kw):
    """`generate` with the draws split round-robin over the ranks of a process group (one
    GPU per rank): every rank solves its share and receives all fields, states and times."""
    world, rank = dist.get_world_size(), dist.get_rank()
    mine = draws_[rank::world]
    fld, st, tm = generate(gg, mine, **kw)
    out, rows = gather_rows(fld, list(zip(st, tm)), len(draws_), dist)
    return out, [r[0] for r in rows], [r[1] for r in rows]


def draws(n, seed, chiN_range=(12.0, 30.0), f_range=(0.30, 0.50)):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(*chiN_range, n), rng.uniform(*f_range, n)], axis=1)


def train(model, sets, epochs, batch=16, lr=1e-3, lr_final=1e-5, seed=0, log=None, max_seconds=None, dist=None):
    """sets: list of (ctx, params (n, 2), fields tensor (n, 2, M...)).  Cosine learning-rate
    decay from lr to lr_final; one mini-batch of one group per step.  Returns the mean
    loss of each epoch; stops after the epoch that passes max_seconds.

    With `dist` (torch.distributed, one GPU per rank, every rank holding the same sets)
    each mini-batch is split over the ranks and the gradients are averaged by one
    all-reduce per step (SpectralNeuralOperator's data-parallel step); every rank draws
    the same shuffles from `seed`, so the ranks agree on the batches and the weights."""
    torch = _torch()
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    gbuf = torch.empty(sno.N_PARAMS + 1, dtype=torch.float32, device="cuda") if world > 1 else None
    t0 = time.time()
    rng = np.random.default_rng(seed)
    steps_per_epoch = sum((len(p) + batch - 1) // batch for _, p, _ in sets)
    total = epochs * steps_per_epoch
    k, hist = 0, []
    for ep in range(epochs):
        jobs = []
        for si, (_, p, _) in enumerate(sets):
            perm = rng.permutation(len(p))
            jobs += [(si, perm[i:i + batch]) for i in range(0, len(p), batch)]
        rng.shuffle(jobs)
        acc = 0.0
        for si, idx in jobs:
            ctx, p, fld = sets[si]
            cur = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(total - 1, 1)))
            if world > 1:
                mine = sno.shard_of(idx, rank, world)
                sel = torch.as_tensor(mine, device="cuda")
                acc += ctx.train_step_data_parallel(p[mine], fld.index_select(0, sel).contiguous(), len(idx), dist,
                                                    lr=cur, grad_buf=gbuf)
            else:
                sel = torch.as_tensor(idx, device="cuda")
                acc += ctx.train_step(p[idx], fld.index_select(0, sel).contiguous(), lr=cur)
            k += 1
        hist.append(acc / len(jobs))
        if log and (ep % 10 == 0 or ep == epochs - 1):
            log(f"epoch {ep}: loss {hist[-1]:.3e}")
        if max_seconds is not None and time.time() - t0 > max_seconds:
            if log:
                log(f"stopped after epoch {ep}: {time.time() - t0:.0f} s")
            break
    return hist


def time_to_tol(gg, chiN, f, start, *, warm, tol=1e-6, switch=1e-5, predict=None, plain=None):
    """Wall time (CUDA events), iterations and final state of a solve: FP32 fields to the
    residual `switch`, then FP64 to `tol`.  `start` is a float tensor 2 x M-grid, or None
    with `predict` a callable returning the start (its time is counted).  `warm` picks
    the schedule of the FP32 phase (WARM, else `plain` or PLAIN)."""
    torch = _torch()
    sch = WARM if warm else (plain or PLAIN)
    p32, s32 = gg.solver(f, chiN, 4, switch, sch, max_iter=600)  # FP64 finishes what FP32 rounding leaves
    p64, s64 = gg.solver(f, chiN, 8, tol, WARM)
    probe = (predict() if start is None else start).to(torch.float32).contiguous()
    s32.evaluate(probe.clone())  # captures the propagator graphs outside the timed region
    s64.evaluate(probe.double())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    w = (predict() if start is None else start).to(torch.float32).contiguous().clone()
    a = s32.solve(w)
    w64 = w.double()
    b = s64.solve(w64)
    e1.record()
    torch.cuda.synchronize()
    res = dict(seconds=e0.elapsed_time(e1) / 1000.0, iterations_fp32=a["iterations"], iterations_fp64=b["iterations"],
               F=b["F"], err=b["err"], converged=bool(b["converged"]))
    for o in (s32, s64, p32, p64):
        o.close()
    return res


def load_pretrained(path):
    model = SpectralNeuralOperator()
    model.load(path)
    return model


__all__ = ["GroupGrid", "generate", "draws", "train", "time_to_tol", "load_pretrained", "PLAIN", "PLAIN_DATA", "WARM",
           "CELL", "GROUP_SLOTS"]
