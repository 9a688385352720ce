"""Mixed batches of plans: the autotuner of each plan's execution choices and the runner
that replays the work of many plans as one CUDA graph.

Neither has a reference counterpart: CrystallographicFFT.jl transforms one field at a
time on the CPU.  They serve batches of fields of uneven space group and grid size.

* autotune_plan times candidate execution choices (cfft_tuning: chunk size, lanes,
  fused-z slots per CTA, the wide backward gather, the bulk-copy plane kernels, the
  fused cluster kernels) on the device with CUDA events, by coordinate descent from the
  defaults, and caches the winner in a JSON file keyed by device, operations, grid,
  precision, batch, operation and path; autotune_path also chooses the decomposition
  (centring fold, plain stride-L, Q-matrix steps).
* MultiPlanStep runs one callable per plan, each on its own stream forked from and
  joined to the caller's stream.  Its first call runs them directly and then captures
  the whole set into a single CUDA graph (capturing runs nothing); every later call
  replays that graph with one launch.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from ._lib import CFFTError
from .plans import KRFFTPlan, _torch

KNOBS = (
    ("lanes", (1, 2, 3)),
    ("chunk_bytes", (16 << 20, 32 << 20, 64 << 20, 128 << 20)),
    ("zr_slots", (2, 4)),
    ("wide", (0, 1)),
    ("tma", (0, 1, 3)),
    ("cluster", (0, 8, 16)),
)


def _default_cache():
    return os.environ.get("CFFT_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cfft_b200",
                                                          "tuning.json"))


def _ops_signature(ops):
    h = hashlib.sha1()
    for op in ops:
        h.update(np.asarray(op.R, dtype=np.int64).tobytes())
        h.update(np.asarray(op.t, dtype=np.int64).tobytes())
    return h.hexdigest()[:12]


def _time_op(plan, op, batch, n_steps, reps):
    """Median device time (ms) of one `op` on `batch` random fields."""
    torch = _torch()
    dt = torch.float64 if plan.precision == 8 else torch.float32
    shape = (batch,) + tuple(reversed(plan.M))
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(shape, generator=g, device="cuda", dtype=dt)
    w = 0.1 * torch.randn(shape, generator=g, device="cuda", dtype=dt)
    y = torch.empty_like(x)
    F = torch.empty((batch, plan.n_spec), dtype=torch.complex128 if plan.precision == 8 else torch.complex64,
                    device="cuda")

    def run():
        if op in ("fwdbwd", "mixed"):
            plan.forward(x, out=F)
            plan.backward(F, out=y)
        if op in ("step", "mixed"):
            plan.step_diffusion(y, w, 0.01, n_steps)

    for _ in range(2):
        run()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        run()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    return float(np.median(times))


def autotune_plan(spec, ops_shifted, *, N=None, precision=4, batch=1, op="fwdbwd", n_steps=50, ds=0.01,
                  lattice=None, path=0, reps=5, cache_path=None, knobs=KNOBS):
    """Execution choices for a plan of these operations, grid, precision and batch that
    minimise the device time of `op` ("fwdbwd", "step": n_steps diffusion steps, or
    "mixed": both).  Returns (tuning dict, best time in ms); cached in cache_path."""
    torch = _torch()
    N = tuple(spec.N if N is None else N)
    cache_path = cache_path or _default_cache()
    key = "|".join([torch.cuda.get_device_name(), _ops_signature(ops_shifted), "x".join(map(str, N)), str(precision),
                    str(batch), op, str(n_steps), str(path),
                    hashlib.sha1(repr(tuple((k, tuple(v)) for k, v in knobs)).encode()).hexdigest()[:8]])
    cache = {}
    if os.path.exists(cache_path):
        try:
            cache = json.load(open(cache_path))
        except (OSError, ValueError):
            cache = {}
    if key in cache:
        return dict(cache[key]["tuning"]), cache[key]["ms"]
    cur = dict(KRFFTPlan.TUNING_DEFAULTS)

    def measure(tu):
        try:
            plan = KRFFTPlan(spec, ops_shifted, N=N, ds=ds, lattice=lattice, precision=precision, max_batch=batch,
                             path=path, tuning=tu)
        except CFFTError:
            return None
        try:
            return _time_op(plan, op, batch, n_steps, reps)
        except CFFTError:
            return None
        finally:
            plan.close()

    best = measure(cur)
    if best is None:
        raise CFFTError(4, "the default execution choices do not run for this plan")
    for name, values in knobs:
        for v in values:
            if v == cur[name]:
                continue
            t = measure(dict(cur, **{name: v}))
            if t is not None and t < best:
                best, cur = t, dict(cur, **{name: v})
    cache[key] = {"tuning": cur, "ms": best}
    os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
    with open(cache_path, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    return dict(cur), best


# Decompositions the autotuner chooses between (cfft_path): the centring fold when the
# lattice is centred (plan_krfft_centered, src/centering_fold.jl:328), the plain stride-L
# transform (plan_krfft + plan_m2_backward, src/krfft.jl:301,1101), and the Q-matrix
# contour steps on either (plan_m2_q, plan_m7_scft, src/q_fused_krfft.jl:83,822).  All
# take the same subgrid fields and give the same spectra and steps.
PATHS = (0, 1, 3, 4)


def autotune_path(spec, ops_shifted, *, paths=PATHS, knobs=KNOBS, **kw):
    """The decomposition and execution choices that minimise the device time of `op`:
    every path in `paths` is timed with the default execution choices, then the
    fastest is tuned by autotune_plan (both cached).  Returns (path, tuning dict, ms);
    paths that do not apply to this plan (a Q-matrix step outside its sizes) are
    skipped."""
    best = None
    for p in paths:
        try:
            _, ms = autotune_plan(spec, ops_shifted, path=p, knobs=(), **kw)
        except CFFTError:
            continue
        if best is None or ms < best[1]:
            best = (p, ms)
    if best is None:
        raise CFFTError(4, "no decomposition runs for this plan")
    tu, ms = autotune_plan(spec, ops_shifted, path=best[0], knobs=knobs, **kw)
    return best[0], tu, ms


class MultiPlanStep:
    """Runs `jobs` (callables that issue their plans' calls on torch's current stream) on
    one stream each, forked from and joined to the caller's stream.  The first call runs
    them directly (so every plan has built its own state, e.g. its captured contour-loop
    graphs) and captures the whole set into one CUDA graph; later calls replay it."""

    def __init__(self, jobs):
        torch = _torch()
        self.jobs = list(jobs)
        self.streams = [torch.cuda.Stream() for _ in self.jobs]
        self.graph = None
        self.kernels_per_run = None  # library kernels one run launches (counted on the direct run)

    def _run(self):
        torch = _torch()
        main = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(main)
        for job, s in zip(self.jobs, self.streams):
            with torch.cuda.stream(s):
                job()
        for s in self.streams:
            main.wait_stream(s)

    def __call__(self):
        torch = _torch()
        from ._lib import LIB

        if self.graph is None:  # direct run (does the work), then capture without running
            before = LIB.cfft_launch_count(0)
            self._run()
            self.kernels_per_run = LIB.cfft_launch_count(0) - before
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._run()
            self.graph = g
            return
        self.graph.replay()
