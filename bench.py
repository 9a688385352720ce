"""Benchmark: symmetry-reduced FFT (KRFFT) forward + backward, Im-3m (No. 229) 128^3
FP32 with the centring fold, batched fields resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]
                    [--workload im3m128|scft-ia3d96|sno-train|pmmm64|ia3d96-step|mixed]

One step = one forward + backward KRFFT over B fields (f0 -> spectral ASU -> f0).
The default workload is the headline line; after its timed region it also measures the
metric's second half, the SCFT time-to-tolerance of the Ia-3d 96^3 gyroid from the
learned warm start and from the plain start, attached as `scft_ia3d96`, and the
secondary workloads below, attached as `secondary` (--no-attach, alias --no-scft, skips
both); --workload selects a secondary single-GPU
measurement (the SCFT time-to-tolerance of an AB diblock in Ia-3d at 96^3 from the
learned warm start and from the plain start; one training step of the warm-start
network; Pmmm 64^3 FP64 forward + backward; the Ia-3d 96^3 FP32 diffusion contour step;
64 fields over four cubic groups and four grid edges, forward + backward and a 50-step
diffusion solve each).
Prints ONE JSON line on rank 0.  Under torchrun each rank runs its own batch
(fields are independent: replicas / weak scaling); the step time is the max over
ranks.  `--impl reference` times the FP64 CPU restatement of the reference's
centred path (fft_reconstruct_centered! + ifft_unrecon_centered!) on a bounded
sample on this host's cores.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "crystallographicfft.jl_b200")
SG, NEDGE = 229, 128
METRIC = "KRFFT fwd+bwd us per field (Im-3m 128^3 FP32, batched, centring fold)"
UNIT = "us/field"


def load_package():
    name = "crystallographicfft_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


# What a DRAM-traffic figure measured by ncu depends on: the device side of the transform
# path (kernels, launch scheduling, the table layouts they read) and the tables the plan
# layer hands it for the measured plan.  The first is keyed by these sources; the plan
# layer (planner.cpp) enters through the hash of the measured plan's tables instead, so
# a faster planner that builds the same tables keeps the figure.  The SCFT driver, the
# warm-start network, the space-group table and the C ABI wrappers do not change it.
TRANSFORM_SOURCES = ("cfft_internal.h", "device_common.cuh", "exec.cu", "exec.h", "fast_api.h", "fast_kernels.cuh",
                     "fast_other_f32.cu", "fast_other_f64.cu", "fast_planes_f32.cu", "fast_planes_f64.cu",
                     "tma_planes.cuh")


def kernel_source_sha():
    """Hash of the transform path's device-side sources."""
    import hashlib

    h = hashlib.sha256()
    csrc = os.path.join(PKG_DIR, "csrc")
    for name in TRANSFORM_SOURCES:
        h.update(name.encode())
        h.update(open(os.path.join(csrc, name), "rb").read())
    return h.hexdigest()[:16]


def plan_table_sha(plan):
    """Hash of the host tables a plan's kernels read: its geometry, spectral ASU,
    representative operations and backward orbit tables."""
    import hashlib

    h = hashlib.sha256()
    for v in (plan.L, plan.M, plan.H, (plan.n_spec, plan.n_channels, plan.info.n_rep, plan.info.P)):
        h.update(np.asarray(v, dtype=np.int64).tobytes())
    idx, mult = plan.spectral_asu()
    for a in (idx, mult, *plan.backward_tables()):
        h.update(np.ascontiguousarray(np.asarray(a, dtype=np.int64)).tobytes())
    for op in plan.rep_ops():
        h.update(np.asarray(op.R, dtype=np.int64).tobytes() + np.asarray(op.t, dtype=np.int64).tobytes())
    return h.hexdigest()[:16]


def algorithmic_bytes_per_field(M, n_spec, real_bytes=4):
    """Forward reads f0 and writes the ASU spectrum; backward does the reverse."""
    return 2 * (real_bytes * int(np.prod(M)) + 2 * real_bytes * n_spec)


def algorithmic_flops_per_field(n_ch, H, n_spec, d):
    """FLOPs of a forward + backward, reported beside the byte roofline (not the bound):
    n_ch complex FFTs of the H^3 channel grid each way at 5 n log2 n, and the d-tap
    complex multiply-add of the reconstruct and of its inverse gather (8 flops a tap) at
    each spectral point."""
    vol = int(np.prod(H))
    return 2 * n_ch * 5 * vol * float(np.log2(vol)) + 2 * d * 8 * n_spec


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.samples, self.proc, self.idx = [], None, gpu_index

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.samples)}
        rows = [r for r in self.samples if len(r) >= 9]
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        out["sm_mhz"] = float(np.median(sm)) if sm else None
        out["sm_max_mhz"] = max(mx) if mx else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, n in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(n)
        out["reasons"] = sorted(reasons)
        return out


# ----------------------------------------------------------------------------- inputs
def symmetric_fields(cf, torch, ops_s, N, L, B, seed, device, with_bases=False):
    """B seeded fields symmetric under ops_s (averaged over the group on the GPU),
    returned as the stride-L subgrid batch (B, M3, M2, M1) in x-fastest layout.
    Each field is a seeded combination of a few symmetric full-grid bases; with
    with_bases=True the bases (n_base, N3, N2, N1) and the coefficients (B, n_base)
    are returned as well, so the FP64 truth of every field is the same combination of
    the bases' FFTs."""
    g = torch.Generator(device=device).manual_seed(seed)
    n1, n2, n3 = N
    z, y, x = torch.meshgrid(torch.arange(n3, device=device), torch.arange(n2, device=device),
                             torch.arange(n1, device=device), indexing="ij")
    X = torch.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)])  # (3, n) in memory order
    Nv = torch.tensor(N, device=device).view(3, 1)
    maps = []
    for op in ops_s:
        R, t = op.Rm, op.tv
        Y = [torch.remainder(sum(int(R[i, j]) * X[j] for j in range(3)) + int(t[i]), int(N[i])) for i in range(3)]
        maps.append(Y[0] + n1 * (Y[1] + n2 * Y[2]))
    n_base = 4
    bases = []
    for _ in range(n_base):
        u = torch.randn(n1 * n2 * n3, generator=g, device=device, dtype=torch.float64)
        s = torch.zeros_like(u)
        for m in maps:
            s.index_add_(0, m, u)
        bases.append((s / len(maps)).view(n3, n2, n1))
    coef = torch.randn(B, n_base, generator=g, device=device, dtype=torch.float64)
    sub = torch.stack([b[::L[2], ::L[1], ::L[0]] for b in bases])  # (n_base, M3, M2, M1)
    out = torch.einsum("bk,kzyx->bzyx", coef, sub).contiguous()
    return (out, torch.stack(bases), coef) if with_bases else out


def forward_truth_error(F, bases, coef, spec_idx):
    """Max over fields of the forward spectrum's relative error against FP64 truth:
    field b's spectrum on the spectral ASU is sum_k coef[b, k] fftn(base_k)[h]."""
    u = bases.cpu().numpy()                                   # (n_base, N3, N2, N1)
    T = np.stack([np.fft.fftn(x)[spec_idx[:, 2], spec_idx[:, 1], spec_idx[:, 0]] for x in u])
    truth = coef.cpu().numpy() @ T                            # (B, n_spec)
    got = F.cpu().numpy().astype(np.complex128)
    err = np.max(np.abs(got - truth), axis=1) / np.max(np.abs(truth), axis=1)
    return float(err.max()), int(np.argmax(err))


# ----------------------------------------------------------------------------- reference arm
_REF = {}


def _oracle_plans():
    """The FP64 CPU restatement of the reference's centred path for Im-3m 128^3
    (plan_krfft_centered + plan_centered_ikrfft), built once per process from the
    oracle alone (its own operations, shift and tables): the library is not loaded."""
    if not _REF:
        sys.path.insert(0, ROOT)
        from oracle import krfft_oracle as O

        N = (NEDGE,) * 3
        _, oops = O.find_optimal_shift(O.get_ops(SG, 3, N), N)  # the oracle's own operation table
        spec = O.calc_spectral_asu(oops, 3, N)
        fwd = O.plan_krfft_centered(spec, oops)
        _REF.update(O=O, fwd=fwd, bwd=O.plan_centered_ikrfft(spec, oops, fwd),
                    f0=np.random.default_rng(0).standard_normal(fwd.krfft.M))
    return _REF


def _ref_fields(n):
    """fft_reconstruct_centered! + ifft_unrecon_centered! on n fields (one worker)."""
    O, fwd, bwd, f0 = _REF["O"], _REF["fwd"], _REF["bwd"], _REF["f0"]
    for _ in range(n):
        O.execute_centered_ikrfft(bwd, O.fft_reconstruct_centered(fwd, f0))
    return n


def _ref_worker_init():
    try:  # one thread per worker, like FFTW.set_num_threads(1) per field
        from threadpoolctl import threadpool_limits

        threadpool_limits(1)
    except ImportError:
        pass


def cpu_reference_sample(budget_s=12.0):
    """Single-thread sample of the CPU restatement (reported beside our own arm)."""
    R = _oracle_plans()
    _ref_fields(1)  # warm-up
    times, t_end = [], time.perf_counter() + budget_s
    while time.perf_counter() < t_end or len(times) < 3:
        t0 = time.perf_counter()
        _ref_fields(1)
        times.append(time.perf_counter() - t0)
        if len(times) >= 50:
            break
    us = float(np.median(times)) * 1e6
    return {"value": us, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{len(times)} single fields of Im-3m 128^3 FP64 (median), numpy/pocketfft single thread"}


def cpu_fullgrid_fft_sample(budget_s=4.0, workers=1):
    """The full-grid baseline the reference's benches time beside the KRFFT
    (test/bench_centered_scft.jl:53-81, test/bench_m7_forward_backward.jl:59-62): an
    in-place complex FP64 FFT of the whole N^3 grid, forward then inverse, here with
    scipy.fft (pocketfft) on `workers` threads.  Median us per field."""
    import scipy.fft as sf

    u = np.random.default_rng(1).standard_normal((NEDGE,) * 3).astype(np.complex128)
    x = u.copy()

    def one():
        y = sf.fftn(x, workers=workers, overwrite_x=True)
        return sf.ifftn(y, workers=workers, overwrite_x=True)

    one()
    times, t_end = [], time.perf_counter() + budget_s
    while time.perf_counter() < t_end or len(times) < 3:
        x[...] = u
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
        if len(times) >= 30:
            break
    return {"value": float(np.median(times)) * 1e6, "unit": UNIT, "cores": workers,
            "sample": f"{len(times)} complex FP64 {NEDGE}^3 fftn + ifftn (median), scipy.fft pocketfft, "
                      f"{workers} thread(s)"}


def cpu_reference_throughput(steps, warmup):
    """All host cores: one forked worker per core (no GPU in this process), each running
    whole fields; one step = one field per worker.  Returns us per field (wall time of
    the timed steps / fields done)."""
    import multiprocessing as mp

    _oracle_plans()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    with mp.get_context("fork").Pool(cores, initializer=_ref_worker_init) as pool:
        pool.map(_ref_fields, [warmup] * cores, chunksize=1)
        t0 = time.perf_counter()
        done = sum(pool.map(_ref_fields, [steps] * cores, chunksize=1))
        dt = time.perf_counter() - t0
    return {"value": dt * 1e6 / done, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} fields of Im-3m 128^3 FP64 ({steps} per worker after {warmup} warm-up), "
                      f"{cores} worker processes x numpy/pocketfft single thread"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_reference_throughput(args.steps, args.warmup)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["value"] * cb["cores"] / 1000.0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": {"workload": "Im-3m (No. 229) centred KRFFT forward+backward 128^3",
                                             "group": SG, "N": NEDGE, "sample": cb["sample"]},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- ranks
def max_over_ranks(value, device, dist=None, world=1):
    """The largest value over all ranks (one float64 all-reduce MAX); the value itself
    on a single rank.  Every rank must call it at the same point."""
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def whole_job_us_per_field(ms_step, fields_per_rank, world):
    """Whole-job time per field: the slowest rank's step time over all ranks' fields."""
    return ms_step * 1000.0 / (fields_per_rank * world)


# ----------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist

    cf = load_package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N = (NEDGE,) * 3
    ops = cf.get_ops(SG, 3, N)
    _, ops_s = cf.find_optimal_shift(ops, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    B = args.batch
    plan = cf.KRFFTPlan(spec, ops_s, precision=4, max_batch=B, path=cf.PATH_CENTERED)
    M = plan.M
    f0, bases, coef = symmetric_fields(cf, torch, ops_s, N, plan.L, B, seed=1234 + rank, device=dev, with_bases=True)
    f0 = f0.float().contiguous()
    F = torch.empty((B, plan.n_spec), dtype=torch.complex64, device=dev)
    out = torch.empty_like(f0)
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    lib = cf.LIB
    h = plan.handle

    def step():
        lib.cfft_forward(h, ctypes.c_void_p(f0.data_ptr()), ctypes.c_void_p(F.data_ptr()), B, sptr)
        lib.cfft_backward(h, ctypes.c_void_p(F.data_ptr()), ctypes.c_void_p(out.data_ptr()), B, sptr)

    # correctness guard on the real workload: every field's forward spectrum against
    # FP64 truth, and backward(forward(x)) == x
    step()
    torch.cuda.synchronize()
    rt_err = (torch.max(torch.abs(out - f0)) / torch.max(torch.abs(f0))).item()
    fwd_err, fwd_worst = forward_truth_error(F, bases, coef, plan.spectral_asu()[0])
    del bases
    if fwd_err > 1e-5 or rt_err > 1e-5:
        raise SystemExit(f"parity guard failed: forward max rel err {fwd_err:.3e} (field {fwd_worst}), "
                         f"round trip {rt_err:.3e}")
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    lib.cfft_launch_count(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = int(lib.cfft_launch_count(1))
    ms_total = e0.elapsed_time(e1)
    # per-stage device times (events between launches), averaged over a few round trips
    stage = np.zeros(6)
    ms_arr = (ctypes.c_float * 8)()
    nst = ctypes.c_int(0)
    reps = 5
    for _ in range(reps):
        lib.cfft_profile_roundtrip(h, ctypes.c_void_p(f0.data_ptr()), ctypes.c_void_p(F.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), B, sptr, ms_arr, ctypes.byref(nst))
        stage += np.array([ms_arr[i] for i in range(6)])
    stage /= reps
    clk = clocks.stop()
    # single-field latency: forward + backward of one field on its own plan, device time
    lat = None
    try:
        plan1 = cf.KRFFTPlan(spec, ops_s, precision=4, max_batch=1, path=cf.PATH_CENTERED)
        x1 = f0[:1].contiguous()
        F1 = torch.empty((1, plan1.n_spec), dtype=torch.complex64, device=dev)
        o1 = torch.empty_like(x1)
        h1 = plan1.handle

        def one():
            lib.cfft_forward(h1, ctypes.c_void_p(x1.data_ptr()), ctypes.c_void_p(F1.data_ptr()), 1, sptr)
            lib.cfft_backward(h1, ctypes.c_void_p(F1.data_ptr()), ctypes.c_void_p(o1.data_ptr()), 1, sptr)

        for _ in range(5):
            one()
        torch.cuda.synchronize()
        ts = []
        for _ in range(20):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        lat = {"value": float(np.median(ts)) * 1000.0, "unit": "us",
               "note": "forward + backward of one field (B = 1 plan), device time by CUDA events, median of 20"}
        plan1.close()
    except Exception as exc:  # reported, never required
        lat = {"error": repr(exc)}
    ms_max = max_over_ranks(ms_total, dev, dist if world > 1 else None, world)
    ms_step = ms_max / args.steps
    fields_total = B * world
    us_field = whole_job_us_per_field(ms_step, B, world)
    # e2e through the host-buffer C entry points with pinned host memory
    e2e = None
    if not args.no_e2e:
        f0_h = torch.empty(f0.shape, dtype=torch.float32, pin_memory=True)
        f0_h.copy_(f0.cpu())
        F_h = torch.empty((B, plan.n_spec), dtype=torch.complex64, pin_memory=True)
        out_h = torch.empty(f0.shape, dtype=torch.float32, pin_memory=True)  # empty_like would be pageable

        def e2e_step():
            lib.cfft_forward_host(h, ctypes.c_void_p(f0_h.data_ptr()), ctypes.c_void_p(F_h.data_ptr()), B)
            lib.cfft_backward_host(h, ctypes.c_void_p(F_h.data_ptr()), ctypes.c_void_p(out_h.data_ptr()), B)

        for _ in range(2):
            e2e_step()
        ke = max(3, args.steps // 2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            e2e_step()
        e2e_s = (time.perf_counter() - t0) / ke
        e2e_us = max_over_ranks(e2e_s, dev, dist if world > 1 else None, world) * 1e6 / fields_total
        fb = 4 * int(np.prod(M)) * B
        sb = 8 * plan.n_spec * B
        # Host-link bound of this step: each call is limited by its larger direction
        # (forward: f0 in; backward: f0 out), timed as plain pinned copies of f0.
        dbuf = torch.empty_like(f0)
        bw = {}
        for name, src, dst in (("h2d", f0_h, dbuf), ("d2h", dbuf, out_h)):
            dst.copy_(src, non_blocking=True)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            for _ in range(3):
                dst.copy_(src, non_blocking=True)
            torch.cuda.synchronize()
            bw[name] = 3 * fb / (time.perf_counter() - t1) / 1e9
        del dbuf
        bound_us = (fb / bw["h2d"] + fb / bw["d2h"]) / 1e3 / B
        e2e = {"value": e2e_us, "unit": UNIT, "h2d_bytes_per_step": fb + sb, "d2h_bytes_per_step": sb + fb,
               "pcie_gbs": {k: round(v, 2) for k, v in bw.items()}, "copy_bound": round(bound_us, 3),
               "note": "cfft_forward_host + cfft_backward_host, pinned host buffers, copies inside the timed region; "
                       "copy_bound = f0 bytes in and out at the measured pinned copy rates, per field"}
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    alg = algorithmic_bytes_per_field(M, plan.n_spec) * B
    achieved = alg / (ms_step * 1e-3) / 1e9
    names = ["plane_fwd (fold+xy FFT)", "z FFT fwd (+ spectral gather when fused)", "spectral gather (separate kernel)",
             "regroup + inverse gather", "expansion + inverse z FFT", "plane_bwd (xy IFFT+unfold)"]
    top = int(np.argmax(stage))
    # The largest stage as a kernel roofline.  The plane kernels move the path's f0 bytes
    # (4 M^3 per field, read by the forward fold, written by the backward unfold); the
    # workspace they write or read is an intermediate and does not count.
    kern = None
    if top in (0, 5) and stage[top] > 0:
        kb = 4.0 * float(np.prod(M)) * B
        ka = kb / (stage[top] * 1e-3) / 1e9
        kern = {"name": "k_plane_fwd_h" if top == 0 else "k_plane_bwd_h", "algorithmic_bytes": kb,
                "ms": float(stage[top]), "achieved": ka, "frac": ka / hbm,
                "note": "f0 bytes of the batch over the stage's CUDA-event time (chunks back to back on one stream)"}
    flops_field = algorithmic_flops_per_field(plan.n_channels, plan.H, plan.n_spec, plan.info.n_rep)
    line = {
        "metric": METRIC, "value": us_field, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"Im-3m (No. 229) centred KRFFT forward+backward, 128^3 FP32, {B} fields per GPU",
                   "group": SG, "N": NEDGE, "batch_per_gpu": B, "fields_total": fields_total,
                   "n_spec": plan.n_spec, "M": list(M), "channels": plan.n_channels,
                   "l2": "inputs larger than L2 (f0 batch %.0f MiB + output %.0f MiB)" % (4 * np.prod(M) * B / 2**20, 4 * np.prod(M) * B / 2**20),
                   "parallelism": f"replicas x{world}", "roundtrip_rel_err": rt_err,
                   "forward_rel_err_vs_fp64": fwd_err},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_src, "traffic": None,
                     "scope": "whole forward+backward per batch (6 launches per 64-field chunk); algorithmic bytes 2*(4*M^3 + 8*n_spec) per field",
                     "stage_ms": {n: float(v) for n, v in zip(names, stage)}, "dominant_stage": names[top],
                     "dominant_kernel": kern, "flops_per_field": flops_field,
                     "achieved_tflops": flops_field / (us_field * 1e-6) / 1e12},
        "latency_1field": lat,
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_reference_sample(budget_s=12.0)
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"error": repr(exc)}
        try:
            cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
            line["cpu_fullgrid_fft"] = {"single_thread": cpu_fullgrid_fft_sample(4.0, 1),
                                        "all_cores": cpu_fullgrid_fft_sample(4.0, cores)}
        except Exception as exc:
            line["cpu_fullgrid_fft"] = {"error": repr(exc)}
    # The metric's second half (SCFT time-to-tolerance, learned start vs plain start),
    # measured after the headline's timed region: two timed pairs of solves.
    if rank == 0 and world == 1 and not args.no_attach:
        try:
            line["scft_ia3d96"] = dict(metric=SCFT_WORKLOAD, unit="s", config=scft_config(),
                                       **scft_summary(scft_learned_vs_plain(2, 1)))
        except Exception as exc:  # reported, never required by the headline
            line["scft_ia3d96"] = {"error": repr(exc)}
    # DRAM traffic per step from the ncu capture of this very build (matched by the hash
    # of the native sources); null when the sources changed since the capture.
    traffic_file = os.path.join(ROOT, "profiles", "traffic_im3m128.json")
    line["roofline"]["kernel_source_sha"] = kernel_source_sha()
    line["roofline"]["plan_table_sha"] = plan_table_sha(plan)
    if os.path.exists(traffic_file):
        try:
            tr = json.load(open(traffic_file))
            if (tr.get("kernel_source_sha") == line["roofline"]["kernel_source_sha"]
                    and tr.get("plan_table_sha") == line["roofline"]["plan_table_sha"]):
                line["roofline"]["traffic"] = tr.get("bytes_per_field", 0) * B
                line["roofline"]["traffic_note"] = tr.get("note")
            else:
                line["roofline"]["traffic_note"] = "no ncu capture of this build's sources"
        except (OSError, ValueError):
            pass
    plan.close()
    if rank == 0 and world == 1 and not args.no_attach:
        line["secondary"] = secondary_lines(args)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


SECONDARY = ("pmmm64", "ia3d96-step", "mixed")


def secondary_lines(args):
    """The secondary workloads, each measured as `--workload NAME` measures it (its own
    CUDA events, with this run's steps and warm-up), summarised for the headline line.
    The mixed batch's autotuner starts from an empty cache unless --tune-cache names one."""
    import tempfile

    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        cache = args.tune_cache or os.path.join(tmp, "tuning.json")
        for name in SECONDARY:
            try:
                t0 = time.perf_counter()
                ln = measure_workload(name, args.steps, args.warmup, cache)
                out[name] = {"metric": ln["metric"], "value": ln["value"], "unit": ln["unit"],
                             "ms_per_step": ln["ms_per_step"], "dtype": ln["dtype"], "fields": ln["config"]["fields"],
                             "roofline_frac": ln["roofline"]["frac"], "gpu_launches": ln["gpu_launches"],
                             "sm_mhz": ln["clocks"].get("sm_mhz"), "clock_reasons": ln["clocks"].get("reasons"),
                             "wall_s": round(time.perf_counter() - t0, 1)}
            except Exception as exc:  # reported, never required by the headline
                out[name] = {"error": repr(exc)}
    return out


# ----------------------------------------------------------------------------- other workloads
WORKLOADS = {
    "pmmm64": dict(sg=47, n=64, precision=8, batch=512, op="fwdbwd",
                   desc="Pmmm (No. 47) KRFFT forward+backward, 64^3 FP64"),
    "ia3d96-step": dict(sg=230, n=96, precision=4, batch=512, op="step",
                        desc="Ia-3d (No. 230) diffusion contour step exp(-w ds/2) IFFT(K FFT(exp(-w ds/2) q)), 96^3 FP32"),
    "mixed": dict(op="mixed", precision=4, batch=64,
                  desc="64 fields drawn from Pm-3m, Im-3m, Fd-3m (origin 2), Ia-3d with edges {32,48,64,96}^3, "
                       "FP32: forward+backward and a 50-step diffusion solve each (one autotuned plan and one "
                       "stream per group and edge, the whole step replayed as one CUDA graph)"),
}


SCFT_CONFIG = dict(sg=230, n=96, f=0.4, chiN=20.0, Ns=100, history=20, tol=1e-6, switch=1e-5, sigma=2.0,
                   amplitude=1.0)
SNO_WEIGHTS = os.path.join(ROOT, "crystallographicfft.jl_b200", "data", "sno_warmstart.npy")


def scft_learned_vs_plain(steps, warmup):
    """Both solves of the SCFT time-to-tolerance comparison (see run_scft), `steps` times
    each after `warmup` untimed pairs.  Returns the seconds of every timed solve and the
    last pair's states."""
    import torch

    cf = load_package()
    from crystallographicfft_b200 import warmstart as ws

    C = SCFT_CONFIG
    gg = ws.GroupGrid(C["sg"], C["n"], Ns=C["Ns"])
    plan = cf.KRFFTPlan(gg.spec, gg.ops, N=gg.N, precision=4, max_batch=32)
    model = cf.SpectralNeuralOperator()
    model.load(SNO_WEIGHTS)
    ctx = model.bind(plan, C["sg"], gg.shift, 1)
    plain0 = torch.tensor(gg.plain_start(C["f"], C["chiN"], plan.L), dtype=torch.float32, device="cuda")

    def predict():
        return ctx.predict([(C["chiN"], C["f"])])[0]

    def once():
        a = ws.time_to_tol(gg, C["chiN"], C["f"], plain0, warm=False, tol=C["tol"], switch=C["switch"])
        b = ws.time_to_tol(gg, C["chiN"], C["f"], None, warm=True, tol=C["tol"], switch=C["switch"], predict=predict)
        return a, b

    for _ in range(warmup):
        once()
    runs = [once() for _ in range(steps)]
    for o in (ctx, model, plan):
        o.close()
    return runs


def scft_summary(runs):
    plain_s = [a["seconds"] for a, _ in runs]
    learned_s = [b["seconds"] for _, b in runs]
    a, b = runs[-1]
    mean_l, mean_p = float(np.mean(learned_s)), float(np.mean(plain_s))
    return {"plain_seconds": mean_p, "learned_seconds": mean_l, "speedup": mean_p / mean_l,
            "F_plain": a["F"], "F_learned": b["F"], "dF": abs(a["F"] - b["F"]),
            "residual_plain": a["err"], "residual_learned": b["err"],
            "converged": bool(a["converged"] and b["converged"]),
            "iterations_plain": [a["iterations_fp32"], a["iterations_fp64"]],
            "iterations_learned": [b["iterations_fp32"], b["iterations_fp64"]],
            "disordered_F": SCFT_CONFIG["chiN"] * SCFT_CONFIG["f"] * (1 - SCFT_CONFIG["f"]),
            "plain_s": [round(t, 4) for t in plain_s], "learned_s": [round(t, 4) for t in learned_s]}


SCFT_WORKLOAD = ("SCFT time-to-tol, s per solve, learned warm start vs plain (AB diblock, Ia-3d 96^3, f=0.4, chiN=20, "
                 "Ns=100, Anderson 20, residual 1e-6)")


def scft_config():
    from crystallographicfft_b200 import warmstart as ws

    C = SCFT_CONFIG
    return {"workload": "scft-ia3d96", "group": C["sg"], "N": C["n"], "f": C["f"], "chiN": C["chiN"],
            "Ns": C["Ns"], "anderson_history": C["history"], "tol": C["tol"],
            "cell": "3.8 b sqrt(N) = %.4f Rg" % ws.CELL,
            "plain_start": "seeded Gaussian-filtered noise, sigma 2 grid points, amplitude 1.0, symmetrised; "
                           "%d simple-mixing iterations, then Anderson" % ws.PLAIN["min_simple"],
            "learned_start": "spectral neural operator prediction (weights %s), Anderson from the start"
                             % os.path.relpath(SNO_WEIGHTS, ROOT),
            "phases": "FP32 to residual %.0e, then FP64 to %.0e" % (C["switch"], C["tol"])}


def run_scft(args):
    """SCFT time-to-tolerance, AB diblock in Ia-3d (No. 230) on 96^3: f = 0.4, chiN = 20,
    Ns = 100, Anderson history 20, residual 1e-6, cell 3.8 b sqrt(N), learned warm start
    against the plain start.  One step = one solve from each start: FP32 fields and
    propagators to a residual of 1e-5, then the same fields in FP64 to 1e-6 (FP32 rounding
    leaves a residual floor near 2e-6 at 96^3); Q, F and the mixing solve are FP64 on the
    device throughout.
    - plain: the seeded start (Gaussian-filtered noise, sigma 2 grid points, amplitude
      1.0, symmetrised), simple mixing for 100 iterations (the gyroid grows out of the
      unstable modes; Anderson mixing from this near-uniform start converges to the
      disordered state), then Anderson mixing;
    - learned: the spectral neural operator's prediction on the 96^3 grid (trained at
      64^3 on the driver's own converged fields; its inference is inside the timed
      region), Anderson mixing from the first iteration."""
    import torch

    cf = load_package()
    torch.cuda.set_device(0)
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    cf.LIB.cfft_launch_count(1)
    runs = scft_learned_vs_plain(args.steps, args.warmup)
    launches = int(cf.LIB.cfft_launch_count(1))
    clk = clocks.stop()
    res = scft_summary(runs)
    line = {"metric": SCFT_WORKLOAD, "value": res["learned_seconds"], "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (res["learned_seconds"] + res["plain_seconds"]) * 1000.0,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (network bf16 weights, f32 accumulate)", "data": "synthetic", "config": scft_config(),
            "result": res, "gpu_launches": launches, "clocks": clk, "e2e": None, "roofline": None}
    print(json.dumps(line), flush=True)


def run_sno_train(args):
    """Training step of the warm-start network (secondary line): Ia-3d 64^3, 16 samples
    per step (the training configuration), targets = seeded plain-start fields.  One step =
    forward (4 Fourier layers: 8 batched KRFFTs of 512 fields, tensor-core channel
    products) + loss + backward + Adam update; device time by CUDA events."""
    import torch

    cf = load_package()
    from crystallographicfft_b200 import warmstart as ws

    torch.cuda.set_device(0)
    S = 16
    gg = ws.GroupGrid(230, 64)
    plan = cf.KRFFTPlan(gg.spec, gg.ops, N=gg.N, precision=4, max_batch=32 * S)
    model = cf.SpectralNeuralOperator()
    ctx = model.bind(plan, 230, gg.shift, S)
    prm = ws.draws(S, seed=5)
    tgt = torch.tensor(np.stack([gg.plain_start(f, c, plan.L) for c, f in prm]), dtype=torch.float32,
                       device="cuda").contiguous()
    for _ in range(args.warmup):
        ctx.train_step(prm, tgt, lr=1e-4)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    cf.LIB.cfft_launch_count(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        ctx.train_step(prm, tgt, lr=1e-4)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = int(cf.LIB.cfft_launch_count(1))
    clk = clocks.stop()
    line = {"metric": "warm-start network training step, ms (Ia-3d 64^3, 16 samples, forward + backward + Adam)",
            "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 weights / tensor-core operands, f32 accumulate and fields", "data": "synthetic",
            "config": {"workload": "sno-train", "group": 230, "N": 64, "samples": S, "width": 32, "modes": 12,
                       "layers": 4, "params": int(cf.sno.N_PARAMS)},
            "samples_per_s": S / (ms / 1000.0), "gpu_launches": launches, "clocks": clk, "e2e": None, "roofline": None}
    for o in (ctx, model, plan):
        o.close()
    print(json.dumps(line), flush=True)


def _field_bytes(plan, rs):
    return 2 * (rs * int(np.prod(plan.M)) + 2 * rs * plan.n_spec)


def run_workload(args):
    """Secondary measurements (one GPU): the same device-event timing as the main arm."""
    print(json.dumps(measure_workload(args.workload, args.steps, args.warmup, args.tune_cache)), flush=True)


def measure_workload(name, steps, warmup, tune_cache=None):
    """One secondary workload (WORKLOADS[name]) timed by CUDA events over `steps` steps
    after `warmup` untimed ones; returns its JSON line."""
    import torch

    cf = load_package()
    W = WORKLOADS[name]
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    rs = W["precision"]
    rdt = torch.float32 if rs == 4 else torch.float64
    jobs = []  # (plan, q, w or None, F or None, fields, algorithmic bytes per step)
    if W["op"] == "mixed":
        rng = np.random.default_rng(64)
        groups = rng.choice([221, 229, 227, 230], size=W["batch"])
        edges = rng.choice([32, 48, 64, 96], size=W["batch"])
        for sg in sorted(set(groups.tolist())):
            for n in sorted(set(edges.tolist())):
                count = int(np.sum((groups == sg) & (edges == n)))
                if count:
                    jobs.append((int(sg), int(n), count))
        built = []
        tunings = []
        for sg, n, count in jobs:
            N = (n,) * 3
            _, ops_s = cf.find_optimal_shift(cf.get_ops(sg, 3, N), N)
            spec = cf.calc_spectral_asu(ops_s, 3, N)
            # execution choices per (group, edge, batch) from the autotuner (cached); choosing the
            # decomposition per plan as well (autotune_path) timed each plan alone and made the
            # overlapped one-graph step slower (49.2 against 46.0 us per field), so it is not used
            tu, tms = cf.autotune_plan(spec, ops_s, N=N, precision=rs, batch=count, op="mixed", n_steps=50,
                                       ds=0.01, cache_path=tune_cache)
            tunings.append({"group": sg, "N": n, "fields": count, "tuning": tu, "tuned_ms": round(tms, 4)})
            plan = cf.KRFFTPlan(spec, ops_s, precision=rs, max_batch=count, ds=0.01, tuning=tu)
            q = symmetric_fields(cf, torch, ops_s, N, plan.L, count, seed=sg * 1000 + n, device=dev).to(rdt).contiguous()
            w = 0.1 * symmetric_fields(cf, torch, ops_s, N, plan.L, count, seed=sg + n, device=dev).to(rdt).contiguous()
            F = torch.empty((count, plan.n_spec), dtype=torch.complex64 if rs == 4 else torch.complex128, device=dev)
            built.append((plan, q, w, F, count, (_field_bytes(plan, rs) * 51 + 3 * rs * int(np.prod(plan.M)) * 50) * count))
        jobs = built
    else:
        N = (W["n"],) * 3
        _, ops_s = cf.find_optimal_shift(cf.get_ops(W["sg"], 3, N), N)
        spec = cf.calc_spectral_asu(ops_s, 3, N)
        B = W["batch"]
        plan = cf.KRFFTPlan(spec, ops_s, precision=rs, max_batch=B, ds=0.01)
        q = symmetric_fields(cf, torch, ops_s, N, plan.L, B, seed=7, device=dev).to(rdt).contiguous()
        w = 0.1 * symmetric_fields(cf, torch, ops_s, N, plan.L, B, seed=8, device=dev).to(rdt).contiguous() \
            if W["op"] == "step" else None
        F = torch.empty((B, plan.n_spec), dtype=torch.complex64 if rs == 4 else torch.complex128, device=dev)
        per = _field_bytes(plan, rs) + (3 * rs * int(np.prod(plan.M)) if W["op"] == "step" else 0)
        jobs = [(plan, q, w, F, B, per * B)]
    fields = sum(j[4] for j in jobs)
    qs = [j[1].clone() for j in jobs]
    main = torch.cuda.current_stream()

    def job(plan, q, w, F, qc):
        def run():
            if W["op"] == "step":
                plan.step_diffusion(qc, w, 0.01, 1)
            else:
                plan.forward(q, out=F)
                plan.backward(F, out=qc)
                if W["op"] == "mixed":
                    plan.step_diffusion(qc, w, 0.01, 50)
        return run

    runs = [job(plan, q, w, F, qc) for (plan, q, w, F, count, _), qc in zip(jobs, qs)]
    if W["op"] == "mixed":
        # every plan's work (its own stream each) replayed as one CUDA graph per step
        step = cf.MultiPlanStep(runs)
    else:
        def step():
            for r in runs:
                r()

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    cf.LIB.cfft_launch_count(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    launches = int(cf.LIB.cfft_launch_count(1))
    if W["op"] == "mixed":
        launches = int(step.kernels_per_run) * steps  # replayed graph: the kernels it holds
    ms_step = e0.elapsed_time(e1) / steps
    clk = clocks.stop()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    alg = sum(j[5] for j in jobs)
    achieved = alg / (ms_step * 1e-3) / 1e9
    line = {"metric": f"{W['desc']}: us per field", "value": ms_step * 1000.0 / fields, "unit": UNIT, "n_gpus": 1,
            "steps": steps, "warmup": warmup, "ms_per_step": ms_step, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if rs == 4 else "f64", "data": "synthetic",
            "config": {"workload": name, "description": W["desc"], "fields": fields,
                       "plans": [{"N": list(j[0].N), "centering": j[0].centering, "centered": j[0].centered,
                                  "fields": j[4]} for j in jobs]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": "measured" if "hbm_gbs" in peaks else "fallback", "traffic": None},
            "gpu_launches": launches, "clocks": clk, "e2e": None}
    if W["op"] == "mixed":
        line["config"]["tuning"] = tunings
        line["config"]["launch"] = "one CUDA graph per step (MultiPlanStep) over one stream per plan"
        step.graph = None  # the graph goes before the plans whose buffers it replays
    torch.cuda.synchronize()
    for j in jobs:
        j[0].close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end timing (profiling runs)")
    ap.add_argument("--no-attach", "--no-scft", dest="no_attach", action="store_true",
                    help="skip what the headline line carries after its timed region: the SCFT learned-vs-plain "
                         "comparison and the secondary workload lines (profiling runs)")
    ap.add_argument("--tune-cache", default=None, help="autotuner cache file (default ~/.cache/cfft_b200/tuning.json)")
    ap.add_argument("--workload", default="im3m128", choices=["im3m128", "scft-ia3d96", "sno-train"] + sorted(WORKLOADS),
                    help="im3m128 is the headline line; the others are secondary single-GPU measurements")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "scft-ia3d96":
        run_scft(args)
    elif args.workload == "sno-train":
        run_sno_train(args)
    elif args.workload != "im3m128":
        run_workload(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
