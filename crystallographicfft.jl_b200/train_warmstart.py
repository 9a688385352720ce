"""Trains the learned SCFT warm start on the GPU and evaluates it (no reference counterpart).

    python crystallographicfft.jl_b200/train_warmstart.py --out WEIGHTS.npy --report REPORT.json

or, data parallel on G GPUs of one node (one process per GPU, NCCL):

    python -m torch.distributed.run --nnodes=1 --nproc-per-node G --master-addr 127.0.0.1 \
        crystallographicfft.jl_b200/train_warmstart.py --out WEIGHTS.npy --report REPORT.json

1. Training and held-out sets: AB diblock melts (b = 1, Ns = 100, cubic cell 3.8 b sqrt(N))
   with (chiN, f) drawn uniformly from [12, 30] x [0.30, 0.50], solved by the library's
   SCFT driver at 64^3 from the seeded plain start to a residual of 1e-4, for Ia-3d
   (No. 230), Im-3m (No. 229) and Pm-3m (No. 221).
2. One network for the three groups, Adam with cosine decay over mini-batches of one
   group, all forward and backward passes on the library's kernels.
3. Held-out evaluation: relative L2 error of the predicted fields; SCFT time to a
   residual of 1e-6 (FP32 to 1e-5, then FP64) from the prediction and from the plain
   start, and the difference of the final free energies.
4. The same comparison for Ia-3d at 96^3, f = 0.4, chiN = 20 (the network predicts on
   the 96^3 grid directly).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _load_package():
    name = "crystallographicfft_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--report", required=True)
    ap.add_argument("--grid", type=int, default=64)
    ap.add_argument("--train", default="230:1000,229:600,221:400", help="group:count of training draws")
    ap.add_argument("--test", default="230:100,229:60,221:40", help="group:count of held-out draws")
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--threads", type=int, default=8)
    ap.add_argument("--time-test", type=int, default=200, help="held-out draws timed (plain vs learned)")
    ap.add_argument("--train-seconds", type=float, default=900.0, help="training time limit")
    ap.add_argument("--max-iter", default="230:1000,229:1000,221:700", help="group:iteration cap of the data solves")
    ap.add_argument("--weights", default=None, help="evaluate these weights: no training set, no training")
    ap.add_argument("--ia3d96", default="20:0.4", help="chiN:f pairs of the Ia-3d 96^3 comparison")
    ap.add_argument("--plain", default="data", choices=["data", "timed"],
                    help="schedule of the timed plain start on held-out draws: that of the training data "
                         "(200 simple-mixing iterations) or the shorter one of the 96^3 gyroid (100)")
    a = ap.parse_args()

    import torch

    cf = _load_package()
    from crystallographicfft_b200 import warmstart as ws

    # Under torchrun (one process per GPU) the data solves are split over the GPUs and the
    # training is data parallel (one NCCL all-reduce of the gradients per step); rank 0
    # saves the weights and runs the evaluation.
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(minutes=20))
    gen = ws.generate if dist is None else (lambda gg, d, **kw: ws.generate_sharded(gg, d, dist, **kw))

    t_start = time.time()
    logs = []

    def log(msg):
        line = f"[{time.time() - t_start:7.1f}s] {msg}"
        logs.append(line)
        if rank == 0:
            print(line, flush=True)

    def parse(spec):
        return [(int(g), int(c)) for g, c in (x.split(":") for x in spec.split(","))]

    train_spec, test_spec = parse(a.train), parse(a.test)
    caps = dict(parse(a.max_iter))
    groups = sorted({g for g, _ in train_spec + test_spec}, key=lambda g: [x for x, _ in train_spec].index(g))
    grids = {g: ws.GroupGrid(g, a.grid) for g in groups}
    data = {}
    for k, (g, cnt) in enumerate(train_spec if a.weights is None else []):
        d = ws.draws(cnt, seed=1000 + k)
        fld, st, tm = gen(grids[g], d, threads=a.threads, log=log, max_iter=caps.get(g, 1000))
        ok = np.array([s["err"] < 1e-3 for s in st])
        data[g] = dict(params=d[ok], fields=fld[torch.as_tensor(np.nonzero(ok)[0], device="cuda")].contiguous(),
                       F=np.array([s["F"] for s in st])[ok], seconds=float(np.sum(tm)), dropped=int((~ok).sum()))
    tests = {}
    for k, (g, cnt) in enumerate(test_spec):
        d = ws.draws(cnt, seed=2000 + k)
        fld, st, tm = gen(grids[g], d, threads=a.threads, log=log, max_iter=caps.get(g, 1000))
        tests[g] = dict(params=d, fields=fld, states=st)
    gen_s = time.time() - t_start
    log(f"data generated in {gen_s:.1f} s")

    model = cf.SpectralNeuralOperator(lr=a.lr)
    plans, ctxs, sets = {}, {}, []
    for g in groups:
        gg = grids[g]
        plans[g] = cf.KRFFTPlan(gg.spec, gg.ops, N=gg.N, precision=4, max_batch=32 * a.batch)
        ctxs[g] = model.bind(plans[g], g, gg.shift, a.batch)
        if g in data:
            sets.append((ctxs[g], data[g]["params"], data[g]["fields"]))
    t0 = time.time()
    if a.weights is None:
        hist = ws.train(model, sets, a.epochs, batch=a.batch, lr=a.lr, log=log, max_seconds=a.train_seconds,
                        dist=dist)
        log(f"trained {a.epochs} epochs in {time.time() - t0:.1f} s on {world} GPU(s), final loss {hist[-1]:.3e}")
        if rank == 0:
            os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
            model.save(a.out)
    else:
        model.load(a.weights)
        hist = [float("nan")]
    train_s = time.time() - t0
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:  # the evaluation runs on rank 0 alone
            for o in list(ctxs.values()) + list(plans.values()) + [model]:
                o.close()
            return

    # held-out: field error of the prediction
    report = dict(grid=a.grid, weights=a.weights or a.out, train={str(g): dict(n=int(len(v["params"])), dropped=v["dropped"],
                                                   solve_seconds=v["seconds"]) for g, v in data.items()},
                  epochs=a.epochs, batch=a.batch, lr=a.lr, gpus=world, loss_history=[float(x) for x in hist[::5]] + [float(hist[-1])],
                  generate_seconds=gen_s, train_seconds=train_s, params=int(cf.sno.N_PARAMS))
    held = []
    for g, t in tests.items():
        for i in range(len(t["params"])):
            chiN, f = t["params"][i]
            pred = ctxs[g].predict([(chiN, f)])[0]
            truth = t["fields"][i]
            dev = (pred - truth).double()
            hom = torch.tensor([chiN * (1 - f), chiN * f], device="cuda", dtype=torch.float64).view(2, 1, 1, 1)
            rel = float(torch.linalg.vector_norm(dev) / torch.linalg.vector_norm(truth.double() - hom))
            held.append(dict(group=g, chiN=float(chiN), f=float(f), field_rel_err=rel, F_plain=t["states"][i]["F"]))
    log(f"held-out field error: median {np.median([h['field_rel_err'] for h in held]):.3e}")
    # held-out: time to 1e-6 from the prediction and from the plain start
    timed = 0
    order = np.random.default_rng(7).permutation(len(held))
    for j in order[:a.time_test]:
        h = held[j]
        gg, ctx = grids[h["group"]], ctxs[h["group"]]
        which = "plain"
        try:
            r_plain = ws.time_to_tol(gg, h["chiN"], h["f"],
                                     torch.tensor(gg.plain_start(h["f"], h["chiN"], plans[h["group"]].L),
                                                  dtype=torch.float32, device="cuda"), warm=False,
                                     plain=ws.PLAIN_DATA if a.plain == "data" else ws.PLAIN)
            which = "learned"
            r_warm = ws.time_to_tol(gg, h["chiN"], h["f"], None, warm=True,
                                    predict=lambda: ctx.predict([(h["chiN"], h["f"])])[0])
        except cf.CFFTError as e:
            h.update(error=str(e), failed_start=which)
            continue
        h.update(plain=r_plain, learned=r_warm, speedup=r_plain["seconds"] / r_warm["seconds"],
                 dF=abs(r_plain["F"] - r_warm["F"]))
        timed += 1
    tm = [h for h in held if "speedup" in h]
    if tm:
        sp = np.array([h["speedup"] for h in tm])
        dF = np.array([h["dF"] for h in tm])
        match = dF <= 1e-7
        report["held_out"] = dict(n=len(tm), failed=len([h for h in held if "error" in h]),
                                  speedup_median=float(np.median(sp)),
                                  speedup_median_matching=float(np.median(sp[match])) if match.any() else None,
                                  speedup_mean_matching=float(np.mean(sp[match])) if match.any() else None,
                                  matching_F=int(match.sum()), matching_F_1e6=int((dF <= 1e-6).sum()),
                                  plain_schedule=a.plain,
                                  failed_plain=len([h for h in held if h.get("failed_start") == "plain"]),
                                  failed_learned=len([h for h in held if h.get("failed_start") == "learned"]),
                                  plain_seconds_mean=float(np.mean([h["plain"]["seconds"] for h in tm])),
                                  learned_seconds_mean=float(np.mean([h["learned"]["seconds"] for h in tm])),
                                  field_rel_err_median=float(np.median([h["field_rel_err"] for h in held])))
        log(f"held-out timing: {report['held_out']}")
    report["held_out_draws"] = held

    # Ia-3d at 96^3 (the network predicts on a grid it was not trained on)
    g96 = ws.GroupGrid(230, 96)
    p96 = cf.KRFFTPlan(g96.spec, g96.ops, N=g96.N, precision=4, max_batch=32)
    c96 = model.bind(p96, 230, g96.shift, 1)
    rows96 = []
    for pair in a.ia3d96.split(","):
        chiN, f = (float(v) for v in pair.split(":"))
        r = {}
        try:
            for rep in range(3):
                r_plain = ws.time_to_tol(g96, chiN, f, torch.tensor(g96.plain_start(f, chiN, p96.L),
                                                                     dtype=torch.float32, device="cuda"), warm=False)
                r_warm = ws.time_to_tol(g96, chiN, f, None, warm=True,
                                        predict=lambda: c96.predict([(chiN, f)])[0])
                r.setdefault("plain", []).append(r_plain)
                r.setdefault("learned", []).append(r_warm)
        except cf.CFFTError as e:
            rows96.append(dict(chiN=chiN, f=f, error=str(e)))
            continue
        ps = min(x["seconds"] for x in r["plain"])
        ls = min(x["seconds"] for x in r["learned"])
        rows96.append(dict(chiN=chiN, f=f, plain=r["plain"][0], learned=r["learned"][0], plain_seconds=ps,
                           learned_seconds=ls, speedup=ps / ls, dF=abs(r["plain"][0]["F"] - r["learned"][0]["F"])))
        log(f"Ia-3d 96^3 chiN {chiN} f {f}: plain {ps:.3f} s, learned {ls:.3f} s, speedup {ps / ls:.2f}, "
            f"dF {rows96[-1]['dF']:.2e}, F {r['plain'][0]['F']:.6f}")
    report["ia3d96"] = rows96
    report["log"] = logs
    with open(a.report, "w") as fh:
        json.dump(report, fh, indent=1)
    for o in list(ctxs.values()) + [c96] + list(plans.values()) + [p96, model]:
        o.close()


if __name__ == "__main__":
    main()
