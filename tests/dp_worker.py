"""One gloo rank (CPU) of the data-parallel host logic of the warm-start training:
sharded mini-batches with share-weighted gradient all-reduce, and the round-robin
gather of generated rows.  Prints one JSON line."""
import json
import os
import sys

import numpy as np
import torch
import torch.distributed as dist

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from conftest import load_package  # noqa: E402


def main():
    dist.init_process_group("gloo", init_method="env://")
    rank, world = dist.get_rank(), dist.get_world_size()
    load_package()
    from crystallographicfft_b200 import sno, warmstart

    # least squares: loss(theta) = mean_i (x_i . theta - y_i)^2 over a global batch of 7
    rng = np.random.default_rng(0)
    X = torch.tensor(rng.standard_normal((7, 5)))
    y = torch.tensor(rng.standard_normal(7))
    theta = torch.tensor(rng.standard_normal(5))
    idx = list(range(7))
    mine = sno.shard_of(idx, rank, world)

    def mean_loss_grad(rows):
        r = X[rows] @ theta - y[rows]
        return float((r ** 2).mean()), (2.0 / len(rows)) * (X[rows].T @ r)

    buf = torch.zeros(6, dtype=torch.float64)
    loss = 0.0
    if mine:
        loss, g = mean_loss_grad(mine)
        buf[:5] = g
    total = sno.allreduce_mean_grads(buf, loss, len(mine), len(idx), dist)
    want_loss, want_g = mean_loss_grad(idx)

    # a rank with no samples still joins the all-reduce (batch of 1 over 2 ranks)
    buf1 = torch.zeros(6, dtype=torch.float64)
    one = sno.shard_of([3], rank, world)
    l1 = 0.0
    if one:
        l1, g1 = mean_loss_grad(one)
        buf1[:5] = g1
    total1 = sno.allreduce_mean_grads(buf1, l1, len(one), 1, dist)
    want1_loss, want1_g = mean_loss_grad([3])

    # round-robin rows (rank r computed rows r, r + world, ...) gathered in order
    n = 5
    rows = list(range(rank, n, world))
    local = torch.tensor([[10.0 * i, i + 0.5] for i in rows]).reshape(len(rows), 2)
    out, objs = warmstart.gather_rows(local, [f"row{i}" for i in rows], n, dist)
    print(json.dumps({
        "rank": rank,
        "grad_err": float((buf[:5] - want_g).abs().max()), "loss_err": abs(total - want_loss),
        "grad1_err": float((buf1[:5] - want1_g).abs().max()), "loss1_err": abs(total1 - want1_loss),
        "rows": out.tolist(), "objs": objs,
    }), flush=True)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
