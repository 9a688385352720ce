"""One rank of the two-rank gloo test of bench.py's multi-rank host logic (launched by
tests/test_bench_ranks.py with RANK, WORLD_SIZE, MASTER_ADDR and MASTER_PORT set).
Prints one JSON line with what this rank computed."""
import importlib.util
import json
import os
import sys
from datetime import timedelta

import torch
import torch.distributed as dist

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def main():
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    cpu = torch.device("cpu")
    # each rank "measured" a different step time; every rank must see the slowest one
    ms = bench.max_over_ranks(2.0 + 3.0 * rank, cpu, dist, world)
    e2e = bench.max_over_ranks(0.5 - 0.25 * rank, cpu, dist, world)
    us = bench.whole_job_us_per_field(ms / 10, 128, world)
    dist.barrier()
    dist.destroy_process_group()
    print(json.dumps({"rank": rank, "ms": ms, "e2e": e2e, "us_field": us}), flush=True)


if __name__ == "__main__":
    sys.exit(main())
