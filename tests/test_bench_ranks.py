"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the step time is the
maximum over ranks, the whole-job value divides it by every rank's fields, and the
reference arm prints only on rank 0."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "tests", "ranks_worker.py")], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["ms"] == 5.0          # the slower rank's time, on both ranks
        assert o["e2e"] == 0.5
        assert abs(o["us_field"] - 0.5 * 1000.0 / 256) < 1e-12  # 5.0 ms / 10 steps over 2 x 128 fields


def test_whole_job_value_single_rank():
    spec_path = os.path.join(ROOT, "bench.py")
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_under_test", spec_path)
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.whole_job_us_per_field(0.16, 128, 1) == 0.16 * 1000.0 / 128


def test_reference_arm_is_silent_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=180, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_fullgrid_fft_baseline_sample():
    # the full-grid complex FFT baseline reported beside cpu_baseline: a positive median
    # over at least three timed fields, with its thread count
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_under_test_fft", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    r = bench.cpu_fullgrid_fft_sample(budget_s=0.1, workers=2)
    assert r["value"] > 0 and r["cores"] == 2 and r["unit"] == bench.UNIT
    assert r["sample"].startswith(("3 ", "4 ", "5 ")) or int(r["sample"].split()[0]) >= 3


def test_warmstart_data_parallel_host_logic_two_gloo_ranks():
    # the warm-start network's data-parallel step on CPU ranks: share-weighted gradients
    # of the ranks' shards sum to the full mini-batch gradient and mean loss (also when a
    # rank has no sample), and round-robin generated rows come back in order
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "tests", "dp_worker.py")], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        o = json.loads(out.strip().splitlines()[-1])
        assert o["grad_err"] < 1e-12 and o["loss_err"] < 1e-12
        assert o["grad1_err"] < 1e-12 and o["loss1_err"] < 1e-12
        assert o["rows"] == [[10.0 * i, i + 0.5] for i in range(5)]
        assert o["objs"] == [f"row{i}" for i in range(5)]


def test_algorithmic_flops_of_the_headline():
    # about 23 MFLOP per Im-3m 128^3 field: 4 channels of 32^3 both ways, 8 taps a point
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_under_test_flops", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    f = bench.algorithmic_flops_per_field(4, (32, 32, 32), 22880, 8)
    assert f == 2 * 4 * 5 * 32768 * 15 + 2 * 8 * 8 * 22880
    assert 22e6 < f < 23e6
