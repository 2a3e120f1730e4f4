"""The multi-process path of bench.py on the CPU (gloo, world size 2).

The solver path does not shard: N GPUs run N independent replicas, each
solving its own system, and the job's time is the slowest rank's.  These
tests cover that host logic without a GPU: the max-over-ranks reduction
every rank takes part in, and the reference arm under torchrun, where rank 0
alone works and prints one JSON line while the other ranks exit 0.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_max(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first = bench.max_over_ranks(values[rank], dist, "cpu")
        second = bench.max_over_ranks(-values[rank], dist, "cpu")
        out.put((rank, first, second))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    values = [0.125, 3.5]
    port = _free_port()
    procs = [ctx.Process(target=_rank_max, args=(r, 2, port, values, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert got == [(0, 3.5, -0.125), (1, 3.5, -0.125)]


def test_max_over_ranks_without_a_process_group_is_the_value():
    import bench
    assert bench.max_over_ranks(2.25) == 2.25


def test_reference_arm_under_torchrun_prints_once_from_rank_zero(built):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--size", "64", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["unit"] == "s/solve" and d["higher_is_better"] is False
    assert d["e2e"] == {"value": d["value"], "unit": "s/solve", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] == 1
    assert d["cpu_baseline"]["host_threads"] >= 1 and "cpu_model" in d["cpu_baseline"]


@pytest.mark.parametrize("line,reasons", [
    ("0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active", []),
    ("0, 1500, 1965, 999.0, 0x4, Not Active, Not Active, Not Active, Active", ["sw_power_cap"]),
    ("0, 900, 1965, 400.0, 0x8, Active, Not Active, Not Active, Not Active", ["hw_slowdown"]),
])
def test_clock_sampler_reads_nvidia_smi_lines(line, reasons):
    import bench
    c = bench.ClockSampler(0)
    c.out = "\n".join([line, line, "garbage"])
    s = c.summary()
    assert s["samples"] == 2 and s["reasons"] == reasons
    assert s["sm_mhz"] == float(line.split(",")[1]) and s["sm_max_mhz"] == 1965.0


def test_cpu_baseline_is_a_median_of_bounded_samples(built):
    """bench.cpu_baseline: the oracle's plain PCG timed as the median of
    three bounded runs, scaled to the full solve's iteration count."""
    import bench
    from programs_b200.mesh import Mesh, poisson_rhs
    A = Mesh.hex(10, jitter=0.15, seed=0, permute=True).pressure(pin=1)
    b = poisson_rhs(A.n_cell, 1)
    v, s, total = bench.cpu_baseline(A, b, 1000, budget_s=0.3)
    assert v > 0 and 2 <= s <= 200 and total > 0
    assert v < 1000 * total          # per-iteration time times 1000, not more
