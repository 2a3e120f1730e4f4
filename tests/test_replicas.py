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

import numpy as np
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
    # the value is an extrapolation and says so; the step time is what was measured
    assert d["cpu_baseline"]["sample"].startswith("EXTRAPOLATED")
    assert d["oracle_iterations"] > 0 and "full oracle solve" in d["oracle_iterations_source"]
    assert d["ms_per_step"] < 1e3 * d["value"]
    chk = d["extrapolation_check"]
    assert set(chk) == {"32^3", "64^3"}
    for v in chk.values():
        assert v["iterations"] > 0 and 0.3 < v["extrapolated_over_full"] < 3.0


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


def test_cpu_oracle_sample_is_bounded(built):
    """bench.cpu_oracle_sample: the oracle's plain PCG timed over bounded
    samples, each a short and a long call, whose difference gives the cost
    per iteration and the rest the fixed cost of a call (the CPU baseline
    extrapolates from these)."""
    import bench
    from programs_b200.mesh import Mesh, poisson_rhs
    A = Mesh.hex(10, jitter=0.15, seed=0, permute=True).pressure(pin=1)
    b = poisson_rhs(A.n_cell, 1)
    per, fixed, s = bench.cpu_oracle_sample(A, b, 0.3, repeats=3)
    assert len(per) == len(fixed) == 3 and 4 <= s <= 400
    assert all(p > 0 for p in per) and all(f >= 0 for f in fixed)


def test_oracle_iteration_counts_are_the_oracles_own(built):
    """The CPU baseline extrapolates with the oracle's own iteration count:
    recorded from a full 256^3 oracle solve, computed in full for small
    systems -- never the GPU solver's count."""
    import bench
    from oracle.oracle import Oracle
    full = bench.oracle_full_solve(256)
    assert full is not None and full["iterations"] > 1000
    A, b = bench.build_system(10)
    it, src = bench.oracle_iterations(A, b, 10)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 100000, np.zeros((A.n_cell, 1)),
                                        b.reshape(-1, 1))
    assert it == int(ref[3][0]) and src == "full oracle solve, this run"


def test_extrapolation_check_compares_full_solves(built):
    import bench
    chk = bench.extrapolation_check(sizes=(8, 12), sample=5)
    assert set(chk) == {"8^3", "12^3"}
    for v in chk.values():
        assert v["full_solve_s"] > 0 and v["extrapolated_s"] > 0 and v["iterations"] > 0
