"""Benchmark: seconds per pressure solve to a 1e-10 relative residual on a
256^3 jittered, permuted hex mesh (16.7M cells, 50.1M interior faces),
plus the SpMV HBM roofline.

One step = one full Krylov solve (the spray-simulation solv_cg call with
reduc=1e-10) of the pressure-correction Poisson system: jitter +-15%,
cells randomly permuted (seed 0) and then renumbered by the framework
(reverse Cuthill-McKee), coefficients area/l_pn, all-Neumann boundaries,
cell 1 pinned, rhs uniform[-1,1] with its mean removed, phi0 = 0.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                  [--size 256] [--method pcg|pcg-mixed] [--imat 0]

The b200 arm times K solves with CUDA events on the solver's stream
(inputs resident in HBM; every input is larger than the 126 MB L2), then
the same solves through the host C-ABI (pinned host buffers, copies
included) for `e2e`.  The reference arm times the CPU oracle -- the
line-faithful C restatement of the Fortran solver -- on a bounded sample
of iterations of the same system and scales to a full solve.
Multi-GPU: the path does not shard (replicas only): each rank solves its
own system, timing is max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Full-solve iteration count of the default workload (256^3, Jacobi PCG,
# reduc 1e-10), recorded from the GPU solver; the oracle matches the GPU
# count to +-2 iterations (tests/test_gpu_parity.py).  Used only by the
# reference arm, which cannot afford to run the ~20-minute CPU solve.
FULL_ITERS = {(256, "pcg", 0): 2616, (64, "pcg", 0): 715}

PEAK_FALLBACK_GBS = 6650.0


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return PEAK_FALLBACK_GBS, "fallback"


def build_system(size: int, seed: int = 0):
    from programs_b200.mesh import Mesh, poisson_rhs
    m = Mesh.hex(size, jitter=0.15, seed=seed, permute=True)
    m.renumber(Mesh.RCM)
    A = m.pressure(pin=1)
    b = poisson_rhs(A.n_cell, seed + 1)
    del m
    return A, b


def spmv_bytes(A, k=1, fp=8):
    """Algorithmic bytes of one matrix product: F*(8+fp*k) + 3*fp*N
    (index pair + k coefficients per interior face; diag, x, y per cell)."""
    F = int((A.inb > 0).sum())
    return F * (8 + fp * k) + 3 * fp * A.n_cell


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _traffic_from_profile(size):
    """DRAM bytes per SpMV launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"spmv_fp64_pressure_{size}.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def cpu_baseline(A, b, imat, iters_full, budget_s=15.0):
    """Oracle (single core, the reference is serial) on a bounded sample."""
    from oracle.oracle import Oracle
    o = Oracle.from_matrix(A)
    rhs = b.reshape(-1, 1)
    t = time.perf_counter()
    o.solv_cg(imat, 1e-10, 2, np.zeros((A.n_cell, 1)), rhs)
    t2 = time.perf_counter() - t
    s = max(2, min(200, int(budget_s / max(t2 / 2, 1e-6))))
    t = time.perf_counter()
    o.solv_cg(imat, 1e-10, s, np.zeros((A.n_cell, 1)), rhs)
    dt = time.perf_counter() - t
    per_iter = dt / s
    return per_iter * iters_full, s, dt


def run_reference(args, rank):
    if rank != 0:
        return
    A, b = build_system(args.size, seed=0)
    key = (args.size, "pcg", args.imat)
    iters = FULL_ITERS.get(key)
    if iters is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"no recorded full-solve iteration count for {key}"}))
        return
    from oracle.oracle import Oracle
    o = Oracle.from_matrix(A)
    rhs = b.reshape(-1, 1)
    t = time.perf_counter()
    o.solv_cg(args.imat, 1e-10, 2, np.zeros((A.n_cell, 1)), rhs)
    per = (time.perf_counter() - t) / 2
    sample = max(2, min(100, int(20.0 / max(per, 1e-6))))
    for _ in range(args.warmup):
        o.solv_cg(args.imat, 1e-10, 1, np.zeros((A.n_cell, 1)), rhs)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        o.solv_cg(args.imat, 1e-10, sample, np.zeros((A.n_cell, 1)), rhs)
        times.append((time.perf_counter() - t) / sample * iters)
    v = statistics.mean(times)
    desc = (f"{sample} PCG iterations of the {args.size}^3 system per step, scaled by the "
            f"{iters}-iteration full solve")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s/solve",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(args, A),
        "cpu_baseline": {"value": v, "unit": "s/solve", "cores": 1, "kind": "port",
                         "sample": desc},
        "e2e": {"value": v, "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


METRIC = "s/solve to 1e-10 rel resid (learned+mixed vs plain FP64 PCG); SpMV HBM GB/s"


def _config(args, A):
    return {"workload": f"pressure Poisson {args.size}^3 jittered hex, PCG to 1e-10 L1-relative",
            "n_cell": A.n_cell, "n_face_interior": int((A.inb > 0).sum()),
            "method": args.method, "imat": args.imat, "ordering": "RCM",
            "l2": "inputs larger than L2 (no flush needed)", "parallelism": "replicas"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--method", default="pcg", choices=["pcg"])
    ap.add_argument("--imat", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    from programs_b200.solver import GpuSolver
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    t0 = time.perf_counter()
    A, b = build_system(args.size, seed=rank)
    setup_s = time.perf_counter() - t0
    N = A.n_cell
    s = GpuSolver(local)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    s.matrix_set(A)
    dev = torch.device("cuda", local)
    b_dev = torch.from_numpy(b).to(dev).reshape(N, 1)
    phi = torch.zeros(N, 1, dtype=torch.float64, device=dev)
    res0 = torch.empty(N, 1, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def solve():
        with torch.cuda.stream(stream):
            phi.zero_()
            res0.copy_(b_dev)
        return s.solv_cg_dev(args.imat, 1e-10, 100000, 1, phi.data_ptr(), res0.data_ptr())

    for _ in range(max(args.warmup, 1)):
        rn, st = solve()
    iters = st["iters"][0]
    launches = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            rn, st = solve()
            launches += st["kernel_launches"] + 2
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = ms_per_step / 1e3 / world  # seconds per solve, whole job

    # solution check: true residual of the last solve
    x = phi.double().cpu().numpy().reshape(-1)
    r_true = b - (A.to_scipy() @ x) if N <= 2_500_000 else None

    # e2e: host C-ABI call, pinned host buffers, copies inside the timed region
    phi_h = torch.zeros(N, 1, dtype=torch.float64).pin_memory().numpy()
    res_h = torch.zeros(N, 1, dtype=torch.float64).pin_memory().numpy()
    res_h_f = np.asfortranarray(res_h)
    e2e = []
    for k in range(args.steps + 1):
        phi_h[:] = 0.0
        res_h_f[:, 0] = b
        rn_h = np.zeros(1)
        torch.cuda.synchronize()
        t = time.perf_counter()
        s.solv_cg(args.imat, 1e-10, 100000, phi_h, res_h_f, rn_h)
        dt = time.perf_counter() - t
        if k > 0:
            e2e.append(dt)
    e2e_v = statistics.mean(e2e) / world

    # roofline of the dominant kernel (the matrix product), CUDA events on the
    # solver's stream around back-to-back launches
    x_dev = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, N)).to(dev)
    y_dev = torch.empty_like(x_dev)
    torch.cuda.synchronize()
    s.spmv_dev(x_dev.data_ptr(), y_dev.data_ptr(), repeat=3)
    spmv_ms = s.spmv_dev(x_dev.data_ptr(), y_dev.data_ptr(), repeat=20)
    alg = spmv_bytes(A, k=1, fp=8)
    peak, peak_kind = _peaks()
    achieved = alg / (spmv_ms * 1e-3) / 1e9
    traffic = _traffic_from_profile(args.size)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, sample, dt = cpu_baseline(A, b, args.imat, iters)
        cpu = {"value": v, "unit": "s/solve", "cores": 1, "kind": "port",
               "sample": f"{sample} oracle PCG iterations ({dt:.1f} s) of this system, "
                         f"scaled to the {iters}-iteration solve"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "s/solve", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": _config(args, A),
            "iterations": iters, "final_ratio": st["ratio"][0],
            "true_rel_resid_l1": (float(np.abs(r_true).sum() / np.abs(b).sum())
                                  if r_true is not None else None),
            "e2e": {"value": e2e_v, "unit": "s/solve", "h2d_bytes_per_step": 2 * N * 8,
                    "d2h_bytes_per_step": 2 * N * 8 + 8},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "SpMV (sliced-ELL face gather)",
                         "alg_bytes_per_launch": alg, "launch_ms": spmv_ms,
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "setup_s": setup_s,
        }
        print(json.dumps(line))
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
