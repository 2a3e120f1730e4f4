"""Benchmark: seconds per pressure solve to a 1e-10 relative residual on a
256^3 jittered, permuted hex mesh (16.8M cells, 50.1M interior faces):
the learned + mixed-precision solve against plain FP64 PCG, plus the
matrix-product HBM rooflines.

One step = one full solve of the pressure-correction Poisson system
(jitter +-15%, cells randomly permuted (seed 0) then renumbered by the
framework (reverse Cuthill-McKee), coefficients area/l_pn, all-Neumann
boundaries, cell 1 pinned, rhs uniform[-1,1] with its mean removed,
phi0 = 0) with the spray-simulation stopping rule |r|_1/|r0|_1 < 1e-10.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                  [--size 256] [--method learned|mg_jacobi|mixed|plain]

Methods (all through the library's C-ABI, same context, same system):
  learned   -- flexible CG, FP32 inner iteration with FP64 reliable
               updates, preconditioned by one V-cycle of the aggregation
               hierarchy whose finest-level smoother is the network's
               operator (solv_gpu_fcg); `value`
  mg_jacobi -- the same V-cycle with damped-Jacobi smoothing (no network)
  one_level -- the network's operator alone as the preconditioner
  mixed     -- Jacobi PCG, FP32 inner iteration with FP64 reliable updates
  plain     -- Jacobi PCG in FP64 (solv_gpu_cg, the reference algorithm)
Each is timed with CUDA events on the solver's stream (inputs resident in
HBM; every array is larger than the 126 MB L2, so no flush is needed); the
measured method is then timed end to end through the host C-ABI with
pinned host buffers (`e2e`).  The hierarchy is built once per mesh (host
aggregation) by the first solve, outside the timed region, like the
matrix structure itself: `first_call_s` reports that first solve.  The reference arm times the CPU oracle -- the
line-faithful C restatement of the Fortran solver -- on a bounded sample of
iterations of the same system, scaled to the full solve.
Multi-GPU: the path does not shard (replicas only): each rank solves its
own system; timing is the max over ranks.
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

# Full-solve iteration counts of plain FP64 Jacobi PCG (reduc 1e-10) on the
# default systems, recorded from the GPU solver (the oracle matches the GPU
# count to +-2 iterations, tests/test_gpu_parity.py).  Only the reference
# arm uses them: it cannot afford the ~20-minute single-core CPU solve.
FULL_ITERS = {256: 2625, 128: 1424, 64: 715}

PEAK_FALLBACK_GBS = 6650.0
METRIC = "s/solve to 1e-10 rel resid (learned+mixed vs plain FP64 PCG); SpMV HBM GB/s"


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def max_over_ranks(x, dist=None, device=None):
    """The largest of every rank's x: a job of replicas takes as long as its
    slowest rank.  Every rank must call it, in the same order."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def host_cpu():
    """The host the CPU baseline ran on: model name and hardware threads."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "host_threads": os.cpu_count()}


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


def spmv_bytes(A, fp=8, k=1):
    """Algorithmic bytes of one matrix product: F*(8+fp*k) + 3*fp*N
    (index pair + k coefficients per interior face; diag, x, y per cell)."""
    F = int((A.inb > 0).sum())
    return F * (8 + fp * k) + 3 * fp * A.n_cell


def apply_bytes(A):
    """Algorithmic bytes of one application of the learned preconditioner:
    per face an index pair and one FP32 weight, per cell q, r, z (FP32)."""
    F = int((A.inb > 0).sum())
    return F * 12 + 12 * A.n_cell


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = ""

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


def _traffic_from_profile(name):
    """DRAM bytes per launch from a committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def cpu_baseline(A, b, iters_full, budget_s=15.0, repeats=3):
    """Oracle plain PCG (single core: the reference is serial) on bounded
    samples: the median over `repeats` runs of s iterations each, scaled to
    the full solve.  Returns (s/solve, s, total seconds timed)."""
    from oracle.oracle import Oracle
    o = Oracle.from_matrix(A)
    rhs = b.reshape(-1, 1)
    t = time.perf_counter()
    o.solv_cg(0, 1e-10, 2, np.zeros((A.n_cell, 1)), rhs)
    per = (time.perf_counter() - t) / 2
    s = max(2, min(200, int(budget_s / repeats / max(per, 1e-6))))
    runs = []
    for _ in range(repeats):
        t = time.perf_counter()
        o.solv_cg(0, 1e-10, s, np.zeros((A.n_cell, 1)), rhs)
        runs.append(time.perf_counter() - t)
    return statistics.median(runs) / s * iters_full, s, sum(runs)


def _config(args, A):
    return {"workload": f"pressure Poisson {args.size}^3 jittered hex, solve to 1e-10 L1-relative",
            "n_cell": A.n_cell, "n_face_interior": int((A.inb > 0).sum()),
            "method": args.method, "baseline_method": "plain FP64 Jacobi PCG",
            "ordering": "RCM", "l2": "inputs larger than L2 (no flush needed)",
            "parallelism": "replicas"}


def run_reference(args, rank):
    if rank != 0:
        return
    A, b = build_system(args.size, seed=0)
    iters = FULL_ITERS.get(args.size)
    if iters is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"no recorded full-solve iteration count for size {args.size}"}))
        return
    from oracle.oracle import Oracle
    o = Oracle.from_matrix(A)
    rhs = b.reshape(-1, 1)
    t = time.perf_counter()
    o.solv_cg(0, 1e-10, 2, np.zeros((A.n_cell, 1)), rhs)
    per = (time.perf_counter() - t) / 2
    sample = max(2, min(100, int(20.0 / max(per, 1e-6))))
    for _ in range(args.warmup):
        o.solv_cg(0, 1e-10, 1, np.zeros((A.n_cell, 1)), rhs)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        o.solv_cg(0, 1e-10, sample, np.zeros((A.n_cell, 1)), rhs)
        times.append((time.perf_counter() - t) / sample * iters)
    v = statistics.mean(times)
    desc = (f"{sample} PCG iterations of the {args.size}^3 system per step (single core; the "
            f"reference is serial), scaled by the {iters}-iteration full solve")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s/solve",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(args, A),
        "cpu_baseline": {"value": v, "unit": "s/solve", "cores": 1, "kind": "port",
                         "sample": desc, **host_cpu()},
        "e2e": {"value": v, "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# The solve methods, as options of one library context.
METHODS = {
    "learned": {"solver": "fcg", "precision": 1, "mg_levels": 12, "smoother": 1},
    "mg_jacobi": {"solver": "fcg", "precision": 1, "mg_levels": 12, "smoother": 0},
    "one_level": {"solver": "fcg", "precision": 1, "mg_levels": 0, "smoother": 1},
    "mixed": {"solver": "cg", "precision": 1, "mg_levels": 12, "smoother": 1},
    "plain": {"solver": "cg", "precision": 0, "mg_levels": 12, "smoother": 1},
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--method", default="learned", choices=["learned", "mg_jacobi", "mixed", "plain"])
    ap.add_argument("--weights", default=None)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    args = ap.parse_args()

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    from programs_b200.learn import DEFAULT_WEIGHTS, load_params
    from programs_b200.solver import (GpuSolver, OPT_MG_LEVELS, OPT_MG_SMOOTHER, OPT_PRECISION)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    t0 = time.perf_counter()
    A, b = build_system(args.size, seed=rank)
    N = A.n_cell
    s = GpuSolver(local)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    s.matrix_set(A)
    setup_s = time.perf_counter() - t0
    s.gnn_set_params(load_params(args.weights or DEFAULT_WEIGHTS))
    dev = torch.device("cuda", local)
    b_dev = torch.from_numpy(b).to(dev).reshape(N, 1)
    phi = torch.zeros(N, 1, dtype=torch.float64, device=dev)
    res0 = torch.empty(N, 1, dtype=torch.float64, device=dev)

    def configure(method):
        m = METHODS[method]
        s.set_option(OPT_PRECISION, m["precision"])
        s.set_option(OPT_MG_LEVELS, m["mg_levels"])
        s.set_option(OPT_MG_SMOOTHER, m["smoother"])

    tune = None
    if not args.no_tune:
        configure("mixed" if args.method != "plain" else "plain")
        tune = s.autotune("cg", 0, 1)
    torch.cuda.synchronize()

    def solve(method, reduc=1e-10):
        configure(method)
        with torch.cuda.stream(stream):
            phi.zero_()
            res0.copy_(b_dev)
        if METHODS[method]["solver"] == "fcg":
            return s.solv_fcg_dev(reduc, 100000, phi.data_ptr(), res0.data_ptr())
        return s.solv_cg_dev(0, reduc, 100000, 1, phi.data_ptr(), res0.data_ptr())

    def first_call(method):
        torch.cuda.synchronize()
        t = time.perf_counter()
        solve(method)
        torch.cuda.synchronize()
        return time.perf_counter() - t

    def timed(method, steps, warmup, clocks=False):
        for _ in range(max(warmup, 1)):
            rn, st = solve(method)
        launches = 0
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local) if clocks else None
        if clk:
            clk.__enter__()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            rn, st = solve(method)
            launches += st["kernel_launches"] + 2
        e1.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        return ms / steps, st, launches, (clk.summary() if clk else None)

    def solution():
        return phi.double().cpu().numpy().reshape(-1).copy()

    first_s = first_call(args.method)  # builds the hierarchy (once per mesh) for multigrid
    ms_step, st, launches, clocks = timed(args.method, args.steps, args.warmup, clocks=True)
    x = solution()
    r_true = b - (A.to_scipy() @ x)
    true_rel = float(np.abs(r_true).sum() / np.abs(b).sum())
    extra = {}
    if args.method == "learned":
        for m, k in (("mg_jacobi", 3), ("one_level", 2)):
            ms_m, st_m, _, _ = timed(m, k, 1)
            extra[m] = {"s_per_solve": ms_m / 1e3, "iterations": st_m["iters"][0]}
    ms_plain, st_plain, _, _ = (timed("plain", 2, 1) if args.method != "plain"
                                else (ms_step, st, 0, None))
    x_plain = solution()
    ms_mixed, st_mixed, _, _ = (timed("mixed", 2, 1) if args.method != "mixed"
                                else (ms_step, st, 0, None))
    # solution agreement with plain FP64 PCG: both stopped at 1e-10 (each
    # carries an error of about cond(A) x 1e-10), and both run to 1e-12
    rel_vs_plain = float(np.linalg.norm(x - x_plain) / np.linalg.norm(x_plain))
    solve(args.method, 1e-12)
    x_t = solution()
    solve("plain", 1e-12)
    x_pt = solution()
    rel_tight = float(np.linalg.norm(x_t - x_pt) / np.linalg.norm(x_pt))

    # e2e: the measured method through the host C-ABI, pinned host buffers,
    # both copies inside the timed region
    phi_h = torch.zeros(N, 1, dtype=torch.float64).pin_memory().numpy()
    res_h = torch.zeros(N, 1, dtype=torch.float64).pin_memory().numpy()
    configure(args.method)
    e2e = []
    for k in range(args.steps + 1):
        phi_h[:] = 0.0
        res_h[:, 0] = b
        rn_h = np.zeros(1)
        torch.cuda.synchronize()
        t = time.perf_counter()
        if METHODS[args.method]["solver"] == "fcg":
            s.solv_fcg(1e-10, 100000, phi_h, res_h, rn_h)
        else:
            s.solv_cg(0, 1e-10, 100000, phi_h, res_h, rn_h)
        dt = time.perf_counter() - t
        if k > 0:
            e2e.append(dt)
    e2e_s = max_over_ranks(statistics.mean(e2e), dist, dev)

    # rooflines: kernels of the solve timed live on the solver's stream
    peak, peak_kind = _peaks()
    kt = {"spmv_fp64": s.kernel_time(0, 20), "spmv_fp32": s.kernel_time(1, 20)}
    alg = {"spmv_fp64": spmv_bytes(A, 8), "spmv_fp32": spmv_bytes(A, 4)}
    if args.method != "plain":
        kt["precond_apply"] = s.kernel_time(2, 20)
        alg["precond_apply"] = apply_bytes(A)
    gbs = {k: alg[k] / (kt[k] * 1e-3) / 1e9 for k in kt}
    vcycle_ms = None
    if METHODS[args.method]["solver"] == "fcg":
        configure(args.method)
        vcycle_ms = s.kernel_time(3, 10)
    dominant = "spmv_fp64" if args.method == "plain" else "spmv_fp32"
    traffic = _traffic_from_profile(f"{dominant}_pressure_{args.size}.txt")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, sample, dt = cpu_baseline(A, b, st_plain["iters"][0])
        cpu = {"value": v, "unit": "s/solve", "cores": 1, "kind": "port",
               "sample": f"median of 3 runs of {sample} oracle PCG iterations ({dt:.1f} s in "
                         f"all, single core) of this system, scaled to the "
                         f"{st_plain['iters'][0]}-iteration plain solve",
               **host_cpu()}

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms_step / 1e3 / world, "unit": "s/solve", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (outer) / f32 (inner) / bf16 (network)" if args.method != "plain"
                     else "f64",
            "data": "synthetic", "config": _config(args, A),
            "iterations": st["iters"][0], "reliable_updates": st["refinements"],
            "fallbacks": st["fallbacks"], "mg_levels": st["mg_levels"],
            "true_rel_resid_l1": true_rel,
            "rel_diff_vs_plain_fp64": rel_vs_plain,
            "rel_diff_vs_plain_fp64_both_at_1e-12": rel_tight,
            "plain_fp64_pcg": {"s_per_solve": ms_plain / 1e3, "iterations": st_plain["iters"][0]},
            "mixed_pcg": {"s_per_solve": ms_mixed / 1e3, "iterations": st_mixed["iters"][0]},
            "multigrid_jacobi_smoother": extra.get("mg_jacobi"),
            "learned_one_level": extra.get("one_level"),
            "speedup_vs_plain_fp64": ms_plain / ms_step,
            "first_call_s": first_s,
            "e2e": {"value": e2e_s / world, "unit": "s/solve",
                    "h2d_bytes_per_step": 2 * N * 8, "d2h_bytes_per_step": 2 * N * 8 + 8},
            "roofline": {"bound": "hbm", "achieved": gbs[dominant], "peak": peak, "unit": "GB/s",
                         "frac": gbs[dominant] / peak, "traffic": traffic,
                         "kernel": f"{dominant} (sliced-ELL face gather)",
                         "alg_bytes_per_launch": alg[dominant], "launch_ms": kt[dominant],
                         "peak_kind": peak_kind},
            "spmv_gbs": {k: round(v, 1) for k, v in gbs.items()},
            "spmv_frac_of_peak": {k: round(v / peak, 3) for k, v in gbs.items()},
            "vcycle_ms": vcycle_ms,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
            "autotune": tune,
            "setup_s": setup_s,
        }
        print(json.dumps(line))
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
