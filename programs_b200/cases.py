"""Run one solver case on cuda:0 and print a JSON line.

  python -m programs_b200.cases solve  --size 128 --system pressure --solver cg --imat 0
  python -m programs_b200.cases spmv   --size 128 --repeat 20
  python -m programs_b200.cases batch  --n-sys 64 --min 8000 --max 500000
  python -m programs_b200.cases kernel --size 160 --which 1 --repeat 5

The systems are the seeded synthetic ones of the benchmarks: jittered
(+-15%), randomly permuted hex meshes renumbered by the framework, the
pressure-correction Poisson matrix (pinned cell 1, zero-mean rhs) or the
upwind momentum matrix (Taylor-Green flux, Pe <= 50, CFL 5).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .mesh import Mesh, poisson_rhs, uniform
from .solver import (GpuSolver, OPT_GRAPH_ITERS, OPT_MG_ALPHA, OPT_MG_LEVELS, OPT_MG_OMEGA,
                     OPT_MG_SMOOTHER, OPT_PERSISTENT, OPT_PRECISION, OPT_RELIABLE_DELTA,
                     OPT_GRAPH_LOOP, OPT_FCG_RELIABLE_DELTA, OPT_FCG_SLOW_ITERS)


def make_system(size, system="pressure", seed=0, renumber="rcm"):
    m = Mesh.hex(size, jitter=0.15, seed=seed, permute=True)
    if renumber == "rcm":
        m.renumber(Mesh.RCM)
    elif renumber == "sfc":
        m.renumber(Mesh.SFC)
    elif renumber == "color":
        m.renumber(Mesh.COLOR)
    if system == "pressure":
        A = m.pressure(pin=1)
        b = poisson_rhs(A.n_cell, seed + 1)
    else:
        A, _ = m.momentum()
        b = uniform(seed + 1, A.n_cell)
    return A, b


def batch_sizes(n_sys, lo, hi, seed=1):
    """Edge lengths of the n_sys hex meshes with log-uniform cell counts in
    [lo, hi] (seeded)."""
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(np.log(lo), np.log(hi), n_sys))
    return [max(2, int(round(nc ** (1.0 / 3.0)))) for nc in cells]


def batch_meshes(n_sys, lo, hi, seed=1, pick=None):
    """n_sys pressure systems with log-uniform cell counts in [lo, hi]; with
    `pick`, only the systems of those indices (the same systems the full
    batch holds at those places)."""
    mats, rhs = [], []
    for k, n in enumerate(batch_sizes(n_sys, lo, hi, seed)):
        if pick is not None and k not in pick:
            continue
        m = Mesh.hex(n, jitter=0.15, seed=1000 + k, permute=True)
        m.renumber(Mesh.RCM)
        A = m.pressure(pin=1)
        mats.append(A)
        rhs.append(poisson_rhs(A.n_cell, 2000 + k))
    return mats, rhs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["solve", "spmv", "batch", "kernel"])
    ap.add_argument("--which", type=int, default=1,
                    help="kernel: 0 FP64 SpMV, 1 FP32 SpMV, 2 network operator, 3 V-cycle")
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--system", default="pressure", choices=["pressure", "momentum"])
    ap.add_argument("--solver", default="cg", choices=["cg", "bicg", "fcg"])
    ap.add_argument("--weights", default=None, help="learned-preconditioner weights (.npz)")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--imat", type=int, default=0)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--n-vc", type=int, default=1)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--graph-iters", type=int, default=16)
    ap.add_argument("--renumber", default="rcm", choices=["rcm", "sfc", "color", "none"])
    ap.add_argument("--n-sys", type=int, default=64)
    ap.add_argument("--min", type=int, default=8000)
    ap.add_argument("--max", type=int, default=500000)
    ap.add_argument("--mg-levels", type=int, default=12, help="fcg: coarse levels (0 = one-level)")
    ap.add_argument("--smoother", type=int, default=1, help="fcg: 1 network, 0 Jacobi")
    ap.add_argument("--omega", type=float, default=0.8)
    ap.add_argument("--alpha", type=float, default=2.0)
    ap.add_argument("--reliable-delta", type=float, default=0.1,
                    help="mixed precision: FP32 residual drop between reliable updates")
    ap.add_argument("--fcg-delta", type=float, default=None,
                    help="fcg: FP32 residual drop at which a lane stops for a reliable update")
    ap.add_argument("--fcg-slow", type=int, default=None,
                    help="fcg: iterations per reliable-update drop before the network smoother "
                         "gives way to Jacobi (0 never)")
    ap.add_argument("--graph-loop", type=int, default=2,
                    help="1: iterations in a conditional WHILE graph; 0: graph_iters per launch; "
                         "2: WHILE for fcg only")
    ap.add_argument("--persistent", type=int, default=0,
                    help="cg, imat 0, FP64: 1 runs the cluster-persistent fused PCG")
    a = ap.parse_args(argv)

    import torch
    s = GpuSolver(0)
    s.set_option(OPT_GRAPH_ITERS, a.graph_iters)
    s.set_option(OPT_PRECISION, a.precision)
    s.set_option(OPT_MG_LEVELS, a.mg_levels)
    s.set_option(OPT_MG_SMOOTHER, a.smoother)
    s.set_option(OPT_MG_OMEGA, a.omega)
    s.set_option(OPT_MG_ALPHA, a.alpha)
    s.set_option(OPT_PERSISTENT, a.persistent)
    s.set_option(OPT_RELIABLE_DELTA, a.reliable_delta)
    s.set_option(OPT_GRAPH_LOOP, a.graph_loop)
    if a.fcg_delta is not None:
        s.set_option(OPT_FCG_RELIABLE_DELTA, a.fcg_delta)
    if a.fcg_slow is not None:
        s.set_option(OPT_FCG_SLOW_ITERS, a.fcg_slow)
    out = {"case": a.what}
    if a.what == "batch":
        mats, rhs = batch_meshes(a.n_sys, a.min, a.max)
        cp = s.matrix_set_batch(mats)
        b = np.concatenate(rhs)
        dev = torch.device("cuda", 0)
        bd = torch.from_numpy(b).to(dev)
        phi = torch.zeros(b.shape[0], dtype=torch.float64, device=dev)
        res0 = torch.empty_like(phi)
        ts = []
        for _ in range(a.repeat):
            phi.zero_()
            res0.copy_(bd)
            torch.cuda.synchronize()
            t = time.perf_counter()
            st = s.solv_batch_dev(a.solver, a.imat, 1e-10, 100000, 1, phi.data_ptr(),
                                  res0.data_ptr())
            ts.append(time.perf_counter() - t)
        out.update(n_sys=a.n_sys, n_cell=int(cp[-1]), s_per_batch=min(ts),
                   iters_max=int(st["iters_all"].max()), iters_min=int(st["iters_all"].min()),
                   ratio_max=float(st["ratio_all"].max()), status=st["status"])
    else:
        A, b = make_system(a.size, a.system, renumber=a.renumber)
        s.matrix_set(A)
        dev = torch.device("cuda", 0)
        if a.solver == "fcg":
            from .learn import DEFAULT_WEIGHTS, load_params
            s.gnn_set_params(load_params(a.weights or DEFAULT_WEIGHTS))
        if a.autotune:
            out["tune"] = s.autotune("cg" if a.solver != "bicg" else "bicg", a.imat, a.n_vc)
        if a.what == "kernel":
            ms = s.kernel_time(a.which, a.repeat)
            out.update(n_cell=A.n_cell, which=a.which, ms_per_launch=ms)
        elif a.what == "spmv":
            x = torch.from_numpy(uniform(3, A.n_cell)).to(dev)
            y = torch.empty_like(x)
            ms = s.spmv_dev(x.data_ptr(), y.data_ptr(), repeat=a.repeat)
            out.update(n_cell=A.n_cell, spmv_ms=ms)
        else:
            V = a.n_vc
            B = np.stack([b] + [uniform(7 + v, A.n_cell) for v in range(1, V)], axis=1)
            bd = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).to(dev)
            phi = torch.zeros(A.n_cell * V, dtype=torch.float64, device=dev)
            res0 = torch.empty_like(bd)
            ts, walls = [], []
            for _ in range(a.repeat):
                phi.zero_()
                res0.copy_(bd)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                if a.solver == "fcg":
                    rn, st = s.solv_fcg_dev(1e-10, 100000, phi.data_ptr(), res0.data_ptr())
                else:
                    fn = s.solv_cg_dev if a.solver == "cg" else s.solv_bicg_dev
                    rn, st = fn(a.imat, 1e-10, 100000, V, phi.data_ptr(), res0.data_ptr())
                walls.append(time.perf_counter() - t0)
                ts.append(st["solve_ms"])
            out.update(n_cell=A.n_cell, levels=s.levels, solve_ms=min(ts), iters=st["iters"],
                       ratio=st["ratio"], refinements=st["refinements"],
                       kernel_launches=st["kernel_launches"], status=st["status"],
                       fallbacks=st["fallbacks"], mg_levels=st["mg_levels"],
                       first_call_s=walls[0])
    s.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
