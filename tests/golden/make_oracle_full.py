"""Full-size oracle solve of the benchmark's pressure system (fixture maker).

TEST INFRASTRUCTURE: runs the CPU oracle (the line-by-line C restatement
of spray-simulation/solv_cg.f90:19-86, single core, FP64, Jacobi
preconditioner, reduc 1e-10) on the 256^3 pressure-correction system that
``bench.py`` times -- jitter +-15%, cells permuted (seed 0), RCM
renumbering, coefficients area/l_pn, cell 1 pinned, rhs uniform[-1,1]
(seed 1) with its mean removed -- to convergence, and writes what a test
needs to hold the GPU to it without the 134 MB solution:

* the oracle's own iteration count, last ratio and initial L1 norm;
* the solution's L1 / L2 norms and its values at 4096 seeded indices;
* the wall time of the solve on this host (single core).

A run takes about half an hour.  Usage:

  python tests/golden/make_oracle_full.py [--size 256] [--out FILE]
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

N_SAMPLE = 4096


def sample_indices(n: int, seed: int = 7) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(n, size=min(N_SAMPLE, n), replace=False))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    from bench import build_system
    from oracle.oracle import Oracle

    t0 = time.perf_counter()
    A, b = build_system(args.size, seed=0)
    t_build = time.perf_counter() - t0
    o = Oracle.from_matrix(A)
    t0 = time.perf_counter()
    phi, _, rn, iters, ratio = o.solv_cg(0, 1e-10, 100000, np.zeros((A.n_cell, 1)),
                                         b.reshape(-1, 1))
    dt = time.perf_counter() - t0
    x = phi[:, 0]
    idx = sample_indices(A.n_cell)
    out = {
        "system": f"pressure Poisson {args.size}^3 jittered hex (bench.build_system, seed 0)",
        "solver": "oracle solv_cg, imat 0 (Jacobi), reduc 1e-10, FP64, single core",
        "n_cell": int(A.n_cell), "iterations": int(iters[0]), "ratio": float(ratio[0]),
        "res0_n": float(rn[0]), "solve_s": dt, "build_s": t_build,
        "host": platform.processor() or platform.machine(),
        "x_l1": float(np.abs(x).sum()), "x_l2": float(np.linalg.norm(x)),
        "sample_seed": 7, "sample_idx": idx.tolist(), "sample_x": x[idx].tolist(),
    }
    path = args.out or os.path.join(HERE, f"oracle_pcg_{args.size}.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print(json.dumps({k: v for k, v in out.items() if not k.startswith("sample_")}))


if __name__ == "__main__":
    main()
