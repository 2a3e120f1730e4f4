"""Generate the golden fixtures in tests/golden/ (run here, committed).

* cavity_3d.npz -- the 125-cell brick mesh shipped with the reference
  (spray-simulation/cavity_3d.neu), read by programs_b200's Gambit reader,
  its face list in the reference's connectivity order, the pressure
  matrix assembled on it, a seeded right-hand side, and the oracle's
  solv_cg / solv_bicg outputs for imat = 0, 1, 2 together with a scipy
  sparse direct solution.  Reading the .neu needs the reference checkout,
  so this part only runs where it is present.
* channel_2d.npz -- the same for the reference's 2-d mesh
  (spray-simulation/channel_2d.neu, 1 554 quadrilaterals, read one unit
  deep).
* hex6.npz -- a 6x6x6 jittered, permuted hex mesh (seed 0): pressure and
  momentum matrices with the same set of outputs (3 right-hand sides for
  the momentum solve).

The tests re-run the oracle on the stored matrices and require the stored
outputs bit for bit, check the solutions against the stored scipy solves,
and run the GPU solvers against the same outputs.

Usage: python tests/golden/make_golden.py [path/to/cavity_3d.neu [path/to/channel_2d.neu]]

Without arguments the two .neu files are looked up in the directory named
by the environment variable SPRAY_SIMULATION_DIR (the reference's
spray-simulation/ checkout); with neither, only hex6.npz is rebuilt.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from programs_b200 import build  # noqa: E402
from programs_b200.mesh import Mesh, poisson_rhs, uniform  # noqa: E402


def reference_mesh(name: str) -> str | None:
    """Path of a mesh the reference ships (spray-simulation/<name>), from
    the directory in SPRAY_SIMULATION_DIR; None when that is not set."""
    d = os.environ.get("SPRAY_SIMULATION_DIR")
    return os.path.join(d, name) if d else None

REDUC = 1e-10
N_ITER = 5000


def _solves(A, b, prefix, out, solvers=("cg", "bicg")):
    import scipy.sparse.linalg as spla
    o = Oracle.from_matrix(A)
    S = A.to_scipy().tocsc()
    V = b.shape[1]
    out[prefix + "x_direct"] = np.stack([spla.spsolve(S, b[:, v]) for v in range(V)], axis=1)
    for solver in solvers:
        for imat in (0, 1, 2):
            phi, r, rn, it, ratio = getattr(o, "solv_" + solver)(
                imat, REDUC, N_ITER, np.zeros((A.n_cell, V)), b)
            k = f"{prefix}{solver}{imat}_"
            out[k + "phi"] = phi
            out[k + "res0"] = np.ascontiguousarray(r)
            out[k + "res0_n"] = rn
            out[k + "iters"] = it
    x = uniform(123, A.n_cell)
    out[prefix + "spmv_x"] = x
    out[prefix + "spmv_y"] = o.spmv(x)
    for imat in (0, 1, 2):
        c, c_r = o.solv_precond(imat)
        out[f"{prefix}c{imat}"] = c
        out[f"{prefix}c_r{imat}"] = c_r
        out[f"{prefix}direct{imat}"] = o.solv_direct(imat, c, c_r, x)


def _matrix(A, prefix, out):
    out[prefix + "n_cell"] = np.int32(A.n_cell)
    out[prefix + "ip"] = A.ip
    out[prefix + "inb"] = A.inb
    out[prefix + "p"] = A.p
    out[prefix + "n"] = A.n
    out[prefix + "pl"] = A.pl


def cavity(path: str, outdir: str = HERE) -> None:
    m = Mesh.read_neu(path)
    A = m.pressure(pin=1)
    b = np.asfortranarray(poisson_rhs(A.n_cell, 7).reshape(-1, 1))
    out = {}
    _matrix(A, "", out)
    out["b"] = b
    _solves(A, b, "", out, solvers=("cg",))
    np.savez_compressed(os.path.join(outdir, "cavity_3d.npz"), **out)
    print("cavity_3d:", A.n_cell, "cells", A.n_face, "faces")


def channel(path: str, outdir: str = HERE) -> None:
    """The reference's 2-d mesh (1 554 quadrilaterals, read one unit deep)."""
    m = Mesh.read_neu(path)
    A = m.pressure(pin=1)
    b = np.asfortranarray(poisson_rhs(A.n_cell, 11).reshape(-1, 1))
    out = {}
    _matrix(A, "", out)
    out["b"] = b
    _solves(A, b, "", out, solvers=("cg",))
    np.savez_compressed(os.path.join(outdir, "channel_2d.npz"), **out)
    print("channel_2d:", A.n_cell, "cells", A.n_face, "faces")


def hex6(outdir: str = HERE) -> None:
    m = Mesh.hex(6, jitter=0.15, seed=0, permute=True)
    P = m.pressure(pin=1)
    M, dt = m.momentum()
    out = {}
    _matrix(P, "p_", out)
    _matrix(M, "m_", out)
    bp = np.asfortranarray(poisson_rhs(P.n_cell, 1).reshape(-1, 1))
    bm = np.asfortranarray(np.stack([uniform(10 + v, M.n_cell) for v in range(3)], axis=1))
    out["p_b"] = bp
    out["m_b"] = bm
    _solves(P, bp, "p_", out, solvers=("cg", "bicg"))
    _solves(M, bm, "m_", out, solvers=("bicg",))
    np.savez_compressed(os.path.join(outdir, "hex6.npz"), **out)
    print("hex6:", P.n_cell, "cells", P.n_face, "faces; momentum dt", dt)


if __name__ == "__main__":
    build.build_all()
    hex6()
    neu = sys.argv[1] if len(sys.argv) > 1 else reference_mesh("cavity_3d.neu")
    if neu and os.path.exists(neu):
        cavity(neu)
    else:
        print("cavity_3d.neu not found; cavity_3d.npz left as is")
    neu2 = sys.argv[2] if len(sys.argv) > 2 else reference_mesh("channel_2d.neu")
    if neu2 and os.path.exists(neu2):
        channel(neu2)
    else:
        print("channel_2d.neu not found; channel_2d.npz left as is")
