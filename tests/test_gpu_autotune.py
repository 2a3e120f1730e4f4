"""The autotuner (solv_gpu_autotune) through the C-ABI.

For each solver it covers -- FP64 and FP32-inner CG, FP32-inner BiCGSTAB on
a batch of two momentum systems, and the learned flexible CG -- the tuned
launch shapes (and, for the FP32 iterations, the products' vector width)
must
* give the same solution as the settings before tuning (both solves run to
  1e-12, where the different reduction trees' paths end within 1e-8);
* be the fastest candidate measured: no slower per iteration than the
  settings before tuning, which are timed the same way in the same call and
  stay eligible;
* have looked at every candidate (10 launch shapes, x 3 vector widths when
  the iteration runs in FP32).
"""
import numpy as np
import pytest

from programs_b200 import learn
from programs_b200.mesh import Mesh, poisson_rhs, uniform
from programs_b200.solver import (OK, OPT_BLOCK, OPT_GRAPH_ITERS, OPT_GRID_PER_SM,
                                  OPT_PRECISION, OPT_VECTOR_WIDTH)

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def _defaults(gpu):
    for k, v in ((OPT_BLOCK, 256), (OPT_GRID_PER_SM, 8), (OPT_GRAPH_ITERS, 16),
                 (OPT_VECTOR_WIDTH, 4), (OPT_PRECISION, 0)):
        gpu.set_option(k, v)


def _solve(gpu, kind, b, imat):
    phi = np.zeros(b.shape, order="C")
    res0 = np.asfortranarray(b.copy())
    if kind == "fcg":
        st = gpu.solv_fcg(1e-12, 20000, phi, res0, np.zeros(1))
    else:
        st = gpu.solv_cg(imat, 1e-12, 20000, phi, res0, np.zeros(b.shape[1]))
    return phi, st


@pytest.mark.parametrize("kind,precision,imat", [("cg", 0, 0), ("cg", 1, 0), ("fcg", 1, 0)])
def test_autotune_keeps_the_solution_and_picks_the_fastest(gpu, kind, precision, imat):
    m = Mesh.hex(40, jitter=0.15, seed=2, permute=True)
    m.renumber(Mesh.RCM)
    A = m.pressure(pin=1)
    gpu.matrix_set(A)
    _defaults(gpu)
    if kind == "fcg":
        gpu.gnn_set_params(learn.load_params())
    gpu.set_option(OPT_PRECISION, precision)
    b = poisson_rhs(A.n_cell, 3).reshape(-1, 1)
    try:
        phi0, st0 = _solve(gpu, kind, b, imat)
        t = gpu.autotune(kind, imat, 1)
        phi1, st1 = _solve(gpu, kind, b, imat)
    finally:
        _defaults(gpu)
    assert st0["status"] == OK and st1["status"] == OK
    assert _rel(phi1, phi0) <= 1e-8
    assert t["candidates"] == (30 if precision == 1 else 10)
    assert t["vector_width"] in (2, 4, 8) and t["block"] in (128, 256)
    assert 0 < t["ms_per_iter"] <= t["ms_per_iter_before"]


def test_autotune_on_a_batch_of_momentum_systems(gpu):
    ms = []
    for k, n in enumerate((20, 26)):
        m = Mesh.hex(n, jitter=0.15, seed=20 + k, permute=True)
        m.renumber(Mesh.RCM)
        ms.append(m.momentum()[0])
    cp = gpu.matrix_set_batch(ms)
    _defaults(gpu)
    gpu.set_option(OPT_PRECISION, 1)
    V = 3
    b = np.asfortranarray(np.stack([uniform(40 + v, cp[-1]) for v in range(V)], axis=1))
    try:
        phi0 = np.zeros((cp[-1], V))
        st0 = gpu.solv_bicg_batch(2, 1e-12, 2000, phi0, np.asfortranarray(b.copy()))
        t = gpu.autotune("bicg", 2, V)
        phi1 = np.zeros((cp[-1], V))
        st1 = gpu.solv_bicg_batch(2, 1e-12, 2000, phi1, np.asfortranarray(b.copy()))
    finally:
        _defaults(gpu)
    assert st0["status"] == OK and st1["status"] == OK
    assert _rel(phi1, phi0) <= 1e-8
    assert t["candidates"] == 30 and 0 < t["ms_per_iter"] <= t["ms_per_iter_before"]
