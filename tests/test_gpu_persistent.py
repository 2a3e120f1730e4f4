"""The cluster-persistent FP64 Jacobi PCG (SOLV_OPT_PERSISTENT 1): the whole
Krylov loop of solv_cg.f90:37-84 in one launch, one cluster of thread blocks
per system, the step kernels fused; systems that fit the cluster keep their
vectors in registers and shared memory, larger ones run from global memory.
Per-cell arithmetic is the graph path's, so against the oracle it is held to
the same bars: iteration counts within 2, solutions within 1e-8 at a 1e-10
residual, the initial residual bit for bit; and it must stop at the
iteration cap like the reference.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from programs_b200.mesh import Mesh, poisson_rhs
from programs_b200.solver import MAXITER, OK, OPT_PERSISTENT

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


@pytest.fixture
def persistent(gpu):
    gpu.set_option(OPT_PERSISTENT, 1)
    yield gpu
    gpu.set_option(OPT_PERSISTENT, 0)


@pytest.mark.parametrize("order", ["as_given", "rcm"])
def test_persistent_pcg_on_the_32_cube(persistent, order):
    gpu = persistent
    m = Mesh.hex(32, jitter=0.15, seed=0, permute=True)
    if order == "rcm":
        m.renumber(Mesh.RCM)
    A = m.pressure(pin=1)
    b = poisson_rhs(A.n_cell, 1).reshape(-1, 1)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b)
    gpu.matrix_set(A)
    phi = np.zeros((A.n_cell, 1))
    res0 = np.asfortranarray(b.copy())
    rn = np.zeros(1)
    st = gpu.solv_cg(0, 1e-10, 20000, phi, res0, rn)
    assert st["status"] == OK and st["graph_launches"] == 0
    assert np.array_equal(res0, ref[1])
    assert abs(rn[0] - ref[2][0]) <= 1e-12 * ref[2][0]
    assert abs(st["iters"][0] - int(ref[3][0])) <= 2, (st["iters"][0], ref[3][0])
    assert _rel(phi, ref[0]) <= 1e-8
    # the graph path on the same system: the same iteration within 2
    gpu.set_option(OPT_PERSISTENT, 0)
    phi_g = np.zeros((A.n_cell, 1))
    st_g = gpu.solv_cg(0, 1e-10, 20000, phi_g, np.asfortranarray(b.copy()), np.zeros(1))
    assert abs(st_g["iters"][0] - st["iters"][0]) <= 2 and _rel(phi_g, phi) <= 1e-8


def test_persistent_pcg_on_a_batch_and_at_the_cap(persistent):
    gpu = persistent
    mats = []
    for k, n in enumerate((6, 11, 17, 23)):
        m = Mesh.hex(n, n + 1, n - 1, jitter=0.15, seed=30 + k, permute=True)
        m.renumber(Mesh.RCM)
        mats.append(m.pressure(pin=1))
    cp = gpu.matrix_set_batch(mats)
    b = np.concatenate([poisson_rhs(A.n_cell, 50 + k) for k, A in enumerate(mats)])
    phi = np.zeros((cp[-1], 1))
    st = gpu.solv_cg_batch(0, 1e-10, 5000, phi, np.asfortranarray(b.reshape(-1, 1).copy()))
    assert st["status"] == OK
    for k, A in enumerate(mats):
        sl = slice(cp[k], cp[k + 1])
        ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 5000, np.zeros((A.n_cell, 1)),
                                            b[sl].reshape(-1, 1))
        assert _rel(phi[sl], ref[0]) <= 1e-8
        assert abs(int(st["iters_all"][k, 0]) - int(ref[3][0])) <= 2
    # the cap: every system stops at n_iter = 7, as the reference's loop does
    phi = np.zeros((cp[-1], 1))
    st = gpu.solv_cg_batch(0, 1e-10, 7, phi, np.asfortranarray(b.reshape(-1, 1).copy()))
    assert st["status"] == MAXITER and np.all(st["iters_all"][:, 0] == 7)


def test_persistent_pcg_above_the_resident_size(persistent):
    """40^3 cells are more than one 16-block cluster holds in registers and
    shared memory (32 768): the loop then runs from global memory, to the
    same bars."""
    gpu = persistent
    m = Mesh.hex(40, jitter=0.15, seed=3, permute=True)
    m.renumber(Mesh.RCM)
    A = m.pressure(pin=1)
    assert A.n_cell > 32768
    b = poisson_rhs(A.n_cell, 4).reshape(-1, 1)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b)
    gpu.matrix_set(A)
    phi = np.zeros((A.n_cell, 1))
    st = gpu.solv_cg(0, 1e-10, 20000, phi, np.asfortranarray(b.copy()), np.zeros(1))
    assert st["status"] == OK and st["graph_launches"] == 0
    assert abs(st["iters"][0] - int(ref[3][0])) <= 2
    assert _rel(phi, ref[0]) <= 1e-8


def test_persistent_pcg_on_a_batch_of_many_small_systems(persistent):
    """More systems than 16-block clusters fit on the GPU at once: each
    system gets an 8-block cluster (its cells in registers and shared
    memory); every system against its own oracle solve."""
    gpu = persistent
    mats = []
    for k in range(24):
        n = 8 + (k % 9)
        m = Mesh.hex(n, n + 1, n, jitter=0.15, seed=60 + k, permute=True)
        m.renumber(Mesh.RCM)
        mats.append(m.pressure(pin=1))
    cp = gpu.matrix_set_batch(mats)
    b = np.concatenate([poisson_rhs(A.n_cell, 80 + k) for k, A in enumerate(mats)])
    phi = np.zeros((cp[-1], 1))
    st = gpu.solv_cg_batch(0, 1e-10, 5000, phi, np.asfortranarray(b.reshape(-1, 1).copy()))
    assert st["status"] == OK
    for k, A in enumerate(mats):
        sl = slice(cp[k], cp[k + 1])
        ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 5000, np.zeros((A.n_cell, 1)),
                                            b[sl].reshape(-1, 1))
        assert _rel(phi[sl], ref[0]) <= 1e-8
        assert abs(int(st["iters_all"][k, 0]) - int(ref[3][0])) <= 2
