"""GPU forms beyond the plain FP64 path: mixed precision (FP32 inner Krylov
with FP64 iterative refinement) and batches of independent systems.

Mixed precision changes the arithmetic on purpose, so it is held to the
solution, not the bits: the true FP64 residual must reach the reference's
stopping rule (|b - A x|_1 / |r0|_1 < 1e-10) and the solution must agree
with the FP64 oracle to 1e-8 relative.  Batches must reproduce, system by
system, what separate solv_cg / solv_bicg calls give.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from programs_b200.mesh import Mesh, poisson_rhs, uniform
from programs_b200.solver import OK, OPT_PRECISION

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-8
# Two different iterations that both stop at |r|_1/|r0|_1 < 1e-10 differ by
# up to about cond(A) x 1e-10; the FP32-inner solves of a batch of uneven
# meshes are held to that (their own FP64 residual is checked exactly).
MIX_BATCH_TOL = 1e-7


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


@pytest.fixture
def mixed(gpu):
    gpu.set_option(OPT_PRECISION, 1)
    yield gpu
    gpu.set_option(OPT_PRECISION, 0)


@pytest.mark.parametrize("imat", [0, 1, 2])
def test_mixed_cg_pressure(mixed, imat):
    m = Mesh.hex(16, seed=1)
    m.renumber(Mesh.RCM)
    A = m.pressure(pin=1)
    o = Oracle.from_matrix(A)
    mixed.matrix_set(A)
    b = np.asfortranarray(poisson_rhs(A.n_cell, 2).reshape(-1, 1))
    ref = o.solv_cg(imat, 1e-10, 5000, np.zeros((A.n_cell, 1)), b)
    phi = np.zeros((A.n_cell, 1))
    res0 = b.copy(order="F")
    rn = np.zeros(1)
    st = mixed.solv_cg(imat, 1e-10, 5000, phi, res0, rn)
    assert st["status"] == OK and st["refinements"] >= 2
    # the reference's stopping rule on the true FP64 residual
    r_true = b[:, 0] - A.to_scipy() @ phi[:, 0]
    assert np.abs(r_true).sum() / rn[0] < 1e-10
    assert _rel(phi, ref[0]) <= SOL_TOL
    assert np.array_equal(res0, ref[1])  # initial residual stays FP64-exact


@pytest.mark.parametrize("imat", [0, 2])
def test_mixed_bicg_momentum_three_components(mixed, imat):
    m = Mesh.hex(14, seed=2)
    m.renumber(Mesh.SFC)
    A, _ = m.momentum()
    o = Oracle.from_matrix(A)
    mixed.matrix_set(A)
    V = 3
    b = np.asfortranarray(np.stack([uniform(30 + v, A.n_cell) for v in range(V)], axis=1))
    ref = o.solv_bicg(imat, 1e-10, 2000, np.zeros((A.n_cell, V)), b)
    phi = np.zeros((A.n_cell, V))
    res0 = b.copy(order="F")
    rn = np.zeros(V)
    st = mixed.solv_bicg(imat, 1e-10, 2000, phi, res0, rn)
    assert st["status"] == OK
    S = A.to_scipy()
    for v in range(V):
        assert np.abs(b[:, v] - S @ phi[:, v]).sum() / rn[v] < 1e-10
        assert _rel(phi[:, v], ref[0][:, v]) <= SOL_TOL


@pytest.mark.parametrize("solver,imat", [("cg", 0), ("cg", 1), ("bicg", 0), ("bicg", 2)])
def test_mixed_solve_of_a_weakly_driven_system(mixed, solver, imat):
    """A right-hand side of size 1e-6 (a SIMPLE pressure correction near
    convergence is driven about this weakly): the inner products of the
    FP32 iteration fall far below the reference's absolute guard 1e-20 well
    before the 1e-10 stopping rule, and the solve must still reach it, with
    the solution 1e-6 times that of the unit right-hand side."""
    m = Mesh.hex(12, seed=3)
    m.renumber(Mesh.RCM)
    A = m.pressure(pin=1) if solver == "cg" else m.momentum()[0]
    mixed.matrix_set(A)
    b1 = poisson_rhs(A.n_cell, 5) if solver == "cg" else uniform(5, A.n_cell)
    S = A.to_scipy()
    sols = []
    for scale in (1.0, 1e-6):
        b = np.asfortranarray((scale * b1).reshape(-1, 1))
        phi = np.zeros((A.n_cell, 1))
        res0 = b.copy(order="F")
        rn = np.zeros(1)
        st = getattr(mixed, "solv_" + solver)(imat, 1e-10, 5000, phi, res0, rn)
        assert st["status"] == OK, scale
        assert np.abs(b[:, 0] - S @ phi[:, 0]).sum() / rn[0] < 1e-10, scale
        sols.append(phi[:, 0] / scale)
    assert _rel(sols[1], sols[0]) <= MIX_BATCH_TOL


def _batch_meshes(k, seed=0):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(4), np.log(11), k)).astype(int)
    out = []
    for j, n in enumerate(sizes):
        m = Mesh.hex(int(n), int(max(3, n - 1)), int(n), seed=100 + j)
        m.renumber(Mesh.RCM if j % 2 else Mesh.SFC)
        out.append(m)
    return out


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("imat", [0, 1])
def test_batch_pressure_matches_separate_solves(gpu, precision, imat):
    meshes = _batch_meshes(7, seed=precision * 10 + imat)
    mats = [m.pressure(pin=1) for m in meshes]
    cell_ptr = gpu.matrix_set_batch(mats)
    gpu.set_option(OPT_PRECISION, precision)
    try:
        b = np.concatenate([poisson_rhs(A.n_cell, 5 + k) for k, A in enumerate(mats)])
        phi = np.zeros((cell_ptr[-1], 1))
        res0 = np.asfortranarray(b.reshape(-1, 1).copy())
        st = gpu.solv_cg_batch(imat, 1e-10, 3000, phi, res0)
    finally:
        gpu.set_option(OPT_PRECISION, 0)
    assert st["status"] == OK
    for k, A in enumerate(mats):
        sl = slice(cell_ptr[k], cell_ptr[k + 1])
        ref = Oracle.from_matrix(A).solv_cg(imat, 1e-10, 3000, np.zeros((A.n_cell, 1)),
                                            b[sl].reshape(-1, 1))
        assert _rel(phi[sl], ref[0]) <= (SOL_TOL if precision == 0 else MIX_BATCH_TOL)
        if precision == 1:
            r = b[sl] - A.to_scipy() @ phi[sl, 0]
            assert np.abs(r).sum() / np.abs(b[sl]).sum() < 1e-10
        assert np.array_equal(res0[sl], ref[1])
        assert np.isclose(st["res0_n"][k, 0], ref[2][0], rtol=1e-12)
        if precision == 0:
            assert abs(int(st["iters_all"][k, 0]) - int(ref[3][0])) <= 2
        assert st["ratio_all"][k, 0] < 1e-10


def test_batch_momentum_bicg_dilu(gpu):
    meshes = _batch_meshes(5, seed=42)
    mats = [m.momentum()[0] for m in meshes]
    cell_ptr = gpu.matrix_set_batch(mats)
    V = 3
    b = np.asfortranarray(np.stack([uniform(60 + v, cell_ptr[-1]) for v in range(V)], axis=1))
    phi = np.zeros((cell_ptr[-1], V))
    res0 = b.copy(order="F")
    st = gpu.solv_bicg_batch(2, 1e-10, 1000, phi, res0)
    assert st["status"] == OK
    for k, A in enumerate(mats):
        sl = slice(cell_ptr[k], cell_ptr[k + 1])
        ref = Oracle.from_matrix(A).solv_bicg(2, 1e-10, 1000, np.zeros((A.n_cell, V)),
                                              np.asfortranarray(b[sl]))
        for v in range(V):
            assert _rel(phi[sl, v], ref[0][:, v]) <= SOL_TOL
            assert abs(int(st["iters_all"][k, v]) - int(ref[3][v])) <= 2


def test_batch_rejects_coupled_systems(gpu):
    from programs_b200.solver import SolverError
    a = Mesh.hex(3, seed=1).pressure(pin=1)
    b = Mesh.hex(3, seed=2).pressure(pin=1)
    ip = np.concatenate([a.ip, b.ip + a.n_cell]).astype(np.int32)
    inb = np.concatenate([a.inb, np.where(b.inb > 0, b.inb + a.n_cell, 0)]).astype(np.int32)
    inb[np.argmax(a.inb == 0)] = a.n_cell + 1  # a face that couples the two
    import ctypes
    cp = np.array([0, a.n_cell, a.n_cell + b.n_cell], np.int32)
    p = np.concatenate([a.p, b.p])
    n = np.concatenate([a.n, b.n])
    pl = np.concatenate([a.pl, b.pl])
    L = gpu._lib
    f64 = ctypes.POINTER(ctypes.c_double)
    i32 = ctypes.POINTER(ctypes.c_int)
    rc = L.solv_gpu_matrix_set_batch(gpu._h, 2, cp.ctypes.data_as(i32), ip.shape[0],
                                     ip.ctypes.data_as(i32), inb.ctypes.data_as(i32),
                                     p.ctypes.data_as(f64), n.ctypes.data_as(f64),
                                     pl.ctypes.data_as(f64))
    assert rc == 4
    with pytest.raises(SolverError):
        gpu._check(rc)


@pytest.mark.parametrize("solver,imat,precision", [("cg", 0, 0), ("cg", 1, 0), ("bicg", 2, 0),
                                                   ("cg", 0, 1), ("bicg", 2, 1)])
def test_while_graph_equals_fixed_graphs(gpu, solver, imat, precision):
    """SOLV_OPT_GRAPH_LOOP 1 runs the iterations in a conditional WHILE graph
    that ends on the device once every lane has stopped; 0 launches graphs of
    SOLV_OPT_GRAPH_ITERS iterations.  The iterations are the same kernels in
    the same order, so the two give the same iterations and the same
    solution, bit for bit; the FP64 solve is one WHILE launch, or one
    launch per 8 iterations."""
    from programs_b200.solver import OPT_GRAPH_ITERS, OPT_GRAPH_LOOP
    m = Mesh.hex(14, seed=8)
    m.renumber(Mesh.RCM)
    if solver == "cg":
        A = m.pressure(pin=1)
        b = poisson_rhs(A.n_cell, 3)
    else:
        A, _ = m.momentum()
        b = uniform(5, A.n_cell)
    gpu.matrix_set(A)
    out = {}
    gpu.set_option(OPT_PRECISION, precision)
    gpu.set_option(OPT_GRAPH_ITERS, 8)
    try:
        for loop in (1, 0):
            gpu.set_option(OPT_GRAPH_LOOP, loop)
            phi = np.zeros((A.n_cell, 1))
            st = getattr(gpu, "solv_" + solver)(imat, 1e-10, 5000, phi,
                                                np.asfortranarray(b.reshape(-1, 1).copy()),
                                                np.zeros(1))
            assert st["status"] == OK
            out[loop] = (phi, st["iters"][0], st["graph_launches"])
    finally:
        gpu.set_option(OPT_GRAPH_LOOP, 2)
        gpu.set_option(OPT_GRAPH_ITERS, 16)
        gpu.set_option(OPT_PRECISION, 0)
    assert out[1][1] == out[0][1]
    assert np.array_equal(out[1][0], out[0][0])
    if precision == 0:
        assert out[1][2] == 1 and out[0][2] == -(-int(out[0][1]) // 8)
