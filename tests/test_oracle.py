"""The CPU oracle (oracle/) against its pins (CPU only).

The reference ships no golden vectors for its solvers and cannot be built
here (Fortran), so the restatement is pinned by:
  1. the committed fixtures in tests/golden/ (bit-for-bit, regression pin);
  2. scipy sparse direct solves of the same matrices (<= 1e-8 relative);
  3. the independent CSR twin of the same algorithms (pcns/src/solv_m.f90);
  4. manufactured solutions (b = A x*) and algebraic identities of the
     preconditioner (M = (D+L) D^-1 (D+U) with D from solv_precond).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle.oracle import Oracle, csr_solve
from programs_b200.mesh import FaceMatrix, Mesh, poisson_rhs, uniform

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def _load(name):
    return np.load(os.path.join(GOLD, name))


def _mat(d, prefix=""):
    return FaceMatrix(int(d[prefix + "n_cell"]), d[prefix + "ip"], d[prefix + "inb"],
                      d[prefix + "p"], d[prefix + "n"], d[prefix + "pl"])


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


GOLDEN = [("cavity_3d.npz", "", ("cg",)), ("channel_2d.npz", "", ("cg",)),
          ("hex6.npz", "p_", ("cg", "bicg")), ("hex6.npz", "m_", ("bicg",))]


@pytest.mark.parametrize("fname,prefix,solvers", GOLDEN)
def test_oracle_reproduces_golden(fname, prefix, solvers):
    d = _load(fname)
    A = _mat(d, prefix)
    o = Oracle.from_matrix(A)
    b = d[prefix + "b"] if prefix + "b" in d else d["b"]
    V = b.shape[1]
    for solver in solvers:
        for imat in (0, 1, 2):
            k = f"{prefix}{solver}{imat}_"
            phi, r, rn, it, _ = getattr(o, "solv_" + solver)(imat, 1e-10, 5000,
                                                            np.zeros((A.n_cell, V)), b)
            assert np.array_equal(phi, d[k + "phi"])
            assert np.array_equal(np.ascontiguousarray(r), d[k + "res0"])
            assert np.array_equal(it, d[k + "iters"])
            # and the solution is the solution of the system
            assert _rel(phi, d[prefix + "x_direct"]) <= 1e-8
    x = d[prefix + "spmv_x"]
    assert np.array_equal(o.spmv(x), d[prefix + "spmv_y"])
    assert np.allclose(o.spmv(x), A.to_scipy() @ x, rtol=1e-13, atol=1e-13)
    for imat in (0, 1, 2):
        c, c_r = o.solv_precond(imat)
        assert np.array_equal(c, d[f"{prefix}c{imat}"])
        assert np.array_equal(c_r, d[f"{prefix}c_r{imat}"])
        assert np.array_equal(o.solv_direct(imat, c, c_r, x), d[f"{prefix}direct{imat}"])


def test_cavity_fixture_matches_reader():
    """The fixture's face list is the Gambit reader's, in reference order
    (owner < neighbour, faces emitted cell by cell)."""
    d = _load("cavity_3d.npz")
    ip, inb = d["ip"], d["inb"]
    assert int(d["n_cell"]) == 125 and ip.shape[0] == 450
    assert np.all(inb[inb > 0] > ip[inb > 0])
    assert np.all(np.diff(ip) >= 0)
    assert (inb == 0).sum() == 150


def test_channel_fixture_matches_reader():
    """The reference's 2-d mesh (1 554 quadrilaterals) read one unit deep:
    every quad edge is an interior face or a wall, and the front and back
    of each cell are boundary faces (4 N = 2 interior + walls)."""
    d = _load("channel_2d.npz")
    ip, inb = d["ip"], d["inb"]
    N = int(d["n_cell"])
    n_int = int((inb > 0).sum())
    walls = int((inb == 0).sum()) - 2 * N
    assert N == 1554 and 4 * N == 2 * n_int + walls and walls > 0
    assert np.all(inb[inb > 0] > ip[inb > 0]) and np.all(np.diff(ip) >= 0)


@pytest.mark.parametrize("imat", [-1, 0, 1, 2, 3])
def test_precond_is_the_incomplete_factorisation(imat):
    """solv_direct applies M^-1 with M = (D+L) D^-1 (D+U), D = c_r.  imat
    outside 0..2 takes the reference's branches as written
    (solv_precond.f90:13-22): <= 0 is Jacobi, >= 3 keeps D = pl (the
    symmetric Gauss-Seidel factorisation) and still runs both sweeps."""
    m = Mesh.hex(5, seed=1)
    A, _ = m.momentum()
    o = Oracle.from_matrix(A)
    c, c_r = o.solv_precond(imat)
    S = A.to_scipy().tocsr()
    if imat <= 0:
        M = sp.diags(A.pl)
        # Jacobi: x = b / (pl + small)
        b = uniform(2, A.n_cell)
        assert np.allclose(o.solv_direct(imat, c, c_r, b), b / (A.pl + 1e-20), rtol=1e-15)
        return
    if imat >= 3:
        assert np.array_equal(c_r, A.pl)
    # the sweeps take L from ng%n and U from ng%p whatever imat is
    # (solv_direct.f90:19,33); imat only changes the diagonal D
    L = sp.tril(S, -1).tocsr()
    U = sp.triu(S, 1).tocsr()
    D = sp.diags(c_r)
    M = (D + L) @ sp.diags(1.0 / c_r) @ (D + U)
    b = uniform(3, A.n_cell)
    x = o.solv_direct(imat, c, c_r, b)
    assert np.allclose(M @ x, b, rtol=1e-10, atol=1e-10)
    # DILU diagonal: d_i = a_ii - sum_{j<i} a_ij a_ji / d_j
    if imat == 2:
        d = np.array(A.pl, dtype=float)
        Sl = S.tolil()
        for i in range(A.n_cell):
            for j in Sl.rows[i]:
                if j < i:
                    d[i] -= S[i, j] * S[j, i] / c_r[j]
        assert np.allclose(d, c_r, rtol=1e-12)


@pytest.mark.parametrize("kind", ["cg", "bicg"])
def test_oracle_agrees_with_csr_twin(kind):
    m = Mesh.hex(7, seed=2)
    if kind == "cg":
        A = m.pressure(pin=1)
        b = poisson_rhs(A.n_cell, 4)
    else:
        A, _ = m.momentum()
        b = uniform(4, A.n_cell)
    o = Oracle.from_matrix(A)
    phi, *_ = getattr(o, "solv_" + kind)(2, 1e-12, 5000, np.zeros((A.n_cell, 1)),
                                          b.reshape(-1, 1))
    x_csr, _ = csr_solve(A.to_scipy(), b, kind=kind, n_iter=5000, reduc=1e-12)
    assert _rel(phi[:, 0], x_csr) <= 1e-9


def test_manufactured_solution():
    m = Mesh.hex(9, seed=3)
    m.renumber(Mesh.SFC)
    A, _ = m.momentum()
    xs = uniform(5, A.n_cell)
    b = A.to_scipy() @ xs
    o = Oracle.from_matrix(A)
    phi, r, rn, it, ratio = o.solv_bicg(2, 1e-12, 5000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    assert _rel(phi[:, 0], xs) <= 1e-9
    assert np.isclose(rn[0], np.abs(b).sum(), rtol=1e-13)


def test_res_not_r0_and_components():
    m = Mesh.hex(4, seed=4)
    A = m.pressure(pin=1)
    o = Oracle.from_matrix(A)
    phi = uniform(1, A.n_cell * 3).reshape(A.n_cell, 3)
    b = np.asfortranarray(uniform(2, A.n_cell * 3).reshape(3, A.n_cell).T)
    r, rn = o.solv_res(phi, b)
    S = A.to_scipy()
    for v in range(3):
        assert np.allclose(r[:, v], b[:, v] - S @ phi[:, v], rtol=1e-13, atol=1e-13)
        assert np.isclose(rn[v], np.abs(r[:, v]).sum(), rtol=1e-14)
    r2, rn2 = o.solv_res(phi, b, not_r0=True)
    assert np.array_equal(r2, b) and np.allclose(rn2, np.abs(b).sum(axis=0))


def test_zero_rhs_early_return():
    A = Mesh.hex(3, seed=0).pressure(pin=1)
    o = Oracle.from_matrix(A)
    phi, r, rn, it, _ = o.solv_cg(0, 1e-10, 10, np.zeros((A.n_cell, 1)), np.zeros((A.n_cell, 1)))
    assert it[0] == 0 and rn[0] == 0.0


def test_scipy_pin_for_each_preconditioner():
    m = Mesh.hex(8, seed=6)
    m.renumber(Mesh.RCM)
    A = m.pressure(pin=1)
    b = poisson_rhs(A.n_cell, 6)
    x = spla.spsolve(A.to_scipy().tocsc(), b)
    o = Oracle.from_matrix(A)
    for imat in (0, 1, 2):
        for solver in ("cg", "bicg"):
            phi, *_ = getattr(o, "solv_" + solver)(imat, 1e-10, 5000, np.zeros((A.n_cell, 1)),
                                                    b.reshape(-1, 1))
            assert _rel(phi[:, 0], x) <= 1e-8


def test_reference_guard_floors_weakly_driven_systems():
    """The reference's step alpha = s / (p.Ap + small), small = 1e-20
    (solv_cg.f90:67-68, precision.f90:8), is not scale-free: on a SIMPLE
    pressure correction driven by its mass imbalance (|b| <= 6e-4) the
    Jacobi-PCG needs many times the iterations it needs for the same system
    driven 1e4 times harder, whose solution is just 1e4 times larger."""
    from test_gpu_gnn import _simple_loop_system
    A, b = _simple_loop_system()
    o = Oracle.from_matrix(A)
    weak = o.solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    strong = o.solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), 1e4 * b.reshape(-1, 1))
    n_weak, n_strong = int(weak[3][0]), int(strong[3][0])
    assert np.abs(b).max() < 1e-3
    assert n_strong < 400 and n_weak > 10 * n_strong, (n_weak, n_strong)
    assert _rel(weak[0] * 1e4, strong[0]) < 1e-6


def test_fixtures_regenerate_bit_for_bit(tmp_path):
    """tests/golden/make_golden.py rebuilds the committed fixtures exactly:
    the mesh generator, the assembly, the seeded right-hand sides and the
    oracle have not drifted from what the fixtures hold.  The fixtures of
    the reference's own meshes are rebuilt only where SPRAY_SIMULATION_DIR
    names the reference's spray-simulation/ directory."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    mg.hex6(str(tmp_path))
    names = ["hex6.npz"]
    neu = mg.reference_mesh("cavity_3d.neu")
    if neu and os.path.exists(neu):
        mg.cavity(neu, str(tmp_path))
        names.append("cavity_3d.npz")
    neu2 = mg.reference_mesh("channel_2d.neu")
    if neu2 and os.path.exists(neu2):
        mg.channel(neu2, str(tmp_path))
        names.append("channel_2d.npz")
    for name in names:
        new, old = np.load(str(tmp_path / name)), _load(name)
        assert sorted(new.files) == sorted(old.files), name
        for k in old.files:
            assert np.array_equal(new[k], old[k]), (name, k)
