"""SIMPLE outer loop: host assembly pieces (CPU) and the loop itself with
the GPU solvers (GPU)."""
import numpy as np
import pytest

from programs_b200.mesh import (Mesh, cavity_field, face_flux, gradient, mass_imbalance,
                                momentum_field, pressure_correction, simple_correct)


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def _mesh(n=8, seed=1):
    m = Mesh.hex(n, jitter=0.15, seed=seed)
    m.renumber(Mesh.RCM)
    m.cache_geometry()
    return m


@pytest.mark.parametrize("jitter,tol", [(0.0, 1e-12), (0.15, 0.6)])
def test_gradient_of_constant_is_zero_and_linear_is_exact_inside(jitter, tol):
    m = Mesh.hex(8, jitter=jitter, seed=1)
    m.renumber(Mesh.RCM)
    m.cache_geometry()
    xc, _ = m.cell_geom()
    assert np.abs(gradient(m, np.ones(m.n_cell))).max() < 1e-12
    # away from the walls (zero-gradient wall values) a linear field's
    # one-sweep Green-Gauss gradient is exact on a regular mesh and
    # first-order on a skewed one (the reference repeats sweeps, n_grad)
    g = gradient(m, 3 * xc[:, 0] - 2 * xc[:, 1] + 0.5 * xc[:, 2])
    inner = np.all((xc > 0.25) & (xc < 0.75), axis=1)
    assert np.abs(g[inner] - [3, -2, 0.5]).max() < tol


def test_mass_imbalance_sums_to_zero_in_a_closed_box():
    m = _mesh()
    u = cavity_field(m, 1.0)
    M, _, F = momentum_field(m, u)
    b, tot = mass_imbalance(m, F, pin=0)
    assert abs(b.sum()) < 1e-14 and tot > 0


def test_correction_removes_the_imbalance():
    """Solving the pressure-correction system exactly and correcting the
    fluxes makes every cell but the pinned one mass-conserving."""
    import scipy.sparse.linalg as spla
    m = _mesh(7, seed=2)
    N = m.n_cell
    u = cavity_field(m, 1.0) + 0.05 * np.random.default_rng(0).normal(size=(N, 3))
    p = np.zeros(N)
    M, _, _ = momentum_field(m, u)
    gp = gradient(m, p)
    F = face_flux(m, u, p, gp, M.pl)
    P = pressure_correction(m, M.pl, pin=1)
    b, tot0 = mass_imbalance(m, F, pin=1)
    pp = spla.spsolve(P.to_scipy().tocsc(), b)
    u2, p2, F2 = u.copy(), p.copy(), F.copy()
    simple_correct(m, pp, gradient(m, pp), M.pl, 1.0, 0.3, u2, p2, F2)
    b2, tot1 = mass_imbalance(m, F2, pin=1)
    assert tot1 < 1e-10 * tot0 + 1e-14
    assert np.allclose(p2, 0.3 * pp)


@pytest.mark.gpu
def test_simple_loop_converges_and_learned_path_agrees(gpu):
    from programs_b200 import learn, simple
    u0, p0, h0, _ = simple.run(size=12, n_outer=40, re=100.0)
    mass = [h["mass"] for h in h0]
    assert mass[-1] < 0.05 * mass[1]
    w = learn.init_params(0)
    if __import__("os").path.exists(learn.DEFAULT_WEIGHTS):
        w = learn.load_params()
    u1, p1, h1, _ = simple.run(size=12, n_outer=40, re=100.0, learned=w)
    for k in range(3):
        assert simple.rel_l2(u1[:, k], u0[:, k]) <= 1e-6
    assert simple.rel_l2(p1, p0) <= 1e-6


@pytest.mark.gpu
def test_device_resident_loop_reproduces_the_host_assembly_loop(gpu):
    """Assembly, gradients, fluxes and corrections on the GPU (fv_gpu) are
    bit-for-bit the host functions and the solves see identical inputs, so
    the whole outer loop reproduces the host-assembly loop exactly."""
    from programs_b200 import simple
    u0, p0, h0, _ = simple.run(size=10, n_outer=6, re=200.0)
    u1, p1, h1, _ = simple.run_device(size=10, n_outer=6, re=200.0)
    assert np.array_equal(u1, u0) and np.array_equal(p1, p0)
    assert [h["p_iters"] for h in h1] == [h["p_iters"] for h in h0]
    for a, b in zip(h0, h1):
        assert abs(a["mass"] - b["mass"]) <= 1e-12 * a["mass"]
