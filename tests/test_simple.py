"""SIMPLE outer loop: host assembly pieces (CPU) and the loop itself with
the GPU solvers (GPU)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
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


def test_one_sweep_with_wall_values_is_the_single_sweep_gradient():
    """solv_grad with n_iter = 1, neu = 1 is the one-sweep gradient above
    (the 1/V factor per face instead of once per cell changes the rounding
    only)."""
    from programs_b200.mesh import gradient_sweeps
    m = _mesh(8)
    phi = np.random.default_rng(0).normal(size=(m.n_cell, 2))
    g = gradient_sweeps(m, phi, 1, 1)
    assert np.abs(g - gradient(m, phi)).max() < 1e-12 * np.abs(g).max()


@pytest.mark.parametrize("jitter", [0.0, 0.2])
def test_sweeps_known_answer_of_the_reference_self_check(jitter):
    """The reference's built-in check (test_grad, cfd_setup.f90:871-921):
    phi = x y with its exact values on the boundary faces (neu = 0), RMS
    error of d/dx -> y and d/dy -> x for 1..6 sweeps.  Exact on a regular
    mesh; on a skewed one the corrected sweeps cut the first sweep's error
    several times and settle by the fourth."""
    from programs_b200.mesh import gradient_sweeps
    m = Mesh.hex(12, jitter=jitter, seed=1, permute=True)
    xc, _ = m.cell_geom()
    _, _, xf, _, _ = m.face_geom()
    phi, bval = xc[:, 0] * xc[:, 1], xf[:, 0] * xf[:, 1]
    exact = np.stack([xc[:, 1], xc[:, 0], np.zeros(m.n_cell)], 1)
    err = [np.sqrt(((gradient_sweeps(m, phi, n, 0, bval) - exact) ** 2).mean(0)).max()
           for n in range(1, 7)]
    if jitter == 0.0:
        assert max(err) < 1e-12
    else:
        assert err[1] < 0.3 * err[0] and abs(err[5] - err[3]) < 0.05 * err[3]
    with pytest.raises(ValueError):
        gradient_sweeps(m, phi, 2, 0)          # Dirichlet walls need their values
    with pytest.raises(ValueError):
        gradient_sweeps(m, phi, 0, 1)


def test_extrapolated_walls_converge_to_a_linear_gradient():
    """neu = 2 (the pressure gradient's walls, cfd_setup.f90:689, 754):
    the wall value is the cell value moved to the face with the previous
    sweep's gradient, so on a regular mesh each sweep halves the error of
    a linear field; zero-gradient walls (neu = 1) keep it."""
    from programs_b200.mesh import gradient_sweeps
    m = Mesh.hex(10, jitter=0.0, seed=1, permute=True)
    xc, _ = m.cell_geom()
    a = np.array([0.7, -1.3, 0.4])
    phi = xc @ a + 2.0
    e = [np.abs(gradient_sweeps(m, phi, n, 2) - a).max() for n in (1, 2, 3, 30)]
    assert abs(e[1] / e[0] - 0.5) < 1e-6 and abs(e[2] / e[1] - 0.5) < 1e-6 and e[3] < 1e-8
    assert abs(np.abs(gradient_sweeps(m, phi, 4, 1) - a).max() - e[0]) < 1e-9


def _cell_sums(m, per_face_p, per_face_n):
    """Sum per-face owner and neighbour contributions into cells."""
    ip, inb = m.faces()
    out = np.zeros(m.n_cell)
    np.add.at(out, ip - 1, per_face_p)
    inner = inb > 0
    np.add.at(out, inb[inner] - 1, per_face_n[inner])
    return out


def test_deferred_diffusion_correction_makes_a_linear_field_harmonic():
    """On a skewed mesh the implicit two-point diffusion d (phi_N - phi_P)
    misses the tangential part of the gradient; with the reference's
    explicit correction d ((phi_N' - phi_P') - (phi_N - phi_P)) the face
    flux is d (phi_N' - phi_P') = mu area grad.n for a linear field, so
    every interior cell balances exactly (cfd_setup.f90:318-322)."""
    from programs_b200.mesh import momentum_deferred
    m = Mesh.hex(8, jitter=0.2, seed=4, permute=True)
    xc, _ = m.cell_geom()
    s, nrm, xf, l, w = m.face_geom()
    ip, inb = m.faces()
    a = np.array([0.7, -1.3, 0.4])
    phi = xc @ a + 2.0
    grad = np.tile(a, (m.n_cell, 1))
    mu = 0.01
    rhs = momentum_deferred(m, phi, grad, np.zeros(m.n_face), mu, c_bl=1.0)
    inner = inb > 0
    d = np.where(inner, mu * s / l, 0.0)
    pb = np.where(inner, phi[np.maximum(inb, 1) - 1], 0.0)
    pa = phi[ip - 1]
    implicit = _cell_sums(m, d * (pa - pb), np.where(inner, d * (pb - pa), 0.0))
    interior = np.bincount(ip - 1, weights=~inner, minlength=m.n_cell) == 0  # no wall face
    scale = np.abs(implicit[interior]).max()
    assert scale > 1e-4                                   # the skew is visible without it
    assert np.abs(implicit[interior] - rhs[interior]).max() < 1e-10 * scale + 1e-15
    assert abs(rhs.sum()) < 1e-12 * np.abs(rhs).sum()     # conservative


def test_deferred_convection_term_is_central_minus_upwind():
    """c_bl c (phi_up - phi_f): zero for a constant field; on a regular mesh
    (auxiliary points at the cell centres, w = 1/2) exactly c (phi_up -
    (phi_P + phi_N) / 2) per face, owner +, neighbour -."""
    from programs_b200.mesh import momentum_deferred
    m = Mesh.hex(6, jitter=0.0, seed=2, permute=True)
    xc, _ = m.cell_geom()
    ip, inb = m.faces()
    c = np.random.default_rng(1).normal(size=m.n_face)
    zero_grad = np.zeros((m.n_cell, 3))
    assert np.abs(momentum_deferred(m, np.full(m.n_cell, 3.0), zero_grad, c, 0.0)).max() == 0.0
    phi = xc[:, 0] - 2 * xc[:, 1]
    grad = np.tile([1.0, -2.0, 0.0], (m.n_cell, 1))
    got = momentum_deferred(m, phi, grad, c, 0.0, c_bl=0.5)
    inner = inb > 0
    pa = phi[ip - 1]
    pb = np.where(inner, phi[np.maximum(inb, 1) - 1], 0.0)
    cor = np.where(inner, 0.5 * c * (np.where(c > 0, pa, pb) - 0.5 * (pa + pb)), 0.0)
    want = _cell_sums(m, cor, -cor)
    assert np.abs(got - want).max() < 1e-13


class _OracleSolver:
    """The loop's solver interface over the CPU oracle -- the reference's
    own solver arithmetic -- so the host loop runs without a GPU."""

    def __init__(self, device=0):
        self.o = None

    def set_option(self, key, value):
        from programs_b200.solver import OPT_PRECISION
        assert key == OPT_PRECISION and value == 0  # the oracle is FP64

    def matrix_set(self, A):
        self.structure = (A.n_cell, A.ip, A.inb)
        self.o = Oracle.from_matrix(A)

    def matrix_values(self, p, n, pl):
        self.o = Oracle(*self.structure, p, n, pl)

    def _solve(self, kind, imat, reduc, n_iter, phi, res0, rn, not_r0):
        x, r, r0n, its, ratio = getattr(self.o, "solv_" + kind)(imat, reduc, n_iter, phi, res0,
                                                               not_r0)
        phi[...] = x.reshape(phi.shape)
        res0[...] = r.reshape(res0.shape)
        rn[...] = r0n
        return {"iters": [int(i) for i in its], "ratio": [float(q) for q in ratio], "status": 0}

    def solv_cg(self, imat, reduc, n_iter, phi, res0, rn, not_r0=False):
        return self._solve("cg", imat, reduc, n_iter, phi, res0, rn, not_r0)

    def solv_bicg(self, imat, reduc, n_iter, phi, res0, rn, not_r0=False):
        return self._solve("bicg", imat, reduc, n_iter, phi, res0, rn, not_r0)

    def close(self):
        self.o = None


def test_host_loop_with_the_reference_solvers_reduces_the_mass_imbalance():
    """The outer loop (host assembly, cfd_solve.f90:131-179) with the
    oracle's solv_bicg / solv_cg at the reference's own settings (momentum
    BiCGSTAB + DILU to 0.1 in at most 5 iterations, pressure DIC-PCG to 0.1
    in at most 20, cfd_setup.f90:528, 662): the caps hold, the fields stay
    finite, and in 30 outer iterations the mass imbalance falls by more
    than three orders of magnitude."""
    from programs_b200 import simple
    u, p, hist, _ = simple.run(size=6, n_outer=30, re=100.0, p_reduc=0.1, p_iter=20, p_imat=1,
                               make_solver=_OracleSolver)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(p))
    assert all(h["p_iters"] <= 20 and max(h["m_iters"]) <= 5 for h in hist)
    mass = [h["mass"] for h in hist]
    assert mass[-1] < 1e-3 * mass[0], mass


def test_tvd_schemes_are_central_on_linear_fields_and_upwind_without_gradient():
    """c_sch 1..3 (min-mod, van Leer, superbee, cfd_setup.f90:253-272): on a
    linear field with its exact gradient the ratio r is 1 and every limiter
    gives psi(1) = 1, the central face value; with zero gradients the
    reconstructed upstream value equals the downwind one, r = -1, psi = 0,
    and the face value is the upwind one (no correction)."""
    from programs_b200.mesh import momentum_deferred
    m = Mesh.hex(6, jitter=0.0, seed=2, permute=True)
    xc, _ = m.cell_geom()
    c = np.random.default_rng(3).normal(size=m.n_face)
    phi = 2 * xc[:, 0] + xc[:, 2]
    grad = np.tile([2.0, 0.0, 1.0], (m.n_cell, 1))
    central = momentum_deferred(m, phi, grad, c, 0.0, scheme=0)
    assert np.abs(central).max() > 1e-3
    for scheme in (1, 2, 3):
        assert np.abs(momentum_deferred(m, phi, grad, c, 0.0, scheme=scheme) - central).max() < 1e-13
        assert np.abs(momentum_deferred(m, phi, 0 * grad, c, 0.0, scheme=scheme)).max() < 1e-15
    assert np.abs(momentum_deferred(m, phi, 0 * grad, c, 0.0, scheme=0)).max() > 1e-3
    with pytest.raises(ValueError):
        momentum_deferred(m, phi, grad, c, 0.0, scheme=4)


def test_host_loop_with_the_reference_explicit_terms():
    """The same loop with the reference's explicit terms and corrected
    gradients (reference_terms): the mass imbalance falls by more than two
    orders of magnitude in 30 outer iterations (the explicit terms lag one
    iteration, so a little slower than the implicit-only loop), and on
    this coarse skewed mesh the central face values move the velocity
    field by some tens of percent against first-order upwind."""
    from programs_b200 import simple
    kw = dict(size=6, n_outer=30, re=100.0, p_reduc=0.1, p_iter=20, p_imat=1,
              make_solver=_OracleSolver)
    u0, p0, _, _ = simple.run(**kw)
    u1, p1, hist, _ = simple.run(reference_terms=True, **kw)
    assert np.all(np.isfinite(u1)) and np.all(np.isfinite(p1))
    mass = [h["mass"] for h in hist]
    assert mass[-1] < 1e-2 * mass[0], mass
    rel = np.linalg.norm(u1 - u0) / np.linalg.norm(u0)
    assert 1e-4 < rel < 0.5, rel
    u2, _, hist2, _ = simple.run(reference_terms=True, reference_weights=True, **kw)
    mass2 = [h["mass"] for h in hist2]
    assert np.all(np.isfinite(u2)) and mass2[-1] < 1e-2 * mass2[0], mass2
    assert not np.array_equal(u2, u1)            # the weights differ on the skewed mesh


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
    the whole outer loop reproduces the host-assembly loop exactly -- with
    the implicit terms alone and with the reference's explicit momentum
    terms, corrected gradient sweeps and auxiliary-point face pressures."""
    from programs_b200 import simple
    for ref in (False, True):  # implicit terms only; with the reference's explicit terms
        u0, p0, h0, _ = simple.run(size=10, n_outer=6, re=200.0, reference_terms=ref)
        u1, p1, h1, _ = simple.run_device(size=10, n_outer=6, re=200.0, reference_terms=ref)
        assert np.array_equal(u1, u0) and np.array_equal(p1, p0), ref
        assert [h["p_iters"] for h in h1] == [h["p_iters"] for h in h0]
        for a, b in zip(h0, h1):
            assert abs(a["mass"] - b["mass"]) <= 1e-12 * a["mass"]


def test_face_flux_at_the_auxiliary_points():
    """The reference's pressure-correction face loop takes the pressures at
    the auxiliary points (cfd_setup.f90:611-620).  On a mesh without jitter
    the auxiliary points are the cell centres (to rounding) and the two
    fluxes agree; on a skewed mesh, for a linear pressure with its exact
    gradient and no velocity, the plain form's smoothing term vanishes and
    the auxiliary form keeps -d g.(x_N' - x_P') (d > 0), as the reference's
    formula does."""
    from programs_b200.mesh import face_flux, momentum_field
    g = np.array([0.3, -0.2, 0.5])
    for jitter in (0.0, 0.2):
        m = Mesh.hex(7, jitter=jitter, seed=4, permute=True)
        m.renumber(Mesh.RCM)
        A, _, _ = momentum_field(m, cavity_field(m, 1.0))
        xc, _ = m.cell_geom()
        p = xc @ g
        gp = np.tile(g, (m.n_cell, 1))
        u0 = np.zeros((m.n_cell, 3))
        f0 = face_flux(m, u0, p, gp, A.pl)
        f1 = face_flux(m, u0, p, gp, A.pl, aux=True)
        assert np.abs(f0).max() < 1e-14
        if jitter == 0.0:
            assert np.abs(f1).max() < 1e-14
            continue
        ip, inb = m.faces()
        _, nrm, xf, _, _ = m.face_geom()
        inner = np.nonzero(inb > 0)[0]
        a, b = ip[inner] - 1, inb[inner] - 1
        def aux(c):
            t = np.einsum("ij,ij->i", xf[inner] - xc[c], nrm[inner])
            return (xf[inner] - nrm[inner] * t[:, None]) - xc[c]
        dp_aux = (aux(b) - aux(a)) @ g
        big = np.abs(dp_aux) > 1e-10
        assert big.sum() > inner.size // 2
        assert np.all(f1[inner][big] / dp_aux[big] < 0)  # -d dp_aux with d > 0


def test_pressure_rhs_scaling_is_exact():
    """p_scale multiplies the pressure right-hand side by a power of two and
    divides the solution by it: exact in floating point, so with the
    oracle's solvers at the reference's settings (where the absolute guard
    is far from binding) the loop's fields come out the same."""
    from programs_b200 import simple
    assert simple.rhs_scale(1000, 1.0) == 1024.0 and simple.rhs_scale(8, 0.0) == 1.0
    kw = dict(size=6, n_outer=6, re=100.0, p_reduc=0.1, p_iter=20, p_imat=1,
              make_solver=_OracleSolver)
    u0, p0, _, _ = simple.run(**kw)
    u1, p1, _, _ = simple.run(p_scale=True, **kw)
    assert np.allclose(u1, u0, rtol=1e-12, atol=1e-15) and np.allclose(p1, p0, rtol=1e-12,
                                                                        atol=1e-15)
