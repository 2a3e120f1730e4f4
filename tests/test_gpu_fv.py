"""The SIMPLE outer-loop pieces on the GPU (fv_gpu.cu) against their host
restatement (fvmesh.cpp): momentum and pressure-correction assembly,
Green-Gauss gradient, Rhie-Chow fluxes, mass imbalance and corrections.
The GPU adds each cell's faces in ascending face order -- the order of the
reference's face loop -- without fused multiply-adds, so every array must
agree bit for bit; only the imbalance total (a tree sum) has a tolerance.
"""
import numpy as np
import pytest

from programs_b200 import mesh as M
from programs_b200.mesh import Mesh, cavity_field

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(built):
    import torch
    from programs_b200.fv import GpuFv
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    m = Mesh.hex(9, 8, 10, jitter=0.2, seed=5, permute=True)
    m.renumber(Mesh.RCM)
    fv = GpuFv(m)
    yield m, fv
    fv.close()


def _d(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float64)).cuda()


def _h(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("given_flux", [False, True])
def test_momentum_assembly_is_bit_exact(case, given_flux):
    m, fv = case
    u = cavity_field(m, 1.3) + 0.05 * M.uniform(3, 3 * m.n_cell).reshape(-1, 3)
    flux = 0.01 * M.uniform(4, m.n_face) if given_flux else None
    A, rhs, fo = M.momentum_field(m, u, flux=flux, rho=1.1, mu=2e-3, u_lid=1.3, urf=0.7)
    p, n, pl, rhs_d, fo_d = fv.momentum_field(_d(u), None if flux is None else _d(flux), rho=1.1,
                                              mu=2e-3, u_lid=1.3, urf=0.7)
    assert np.array_equal(_h(p), A.p) and np.array_equal(_h(n), A.n)
    assert np.array_equal(_h(pl), A.pl)
    assert np.array_equal(_h(rhs_d), rhs) and np.array_equal(_h(fo_d), fo)
    assert np.abs(rhs[:, 0]).max() > 0  # the lid term is exercised


@pytest.mark.parametrize("pin", [0, 1, 17])
def test_pressure_correction_assembly_is_bit_exact(case, pin):
    m, fv = case
    A, _, _ = M.momentum_field(m, cavity_field(m, 1.0))
    P = M.pressure_correction(m, A.pl, rho=1.2, pin=pin)
    p, n, pl = fv.pressure_correction(_d(A.pl), rho=1.2, pin=pin)
    assert np.array_equal(_h(p), P.p) and np.array_equal(_h(n), P.n)
    assert np.array_equal(_h(pl), P.pl)


@pytest.mark.parametrize("k", [1, 3])
def test_gradient_is_bit_exact(case, k):
    m, fv = case
    phi = M.uniform(7, m.n_cell * k).reshape(m.n_cell, k) if k > 1 else M.uniform(7, m.n_cell)
    assert np.array_equal(_h(fv.gradient(_d(phi))), M.gradient(m, phi))


def test_flux_imbalance_and_corrections_are_bit_exact(case):
    m, fv = case
    u = cavity_field(m, 1.0)
    A, _, _ = M.momentum_field(m, u)
    p = M.uniform(8, m.n_cell)
    gp = M.gradient(m, p)
    f_h = M.face_flux(m, u, p, gp, A.pl, rho=1.0)
    f_d = fv.face_flux(_d(u), _d(p), _d(gp), _d(A.pl), rho=1.0)
    assert np.array_equal(_h(f_d), f_h)
    b_h, t_h = M.mass_imbalance(m, f_h, pin=1)
    b_d, t_d = fv.mass_imbalance(f_d, pin=1)
    assert np.array_equal(_h(b_d), b_h)
    assert abs(t_d - t_h) <= 1e-12 * t_h
    pp = M.uniform(9, m.n_cell)
    gpp = M.gradient(m, pp)
    u_h, p_h, fl_h = u.copy(), p.copy(), f_h.copy()
    M.simple_correct(m, pp, gpp, A.pl, 1.0, 0.3, u_h, p_h, fl_h)
    u_d, p_d, fl_d = _d(u), _d(p), _d(f_h)
    fv.simple_correct(_d(pp), _d(gpp), _d(A.pl), 1.0, 0.3, u_d, p_d, fl_d)
    assert np.array_equal(_h(u_d), u_h) and np.array_equal(_h(p_d), p_h)
    assert np.array_equal(_h(fl_d), fl_h)


@pytest.mark.parametrize("n_iter", [1, 2, 3])
@pytest.mark.parametrize("neu", [0, 1, 2])
@pytest.mark.parametrize("k", [1, 3])
def test_gradient_sweeps_are_bit_exact(case, n_iter, neu, k):
    """solv_grad in full on the GPU (corrected sweeps, walls by neu)
    against fvm_gradient_sweeps."""
    m, fv = case
    phi = M.uniform(11, m.n_cell * k).reshape(m.n_cell, k) if k > 1 else M.uniform(11, m.n_cell)
    bval = M.uniform(12, m.n_face * k).reshape(m.n_face, k)
    g_h = M.gradient_sweeps(m, phi, n_iter, neu, bval if neu == 0 else None)
    g_d = fv.gradient_sweeps(_d(phi), n_iter, neu, _d(bval) if neu == 0 else None)
    assert np.array_equal(_h(g_d).reshape(g_h.shape), g_h)


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
@pytest.mark.parametrize("c_bl", [1.0, 0.7])
def test_momentum_deferred_is_bit_exact(case, scheme, c_bl):
    """The explicit momentum terms on the GPU against fvm_momentum_deferred,
    added to a right-hand side that is not zero."""
    m, fv = case
    u = cavity_field(m, 1.0) + 0.05 * M.uniform(13, 3 * m.n_cell).reshape(-1, 3)
    _, _, flux = M.momentum_field(m, u)
    assert (flux > 0).any() and (flux < 0).any()
    g = M.gradient_sweeps(m, u, 2, 1)
    rhs0 = M.uniform(14, 3 * m.n_cell).reshape(-1, 3)
    r_h = rhs0 + M.momentum_deferred(m, u, g, flux, 1e-3, c_bl, scheme)
    r_d = _d(rhs0)
    dcor = _d(np.zeros_like(rhs0))
    fv.momentum_deferred(_d(u), _d(g), _d(flux), 1e-3, dcor, c_bl=c_bl, scheme=scheme)
    r_d += dcor
    assert np.array_equal(_h(r_d), r_h)
    # accumulated straight into a right-hand side: the same terms, other rounding
    r_d2 = _d(rhs0)
    fv.momentum_deferred(_d(u), _d(g), _d(flux), 1e-3, r_d2, c_bl=c_bl, scheme=scheme)
    assert np.allclose(_h(r_d2), r_h, rtol=1e-12, atol=1e-15)


def test_face_flux_at_the_auxiliary_points_is_bit_exact(case):
    m, fv = case
    u = cavity_field(m, 1.0)
    A, _, _ = M.momentum_field(m, u)
    p = M.uniform(15, m.n_cell)
    gp = M.gradient_sweeps(m, p, 2, 2)
    f_h = M.face_flux(m, u, p, gp, A.pl, rho=1.0, aux=True)
    f_d = fv.face_flux(_d(u), _d(p), _d(gp), _d(A.pl), rho=1.0, aux=True)
    assert np.array_equal(_h(f_d), f_h)
    assert not np.array_equal(f_h, M.face_flux(m, u, p, gp, A.pl, rho=1.0))  # skewed mesh
