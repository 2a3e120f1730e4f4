"""CPU checks of the learned preconditioner's reference implementation
(oracle/gnn_ref.py) and of the parameter layout shared with gnn.cuh."""
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle import gnn_ref
from programs_b200 import learn
from programs_b200.mesh import Mesh, cavity_field, momentum_field, pressure_correction, uniform

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def _system(n=6, seed=1):
    m = Mesh.hex(n, jitter=0.2, seed=seed)
    m.renumber(Mesh.RCM)
    M, _, _ = momentum_field(m, cavity_field(m, 1.0), u_lid=1.0)
    return pressure_correction(m, M.pl, pin=1)


def _active(seed=1):
    p = learn.init_params(seed).astype(np.float64)
    rng = np.random.default_rng(seed)
    p[learn.P_WA:learn.P_WA + 32] = rng.normal(0, 0.3, 32)
    p[learn.P_WE:learn.P_WE + 32] = rng.normal(0, 0.3, 32)
    p[learn.P_BE] = 0.2
    return p


def test_layout_matches_cuda_header():
    src = open(os.path.join(ROOT, "programs_b200", "csrc", "gnn.cuh")).read()
    assert re.search(r"constexpr int H = 32;", src) and re.search(r"constexpr int NL = 3;", src)
    assert re.search(r"kGamma = 0\.95f", src) and gnn_ref.GAMMA == 0.95
    assert learn.N_PARAM == gnn_ref.N_PARAM == 128 + 3 * (2 * 32 * 32 + 32) + 66
    assert (learn.P_WA, learn.P_BA, learn.P_WE, learn.P_BE) == (
        gnn_ref.P_WA, gnn_ref.P_BA, gnn_ref.P_WE, gnn_ref.P_BE)


def test_untrained_network_is_the_jacobi_step():
    A = _system()
    r = uniform(3, A.n_cell)
    z = gnn_ref.precondition(A, r, r, learn.init_params(0))
    assert np.allclose(z, r.astype(np.float32) / A.pl, rtol=1e-6)


def test_preconditioner_is_symmetric_positive_definite():
    A = _system(5, seed=2)
    p = _active(4)
    N = A.n_cell
    r0 = uniform(1, N)
    M = np.stack([gnn_ref.precondition(A, r0, e, p) for e in np.eye(N)], axis=1)
    assert np.allclose(M, M.T, rtol=1e-6, atol=1e-9)
    assert np.linalg.eigvalsh(0.5 * (M + M.T)).min() > 0


def test_bf16_rounding_is_round_to_nearest_even():
    import torch
    x = torch.tensor([1.0, 1.00390625, 1.01171875, -3.3, 1e-3], dtype=torch.float64)
    y = gnn_ref.bf16_round(x).numpy()
    assert y[0] == 1.0 and y[1] == 1.0 and y[2] == 1.015625  # ties to even
    assert abs(y[3] + 3.3) < 3.3 * 2 ** -8


@pytest.mark.parametrize("kind", [0, 1])
def test_reference_gradient_matches_finite_differences(kind):
    gnn_ref.ROUND = False
    try:
        A = _system(5, seed=2)
        r0 = uniform(4, A.n_cell)
        samples = [r0, uniform(5, A.n_cell)]
        p = _active(1)
        J0, g = gnn_ref.loss_and_grad(A, r0, samples, p, kind=kind)
        rng = np.random.default_rng(0)
        idx = np.concatenate([rng.choice(learn.N_PARAM, 20, replace=False),
                              [learn.P_BA, learn.P_BE, learn.P_WA, learn.P_WE + 3]])
        for k in idx:
            e = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[k] += e
            pm[k] -= e
            fd = (float(gnn_ref.loss(A, r0, samples, pp, kind=kind)[0]) -
                  float(gnn_ref.loss(A, r0, samples, pm, kind=kind)[0])) / (2 * e)
            assert abs(fd - g[k]) <= 1e-7 + 1e-4 * abs(g[k]), k
    finally:
        gnn_ref.ROUND = True


def test_energy_loss_minimiser_is_the_solution():
    """J(z) = 1/2 z.Â z - z.u is minimised by z = Â^-1 u."""
    import scipy.sparse.linalg as spla
    A = _system(5, seed=3)
    rsd = 1.0 / np.sqrt(A.pl)
    S = sp.diags(rsd) @ A.to_scipy() @ sp.diags(rsd)
    u = uniform(5, A.n_cell)
    x = spla.spsolve(S.tocsc(), u)
    J = lambda o: 0.5 * o @ (S @ o) - o @ u
    for k in range(5):
        d = np.random.default_rng(k).normal(size=A.n_cell) * 1e-3
        assert J(x + d) > J(x)


def test_scale_free_loss_ignores_the_scale_of_z():
    """L(z) = -(z.u)^2/(z.Â z) is twice the energy after the best step along
    z: the same for every multiple of z, at most twice the energy of z, and
    minimal (-u.Â^-1 u) at z = Â^-1 u."""
    import scipy.sparse.linalg as spla
    A = _system(5, seed=3)
    rsd = 1.0 / np.sqrt(A.pl)
    S = sp.diags(rsd) @ A.to_scipy() @ sp.diags(rsd)
    u = uniform(6, A.n_cell)
    L = lambda z: -(z @ u) ** 2 / (z @ (S @ z))
    E = lambda z: 0.5 * z @ (S @ z) - z @ u
    z = u * np.random.default_rng(1).uniform(0.5, 2.0, A.n_cell)
    assert abs(L(3.7 * z) - L(z)) <= 1e-12 * abs(L(z))
    assert 0.5 * L(z) <= E(z) + 1e-12 * abs(E(z))
    x = spla.spsolve(S.tocsc(), u)
    assert abs(L(x) - 2 * E(x)) <= 1e-9 * abs(E(x))


def _aggs(A):
    """A two-level aggregation of consecutive cell indices (the reference's
    V-cycle takes any aggregation; the GPU's own comes from its API)."""
    a = np.arange(A.n_cell) // 8
    return [a]


def test_reference_vcycle_is_symmetric_and_untrained_is_jacobi_smoothing():
    A = _system(5, seed=4)
    mats, Ps = gnn_ref.hierarchy(A, _aggs(A))
    p0 = learn.init_params(0)
    s, gE, rows_t, cols_t, wt, P, rsd = gnn_ref.build(A, uniform(1, A.n_cell), p0)
    rsd_t = torch.tensor(rsd, dtype=torch.float64)
    K = lambda v: rsd_t * gnn_ref._apply(s, gE, rows_t, cols_t, rsd_t * v)
    D = torch.tensor(1.0 / A.pl)
    x = torch.tensor(uniform(2, A.n_cell))
    y = torch.tensor(uniform(3, A.n_cell))
    assert torch.allclose(K(x), D * x, rtol=1e-6)  # untrained network = Jacobi (FP32 rsd)
    Vx = gnn_ref.vcycle(mats, Ps, x, K, 0.8, 2.0)
    Vy = gnn_ref.vcycle(mats, Ps, y, K, 0.8, 2.0)
    assert abs(float(Vx @ y - x @ Vy)) <= 1e-10 * abs(float(Vx @ y))


def test_reference_vcycle_gradient_matches_finite_differences():
    gnn_ref.ROUND = False
    try:
        A = _system(5, seed=2)
        r0 = uniform(4, A.n_cell)
        samples = [r0, uniform(5, A.n_cell)]
        p = _active(1)
        aggs = _aggs(A)
        J0, g = gnn_ref.loss_mg_and_grad(A, r0, samples, p, aggs, 0.8, 2.0)
        rng = np.random.default_rng(1)
        idx = np.concatenate([rng.choice(learn.N_PARAM, 12, replace=False),
                              [learn.P_BA, learn.P_BE, learn.P_WA + 1, learn.P_WE + 2]])
        for k in idx:
            e = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[k] += e
            pm[k] -= e
            fd = (float(gnn_ref.loss_mg(A, r0, samples, pp, aggs, 0.8, 2.0)[0]) -
                  float(gnn_ref.loss_mg(A, r0, samples, pm, aggs, 0.8, 2.0)[0])) / (2 * e)
            assert abs(fd - g[k]) <= 1e-7 + 1e-4 * abs(g[k]), k
    finally:
        gnn_ref.ROUND = True


def test_shipped_weights_load_and_record_their_training(tmp_path):
    """The committed network: the library's layout, finite, not the untrained
    Jacobi network, trained on 2,000 pressure systems of 64^3 meshes; a file
    of another layout is refused rather than misread."""
    import json
    p = learn.load_params()
    assert p.shape == (learn.N_PARAM,) and p.dtype == np.float32 and np.all(np.isfinite(p))
    assert np.any(p[learn.P_WE:learn.P_WE + 32] != 0)    # face heads trained away from zero
    meta = json.loads(str(np.load(learn.DEFAULT_WEIGHTS)["meta"]))
    assert meta["size"] == 64 and meta["systems"] == 2000
    bad = str(tmp_path / "bad.npz")
    np.savez(bad, params=p[:-1], n_param=learn.N_PARAM - 1, layout=learn.LAYOUT, meta="{}")
    with pytest.raises(ValueError):
        learn.load_params(bad)


def test_training_systems_are_seeded_symmetric_pinned_pressure_corrections():
    """The generator behind the shipped network's training data: per mesh
    (jitter drawn in [0, 0.25]) several flow states; every system is the
    symmetric pressure-correction matrix with cell 1 pinned, driven by a
    uniform right-hand side with its mean removed and zero at the pinned
    cell, and the same seed gives the same systems."""
    def draw():
        return [(P.p.copy(), P.n.copy(), P.pl.copy(), b.copy())
                for _, P, b in learn.simple_systems(5, n_mesh=3, per_mesh=2, seed=4)]
    first, again = draw(), draw()
    assert len(first) == 6
    for (p, n, pl, b), (p2, n2, pl2, b2) in zip(first, again):
        assert np.array_equal(p, p2) and np.array_equal(pl, pl2) and np.array_equal(b, b2)
        assert np.array_equal(p, n) and np.all(p <= 0)
        assert np.all(pl > 0) and b[0] == 0.0 and np.all(np.abs(b) <= 2.0)
    # different flow states on one mesh give different coefficients
    assert not np.array_equal(first[0][2], first[1][2])
