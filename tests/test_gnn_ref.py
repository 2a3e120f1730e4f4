"""CPU checks of the learned preconditioner's reference implementation
(oracle/gnn_ref.py) and of the parameter layout shared with gnn.cuh."""
import os
import re

import numpy as np
import pytest

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


def test_layout_matches_cuda_header():
    src = open(os.path.join(ROOT, "programs_b200", "csrc", "gnn.cuh")).read()
    assert re.search(r"constexpr int H = 32;", src) and re.search(r"constexpr int NL = 3;", src)
    assert learn.N_PARAM == gnn_ref.N_PARAM == 128 + 3 * (2 * 32 * 32 + 32) + 33


def test_untrained_network_is_the_jacobi_step():
    A = _system()
    r = uniform(3, A.n_cell)
    z, _, _ = gnn_ref.forward(A, r, learn.init_params(0))
    assert np.allclose(z, r / A.pl, rtol=2e-6)


def test_bf16_rounding_is_round_to_nearest_even():
    import torch
    x = torch.tensor([1.0, 1.00390625, 1.01171875, -3.3, 1e-3], dtype=torch.float64)
    y = gnn_ref.bf16_round(x).numpy()
    assert y[0] == 1.0 and y[1] == 1.0 and y[2] == 1.015625  # ties to even
    assert abs(y[3] + 3.3) < 3.3 * 2 ** -8


def test_reference_gradient_matches_finite_differences():
    gnn_ref.ROUND = False
    try:
        A = _system(5, seed=2)
        r = uniform(4, A.n_cell)
        p = learn.init_params(1).astype(np.float64)
        rng = np.random.default_rng(0)
        p[learn.P_WOUT:learn.P_WOUT + 32] = rng.normal(0, 0.3, 32)  # open the correction path
        J0, g = gnn_ref.loss_and_grad(A, r, p)
        idx = rng.choice(learn.N_PARAM, 25, replace=False)
        for k in idx:
            e = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[k] += e
            pm[k] -= e
            fd = (float(gnn_ref.forward(A, r, pp)[1]) - float(gnn_ref.forward(A, r, pm)[1])) / (2 * e)
            assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(g[k])
    finally:
        gnn_ref.ROUND = True


def test_energy_loss_minimiser_is_the_solution():
    """J(out) = 1/2 out.Â out - out.u is minimised by out = Â^-1 u."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    A = _system(5, seed=3)
    rsd = 1.0 / np.sqrt(A.pl)
    S = sp.diags(rsd) @ A.to_scipy() @ sp.diags(rsd)
    u = uniform(5, A.n_cell)
    x = spla.spsolve(S.tocsc(), u)
    J = lambda o: 0.5 * o @ (S @ o) - o @ u
    for _ in range(5):
        d = np.random.default_rng(_).normal(size=A.n_cell) * 1e-3
        assert J(x + d) > J(x)
