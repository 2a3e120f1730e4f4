"""GPU checks of the learned preconditioner (gnn.cuh) and of flexible CG.

* forward: the preconditioner the training kernels (FP32 CUDA cores) build
  agrees with the CPU reference oracle/gnn_ref.py; the inference kernels
  (BF16 tensor cores) agree with the training kernels to BF16 accuracy;
* backward: the hand-written gradient kernels agree with torch autograd on
  the CPU reference;
* flexible CG: the untrained network (= the Jacobi step) reproduces PCG;
  any network converges to the FP64 oracle's solution (the FP64 residual
  decides); a broken network hands over to plain PCG;
* training lowers the loss and the FCG iteration count (the gain test).
"""
import os

import numpy as np
import pytest

from oracle import gnn_ref
from oracle.oracle import Oracle
from programs_b200 import learn
from programs_b200.mesh import Mesh, cavity_field, momentum_field, pressure_correction, uniform
from programs_b200.solver import OK

pytestmark = pytest.mark.gpu


def _system(n=10, seed=1, lid=1.0, jitter=0.2):
    m = Mesh.hex(n, jitter=jitter, seed=seed, permute=True)
    m.renumber(Mesh.RCM)
    M, _, _ = momentum_field(m, cavity_field(m, lid), u_lid=lid)
    return pressure_correction(m, M.pl, pin=1)


def _active_params(seed=1):
    p = learn.init_params(seed)
    rng = np.random.default_rng(seed)
    p[learn.P_WA:learn.P_WA + 32] = rng.normal(0, 0.3, 32).astype(np.float32)
    p[learn.P_WE:learn.P_WE + 32] = rng.normal(0, 0.3, 32).astype(np.float32)
    p[learn.P_BE] = 0.2
    for l in range(3):  # non-zero biases exercise every term
        o = learn.P_LAYER + l * learn.LAYER_SZ + 2 * 32 * 32
        p[o:o + 32] = rng.normal(0, 0.1, 32).astype(np.float32)
    return p


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.float64)).cuda()


def _rhs(A, seed):
    b = uniform(seed, A.n_cell)
    b -= b.mean()
    b[0] = 0.0
    return b


def test_forward_kernels_match_reference(gpu):
    A = _system(10)
    gpu.matrix_set(A)
    p = _active_params()
    gpu.gnn_set_params(p)
    r0, r = uniform(3, A.n_cell), uniform(4, A.n_cell)
    r0d, rd = _dev(r0), _dev(r)
    z0 = _dev(np.zeros(A.n_cell))
    z1 = _dev(np.zeros(A.n_cell))
    gpu.gnn_forward_dev(r0d.data_ptr(), rd.data_ptr(), z1.data_ptr(), path=1)
    gpu.gnn_forward_dev(r0d.data_ptr(), rd.data_ptr(), z0.data_ptr(), path=0)
    zc = gnn_ref.precondition(A, r0, r, p)
    z1, z0 = z1.cpu().numpy(), z0.cpu().numpy()
    assert _rel(z1, zc) < 2e-3          # FP32 vs FP64 sums; BF16 roundings at the same points
    assert _rel(z0, z1) < 2e-2          # tensor-core accumulation order vs CUDA cores


def test_gradient_kernels_match_autograd(gpu):
    import torch
    A = _system(8, seed=2)
    gpu.matrix_set(A)
    p = _active_params(3)
    gpu.gnn_set_params(p)
    r0 = uniform(5, A.n_cell)
    samples = [r0, uniform(6, A.n_cell), uniform(7, A.n_cell)]
    sd = torch.from_numpy(np.stack(samples)).cuda()
    r0d = _dev(r0)
    loss_g = gpu.gnn_grad_dev(r0d.data_ptr(), sd.data_ptr(), len(samples))
    g_g = gpu.gnn_get_grad()
    loss_c, g_c = gnn_ref.loss_and_grad(A, r0, samples, p)
    assert abs(loss_g - loss_c) <= 1e-3 * abs(loss_c)
    blocks = [("w_in", 0, learn.P_LAYER)]
    for l in range(3):
        o = learn.P_LAYER + l * learn.LAYER_SZ
        blocks += [(f"Ws{l}", o, o + 1024), (f"Wn{l}", o + 1024, o + 2048),
                   (f"b{l}", o + 2048, o + 2080)]
    blocks += [("w_a", learn.P_WA, learn.P_BA), ("b_a", learn.P_BA, learn.P_WE),
               ("w_e", learn.P_WE, learn.P_BE), ("b_e", learn.P_BE, learn.N_PARAM)]
    for name, a, b in blocks:
        assert _rel(g_g[a:b], g_c[a:b]) < 3e-2, name


def _solve_fcg(gpu, A, b):
    phi = np.zeros((A.n_cell, 1))
    res0 = np.asfortranarray(b.reshape(-1, 1).copy())
    rn = np.zeros(1)
    st = gpu.solv_fcg(1e-10, 20000, phi, res0, rn)
    return phi, st, rn


def test_untrained_network_reproduces_pcg(gpu):
    A = _system(12, seed=4)
    gpu.matrix_set(A)
    gpu.gnn_set_params(learn.init_params(0))
    b = _rhs(A, 6)
    phi, st, rn = _solve_fcg(gpu, A, b)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    assert st["status"] == OK and st["fallbacks"] == 0
    assert _rel(phi, ref[0]) <= 1e-8
    # FCG(1) with the fixed SPD Jacobi preconditioner is PCG; FP32 with
    # reliable updates may cost a few iterations
    assert st["iters"][0] <= 1.15 * int(ref[3][0])


def test_broken_network_falls_back_to_pcg(gpu):
    A = _system(10, seed=5)
    gpu.matrix_set(A)
    p = learn.init_params(0)
    p[learn.P_BA] = np.nan  # z = NaN: no curvature, FCG stalls at once
    gpu.gnn_set_params(p)
    b = _rhs(A, 7)
    phi, st, rn = _solve_fcg(gpu, A, b)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    assert st["status"] == OK and st["fallbacks"] >= 1
    assert _rel(phi, ref[0]) <= 1e-8


def test_training_gains_over_the_untrained_network(gpu):
    """A short training run lowers the energy loss and the FCG iteration
    count below the untrained network's (which is Jacobi-PCG)."""
    p0 = learn.init_params(0)
    p, hist = learn.train(size=12, n_mesh=4, per_mesh=12, samples=4, epochs=3, lr=3e-3, seed=0,
                          init=p0, log_every=0)
    assert np.mean(hist[-10:]) < np.mean(hist[:10])
    A = _system(14, seed=11, lid=0.7, jitter=0.12)
    gpu.matrix_set(A)
    b = _rhs(A, 8)
    gpu.gnn_set_params(p0)
    _, st0, _ = _solve_fcg(gpu, A, b)
    gpu.gnn_set_params(p)
    phi, st1, _ = _solve_fcg(gpu, A, b)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    assert _rel(phi, ref[0]) <= 1e-8
    assert st1["iters"][0] < 0.9 * st0["iters"][0], (st0["iters"], st1["iters"])


@pytest.mark.skipif(not os.path.exists(learn.DEFAULT_WEIGHTS), reason="no trained weights")
def test_committed_weights_solve_to_the_oracle_solution(gpu):
    A = _system(24, seed=21, lid=1.3, jitter=0.18)
    gpu.matrix_set(A)
    gpu.gnn_set_params(learn.load_params())
    b = _rhs(A, 9)
    phi, st, rn = _solve_fcg(gpu, A, b)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    assert st["status"] == OK
    assert _rel(phi, ref[0]) <= 1e-8
    S = A.to_scipy()
    assert np.abs(b - S @ phi[:, 0]).sum() / rn[0] < 1e-10
    assert st["iters"][0] < int(ref[3][0])  # fewer iterations than Jacobi-PCG
