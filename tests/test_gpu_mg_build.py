"""The aggregation hierarchy built on the GPU (programs_b200/csrc/mg_build.cuh).

* every level's aggregation covers all aggregates 0..nc-1, each aggregate is
  connected in the finer level's face graph (pairs of neighbours, joined
  singletons), and every level coarsens at least twofold;
* the build is deterministic: a second build of the same structure gives the
  same aggregations;
* the V-cycle over it preconditions as well as the host build's (sequential
  greedy matching): iteration counts of the Jacobi-smoothed multigrid FCG
  within 25% of each other, both converging to the oracle's solution.
(three passes of pairing aim at eightfold)
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

from oracle.oracle import Oracle
from programs_b200 import learn
from programs_b200.mesh import Mesh, poisson_rhs
from programs_b200.solver import (OK, OPT_MG_BUILD, OPT_MG_SMOOTHER, OPT_PRECISION, SolverError)

pytestmark = pytest.mark.gpu


def _system(n, seed=3):
    m = Mesh.hex(n, jitter=0.15, seed=seed, permute=True)
    m.renumber(Mesh.RCM)
    return m.pressure(pin=1)


def _levels(gpu, n0):
    aggs, n = [], n0
    while True:
        try:
            agg, nc = gpu.mg_aggregates(len(aggs) + 1, n)
        except SolverError:
            return aggs
        aggs.append((agg, nc))
        n = nc


def _graph(A):
    m = A.inb > 0
    a, b = A.ip[m] - 1, A.inb[m] - 1
    G = sp.coo_matrix((np.ones(a.size), (a, b)), shape=(A.n_cell, A.n_cell))
    return (G + G.T).tocsr()


def test_gpu_hierarchy_is_a_connected_aggregation(gpu):
    A = _system(24)
    gpu.matrix_set(A)
    gpu.set_option(OPT_MG_BUILD, 0)
    levels = _levels(gpu, A.n_cell)
    assert len(levels) >= 2 and levels[-1][1] <= 256
    G = _graph(A)
    for agg, nc in levels:
        assert agg.min() == 0 and agg.max() == nc - 1
        assert np.bincount(agg, minlength=nc).min() >= 1
        assert nc * 2 <= G.shape[0]
        # each aggregate is connected in the finer level's graph
        rows, cols = G.nonzero()
        same = agg[rows] == agg[cols]
        H = sp.coo_matrix((np.ones(same.sum()), (rows[same], cols[same])), shape=G.shape)
        n_comp, _ = connected_components(H, directed=False)
        assert n_comp == nc
        # the next finer graph: aggregates coupled where their members are
        P = sp.coo_matrix((np.ones(agg.size), (np.arange(agg.size), agg)), shape=(agg.size, nc))
        G = (P.T @ G @ P).tocsr()
        G.setdiag(0)
        G.eliminate_zeros()


def test_gpu_hierarchy_is_deterministic(gpu):
    A = _system(20, seed=4)
    gpu.set_option(OPT_MG_BUILD, 0)
    gpu.matrix_set(A)
    first = _levels(gpu, A.n_cell)
    gpu.matrix_set(A)
    second = _levels(gpu, A.n_cell)
    assert len(first) == len(second)
    for (a1, n1), (a2, n2) in zip(first, second):
        assert n1 == n2 and np.array_equal(a1, a2)


def test_gpu_and_host_builds_precondition_alike(gpu):
    A = _system(32, seed=5)
    b = poisson_rhs(A.n_cell, 6)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-10, 20000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    gpu.gnn_set_params(learn.init_params(0))
    gpu.set_option(OPT_MG_SMOOTHER, 0)
    its = {}
    try:
        for build in (0, 1):
            gpu.set_option(OPT_MG_BUILD, build)
            gpu.matrix_set(A)
            phi = np.zeros((A.n_cell, 1))
            res0 = np.asfortranarray(b.reshape(-1, 1).copy())
            st = gpu.solv_fcg(1e-10, 20000, phi, res0, np.zeros(1))
            assert st["status"] == OK and st["fallbacks"] == 0 and st["mg_levels"] >= 2
            rel = np.linalg.norm(phi - ref[0]) / np.linalg.norm(ref[0])
            assert rel <= 1e-7
            its[build] = st["iters"][0]
    finally:
        gpu.set_option(OPT_MG_BUILD, 0)
        gpu.set_option(OPT_MG_SMOOTHER, 1)
        gpu.set_option(OPT_PRECISION, 0)
    assert abs(its[0] - its[1]) <= 0.25 * its[1] + 2, its


def _hub_system(per_hub=250, seed=7):
    """Two strongly coupled hub cells, each with per_hub neighbours; every
    neighbour has a private, strongly coupled partner and the partners form a
    weak chain.  The first matching pass pairs the hubs and each neighbour
    with its partner, so the hubs' aggregate touches 2 x per_hub others: a
    pass graph (and a coarse level) whose row is wider than the 255 slots of
    the slice format."""
    from programs_b200.mesh import FaceMatrix
    rng = np.random.default_rng(seed)
    L = 2 * per_hub
    leaf = 2 + np.arange(L)
    part = 2 + L + np.arange(L)
    a = [np.array([0]), np.where(np.arange(L) < per_hub, 0, 1), leaf, part[:-1]]
    b = [np.array([1]), leaf, part, part[1:]]
    w = [np.array([50.0]), rng.uniform(0.5, 1.0, L), rng.uniform(20.0, 30.0, L),
         rng.uniform(0.1, 0.2, L - 1)]
    ip, inb, wf = (np.concatenate(x) for x in (a, b, w))
    N = 2 + 2 * L
    diag = np.bincount(ip, wf, N) + np.bincount(inb, wf, N) + 1.0
    return FaceMatrix(N, (ip + 1).astype(np.int32), (inb + 1).astype(np.int32), -wf, -wf.copy(),
                      diag)


@pytest.mark.parametrize("build", [0, 1])
def test_too_dense_a_coarse_row_means_one_level(gpu, build):
    """Where coarsening meets a row wider than the slice format holds, the
    flexible CG still returns a solution, not an error: the GPU build gives
    the hierarchy up and runs the one-level preconditioner (the host build's
    sequential matching finds a coarse level that fits)."""
    A = _hub_system()
    b = poisson_rhs(A.n_cell, 9)
    ref = Oracle.from_matrix(A).solv_cg(0, 1e-12, 20000, np.zeros((A.n_cell, 1)), b.reshape(-1, 1))
    gpu.gnn_set_params(learn.init_params(0))
    gpu.set_option(OPT_MG_BUILD, build)
    try:
        gpu.matrix_set(A)
        phi = np.zeros((A.n_cell, 1))
        st = gpu.solv_fcg(1e-12, 20000, phi, np.asfortranarray(b.reshape(-1, 1).copy()), np.zeros(1))
    finally:
        gpu.set_option(OPT_MG_BUILD, 0)
    assert st["status"] == OK
    if build == 0:
        assert st["mg_levels"] == 0
    assert np.linalg.norm(phi - ref[0]) / np.linalg.norm(ref[0]) <= 1e-8
