"""The multigrid hierarchy's aggregation rule (host code in mg.cuh, called
through the C-ABI without a GPU): about 2^passes cells per aggregate, every
aggregate connected in the coupling graph, no cell left alone where it has
a neighbour, deterministic."""
import numpy as np
import pytest

from programs_b200.mesh import Mesh


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def _graph(n=14, seed=2):
    m = Mesh.hex(n, jitter=0.2, seed=seed, permute=True)
    m.renumber(Mesh.RCM)
    A = m.pressure(pin=0)
    S = A.to_scipy().tocsr()
    S.setdiag(0)
    S.eliminate_zeros()
    return S.indptr.astype(np.int64), S.indices.astype(np.int32), np.abs(S.data).astype(np.float32)


def test_aggregates_are_connected_and_about_eight_cells():
    from programs_b200.solver import mg_aggregate
    ptr, adj, w = _graph()
    n = len(ptr) - 1
    agg, na = mg_aggregate(ptr, adj, w, 3)
    assert agg.min() == 0 and agg.max() == na - 1
    size = np.bincount(agg, minlength=na)
    assert size.min() >= 2                 # no cell alone: every cell has a neighbour
    assert 6.5 <= n / na <= 9.0            # three pairwise passes: about 8 cells each
    assert size.max() <= 16
    # each aggregate is connected through the graph's edges
    for a in range(0, na, max(1, na // 200)):
        cells = set(np.nonzero(agg == a)[0].tolist())
        seen, todo = {min(cells)}, [min(cells)]
        while todo:
            i = todo.pop()
            for j in adj[ptr[i]:ptr[i + 1]]:
                if j in cells and j not in seen:
                    seen.add(int(j))
                    todo.append(int(j))
        assert seen == cells, a
    agg2, na2 = mg_aggregate(ptr, adj, w, 3)
    assert na2 == na and np.array_equal(agg2, agg)


def test_one_pass_is_a_matching_and_bad_graphs_are_rejected():
    from programs_b200.solver import SolverError, mg_aggregate
    ptr, adj, w = _graph(8)
    agg, na = mg_aggregate(ptr, adj, w, 1)
    assert np.bincount(agg).max() <= 3     # pairs, plus cells joined afterwards
    bad = adj.copy()
    bad[0] = len(ptr) + 5
    with pytest.raises(SolverError):
        mg_aggregate(ptr, bad, w, 3)


def test_isolated_cells_stay_alone_and_components_never_mix():
    """A cell without neighbours (a row with its diagonal only) is its own
    aggregate; two disconnected systems share no aggregate."""
    import scipy.sparse as sp
    from programs_b200.solver import mg_aggregate
    A = Mesh.hex(6, jitter=0.2, seed=1).pressure(pin=0).to_scipy()
    n1 = A.shape[0]
    S = sp.block_diag([A, A, sp.identity(5)]).tocsr()
    S.setdiag(0)
    S.eliminate_zeros()
    agg, na = mg_aggregate(S.indptr.astype(np.int64), S.indices.astype(np.int32),
                           np.abs(S.data).astype(np.float32), 3)
    size = np.bincount(agg, minlength=na)
    assert np.all(size[agg[-5:]] == 1) and len(set(agg[-5:].tolist())) == 5
    assert not set(agg[:n1].tolist()) & set(agg[n1:2 * n1].tolist())
    assert size[np.unique(agg[:2 * n1])].min() >= 2
    ptr = np.arange(8, dtype=np.int64) * 0
    agg, na = mg_aggregate(ptr, np.zeros(0, np.int32), np.zeros(0, np.float32), 3)
    assert na == 7 and np.array_equal(agg, np.arange(7))


def test_self_loops_change_nothing():
    """A graph that keeps the matrix diagonal (every row its own neighbour)
    aggregates exactly as the graph without it."""
    from programs_b200.solver import mg_aggregate
    A = Mesh.hex(5, jitter=0.2, seed=1).pressure(pin=0).to_scipy().tocsr()
    S = A.copy()
    S.data = np.abs(S.data)
    T = A.copy()
    T.setdiag(0)
    T.eliminate_zeros()
    T.data = np.abs(T.data)
    got = [mg_aggregate(M.indptr.astype(np.int64), M.indices.astype(np.int32),
                        M.data.astype(np.float32), 3) for M in (S, T)]
    assert got[0][1] == got[1][1] and np.array_equal(got[0][0], got[1][0])
