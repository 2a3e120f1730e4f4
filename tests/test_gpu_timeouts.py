"""The bounded waits of the DIC/DILU recurrences (kernels.cuh: sweep_slices,
at most kSweepPolls polls each).  A wait that runs out must come back as a
status the host reads, SOLV_GPU_TIMEOUT, and leave the context usable: the
next sweep rebuilds its pending state and solves as before.  The wait is
made to run out without any fault: one cell waits on a value that nothing
ever writes (solv_gpu_selftest_sweep_wait)."""
import time

import numpy as np
import pytest

from oracle.oracle import Oracle
from programs_b200.mesh import Mesh, uniform
from programs_b200.solver import OK, TIMEOUT

pytestmark = pytest.mark.gpu


def test_a_sweep_wait_runs_out_and_the_context_stays_usable(gpu):
    m = Mesh.hex(10, seed=5)
    m.renumber(Mesh.RCM)
    A, _ = m.momentum()
    b = uniform(7, A.n_cell).reshape(-1, 1)
    ref = Oracle.from_matrix(A).solv_bicg(2, 1e-10, 500, np.zeros((A.n_cell, 1)), b)
    gpu.matrix_set(A)
    t = time.perf_counter()
    assert gpu.selftest_sweep_wait() == TIMEOUT
    assert time.perf_counter() - t < 30.0  # bounded, about a second
    for _ in range(2):  # the context and its sweeps work afterwards
        phi = np.zeros((A.n_cell, 1))
        res0 = np.asfortranarray(b.copy())
        st = gpu.solv_bicg(2, 1e-10, 500, phi, res0, np.zeros(1))
        assert st["status"] == OK
        assert np.array_equal(res0, ref[1])
        assert abs(st["iters"][0] - int(ref[3][0])) <= 2
        assert np.linalg.norm(phi - ref[0]) / np.linalg.norm(ref[0]) <= 1e-8
