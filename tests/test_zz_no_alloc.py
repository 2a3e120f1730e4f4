"""The no-allocation residual entry point against the context-based one.

solv_gpu_res_noalloc serves callers that cannot allocate device memory
(their memory pool belongs to another runtime, or a service forbids
allocation once running): it computes solv_res from device arrays the
caller already owns and keeps its reduction scratch in one fixed device
array inside the library.  Every call reuses that array, so two calls in a
row are checked; both must agree with solv_gpu_res, the entry point that
works through a context and its own workspace, within the rounding that
the different order of the face sums (atomic adds) allows.

This file is named to be collected last, so a run that stops at the first
failure has run every other test first; it also passes alone in a fresh
process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc():
    from programs_b200.solver import lib
    L = lib()
    vp = ctypes.c_void_p
    L.solv_gpu_res_noalloc.restype = ctypes.c_int
    L.solv_gpu_res_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int,
                                       vp, vp, vp, ctypes.c_int, vp]
    return L.solv_gpu_res_noalloc


def _system(kind):
    from programs_b200.mesh import Mesh
    m = Mesh.hex(12, jitter=0.15, seed=3)
    m.renumber(Mesh.RCM)
    return m.pressure(pin=1) if kind == "pressure" else m.momentum()[0]


@pytest.mark.parametrize("kind,V", [("pressure", 1), ("momentum", 3)])
@pytest.mark.parametrize("not_r0", [False, True])
def test_noalloc_matches_solv_gpu_res_on_two_calls(kind, V, not_r0):
    import torch
    from programs_b200.mesh import uniform
    from programs_b200.solver import GpuSolver
    A = _system(kind)
    N, F = A.n_cell, A.n_face
    dev = torch.device("cuda", 0)
    ip = torch.from_numpy(A.ip.astype(np.int32)).to(dev)
    inb = torch.from_numpy(A.inb.astype(np.int32)).to(dev)
    p = torch.from_numpy(A.p).to(dev)
    n = torch.from_numpy(A.n).to(dev)
    pl = torch.from_numpy(A.pl).to(dev)
    s = GpuSolver(0)
    s.matrix_set(A)
    fn = _noalloc()
    try:
        for call in range(2):
            phi = uniform(10 + call, N * V).reshape(N, V).copy()
            b = np.asfortranarray(uniform(20 + call, N * V).reshape(V, N).T)
            r_ref = b.copy(order="F")
            rn_ref = np.zeros(V)
            s.solv_res(phi, r_ref, rn_ref, not_r0)
            phi_d = torch.from_numpy(phi).to(dev)
            r_d = torch.from_numpy(np.ascontiguousarray(b.T)).to(dev)  # column-major res0
            rn_d = torch.full((V,), -1.0, dtype=torch.float64, device=dev)
            rc = fn(N, F, ip.data_ptr(), inb.data_ptr(), p.data_ptr(), n.data_ptr(), pl.data_ptr(),
                    V, phi_d.data_ptr(), r_d.data_ptr(), rn_d.data_ptr(), int(not_r0), None)
            assert rc == 0
            r = r_d.cpu().numpy().T
            rn = rn_d.cpu().numpy()
            scale = np.abs(b).max() + np.abs(phi).max() * np.abs(A.pl).max()
            assert np.allclose(r, r_ref, rtol=1e-12, atol=1e-13 * scale)
            assert np.allclose(rn, rn_ref, rtol=1e-12)
    finally:
        s.close()


def test_noalloc_rejects_what_it_cannot_hold():
    import torch
    A = _system("pressure")
    N, F = A.n_cell, A.n_face
    dev = torch.device("cuda", 0)
    ip = torch.from_numpy(A.ip.astype(np.int32)).to(dev)
    inb_bad = A.inb.astype(np.int32).copy()
    inb_bad[np.argmax(A.inb > 0)] = N + 7  # one face points past the last cell
    inb = torch.from_numpy(inb_bad).to(dev)
    p, n, pl = (torch.from_numpy(x).to(dev) for x in (A.p, A.n, A.pl))
    phi = torch.ones(N * 5, dtype=torch.float64, device=dev)
    r = torch.full((N * 5,), 2.0, dtype=torch.float64, device=dev)
    rn = torch.full((5,), 3.0, dtype=torch.float64, device=dev)
    fn = _noalloc()
    args = (ip.data_ptr(), inb.data_ptr(), p.data_ptr(), n.data_ptr(), pl.data_ptr())
    assert fn(N, F, *args, 5, phi.data_ptr(), r.data_ptr(), rn.data_ptr(), 0, None) == 9  # n_vc > 4
    assert fn(N, F, *args, 0, phi.data_ptr(), r.data_ptr(), rn.data_ptr(), 0, None) == 4  # n_vc < 1
    assert fn(N, F, *args, -1, phi.data_ptr(), r.data_ptr(), rn.data_ptr(), 0, None) == 4
    assert fn(N, F, *args, 1, phi.data_ptr(), r.data_ptr(), rn.data_ptr(), 0, None) == 4  # bad index
    # the bad index is found before anything is written
    assert bool((r == 2.0).all()) and bool((rn == 3.0).all())
    # and the scratch is left usable: a valid call right after succeeds
    inb_ok = torch.from_numpy(A.inb.astype(np.int32)).to(dev)
    args_ok = (ip.data_ptr(), inb_ok.data_ptr(), p.data_ptr(), n.data_ptr(), pl.data_ptr())
    assert fn(N, F, *args_ok, 1, phi.data_ptr(), r.data_ptr(), rn.data_ptr(), 0, None) == 0
    assert float(rn[0]) >= 0.0 and float(rn[0]) != 3.0
