"""ctypes wrapper of the CPU oracle (``oracle/liborc.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``, as the oracle results are
compared with -- never by the product path.  Function names and argument meanings follow the Fortran
subroutines they restate (spray-simulation/solv_*.f90).  Parity of the
restatement is not pinned by the reference itself (no Fortran compiler, no
golden vectors); it is cross-checked in tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


class _OrcMatrix(ctypes.Structure):
    _fields_ = [("n_cell", ctypes.c_int), ("n_face", ctypes.c_int),
                ("ip", _i32p), ("in_", _i32p), ("p", _f64p), ("n", _f64p), ("pl", _f64p),
                ("v_ptr", _i32p), ("v_fce", _i32p), ("v_ng", _i32p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liborc.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.orc_vlst_size.restype = ctypes.c_int
        L.orc_vlst_size.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p]
        L.orc_build_vlst.restype = ctypes.c_int
        L.orc_build_vlst.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p, _i32p, _i32p]
        mp = ctypes.POINTER(_OrcMatrix)
        L.orc_solv_res.argtypes = [mp, ctypes.c_int, _f64p, _f64p, _f64p, ctypes.c_int]
        L.orc_solv_precond.argtypes = [mp, ctypes.c_int, _f64p, _f64p]
        L.orc_solv_direct.argtypes = [mp, ctypes.c_int, _f64p, _f64p, _f64p, _f64p]
        L.orc_spmv.argtypes = [mp, _f64p, _f64p]
        for fn in (L.orc_solv_cg, L.orc_solv_bicg):
            fn.argtypes = [mp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _f64p,
                           _f64p, _f64p, ctypes.c_int, _i32p, _f64p]
        for fn in (L.csr_cg_solver, L.csr_bicg_solver):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, ctypes.c_int,
                           ctypes.c_double]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


class Oracle:
    """The matrix of solv_data.f90 plus the restated subroutines."""

    def __init__(self, n_cell, ip, inb, p, n, pl):
        L = lib()
        self.N = int(n_cell)
        self.ip = np.ascontiguousarray(ip, np.int32)
        self.inb = np.ascontiguousarray(inb, np.int32)
        self.p = np.ascontiguousarray(p, np.float64)
        self.n = np.ascontiguousarray(n, np.float64)
        self.pl = np.ascontiguousarray(pl, np.float64)
        F = self.ip.shape[0]
        size = L.orc_vlst_size(self.N, F, _p(self.ip, _i32p), _p(self.inb, _i32p))
        if size < 0:
            raise ValueError("face index out of range")
        self.v_ptr = np.zeros(self.N + 1, np.int32)
        self.v_fce = np.zeros(max(size, 1), np.int32)
        self.v_ng = np.zeros(max(size, 1), np.int32)
        L.orc_build_vlst(self.N, F, _p(self.ip, _i32p), _p(self.inb, _i32p),
                         _p(self.v_ptr, _i32p), _p(self.v_fce, _i32p), _p(self.v_ng, _i32p))
        self._m = _OrcMatrix(self.N, F, _p(self.ip, _i32p), _p(self.inb, _i32p),
                             _p(self.p, _f64p), _p(self.n, _f64p), _p(self.pl, _f64p),
                             _p(self.v_ptr, _i32p), _p(self.v_fce, _i32p), _p(self.v_ng, _i32p))

    @classmethod
    def from_matrix(cls, m):
        return cls(m.n_cell, m.ip, m.inb, m.p, m.n, m.pl)

    def solv_res(self, phi, res0, not_r0=False):
        """phi (N,V) cell-major, res0 (N,V) as Fortran res0(ip,ivc); both copied."""
        phi = np.ascontiguousarray(phi, np.float64).reshape(self.N, -1)
        V = phi.shape[1]
        r = np.asfortranarray(np.array(res0, np.float64).reshape(self.N, V))
        rn = np.zeros(V)
        lib().orc_solv_res(ctypes.byref(self._m), V, _p(phi, _f64p), _p(r, _f64p),
                           _p(rn, _f64p), int(bool(not_r0)))
        return r, rn

    def solv_precond(self, imat):
        c = np.empty(self.N)
        c_r = np.empty(self.N)
        lib().orc_solv_precond(ctypes.byref(self._m), imat, _p(c, _f64p), _p(c_r, _f64p))
        return c, c_r

    def solv_direct(self, imat, c, c_r, b):
        x = np.zeros(self.N)
        c = np.ascontiguousarray(c, np.float64)
        c_r = np.ascontiguousarray(c_r, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        lib().orc_solv_direct(ctypes.byref(self._m), imat, _p(c, _f64p), _p(c_r, _f64p),
                              _p(x, _f64p), _p(b, _f64p))
        return x

    def spmv(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.N)
        lib().orc_spmv(ctypes.byref(self._m), _p(x, _f64p), _p(y, _f64p))
        return y

    def _solve(self, fn, imat, reduc, n_iter, phi, res0, not_r0):
        phi = np.array(phi, np.float64).reshape(self.N, -1)
        V = phi.shape[1]
        r = np.asfortranarray(np.array(res0, np.float64).reshape(self.N, V))
        rn = np.zeros(V)
        iters = np.zeros(V, np.int32)
        ratio = np.zeros(V)
        fn(ctypes.byref(self._m), imat, reduc, n_iter, V, _p(phi, _f64p), _p(r, _f64p),
           _p(rn, _f64p), int(bool(not_r0)), _p(iters, _i32p), _p(ratio, _f64p))
        return phi, r, rn, iters, ratio

    def solv_cg(self, imat, reduc, n_iter, phi, res0, not_r0=False):
        """Returns phi, res0 (initial residual), res0_n, iterations, last ratio."""
        return self._solve(lib().orc_solv_cg, imat, reduc, n_iter, phi, res0, not_r0)

    def solv_bicg(self, imat, reduc, n_iter, phi, res0, not_r0=False):
        return self._solve(lib().orc_solv_bicg, imat, reduc, n_iter, phi, res0, not_r0)


def csr_solve(A, b, phi0=None, kind="cg", n_iter=1000, reduc=1e-10):
    """pcns/src/solv_m.f90 twin on a scipy CSR matrix (1 RHS, DILU)."""
    import scipy.sparse as sp
    A = sp.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    ia = (A.indptr + 1).astype(np.int32)
    ja = (A.indices + 1).astype(np.int32)
    a = A.data.astype(np.float64).copy()
    phi = np.zeros(n) if phi0 is None else np.array(phi0, np.float64)
    res = np.array(b, np.float64)
    norm = ctypes.c_double()
    fn = lib().csr_cg_solver if kind == "cg" else lib().csr_bicg_solver
    it = fn(n, _p(ia, _i32p), _p(ja, _i32p), _p(a, _f64p), _p(phi, _f64p), _p(res, _f64p),
            ctypes.byref(norm), n_iter, reduc)
    return phi, it
