"""Python mirror of the spray-simulation solver subroutines on the C-ABI of
``libsolv_gpu.so`` (include/solv_gpu.h).

The reference keeps the matrix in module globals (solv_data.f90:10-22) and
exposes

    solv_cg(imat, reduc, n_iter, phi, res0, res0_n, not_r0)     solv_cg.f90:7
    solv_bicg(imat, reduc, n_iter, phi, res0, res0_n, not_r0)   solv_bicg.f90:7
    solv_res(phi, res0, res0_n, not_r0)                         solv_res.f90:5
    solv_precond(imat, c, c_r)                                  solv_precond.f90:5
    solv_direct(imat, c, c_r, x, b)                             solv_direct.f90:5

:class:`GpuSolver` holds one device context with the matrix resident in
HBM and offers the same calls.  ``phi`` is (n_cell, n_vc) cell-major like
``phi(ip)%vc``; ``res0`` is (n_cell, n_vc) like Fortran ``res0(ip,ivc)``
(passed column-major to the library).  Arrays are updated in place, as the
Fortran ``intent(inout)`` arguments are.  There is no CPU fallback: without
a GPU or the built library every call raises.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import load

OK, MAXITER, NAN, BAD_INPUT, DEVICE_ERROR, NO_MATRIX, ZERO_RHS = 0, 1, 3, 4, 5, 7, 8
TIMEOUT = 6
MAX_VC = 4
OPT_PRECISION, OPT_INNER_REDUC, OPT_GRAPH_ITERS, OPT_BLOCK, OPT_GRID_PER_SM, OPT_MAX_REFINE = (
    1, 2, 3, 4, 5, 6)
OPT_INNER_MAX_ITER, OPT_RELIABLE_DELTA, OPT_GNN_LOSS = 7, 8, 9
OPT_MG_LEVELS, OPT_MG_SMOOTHER, OPT_MG_OMEGA, OPT_MG_ALPHA = 10, 11, 12, 13
OPT_FCG_STALL_ITERS, OPT_FCG_STALL_DROP, OPT_MG_SCALE_MIN, OPT_MG_BUILD = 14, 15, 16, 17
OPT_VECTOR_WIDTH, OPT_PERSISTENT, OPT_FCG_RELIABLE_DELTA, OPT_GRAPH_LOOP = 18, 19, 20, 21
OPT_FCG_FALLBACK, OPT_FCG_SLOW_ITERS = 22, 23

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


class Stats(ctypes.Structure):
    _fields_ = [("n_vc", ctypes.c_int), ("iters", ctypes.c_int * MAX_VC),
                ("ratio", ctypes.c_double * MAX_VC), ("status", ctypes.c_int),
                ("n_levels", ctypes.c_int), ("refinements", ctypes.c_int),
                ("graph_launches", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("solve_ms", ctypes.c_double), ("fallbacks", ctypes.c_int),
                ("mg_levels", ctypes.c_int), ("smoother_switches", ctypes.c_int)]

    def as_dict(self):
        V = self.n_vc
        return {"iters": list(self.iters[:V]), "ratio": list(self.ratio[:V]),
                "status": self.status, "n_levels": self.n_levels,
                "refinements": self.refinements, "graph_launches": self.graph_launches,
                "kernel_launches": self.kernel_launches, "solve_ms": self.solve_ms,
                "fallbacks": self.fallbacks, "mg_levels": self.mg_levels,
                "smoother_switches": self.smoother_switches}


class Tune(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int), ("grid_per_sm", ctypes.c_int),
                ("graph_iters", ctypes.c_int), ("candidates", ctypes.c_int),
                ("ms_per_iter", ctypes.c_double), ("vector_width", ctypes.c_int),
                ("ms_per_iter_before", ctypes.c_double)]


# Exported symbols of include/solv_gpu.h (the tests check them all).
EXPORTS = [
    "solv_gpu_create", "solv_gpu_destroy", "solv_gpu_set_stream", "solv_gpu_set_option",
    "solv_gpu_status_string", "solv_gpu_last_error", "solv_gpu_matrix_set",
    "solv_gpu_matrix_values", "solv_gpu_matrix_values_dev", "solv_gpu_matrix_levels",
    "solv_gpu_res", "solv_gpu_precond", "solv_gpu_direct", "solv_gpu_spmv", "solv_gpu_cg",
    "solv_gpu_bicg", "solv_gpu_cg_dev", "solv_gpu_bicg_dev", "solv_gpu_spmv_dev",
    "solv_gpu_matrix_set_batch", "solv_gpu_n_systems", "solv_gpu_cg_batch", "solv_gpu_bicg_batch",
    "solv_gpu_cg_batch_dev", "solv_gpu_bicg_batch_dev", "solv_gpu_autotune",
    "solv_gpu_fcg", "solv_gpu_fcg_dev", "solv_gpu_gnn_n_params", "solv_gpu_gnn_set_params",
    "solv_gpu_gnn_get_params", "solv_gpu_gnn_forward_dev", "solv_gpu_gnn_grad_dev",
    "solv_gpu_gnn_get_grad", "solv_gpu_gnn_zero_grad", "solv_gpu_gnn_adam",
    "solv_gpu_kernel_time", "solv_gpu_selftest_sweep_wait", "solv_gpu_mg_aggregates",
    "solv_gpu_mg_aggregate",
    "solv_gpu_create_", "solv_gpu_destroy_", "solv_gpu_matrix_set_", "solv_gpu_matrix_values_",
    "solv_gpu_res_", "solv_gpu_precond_", "solv_gpu_direct_", "solv_gpu_cg_", "solv_gpu_bicg_",
]


def lib():
    L = load("libsolv_gpu.so")
    if getattr(L, "_typed", False):
        return L
    vp = ctypes.c_void_p
    L.solv_gpu_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int]
    L.solv_gpu_destroy.argtypes = [vp]
    L.solv_gpu_set_stream.argtypes = [vp, vp]
    L.solv_gpu_set_option.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.solv_gpu_status_string.restype = ctypes.c_char_p
    L.solv_gpu_status_string.argtypes = [ctypes.c_int]
    L.solv_gpu_last_error.restype = ctypes.c_char_p
    L.solv_gpu_last_error.argtypes = [vp]
    L.solv_gpu_matrix_set.argtypes = [vp, ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
    L.solv_gpu_matrix_values.argtypes = [vp, _f64p, _f64p, _f64p]
    L.solv_gpu_matrix_values_dev.argtypes = [vp, vp, vp, vp]
    L.solv_gpu_matrix_levels.argtypes = [vp]
    L.solv_gpu_res.argtypes = [vp, ctypes.c_int, _f64p, _f64p, _f64p, ctypes.c_int]
    L.solv_gpu_precond.argtypes = [vp, ctypes.c_int, _f64p, _f64p]
    L.solv_gpu_direct.argtypes = [vp, ctypes.c_int, _f64p, _f64p, _f64p, _f64p]
    L.solv_gpu_spmv.argtypes = [vp, _f64p, _f64p]
    for fn in (L.solv_gpu_cg, L.solv_gpu_bicg):
        fn.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _f64p,
                       _f64p, _f64p, ctypes.c_int, ctypes.POINTER(Stats)]
    for fn in (L.solv_gpu_cg_dev, L.solv_gpu_bicg_dev):
        fn.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, vp, vp,
                       _f64p, ctypes.c_int, ctypes.POINTER(Stats)]
    L.solv_gpu_spmv_dev.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.solv_gpu_matrix_set_batch.argtypes = [vp, ctypes.c_int, _i32p, ctypes.c_int, _i32p, _i32p,
                                            _f64p, _f64p, _f64p]
    L.solv_gpu_n_systems.argtypes = [vp]
    L.solv_gpu_autotune.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(Tune)]
    L.solv_gpu_fcg.argtypes = [vp, ctypes.c_double, ctypes.c_int, _f64p, _f64p, _f64p,
                               ctypes.c_int, ctypes.POINTER(Stats)]
    L.solv_gpu_fcg_dev.argtypes = [vp, ctypes.c_double, ctypes.c_int, vp, vp, _f64p,
                                   ctypes.c_int, ctypes.POINTER(Stats)]
    L.solv_gpu_gnn_n_params.argtypes = []
    _f32p = ctypes.POINTER(ctypes.c_float)
    L.solv_gpu_gnn_set_params.argtypes = [vp, _f32p, ctypes.c_int]
    L.solv_gpu_gnn_get_params.argtypes = [vp, _f32p, ctypes.c_int]
    L.solv_gpu_gnn_get_grad.argtypes = [vp, _f32p, ctypes.c_int]
    L.solv_gpu_gnn_zero_grad.argtypes = [vp]
    L.solv_gpu_gnn_forward_dev.argtypes = [vp, vp, vp, vp, ctypes.c_int]
    L.solv_gpu_gnn_grad_dev.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.c_int]
    L.solv_gpu_gnn_adam.argtypes = [vp, ctypes.c_float, ctypes.c_float]
    L.solv_gpu_selftest_sweep_wait.argtypes = [vp]
    L.solv_gpu_kernel_time.argtypes = [vp, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_float)]
    L.solv_gpu_mg_aggregates.argtypes = [vp, ctypes.c_int, _i32p, ctypes.c_int, _i32p]
    L.solv_gpu_mg_aggregate.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), _i32p,
                                        ctypes.POINTER(ctypes.c_float), ctypes.c_int, _i32p, _i32p]
    for fn in (L.solv_gpu_cg_batch, L.solv_gpu_bicg_batch):
        fn.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _f64p,
                       _f64p, _f64p, ctypes.c_int, _i32p, _f64p, ctypes.POINTER(Stats)]
    for fn in (L.solv_gpu_cg_batch_dev, L.solv_gpu_bicg_batch_dev):
        fn.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, vp, vp,
                       _f64p, ctypes.c_int, _i32p, _f64p, ctypes.POINTER(Stats)]
    L._typed = True
    return L


class SolverError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"status {code}: {msg}")
        self.code = code


def _p(a, t):
    return a.ctypes.data_as(t)


class GpuSolver:
    """One device context: the matrix of solv_data.f90 resident in HBM."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = ctypes.c_void_p()
        rc = self._lib.solv_gpu_create(ctypes.byref(h), device)
        if rc != OK:
            raise SolverError(rc, "solv_gpu_create failed (no CUDA device?)")
        self._h = h
        self.n_cell = 0

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.solv_gpu_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, allow=(OK,)):
        if rc not in allow:
            msg = self._lib.solv_gpu_last_error(self._h).decode()
            raise SolverError(rc, msg or self._lib.solv_gpu_status_string(rc).decode())
        return rc

    # -- configuration -------------------------------------------------------
    def set_option(self, key: int, value: float):
        self._check(self._lib.solv_gpu_set_option(self._h, key, float(value)))

    def set_stream(self, stream_handle: int | None):
        self._check(self._lib.solv_gpu_set_stream(self._h, stream_handle or None))

    # -- matrix (grd_solv + coefficient fill) ----------------------------------
    def matrix_set(self, m) -> None:
        """m: programs_b200.mesh.FaceMatrix (or anything with n_cell, ip, inb, p, n, pl)."""
        self._keep = [np.ascontiguousarray(m.ip, np.int32), np.ascontiguousarray(m.inb, np.int32),
                      np.ascontiguousarray(m.p, np.float64), np.ascontiguousarray(m.n, np.float64),
                      np.ascontiguousarray(m.pl, np.float64)]
        ip, inb, p, n, pl = self._keep
        self._check(self._lib.solv_gpu_matrix_set(self._h, int(m.n_cell), ip.shape[0],
                                                  _p(ip, _i32p), _p(inb, _i32p), _p(p, _f64p),
                                                  _p(n, _f64p), _p(pl, _f64p)))
        self.n_cell = int(m.n_cell)
        self._keep = None

    def matrix_values(self, p, n, pl) -> None:
        p = np.ascontiguousarray(p, np.float64)
        n = np.ascontiguousarray(n, np.float64)
        pl = np.ascontiguousarray(pl, np.float64)
        self._check(self._lib.solv_gpu_matrix_values(self._h, _p(p, _f64p), _p(n, _f64p),
                                                     _p(pl, _f64p)))

    def matrix_values_dev(self, p_ptr: int, n_ptr: int, pl_ptr: int) -> None:
        self._check(self._lib.solv_gpu_matrix_values_dev(self._h, p_ptr, n_ptr, pl_ptr))

    @property
    def levels(self) -> int:
        return int(self._lib.solv_gpu_matrix_levels(self._h))

    # -- the hot path ----------------------------------------------------------
    @staticmethod
    def _as_phi(phi):
        if not (isinstance(phi, np.ndarray) and phi.dtype == np.float64 and phi.flags.c_contiguous):
            raise TypeError("phi must be a C-contiguous float64 array (n_cell, n_vc)")
        return phi.reshape(phi.shape[0], -1)

    @staticmethod
    def _as_res0(res0):
        if not (isinstance(res0, np.ndarray) and res0.dtype == np.float64):
            raise TypeError("res0 must be a float64 array (n_cell, n_vc)")
        if res0.ndim == 2 and not res0.flags.f_contiguous:
            raise TypeError("res0 must be Fortran-ordered like res0(ip,ivc)")
        return res0

    def solv_res(self, phi, res0, res0_n, not_r0=False):
        phi2 = self._as_phi(phi)
        V = phi2.shape[1]
        self._as_res0(res0)
        self._check(self._lib.solv_gpu_res(self._h, V, _p(phi2, _f64p), _p(res0, _f64p),
                                           _p(res0_n, _f64p), int(bool(not_r0))))

    def solv_precond(self, imat, c, c_r):
        self._check(self._lib.solv_gpu_precond(self._h, imat, _p(c, _f64p), _p(c_r, _f64p)))

    def solv_direct(self, imat, c, c_r, x, b):
        c = np.ascontiguousarray(c, np.float64)
        c_r = np.ascontiguousarray(c_r, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        self._check(self._lib.solv_gpu_direct(self._h, imat, _p(c, _f64p), _p(c_r, _f64p),
                                              _p(x, _f64p), _p(b, _f64p)))

    def spmv(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        self._check(self._lib.solv_gpu_spmv(self._h, _p(x, _f64p), _p(y, _f64p)))
        return y

    def _solve(self, fn, imat, reduc, n_iter, phi, res0, res0_n, not_r0):
        phi2 = self._as_phi(phi)
        V = phi2.shape[1]
        self._as_res0(res0)
        st = Stats()
        rc = fn(self._h, imat, float(reduc), int(n_iter), V, _p(phi2, _f64p), _p(res0, _f64p),
                _p(res0_n, _f64p), int(bool(not_r0)), ctypes.byref(st))
        self._check(rc, allow=(OK, MAXITER))
        return st.as_dict()

    def solv_cg(self, imat, reduc, n_iter, phi, res0, res0_n, not_r0=False):
        """solv_cg.f90:7 -- updates phi, res0 (-> initial residual), res0_n in place."""
        return self._solve(self._lib.solv_gpu_cg, imat, reduc, n_iter, phi, res0, res0_n, not_r0)

    def solv_bicg(self, imat, reduc, n_iter, phi, res0, res0_n, not_r0=False):
        """solv_bicg.f90:7 -- same arguments as solv_cg."""
        return self._solve(self._lib.solv_gpu_bicg, imat, reduc, n_iter, phi, res0, res0_n, not_r0)

    # -- device-resident forms (torch CUDA tensors or raw device pointers) ----
    def _solve_dev(self, fn, imat, reduc, n_iter, n_vc, phi_ptr, res0_ptr, not_r0):
        res0_n = np.zeros(n_vc)
        st = Stats()
        rc = fn(self._h, imat, float(reduc), int(n_iter), n_vc, phi_ptr, res0_ptr,
                _p(res0_n, _f64p), int(bool(not_r0)), ctypes.byref(st))
        self._check(rc, allow=(OK, MAXITER))
        return res0_n, st.as_dict()

    def solv_cg_dev(self, imat, reduc, n_iter, n_vc, phi_ptr, res0_ptr, not_r0=False):
        return self._solve_dev(self._lib.solv_gpu_cg_dev, imat, reduc, n_iter, n_vc, phi_ptr,
                               res0_ptr, not_r0)

    def solv_bicg_dev(self, imat, reduc, n_iter, n_vc, phi_ptr, res0_ptr, not_r0=False):
        return self._solve_dev(self._lib.solv_gpu_bicg_dev, imat, reduc, n_iter, n_vc, phi_ptr,
                               res0_ptr, not_r0)

    # -- learned preconditioner --------------------------------------------------
    def solv_fcg(self, reduc, n_iter, phi, res0, res0_n, not_r0=False):
        """Flexible CG with the learned preconditioner (FP32 inner, FP64
        refinement, plain PCG fallback); arguments as solv_cg minus imat."""
        phi2 = self._as_phi(phi)
        self._as_res0(res0)
        st = Stats()
        rc = self._lib.solv_gpu_fcg(self._h, float(reduc), int(n_iter), _p(phi2, _f64p),
                                    _p(res0, _f64p), _p(res0_n, _f64p), int(bool(not_r0)),
                                    ctypes.byref(st))
        self._check(rc, allow=(OK, MAXITER))
        return st.as_dict()

    def solv_fcg_dev(self, reduc, n_iter, phi_ptr, res0_ptr, not_r0=False):
        res0_n = np.zeros(1)
        st = Stats()
        rc = self._lib.solv_gpu_fcg_dev(self._h, float(reduc), int(n_iter), phi_ptr, res0_ptr,
                                        _p(res0_n, _f64p), int(bool(not_r0)), ctypes.byref(st))
        self._check(rc, allow=(OK, MAXITER))
        return res0_n, st.as_dict()

    @staticmethod
    def gnn_n_params() -> int:
        return int(lib().solv_gpu_gnn_n_params())

    def gnn_set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        self._check(self._lib.solv_gpu_gnn_set_params(
            self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.shape[0]))

    def gnn_get_params(self) -> np.ndarray:
        p = np.empty(self.gnn_n_params(), np.float32)
        self._check(self._lib.solv_gpu_gnn_get_params(
            self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.shape[0]))
        return p

    def gnn_get_grad(self) -> np.ndarray:
        g = np.empty(self.gnn_n_params(), np.float32)
        self._check(self._lib.solv_gpu_gnn_get_grad(
            self._h, g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), g.shape[0]))
        return g

    def gnn_forward_dev(self, r0_ptr: int, r_ptr: int, z_ptr: int, path: int = 0) -> None:
        """z = M^-1 r, the preconditioner built from r0 (device pointers, caller order)."""
        self._check(self._lib.solv_gpu_gnn_forward_dev(self._h, r0_ptr, r_ptr, z_ptr, path))

    def gnn_grad_dev(self, r0_ptr: int, samples_ptr: int, n_samples: int,
                     accumulate: bool = False) -> float:
        loss = ctypes.c_double()
        self._check(self._lib.solv_gpu_gnn_grad_dev(self._h, r0_ptr, samples_ptr, n_samples,
                                                    ctypes.byref(loss), int(bool(accumulate))))
        return loss.value

    def mg_aggregates(self, level: int, n_finer: int) -> tuple[np.ndarray, int]:
        """Aggregate index of every cell of level-1 (caller order for level 1)
        and the size of `level`."""
        agg = np.zeros(n_finer, np.int32)
        nc = ctypes.c_int()
        self._check(self._lib.solv_gpu_mg_aggregates(self._h, level, _p(agg, _i32p), n_finer,
                                                     ctypes.byref(nc)))
        return agg, nc.value

    def gnn_zero_grad(self) -> None:
        """Clear the accumulated gradient."""
        self._check(self._lib.solv_gpu_gnn_zero_grad(self._h))

    def gnn_adam(self, lr: float, grad_scale: float = 1.0) -> None:
        self._check(self._lib.solv_gpu_gnn_adam(self._h, lr, grad_scale))

    def autotune(self, solver: str = "cg", imat: int = 0, n_vc: int = 1) -> dict:
        """Pick launch shapes (and, for FP32 iterations, the products' vector
        width) for this matrix and solver ("cg", "bicg" or "fcg", the learned
        solve); the choice is left set on the context."""
        t = Tune()
        code = {"cg": 0, "bicg": 1, "fcg": 2}[solver]
        self._check(self._lib.solv_gpu_autotune(self._h, code, imat, n_vc, ctypes.byref(t)))
        return {"block": t.block, "grid_per_sm": t.grid_per_sm, "graph_iters": t.graph_iters,
                "vector_width": t.vector_width, "candidates": t.candidates,
                "ms_per_iter": t.ms_per_iter, "ms_per_iter_before": t.ms_per_iter_before}

    # -- batches of independent systems ----------------------------------------
    def matrix_set_batch(self, mats) -> np.ndarray:
        """Concatenate independent face matrices into one block-diagonal batch.
        Returns cell_ptr (0-based offsets of each system)."""
        ns = len(mats)
        cell_ptr = np.zeros(ns + 1, np.int32)
        for k, m in enumerate(mats):
            cell_ptr[k + 1] = cell_ptr[k] + m.n_cell
        ip = np.concatenate([m.ip + cell_ptr[k] for k, m in enumerate(mats)]).astype(np.int32)
        inb = np.concatenate([np.where(m.inb > 0, m.inb + cell_ptr[k], 0)
                              for k, m in enumerate(mats)]).astype(np.int32)
        p = np.concatenate([m.p for m in mats]).astype(np.float64)
        n = np.concatenate([m.n for m in mats]).astype(np.float64)
        pl = np.concatenate([m.pl for m in mats]).astype(np.float64)
        self._check(self._lib.solv_gpu_matrix_set_batch(
            self._h, ns, _p(cell_ptr, _i32p), ip.shape[0], _p(ip, _i32p), _p(inb, _i32p),
            _p(p, _f64p), _p(n, _f64p), _p(pl, _f64p)))
        self.n_cell = int(cell_ptr[-1])
        self.cell_ptr = cell_ptr
        return cell_ptr

    @property
    def n_systems(self) -> int:
        return int(self._lib.solv_gpu_n_systems(self._h))

    def _solve_batch(self, fn, imat, reduc, n_iter, phi, res0, not_r0):
        phi2 = self._as_phi(phi)
        V = phi2.shape[1]
        self._as_res0(res0)
        nl = self.n_systems * V
        rn = np.zeros(nl)
        iters = np.zeros(nl, np.int32)
        ratio = np.zeros(nl)
        st = Stats()
        rc = fn(self._h, imat, float(reduc), int(n_iter), V, _p(phi2, _f64p), _p(res0, _f64p),
                _p(rn, _f64p), int(bool(not_r0)), _p(iters, _i32p), _p(ratio, _f64p),
                ctypes.byref(st))
        self._check(rc, allow=(OK, MAXITER))
        d = st.as_dict()
        d.update(res0_n=rn.reshape(-1, V), iters_all=iters.reshape(-1, V),
                 ratio_all=ratio.reshape(-1, V))
        return d

    def solv_cg_batch(self, imat, reduc, n_iter, phi, res0, not_r0=False):
        return self._solve_batch(self._lib.solv_gpu_cg_batch, imat, reduc, n_iter, phi, res0, not_r0)

    def solv_bicg_batch(self, imat, reduc, n_iter, phi, res0, not_r0=False):
        return self._solve_batch(self._lib.solv_gpu_bicg_batch, imat, reduc, n_iter, phi, res0,
                                 not_r0)

    def solv_batch_dev(self, solver, imat, reduc, n_iter, n_vc, phi_ptr, res0_ptr, not_r0=False):
        fn = self._lib.solv_gpu_cg_batch_dev if solver == "cg" else self._lib.solv_gpu_bicg_batch_dev
        nl = self.n_systems * n_vc
        rn = np.zeros(nl)
        iters = np.zeros(nl, np.int32)
        ratio = np.zeros(nl)
        st = Stats()
        rc = fn(self._h, imat, float(reduc), int(n_iter), n_vc, phi_ptr, res0_ptr, _p(rn, _f64p),
                int(bool(not_r0)), _p(iters, _i32p), _p(ratio, _f64p), ctypes.byref(st))
        self._check(rc, allow=(OK, MAXITER))
        d = st.as_dict()
        d.update(res0_n=rn.reshape(-1, n_vc), iters_all=iters.reshape(-1, n_vc),
                 ratio_all=ratio.reshape(-1, n_vc))
        return d

    def selftest_sweep_wait(self) -> int:
        """Status of one bounded sweep wait on a value nothing writes
        (solv_gpu_selftest_sweep_wait): TIMEOUT when the bound works."""
        return int(self._lib.solv_gpu_selftest_sweep_wait(self._h))

    def kernel_time(self, which: int, repeat: int = 20) -> float:
        """ms per launch (solv_gpu_kernel_time): 0 FP64 SpMV, 1 FP32 SpMV, 2 the
        network operator, 3 one V-cycle, 4 level-0 residual of the V-cycle,
        5 the network's smoothing step, 6 flexible-CG product, 7 FP64 CG
        product, 8 one DILU application (both recurrences)."""
        ms = ctypes.c_float()
        self._check(self._lib.solv_gpu_kernel_time(self._h, which, repeat, ctypes.byref(ms)))
        return ms.value

    def spmv_dev(self, x_ptr: int, y_ptr: int, repeat: int = 1) -> float:
        ms = ctypes.c_float()
        self._check(self._lib.solv_gpu_spmv_dev(self._h, x_ptr, y_ptr, repeat, ctypes.byref(ms)))
        return ms.value


def mg_aggregate(ptr, adj, w, passes: int = 3):
    """The hierarchy's aggregation rule on a CSR graph (host only)."""
    L = lib()
    n = len(ptr) - 1
    ptr = np.ascontiguousarray(ptr, np.int64)
    adj = np.ascontiguousarray(adj, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    agg = np.zeros(n, np.int32)
    na = ctypes.c_int()
    rc = L.solv_gpu_mg_aggregate(n, ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                 _p(adj, _i32p), w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                 passes, _p(agg, _i32p), ctypes.byref(na))
    if rc:
        raise SolverError(rc, "mg_aggregate: bad graph")
    return agg, na.value


def new_res0(n_cell: int, n_vc: int) -> np.ndarray:
    """A Fortran-ordered res0(n_cell, n_vc) array."""
    return np.zeros((n_cell, n_vc), order="F")
