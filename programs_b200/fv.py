"""The SIMPLE outer-loop pieces on the GPU (include/fv_gpu.h) for a Mesh.

:class:`GpuFv` uploads a mesh's geometry once and offers, on torch CUDA
tensors in the caller's layout, what ``mesh.py`` offers on the host:
momentum and pressure-correction assembly (cfd_setup.f90:178-431, 473-518,
604-646), the Green-Gauss gradient (solv_grad, :765-866), Rhie-Chow face
fluxes, the mass imbalance and the SIMPLE corrections.  Results are
bit-for-bit those of the host functions.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes

from .solver import SolverError, lib

_vp = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int


def _typed():
    L = lib()
    if getattr(L, "_fv_typed", False):
        return L
    L.fv_gpu_create.argtypes = [ctypes.POINTER(_vp), _i, _i, _i] + [_vp] * 9
    L.fv_gpu_destroy.argtypes = [_vp]
    L.fv_gpu_set_stream.argtypes = [_vp, _vp]
    L.fv_gpu_momentum.argtypes = [_vp, _vp, _vp, _d, _d, _d, _d, _vp, _vp, _vp, _vp, _vp]
    L.fv_gpu_pressure_correction.argtypes = [_vp, _vp, _d, _i, _vp, _vp, _vp]
    L.fv_gpu_gradient.argtypes = [_vp, _i, _vp, _vp]
    L.fv_gpu_face_flux.argtypes = [_vp, _vp, _vp, _vp, _vp, _d, _vp]
    L.fv_gpu_face_flux_aux.argtypes = [_vp, _vp, _vp, _vp, _vp, _d, _vp]
    L.fv_gpu_gradient_sweeps.argtypes = [_vp, _i, _vp, _vp, _i, _i, _vp]
    L.fv_gpu_momentum_deferred.argtypes = [_vp, _i, _vp, _vp, _vp, _d, _d, _i, _vp]
    L.fv_gpu_mass_imbalance.argtypes = [_vp, _vp, _i, _vp, ctypes.POINTER(_d)]
    L.fv_gpu_simple_correct.argtypes = [_vp, _vp, _vp, _vp, _d, _d, _vp, _vp, _vp]
    L._fv_typed = True
    return L


def _ptr(t):
    return None if t is None else t.data_ptr()


class GpuFv:
    """Device geometry of one mesh and the SIMPLE pieces on it."""

    def __init__(self, mesh, device: int = 0):
        import numpy as np
        import torch
        self._lib = _typed()
        self.device = torch.device("cuda", device)
        ip, inb = mesh.faces()
        s, nrm, xf, l_pn, w_fp = mesh.face_geom()
        xc, vol = mesh.cell_geom()
        self.n_cell, self.n_face = mesh.n_cell, ip.shape[0]
        arrs = [np.ascontiguousarray(a) for a in (ip, inb, s, nrm, xf, l_pn, w_fp, xc, vol)]
        h = _vp()
        rc = self._lib.fv_gpu_create(ctypes.byref(h), device, self.n_cell, self.n_face,
                                     *[a.ctypes.data for a in arrs])
        if rc:
            raise SolverError(rc, "fv_gpu_create failed")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fv_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise SolverError(rc, "fv_gpu call failed")

    def _new(self, *shape):
        import torch
        return torch.empty(*shape, dtype=torch.float64, device=self.device)

    def momentum_field(self, u, flux=None, rho=1.0, mu=1e-3, u_lid=1.0, urf=0.7):
        """(p, n, pl, rhs (n_cell, 3), face fluxes) for the velocity u (n_cell, 3)."""
        p, n, pl = self._new(self.n_face), self._new(self.n_face), self._new(self.n_cell)
        rhs, fo = self._new(self.n_cell, 3), self._new(self.n_face)
        self._check(self._lib.fv_gpu_momentum(self._h, _ptr(u), _ptr(flux), rho, mu, u_lid, urf,
                                              _ptr(p), _ptr(n), _ptr(pl), _ptr(rhs), _ptr(fo)))
        return p, n, pl, rhs, fo

    def pressure_correction(self, ap, rho=1.0, pin=1):
        p, n, pl = self._new(self.n_face), self._new(self.n_face), self._new(self.n_cell)
        self._check(self._lib.fv_gpu_pressure_correction(self._h, _ptr(ap), rho, pin, _ptr(p),
                                                         _ptr(n), _ptr(pl)))
        return p, n, pl

    def gradient(self, phi):
        k = 1 if phi.dim() == 1 else phi.shape[1]
        g = self._new(self.n_cell, k, 3) if k > 1 else self._new(self.n_cell, 3)
        self._check(self._lib.fv_gpu_gradient(self._h, k, _ptr(phi), _ptr(g)))
        return g

    def face_flux(self, u, p, gradp, ap, rho=1.0, aux=False):
        """Rhie-Chow face fluxes; aux takes the pressures at the auxiliary
        points (cfd_setup.f90:611-620)."""
        f = self._new(self.n_face)
        fn = self._lib.fv_gpu_face_flux_aux if aux else self._lib.fv_gpu_face_flux
        self._check(fn(self._h, _ptr(u), _ptr(p), _ptr(gradp), _ptr(ap), rho, _ptr(f)))
        return f

    def gradient_sweeps(self, phi, n_iter=2, neu=2, bval=None):
        """solv_grad in full: n_iter corrected sweeps, walls by neu (bval:
        (n_face, ncomp) wall values for neu = 0)."""
        k = 1 if phi.dim() == 1 else phi.shape[1]
        g = self._new(self.n_cell, k, 3) if k > 1 else self._new(self.n_cell, 3)
        self._check(self._lib.fv_gpu_gradient_sweeps(self._h, k, _ptr(phi), _ptr(bval), n_iter,
                                                     neu, _ptr(g)))
        return g

    def momentum_deferred(self, u, grad, flux, mu, rhs, c_bl=1.0, scheme=0):
        """Adds the explicit momentum terms to rhs (in place)."""
        k = 1 if u.dim() == 1 else u.shape[1]
        self._check(self._lib.fv_gpu_momentum_deferred(self._h, k, _ptr(u), _ptr(grad), _ptr(flux),
                                                       mu, c_bl, scheme, _ptr(rhs)))
        return rhs

    def mass_imbalance(self, flux, pin=1):
        b = self._new(self.n_cell)
        t = _d()
        self._check(self._lib.fv_gpu_mass_imbalance(self._h, _ptr(flux), pin, _ptr(b),
                                                    ctypes.byref(t)))
        return b, t.value

    def simple_correct(self, pp, gradpp, ap, rho, urf_p, u, p, flux):
        """In place on u, p, flux (device tensors)."""
        self._check(self._lib.fv_gpu_simple_correct(self._h, _ptr(pp), _ptr(gradpp), _ptr(ap),
                                                    rho, urf_p, _ptr(u), _ptr(p), _ptr(flux)))
