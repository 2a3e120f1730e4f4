"""Face-addressed meshes and matrices (host side, ``libfvmesh.so``).

A :class:`Mesh` owns a hex mesh and exposes the spray-simulation face list
(``ng(:)%ip``, ``ng(:)%in``, 1-based, ``in = 0`` on boundary faces; see
spray-simulation/grd_conn.f90:99-113) plus the matrices the solvers take:

* :meth:`Mesh.pressure` -- the pressure-correction Poisson system
  (p = n = -area/l_pn, pl = sum area/l_pn, one pinned cell);
* :meth:`Mesh.momentum` -- first-order upwind convection-diffusion with a
  Taylor-Green flux and a 1/dt diagonal (cfd_setup.f90:324-330, 473-518).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import load

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


def _lib():
    lib = load("libfvmesh.so")
    if not getattr(lib, "_typed", False):
        lib.fvm_mesh_hex.restype = ctypes.c_void_p
        lib.fvm_mesh_hex.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_uint64, ctypes.c_int]
        lib.fvm_mesh_read_neu.restype = ctypes.c_void_p
        lib.fvm_mesh_read_neu.argtypes = [ctypes.c_char_p]
        lib.fvm_mesh_free.argtypes = [ctypes.c_void_p]
        lib.fvm_mesh_sizes.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p]
        lib.fvm_mesh_faces.argtypes = [ctypes.c_void_p, _i32p, _i32p]
        lib.fvm_mesh_face_geom.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p]
        lib.fvm_mesh_cell_geom.argtypes = [ctypes.c_void_p, _f64p, _f64p]
        lib.fvm_mesh_renumber.restype = ctypes.c_int
        lib.fvm_mesh_renumber.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p]
        lib.fvm_assemble_pressure.argtypes = [ctypes.c_void_p, ctypes.c_int, _f64p, _f64p, _f64p]
        lib.fvm_assemble_momentum.restype = ctypes.c_double
        lib.fvm_assemble_momentum.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, _f64p, _f64p, _f64p]
        lib.fvm_uniform.argtypes = [ctypes.c_uint64, ctypes.c_int64, _f64p]
        lib.fvm_cavity_field.argtypes = [ctypes.c_void_p, ctypes.c_double, _f64p]
        lib.fvm_mesh_cache_geometry.argtypes = [ctypes.c_void_p]
        lib.fvm_mesh_set_face_weights.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.fvm_gradient.argtypes = [ctypes.c_void_p, ctypes.c_int, _f64p, _f64p]
        lib.fvm_momentum_deferred.restype = ctypes.c_int
        lib.fvm_momentum_deferred.argtypes = [ctypes.c_void_p, ctypes.c_int, _f64p, _f64p, _f64p,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                              _f64p]
        lib.fvm_gradient_sweeps.restype = ctypes.c_int
        lib.fvm_gradient_sweeps.argtypes = [ctypes.c_void_p, ctypes.c_int, _f64p, _f64p,
                                            ctypes.c_int, ctypes.c_int, _f64p]
        lib.fvm_face_flux.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p, ctypes.c_double,
                                      _f64p]
        lib.fvm_face_flux_aux.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p, ctypes.c_double,
                                      _f64p]
        lib.fvm_mass_imbalance.restype = ctypes.c_double
        lib.fvm_mass_imbalance.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int, _f64p]
        lib.fvm_simple_correct.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, ctypes.c_double,
                                           ctypes.c_double, _f64p, _f64p, _f64p]
        lib.fvm_assemble_momentum_field.argtypes = [
            ctypes.c_void_p, _f64p, _f64p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, _f64p, _f64p, _f64p, _f64p, _f64p]
        lib.fvm_assemble_pressure_correction.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_double,
                                                         ctypes.c_int, _f64p, _f64p, _f64p]
        lib._typed = True
    return lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


@dataclass
class FaceMatrix:
    """The solver's matrix: ng(:)%{ip,in,p,n} and pl (solv_data.f90:14-22)."""
    n_cell: int
    ip: np.ndarray  # int32, 1-based
    inb: np.ndarray  # int32, 1-based, 0 = boundary
    p: np.ndarray
    n: np.ndarray
    pl: np.ndarray

    @property
    def n_face(self) -> int:
        return int(self.ip.shape[0])

    def to_scipy(self):
        """Assemble A as scipy CSR (test / reference use)."""
        import scipy.sparse as sp
        m = self.inb > 0
        a = self.ip[m] - 1
        b = self.inb[m] - 1
        rows = np.concatenate([np.arange(self.n_cell), a, b])
        cols = np.concatenate([np.arange(self.n_cell), b, a])
        vals = np.concatenate([self.pl, self.p[m], self.n[m]])
        return sp.csr_matrix((vals, (rows, cols)), shape=(self.n_cell, self.n_cell))


class Mesh:
    RCM = 1
    SFC = 2
    COLOR = 4  # multicolour: colour by colour, RCM order inside a colour

    def __init__(self, handle: int):
        if not handle:
            raise RuntimeError("mesh construction failed")
        self._h = ctypes.c_void_p(handle)
        self._lib = _lib()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.fvm_mesh_free(h)
            self._h = ctypes.c_void_p(0)

    @classmethod
    def hex(cls, nx: int, ny: int | None = None, nz: int | None = None, jitter: float = 0.15,
            seed: int = 0, permute: bool = True) -> "Mesh":
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        return cls(_lib().fvm_mesh_hex(nx, ny, nz, jitter, seed, 1 if permute else 0))

    @classmethod
    def read_neu(cls, path: str) -> "Mesh":
        h = _lib().fvm_mesh_read_neu(path.encode())
        if not h:
            raise RuntimeError(f"cannot read Gambit neutral file {path}")
        return cls(h)

    def sizes(self):
        v = [ctypes.c_int() for _ in range(4)]
        self._lib.fvm_mesh_sizes(self._h, *[ctypes.byref(x) for x in v])
        return tuple(x.value for x in v)  # n_cell, n_face, n_bface, n_vert

    @property
    def n_cell(self) -> int:
        return self.sizes()[0]

    @property
    def n_face(self) -> int:
        return self.sizes()[1]

    def faces(self):
        F = self.n_face
        ip = np.empty(F, np.int32)
        inb = np.empty(F, np.int32)
        self._lib.fvm_mesh_faces(self._h, _p(ip, _i32p), _p(inb, _i32p))
        return ip, inb

    def face_geom(self):
        F = self.n_face
        s = np.empty(F)
        nrm = np.empty((F, 3))
        xf = np.empty((F, 3))
        l_pn = np.empty(F)
        w_fp = np.empty(F)
        self._lib.fvm_mesh_face_geom(self._h, _p(s, _f64p), _p(nrm, _f64p), _p(xf, _f64p),
                                     _p(l_pn, _f64p), _p(w_fp, _f64p))
        return s, nrm, xf, l_pn, w_fp

    def cell_geom(self):
        N = self.n_cell
        xc = np.empty((N, 3))
        vol = np.empty(N)
        self._lib.fvm_mesh_cell_geom(self._h, _p(xc, _f64p), _p(vol, _f64p))
        return xc, vol

    def renumber(self, method: int) -> np.ndarray:
        """Renumber cells in place (RCM, SFC or COLOR); returns new index of old
        cell (1-based)."""
        perm = np.empty(self.n_cell, np.int32)
        rc = self._lib.fvm_mesh_renumber(self._h, method, _p(perm, _i32p))
        if rc != 0:
            raise ValueError("renumber failed")
        return perm

    def cache_geometry(self) -> None:
        """Keep face geometry and volumes for repeated assembly on this mesh."""
        self._lib.fvm_mesh_cache_geometry(self._h)

    def set_face_weights(self, reference: bool) -> None:
        """Face distance and interpolation weight of every assembly: False
        (default) along the face normal between the auxiliary points, with
        the linear weight; True the reference's centre distance and
        w_fp = 1 - |x_f - x_P| / l_pn (cfd_grid.f90:520, 524)."""
        self._lib.fvm_mesh_set_face_weights(self._h, 1 if reference else 0)

    def permute(self, perm: np.ndarray) -> None:
        """Apply a given permutation (new 1-based index of old cell i)."""
        perm = np.ascontiguousarray(perm, np.int32)
        if self._lib.fvm_mesh_renumber(self._h, 3, _p(perm, _i32p)) != 0:
            raise ValueError("bad permutation")

    def pressure(self, pin: int = 1) -> FaceMatrix:
        ip, inb = self.faces()
        F, N = ip.shape[0], self.n_cell
        p = np.empty(F)
        n = np.empty(F)
        pl = np.empty(N)
        self._lib.fvm_assemble_pressure(self._h, pin, _p(p, _f64p), _p(n, _f64p), _p(pl, _f64p))
        return FaceMatrix(N, ip, inb, p, n, pl)

    def momentum(self, gamma: float = 1e-3, pe_max: float = 50.0, cfl: float = 5.0):
        ip, inb = self.faces()
        F, N = ip.shape[0], self.n_cell
        p = np.empty(F)
        n = np.empty(F)
        pl = np.empty(N)
        dt = self._lib.fvm_assemble_momentum(self._h, gamma, pe_max, cfl, _p(p, _f64p),
                                             _p(n, _f64p), _p(pl, _f64p))
        return FaceMatrix(N, ip, inb, p, n, pl), dt


def cavity_field(mesh: "Mesh", u_lid: float) -> np.ndarray:
    """A divergence-free cavity-like velocity field (n_cell, 3)."""
    u = np.empty((mesh.n_cell, 3))
    _lib().fvm_cavity_field(mesh._h, u_lid, _p(u, _f64p))
    return u


def momentum_field(mesh: "Mesh", u: np.ndarray, flux=None, rho=1.0, mu=1e-3, u_lid=1.0,
                   urf=0.7):
    """Momentum matrix for velocity field u (cfd_setup.f90:324-330, 517-518).
    Returns (FaceMatrix, rhs (n_cell, 3), face fluxes)."""
    ip, inb = mesh.faces()
    F, N = ip.shape[0], mesh.n_cell
    u = np.ascontiguousarray(u, np.float64)
    p, n, pl = np.empty(F), np.empty(F), np.empty(N)
    rhs = np.empty((N, 3))
    fo = np.empty(F)
    fl = None if flux is None else _p(np.ascontiguousarray(flux, np.float64), _f64p)
    _lib().fvm_assemble_momentum_field(mesh._h, _p(u, _f64p), fl, rho, mu, u_lid, urf,
                                       _p(p, _f64p), _p(n, _f64p), _p(pl, _f64p),
                                       _p(rhs, _f64p), _p(fo, _f64p))
    return FaceMatrix(N, ip, inb, p, n, pl), rhs, fo


def pressure_correction(mesh: "Mesh", ap: np.ndarray, rho=1.0, pin=1) -> FaceMatrix:
    """Pressure-correction matrix from the momentum diagonal (cfd_setup.f90:604-634)."""
    ip, inb = mesh.faces()
    F, N = ip.shape[0], mesh.n_cell
    ap = np.ascontiguousarray(ap, np.float64)
    p, n, pl = np.empty(F), np.empty(F), np.empty(N)
    _lib().fvm_assemble_pressure_correction(mesh._h, _p(ap, _f64p), rho, pin, _p(p, _f64p),
                                            _p(n, _f64p), _p(pl, _f64p))
    return FaceMatrix(N, ip, inb, p, n, pl)


def _c(a):
    return np.ascontiguousarray(a, np.float64)


def gradient(mesh: "Mesh", phi: np.ndarray) -> np.ndarray:
    """Green-Gauss gradient of a cell field (n_cell,) or (n_cell, k)."""
    phi = _c(phi)
    k = 1 if phi.ndim == 1 else phi.shape[1]
    g = np.empty((mesh.n_cell, k, 3)) if k > 1 else np.empty((mesh.n_cell, 3))
    _lib().fvm_gradient(mesh._h, k, _p(phi, _f64p), _p(g, _f64p))
    return g


def gradient_sweeps(mesh: "Mesh", phi: np.ndarray, n_iter: int = 2, neu: int = 2,
                    bval: np.ndarray | None = None) -> np.ndarray:
    """solv_grad (cfd_setup.f90:765-866) with its sweeps and boundary modes:
    n_iter Green-Gauss sweeps, later ones corrected with the previous
    gradient; boundary faces neu = 0 Dirichlet from bval (one value per
    face and component, boundary entries read), 1 the cell value, 2 the
    cell value extrapolated to the face.  The reference's loop calls it
    with n_iter = 2 (cfd_solve.f90:38), neu = 0 for velocity and 2 for
    pressure (cfd_setup.f90:124, 689, 754)."""
    phi = _c(phi)
    k = 1 if phi.ndim == 1 else phi.shape[1]
    g = np.empty((mesh.n_cell, k, 3)) if k > 1 else np.empty((mesh.n_cell, 3))
    bv = None if bval is None else _c(np.broadcast_to(
        np.asarray(bval, np.float64).reshape(mesh.n_face, -1), (mesh.n_face, k)))
    rc = _lib().fvm_gradient_sweeps(mesh._h, k, _p(phi, _f64p), None if bv is None else
                                    _p(bv, _f64p), int(n_iter), int(neu), _p(g, _f64p))
    if rc != 0:
        raise ValueError("gradient_sweeps: n_iter >= 1, neu in 0..2, bval needed for neu = 0")
    return g


def momentum_deferred(mesh: "Mesh", u: np.ndarray, grad: np.ndarray, flux: np.ndarray,
                      mu: float, c_bl: float = 1.0, scheme: int = 0) -> np.ndarray:
    """The reference's explicit momentum terms (deferred correction toward
    the face values of `scheme` -- 0 central, 1 min-mod, 2 van Leer,
    3 superbee -- blended by c_bl, and the non-orthogonal diffusion
    correction, cfd_setup.f90:185-328) for a cell field u (n_cell,) or
    (n_cell, k), its gradient (as gradient_sweeps returns it) and the face
    mass fluxes; returns the right-hand-side increments, shaped like u."""
    u = _c(u)
    k = 1 if u.ndim == 1 else u.shape[1]
    g = _c(grad).reshape(mesh.n_cell, k, 3)
    out = np.zeros((mesh.n_cell, k))
    rc = _lib().fvm_momentum_deferred(mesh._h, k, _p(u, _f64p), _p(g, _f64p),
                                      _p(_c(flux), _f64p), float(mu), float(c_bl), int(scheme),
                                      _p(out, _f64p))
    if rc != 0:
        raise ValueError("momentum_deferred: scheme is 0 (central) .. 3 (superbee)")
    return out[:, 0].copy() if u.ndim == 1 else out


def face_flux(mesh: "Mesh", u, p, gradp, ap, rho=1.0, aux=False) -> np.ndarray:
    """Rhie-Chow face fluxes; aux takes the pressures at the face's
    auxiliary points, as the reference does (cfd_setup.f90:611-620)."""
    f = np.empty(mesh.n_face)
    u, p, gradp, ap = _c(u), _c(p), _c(gradp), _c(ap)
    fn = _lib().fvm_face_flux_aux if aux else _lib().fvm_face_flux
    fn(mesh._h, _p(u, _f64p), _p(p, _f64p), _p(gradp, _f64p), _p(ap, _f64p), rho, _p(f, _f64p))
    return f


def mass_imbalance(mesh: "Mesh", flux, pin=1):
    b = np.empty(mesh.n_cell)
    flux = _c(flux)
    t = _lib().fvm_mass_imbalance(mesh._h, _p(flux, _f64p), pin, _p(b, _f64p))
    return b, t


def simple_correct(mesh: "Mesh", pp, gradpp, ap, rho, urf_p, u, p, flux) -> None:
    """In place: p += urf_p pp; u -= V/a_P grad pp; flux -= d (pp_N - pp_P)."""
    for a in (u, p, flux):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    pp, gradpp, ap = _c(pp), _c(gradpp), _c(ap)
    _lib().fvm_simple_correct(mesh._h, _p(pp, _f64p), _p(gradpp, _f64p), _p(ap, _f64p), rho,
                              urf_p, _p(u, _f64p), _p(p, _f64p), _p(flux, _f64p))


def uniform(seed: int, count: int) -> np.ndarray:
    """Uniform [-1, 1) from std::mt19937_64(seed), as the C++ generator draws."""
    out = np.empty(count)
    _lib().fvm_uniform(seed, count, _p(out, _f64p))
    return out


def poisson_rhs(n_cell: int, seed: int, pin: int = 1) -> np.ndarray:
    """uniform[-1,1] with its mean removed; zero at the pinned cell."""
    b = uniform(seed, n_cell)
    b -= b.mean()
    if pin > 0:
        b[pin - 1] = 0.0
    return b
