/*
 * fvmesh.h -- host-side unstructured hex mesh, face list and matrix
 * assembly for the face-addressed solvers.
 *
 * The face list follows the spray-simulation connectivity rules: faces are
 * emitted cell by cell in ascending cell order, each cell's local faces in
 * its element-table order; a face shared with an already visited
 * (lower-numbered) cell is not emitted again, so every interior face has
 * owner ip < neighbour in and boundary faces have in = 0
 * (grd_conn.f90:45-113).  Geometry follows grd_geom.f90:31-43 (cell centre
 * = vertex average) and :119-208 (triangle-fan area and normal, face centre,
 * auxiliary poles, l_pn, w_fp).  All indices exposed here are 1-based.
 */
#ifndef FVMESH_H
#define FVMESH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fvm_mesh fvm_mesh;

/* nx*ny*nz hex cells on the unit box, interior vertices jittered uniformly
 * by +-jitter*h per axis, cells randomly permuted when permute != 0.  The
 * generator draws from std::mt19937_64(seed). */
fvm_mesh *fvm_mesh_hex(int nx, int ny, int nz, double jitter, uint64_t seed,
                       int permute);

/* Gambit neutral file reader (grd_read.f90) with hashed face matching in
 * place of the quadratic search of grd_conn.f90:77-93.  NULL on error. */
fvm_mesh *fvm_mesh_read_neu(const char *path);

void fvm_mesh_free(fvm_mesh *m);

/* n_cell, n_face (interior + boundary), n_bface, n_vert */
void fvm_mesh_sizes(const fvm_mesh *m, int *n_cell, int *n_face, int *n_bface,
                    int *n_vert);

/* ng(:)%ip / ng(:)%in, 1-based, in = 0 on boundary faces. */
void fvm_mesh_faces(const fvm_mesh *m, int *ip, int *in);

/* Per-face geometry (any output may be NULL): area s, normal (3 per face,
 * outward from the owner), centre (3 per face), l_pn, w_fp. */
void fvm_mesh_face_geom(const fvm_mesh *m, double *s, double *nrm, double *xf,
                        double *l_pn, double *w_fp);

/* Keep the face geometry and cell volumes in memory (9 + 1 doubles per
 * face / cell) so repeated assemblies on one mesh skip the geometry;
 * dropped by renumbering. */
void fvm_mesh_cache_geometry(fvm_mesh *m);
/* Which face distance l_pn and interpolation weight w_fp (on phi_N) the
 * geometry reports, and with it every assembly: 0 (default) the distance
 * between the two auxiliary points on the face normal and the linear
 * weight |x_f - x_P,aux| / l_pn; 1 the reference's centre distance
 * |x_N - x_P| and w_fp = 1 - |x_f - x_P| / l_pn (cfd_grid.f90:520, 524;
 * boundary faces |x_f - x_P|, :534).  Both agree on regular meshes. */
void fvm_mesh_set_face_weights(fvm_mesh *m, int reference);

/* Cell centres (3 per cell) and volumes (either may be NULL). */
void fvm_mesh_cell_geom(const fvm_mesh *m, double *xc, double *vol);

/* Renumber cells.  method 1 = reverse Cuthill-McKee, 2 = Morton
 * space-filling curve of the cell centres, 3 = a given permutation in
 * perm (new 1-based index of old cell i), 4 = multicolour (a greedy
 * colouring in RCM order, cells colour by colour, RCM order inside a
 * colour: the DIC / DILU recurrences become as deep as the colour count).  The face list is re-emitted
 * under the new numbering.  On return perm (if not NULL and method != 3)
 * holds the permutation applied.  Returns 0, or -1 on bad input. */
int fvm_mesh_renumber(fvm_mesh *m, int method, int *perm);

/* Pressure-correction Poisson matrix: p = n = -area/l_pn on interior
 * faces, pl = sum of area/l_pn, boundaries all-Neumann; cell `pin`
 * (1-based, 0 for none) is pinned by zeroing both off-diagonals of every
 * face that touches it, which keeps the matrix symmetric positive definite.
 * Boundary faces get p = n = 0. */
void fvm_assemble_pressure(const fvm_mesh *m, int pin, double *p, double *n,
                           double *pl);

/* Momentum convection-diffusion matrix, first-order upwind
 * (cfd_setup.f90:324-330): p = -d + min(c,0), n = -d - max(c,0),
 * pl = -sum(off-diagonals) + V/dt, with d = gamma*area/l_pn and c the
 * face flux of a Taylor-Green field u = U0 (sin X cos Y cos Z,
 * -cos X sin Y cos Z, 0), X = 2 pi x, scaled so the largest cell Peclet
 * number U0*h/gamma is pe_max.  Walls are Dirichlet (d on the boundary
 * face, zero flux).  dt = cfl*h/U0.  Returns dt. */
double fvm_assemble_momentum(const fvm_mesh *m, double gamma, double pe_max,
                             double cfl, double *p, double *n, double *pl);

/* Momentum matrix of a lid-driven cavity for a given cell velocity field
 * u (3 per cell) and face mass fluxes flux (per face, owner -> neighbour;
 * NULL = from the linearly interpolated u): upwind convection, central
 * diffusion d = mu*area/l_pn, walls no-slip, the y = 1 wall moving with
 * (u_lid, 0, 0), under-relaxation urf (cfd_setup.f90:324-330, 473-518):
 * pl = (-sum off-diagonals) / urf.  rhs (3 per cell, may be NULL) gets
 * the wall terms and (1-urf) pl u.  Returns the face fluxes used in flux_out
 * (may be NULL). */
void fvm_assemble_momentum_field(const fvm_mesh *m, const double *u, const double *flux,
                                 double rho, double mu, double u_lid, double urf,
                                 double *p, double *n, double *pl, double *rhs,
                                 double *flux_out);

/* Pressure-correction matrix of cfd_setup.f90:604-634:
 * d = rho * p_r * area * v / l_pn with p_r, v the w_fp-weighted face
 * values of 1/a_P (a_P = the momentum diagonal `ap`) and of the cell
 * volume; p = n = -d, pl = sum d; boundaries all-Neumann; cell `pin`
 * (1-based, 0 none) pinned as in fvm_assemble_pressure. */
void fvm_assemble_pressure_correction(const fvm_mesh *m, const double *ap, double rho,
                                      int pin, double *p, double *n, double *pl);

/* A cavity-like divergence-free velocity field (3 per cell): stream
 * function psi = u_lid x^2 (1-x)^2 y^2 (1-y) (scaled so u(0.5,1) = u_lid),
 * u = dpsi/dy, v = -dpsi/dx, modulated by sin(pi z); w = 0. */
void fvm_cavity_field(const fvm_mesh *m, double u_lid, double *u);

/* -- SIMPLE outer-loop pieces (lid-driven cavity) ------------------------ */
/* Green-Gauss gradient (solv_grad, cfd_setup.f90:765-866, one sweep):
 * grad_i = sum_f phi_f area n / V_i, phi_f = w phi_N + (1-w) phi_P inside,
 * phi_P on walls (zero normal gradient); `ncomp` components per cell,
 * grad has 3*ncomp per cell. */
void fvm_gradient(const fvm_mesh *m, int ncomp, const double *phi, double *grad);

/* solv_grad in full (cfd_setup.f90:765-866, 3-d): n_iter Green-Gauss
 * sweeps.  Sweep 1 takes interior face values phi_f = w phi_N + (1-w) phi_P;
 * later sweeps first move phi_P and phi_N to their auxiliary points on the
 * face normal through the face centre with the previous sweep's gradient,
 * phi_P + g_P.dx_P (dx_P = x_P_aux - x_P, cfd_grid.f90:487-491, 512-516).
 * Boundary faces: neu = 0 takes bval[f*ncomp + k] (values per face and
 * component; only boundary entries are read), neu = 1 the cell value,
 * neu = 2 the cell value plus,
 * after sweep 1, g_P.(x_f - x_P).  Each face adds ((phi_f s) n) / V in the
 * reference's face order, 1/V formed once per cell.  grad has 3*ncomp per
 * cell.  Returns 0, or -1 for n_iter < 1, neu outside 0..2 or neu = 0
 * without bval. */
int fvm_gradient_sweeps(const fvm_mesh *m, int ncomp, const double *phi, const double *bval,
                        int n_iter, int neu, double *grad);

/* The explicit (deferred-correction) right-hand-side terms of the
 * reference's momentum face loop (cfd_setup.f90:185-272, 306-328): per
 * interior face
 *   cor = c_bl c (phi_up - phi_f) + d ((phi_N' - phi_P') - (phi_N - phi_P)),
 * phi_P' = phi_P + g_P.dx_P at the auxiliary points, phi_up the upwind
 * cell value of the face mass flux c (flux[f], owner -> neighbour),
 * d = mu area / l_pn; rhs_P += cor and rhs_N -= cor for each of the ncomp
 * components (grad: 3 per component per cell).  The face value phi_f is
 * by `scheme` (the reference's c_sch): 0 central, w phi_N' + (1-w) phi_P';
 * 1 min-mod, 2 van Leer, 3 superbee: with C the upwind and D the downwind
 * auxiliary value and U = D - 2 g_C.(x_D' - x_C'), r = (C - U) / (D - C +
 * small), phi_f = C + psi(r) (D - C) / 2.  rhs is accumulated into, not
 * cleared; the implicit part is the matrix of fvm_assemble_momentum_field.
 * Returns 0, or -1 for a scheme outside 0..3. */
int fvm_momentum_deferred(const fvm_mesh *m, int ncomp, const double *phi, const double *grad,
                          const double *flux, double mu, double c_bl, int scheme, double *rhs);

/* Face mass fluxes from the momentum-predicted velocity with Rhie-Chow
 * pressure smoothing (cfd_setup.f90:615-634): F = rho area (u_f . n)
 * - d ((p_N - p_P) - grad(p)_f . (x_N - x_P)), d = rho (V/a_P)_f area / l_pn;
 * zero on walls. */
void fvm_face_flux(const fvm_mesh *m, const double *u, const double *p, const double *gradp,
                   const double *ap, double rho, double *flux);
/* The same fluxes with the pressures taken at the auxiliary points of the
 * face, p_P + grad(p)_P . dx_P, as the reference's pressure-correction face
 * loop does (cfd_setup.f90:611-620):
 * dp = (p_N' - p_P') - grad(p)_f . (x_N - x_P). */
void fvm_face_flux_aux(const fvm_mesh *m, const double *u, const double *p, const double *gradp,
                       const double *ap, double rho, double *flux);

/* Mass imbalance right-hand side b_i = -sum of outflow of cell i; cell
 * `pin` (1-based) gets 0.  Returns sum |b|. */
double fvm_mass_imbalance(const fvm_mesh *m, const double *flux, int pin, double *b);

/* SIMPLE corrections with the pressure correction pp:
 * p += urf_p pp; u_i -= (V_i / a_P,i) grad(pp)_i; F -= d (pp_N - pp_P). */
void fvm_simple_correct(const fvm_mesh *m, const double *pp, const double *gradpp,
                        const double *ap, double rho, double urf_p, double *u, double *p,
                        double *flux);

/* Uniform [-1,1) values from std::mt19937_64(seed) (53-bit mantissa). */
void fvm_uniform(uint64_t seed, int64_t count, double *out);

#ifdef __cplusplus
}
#endif
#endif
