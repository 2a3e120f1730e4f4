/*
 * fv_gpu.h -- C-ABI of the SIMPLE outer-loop pieces on the GPU: momentum and
 * pressure-correction assembly, Green-Gauss gradient, Rhie-Chow face fluxes,
 * mass imbalance and the SIMPLE corrections, for the lid-driven cavity of the
 * spray-simulation SIMPLE solver.
 *
 * The reference does these in face loops inside cfd_setup.f90 (momentum
 * assembly :178-431 and :473-518, pressure correction :604-646, solv_grad
 * :765-866) before and after every call of the solvers this library
 * replaces.  Here they run on device arrays in the caller's layout, so an
 * outer iteration never leaves the GPU: their outputs (ng%p, ng%n, pl in
 * face / cell order) go straight to solv_gpu_matrix_values_dev.
 *
 * Every output is bit-for-bit the host restatement's (fvmesh.h): face terms
 * use the same operations in the same order without fused multiply-adds,
 * and each cell adds its faces' contributions in ascending face order, the
 * order in which the reference's face loop adds them.
 *
 * Layouts: ip / in 1-based, in = 0 on boundary faces; cell vectors with 3
 * components are cell-major (u[3*c + k]); gradients are 3 per component
 * (grad[(c*ncomp + k)*3 + d]).  All array arguments of the operations are
 * DEVICE pointers; the geometry given to fv_gpu_create is host memory,
 * copied once.  Functions return 0 on success, SOLV_GPU_* codes otherwise.
 */
#ifndef FV_GPU_H
#define FV_GPU_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct fv_gpu fv_gpu;

/* Mesh and geometry (host arrays): n_face faces (interior and boundary),
 * area, unit normal (3 per face, outward from ip), face centre (3 per
 * face), l_pn, w_fp per face; cell centre (3 per cell) and volume.
 * No counterpart in the reference: it keeps these in module globals
 * (grd_geom.f90). */
int fv_gpu_create(fv_gpu **out, int device, int n_cell, int n_face, const int *ip,
                  const int *in, const double *area, const double *nrm, const double *xf,
                  const double *l_pn, const double *w_fp, const double *xc,
                  const double *vol);
int fv_gpu_destroy(fv_gpu *fv);
/* Run on a caller stream (a cudaStream_t); NULL = the default stream. */
int fv_gpu_set_stream(fv_gpu *fv, void *stream);

/* Momentum matrix (cfd_setup.f90:178-431, 473-518): upwind convection of
 * the face flux (flux, or NULL = rho area u_f.n from the linearly
 * interpolated u), central diffusion d = mu area / l_pn, no-slip walls, the
 * y = 1 wall moving with (u_lid, 0, 0), under-relaxation urf:
 * p = -d + min(F,0), n = -d - max(F,0), pl = (-sum off-diagonals) / urf;
 * rhs (3 per cell, may be NULL) gets the lid terms and (1-urf) pl u;
 * flux_out (may be NULL) the face fluxes used. */
int fv_gpu_momentum(fv_gpu *fv, const double *u, const double *flux, double rho, double mu,
                    double u_lid, double urf, double *p, double *n, double *pl, double *rhs,
                    double *flux_out);
/* Pressure-correction matrix (cfd_setup.f90:604-634):
 * d = rho (1/a_P)_f area V_f / l_pn, p = n = -d, pl = sum d, all-Neumann
 * walls; cell `pin` (1-based, 0 for none) pinned by zeroing the
 * off-diagonals of its faces. */
int fv_gpu_pressure_correction(fv_gpu *fv, const double *ap, double rho, int pin, double *p,
                               double *n, double *pl);
/* Green-Gauss gradient (solv_grad, cfd_setup.f90:765-866, one sweep) of
 * ncomp components per cell (phi[c*ncomp + k]). */
int fv_gpu_gradient(fv_gpu *fv, int ncomp, const double *phi, double *grad);
/* Face mass fluxes with Rhie-Chow pressure smoothing (cfd_setup.f90:615-634). */
int fv_gpu_face_flux(fv_gpu *fv, const double *u, const double *p, const double *gradp,
                     const double *ap, double rho, double *flux);
/* The same with the pressures taken at the face's auxiliary points,
 * p_P + grad(p)_P . dx_P, as the reference's pressure-correction face loop
 * does (cfd_setup.f90:611-620); bit-for-bit fvm_face_flux_aux. */
int fv_gpu_face_flux_aux(fv_gpu *fv, const double *u, const double *p, const double *gradp,
                         const double *ap, double rho, double *flux);
/* solv_grad in full (cfd_setup.f90:765-866): n_iter Green-Gauss sweeps,
 * the later ones with the face values moved to the auxiliary points by the
 * previous sweep's gradient; walls by neu (0 the values bval[f*ncomp + k],
 * 1 the cell value, 2 the cell value extrapolated with the previous
 * gradient); bit-for-bit fvm_gradient_sweeps. */
int fv_gpu_gradient_sweeps(fv_gpu *fv, int ncomp, const double *phi, const double *bval,
                           int n_iter, int neu, double *grad);
/* The explicit momentum terms (cfd_setup.f90:185-272, 306-328), added to
 * rhs: deferred correction toward the face value of `scheme` (0 central,
 * 1 min-mod, 2 van Leer, 3 superbee) on the auxiliary-point values,
 * blended by c_bl, and the non-orthogonal diffusion correction;
 * bit-for-bit fvm_momentum_deferred. */
int fv_gpu_momentum_deferred(fv_gpu *fv, int ncomp, const double *phi, const double *grad,
                             const double *flux, double mu, double c_bl, int scheme,
                             double *rhs);
/* Mass imbalance b_i = -(net outflow of cell i), b = 0 at cell `pin`;
 * *total (host) = sum |b| (a deterministic tree sum). */
int fv_gpu_mass_imbalance(fv_gpu *fv, const double *flux, int pin, double *b, double *total);
/* SIMPLE corrections with the pressure correction pp: p += urf_p pp,
 * u -= (V / a_P) grad(pp), F -= d (pp_N - pp_P). */
int fv_gpu_simple_correct(fv_gpu *fv, const double *pp, const double *gradpp, const double *ap,
                          double rho, double urf_p, double *u, double *p, double *flux);

#ifdef __cplusplus
}
#endif
#endif
