/*
 * solv_oracle.h -- CPU restatement of the spray-simulation linear solvers.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is compared
 * against (and the timed single-core CPU baseline); no product code links it.
 *
 * Parity status: the reference solver is Fortran 90 and no Fortran compiler
 * exists on either machine, and the reference ships no golden vectors for
 * these routines, so parity is NOT pinned by the reference itself.  The
 * restatement is cross-checked instead against (1) scipy sparse direct
 * solves, (2) an independent restatement of the CSR twin of the same
 * algorithms (pcns/src/solv_m.f90:32-289, csr_oracle.c) and (3)
 * manufactured solutions -- see tests/test_oracle.py.
 *
 * Conventions follow the Fortran exactly:
 *   - cell and face indices are 1-based; ng(f)%in == 0 marks a boundary face;
 *   - phi is cell-major  phi[(ip-1)*n_vc + ivc]   (phi(ip)%vc(ivc));
 *   - res0 is column-major res0[ivc*n_cell + ip-1] (res0(ip,ivc));
 *   - small = 1e-20, large = 1e20 (spray-simulation/precision.f90:8-9).
 */
#ifndef SOLV_ORACLE_H
#define SOLV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Face-addressed matrix: solv_data.f90:6-22 (ng_t, pl, v_lst_t). */
typedef struct {
  int n_cell;           /* size(pl)                                  */
  int n_face;           /* size(ng): interior + boundary faces        */
  const int *ip;        /* ng(:)%ip, 1-based owner                    */
  const int *in;        /* ng(:)%in, 1-based neighbour, 0 = boundary  */
  const double *p;      /* ng(:)%p = A(ip,in)                         */
  const double *n;      /* ng(:)%n = A(in,ip)                         */
  const double *pl;     /* pl(:)   = A(ip,ip)                         */
  const int *v_ptr;     /* n_cell+1 offsets (0-based) into v_fce/v_ng */
  const int *v_fce;     /* v_lst(ip)%fce_lst, 1-based face numbers    */
  const int *v_ng;      /* v_lst(ip)%ng_lst, 1-based cell, 0 = none   */
} orc_matrix;

/* Per-cell face / neighbour lists, built the way grd_conn builds them
 * (grd_conn.f90:129-152 face lists in ascending face order, :218-238
 * neighbour lists).  v_ptr has n_cell+1 entries; v_fce / v_ng have
 * v_ptr[n_cell] entries.  Returns the list length, or -1 on a bad index. */
int orc_build_vlst(int n_cell, int n_face, const int *ip, const int *in,
                   int *v_ptr, int *v_fce, int *v_ng);
int orc_vlst_size(int n_cell, int n_face, const int *ip, const int *in);

/* solv_res.f90:5-30 */
void orc_solv_res(const orc_matrix *m, int n_vc, const double *phi,
                  double *res0, double *res0_n, int not_r0);

/* solv_precond.f90:5-30 */
void orc_solv_precond(const orc_matrix *m, int imat, double *c, double *c_r);

/* solv_direct.f90:5-43 */
void orc_solv_direct(const orc_matrix *m, int imat, const double *c,
                     const double *c_r, double *x, const double *b);

/* y = A x with the face-loop order of solv_cg.f90:56-64. */
void orc_spmv(const orc_matrix *m, const double *x, double *y);

/* solv_cg.f90:7-87.  iters[ivc] / ratio[ivc] (optional, may be NULL)
 * receive the iteration count and the last |r|_1/|r0|_1 per component. */
void orc_solv_cg(const orc_matrix *m, int imat, double reduc, int n_iter,
                 int n_vc, double *phi, double *res0, double *res0_n,
                 int not_r0, int *iters, double *ratio);

/* solv_bicg.f90:7-121 */
void orc_solv_bicg(const orc_matrix *m, int imat, double reduc, int n_iter,
                   int n_vc, double *phi, double *res0, double *res0_n,
                   int not_r0, int *iters, double *ratio);

/* Independent CSR restatement of pcns/src/solv_m.f90 (cg_solver :32-105,
 * bicg_solver :110-204, preconditioner :209-238, direct_solve :243-289).
 * Rows sorted by column (csr_index / "exit" loops need that), 1-based
 * ja / ia as in Fortran.  One right-hand side.  Returns iterations. */
int csr_cg_solver(int n, const int *ia, const int *ja, const double *a,
                  double *phi, double *res, double *norm, int n_iter,
                  double reduc);
int csr_bicg_solver(int n, const int *ia, const int *ja, const double *a,
                    double *phi, double *res, double *norm, int n_iter,
                    double reduc);

#ifdef __cplusplus
}
#endif
#endif
