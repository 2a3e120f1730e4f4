/*
 * csr_oracle.c -- independent restatement of the CSR twin of the spray
 * solvers, pcns/src/solv_m.f90 (TEST INFRASTRUCTURE ONLY).
 *
 * pcns runs the same DILU-preconditioned CG and right-preconditioned
 * BiCGSTAB on CSR storage.  Used only to cross-check solv_oracle.c: both
 * must converge to the same solution of the same system.  Differences from
 * the face-addressed code are kept as pcns has them (beta = 1/(s+small),
 * (v+small)^2 in the BiCGSTAB denominator, the preconditioner is always
 * DILU).  Index arrays are 1-based (Fortran CSR), rows sorted by column.
 */
#include "solv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SMALL 1e-20
#define LARGE 1e20

/* matrix_utils_m.f90:74-89 csr_matvec_prod */
static void csr_matvec(int n, const int *ia, const int *ja, const double *a,
                       const double *x, double *y) {
  for (int i = 1; i <= n; ++i) {
    double s = 0.0;
    for (int k = ia[i - 1]; k <= ia[i] - 1; ++k) s = s + a[k - 1] * x[ja[k - 1] - 1];
    y[i - 1] = s;
  }
}

/* matrix_utils_m.f90:57-70 csr_index (returns 1-based k, or -1) */
static int csr_index(int i, int j, const int *ia, const int *ja) {
  for (int k = ia[i - 1]; k <= ia[i] - 1; ++k)
    if (ja[k - 1] == j) return k;
  return -1;
}

/* vector_utils_m.f90:8-13 p_norm with p=1 */
static double p1_norm(int n, const double *v) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + fabs(v[i]);
  return s;
}

/* solv_m.f90:209-238 preconditioner (DILU diagonal, stored inverted) */
static void csr_precond(int n, const int *ia, const int *ja, const double *a,
                        double *c) {
  for (int i = 1; i <= n; ++i) {
    int kii = csr_index(i, i, ia, ja);
    double summ = a[kii - 1];
    for (int kij = ia[i - 1]; kij <= ia[i] - 1; ++kij) {
      int j = ja[kij - 1];
      if (j < i) {
        int kji = csr_index(j, i, ia, ja);
        summ = summ - a[kij - 1] * c[j - 1] * a[kji - 1];
      } else {
        break;
      }
    }
    c[i - 1] = 1.0 / (summ + SMALL);
  }
}

/* solv_m.f90:243-289 direct_solve */
static void csr_direct(int n, const int *ia, const int *ja, const double *a,
                       const double *c, const double *b, double *x) {
  for (int i = 1; i <= n; ++i) {
    double summ = b[i - 1];
    for (int kij = ia[i - 1]; kij <= ia[i] - 1; ++kij) {
      int j = ja[kij - 1];
      if (j < i) summ = summ - a[kij - 1] * x[j - 1];
      else break;
    }
    x[i - 1] = summ * c[i - 1];
  }
  for (int i = 1; i <= n; ++i) {
    double cof = 1.0 / (c[i - 1] + SMALL);
    x[i - 1] = cof * x[i - 1];
  }
  for (int i = n; i >= 1; --i) {
    double summ = x[i - 1];
    for (int kij = ia[i] - 1; kij >= ia[i - 1]; --kij) {
      int j = ja[kij - 1];
      if (j > i) summ = summ - a[kij - 1] * x[j - 1];
      else break;
    }
    x[i - 1] = summ * c[i - 1];
  }
}

static double dotp(int n, const double *a, const double *b) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

/* solv_m.f90:32-105 cg_solver */
int csr_cg_solver(int n, const int *ia, const int *ja, const double *a,
                  double *phi, double *res, double *norm, int n_iter,
                  double reduc) {
  double *wk = (double *)calloc((size_t)n * 6, sizeof(double));
  double *w1 = wk, *w2 = wk + n, *w3 = wk + 2 * (size_t)n, *w6 = wk + 5 * (size_t)n;
  double cof[6] = {0, 0, 0, 0, 0, 0};
  csr_matvec(n, ia, ja, a, phi, w1);
  for (int i = 0; i < n; ++i) res[i] = res[i] - w1[i];
  *norm = p1_norm(n, res);
  double norm0 = *norm;
  csr_precond(n, ia, ja, a, w6);
  cof[3] = LARGE;
  memcpy(w1, res, sizeof(double) * (size_t)n);
  memset(w2, 0, sizeof(double) * 2 * (size_t)n);
  int iter;
  for (iter = 1; iter <= n_iter; ++iter) {
    cof[0] = 0;
    csr_direct(n, ia, ja, a, w6, w1, w3);
    cof[2] = 1.0 / (cof[3] + SMALL);
    cof[3] = dotp(n, w1, w3);
    cof[2] = cof[2] * cof[3];
    for (int i = 0; i < n; ++i) w2[i] = w3[i] + cof[2] * w2[i];
    csr_matvec(n, ia, ja, a, w2, w3);
    cof[1] = dotp(n, w2, w3);
    cof[1] = cof[3] / (cof[1] + SMALL);
    for (int i = 0; i < n; ++i) phi[i] = phi[i] + cof[1] * w2[i];
    for (int i = 0; i < n; ++i) w1[i] = w1[i] - cof[1] * w3[i];
    *norm = p1_norm(n, w1);
    cof[0] = *norm / (norm0 + SMALL);
    if (cof[0] < reduc) break;
  }
  free(wk);
  return iter > n_iter ? n_iter : iter;
}

/* solv_m.f90:110-204 bicg_solver */
int csr_bicg_solver(int n, const int *ia, const int *ja, const double *a,
                    double *phi, double *res, double *norm, int n_iter,
                    double reduc) {
  double *wk = (double *)calloc((size_t)n * 6, sizeof(double));
  double *w1 = wk, *w2 = wk + n, *w3 = wk + 2 * (size_t)n, *w4 = wk + 3 * (size_t)n,
         *w5 = wk + 4 * (size_t)n, *w6 = wk + 5 * (size_t)n;
  double cof[6];
  csr_matvec(n, ia, ja, a, phi, w1);
  for (int i = 0; i < n; ++i) res[i] = res[i] - w1[i];
  *norm = p1_norm(n, res);
  double norm0 = *norm;
  csr_precond(n, ia, ja, a, w6);
  for (int k = 0; k < 6; ++k) cof[k] = 0;
  cof[1] = cof[2] = 1;
  cof[4] = 1;
  memcpy(w1, res, sizeof(double) * (size_t)n);
  memset(w2, 0, sizeof(double) * 4 * (size_t)n);
  int iter;
  for (iter = 1; iter <= n_iter; ++iter) {
    cof[0] = 0;
    cof[3] = dotp(n, w1, res);
    cof[5] = cof[3] * cof[4] / (cof[1] * cof[2] + SMALL);
    cof[2] = cof[3];
    for (int i = 0; i < n; ++i) w2[i] = w1[i] + cof[5] * (w2[i] - cof[1] * w3[i]);
    csr_direct(n, ia, ja, a, w6, w2, w5);
    csr_matvec(n, ia, ja, a, w5, w3);
    cof[4] = dotp(n, w3, res);
    cof[4] = cof[3] / (cof[4] + SMALL);
    for (int i = 0; i < n; ++i) phi[i] = phi[i] + cof[4] * w5[i];
    for (int i = 0; i < n; ++i) w1[i] = w1[i] - cof[4] * w3[i];
    csr_direct(n, ia, ja, a, w6, w1, w5);
    csr_matvec(n, ia, ja, a, w5, w4);
    cof[0] = cof[1] = 0;
    for (int i = 0; i < n; ++i) {
      cof[0] = cof[0] + w4[i] * w1[i];
      cof[1] = cof[1] + (w4[i] + SMALL) * (w4[i] + SMALL);
    }
    cof[1] = cof[0] / (cof[1] + SMALL);
    for (int i = 0; i < n; ++i) phi[i] = phi[i] + cof[1] * w5[i];
    for (int i = 0; i < n; ++i) w1[i] = w1[i] - cof[1] * w4[i];
    *norm = p1_norm(n, w1);
    cof[0] = *norm / (norm0 + SMALL);
    if (cof[0] < reduc) break;
  }
  free(wk);
  return iter > n_iter ? n_iter : iter;
}
