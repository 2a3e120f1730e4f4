/*
 * solv_oracle.c -- line-faithful CPU restatement of the spray-simulation
 * linear-solver hot path (TEST INFRASTRUCTURE ONLY: the oracle the GPU
 * path is tested against and the single-core CPU baseline, never linked
 * into the product library).
 *
 * Each routine follows the Fortran loop order statement by statement so
 * that floating-point results match a gfortran build without -ffast-math:
 * sequential dot products / sums in cell order, face order for the matrix
 * products, ascending / descending cell order for the sweeps.  Build with
 * -O2 -ffp-contract=off (no FMA contraction, no reassociation).
 *
 * Parity unpinned by the reference (no Fortran compiler; no golden vectors
 * in the reference) -- cross-checked against scipy, the CSR twin below and
 * manufactured solutions by the tests.
 */
#include "solv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SMALL 1e-20 /* precision.f90:8  small = ten**(-20) */
#define LARGE 1e20  /* precision.f90:9  large = one/small  */

/* ------------------------------------------------------------------ */
/* v_lst construction: grd_conn.f90:128-152 (volume face lists, faces  */
/* appended in ascending global face order to owner then neighbour) and */
/* grd_conn.f90:218-238 (neighbour list = the other cell of the face).  */
/* ------------------------------------------------------------------ */
int orc_vlst_size(int n_cell, int n_face, const int *ip, const int *in) {
  long total = 0;
  for (int f = 0; f < n_face; ++f) {
    if (ip[f] < 1 || ip[f] > n_cell || in[f] < 0 || in[f] > n_cell) return -1;
    total += 1 + (in[f] > 0);
  }
  (void)n_cell;
  return (int)total;
}

int orc_build_vlst(int n_cell, int n_face, const int *ip, const int *in,
                   int *v_ptr, int *v_fce, int *v_ng) {
  int total = orc_vlst_size(n_cell, n_face, ip, in);
  if (total < 0) return -1;
  memset(v_ptr, 0, sizeof(int) * (size_t)(n_cell + 1));
  for (int f = 0; f < n_face; ++f) {
    v_ptr[ip[f]] += 1;
    if (in[f] > 0) v_ptr[in[f]] += 1;
  }
  for (int i = 0; i < n_cell; ++i) v_ptr[i + 1] += v_ptr[i];
  int *fill = (int *)malloc(sizeof(int) * (size_t)(n_cell > 0 ? n_cell : 1));
  for (int i = 0; i < n_cell; ++i) fill[i] = v_ptr[i];
  for (int f = 0; f < n_face; ++f) {
    int a = ip[f] - 1;
    v_fce[fill[a]] = f + 1;
    v_ng[fill[a]] = in[f] > 0 ? in[f] : 0; /* c_neig_lst: other cell */
    fill[a]++;
    if (in[f] > 0) {
      int b = in[f] - 1;
      v_fce[fill[b]] = f + 1;
      v_ng[fill[b]] = ip[f];
      fill[b]++;
    }
  }
  free(fill);
  return total;
}

/* ------------------------------------------------------------------ */
/* solv_res.f90:5-30                                                   */
/* ------------------------------------------------------------------ */
void orc_solv_res(const orc_matrix *m, int n_vc, const double *phi,
                  double *res0, double *res0_n, int not_r0) {
  const int N = m->n_cell;
  if (!not_r0) {
    /* :13-15  res0(ip,:)=res0(ip,:)-pl(ip)*phi(ip)%vc */
    for (int ip = 0; ip < N; ++ip)
      for (int v = 0; v < n_vc; ++v)
        res0[(size_t)v * N + ip] =
            res0[(size_t)v * N + ip] - m->pl[ip] * phi[(size_t)ip * n_vc + v];
    /* :16-23  face loop */
    for (int f = 0; f < m->n_face; ++f) {
      if (m->in[f] > 0) {
        int a = m->ip[f] - 1, b = m->in[f] - 1;
        for (int v = 0; v < n_vc; ++v)
          res0[(size_t)v * N + a] =
              res0[(size_t)v * N + a] - m->p[f] * phi[(size_t)b * n_vc + v];
        for (int v = 0; v < n_vc; ++v)
          res0[(size_t)v * N + b] =
              res0[(size_t)v * N + b] - m->n[f] * phi[(size_t)a * n_vc + v];
      }
    }
  }
  /* :26-29  res0_n = sum over cells of |res0| */
  for (int v = 0; v < n_vc; ++v) res0_n[v] = 0.0;
  for (int ip = 0; ip < N; ++ip)
    for (int v = 0; v < n_vc; ++v)
      res0_n[v] = res0_n[v] + fabs(res0[(size_t)v * N + ip]);
}

/* ------------------------------------------------------------------ */
/* solv_precond.f90:5-30                                               */
/* ------------------------------------------------------------------ */
void orc_solv_precond(const orc_matrix *m, int imat, double *c, double *c_r) {
  const int N = m->n_cell;
  for (int ip = 0; ip < N; ++ip) {
    c[ip] = m->pl[ip];
    if (imat > 0) {
      for (int k = m->v_ptr[ip]; k < m->v_ptr[ip + 1]; ++k) {
        int in = m->v_ng[k]; /* 1-based, 0 = none */
        if (in > 0 && in < ip + 1) {
          int f = m->v_fce[k] - 1;
          if (imat == 1) {
            c[ip] = c[ip] - (m->n[f] * m->n[f]) * c[in - 1]; /* :19 */
          } else if (imat == 2) {
            c[ip] = c[ip] - m->p[f] * c[in - 1] * m->n[f]; /* :21 */
          }
        }
      }
    }
    c_r[ip] = c[ip];                 /* :27 */
    c[ip] = 1.0 / (c[ip] + SMALL);   /* :28 */
  }
}

/* ------------------------------------------------------------------ */
/* solv_direct.f90:5-43                                                */
/* ------------------------------------------------------------------ */
void orc_solv_direct(const orc_matrix *m, int imat, const double *c,
                     const double *c_r, double *x, const double *b) {
  const int N = m->n_cell;
  if (imat > 0) {
    for (int ip = 0; ip < N; ++ip) { /* :12-24 forward */
      x[ip] = b[ip];
      for (int k = m->v_ptr[ip]; k < m->v_ptr[ip + 1]; ++k) {
        int in = m->v_ng[k];
        if (in > 0 && in < ip + 1) {
          int f = m->v_fce[k] - 1;
          x[ip] = x[ip] - m->n[f] * x[in - 1];
        }
      }
      x[ip] = x[ip] * c[ip];
    }
    for (int ip = 0; ip < N; ++ip) x[ip] = x[ip] * c_r[ip]; /* :26 */
    for (int ip = N - 1; ip >= 0; --ip) {                  /* :28-38 */
      for (int k = m->v_ptr[ip]; k < m->v_ptr[ip + 1]; ++k) {
        int in = m->v_ng[k];
        if (in > 0 && in > ip + 1) {
          int f = m->v_fce[k] - 1;
          x[ip] = x[ip] - m->p[f] * x[in - 1];
        }
      }
      x[ip] = x[ip] * c[ip];
    }
  } else {
    for (int ip = 0; ip < N; ++ip) x[ip] = b[ip] * c[ip]; /* :41 */
  }
}

/* ------------------------------------------------------------------ */
/* face-loop matrix product, solv_cg.f90:56-64 / solv_bicg.f90:61-69    */
/* ------------------------------------------------------------------ */
void orc_spmv(const orc_matrix *m, const double *x, double *y) {
  const int N = m->n_cell;
  for (int ip = 0; ip < N; ++ip) y[ip] = m->pl[ip] * x[ip];
  for (int f = 0; f < m->n_face; ++f) {
    if (m->in[f] > 0) {
      int a = m->ip[f] - 1, b = m->in[f] - 1;
      y[a] = y[a] + m->p[f] * x[b];
      y[b] = y[b] + m->n[f] * x[a];
    }
  }
}

static double dot_product(int n, const double *a, const double *b) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

static double sum_abs(int n, const double *a) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + fabs(a[i]);
  return s;
}

/* ------------------------------------------------------------------ */
/* solv_cg.f90:7-87                                                    */
/* ------------------------------------------------------------------ */
void orc_solv_cg(const orc_matrix *m, int imat, double reduc, int n_iter,
                 int n_vc, double *phi, double *res0, double *res0_n,
                 int not_r0, int *iters, double *ratio) {
  const int N = m->n_cell;
  double w_sc[4];
  for (int v = 0; v < n_vc; ++v) {
    if (iters) iters[v] = 0;
    if (ratio) ratio[v] = 0.0;
  }

  orc_solv_res(m, n_vc, phi, res0, res0_n, not_r0); /* :20 */
  double mx = -HUGE_VAL;
  for (int v = 0; v < n_vc; ++v) mx = res0_n[v] > mx ? res0_n[v] : mx;
  if (mx < SMALL) return; /* :21 */

  double *c = (double *)malloc(sizeof(double) * (size_t)N);
  double *c_r = (double *)malloc(sizeof(double) * (size_t)N);
  double *w1 = (double *)malloc(sizeof(double) * (size_t)N); /* res */
  double *w2 = (double *)malloc(sizeof(double) * (size_t)N); /* p   */
  double *w3 = (double *)malloc(sizeof(double) * (size_t)N); /* z   */
  orc_solv_precond(m, imat, c, c_r); /* :24 */

  for (int ivc = 0; ivc < n_vc; ++ivc) {
    w_sc[0] = w_sc[1] = w_sc[2] = 0.0; /* :29 */
    w_sc[3] = LARGE;
    memcpy(w1, res0 + (size_t)ivc * N, sizeof(double) * (size_t)N); /* :32 */
    memset(w2, 0, sizeof(double) * (size_t)N);
    memset(w3, 0, sizeof(double) * (size_t)N);
    int num = 0;
    double last = 0.0;
    for (int iter = 1; iter <= n_iter; ++iter) {
      num = num + 1;
      orc_solv_direct(m, imat, c, c_r, w3, w1); /* :41 */
      w_sc[2] = 1.0 / w_sc[3];                  /* :44 */
      w_sc[3] = dot_product(N, w1, w3);         /* :47 */
      w_sc[2] = w_sc[2] * w_sc[3];              /* :50 */
      for (int i = 0; i < N; ++i) w2[i] = w3[i] + w_sc[2] * w2[i]; /* :53 */
      orc_spmv(m, w2, w3);                      /* :56-64 */
      w_sc[1] = dot_product(N, w2, w3);         /* :67 */
      w_sc[1] = w_sc[3] / (w_sc[1] + SMALL);    /* :68 */
      for (int i = 0; i < N; ++i)               /* :73-76 */
        phi[(size_t)i * n_vc + ivc] = phi[(size_t)i * n_vc + ivc] + w_sc[1] * w2[i];
      for (int i = 0; i < N; ++i) w1[i] = w1[i] - w_sc[1] * w3[i]; /* :77 */
      w_sc[0] = sum_abs(N, w1);                         /* :78 */
      w_sc[0] = w_sc[0] / (res0_n[ivc] + SMALL);        /* :81 */
      last = w_sc[0];
      if (w_sc[0] < reduc) break;                       /* :82 */
      w_sc[0] = 0.0;
    }
    if (iters) iters[ivc] = num;
    if (ratio) ratio[ivc] = last;
  }
  free(c); free(c_r); free(w1); free(w2); free(w3);
}

/* ------------------------------------------------------------------ */
/* solv_bicg.f90:7-121                                                 */
/* ------------------------------------------------------------------ */
void orc_solv_bicg(const orc_matrix *m, int imat, double reduc, int n_iter,
                   int n_vc, double *phi, double *res0, double *res0_n,
                   int not_r0, int *iters, double *ratio) {
  const int N = m->n_cell;
  /* w_sc: res_n=0 alpha=1 beta0=2 beta=3 gam=4 omeg=5 (0-based) */
  double w_sc[6];
  for (int v = 0; v < n_vc; ++v) {
    if (iters) iters[v] = 0;
    if (ratio) ratio[v] = 0.0;
  }

  orc_solv_res(m, n_vc, phi, res0, res0_n, not_r0); /* :20 */
  double mx = -HUGE_VAL;
  for (int v = 0; v < n_vc; ++v) mx = res0_n[v] > mx ? res0_n[v] : mx;
  if (mx < SMALL) return; /* :21 */

  double *c = (double *)malloc(sizeof(double) * (size_t)N);
  double *c_r = (double *)malloc(sizeof(double) * (size_t)N);
  double *w[5];
  for (int k = 0; k < 5; ++k) w[k] = (double *)malloc(sizeof(double) * (size_t)N);
  double *res = w[0], *p = w[1], *u = w[2], *vv = w[3], *z = w[4];
  orc_solv_precond(m, imat, c, c_r); /* :24 */

  for (int ivc = 0; ivc < n_vc; ++ivc) {
    const double *r0 = res0 + (size_t)ivc * N;
    for (int k = 0; k < 6; ++k) w_sc[k] = 0.0; /* :31-33 */
    w_sc[1] = w_sc[2] = 1.0;
    w_sc[4] = 1.0;
    memcpy(res, r0, sizeof(double) * (size_t)N); /* :37 */
    for (int k = 1; k < 5; ++k) memset(w[k], 0, sizeof(double) * (size_t)N);
    int num = 0;
    double last = 0.0;
    for (int iter = 1; iter <= n_iter; ++iter) {
      num = num + 1;
      w_sc[3] = dot_product(N, res, r0);                               /* :48 */
      w_sc[5] = w_sc[3] * w_sc[4] / (w_sc[1] * w_sc[2] + SMALL);       /* :49 */
      w_sc[2] = w_sc[3];                                               /* :50 */
      for (int i = 0; i < N; ++i)                                      /* :54-55 */
        p[i] = res[i] + w_sc[5] * (p[i] - w_sc[1] * u[i]);
      orc_solv_direct(m, imat, c, c_r, z, p);                          /* :58 */
      orc_spmv(m, z, u);                                               /* :61-69 */
      w_sc[4] = dot_product(N, u, r0);                                 /* :72 */
      w_sc[4] = w_sc[3] / (w_sc[4] + SMALL);                           /* :73 */
      for (int i = 0; i < N; ++i)                                      /* :77-80 */
        phi[(size_t)i * n_vc + ivc] = phi[(size_t)i * n_vc + ivc] + w_sc[4] * z[i];
      for (int i = 0; i < N; ++i) res[i] = res[i] - w_sc[4] * u[i];   /* :81 */
      orc_solv_direct(m, imat, c, c_r, z, res);                        /* :84 */
      orc_spmv(m, z, vv);                                              /* :87-95 */
      w_sc[0] = dot_product(N, vv, res);                               /* :98 */
      w_sc[1] = dot_product(N, vv, vv);                                /* :99 */
      w_sc[1] = w_sc[0] / (w_sc[1] + SMALL);                           /* :100 */
      for (int i = 0; i < N; ++i)                                      /* :105-108 */
        phi[(size_t)i * n_vc + ivc] = phi[(size_t)i * n_vc + ivc] + w_sc[1] * z[i];
      for (int i = 0; i < N; ++i) res[i] = res[i] - w_sc[1] * vv[i];  /* :109 */
      w_sc[0] = sum_abs(N, res);                                       /* :110 */
      w_sc[0] = w_sc[0] / (res0_n[ivc] + SMALL);                       /* :115 */
      last = w_sc[0];
      if (w_sc[0] < reduc) break;                                      /* :116 */
      w_sc[0] = 0.0;
    }
    if (iters) iters[ivc] = num;
    if (ratio) ratio[ivc] = last;
  }
  free(c); free(c_r);
  for (int k = 0; k < 5; ++k) free(w[k]);
}
