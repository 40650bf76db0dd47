/*
 * Test infrastructure only (oracle build): never linked into the product.
 *
 * Harness around the reference compiled from its own, unmodified sources into
 * oracle/_ref/libkfun3d_ref.so.  It adds what the reference cannot do from its
 * command line:
 *   - ref_set_aoa: the angle of attack, a compile-time macro in inc/phy.h:8-9,
 *     becomes a run-time setting through oracle/shadow/phy.h;
 *   - ref_setup / ref_free: src/mesh.c:22-154 Setup for any mesh path and
 *     thread count, and the teardown of src/main.c:65-122;
 *   - ref_solve: the Newton/SER + left-preconditioned GMRES driver of
 *     src/kernel.c:47-232, restated with its #define constants
 *     (src/kernel.c:12-22) turned into parameters, recording every step.
 *     With the default parameters it follows kernel.c statement for statement,
 *     so its history is bit-identical to the unmodified binary's.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "geometry.h"
#include "core_kernel.h"
#include "utils.h"

extern void Setup(const char *, GEOMETRY *);
extern void CXX_Matrix_Delete(void *ptr);
extern void iJacVec(const GEOMETRY *g, const double *x, const double *r,
                    const double norm, GRADIENT *grad, double *w, double *y);
extern void fun3d_init_log(void);

double kf_ref_phy_u = 0.99862953475457383;  /* cos(3 deg), replaced by ref_set_aoa */
double kf_ref_phy_v = 0.052335956242943835; /* sin(3 deg) */

/* inc/phy.h:8-9: U = cos(a / (180 / M_PI)), V = sin(a / (180 / M_PI)). */
void ref_set_aoa(double deg)
{
  kf_ref_phy_u = cos(deg / (180 / M_PI));
  kf_ref_phy_v = sin(deg / (180 / M_PI));
}

void ref_get_uv(double *u, double *v)
{
  *u = kf_ref_phy_u;
  *v = kf_ref_phy_v;
}

static int log_ready = 0;

GEOMETRY *ref_setup(const char *path, int threads)
{
  if (!log_ready) { fun3d_init_log(); log_ready = 1; }
  omp_set_num_threads(threads);
  GEOMETRY *g = (GEOMETRY *) calloc(1, sizeof(GEOMETRY));
  Setup(path, g);
  return g;
}

/* Mirrors the teardown in src/main.c:65-122. */
void ref_free(GEOMETRY *g)
{
  if (!g) return;
  free(g->e->xyzn->x0); free(g->e->xyzn->x1); free(g->e->xyzn->x2); free(g->e->xyzn->x3);
  free(g->e->xyzn);
  free(g->e->w->w0->x0); free(g->e->w->w0->x1); free(g->e->w->w0->x2); free(g->e->w->w0);
  free(g->e->w->w1->x0); free(g->e->w->w1->x1); free(g->e->w->w1->x2); free(g->e->w->w1);
  free(g->e->w);
  free(g->e->eptr->n0); free(g->e->eptr->n1); free(g->e->eptr); free(g->e);
  free(g->s->i); free(g->s); free(g->t->i); free(g->t);
  free(g->c);
  free(g->b->s->xyz->x0); free(g->b->s->xyz->x1); free(g->b->s->xyz->x2); free(g->b->s->xyz);
  free(g->b->s->nptr); free(g->b->s);
  free(g->b->f->xyz->x0); free(g->b->f->xyz->x1); free(g->b->f->xyz->x2); free(g->b->f->xyz);
  free(g->b->f->nptr); free(g->b->f);
  free(g->b->fc->fptr->n0); free(g->b->fc->fptr->n1); free(g->b->fc->fptr->n2);
  free(g->b->fc->fptr); free(g->b->fc); free(g->b);
  free(g->n->xyz->x0); free(g->n->xyz->x1); free(g->n->xyz->x2); free(g->n->xyz);
  free(g->n->cdt); free(g->n->part); free(g->n);
  free(g->q->q); free(g->q);
  CXX_Matrix_Delete(g->matrix);
  free(g);
}

typedef struct {
  int ts_max;           /* TS_MAX 15 */
  double stop_ratio;    /* FNORM_MAX 1e7: stop once round(|r0|/|r|) >= stop_ratio */
  double gmres_rtol;    /* GMRES_RELATIVE_TOLERANCE 0.01 */
  int gmres_restart;    /* GMRES_RESTART 30 (<= 30) */
  int gmres_max_it;     /* GMRES_MAX_IT 10000 */
  double cfl_init;      /* CFL_INIT 50 */
  double cfl_max;       /* CLF_MAX 100000 */
} ref_params;

typedef struct {
  int step;
  int gmres_its;
  double cfl;
  double fnorm;
  double lift, drag, momn;
} ref_step;

#define KF_BASIS 31

/* src/kernel.c:47-232 with parameters; returns the number of steps recorded. */
int ref_solve(GEOMETRY *g, const ref_params *p, ref_step *hist, int max_hist)
{
  const size_t sz = g->c->sz;
  GRADIENT grad;
  grad.x0 = (double *) calloc(sz, sizeof(double));
  grad.x1 = (double *) calloc(sz, sizeof(double));
  grad.x2 = (double *) calloc(sz, sizeof(double));
  double *x = (double *) calloc(sz, sizeof(double));
  double *r = (double *) calloc(sz, sizeof(double));
  double *w = (double *) calloc(sz, sizeof(double));
  double *t = (double *) calloc(sz, sizeof(double));
  double *ghh = (double *) calloc(KF_BASIS * KF_BASIS, sizeof(double));
  double *vecs[KF_BASIS];
  for (int v = 0; v < KF_BASIS; v++) vecs[v] = (double *) calloc(sz, sizeof(double));
  double cc[KF_BASIS], ss[KF_BASIS], rs[KF_BASIS];
  double forces[3];
  const unsigned int restart = (unsigned int) p->gmres_restart;

  double fnorm_init = 0.f;
  double cfl = p->cfl_init;
  int nrec = 0;

  uint32_t its = 0;
  while (its < (uint32_t) p->ts_max) {
    ComputeFlux(g, g->q->q, &grad, r);
    double fnorm = Compute2ndNorm(sz, r);
    if (its == 0) fnorm_init = fnorm;
    else {
      double cfl0 = 1.1 * p->cfl_init * fnorm_init;
      cfl0 /= fnorm;
      cfl = (cfl0 < p->cfl_max) ? cfl0 : p->cfl_max;
    }
    ComputeTimeStep(cfl, g);
    ComputeA(g);
    double qnorm = sqrt(1.f + Compute2ndNorm(sz, g->q->q));
    memset(x, 0, sz * sizeof(double));
    ComputeNumericalILU(g);
    ComputeSparseTriangularSolve(g, r, vecs[0]);

    double tol = 0.f;
    uint32_t total = 0;
    unsigned int flag = 0;
    while (total <= (uint32_t) p->gmres_max_it) {
      if (total > 0) {
        iJacVec(g, x, r, qnorm, &grad, w, t);
        ComputeNewAXPY(sz, -1.f, t, r, w);
        ComputeSparseTriangularSolve(g, w, vecs[0]);
      }
      rs[0] = Normalize(sz, vecs[0]);
      tol = (total == 0) ? p->gmres_rtol * rs[0] : tol;
      uint32_t k = 0;
      while (k < restart) {
        iJacVec(g, vecs[k], r, qnorm, &grad, w, t);
        ComputeSparseTriangularSolve(g, t, vecs[1 + k]);
        double *hh = ghh + k * (KF_BASIS + 1);
        for (unsigned int v = 0; v < k + 1; v++) {
          double dot = 0.f;
#pragma omp parallel for reduction(+ : dot)
          for (size_t i = 0; i < sz; i++) dot += vecs[k + 1][i] * vecs[v][i];
          hh[v] = dot;
          ComputeAXPY(sz, -hh[v], vecs[v], vecs[k + 1]);
        }
        hh[k + 1] = Normalize(sz, vecs[1 + k]);
        for (unsigned int i = 0; i < k; i++) {
          const double tt = *hh;
          *hh = cc[i] * *hh + ss[i] * *(hh + 1);
          hh++;
          *hh = cc[i] * *hh - ss[i] * tt;
        }
        const double tt = sqrt(*hh * *hh + *(hh + 1) * *(hh + 1));
        double c = *hh / tt;
        double s = *(hh + 1) / tt;
        cc[k] = c;
        ss[k] = s;
        rs[k + 1] = -(s * rs[k]);
        rs[k] = c * rs[k];
        *hh = c * *hh + s * *(hh + 1);
        const double res = fabs(rs[k + 1]);
        k++;
        if (res <= tol) { flag = 1; break; }
      }
      total += k;
      rs[k - 1] /= ghh[(k - 1) * (KF_BASIS + 1) + (k - 1)];
      for (unsigned int i = 1; i <= k - 1; i++) {
        uint32_t m = (k - 1) - i;
        double tt = rs[m];
        for (unsigned int j = m + 1; j <= k - 1; j++) tt -= ghh[j * (KF_BASIS + 1) + m] * rs[j];
        rs[m] = tt / ghh[m * (KF_BASIS + 1) + m];
      }
      for (unsigned int v = 0; v < k; v++) ComputeAXPY(sz, rs[v], vecs[v], x);
      if (flag) break;
    }

    ComputeAXPY(sz, -1.f, x, g->q->q);
    ComputeForces(g, forces);
    if (nrec < max_hist) {
      hist[nrec].step = (int) its;
      hist[nrec].gmres_its = (int) total;
      hist[nrec].cfl = cfl;
      hist[nrec].fnorm = fnorm;
      hist[nrec].lift = forces[0];
      hist[nrec].drag = forces[1];
      hist[nrec].momn = forces[2];
      nrec++;
    }
    /* kernel.c:214 casts round(...) to uint32_t; the ratio is compared as a
       double here so ratios above 2^32 cannot wrap around. */
    if (round(fnorm_init / fnorm) >= p->stop_ratio) break;
    its++;
  }

  free(grad.x0); free(grad.x1); free(grad.x2);
  free(x); free(r); free(w); free(t); free(ghh);
  for (int v = 0; v < KF_BASIS; v++) free(vecs[v]);
  return nrec;
}
