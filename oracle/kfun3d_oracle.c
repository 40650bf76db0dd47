/*
 * Test infrastructure only: the CPU oracle for the kfun3d_b200 hot path.
 *
 * Restates the reference's kernels at one OpenMP thread.  Each routine names
 * the reference lines it follows.  The arithmetic is kept in the reference's
 * operation order (same parenthesisation, no contraction: built with
 * -ffp-contract=off) because bit-identical results are the point; everything
 * else (data layout, loop structure, helpers) is this file's own.
 *
 * Constants of inc/phy.h: B = 15 (an int in the reference, so every use is an
 * exact conversion to 15.0), P = 1, W = 0; U and V come from orc_phys.
 * Float literals of the reference (0.5f, 1.f, 2.f, 0.125f, 0.75f, 0.25f, 3.f)
 * are exact in double except 0.95f, kept as (double)0.95f.
 */
#include "kfun3d_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KB 15.0                     /* inc/phy.h:6 */
#define KP 1.0                      /* inc/phy.h:7 */
#define KW 0.0                      /* inc/phy.h:10 */
#define SWITCH ((double) 0.95f)     /* src/flux.c:181 */
#define MAG0 (0.5 / 3)              /* src/flux.c:11-12 */
#define MAG1 (-MAG0)
#define JV_EPS 1.490116119384766e-08 /* src/kernel.c:12 */

orc_phys orc_phys_from_aoa(double aoa_deg)
{
  orc_phys p;
  p.u = cos(aoa_deg / (180 / M_PI));
  p.v = sin(aoa_deg / (180 / M_PI));
  return p;
}

/* ------------------------------------------------------------------ helpers */

typedef struct { double x1, y1, z1, x2, y2, z2; } frame_t;

/* Two unit tangents completing the unit normal (src/flux.c:173-217,
   src/fill.c:181-225, src/flux.c:565-612, src/fill.c:544-582). */
static frame_t tangents(double xn, double yn, double zn)
{
  frame_t f;
  double d;
  if (fabs(xn) < SWITCH) {
    d = xn;
    f.x1 = 1.0 - d * xn;
    f.y1 = -d * yn;
    f.z1 = -d * zn;
  } else {
    d = yn;
    f.x1 = -d * xn;
    f.y1 = 1.0 - d * yn;
    f.z1 = -d * zn;
  }
  double s = f.x1 * f.x1;
  s += f.y1 * f.y1;
  s += f.z1 * f.z1;
  s = sqrt(s);
  f.x1 /= s;
  f.y1 /= s;
  f.z1 /= s;
  f.x2 = yn * f.z1;
  f.x2 -= zn * f.y1;
  f.y2 = zn * f.x1;
  f.y2 -= xn * f.z1;
  f.z2 = xn * f.y1;
  f.z2 -= yn * f.x1;
  return f;
}

/* phi1..phi9 of src/flux.c:299-324 for averaged velocity (u,v,w), normal
   velocity ubar; the same expressions appear in fill.c and the far-field code. */
static void phis(double xn, double yn, double zn, double u, double v, double w,
                 double ubar, const frame_t *f, double ph[10])
{
  double p1 = xn * KB; p1 += u * ubar;
  double p2 = yn * KB; p2 += v * ubar;
  double p3 = zn * KB; p3 += w * ubar;
  ph[1] = p1; ph[2] = p2; ph[3] = p3;
  ph[4] = f->y2 * p3; ph[4] -= f->z2 * p2;
  ph[5] = f->z2 * p1; ph[5] -= f->x2 * p3;
  ph[6] = f->x2 * p2; ph[6] -= f->y2 * p1;
  ph[7] = f->z1 * p2; ph[7] -= f->y1 * p3;
  ph[8] = f->x1 * p3; ph[8] -= f->z1 * p1;
  ph[9] = f->y1 * p1; ph[9] -= f->x1 * p2;
}

/* ------------------------------------------------------------------ residual */

/* Roe-type dissipative edge flux, src/flux.c:161-448, for one edge given the
   end-point states, gradients and coordinates.  Writes res[4]. */
static void edge_flux(double xn, double yn, double zn, double ln,
                      const double *xa, const double *xb,
                      const double *qa, const double *qb,
                      const double *ga[3], const double *gb[3], double res[4])
{
  double xmean = 0.5 * (xa[0] + xb[0]);
  double ymean = 0.5 * (xa[1] + xb[1]);
  double zmean = 0.5 * (xa[2] + xb[2]);
  frame_t f = tangents(xn, yn, zn);

  double rx = xmean - xa[0], ry = ymean - xa[1], rz = zmean - xa[2];
  double sL[4];
  for (int k = 0; k < 4; k++) {
    double s = qa[k] + ga[0][k] * rx;
    s += ga[1][k] * ry;
    s += ga[2][k] * rz;
    sL[k] = s;
  }
  double ubarL = xn * sL[1]; ubarL += yn * sL[2]; ubarL += zn * sL[3];

  rx = xmean - xb[0]; ry = ymean - xb[1]; rz = zmean - xb[2];
  double sR[4];
  for (int k = 0; k < 4; k++) {
    double s = qb[k] + gb[0][k] * rx;
    s += gb[1][k] * ry;
    s += gb[2][k] * rz;
    sR[k] = s;
  }
  double ubarR = xn * sR[1]; ubarR += yn * sR[2]; ubarR += zn * sR[3];

  double u = 0.5 * (sL[1] + sR[1]);
  double v = 0.5 * (sL[2] + sR[2]);
  double w = 0.5 * (sL[3] + sR[3]);
  double ubar = xn * u; ubar += yn * v; ubar += zn * w;

  double ph[10];
  phis(xn, yn, zn, u, v, w, ubar, &f, ph);

  double c2 = ubar * ubar + KB;
  double c = sqrt(c2);
  double e12 = fabs(ubar), e3 = fabs(ubar + c), e4 = fabs(ubar - c);

  double dp = sR[0] - sL[0], du = sR[1] - sL[1], dv = sR[2] - sL[2], dw = sR[3] - sL[3];

  double ti11 = u * ph[4]; ti11 += v * ph[5]; ti11 += w * ph[6]; ti11 = -ti11 / KB;
  double ti21 = u * ph[7]; ti21 += v * ph[8]; ti21 += w * ph[9]; ti21 = -ti21 / KB;
  double ti31 = 0.5 * (c - ubar); ti31 /= KB;
  double ti41 = -0.5 * (c + ubar); ti41 /= KB;

  double dv1 = ti11 * dp; dv1 += ph[4] * du; dv1 += ph[5] * dv; dv1 += ph[6] * dw; dv1 /= c2;
  double dv2 = ti21 * dp; dv2 += ph[7] * du; dv2 += ph[8] * dv; dv2 += ph[9] * dw; dv2 /= c2;
  double dv3 = 2.0 * ti31 * dp; dv3 += xn * du; dv3 += yn * dv; dv3 += zn * dw; dv3 *= 0.5 / c2;
  double dv4 = 2.0 * ti41 * dp; dv4 += xn * du; dv4 += yn * dv; dv4 += zn * dw; dv4 *= 0.5 / c2;

  double r13 = c * KB;
  double r23 = u * (ubar + c); r23 += xn * KB;
  double r33 = v * (ubar + c); r33 += yn * KB;
  double r43 = w * (ubar + c); r43 += zn * KB;
  double r14 = -c * KB;
  double r24 = u * (ubar - c); r24 += xn * KB;
  double r34 = v * (ubar - c); r34 += yn * KB;
  double r44 = w * (ubar - c); r44 += zn * KB;

  double t1 = e3 * r13 * dv3 + e4 * r14 * dv4;
  double t2 = e12 * f.x1 * dv1 + e12 * f.x2 * dv2;
  t2 += e3 * r23 * dv3 + e4 * r24 * dv4;
  double t3 = e12 * f.y1 * dv1 + e12 * f.y2 * dv2;
  t3 += e3 * r33 * dv3 + e4 * r34 * dv4;
  double t4 = e12 * f.z1 * dv1 + e12 * f.z2 * dv2;
  t4 += e3 * r43 * dv3 + e4 * r44 * dv4;

  double fp1 = ln * KB * ubarL;
  double fp2 = ln * (sL[1] * ubarL + xn * sL[0]);
  double fp3 = ln * (sL[2] * ubarL + yn * sL[0]);
  double fp4 = ln * (sL[3] * ubarL + zn * sL[0]);
  double fm1 = ln * KB * ubarR;
  double fm2 = ln * (sR[1] * ubarR + xn * sR[0]);
  double fm3 = ln * (sR[2] * ubarR + yn * sR[0]);
  double fm4 = ln * (sR[3] * ubarR + zn * sR[0]);

  res[0] = 0.5 * (fp1 + fm1 - ln * t1);
  res[1] = 0.5 * (fp2 + fm2 - ln * t2);
  res[2] = 0.5 * (fp3 + fm3 - ln * t3);
  res[3] = 0.5 * (fp4 + fm4 - ln * t4);
}

/* Characteristic far-field flux at one node, src/flux.c:541-779. */
static void farfield_flux(orc_phys ph_, double fx, double fy, double fz,
                          const double *qi, double out[4])
{
  const double U = ph_.u, V = ph_.v;
  double area = fx * fx; area += fy * fy; area += fz * fz; area = sqrt(area);
  double xn = fx / area, yn = fy / area, zn = fz / area;
  frame_t f = tangents(xn, yn, zn);

  double ubar0 = xn * U; ubar0 += yn * V; ubar0 += zn * KW;
  double c20 = ubar0 * ubar0 + KB;
  double c0 = sqrt(c20);
  double ph[10];
  phis(xn, yn, zn, U, V, KW, ubar0, &f, ph);

  double t13 = c0 * KB;
  double t23 = U * (ubar0 + c0); t23 += xn * KB;
  double t33 = V * (ubar0 + c0); t33 += yn * KB;
  double t43 = KW * (ubar0 + c0); t43 += zn * KB;
  double t14 = -c0 * KB;
  double t24 = U * (ubar0 - c0); t24 += xn * KB;
  double t34 = V * (ubar0 - c0); t34 += yn * KB;
  double t44 = KW * (ubar0 - c0); t44 += zn * KB;

  double ti11 = U * ph[4]; ti11 += V * ph[5]; ti11 += KW * ph[6]; ti11 = -ti11 / KB;
  double ti21 = U * ph[7]; ti21 += V * ph[8]; ti21 += KW * ph[9]; ti21 = -ti21 / KB;
  double ti31 = 0.5 * (c0 - ubar0); ti31 /= KB;
  double ti41 = -0.5 * (c0 + ubar0); ti41 /= KB;

  double pi = qi[0], ui = qi[1], vi = qi[2], wi = qi[3];
  double un = xn * ui; un += yn * vi; un += zn * wi;
  double pr, ur, vr, wr;
  if (un > 0.0) { pr = pi; ur = ui; vr = vi; wr = wi; }
  else { pr = KP; ur = U; vr = V; wr = KW; }

  double rhs1 = ti11 * pr; rhs1 += ph[4] * ur; rhs1 += ph[5] * vr; rhs1 += ph[6] * wr; rhs1 /= c20;
  double rhs2 = ti21 * pr; rhs2 += ph[7] * ur; rhs2 += ph[8] * vr; rhs2 += ph[9] * wr; rhs2 /= c20;
  double rhs3 = 2.0 * ti31 * pi; rhs3 += xn * ui; rhs3 += yn * vi; rhs3 += zn * wi;
  rhs3 = 0.5 * rhs3 / c20;
  double rhs4 = 2.0 * ti41 * KP; rhs4 += xn * U; rhs4 += yn * V; rhs4 += zn * KW;
  rhs4 = 0.5 * rhs4 / c20;

  double pb = t13 * rhs3; pb += t14 * rhs4;
  double ub = f.x1 * rhs1; ub += f.x2 * rhs2; ub += t23 * rhs3; ub += t24 * rhs4;
  double vb = f.y1 * rhs1; vb += f.y2 * rhs2; vb += t33 * rhs3; vb += t34 * rhs4;
  double wb = f.z1 * rhs1; wb += f.z2 * rhs2; wb += t43 * rhs3; wb += t44 * rhs4;
  double ubar = xn * ub; ubar += yn * vb; ubar += zn * wb;

  out[0] = area * KB * ubar;
  out[1] = area * (ub * ubar + xn * pb);
  out[2] = area * (vb * ubar + yn * pb);
  out[3] = area * (wb * ubar + zn * pb);
}

void orc_flux(const GEOMETRY *g, orc_phys ph, const double *q, double *gx,
              double *gy, double *gz, double *r, int first_order)
{
  const size_t E = g->e->sz, N = g->n->sz, dofs = 4 * N;
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
  const double *xs = g->n->xyz->x0, *ys = g->n->xyz->x1, *zs = g->n->xyz->x2;

  memset(gx, 0, dofs * sizeof(double));
  memset(gy, 0, dofs * sizeof(double));
  memset(gz, 0, dofs * sizeof(double));
  memset(r, 0, dofs * sizeof(double));

  /* Least-squares gradients, src/flux.c:60-145 (single thread: every edge
     updates both end points, in edge order). */
  if (!first_order) {
    const double *w0[3] = {g->e->w->w0->x0, g->e->w->w0->x1, g->e->w->w0->x2};
    const double *w1[3] = {g->e->w->w1->x0, g->e->w->w1->x1, g->e->w->w1->x2};
    for (size_t e = 0; e < E; e++) {
      const size_t a = 4 * (size_t) n0[e], b = 4 * (size_t) n1[e];
      for (int k = 0; k < 4; k++) {
        double dq = q[b + k] - q[a + k];
        gx[a + k] += w0[0][e] * dq;
        gy[a + k] += w0[1][e] * dq;
        gz[a + k] += w0[2][e] * dq;
      }
      for (int k = 0; k < 4; k++) {
        double dq = q[a + k] - q[b + k];
        gx[b + k] += w1[0][e] * dq;
        gy[b + k] += w1[1][e] * dq;
        gz[b + k] += w1[2][e] * dq;
      }
    }
  }

  /* Edge fluxes, src/flux.c:151-465. */
  const double *xn = g->e->xyzn->x0, *yn = g->e->xyzn->x1, *zn = g->e->xyzn->x2,
               *ln = g->e->xyzn->x3;
  for (size_t e = 0; e < E; e++) {
    const size_t a = 4 * (size_t) n0[e], b = 4 * (size_t) n1[e];
    const double xa[3] = {xs[n0[e]], ys[n0[e]], zs[n0[e]]};
    const double xb[3] = {xs[n1[e]], ys[n1[e]], zs[n1[e]]};
    const double *ga[3] = {gx + a, gy + a, gz + a};
    const double *gb[3] = {gx + b, gy + b, gz + b};
    double res[4];
    edge_flux(xn[e], yn[e], zn[e], ln[e], xa, xb, q + a, q + b, ga, gb, res);
    for (int k = 0; k < 4; k++) r[a + k] = r[a + k] + res[k];
    for (int k = 0; k < 4; k++) r[b + k] = r[b + k] - res[k];
  }

  /* Slip-wall pressure flux by colour, src/flux.c:467-539. */
  const unsigned int *f0 = g->b->fc->fptr->n0, *f1 = g->b->fc->fptr->n1,
                     *f2 = g->b->fc->fptr->n2, *col = g->t->i;
  for (size_t c = 0; c < g->t->sz; c++) {
    for (unsigned int j = col[c]; j < col[c + 1]; j++) {
      const unsigned int a = f0[j], b = f1[j], d = f2[j];
      double p1 = q[4 * (size_t) a], p2 = q[4 * (size_t) b], p3 = q[4 * (size_t) d];
      double ax = xs[b] - xs[a], ay = ys[b] - ys[a], az = zs[b] - zs[a];
      double bx = xs[d] - xs[a], by = ys[d] - ys[a], bz = zs[d] - zs[a];
      double nx = ay * bz; nx -= az * by; nx *= MAG1;
      double ny = ax * bz; ny -= az * bx; ny *= MAG0;
      double nz = ax * by; nz -= ay * bx; nz *= MAG1;
      double pa = 0.125 * (p2 + p3); pa += 0.75 * p1;
      double pb = 0.125 * (p3 + p1); pb += 0.75 * p2;
      double pc = 0.125 * (p1 + p2); pc += 0.75 * p3;
      const unsigned int nodes[3] = {a, b, d};
      const double pp[3] = {pa, pb, pc};
      for (int t = 0; t < 3; t++) {
        double *rr = r + 4 * (size_t) nodes[t];
        rr[1] += nx * pp[t];
        rr[2] += ny * pp[t];
        rr[3] += nz * pp[t];
      }
    }
  }

  /* Far-field nodes, src/flux.c:541-779. */
  const unsigned int *fn = g->b->f->nptr;
  const double *fx = g->b->f->xyz->x0, *fy = g->b->f->xyz->x1, *fz = g->b->f->xyz->x2;
  for (size_t i = 0; i < g->b->f->sz; i++) {
    double out[4];
    const size_t o = 4 * (size_t) fn[i];
    farfield_flux(ph, fx[i], fy[i], fz[i], q + o, out);
    for (int k = 0; k < 4; k++) r[o + k] += out[k];
  }
}

/* ------------------------------------------------------------------ time step */

static double boundary_rate(double xn, double yn, double zn, const double *qi)
{
  /* src/timestep.c:98-118 (wall) and 126-146 (far field) */
  double ln = sqrt(xn * xn + yn * yn + zn * zn);
  double ubar = qi[1] * xn + qi[2] * yn + qi[3] * zn;
  double ub = ubar / ln;
  double c = sqrt(ub * ub + KB);
  return fabs(ubar) + c * ln;
}

void orc_timestep(const GEOMETRY *g, double cfl, const double *q, double *cdt)
{
  const size_t E = g->e->sz, N = g->n->sz;
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
  const double *xn = g->e->xyzn->x0, *yn = g->e->xyzn->x1, *zn = g->e->xyzn->x2,
               *ln = g->e->xyzn->x3;
  memset(cdt, 0, N * sizeof(double));
  for (size_t e = 0; e < E; e++) {   /* src/timestep.c:58-91 */
    const double *qa = q + 4 * (size_t) n0[e], *qb = q + 4 * (size_t) n1[e];
    double xnorm = xn[e] * ln[e], ynorm = yn[e] * ln[e], znorm = zn[e] * ln[e];
    double u = 0.5 * (qa[1] + qb[1]);
    double v = 0.5 * (qa[2] + qb[2]);
    double w = 0.5 * (qa[3] + qb[3]);
    double ubar = xn[e] * u + yn[e] * v + zn[e] * w;
    double c = sqrt(ubar * ubar + KB);
    double term = u * xnorm; term += v * ynorm; term += w * znorm;
    term = fabs(term) + c * ln[e];
    cdt[n0[e]] = cdt[n0[e]] + term;
    cdt[n1[e]] = cdt[n1[e]] + term;
  }
  const struct bntbl *s = g->b->s, *f = g->b->f;
  for (size_t i = 0; i < s->sz; i++)
    cdt[s->nptr[i]] += boundary_rate(s->xyz->x0[i], s->xyz->x1[i], s->xyz->x2[i],
                                     q + 4 * (size_t) s->nptr[i]);
  for (size_t i = 0; i < f->sz; i++)
    cdt[f->nptr[i]] += boundary_rate(f->xyz->x0[i], f->xyz->x1[i], f->xyz->x2[i],
                                     q + 4 * (size_t) f->nptr[i]);
  for (size_t i = 0; i < N; i++) cdt[i] /= cfl;
}

/* ------------------------------------------------------------------ forces */

void orc_forces(const GEOMETRY *g, orc_phys ph, const double *q, double out[3])
{
  const double *xs = g->n->xyz->x0, *ys = g->n->xyz->x1, *zs = g->n->xyz->x2;
  const unsigned int *f0 = g->b->fc->fptr->n0, *f1 = g->b->fc->fptr->n1,
                     *f2 = g->b->fc->fptr->n2, *col = g->t->i;
  double lift = 0.0, drag = 0.0, momn = 0.0;
  for (size_t c = 0; c < g->t->sz; c++) {
    /* src/forces.c:33 is an OpenMP reduction per colour: each colour sums
       from zero, then the partial sum is added to the total. */
    double l = 0.0, d = 0.0, m = 0.0;
    for (unsigned int j = col[c]; j < col[c + 1]; j++) {
      const unsigned int a = f0[j], b = f1[j], e = f2[j];
      double ax = xs[b] - xs[a], ay = ys[b] - ys[a], az = zs[b] - zs[a];
      double bx = xs[e] - xs[a], by = ys[e] - ys[a], bz = zs[e] - zs[a];
      double xnorm = ay * bz; xnorm -= az * by; xnorm = -0.5 * xnorm;
      double ynorm = ax * bz; ynorm -= az * bx; ynorm = 0.5 * ynorm;
      double press = (q[4 * (size_t) a] + q[4 * (size_t) b] + q[4 * (size_t) e]) / 3.0;
      double cp = 2.0 * (press - 1.0);
      double dcx = cp * xnorm, dcy = cp * ynorm;
      double xmid = xs[a] + xs[b] + xs[e];
      double ymid = ys[a] + ys[b] + ys[e];
      l = l - dcx * ph.v + dcy * ph.u;
      d = d + dcx * ph.u + dcy * ph.v;
      m = m + (xmid - 0.25) * dcy - ymid * dcx;
    }
    lift += l;
    drag += d;
    momn += m;
  }
  out[0] = lift;
  out[1] = drag;
  out[2] = momn;
}

/* ------------------------------------------------------------------ BSR */

static int cmp_u32(const void *a, const void *b)
{
  unsigned int x = *(const unsigned int *) a, y = *(const unsigned int *) b;
  return (x > y) - (x < y);
}

/* Pattern of matrix/init.cpp:7-74: every node row holds its diagonal and one
   block per incident edge, columns sorted.  Also records, per row, which
   lower block the reference's fill touches last (its first L slot then holds
   that block, matrix/matrix.cpp:239). */
orc_bsr *orc_bsr_create(const GEOMETRY *g)
{
  const size_t N = g->n->sz, E = g->e->sz;
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
  orc_bsr *m = (orc_bsr *) calloc(1, sizeof(orc_bsr));
  m->n = N;
  m->ia = (unsigned int *) calloc(N + 1, sizeof(unsigned int));
  for (size_t e = 0; e < E; e++) { m->ia[n0[e] + 1]++; m->ia[n1[e] + 1]++; }
  for (size_t i = 0; i < N; i++) m->ia[i + 1] += m->ia[i] + 1;
  m->nnz = m->ia[N];
  m->ja = (unsigned int *) malloc(m->nnz * sizeof(unsigned int));
  unsigned int *fillp = (unsigned int *) malloc(N * sizeof(unsigned int));
  for (size_t i = 0; i < N; i++) { m->ja[m->ia[i]] = (unsigned int) i; fillp[i] = m->ia[i] + 1; }
  for (size_t e = 0; e < E; e++) {
    m->ja[fillp[n0[e]]++] = n1[e];
    m->ja[fillp[n1[e]]++] = n0[e];
  }
  free(fillp);
  m->diag = (unsigned int *) malloc(N * sizeof(unsigned int));
  m->lpos = (unsigned int *) calloc(N + 1, sizeof(unsigned int));
  for (size_t i = 0; i < N; i++) {
    qsort(m->ja + m->ia[i], m->ia[i + 1] - m->ia[i], sizeof(unsigned int), cmp_u32);
    for (unsigned int j = m->ia[i]; j < m->ia[i + 1]; j++)
      if (m->ja[j] == i) { m->diag[i] = j; break; }
    m->lpos[i + 1] = m->lpos[i] + (m->diag[i] - m->ia[i]);
  }
  m->a = (double *) calloc(m->nnz * 16, sizeof(double));
  m->af = (float *) calloc(m->nnz * 16, sizeof(float));
  m->lslot = (double *) calloc((size_t) m->lpos[N] * 16 + 16, sizeof(double));
  m->last_lower = (unsigned int *) malloc(N * sizeof(unsigned int));
  for (size_t i = 0; i < N; i++) m->last_lower[i] = ~0u;
  /* fill order: per edge (n0,n0), (n0,n1), (n1,n0), (n1,n1) (src/fill.c:496-511) */
  for (size_t e = 0; e < E; e++) {
    unsigned int a = n0[e], b = n1[e];
    if (b < a) m->last_lower[a] = b;  /* (a,b) is lower in row a */
    if (a < b) m->last_lower[b] = a;  /* (b,a) is lower in row b */
  }
  for (size_t i = 0; i < N; i++) {
    if (m->last_lower[i] == ~0u) continue;
    unsigned int col = m->last_lower[i], j = m->ia[i];
    while (m->ja[j] != col) j++;
    m->last_lower[i] = j;
  }
  return m;
}

void orc_bsr_free(orc_bsr *m)
{
  if (!m) return;
  free(m->ia); free(m->ja); free(m->diag); free(m->a); free(m->af);
  free(m->lslot); free(m->lpos); free(m->last_lower);
  free(m);
}

static double *block(orc_bsr *m, unsigned int row, unsigned int col)
{
  for (unsigned int j = m->ia[row]; j < m->ia[row + 1]; j++)
    if (m->ja[j] == col) return m->a + 16 * (size_t) j;
  return NULL;
}

/* ------------------------------------------------------------------ Jacobian */

/* First-order edge Jacobians v0 = 0.5(A_L + |A|), v1 = 0.5(A_R - |A|),
   src/fill.c:171-494. */
static void edge_jacobians(double xn, double yn, double zn, double ln,
                           const double *qa, const double *qb, double v0[16], double v1[16])
{
  frame_t f = tangents(xn, yn, zn);
  double uL = qa[1], vL = qa[2], wL = qa[3];
  double ubarL = xn * uL; ubarL += yn * vL; ubarL += zn * wL;
  double uR = qb[1], vR = qb[2], wR = qb[3];
  double ubarR = xn * uR; ubarR += yn * vR; ubarR += zn * wR;
  double u = 0.5 * (uL + uR), v = 0.5 * (vL + vR), w = 0.5 * (wL + wR);
  double ubar = xn * u; ubar += yn * v; ubar += zn * w;
  double c2 = ubar * ubar + KB;
  double c = sqrt(c2);
  double e12 = ln * fabs(ubar), e3 = ln * fabs(ubar + c), e4 = ln * fabs(ubar - c);
  double ph[10];
  phis(xn, yn, zn, u, v, w, ubar, &f, ph);

  double c2inv = 1.0 / c2;
  double y[5][5];   /* T^-1, 1-based */
  double t;
  t = u * ph[4]; t += v * ph[5]; t += w * ph[6]; y[1][1] = -c2inv * t / KB;
  t = u * ph[7]; t += v * ph[8]; t += w * ph[9]; y[2][1] = -c2inv * t / KB;
  t = c2inv * (c - ubar); y[3][1] = 0.5 * t / KB;
  t = c2inv * (c + ubar); y[4][1] = -0.5 * t / KB;
  y[1][2] = c2inv * ph[4]; y[2][2] = c2inv * ph[7];
  y[3][2] = c2inv * 0.5 * xn; y[4][2] = c2inv * 0.5 * xn;
  y[1][3] = c2inv * ph[5]; y[2][3] = c2inv * ph[8];
  y[3][3] = c2inv * 0.5 * yn; y[4][3] = c2inv * 0.5 * yn;
  y[1][4] = c2inv * ph[6]; y[2][4] = c2inv * ph[9];
  y[3][4] = c2inv * 0.5 * zn; y[4][4] = c2inv * 0.5 * zn;

  double t13 = c * KB;
  double t23 = u * (ubar + c); t23 += xn * KB;
  double t33 = v * (ubar + c); t33 += yn * KB;
  double t43 = w * (ubar + c); t43 += zn * KB;
  double t14 = -c * KB;
  double t24 = u * (ubar - c); t24 += xn * KB;
  double t34 = v * (ubar - c); t34 += yn * KB;
  double t44 = w * (ubar - c); t44 += zn * KB;

  /* |A| = T |Lambda| T^-1 (src/fill.c:367-439), 1-based */
  double a[5][5];
  const double X[4] = {0, f.x1, f.y1, f.z1};   /* rows 2..4 use X1,Y1,Z1 */
  const double Y[4] = {0, f.x2, f.y2, f.z2};
  const double T3[5] = {0, 0, t23, t33, t43};
  const double T4[5] = {0, 0, t24, t34, t44};
  for (int j = 1; j <= 4; j++) {
    double s = e3 * t13 * y[3][j];
    s += e4 * t14 * y[4][j];
    a[1][j] = s;
  }
  for (int i = 2; i <= 4; i++)
    for (int j = 1; j <= 4; j++) {
      double s = e12 * X[i - 1] * y[1][j];
      s += e12 * Y[i - 1] * y[2][j];
      s += e3 * T3[i] * y[3][j];
      s += e4 * T4[i] * y[4][j];
      a[i][j] = s;
    }

  double lb = ln * KB, lx = ln * xn, ly = ln * yn, lz = ln * zn;
  /* row-major block index 4*row + col; row = flux component, col = (p,u,v,w) */
  v0[0] = 0.5 * a[1][1];
  v0[4] = 0.5 * (lx + a[2][1]);
  v0[8] = 0.5 * (ly + a[3][1]);
  v0[12] = 0.5 * (lz + a[4][1]);
  v0[1] = 0.5 * ((lb * xn) + a[1][2]);
  v0[5] = 0.5 * ((ln * (ubarL + xn * uL)) + a[2][2]);
  v0[9] = 0.5 * ((lx * vL) + a[3][2]);
  v0[13] = 0.5 * ((lx * wL) + a[4][2]);
  v0[2] = 0.5 * ((lb * yn) + a[1][3]);
  v0[6] = 0.5 * ((ly * uL) + a[2][3]);
  v0[10] = 0.5 * ((ln * (ubarL + yn * vL)) + a[3][3]);
  v0[14] = 0.5 * ((ly * wL) + a[4][3]);
  v0[3] = 0.5 * ((lb * zn) + a[1][4]);
  v0[7] = 0.5 * ((lz * uL) + a[2][4]);
  v0[11] = 0.5 * ((lz * vL) + a[3][4]);
  v0[15] = 0.5 * ((ln * (ubarL + zn * wL)) + a[4][4]);

  v1[0] = 0.5 * -a[1][1];
  v1[4] = 0.5 * (lx - a[2][1]);
  v1[8] = 0.5 * (ly - a[3][1]);
  v1[12] = 0.5 * (lz - a[4][1]);
  v1[1] = 0.5 * ((lb * xn) - a[1][2]);
  v1[5] = 0.5 * ((ln * (ubarR + xn * uR)) - a[2][2]);
  v1[9] = 0.5 * ((lx * vR) - a[3][2]);
  v1[13] = 0.5 * ((lx * wR) - a[4][2]);
  v1[2] = 0.5 * ((lb * yn) - a[1][3]);
  v1[6] = 0.5 * ((ly * uR) - a[2][3]);
  v1[10] = 0.5 * ((ln * (ubarR + yn * vR)) - a[3][3]);
  v1[14] = 0.5 * ((ly * wR) - a[4][3]);
  v1[3] = 0.5 * ((lb * zn) - a[1][4]);
  v1[7] = 0.5 * ((lz * uR) - a[2][4]);
  v1[11] = 0.5 * ((lz * vR) - a[3][4]);
  v1[15] = 0.5 * ((ln * (ubarR + zn * wR)) - a[4][4]);
}

/* Far-field diagonal block with frozen free-stream T, src/fill.c:527-877. */
static void farfield_jacobian(orc_phys ph_, double fx, double fy, double fz,
                              const double *qi, double vb[16])
{
  const double U = ph_.u, V = ph_.v;
  double ln = sqrt(fx * fx + fy * fy + fz * fz);
  double xn = fx / ln, yn = fy / ln, zn = fz / ln;
  frame_t f = tangents(xn, yn, zn);
  double ubar0 = xn * U; ubar0 += yn * V; ubar0 += zn * KW;
  double c20 = ubar0 * ubar0 + KB;
  double c0 = sqrt(c20);
  double ph[10];
  phis(xn, yn, zn, U, V, KW, ubar0, &f, ph);

  double t13 = c0 * KB;
  double t23 = U * (ubar0 + c0); t23 += xn * KB;
  double t33 = V * (ubar0 + c0); t33 += yn * KB;
  double t43 = KW * (ubar0 + c0); t43 += zn * KB;
  double t14 = -c0 * KB;
  double t24 = U * (ubar0 - c0); t24 += xn * KB;
  double t34 = V * (ubar0 - c0); t34 += yn * KB;
  double t44 = KW * (ubar0 - c0); t44 += zn * KB;

  double ti11 = U * ph[4]; ti11 += V * ph[5]; ti11 += KW * ph[6]; ti11 = -ti11 / KB / c20;
  double ti21 = U * ph[7]; ti21 += V * ph[8]; ti21 += KW * ph[9]; ti21 = -ti21 / KB / c20;
  double ti31 = (c0 - ubar0) / (2.0 * KB * c20);
  double ti41 = -(c0 + ubar0) / (2.0 * KB * c20);
  double ti12 = ph[4] / c20, ti22 = ph[7] / c20, ti32 = 0.5 * xn / c20, ti42 = 0.5 * xn / c20;
  double ti13 = ph[5] / c20, ti23 = ph[8] / c20, ti33 = 0.5 * yn / c20, ti43 = 0.5 * yn / c20;
  double ti14 = ph[6] / c20, ti24 = ph[9] / c20, ti34 = 0.5 * zn / c20, ti44 = 0.5 * zn / c20;

  double pi = qi[0], ui = qi[1], vi = qi[2], wi = qi[3];
  double un = xn * ui; un += yn * vi; un += zn * wi;
  double pr, prp, ur, uru, vr, vrv, wr, wrw;
  if (un > 0.0) { pr = pi; prp = 1.0; ur = ui; uru = 1.0; vr = vi; vrv = 1.0; wr = wi; wrw = 1.0; }
  else { pr = KP; prp = 0.0; ur = U; uru = 0.0; vr = V; vrv = 0.0; wr = KW; wrw = 0.0; }

  double rhs1 = ti11 * pr; rhs1 += ti12 * ur; rhs1 += ti13 * vr; rhs1 += ti14 * wr;
  double rhs1p = ti11 * prp, rhs1u = ti12 * uru, rhs1v = ti13 * vrv, rhs1w = ti14 * wrw;
  double rhs2 = ti21 * pr; rhs2 += ti22 * ur; rhs2 += ti23 * vr; rhs2 += ti24 * wr;
  double rhs2p = ti21 * prp, rhs2u = ti22 * uru, rhs2v = ti23 * vrv, rhs2w = ti24 * wrw;
  double rhs3 = ti31 * pi; rhs3 += ti32 * ui; rhs3 += ti33 * vi; rhs3 += ti34 * wi;
  double rhs4 = ti41 * KP; rhs4 += ti42 * U; rhs4 += ti43 * V; rhs4 += ti44 * KW;

  double pb = t13 * rhs3; pb += t14 * rhs4;
  double pbd[4] = {t13 * ti31, t13 * ti32, t13 * ti33, t13 * ti34};
  const double r1d[4] = {rhs1p, rhs1u, rhs1v, rhs1w};
  const double r2d[4] = {rhs2p, rhs2u, rhs2v, rhs2w};
  const double tid[4] = {ti31, ti32, ti33, ti34};

  double ub = f.x1 * rhs1; ub += f.x2 * rhs2; ub += t23 * rhs3; ub += t24 * rhs4;
  double vb_ = f.y1 * rhs1; vb_ += f.y2 * rhs2; vb_ += t33 * rhs3; vb_ += t34 * rhs4;
  double wb = f.z1 * rhs1; wb += f.z2 * rhs2; wb += t43 * rhs3; wb += t44 * rhs4;
  double ubd[4], vbd[4], wbd[4];
  for (int k = 0; k < 4; k++) {
    ubd[k] = f.x1 * r1d[k]; ubd[k] += f.x2 * r2d[k]; ubd[k] += t23 * tid[k];
    vbd[k] = f.y1 * r1d[k]; vbd[k] += f.y2 * r2d[k]; vbd[k] += t33 * tid[k];
    wbd[k] = f.z1 * r1d[k]; wbd[k] += f.z2 * r2d[k]; wbd[k] += t43 * tid[k];
  }
  double unb = xn * ub; unb += yn * vb_; unb += zn * wb;
  double unbd[4];
  for (int k = 0; k < 4; k++) {
    unbd[k] = xn * ubd[k]; unbd[k] += yn * vbd[k]; unbd[k] += zn * wbd[k];
  }
  for (int k = 0; k < 4; k++) {   /* column k = d/d(p,u,v,w) */
    vb[k] = ln * KB * unbd[k];
    vb[4 + k] = ln * (ub * unbd[k] + unb * ubd[k] + xn * pbd[k]);
    vb[8 + k] = ln * (vb_ * unbd[k] + unb * vbd[k] + yn * pbd[k]);
    vb[12 + k] = ln * (wb * unbd[k] + unb * wbd[k] + zn * pbd[k]);
  }
}

void orc_fill(orc_bsr *m, const GEOMETRY *g, orc_phys ph, const double *q, const double *cdt)
{
  const size_t E = g->e->sz, N = g->n->sz;
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
  const double *xn = g->e->xyzn->x0, *yn = g->e->xyzn->x1, *zn = g->e->xyzn->x2,
               *ln = g->e->xyzn->x3;
  memset(m->a, 0, m->nnz * 16 * sizeof(double));          /* matrix.cpp:298-301 */
  for (size_t i = 0; i < N; i++) {                          /* fill.c:154-161 */
    double *d = m->a + 16 * (size_t) m->diag[i];
    d[0] += cdt[i]; d[5] += cdt[i]; d[10] += cdt[i]; d[15] += cdt[i];
  }
  for (size_t e = 0; e < E; e++) {                          /* fill.c:171-512 */
    double v0[16], v1[16];
    edge_jacobians(xn[e], yn[e], zn[e], ln[e], q + 4 * (size_t) n0[e], q + 4 * (size_t) n1[e], v0, v1);
    double *aa = block(m, n0[e], n0[e]), *ab = block(m, n0[e], n1[e]);
    double *ba = block(m, n1[e], n0[e]), *bb = block(m, n1[e], n1[e]);
    for (int k = 0; k < 16; k++) aa[k] += v0[k];
    for (int k = 0; k < 16; k++) ab[k] += v1[k];
    for (int k = 0; k < 16; k++) ba[k] += -1.0 * v0[k];
    for (int k = 0; k < 16; k++) bb[k] += -1.0 * v1[k];
  }
  const struct bntbl *s = g->b->s, *f = g->b->f;
  for (size_t i = 0; i < s->sz; i++) {                     /* fill.c:516-523, matrix.cpp:282-296 */
    double *d = m->a + 16 * (size_t) m->diag[s->nptr[i]];
    d[4] += s->xyz->x0[i];
    d[8] += s->xyz->x1[i];
    d[12] += s->xyz->x2[i];
  }
  for (size_t i = 0; i < f->sz; i++) {                     /* fill.c:527-877 */
    double v[16];
    farfield_jacobian(ph, f->xyz->x0[i], f->xyz->x1[i], f->xyz->x2[i], q + 4 * (size_t) f->nptr[i], v);
    double *d = m->a + 16 * (size_t) m->diag[f->nptr[i]];
    for (int k = 0; k < 16; k++) d[k] += v[k];
  }
  /* matrix.cpp:239: every lower fill copies the block into the row's first L
     slot, so after the fill that slot holds the last lower block filled. */
  for (size_t i = 0; i < N; i++)
    if (m->last_lower[i] != ~0u)
      memcpy(m->lslot + 16 * (size_t) m->lpos[i], m->a + 16 * (size_t) m->last_lower[i], 16 * sizeof(double));
}

/* ------------------------------------------------------------------ ILU(0) */

/* matrix/init.cpp:105-116: C = A B, each entry summed over k from 0. */
static void gemm4(const double *a, const double *b, double *c)
{
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.0;
      for (int k = 0; k < 4; k++) s += a[4 * i + k] * b[4 * k + j];
      c[4 * i + j] = s;
    }
}

static const double IDENT[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};

void orc_inv4(const double *s, double *dst)
{
  /* matrix/inverse.cpp:195-355: cofactors as sums of triple products in the
     listed order, determinant along the first row, then scale by 1/det. */
  double d[16];
  d[0] = s[5] * s[10] * s[15] - s[5] * s[11] * s[14] - s[9] * s[6] * s[15]
       + s[9] * s[7] * s[14] + s[13] * s[6] * s[11] - s[13] * s[7] * s[10];
  d[1] = -s[1] * s[10] * s[15] + s[1] * s[11] * s[14] + s[9] * s[2] * s[15]
       - s[9] * s[3] * s[14] - s[13] * s[2] * s[11] + s[13] * s[3] * s[10];
  d[2] = s[1] * s[6] * s[15] - s[1] * s[7] * s[14] - s[5] * s[2] * s[15]
       + s[5] * s[3] * s[14] + s[13] * s[2] * s[7] - s[13] * s[3] * s[6];
  d[3] = -s[1] * s[6] * s[11] + s[1] * s[7] * s[10] + s[5] * s[2] * s[11]
       - s[5] * s[3] * s[10] - s[9] * s[2] * s[7] + s[9] * s[3] * s[6];
  d[4] = -s[4] * s[10] * s[15] + s[4] * s[11] * s[14] + s[8] * s[6] * s[15]
       - s[8] * s[7] * s[14] - s[12] * s[6] * s[11] + s[12] * s[7] * s[10];
  d[5] = s[0] * s[10] * s[15] - s[0] * s[11] * s[14] - s[8] * s[2] * s[15]
       + s[8] * s[3] * s[14] + s[12] * s[2] * s[11] - s[12] * s[3] * s[10];
  d[6] = -s[0] * s[6] * s[15] + s[0] * s[7] * s[14] + s[4] * s[2] * s[15]
       - s[4] * s[3] * s[14] - s[12] * s[2] * s[7] + s[12] * s[3] * s[6];
  d[7] = s[0] * s[6] * s[11] - s[0] * s[7] * s[10] - s[4] * s[2] * s[11]
       + s[4] * s[3] * s[10] + s[8] * s[2] * s[7] - s[8] * s[3] * s[6];
  d[8] = s[4] * s[9] * s[15] - s[4] * s[11] * s[13] - s[8] * s[5] * s[15]
       + s[8] * s[7] * s[13] + s[12] * s[5] * s[11] - s[12] * s[7] * s[9];
  d[9] = -s[0] * s[9] * s[15] + s[0] * s[11] * s[13] + s[8] * s[1] * s[15]
       - s[8] * s[3] * s[13] - s[12] * s[1] * s[11] + s[12] * s[3] * s[9];
  d[10] = s[0] * s[5] * s[15] - s[0] * s[7] * s[13] - s[4] * s[1] * s[15]
        + s[4] * s[3] * s[13] + s[12] * s[1] * s[7] - s[12] * s[3] * s[5];
  d[11] = -s[0] * s[5] * s[11] + s[0] * s[7] * s[9] + s[4] * s[1] * s[11]
        - s[4] * s[3] * s[9] - s[8] * s[1] * s[7] + s[8] * s[3] * s[5];
  d[12] = -s[4] * s[9] * s[14] + s[4] * s[10] * s[13] + s[8] * s[5] * s[14]
        - s[8] * s[6] * s[13] - s[12] * s[5] * s[10] + s[12] * s[6] * s[9];
  d[13] = s[0] * s[9] * s[14] - s[0] * s[10] * s[13] - s[8] * s[1] * s[14]
        + s[8] * s[2] * s[13] + s[12] * s[1] * s[10] - s[12] * s[2] * s[9];
  d[14] = -s[0] * s[5] * s[14] + s[0] * s[6] * s[13] + s[4] * s[1] * s[14]
        - s[4] * s[2] * s[13] - s[12] * s[1] * s[6] + s[12] * s[2] * s[5];
  d[15] = s[0] * s[5] * s[10] - s[0] * s[6] * s[9] - s[4] * s[1] * s[10]
        + s[4] * s[2] * s[9] + s[8] * s[1] * s[6] - s[8] * s[2] * s[5];
  double det = s[0] * d[0] + s[1] * d[4] + s[2] * d[8] + s[3] * d[12];
  det = 1.0 / det;
  for (int k = 0; k < 16; k++) dst[k] = d[k] * det;
}

/*
 * One in-order pass of the Chow-Patel sweep of matrix/ilu.cpp:49-97.  For block
 * (i,k) the sweep walks L's row i (its diagonal slot is the identity) against
 * U's column k in index order, subtracting every product L(i,m) U(m,k); the
 * last product is added back afterwards (ilu.cpp:86), and that last product
 * is taken with the slot's value before this pass: the row's persistent L slot
 * when k < i (m == k), the freshly filled A(i,k) when k >= i (m == i).  Lower
 * blocks are then multiplied by the inverse of U(k,k) (ilu.cpp:88-93).  Finally
 * (ilu.cpp:115-136) the factor is written over A and the diagonal inverted.
 */
void orc_ilu(orc_bsr *m)
{
  const size_t N = m->n;
  double *U = (double *) malloc(m->nnz * 16 * sizeof(double)); /* U part, this pass */
  memcpy(U, m->a, m->nnz * 16 * sizeof(double));
  unsigned int *cur = (unsigned int *) malloc(N * sizeof(unsigned int));

  for (size_t i = 0; i < N; i++) {
    const unsigned int j0 = m->ia[i], jd = m->diag[i], j1 = m->ia[i + 1];
    for (unsigned int j = j0; j < j1; j++) {
      const unsigned int k = m->ja[j];
      double a[16], d[16] = {0};
      memcpy(a, m->a + 16 * (size_t) j, sizeof(a));
      /* L row i: columns ja[j0..jd) then the identity at i.
         U column k: rows m <= k with a block (m,k); found by searching row m. */
      for (unsigned int jl = j0; jl <= jd; jl++) {
        const unsigned int mm = m->ja[jl];
        if (mm > k) break;
        /* U(mm, k) exists iff row mm has column k (pattern is symmetric) */
        const double *ublk = NULL;
        size_t uidx = 0;
        for (unsigned int t = m->diag[mm]; t < m->ia[mm + 1]; t++)
          if (m->ja[t] == k) { ublk = U + 16 * (size_t) t; uidx = t; break; }
        if (!ublk) continue;
        const double *lblk;
        if (mm == i) lblk = IDENT;
        else lblk = m->lslot + 16 * (size_t) (m->lpos[i] + (jl - j0));
        (void) uidx;
        gemm4(lblk, ublk, d);
        for (int t = 0; t < 16; t++) a[t] = -1.0 * d[t] + a[t];
      }
      for (int t = 0; t < 16; t++) a[t] = 1.0 * d[t] + a[t];
      if (i > k) {
        double inv[16];
        orc_inv4(U + 16 * (size_t) m->diag[k], inv);
        gemm4(a, inv, m->lslot + 16 * (size_t) (m->lpos[i] + (j - j0)));
      } else {
        memcpy(U + 16 * (size_t) j, a, sizeof(a));
      }
    }
  }
  for (size_t i = 0; i < N; i++) {
    for (unsigned int j = m->ia[i]; j < m->ia[i + 1]; j++) {
      double *dst = m->a + 16 * (size_t) j;
      if (j < m->diag[i]) memcpy(dst, m->lslot + 16 * (size_t) (m->lpos[i] + (j - m->ia[i])), 16 * sizeof(double));
      else memcpy(dst, U + 16 * (size_t) j, 16 * sizeof(double));
    }
    double inv[16];
    orc_inv4(m->a + 16 * (size_t) m->diag[i], inv);
    memcpy(m->a + 16 * (size_t) m->diag[i], inv, sizeof(inv));
  }
  free(U);
  free(cur);
}

/* matrix/init.cpp:96-103: y = A x, each entry summed from zero. */
static void gemv4(const double *a, const double *x, double *y)
{
  for (int i = 0; i < 4; i++) {
    double s = 0.0;
    for (int j = 0; j < 4; j++) s += a[4 * i + j] * x[j];
    y[i] = s;
  }
}

void orc_sptrsv(const orc_bsr *m, const double *b, double *x)
{
  const size_t N = m->n;
  for (size_t r = 0; r < N; r++) {                 /* sptrsv.cpp:173-189 */
    double *xr = x + 4 * r;
    memcpy(xr, b + 4 * r, 4 * sizeof(double));
    for (unsigned int j = m->ia[r]; j < m->diag[r]; j++) {
      double t[4];
      gemv4(m->a + 16 * (size_t) j, x + 4 * (size_t) m->ja[j], t);
      for (int k = 0; k < 4; k++) xr[k] = -1.0 * t[k] + xr[k];
    }
  }
  for (size_t rr = N; rr-- > 0;) {                  /* sptrsv.cpp:191-209 */
    double *xr = x + 4 * rr;
    for (unsigned int j = m->diag[rr] + 1; j < m->ia[rr + 1]; j++) {
      double t[4];
      gemv4(m->a + 16 * (size_t) j, x + 4 * (size_t) m->ja[j], t);
      for (int k = 0; k < 4; k++) xr[k] = -1.0 * t[k] + xr[k];
    }
    double t[4];
    gemv4(m->a + 16 * (size_t) m->diag[rr], xr, t);
    memcpy(xr, t, sizeof(t));
  }
}

/* ------------------------------------------------------------------ FP32 form */

void orc_round_f32(orc_bsr *m)
{
  for (size_t k = 0; k < m->nnz * 16; k++) m->af[k] = (float) m->a[k];
}

static void gemm4f(const float *a, const float *b, float *c)
{
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      float s = 0.0f;
      for (int k = 0; k < 4; k++) s += a[4 * i + k] * b[4 * k + j];
      c[4 * i + j] = s;
    }
}

static void inv4f(const float *s, float *dst)
{
  double sd[16], dd[16];
  for (int k = 0; k < 16; k++) sd[k] = s[k];
  orc_inv4(sd, dd);
  for (int k = 0; k < 16; k++) dst[k] = (float) dd[k];
}

/* Block ILU(0) in natural order on float blocks: L(i,k) = (A(i,k) -
   sum_m L(i,m) U(m,k)) U(k,k)^-1 for k < i, U(i,k) = A(i,k) - sum_m L(i,m) U(m,k)
   for k >= i, products summed in increasing m; the 4x4 inverses are formed in
   double from the float block and rounded.  Diagonal stored inverted. */
void orc_ilu_f32(orc_bsr *m)
{
  const size_t N = m->n;
  float *dinv = (float *) malloc(N * 16 * sizeof(float));
  for (size_t i = 0; i < N; i++) {
    const unsigned int j0 = m->ia[i], j1 = m->ia[i + 1];
    for (unsigned int j = j0; j < j1; j++) {
      const unsigned int k = m->ja[j];
      float *a = m->af + 16 * (size_t) j;
      for (unsigned int jl = j0; jl < j1; jl++) {
        const unsigned int mm = m->ja[jl];
        if (mm >= i || mm >= k) break;
        const float *ublk = NULL;
        for (unsigned int t = m->diag[mm] + 1; t < m->ia[mm + 1]; t++)
          if (m->ja[t] == k) { ublk = m->af + 16 * (size_t) t; break; }
        if (!ublk) continue;
        float p[16];
        gemm4f(m->af + 16 * (size_t) jl, ublk, p);
        for (int t = 0; t < 16; t++) a[t] -= p[t];
      }
      if (k < i) {
        float tmp[16];
        gemm4f(a, dinv + 16 * (size_t) k, tmp);
        memcpy(a, tmp, sizeof(tmp));
      } else if (k == i) {
        inv4f(a, dinv + 16 * i);
      }
    }
    memcpy(m->af + 16 * (size_t) m->diag[i], dinv + 16 * i, 16 * sizeof(float));
  }
  free(dinv);
}

void orc_sptrsv_f32(const orc_bsr *m, const double *b, double *x)
{
  const size_t N = m->n;
  for (size_t r = 0; r < N; r++) {
    double *xr = x + 4 * r;
    memcpy(xr, b + 4 * r, 4 * sizeof(double));
    for (unsigned int j = m->ia[r]; j < m->diag[r]; j++) {
      const float *a = m->af + 16 * (size_t) j;
      const double *xc = x + 4 * (size_t) m->ja[j];
      for (int i = 0; i < 4; i++) {
        double s = 0.0;
        for (int k = 0; k < 4; k++) s += (double) a[4 * i + k] * xc[k];
        xr[i] -= s;
      }
    }
  }
  for (size_t rr = N; rr-- > 0;) {
    double *xr = x + 4 * rr;
    for (unsigned int j = m->diag[rr] + 1; j < m->ia[rr + 1]; j++) {
      const float *a = m->af + 16 * (size_t) j;
      const double *xc = x + 4 * (size_t) m->ja[j];
      for (int i = 0; i < 4; i++) {
        double s = 0.0;
        for (int k = 0; k < 4; k++) s += (double) a[4 * i + k] * xc[k];
        xr[i] -= s;
      }
    }
    const float *d = m->af + 16 * (size_t) m->diag[rr];
    double t[4];
    for (int i = 0; i < 4; i++) {
      double s = 0.0;
      for (int k = 0; k < 4; k++) s += (double) d[4 * i + k] * xr[k];
      t[i] = s;
    }
    memcpy(xr, t, sizeof(t));
  }
}

/* ------------------------------------------------------------------ BLAS-1 */

double orc_norm2(size_t n, const double *v)
{
  double s = 0.0;                                  /* utils.c:53-67 */
  for (size_t i = 0; i < n; i++) s += v[i] * v[i];
  return sqrt(s);
}

static double dot(size_t n, const double *a, const double *b)
{
  double s = 0.0;                                  /* kernel.c:131-134 */
  for (size_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

static void axpy(size_t n, double a, const double *x, double *y)
{
  for (size_t i = 0; i < n; i++) y[i] = a * x[i] + y[i];   /* utils.c:69-87 */
}

static void waxpy(size_t n, double a, const double *x, const double *y, double *w)
{
  for (size_t i = 0; i < n; i++) w[i] = a * x[i] + y[i];   /* utils.c:89-107 */
}

static double normalize(size_t n, double *x)
{
  double nrm = orc_norm2(n, x);                    /* utils.c:109-122 */
  double s = 1.0 / nrm;
  for (size_t i = 0; i < n; i++) x[i] *= s;
  return nrm;
}

/* ------------------------------------------------------------------ driver */

typedef struct {
  const GEOMETRY *g;
  orc_phys ph;
  const orc_params *p;
  orc_bsr *m;
  double *gx, *gy, *gz;
} ctx_t;

static void precondition(ctx_t *c, const double *b, double *x)
{
  if (c->p->precision) orc_sptrsv_f32(c->m, b, x);
  else orc_sptrsv(c->m, b, x);
}

/* iJacVec, src/kernel.c:24-45: y = (F(q + h x/|x|) - r + cdt (w - q)) |x| / h */
static void jacvec(ctx_t *c, const double *q, const double *cdt, const double *x,
                   const double *r, double qnorm, double *w, double *y)
{
  const size_t sz = 4 * c->g->n->sz;
  const double xnorm = orc_norm2(sz, x);
  const double h = JV_EPS * qnorm;
  waxpy(sz, h / xnorm, x, q, w);
  orc_flux(c->g, c->ph, w, c->gx, c->gy, c->gz, y, c->p->first_order);
  const double a = xnorm / h;
  for (size_t i = 0; i < c->g->n->sz; i++)
    for (int k = 0; k < 4; k++) {
      const size_t o = 4 * i + k;
      y[o] = (y[o] - r[o] + cdt[i] * (w[o] - q[o])) * a;
    }
}

#define NB 31

int orc_solve(const GEOMETRY *g, orc_phys ph, double *q, const orc_params *p,
              orc_step *hist, int max_hist)
{
  const size_t N = g->n->sz, sz = 4 * N;
  ctx_t c;
  c.g = g; c.ph = ph; c.p = p;
  c.m = orc_bsr_create(g);
  c.gx = (double *) calloc(sz, sizeof(double));
  c.gy = (double *) calloc(sz, sizeof(double));
  c.gz = (double *) calloc(sz, sizeof(double));
  double *x = (double *) calloc(sz, sizeof(double));
  double *r = (double *) calloc(sz, sizeof(double));
  double *w = (double *) calloc(sz, sizeof(double));
  double *t = (double *) calloc(sz, sizeof(double));
  double *cdt = (double *) calloc(N, sizeof(double));
  double *hh = (double *) calloc(NB * (NB + 1), sizeof(double));
  double *V[NB];
  for (int v = 0; v < NB; v++) V[v] = (double *) calloc(sz, sizeof(double));
  double cs[NB], sn[NB], rs[NB];
  const unsigned int restart = (unsigned int) p->gmres_restart;

  double fnorm0 = 0.0, cfl = p->cfl_init;
  int nrec = 0;
  for (int step = 0; step < p->ts_max; step++) {     /* kernel.c:77-217 */
    orc_flux(g, ph, q, c.gx, c.gy, c.gz, r, p->first_order);
    const double fnorm = orc_norm2(sz, r);
    if (step == 0) fnorm0 = fnorm;
    else {
      double cfl0 = 1.1 * p->cfl_init * fnorm0;
      cfl0 /= fnorm;
      cfl = (cfl0 < p->cfl_max) ? cfl0 : p->cfl_max;
    }
    orc_timestep(g, cfl, q, cdt);
    orc_fill(c.m, g, ph, q, cdt);
    const double qnorm = sqrt(1.0 + orc_norm2(sz, q));
    memset(x, 0, sz * sizeof(double));
    if (p->precision) { orc_round_f32(c.m); orc_ilu_f32(c.m); }
    else orc_ilu(c.m);
    precondition(&c, r, V[0]);

    double tol = 0.0;
    unsigned int total = 0;
    int done = 0;
    while (total <= (unsigned int) p->gmres_max_it) {   /* kernel.c:107-196 */
      if (total > 0) {
        jacvec(&c, q, cdt, x, r, qnorm, w, t);
        waxpy(sz, -1.0, t, r, w);
        precondition(&c, w, V[0]);
      }
      rs[0] = normalize(sz, V[0]);
      if (total == 0) tol = p->gmres_rtol * rs[0];
      unsigned int k = 0;
      while (k < restart) {
        jacvec(&c, q, cdt, V[k], r, qnorm, w, t);
        precondition(&c, t, V[k + 1]);
        double *h = hh + k * (NB + 1);
        for (unsigned int v = 0; v <= k; v++) {       /* modified Gram-Schmidt */
          h[v] = dot(sz, V[k + 1], V[v]);
          axpy(sz, -h[v], V[v], V[k + 1]);
        }
        h[k + 1] = normalize(sz, V[k + 1]);
        for (unsigned int i = 0; i < k; i++) {       /* old rotations */
          const double h0 = h[i], h1 = h[i + 1];
          h[i] = cs[i] * h0 + sn[i] * h1;
          h[i + 1] = cs[i] * h1 - sn[i] * h0;
        }
        const double hk = h[k], hk1 = h[k + 1];
        const double nrm = sqrt(hk * hk + hk1 * hk1);
        const double cr = hk / nrm, sr = hk1 / nrm;
        cs[k] = cr;
        sn[k] = sr;
        rs[k + 1] = -(sr * rs[k]);
        rs[k] = cr * rs[k];
        h[k] = cr * hk + sr * hk1;
        const double res = fabs(rs[k + 1]);
        k++;
        if (res <= tol) { done = 1; break; }
      }
      total += k;
      rs[k - 1] /= hh[(k - 1) * (NB + 1) + (k - 1)];   /* back substitution */
      for (unsigned int i = 1; i <= k - 1; i++) {
        const unsigned int mm = (k - 1) - i;
        double s = rs[mm];
        for (unsigned int j = mm + 1; j <= k - 1; j++) s -= hh[j * (NB + 1) + mm] * rs[j];
        rs[mm] = s / hh[mm * (NB + 1) + mm];
      }
      for (unsigned int v = 0; v < k; v++) axpy(sz, rs[v], V[v], x);
      if (done) break;
    }
    axpy(sz, -1.0, x, q);
    double f[3];
    orc_forces(g, ph, q, f);
    if (nrec < max_hist) {
      hist[nrec].step = step;
      hist[nrec].gmres_its = (int) total;
      hist[nrec].cfl = cfl;
      hist[nrec].fnorm = fnorm;
      hist[nrec].lift = f[0];
      hist[nrec].drag = f[1];
      hist[nrec].momn = f[2];
      nrec++;
    }
    if (round(fnorm0 / fnorm) >= p->stop_ratio) break;
  }
  orc_bsr_free(c.m);
  free(c.gx); free(c.gy); free(c.gz);
  free(x); free(r); free(w); free(t); free(cdt); free(hh);
  for (int v = 0; v < NB; v++) free(V[v]);
  return nrec;
}
