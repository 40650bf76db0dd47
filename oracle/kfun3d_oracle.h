/*
 * Test infrastructure only: the CPU oracle for the kfun3d_b200 hot path.
 *
 * A plain-C restatement of the reference's pseudo-transient Newton-Krylov
 * solve at one OpenMP thread (the only thread count at which the reference is
 * deterministic).  Every function follows one reference function operation by
 * operation, so on the same GEOMETRY its results are bit-identical to the
 * reference's; that is checked against the reference itself (oracle/_ref) and
 * against committed golden fixtures.  Only tests, smoke() and bench.py's CPU
 * baseline may use it, and only as the checker; the product never links it.
 */
#ifndef KFUN3D_ORACLE_H
#define KFUN3D_ORACLE_H

#include <stddef.h>
#include "kfun3d_geometry.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Free stream of inc/phy.h:6-10 with the angle of attack as data:
   B = 15, P = 1, W = 0 stay the reference's constants. */
typedef struct {
  double u;   /* cos(aoa / (180 / M_PI)) */
  double v;   /* sin(aoa / (180 / M_PI)) */
} orc_phys;

orc_phys orc_phys_from_aoa(double aoa_deg);

/* ComputeFlux (src/flux.c:14-825).  first_order != 0 skips the gradient and
   reconstructs with zero gradients (a mode the reference does not have). */
void orc_flux(const GEOMETRY *g, orc_phys ph, const double *q, double *gx,
              double *gy, double *gz, double *r, int first_order);

/* ComputeTimeStep (src/timestep.c:21-188): cdt[N]. */
void orc_timestep(const GEOMETRY *g, double cfl, const double *q, double *cdt);

/* ComputeForces (src/forces.c:8-120): lift, drag, moment. */
void orc_forces(const GEOMETRY *g, orc_phys ph, const double *q, double out[3]);

/* Block-sparse 4x4 matrix of matrix/matrix.h:9-14 with the state the
   reference's ILU keeps between calls. */
typedef struct {
  size_t n, nnz;
  unsigned int *ia, *ja, *diag;   /* CSR of blocks, sorted columns, diagonal slot */
  double *a;                      /* nnz * 16, row-major blocks */
  float *af;                      /* nnz * 16, single-precision copy (mixed form) */
  double *lslot;                  /* lower blocks' persistent slots (one per a lower entry) */
  unsigned int *lpos;             /* n+1: first lower slot of each row */
  unsigned int *last_lower;       /* per row: block index of the last lower fill, or ~0 */
} orc_bsr;

orc_bsr *orc_bsr_create(const GEOMETRY *g);
void orc_bsr_free(orc_bsr *m);

/* ComputeA (src/fill.c:115-917 through matrix/matrix.cpp:231-301). */
void orc_fill(orc_bsr *m, const GEOMETRY *g, orc_phys ph, const double *q, const double *cdt);

/* ComputeNumericalILU: one in-order sweep of matrix/ilu.cpp:49-138, which at one
   thread is block ILU(0) in natural order, then the diagonal blocks inverted by
   matrix/inverse.cpp:195-355.  Keeps the reference's slot semantics. */
void orc_ilu(orc_bsr *m);

/* ComputeSparseTriangularSolve (matrix/sptrsv.cpp:34-73). */
void orc_sptrsv(const orc_bsr *m, const double *b, double *x);

/* Mixed-precision form (no reference counterpart): the filled blocks rounded to
   float, block ILU(0) in float, and triangular solves with float blocks and
   double vectors. */
void orc_round_f32(orc_bsr *m);
void orc_ilu_f32(orc_bsr *m);
void orc_sptrsv_f32(const orc_bsr *m, const double *b, double *x);

/* 4x4 inverse of matrix/inverse.cpp:195-355 (adjugate / determinant). */
void orc_inv4(const double *src, double *dst);

/* Compute2ndNorm (src/utils.c:53-67), in index order. */
double orc_norm2(size_t n, const double *v);

typedef struct {
  int ts_max;
  double stop_ratio;
  double gmres_rtol;
  int gmres_restart;
  int gmres_max_it;
  double cfl_init;
  double cfl_max;
  int first_order;   /* residual without gradients */
  int precision;     /* 0: FP64 preconditioner, 1: FP32 blocks/factors/solves */
} orc_params;

typedef struct {
  int step;
  int gmres_its;
  double cfl;
  double fnorm;
  double lift, drag, momn;
} orc_step;

/* Newton/SER + GMRES driver (src/kernel.c:24-232) on state q (in/out). */
int orc_solve(const GEOMETRY *g, orc_phys ph, double *q, const orc_params *p,
              orc_step *hist, int max_hist);

#ifdef __cplusplus
}
#endif
#endif
