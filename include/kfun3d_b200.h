/*
 * kfun3d_b200: B200 (sm_100a) implementation of KFUN3D's pseudo-transient
 * Newton-Krylov solve, exported as a C ABI.
 *
 * Part 1 re-exports the reference's own entry points with their exact
 * signatures, so the reference's C host driver (src/main.c, src/mesh.c and the
 * set-up files) links against libkfun3d_b200.so in place of src/flux.c,
 * src/timestep.c, src/fill.c, src/ilu.c, src/sptrsv.c, src/forces.c,
 * src/utils.c, src/kernel.c and the matrix/ C++ files.  Every call runs on the GPU;
 * there is no CPU fallback.  Host arrays passed in are copied to device
 * mirrors kept per GEOMETRY (geometry uploaded once, on first use) and results
 * are copied back.  Kernel() runs the whole solve on the device.
 *
 * Part 2 adds what the fixed ABI cannot express: status, physics and solver
 * settings, a native mesh loader/generator, a parameterised solve with
 * per-step history, and device-resident timing hooks.
 *
 * Failures: the reference's entry points return void and assert.  Here every
 * call records a status (kfun3d_gpu_last_status); by default a CUDA error,
 * a missing CUDA device, or a GEOMETRY set up with more than one OpenMP
 * thread also aborts the process, as the reference's asserts do.
 */
#ifndef KFUN3D_B200_H
#define KFUN3D_B200_H

#include <stddef.h>
#include <stdint.h>

#include "kfun3d_geometry.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ===================================================================== */
/* Part 1: the reference's entry points                                  */
/* ===================================================================== */

/* inc/core_kernel.h:9 -> src/fill.c:881-917.  First-order 4x4-block Jacobian
   at g->q->q with diagonal g->n->cdt, kept on the device behind g->matrix. */
void ComputeA(GEOMETRY *g);

/* inc/core_kernel.h:12 -> src/timestep.c:156-188.  Writes g->n->cdt. */
void ComputeTimeStep(const double cfl, GEOMETRY *g);

/* inc/core_kernel.h:15 -> src/flux.c:782-825.  Residual r[4N] of state q[4N];
   also writes the least-squares gradients grad->x0/x1/x2 [4N]. */
void ComputeFlux(const GEOMETRY *g, const double *q, GRADIENT *grad, double *r);

/* inc/core_kernel.h:18 -> src/forces.c:101-120.  forces = {lift, drag, moment}. */
void ComputeForces(const GEOMETRY *g, double *forces);

/* inc/core_kernel.h:21 -> src/ilu.c:271-288 (matrix/ilu.cpp:49-138).
   Block ILU(0) of the matrix in place, diagonal blocks stored inverted. */
void ComputeNumericalILU(GEOMETRY *g);

/* inc/core_kernel.h:22 -> src/sptrsv.c:86-105 (matrix/sptrsv.cpp:34-73).
   x = (LU)^-1 b with the factor of ComputeNumericalILU. */
void ComputeSparseTriangularSolve(const GEOMETRY *g, const double *b, double *x);

/* inc/utils.h:18 -> src/utils.c:53-67 */
double Compute2ndNorm(const size_t sz, const double *v);
/* inc/utils.h:21 -> src/utils.c:69-87: y = a x + y */
void ComputeAXPY(const size_t sz, const double a, const double *x, double *y);
/* inc/utils.h:24 -> src/utils.c:89-107: w = a x + y */
void ComputeNewAXPY(const size_t sz, const double a, const double *x, const double *y, double *w);
/* inc/utils.h:27 -> src/utils.c:109-122: x /= |x|, returns |x| */
double Normalize(const size_t sz, double *x);
/* inc/utils.h:15 -> src/utils.c:5-51 (coloured printf used by src/bench.c) */
void fun3d_printf(const uint32_t c, const char *format, ...);

/* src/main.c:19 -> src/kernel.c:47-232.  The whole pseudo-transient solve on
   the device with the reference's constants; updates g->q->q and prints the
   reference's per-step report unless kfun3d_set_verbose(0). */
void Kernel(GEOMETRY *g);

/* matrix/wrapper.cpp:23-28.  Creates the opaque matrix handle stored in
   g->matrix.  The handle keeps the edges; the block pattern of the edge graph
   (with its level sets and ILU(0) product lists) is built on the device with
   the mirror, at the first kernel call.  No device memory is touched before. */
void *CXX_Matrix_Init(const size_t nnodes, const size_t nedges, const unsigned int block_size,
                      const unsigned int nthreads, const unsigned int *n0, const unsigned int *n1);
/* matrix/wrapper.cpp:30-34 */
void CXX_Matrix_Delete(void *ptr);
/* matrix/wrapper.cpp:36-40.  The reference partitions with METIS for its
   OpenMP threads; the device path does not use the partition, so this assigns
   contiguous node ranges. */
void CXX_METIS(const unsigned int nparts, unsigned int *parts, void *ptr);
/* matrix/wrapper.cpp:13-21: big-endian walkers of the .msh reader */
void CXX_Walk_Int(char *l, const char *h, const size_t sz, unsigned int *b);
void CXX_Walk_Double(char *l, const char *h, const size_t sz, double *b);

/* ===================================================================== */
/* Part 2: extensions (no counterpart in the reference's ABI)            */
/* ===================================================================== */

enum kfun3d_status {
  KFUN3D_OK = 0,
  KFUN3D_ERR_CUDA = 1,        /* a CUDA call failed */
  KFUN3D_ERR_NONFINITE = 2,   /* NaN or Inf in a residual or norm */
  KFUN3D_ERR_PIVOT = 3,       /* zero or non-finite pivot block in ILU(0) */
  KFUN3D_ERR_ARG = 4,         /* invalid argument or unsupported GEOMETRY */
  KFUN3D_ERR_IO = 5,          /* mesh file error */
  KFUN3D_ERR_NO_DEVICE = 6,   /* no CUDA device */
  KFUN3D_ERR_DIVERGED = 7,    /* linear or nonlinear solve failed */
  KFUN3D_ERR_TIMEOUT = 8      /* a device-side wait exceeded its bound (results invalid) */
};

/* Status of the most recent call (KFUN3D_OK or an error code) and its text. */
int kfun3d_gpu_last_status(void);
const char *kfun3d_gpu_last_error(void);
void kfun3d_clear_status(void);
/* 1 (default): a CUDA error, a missing CUDA device or a GEOMETRY set up with
   more than one OpenMP thread aborts the process like the reference's
   asserts.  0: the error is only recorded. */
void kfun3d_set_abort_on_error(int on);

/* Angle of attack in degrees (inc/phy.h:8-9 hard-codes 3).  Free stream
   U = cos(a / (180/pi)), V = sin(a / (180/pi)), W = 0, P = 1, beta = 15. */
void kfun3d_set_aoa(double deg);
double kfun3d_get_aoa(void);
void kfun3d_get_freestream(double *u, double *v);

/* Arithmetic of the device kernels.
   KFUN3D_MODE_EXACT: the reference's operation order everywhere (no fused
     multiply-add, per-node sums in edge order, reductions in index order);
     results are bit-identical to the reference at one OpenMP thread.
   KFUN3D_MODE_FAST: fused multiply-add, tree reductions, reciprocals
     hoisted; results differ from the reference at rounding level. */
enum { KFUN3D_MODE_EXACT = 0, KFUN3D_MODE_FAST = 1 };
void kfun3d_set_mode(int mode);
int kfun3d_get_mode(void);

/* Preconditioner precision: 0 = FP64 (the reference), 1 = FP32 Jacobian
   blocks, FP32 ILU(0) factors and FP32-block triangular solves. */
void kfun3d_set_precision(int p);
/* Elimination order of ILU(0) and the triangular solves.
   0 = the mesh's node numbering (the reference: matrix/matrix.cpp factors
       rows in node order);
   1 = spatial: rows and columns renumbered by sweeps of the node
       coordinates (s = x + y + z cut into 4 slabs, each swept from both
       faces towards its middle; P A P^T is factored, x = P^T (LU)^-1 P b).  Same Jacobian blocks and sparsity, a different
       (and on randomly numbered meshes a much stronger) preconditioner; not
       a parity path.  Built on first use per mesh.  While it is active
       kfun3d_matrix_read(blocks) and kfun3d_sptrsv_device_noalloc return
       KFUN3D_ERR_ARG.
   KFUN3D_ILU_PERM in the environment, read when the order is built:
   "sweep" renumbers by ascending x + y + z over the whole mesh, "tiles" tile
   by tile (one tile per SM, each tile swept by x + y + z), "morton" by
   the Morton order of the coordinates; KFUN3D_ILU_SLABS sets the number of
   slabs of the default order;
   "identity" keeps the mesh numbering through the same renumbering code
   (a test hook). */
void kfun3d_set_ilu_order(int order);
int kfun3d_get_ilu_order(void);
/* Row of every node (rank[node], N entries) in the spatial order built for
   this GEOMETRY; returns N, or -1 when it has not been built. */
long kfun3d_ilu_rank(const GEOMETRY *g, unsigned int *rank);
/* Host only (no GPU needed): the spatial order kfun3d_set_ilu_order(1) would
   build for this GEOMETRY under the current environment, with `tiles` column
   tiles (the device uses one per SM): rank[node] (N entries, may be NULL)
   and the numbers of levels of the lower and upper triangular sweeps of the
   renumbered pattern (may be NULL).  Returns 0, or -1 on bad arguments. */
int kfun3d_ilu_order_plan(const GEOMETRY *g, unsigned int tiles, unsigned int *rank, unsigned int *nlev_lower,
                          unsigned int *nlev_upper);
/* Additive Schwarz preconditioner without overlap (the "Schwarz" of
   Newton-Krylov-Schwarz: PETSc's -pc_type asm -sub_pc_type ilu in
   archive/base2/incomp/petsc.opt, the reference's partition being METIS's,
   matrix/matrix.cpp:99-135), on one device: with parts > 1 the nodes are cut
   into `parts` subdomains by recursive coordinate bisection
   (kfun3d_schwarz_partition) and every Jacobian block that couples two
   subdomains is removed before ILU(0), which then factors each subdomain on
   its own (block-Jacobi ILU(0) in the active elimination order; the
   triangular solves are the subdomains' own).  What one GPU per subdomain
   would compute, without the halo exchange and the reductions across GPUs.
   0 or 1: off (default).  Applied at the next factorisation; changes the
   iteration counts, not the Jacobian-vector products. */
void kfun3d_set_schwarz(unsigned int parts);
unsigned int kfun3d_get_schwarz(void);
/* Host only (no GPU needed): part[node] (N entries) of the `parts`
   subdomains kfun3d_set_schwarz(parts) uses.  Returns 0, or -1 on bad
   arguments. */
int kfun3d_schwarz_partition(const GEOMETRY *g, unsigned int parts, unsigned int *part);
/* 1: residual reconstructed without gradients (first-order flux). */
void kfun3d_set_first_order(int on);
/* 0 silences Kernel()'s per-step report. */
void kfun3d_set_verbose(int on);

typedef struct {
  int ts_max;          /* Newton steps (src/kernel.c:21: 15) */
  double stop_ratio;   /* stop once round(|r0|/|r|) >= stop_ratio (kernel.c:22: 1e7) */
  double gmres_rtol;   /* kernel.c:14: 0.01 */
  int gmres_restart;   /* kernel.c:15: 30 (at most 30) */
  int gmres_max_it;    /* kernel.c:17: 10000 */
  double cfl_init;     /* kernel.c:19: 50 */
  double cfl_max;      /* kernel.c:20: 1e5 */
} kfun3d_solver_params;

typedef struct {
  int step;
  int gmres_its;
  double cfl;
  double fnorm;        /* residual norm before this step's update */
  double lift, drag, momn;
  double seconds;      /* device time of the step */
} kfun3d_step;

/* Reference defaults (src/kernel.c:12-22). */
void kfun3d_default_params(kfun3d_solver_params *p);

/* Kernel() with parameters: solves from g->q->q (updated in place), records
   up to max_hist steps, returns the number of steps taken or -1 on error. */
int kfun3d_solve(GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_step *hist, int max_hist);

/* Native .msh loader: the GEOMETRY the reference's Setup builds at one
   thread (same edge order, wall colouring and least-squares weights), with
   the free-stream initial state of the current angle of attack. */
GEOMETRY *kfun3d_setup_load(const char *path);
void kfun3d_setup_free(GEOMETRY *g);
void kfun3d_initial_guess(GEOMETRY *g);

/* Synthetic Kuhn-box mesh writer: n^3 nodes on [0,1]^3, each hex split into
   six tets, interior nodes jittered by U(+-jitter h), bottom face a slip wall
   with a Gaussian bump height*exp(-r^2/(2 sigma^2))*(1-z), other faces far
   field, node numbering by permute: 0 the lattice order, 1 seeded random,
   2 Morton order of the lattice.  Returns 0 on success. */
typedef struct {
  unsigned int n;
  double bump_height;
  double bump_sigma;
  double jitter;
  unsigned long long seed;
  int permute;
} kfun3d_mesh_spec;
int kfun3d_mesh_generate(const char *path, const kfun3d_mesh_spec *spec);

/* Device-resident timing: runs kernel family `which` reps times on the
   device copy of g (state g->q->q uploaded once), returns the mean time of
   one call in milliseconds measured with CUDA events on the solver's stream,
   or a negative value on error.  which: 0 flux (gradient + edge flux +
   boundary), 1 time step, 2 Jacobian fill, 3 ILU(0), 4 triangular solves,
   5 one GMRES iteration at Arnoldi index 15 (J.v + solve + MGS),
   6 modified Gram-Schmidt and normalisation alone at Arnoldi index 15,
   7 the gradient alone, 8 the edge flux and boundary terms alone. */
double kfun3d_time_kernel(GEOMETRY *g, int which, int reps);

/* Device-resident solve timing: the initial state g->q->q is uploaded once;
   each of reps solves restarts from it on the device and runs kfun3d_solve's
   algorithm.  Returns the mean seconds per solve (CUDA events on the solver's
   stream) and fills hist with the last solve's steps; negative on error. */
double kfun3d_time_solve(GEOMETRY *g, const kfun3d_solver_params *p, int reps, kfun3d_step *hist,
                         int max_hist, int *nsteps);

/* Number of kernel launches the library issued since the last reset. */
unsigned long long kfun3d_launch_count(void);
void kfun3d_reset_launch_count(void);

/* The device matrix behind g->matrix, for inspection: the block pattern of
   matrix/init.cpp:7-74 (row pointers nnodes+1, sorted columns nnz) and the
   4x4 row-major blocks (nnz*16, FP32 blocks widened) as left by the last
   ComputeA (the Jacobian) or ComputeNumericalILU (the factor, diagonal blocks
   inverted).  Returns nnz, or -1 on error; NULL outputs are skipped. */
long kfun3d_matrix_read(const GEOMETRY *g, unsigned int *ia, unsigned int *ja, double *blocks);

/* No counterpart in the reference.  Allocation-free triangular solve, for
   callers that cannot allocate device memory: a framework that owns every
   device allocation (its own pooled allocator, or all device memory sized at
   start-up) and forbids libraries from calling cudaMalloc afterwards.
   x = (LU)^-1 b with the factor of the last ComputeNumericalILU on this
   GEOMETRY, in the mesh's ILU(0) order and in the precision that is still
   set (a changed kfun3d_set_precision or the spatial order is refused with
   KFUN3D_ERR_ARG); d_b and d_x are the caller's device arrays of 4*nnodes
   doubles (16-byte aligned, distinct).  Runs the sync-free sweep, whose
   per-row completion flags live in a fixed device array of the library
   (8 MiB, held by every GPU that loads the library until exit, cleared by
   each call), so the call allocates nothing; at most 2,097,152 rows, larger
   matrices are rejected (KFUN3D_ERR_ARG).  The first call on a device looks
   up that array's device address (cudaGetSymbolAddress).  The call waits for
   all work already queued on the device (so b may be written on any stream
   just before), runs on the library's stream and returns once x is written.
   Calls share the array: calls that overlap on the GPU (from several host
   threads) race.  Returns KFUN3D_OK or an error code (also recorded). */
int kfun3d_sptrsv_device_noalloc(const GEOMETRY *g, const double *d_b, double *d_x);

/* Release the device mirror of g (also done by CXX_Matrix_Delete). */
void kfun3d_device_release(GEOMETRY *g);

/* Self-check of the device-side bounded waits, without a fault: one thread
   waits, the way the sync-free triangular sweep waits for a row, on a flag
   that nothing sets, and must give up after the library's poll limit (about
   a second at most); a second wait on a flag that is set must return at once,
   in the same context.  Returns KFUN3D_ERR_TIMEOUT when both behave so,
   KFUN3D_ERR_ARG when either does not, KFUN3D_ERR_CUDA / _NO_DEVICE on a
   CUDA failure or without a device.  For tests and bring-up; no counterpart
   in the reference. */
int kfun3d_check_bounded_wait(void);

/* Which device paths g's mirror uses (for tests and reports; builds the
   mirror on first use): key "sptrsv_schedule" -> the triangular-solve
   schedule of the active ILU(0) order (8 packed level launches, 7 four-lane
   level launches, ...), "lsq_terms_match" -> 1 when the least-squares
   terms recomputed on the device from per-node coefficients made there equal
   the GEOMETRY's stored terms bit for bit, "visit_order_copies" -> 1 when
   the residual passes work on copies of the node data in their spatial visit
   order, "mgs_resident" -> 1 when Gram-Schmidt keeps the vector on chip,
   "pattern_matches_host" / "spatial_pattern_matches_host" -> 1 when the
   block pattern, level lists and ILU(0) product lists built on the device
   (mesh numbering / spatial renumbering; -1 while the latter is not built)
   equal a host build from the same edges element for element, else 0,
   "setup_us" / "pattern_us" / "spatial_setup_us" -> host wall time in
   microseconds of building the mirror / its block pattern on the device /
   the spatial order's set, "host_pattern_us" -> that of the host build the
   last "pattern_matches_host" made (-1 before one).  -1 for an unknown key
   or on error. */
long kfun3d_device_query(const GEOMETRY *g, const char *key);

/* ---------------------------------------------------------------------
 * Part 3: the learned right preconditioner (no reference counterpart).
 *
 * An edge-based message-passing network, hidden width 32: an encoder MLP on
 * node features [y/s, q], three message-passing layers (edge MLP on
 * [h_i, h_j, n_ij, a_ij], sum over a node's edges, residual node MLP on
 * [h_i, sum]), and a decoder MLP to 4 outputs.  Every MLP has two linear
 * layers with a ReLU between; layer L maps kin inputs (its bias is the column
 * at the ones feature, index nreal) to out outputs, weights W~[out x kin] in
 * one FP32 parameter vector at `offset`.  Forward, backward and Adam run on
 * the GPU with BF16 tensor-core operands and FP32 accumulation.
 *
 * All d_* arguments are device pointers.  x0 is [nodes x 8] BF16
 * ([y/s (4), q (4)]); targets and outputs are [nodes x 4] FP32.
 * --------------------------------------------------------------------- */
typedef struct kfun3d_mpnn kfun3d_mpnn;
typedef struct kfun3d_mpnn_graph kfun3d_mpnn_graph;

size_t kfun3d_mpnn_param_count(void);
int kfun3d_mpnn_layer_shape(int layer, int *out, int *kin, int *nreal, int *offset);
/* Seeded initialisation on the current device; NULL on failure. */
kfun3d_mpnn *kfun3d_mpnn_create(unsigned long long seed);
void kfun3d_mpnn_free(kfun3d_mpnn *net);
/* Host FP32 parameters in and out; set_params also resets the Adam state. */
int kfun3d_mpnn_set_params(kfun3d_mpnn *net, const float *host, size_t n);
int kfun3d_mpnn_get_params(const kfun3d_mpnn *net, float *host, size_t n);
int kfun3d_mpnn_get_grad(const kfun3d_mpnn *net, float *host, size_t n);
int kfun3d_mpnn_zero_grad(kfun3d_mpnn *net);
/* The directed-edge graph of a mesh (node-incidence rows, edge features). */
kfun3d_mpnn_graph *kfun3d_mpnn_graph_create(const GEOMETRY *g);
void kfun3d_mpnn_graph_free(kfun3d_mpnn_graph *G);
/* d_out = N(x0). */
int kfun3d_mpnn_forward(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const void *d_x0, float *d_out);
/* Adds the gradient of weight * sum (N(x0) - target)^2 to the network's
 * gradient; *loss (optional) receives weight * sum (...)^2. */
int kfun3d_mpnn_accumulate(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const void *d_x0, const float *d_target,
                           double weight, double *loss);
/* One Adam step on the accumulated gradient, which it then clears. */
int kfun3d_mpnn_adam_step(kfun3d_mpnn *net, double lr, double beta1, double beta2, double eps);
/* Features and target of a training pair from FP64 device vectors of
 * 4 * nnodes: x0 = BF16([y/s, q]), target = (x - y)/s, s = RMS(y). */
int kfun3d_mpnn_make_pair(size_t nnodes, const double *d_y, const double *d_q, const double *d_x, void *d_x0,
                          float *d_target);
/* z = y + s N([y/s, q]): the network's correction of an ILU(0)-preconditioned
 * vector y. */
int kfun3d_mpnn_apply(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const double *d_y, const double *d_q, double *d_z);
/* Statistics of a flexible solve. */
typedef struct {
  int newton_steps;     /* Newton steps taken */
  int gmres_its;        /* FGMRES iterations over the solve */
  int learned_its;      /* iterations preconditioned by the network */
  int fallback_solves;  /* linear solves run (or finished) without the network */
  int rejected_steps;   /* updates undone because the nonlinear residual grew tenfold */
  int disabled;         /* 1: the network was switched off for the rest of the solve */
  int pairs;            /* training pairs written (kfun3d_collect_pairs) */
  double seconds;       /* device time of the whole solve */
} kfun3d_flex_stats;

/* The pseudo-transient solve of Kernel() with flexible GMRES(restart) on the
 * reference's left-preconditioned system (Arnoldi on ILU(0)^-1 J, the
 * reference's residual measure and stopping test) and a right preconditioner
 * that may change per iteration: the identity (net == NULL: the reference's
 * GMRES, iteration for iteration) or the network's correction
 * v + s N([v/s, q]), from Newton step 1 on.  The network falls back to
 * the identity: for a linear solve whose first direction it does not improve
 * (its image under ILU(0)^-1 J farther from v0), for the rest of a solve
 * whose residual falls at less than half the previous solve's rate or that
 * has used 1.5x the previous solve's iterations, for good after three such
 * fallbacks in a row,
 * and for an update after which the FP64 nonlinear residual grows tenfold
 * (the update is undone).  Solves from g->q->q and updates it; returns the
 * number of history entries or -1. */
int kfun3d_solve_flexible(GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_mpnn *net, kfun3d_step *hist,
                          int max_hist, kfun3d_flex_stats *stats);
/* The flexible solve without a network, writing training pairs (x, y) with
 * ILU(0)^-1 J x = y: the pair (BF16([y/s, q]), (x - y)/s), s = RMS(y), goes
 * to slot i of d_x0 ([cap][N x 8] BF16) and d_target ([cap][N x 4] FP32).  x
 * is each Newton step's final correction (y = ILU(0)^-1 J x formed for it)
 * and, for stride > 0, the iterate after every `stride` iterations of the
 * step's first cycle; for stride < 0, the Krylov vector v_k of every
 * -stride-th iteration with y = ILU(0)^-1 J v_k, the product the iteration
 * forms anyway.  Returns the number of pairs or -1. */
int kfun3d_collect_pairs(GEOMETRY *g, const kfun3d_solver_params *p, int stride, void *d_x0, float *d_target,
                         int cap, kfun3d_flex_stats *stats);
/* Mean device seconds of `reps` flexible solves from g->q->q (not updated). */
double kfun3d_time_solve_flexible(GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_mpnn *net, int reps,
                                  kfun3d_step *hist, int max_hist, int *nsteps, kfun3d_flex_stats *stats);

/* Milliseconds of one application of the learned preconditioner's network
 * (features, encoder, three message-passing layers, decoder) on g's device
 * mirror, averaged over reps. */
double kfun3d_time_learned_apply(GEOMETRY *g, kfun3d_mpnn *net, int reps);

/* Test hook: Y = X Wt^T, one BF16 tensor-core tile per 128 rows. */
int kfun3d_umma_selftest(const void *X, const void *Wt, float *Y, int rows, int K, int N);

#ifdef __cplusplus
}
#endif
#endif /* KFUN3D_B200_H */
