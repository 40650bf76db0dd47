// kfun3d_b200 internals shared by the host and CUDA translation units.
#pragma once

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <memory>
#include <thread>
#include <vector>

#include "kfun3d_b200.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#else
struct double4_host { double x, y, z, w; };
#endif

void kf_set_error(int code, const char *msg);

// ord = 0 .. n-1 ordered by key, ties by index (what a stable sort by key
// gives), on the host's threads: chunks sorted under that total order, then
// merged pairwise.
template <class K> void kf_sort_by_key(std::vector<uint32_t> &ord, const std::vector<K> &key)
{
  const size_t n = key.size();
  ord.resize(n);
  for (size_t i = 0; i < n; i++) ord[i] = (uint32_t)i;
  auto less = [&key](uint32_t a, uint32_t b) { return key[a] < key[b] || (!(key[b] < key[a]) && a < b); };
  unsigned T = 1;
  while (T * 2 <= std::min(16u, std::thread::hardware_concurrency())) T *= 2;
  if (n < 65536 || T == 1) {
    std::sort(ord.begin(), ord.end(), less);
    return;
  }
  std::vector<size_t> cut(T + 1);
  for (unsigned t = 0; t <= T; t++) cut[t] = n * t / T;
  {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++)
      th.emplace_back([&, t] { std::sort(ord.begin() + cut[t], ord.begin() + cut[t + 1], less); });
    for (auto &x : th) x.join();
  }
  std::vector<uint32_t> tmp(n);
  for (unsigned w = 1; w < T; w *= 2) {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t += 2 * w)
      th.emplace_back([&, t] {
        std::merge(ord.begin() + cut[t], ord.begin() + cut[t + w], ord.begin() + cut[t + w],
                   ord.begin() + cut[t + 2 * w], tmp.begin() + cut[t], less);
      });
    for (auto &x : th) x.join();
    ord.swap(tmp);
  }
}

// Set-up phase trace: with KFUN3D_SETUP_TRACE=1 in the environment, each
// mark() prints to stderr the host wall time since the tracer's previous mark.
struct SetupTrace {
  const char *scope;
  bool on;
  std::chrono::steady_clock::time_point t;
  explicit SetupTrace(const char *s)
      : scope(s), on(getenv("KFUN3D_SETUP_TRACE") && atoi(getenv("KFUN3D_SETUP_TRACE")) > 0),
        t(std::chrono::steady_clock::now()) {}
  void mark(const char *phase)
  {
    if (!on) return;
    const auto n = std::chrono::steady_clock::now();
    fprintf(stderr, "kfun3d_b200 set-up: %s: %s %.3f s\n", scope, phase, std::chrono::duration<double>(n - t).count());
    t = n;
  }
};
int kf_mode();
int kf_precision();
int kf_first_order();

// Host-side block pattern of the edge graph (matrix/init.cpp:7-74): row i
// holds its diagonal and one block per incident edge, columns sorted.
// std::allocator that leaves new elements uninitialised (for arrays every
// element of which is written right after they are sized)
template <class T> struct uninit_alloc : std::allocator<T> {
  template <class U> struct rebind { using other = uninit_alloc<U>; };
  uninit_alloc() = default;
  template <class U> uninit_alloc(const uninit_alloc<U> &) noexcept {}
  template <class U> void construct(U *p) noexcept { ::new ((void *)p) U; }
  template <class U, class... A> void construct(U *p, A &&...a) { ::new ((void *)p) U(static_cast<A &&>(a)...); }
};

struct HostPattern {
  size_t n = 0, nnz = 0;
  std::vector<uint32_t> ia, ja, diag;
  std::vector<uint32_t> tblk;        // block (i,j) -> index of block (j,i)
  std::vector<uint32_t> lpos;        // first persistent L slot of each row
  std::vector<uint32_t> last_lower;  // per row: lower block the fill touches last (or ~0)
  std::vector<uint32_t> lev_l, lev_l_ptr;   // rows by forward level (matrix/init.cpp:194-232)
  std::vector<uint32_t> lev_u, lev_u_ptr;   // rows by backward level (matrix/init.cpp:234-270)
  // ILU(0) products of block j = (i,k) in merge order (matrix/ilu.cpp:71-84):
  // pairs [pair_ptr[j], pair_ptr[j+1]) of (L slot index or ~0 for the
  // identity, block index of U(m,k)); the last pair is the product the
  // reference adds back.
  std::vector<uint32_t> pair_ptr;
  std::vector<uint32_t, uninit_alloc<uint32_t>> pairs;
  // built on the device (kf_build_pattern_device): tblk, pair_ptr and pairs
  // are then only on the device
  bool on_device = false;
};

void kf_build_pattern(HostPattern &p, size_t nnodes, size_t nedges, const unsigned int *n0,
                      const unsigned int *n1);

struct DevMesh;

// The opaque handle behind GEOMETRY::matrix.  The edges given to
// CXX_Matrix_Init are kept; the block pattern is built on the device with the
// device mirror, or on the host threads when host code asks for it first
// (kf_host_pattern).
struct MatrixHandle {
  uint32_t magic = 0x4B463344u;   // "KF3D"
  std::vector<uint32_t> e0, e1;   // the edges (n0, n1)
  HostPattern pat;                // pat.n is set at CXX_Matrix_Init, the rest when built
  DevMesh *dev = nullptr;
  const GEOMETRY *owner = nullptr;
};

MatrixHandle *kf_handle(const GEOMETRY *g);
// The handle's host pattern, built on the host threads if it has not been
// built yet (with the full product lists), for host-side readers.
const HostPattern &kf_host_pattern(MatrixHandle *h);

#ifdef __CUDACC__

constexpr int KF_NBASIS = 31;

// Grid-wide barrier for cooperative launches, with a bounded wait.  bar[0]
// counts arrivals, bar[1] is the generation; both start at zero.  Returns
// false (and sets *err) if the wait gave up, after which every caller skips
// the rest of its work.
constexpr uint32_t KF_BARRIER_LIMIT = 1u << 22;
__device__ __forceinline__ bool kf_grid_barrier(unsigned *bar, int *err)
{
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned *gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x * gridDim.y * gridDim.z - 1) {
      bar[0] = 0;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned spins = 0;
      while (*gen == g) {
        if (++spins > KF_BARRIER_LIMIT) { atomicExch(err, 1); ok = 0; break; }
        if ((spins & 255) == 0 && *(volatile int *)err) { ok = 0; break; }
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// The matrix pattern the Jacobian fill, ILU(0) and the triangular solves use:
// the reference's numbering (set 0), or its rows and columns renumbered in a
// spatial order (set 1, kfun3d_set_ilu_order).  fill_* are indexed by node in
// the mesh's numbering and point into the set's pattern.

// Packed level schedule of the triangular solves (trsv_mode 8), one per
// sweep (0 lower, 1 upper): the factor's blocks streamed in level-slot order
// (per slot its lower blocks, or its inverted diagonal block then its upper
// blocks, in column order), so that the rows one CTA solves in one level are
// one contiguous run of the stream.  The blocks are copied into the stream
// after every factorisation (k_trsv_pack, through src).
constexpr uint32_t KF_PK_ROW_MAX = 1536;   // blocks of one row, at most (larger: no packed schedule)
struct PackedSweep {
  uint32_t *row = nullptr;     // [N] matrix row of each slot
  uint32_t *first = nullptr;   // [N+1] first streamed block of each slot
  uint32_t *col = nullptr;     // [nblk] column of each streamed block
  uint32_t *src = nullptr;     // [nblk] matrix block copied to each stream position
  // two cuts of the levels into chunks, [0] of at most 32 rows and 256 blocks
  // (one CTA of 128 threads), [1] of at most 64 rows and 512 blocks (256
  // threads); a row longer than the budget is a chunk of its own
  uint4 *chunk[2] = {nullptr, nullptr};   // per CTA: (first slot, end slot, first block, end block)
  std::vector<uint32_t> lev[2];           // first chunk of each level, nlev + 1 entries
  uint32_t maxblk[2] = {0, 0};            // blocks of the largest chunk
  uint32_t nblk = 0;                      // blocks in the stream
};

struct IluSet {
  bool valid = false;
  uint32_t *ia = nullptr, *ja = nullptr, *diag = nullptr, *tblk = nullptr, *lpos = nullptr;
  uint32_t *last_lower = nullptr, *pair_ptr = nullptr;
  uint2 *pairs = nullptr;
  uint32_t *lev_l = nullptr, *lev_u = nullptr, *lev_ptr_d = nullptr;
  std::vector<uint32_t> lev_l_ptr, lev_u_ptr;
  uint32_t nlev_l = 0, nlev_u = 0;
  uint4 *desc_l = nullptr, *desc_u = nullptr;
  int trsv_mode = 4;
  uint32_t *fill_blk = nullptr;    // [2E] block of (node, other) per incidence (CSR order)
  uint32_t *fill_diag = nullptr;   // [N] diagonal block of each node
  uint32_t *fill_last = nullptr;   // [N] the node's row's last-touched lower block (or ~0)
  uint32_t *fill_lpos = nullptr;   // [N] the node's row's first persistent L slot
  uint32_t *row_node = nullptr;    // [N] node of each matrix row (null: the identity)
  PackedSweep pk[2];               // packed level schedule (trsv_mode 8)
};

// Level-slot descriptors of both sweeps, (row, first block, end block, 0):
// the lower sweep's blocks left of the diagonal, the upper sweep's right of
// it; within a level the longest rows first (stable), so that the groups that
// take a second row take short ones.
void kf_level_descriptors(const HostPattern &p, std::vector<uint4> &desc_l, std::vector<uint4> &desc_u);
// Builds the packed level schedule of one pattern from its level-slot
// descriptors (host copies for the chunk cuts, device copies for the
// streams) and level offsets; ja and diag are the pattern's device arrays.
// KFUN3D_OK, KFUN3D_ERR_ARG (a row too long: no packed schedule) or
// KFUN3D_ERR_CUDA, with nothing left allocated on error.
int kf_build_packed(PackedSweep pk[2], const HostPattern &p, const std::vector<uint4> &desc_l,
                    const std::vector<uint4> &desc_u, const uint4 *ddesc_l, const uint4 *ddesc_u,
                    const uint32_t *ja, const uint32_t *diag, cudaStream_t st);
int kf_packed_streams_device(uint32_t N, bool upper, const uint4 *desc, const uint32_t *first, const uint32_t *ja,
                             const uint32_t *diag, uint32_t *row, uint32_t *col, uint32_t *src, cudaStream_t st);
void kf_free_packed(PackedSweep pk[2]);

// The block pattern built on the device (setup_device.cu): the device arrays,
// and into `host` the arrays the host set-up code reads (ia, ja, diag, lpos,
// last_lower, the level lists).  KFUN3D_OK or an error code, nothing left
// allocated on error.
struct DevPattern {
  uint32_t *ia = nullptr, *ja = nullptr, *diag = nullptr, *tblk = nullptr, *lpos = nullptr;
  uint32_t *last_lower = nullptr, *pair_ptr = nullptr;
  uint2 *pairs = nullptr;
  size_t npairs = 0;
};
int kf_build_pattern_device(HostPattern &host, DevPattern &d, size_t N, size_t E, const unsigned int *n0,
                            const unsigned int *n1, cudaStream_t st);
void kf_free_device_pattern(DevPattern &d);
// The mirror's edge geometry (egeo), node incidence lists (inc_*), two-pass
// edge storage (eoff, n0s, n1, egeo_s, in1_*) and visit-order copies
// (inc_othv, inc_geo, n0v, n1v, xyzv), built on the device from the
// GEOMETRY's edges, edge geometry and least-squares terms; m.ord, m.rowof,
// m.xyz, the block pattern, m.two_pass and m.visit are set before.  KFUN3D_OK
// or an error code (the arrays made so far are the mirror's, freed with it).
int kf_build_mesh_lists_device(DevMesh &m, const GEOMETRY *g);
// The fill's targets in the renumbered pattern of `s` (fill_blk per
// incidence, fill_diag / fill_last / fill_lpos per node, row_node per row),
// from m.ilu_rank and the mirror's incidence lists, on the device.
int kf_fill_targets_device(const DevMesh &m, IluSet &s);
// 1 when every pattern array of `s` (on the device) and its level lists equal
// kf_build_pattern's for the same edges, 0 when one differs, -1 on a CUDA error;
// *host_us (if given) the host build's wall time in microseconds
int kf_pattern_matches(const IluSet &s, size_t N, size_t E, const unsigned int *n0, const unsigned int *n1,
                       cudaStream_t st, long *host_us);

// Device mirror of one GEOMETRY.  Node-indexed arrays follow the reference's
// numbering; edge-indexed arrays its (sorted) edge order.
struct DevMesh {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t N = 0, E = 0, Ns = 0, Nf = 0, F = 0, ncol = 0, nnz = 0, nlower = 0;
  // static geometry
  double4 *egeo = nullptr;        // [E] unit normal n0->n1, area
  double4 *xyz = nullptr;         // [N] coordinates, w = 0
  uint32_t *ord = nullptr;        // [N] node visited at position p by the node-centric gathers
  uint32_t *rowof = nullptr;      // [N] position (CSR row) of each node
  bool spatial_order = false;     // ord is the Morton order (not the mesh's own)
  uint32_t *inc_ptr = nullptr;    // [N+1] incident edges of node ord[p] (row p), in edge order
  uint32_t *inc_oth = nullptr;    // [2E] the other end point
  uint32_t *inc_edge = nullptr;   // [2E] edge index | (1u<<31 when the node is n1)
  uint32_t *inc_blk = nullptr;    // [2E] block index of (node, other)
  double *inc_w = nullptr;        // [3][wstride] least-squares terms seen from the node
  uint32_t wstride = 0;           // 2E rounded up to a multiple of 4 (16-byte aligned rows)
  unsigned grad_smem = 0;         // dynamic shared memory of k_gradient_tma (0: not used)
  double4 *lsq_coef = nullptr;    // [2N] least-squares coefficients per node, computed on the device
  // host wall time of the set-up, microseconds: the whole device mirror, its
  // block pattern on the device, the spatial ILU(0) order's set (0 until built)
  long setup_us = 0, pattern_us = 0, spatial_us = 0;
  long host_pattern_us = -1;      // the same pattern on the host threads (set by the pattern check)
  bool lsq_match = false;         // the terms recomputed from lsq_coef equal the stored ones bit for bit
  int grad_lanes = 1;             // lanes per node of the gradient in the mesh's order (1 or 4)
  // visit-order copies for the residual passes on large meshes (spatial_order
  // and two_pass): state, coordinates, gradients, the other end of each
  // incidence and the end points of each stored edge as visit positions
  bool visit = false;
  double4 *qv = nullptr, *xyzv = nullptr, *gxv = nullptr, *gyv = nullptr, *gzv = nullptr;
  uint32_t *inc_othv = nullptr, *n0v = nullptr, *n1v = nullptr;
  double4 *inc_geo = nullptr;     // [2E] edge geometry per incidence (CSR order), for the time step and fill
  // two-pass residual (every edge has n0 < n1); edge arrays in storage
  // order: grouped by n0 in node-visit order (ord), each group in edge order
  bool two_pass = false;
  uint32_t *eoff = nullptr;       // [N+1] storage range of the edges with n0 = ord[p]
  uint32_t *n0s = nullptr;        // [E] n0 of each stored edge
  uint32_t *n1 = nullptr;         // [E] n1 of each stored edge
  double4 *egeo_s = nullptr;      // [E] edge geometry in storage order
  uint32_t *in1_ptr = nullptr;    // [N+1] edges with n1 = ord[p], in edge order
  uint32_t *in1_edge = nullptr;   // [E] their storage positions
  double4 *eres = nullptr;        // [E] edge fluxes, storage order
  uint32_t *wf_nodes = nullptr;   // [3F] wall faces in colour order
  double *wf_n = nullptr;         // [3F] wall-face normals -(1/6) a x b
  uint32_t *col = nullptr;        // [ncol+1] wall-face colour offsets
  double *s_n = nullptr;          // [3 Ns] wall-node normals
  double *f_n = nullptr;          // [3 Nf] far-field node normals
  uint32_t nb = 0;                // boundary nodes
  uint32_t *bnd_of = nullptr;     // [N] position in bnd_node, or ~0
  uint32_t *bnd_node = nullptr;   // [nb]
  uint32_t *bnd_ptr = nullptr;    // [nb+1]
  uint32_t *bnd_ent = nullptr;    // entries: kind << 29 | index
  // block matrix
  uint32_t *ia = nullptr, *ja = nullptr, *diag = nullptr, *tblk = nullptr;
  uint32_t *lpos = nullptr, *last_lower = nullptr;
  uint32_t nlev_l = 0, nlev_u = 0;
  std::vector<uint32_t> lev_l_ptr, lev_u_ptr;   // host copies of level offsets
  uint32_t *lev_l = nullptr, *lev_u = nullptr;
  uint32_t *pair_ptr = nullptr;   // [nnz+1]
  uint2 *pairs = nullptr;         // [npairs] (L slot or ~0, U block)
  double *A = nullptr;            // [nnz*16]
  double *lslot = nullptr;        // [nlower*16] persistent L slots
  double *dinv = nullptr;         // [N*16] inverse diagonal blocks
  float *Af = nullptr;            // [nnz*16] FP32 form
  float *dinvf = nullptr;         // [N*16]
  // state and work vectors (4N doubles each)
  double *q = nullptr, *r = nullptr, *gx = nullptr, *gy = nullptr, *gz = nullptr;
  double *cdt = nullptr, *w = nullptr, *t = nullptr, *x = nullptr, *rhs = nullptr;
  double *V = nullptr;            // [KF_NBASIS][4N]
  double *red = nullptr;          // reduction scratch
  double *scal = nullptr;         // device scalars
  double *forces = nullptr;       // [3]
  double *dscr = nullptr;         // [nb*16] double diagonal blocks of boundary rows (FP32 fill)
  int *status = nullptr;          // device status words: [0] pivot failure, [1] wait timeout
  // sync-free triangular solves
  bool syncfree = true;
  int trsv_mode = 8;               // 0 levels (4 lanes/row), 1 sync-free, 3 one persistent launch,
                                   // grid barrier between levels, 4 levels with programmatic
                                   // dependent launch (16 lanes/row), 5 one persistent launch,
                                   // 1-3 CTAs per SM, counter barrier, 7 the same with 4 lanes/row,
                                   // 8 packed level launches (default)
  unsigned trsv_grid = 0;          // persistent grid (whole blocks resident on every SM)
  uint32_t *flags = nullptr;       // [N] per-row completion epoch
  unsigned long long *ticket = nullptr;   // unused (kept zero)
  uint4 *desc_l = nullptr, *desc_u = nullptr;   // [N] (row, first block, end block) in level order
  // fast mode: one CUDA graph per Arnoldi index (jacobian-vector product,
  // triangular solves, Gram-Schmidt, read-back of the Hessenberg column)
  cudaGraphExec_t arnoldi[2][2][KF_NBASIS] = {};   // [precision][first order][k]
  unsigned arnoldi_nodes[2][2][KF_NBASIS] = {};
  double graph_aoa = 0.0;
  bool use_graphs = true;
  unsigned mgs_grid = 0;          // cooperative grid for the Gram-Schmidt kernel
  bool mgs_resident = true;       // Gram-Schmidt with w kept on chip (k_mgs_resident)
  int mgs_ts = 0;                 // its double2 elements per thread in shared memory
  double *part = nullptr;         // [2][mgs_grid] block partial sums
  unsigned *bar = nullptr;        // grid-barrier words: [0..1] persistent sweep, [2..3] Gram-Schmidt,
                                  // [4] counter of the one-CTA-per-SM sweep
  uint32_t *lev_ptr_d = nullptr;  // [nlev_l+1 + nlev_u+1] level offsets on the device
  unsigned trsv_pgrid = 0;        // persistent sweep grid
  unsigned trsv_mgrid = 0;        // persistent sweep grid of mode 5 (SMs x trsv_mgrid_per)
  int trsv_mgrid_per = 2;         // 512-thread CTAs per SM in mode 5 (1, 2 or 3)
  int trsv_lanes = 8;             // lanes per row in mode 5 (8 or 16)
  double *h_scal = nullptr;       // pinned host mirror of scal
  // ILU(0) ordering: the active set's fields are copied into the fields above
  IluSet iset[2];
  PackedSweep pk[2];              // active set's packed level schedule
  int pk_cut[2] = {0, 0};         // chunk cut used with FP64 / FP32 factors (0: 32 rows, 1: 64 rows)
  bool pk_fp64 = false;           // FP64 factors also take the packed schedule (KFUN3D_PK_FP64=1)
  void *pk_buf = nullptr;         // the packed factor: lower stream, then upper stream (FP64 or FP32 blocks)
  int ilu_active = 0;             // 1: the spatial set is active
  uint32_t *ilu_rank = nullptr;   // [N] row of each node in the spatial set
  double *pb = nullptr, *px = nullptr;   // [4N] right-hand side and solution, spatial numbering
  int graph_ilu = 0;              // ILU set the Arnoldi graphs were captured with
  uint32_t *fill_blk = nullptr, *fill_diag = nullptr, *fill_last = nullptr, *fill_lpos = nullptr;
  uint32_t *row_node = nullptr;   // active set's node of each matrix row (null: the identity)
  // additive Schwarz subdomains (kfun3d_set_schwarz): sub_part[node] for
  // sub_parts subdomains; 0 parts: the whole mesh is one domain
  uint32_t *sub_part = nullptr;
  uint32_t sub_parts = 0;
  // the state whose visit-order copy qv already holds, written together with
  // it by its producer; the next visit-order gather of that state is skipped
  // (one-shot)
  const double *qv_of = nullptr;
  // flexible GMRES (right preconditioning) and the learned preconditioner
  double *Z = nullptr;            // [30][4N] preconditioned basis vectors
  double *qold = nullptr;         // [4N] state before the last update
  double *fy = nullptr;           // [4N] ILU(0)-preconditioned vector
  double *fx = nullptr;           // [4N] iterate of a training pair
  double *pscr = nullptr;         // [264] scratch of the pair features
  kfun3d_mpnn_graph *mgraph = nullptr;   // the network's graph of this mesh
  bool factored = false;
  int factor_precision = 0;       // precision of the last ILU(0) factorisation (0 FP64, 1 FP32)
  bool a_valid = false;
};

DevMesh *kf_device(const GEOMETRY *g);   // creates and uploads on first use
int kf_ilu_order();
// Makes the ILU(0) ordering `order` (0 the mesh's numbering, 1 spatial) the
// active one, building set 1 on first use; KFUN3D_OK or an error code.
int kf_ilu_select(DevMesh &m, const GEOMETRY *g, int order);
unsigned kf_schwarz();
// Makes `parts` additive Schwarz subdomains (0 or 1: none) the mesh's
// current ones, computing and uploading the partition on a change.
int kf_schwarz_select(DevMesh &m, const GEOMETRY *g, unsigned parts);
// Recursive coordinate bisection of the nodes into `parts` subdomains.
std::vector<uint32_t> kf_partition_rcb(const double *X, const double *Y, const double *Z, size_t N, uint32_t parts);

void kf_count_launch(unsigned n = 1);
void kfun3d_reset_launch_count_by(unsigned long long n);   // undo counts taken during graph capture

// Kernel families, one set per arithmetic mode (kernels_exact.cu, kernels_fast.cu).
#define KF_DECLARE_KERNELS(NS)                                                          \
  namespace NS {                                                                        \
  void gradient(DevMesh &m, const double *q);                                           \
  int bounded_wait_check(cudaStream_t st);                                              \
  void residual(DevMesh &m, const double *q, double *r, int first_order, double u, double v); \
  void timestep(DevMesh &m, const double *q, double cfl);                               \
  void fill(DevMesh &m, const double *q, double u, double v, int precision);            \
  void ilu(DevMesh &m, int precision);                                                  \
  void sptrsv(DevMesh &m, const double *b, double *x, int precision);                   \
  bool sptrsv_permuted(DevMesh &m, const double *b, double *x, int precision);         \
  void sptrsv_flags(DevMesh &m, const double *b, double *x, int precision, uint32_t *flags); \
  int lsq_setup(DevMesh &m);                                                            \
  void gradient_to_mesh_order(DevMesh &m);                                              \
  void jv_combine(DevMesh &m, double *y, const double *r, const double *w,              \
                  const double *q, const double *scal, int ia);                          \
  }
KF_DECLARE_KERNELS(kf_exact)
KF_DECLARE_KERNELS(kf_fast)

// Learned preconditioner (mpnn.cu), for the solver: workspace for a graph
// (allocates; call before any capture), the correction z = y + s N([y/s, q])
// enqueued on a stream, the completion status of its bounded waits, and the
// features/target of a training pair (scr: 264 doubles of device scratch).
int kf_mpnn_prepare(kfun3d_mpnn *net, kfun3d_mpnn_graph *G);
int kf_mpnn_apply_async(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const double *y, const double *q, double *z,
                        cudaStream_t st);
int kf_mpnn_status(kfun3d_mpnn *net, cudaStream_t st);
int kf_mpnn_pair_async(size_t nnodes, const double *y, const double *q, const double *x, void *x0, float *tgt,
                       double *scr, cudaStream_t st);

#endif
