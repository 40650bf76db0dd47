// kfun3d_b200: ILU(0) in a spatial ordering (option for the fast forms).
//
// With a random node numbering (the meshes here are numbered at random, as
// the reference's inputs may be) ILU(0) of the Jacobian in the mesh's own
// order is weak: on the 120^3 box the solve needs 1556 GMRES iterations
// against 761 when rows and columns are eliminated in a spatially coherent
// order.  Set 1 renumbers the block pattern by a spatial order of the nodes:
// the matrix becomes P A P^T, ILU(0) factors that (same sparsity, different
// elimination order) and a triangular solve runs x = P^T (L U)^-1 P b.  The
// Jacobian blocks themselves are unchanged; the fill writes them into the
// renumbered pattern.  Not a parity path: the reference factors in its own
// order, which stays the default (kfun3d_set_ilu_order(0)).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace {

// (waits for the copy to land: see device_mesh.cu's upload)
template <class T> cudaError_t upload(T **dst, const T *src, size_t n)
{
  cudaError_t e = cudaMalloc((void **)dst, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess || n == 0) return e;
  e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
}

template <class F> void parallel_ranges(size_t n, F f)
{
  const unsigned T = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (n < 65536 || T == 1) {
    f((size_t)0, n);
    return;
  }
  std::vector<std::thread> th;
  const size_t chunk = (n + T - 1) / T;
  for (unsigned t = 0; t < T; t++) {
    const size_t a = t * chunk, b = std::min(n, a + chunk);
    if (a < b) th.emplace_back(f, a, b);
  }
  for (auto &x : th) x.join();
}

void activate(DevMesh &m, const IluSet &s)
{
  m.ia = s.ia; m.ja = s.ja; m.diag = s.diag; m.tblk = s.tblk; m.lpos = s.lpos;
  m.last_lower = s.last_lower; m.pair_ptr = s.pair_ptr; m.pairs = s.pairs;
  m.lev_l = s.lev_l; m.lev_u = s.lev_u; m.lev_ptr_d = s.lev_ptr_d;
  m.lev_l_ptr = s.lev_l_ptr; m.lev_u_ptr = s.lev_u_ptr;
  m.nlev_l = s.nlev_l; m.nlev_u = s.nlev_u;
  m.desc_l = s.desc_l; m.desc_u = s.desc_u;
  m.trsv_mode = s.trsv_mode;
  m.syncfree = s.trsv_mode == 1;
  m.fill_blk = s.fill_blk; m.fill_diag = s.fill_diag; m.fill_last = s.fill_last; m.fill_lpos = s.fill_lpos;
  m.pk[0] = s.pk[0];
  m.pk[1] = s.pk[1];
  m.row_node = s.row_node;
}

// Tiles of the tile-major order (KFUN3D_ILU_PERM=tiles): columns along the
// sweep direction (1,1,1), cut in the plane across it (u = x - y, w = x + y - 2z) into
// floor(sqrt(T)) strips by u, each strip into cells by w, with equal shares
// of the cross-section rather than of the nodes: a node weighs 1 / (the
// extent in s = x + y + z of the nodes that project near it, on a 64 x 64
// grid of the (u, w) plane), so every tile holds about the same number of
// rows of each level.  Tile ids run strip by strip.
std::vector<uint32_t> partition_tiles(const double *X, const double *Y, const double *Z, size_t N, uint32_t T)
{
  std::vector<uint32_t> tile(N, 0);
  if (T <= 1 || N == 0) return tile;
  const uint32_t Tu = std::max(1u, (uint32_t)std::floor(std::sqrt((double)T)));
  std::vector<uint32_t> idx(N);
  std::vector<double> u(N), w(N), sv(N), wt(N);
  double ulo = 1e300, uhi = -1e300, wlo = 1e300, whi = -1e300;
  for (size_t i = 0; i < N; i++) {
    idx[i] = (uint32_t)i;
    u[i] = X[i] - Y[i];
    w[i] = (X[i] + Y[i]) - 2.0 * Z[i];
    sv[i] = (X[i] + Y[i]) + Z[i];
    ulo = std::min(ulo, u[i]); uhi = std::max(uhi, u[i]);
    wlo = std::min(wlo, w[i]); whi = std::max(whi, w[i]);
  }
  constexpr int B = 64;
  auto bin = [&](size_t i) {
    const int bu = (int)std::min<double>(B - 1, std::max(0.0, (u[i] - ulo) / std::max(uhi - ulo, 1e-300) * B));
    const int bw = (int)std::min<double>(B - 1, std::max(0.0, (w[i] - wlo) / std::max(whi - wlo, 1e-300) * B));
    return bu * B + bw;
  };
  std::vector<double> smin(B * B, 1e300), smax(B * B, -1e300);
  double slo = 1e300, shi = -1e300;
  for (size_t i = 0; i < N; i++) {
    const int k = bin(i);
    smin[k] = std::min(smin[k], sv[i]);
    smax[k] = std::max(smax[k], sv[i]);
    slo = std::min(slo, sv[i]);
    shi = std::max(shi, sv[i]);
  }
  const double floor_ext = std::max(shi - slo, 1e-300) / 64.0;
  double total = 0.0;
  for (size_t i = 0; i < N; i++) {
    const int k = bin(i);
    wt[i] = 1.0 / std::max(smax[k] - smin[k], floor_ext);
    total += wt[i];
  }
  // consecutive runs of idx[a, b) with equal shares of weight
  auto cut = [&](size_t a, size_t b, uint32_t parts, double share, auto &&emit) {
    double acc = 0.0;
    uint32_t part = 0;
    size_t c0 = a;
    for (size_t q = a; q < b; q++) {
      acc += wt[idx[q]];
      if (part + 1 < parts && acc >= share * (part + 1)) {
        emit(part, c0, q + 1);
        c0 = q + 1;
        part++;
      }
    }
    emit(part, c0, b);
    for (uint32_t rest = part + 1; rest < parts; rest++) emit(rest, b, b);
  };
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return u[a] < u[b]; });
  // strip k takes cells[k] / T of the weight
  std::vector<uint32_t> cells(Tu);
  for (uint32_t k = 0; k < Tu; k++) cells[k] = T / Tu + (k < T % Tu ? 1u : 0u);
  std::vector<std::pair<size_t, size_t>> strips(Tu, {N, N});
  {
    double acc = 0.0, target = total * cells[0] / T;
    size_t start = 0;
    uint32_t k = 0;
    for (size_t q = 0; q < N && k + 1 < Tu; q++) {
      acc += wt[idx[q]];
      if (acc >= target) {
        strips[k] = {start, q + 1};
        start = q + 1;
        k++;
        target += total * cells[k] / T;
      }
    }
    strips[k] = {start, N};
  }
  uint32_t t0 = 0;
  for (uint32_t k = 0; k < Tu; k++) {
    const size_t a = strips[k].first, b = strips[k].second;
    std::stable_sort(idx.begin() + a, idx.begin() + b, [&](uint32_t x0, uint32_t x1) { return w[x0] < w[x1]; });
    double sw = 0.0;
    for (size_t q = a; q < b; q++) sw += wt[idx[q]];
    cut(a, b, cells[k], sw / cells[k], [&](uint32_t c, size_t c0, size_t c1) {
      for (size_t q = c0; q < c1; q++) tile[idx[q]] = t0 + c;
    });
    t0 += cells[k];
  }
  return tile;
}

// Position of every node in the spatial elimination order.  ILU(0) depends
// only on which of two neighbours is eliminated first; orders that follow a
// sweep of the coordinates orient the edges as the lexicographic order of a
// lattice does (the strong ordering) while keeping the level sets few.  With
// s = x + y + z:
//   slabs (default): the range of s cut into K slabs (KFUN3D_ILU_SLABS,
//     default 4), each swept from both of its faces towards its middle
//     (descending |s - middle of the slab|, ties in node order).  On the
//     120^3 box: 803 GMRES iterations and a 2.1 ms FP32 triangular solve,
//     against 728 and 2.7 ms for K = 1, 704 and 3.6 ms for one sweep, 1556
//     and 1.3 ms in the mesh's random numbering;
//   KFUN3D_ILU_PERM=tiles: tile by tile (ids as above), ascending s within a
//     tile: between tiles the edges point from the lower tile id to the
//     higher (an order whose tiles depend on their neighbours one way only);
//   KFUN3D_ILU_PERM=sweep: ascending s over the whole mesh (level sets: about
//     3n on an n^3 Kuhn box, against about 9n for the Morton order of the
//     jittered coordinates);
//   KFUN3D_ILU_PERM=morton: Morton order of the coordinates, 21 bits per axis
//     over the bounding box;
//   KFUN3D_ILU_PERM=identity: the mesh's own order through the renumbering
//     code (reproduces the mesh order bit for bit; a test hook).
// Ties keep node order in every case.
std::vector<uint32_t> spatial_rank(const GEOMETRY *g, size_t N, const std::vector<uint32_t> &tile)
{
  std::vector<uint32_t> rank(N), ord(N);
  for (size_t i = 0; i < N; i++) ord[i] = (uint32_t)i;
  const char *env = getenv("KFUN3D_ILU_PERM");
  const std::string kind = env ? env : "slabs";
  if (kind == "identity") return ord;
  const double *X = g->n->xyz->x0, *Y = g->n->xyz->x1, *Z = g->n->xyz->x2;
  if (kind == "morton") {
    double lo[3] = {X[0], Y[0], Z[0]}, hi[3] = {X[0], Y[0], Z[0]};
    for (size_t i = 0; i < N; i++) {
      const double c[3] = {X[i], Y[i], Z[i]};
      for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], c[d]); hi[d] = std::max(hi[d], c[d]); }
    }
    auto spread = [](uint64_t v) {
      v &= 0x1fffffull;
      v = (v | v << 32) & 0x1f00000000ffffull;
      v = (v | v << 16) & 0x1f0000ff0000ffull;
      v = (v | v << 8) & 0x100f00f00f00f00full;
      v = (v | v << 4) & 0x10c30c30c30c30c3ull;
      v = (v | v << 2) & 0x1249249249249249ull;
      return v;
    };
    std::vector<uint64_t> key(N);
    for (size_t i = 0; i < N; i++) {
      const double c[3] = {X[i], Y[i], Z[i]};
      uint64_t k = 0;
      for (int d = 0; d < 3; d++) {
        const double span = hi[d] > lo[d] ? hi[d] - lo[d] : 1.0;
        const uint64_t b = (uint64_t)std::min(2097151.0, std::max(0.0, (c[d] - lo[d]) / span * 2097151.0));
        k |= spread(b) << d;
      }
      key[i] = k;
    }
    kf_sort_by_key(ord, key);
  } else {
    std::vector<double> key(N);
    for (size_t i = 0; i < N; i++) key[i] = (X[i] + Y[i]) + Z[i];
    if (kind == "tiles") {
      std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
        return tile[a] != tile[b] ? tile[a] < tile[b] : key[a] < key[b];
      });
    } else {
      if (kind != "sweep") {
        double lo = 1e300, hi = -1e300;
        for (size_t i = 0; i < N; i++) { lo = std::min(lo, key[i]); hi = std::max(hi, key[i]); }
        int K = 4;
        const char *kenv = getenv("KFUN3D_ILU_SLABS");
        if (kenv && atoi(kenv) >= 1 && atoi(kenv) <= 64) K = atoi(kenv);
        const double w = std::max((hi - lo) / K, 1e-300);
        for (size_t i = 0; i < N; i++) {
          const int sl = std::min(K - 1, (int)((key[i] - lo) / w));
          key[i] = -std::fabs(key[i] - (lo + (sl + 0.5) * w));
        }
      }
      kf_sort_by_key(ord, key);
    }
  }
  for (size_t p = 0; p < N; p++) rank[ord[p]] = (uint32_t)p;
  return rank;
}


int build_spatial(DevMesh &m, const GEOMETRY *g)
{
  const size_t N = m.N, E = m.E;
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m.device);
  const uint32_t T = (uint32_t)std::max(1, nsm);
  SetupTrace tr("spatial order");
  // tiles only for the tile-major order
  const char *perm = getenv("KFUN3D_ILU_PERM");
  const std::vector<uint32_t> tile = perm && strcmp(perm, "tiles") == 0
                                         ? partition_tiles(g->n->xyz->x0, g->n->xyz->x1, g->n->xyz->x2, N, T)
                                         : std::vector<uint32_t>();
  const std::vector<uint32_t> rank = spatial_rank(g, N, tile);
  tr.mark("rank");
  std::vector<uint32_t> pn0(E), pn1(E);
  for (size_t e = 0; e < E; e++) { pn0[e] = rank[n0[e]]; pn1[e] = rank[n1[e]]; }
  // the permuted block pattern, built on the device
  HostPattern p;
  DevPattern dp;
  if (kf_build_pattern_device(p, dp, N, E, pn0.data(), pn1.data(), m.stream) != KFUN3D_OK) return KFUN3D_ERR_CUDA;
  tr.mark("renumbered edges, block pattern on the device");
  IluSet &s = m.iset[1];
  s.ia = dp.ia; s.ja = dp.ja; s.diag = dp.diag; s.tblk = dp.tblk; s.lpos = dp.lpos;
  s.last_lower = dp.last_lower; s.pair_ptr = dp.pair_ptr; s.pairs = dp.pairs;
  bool ok = true;
  auto up = [&](auto **dst, const auto &vec) {
    if (ok && upload(dst, vec.data(), vec.size()) != cudaSuccess) ok = false;
  };
  up(&s.lev_l, p.lev_l);
  up(&s.lev_u, p.lev_u);
  s.lev_l_ptr = p.lev_l_ptr;
  s.lev_u_ptr = p.lev_u_ptr;
  s.nlev_l = (uint32_t)p.lev_l_ptr.size() - 1;
  s.nlev_u = (uint32_t)p.lev_u_ptr.size() - 1;
  {
    std::vector<uint32_t> lp(p.lev_l_ptr);
    lp.insert(lp.end(), p.lev_u_ptr.begin(), p.lev_u_ptr.end());
    up(&s.lev_ptr_d, lp);
  }
  {
    std::vector<uint4> dl, du;
    kf_level_descriptors(p, dl, du);
    up(&s.desc_l, dl);
    up(&s.desc_u, du);
    if (ok && kf_build_packed(s.pk, p, dl, du, s.desc_l, s.desc_u, s.ja, s.diag, m.stream) == KFUN3D_ERR_CUDA)
      ok = false;
  }
  tr.mark("level descriptors, packed schedule");
  // the fill's view of the renumbered pattern, per node of the mesh, and
  // the node of each renumbered row (on the device)
  up(&m.ilu_rank, rank);
  if (ok && kf_fill_targets_device(m, s) != KFUN3D_OK) ok = false;
  if (ok && cudaMalloc(&m.pb, 4 * N * sizeof(double)) != cudaSuccess) ok = false;
  if (ok && cudaMalloc(&m.px, 4 * N * sizeof(double)) != cudaSuccess) ok = false;
  // one launch per level (programmatic dependent launch, each CTA's rows one
  // contiguous run of the packed factor) by default; KFUN3D_SPTRSV picks
  // another schedule
  s.trsv_mode = s.pk[0].chunk[0] ? 8 : 7;
  const char *env = getenv("KFUN3D_SPTRSV");
  if (env && strcmp(env, "pdl4") == 0) s.trsv_mode = 7;
  if (env && strcmp(env, "packed") == 0 && s.pk[0].chunk[0]) s.trsv_mode = 8;
  if (env && strcmp(env, "pdl") == 0) s.trsv_mode = 4;
  if (env && strcmp(env, "mono") == 0) s.trsv_mode = 5;
  if (env && strcmp(env, "syncfree") == 0) s.trsv_mode = 1;
  if (!ok) {
    kf_set_error(KFUN3D_ERR_CUDA, "spatial ILU(0) order: out of device memory");
    return KFUN3D_ERR_CUDA;
  }
  tr.mark("fill targets");
  s.valid = true;
  return KFUN3D_OK;
}

}  // namespace

void kf_ilu_release(DevMesh &m);

int kf_ilu_select(DevMesh &m, const GEOMETRY *g, int order)
{
  order = order ? 1 : 0;
  if (order == m.ilu_active) return KFUN3D_OK;
  if (order == 1 && !m.iset[1].valid) {
    kf_ilu_release(m);   // what an earlier attempt that ran out of memory left
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = build_spatial(m, g);
    if (rc != KFUN3D_OK) return rc;
    m.spatial_us = (long)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0)
                       .count();
  }
  activate(m, m.iset[order]);
  m.ilu_active = order;
  m.factored = false;
  // the persistent L slots hold the other numbering's factor: start afresh
  if (cudaMemsetAsync(m.lslot, 0, (16 * (size_t)m.nlower + 16) * sizeof(double), m.stream) != cudaSuccess) {
    kf_set_error(KFUN3D_ERR_CUDA, "spatial ILU(0) order: clearing the L slots failed");
    return KFUN3D_ERR_CUDA;
  }
  return KFUN3D_OK;
}

void kf_ilu_release(DevMesh &m)
{
  if (m.ilu_active && m.iset[0].valid) {
    activate(m, m.iset[0]);
    m.ilu_active = 0;
  }
  IluSet &s = m.iset[1];
  void *ptrs[] = {s.ia, s.ja, s.diag, s.tblk, s.lpos, s.last_lower, s.pair_ptr, s.pairs, s.lev_l, s.lev_u,
                  s.lev_ptr_d, s.desc_l, s.desc_u, s.fill_blk, s.fill_diag, s.fill_last, s.fill_lpos, s.row_node,
                  m.ilu_rank, m.pb, m.px};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  kf_free_packed(s.pk);
  s = IluSet{};
  m.ilu_rank = nullptr;
  m.pb = m.px = nullptr;
}

extern "C" long kfun3d_ilu_rank(const GEOMETRY *g, unsigned int *rank)
{
  MatrixHandle *h = kf_handle(g);
  if (!h || !h->dev || !h->dev->iset[1].valid || !h->dev->ilu_rank) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_ilu_rank: the spatial ILU order has not been built for this GEOMETRY");
    return -1;
  }
  DevMesh &m = *h->dev;
  if (rank && cudaMemcpy(rank, m.ilu_rank, (size_t)m.N * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
    kf_set_error(KFUN3D_ERR_CUDA, "kfun3d_ilu_rank: copy failed");
    return -1;
  }
  return (long)m.N;
}

extern "C" int kfun3d_ilu_order_plan(const GEOMETRY *g, unsigned int tiles, unsigned int *rank,
                                     unsigned int *nlev_lower, unsigned int *nlev_upper)
{
  if (!g || !g->n || !g->e || !g->n->xyz || tiles < 1) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_ilu_order_plan: bad arguments");
    return -1;
  }
  const size_t N = g->n->sz, E = g->e->sz;
  const char *perm = getenv("KFUN3D_ILU_PERM");
  const std::vector<uint32_t> tile = perm && strcmp(perm, "tiles") == 0
                                         ? partition_tiles(g->n->xyz->x0, g->n->xyz->x1, g->n->xyz->x2, N, tiles)
                                         : std::vector<uint32_t>();
  const std::vector<uint32_t> r = spatial_rank(g, N, tile);
  if (rank) std::copy(r.begin(), r.end(), rank);
  if (nlev_lower || nlev_upper) {
    const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
    std::vector<uint32_t> pn0(E), pn1(E);
    for (size_t e = 0; e < E; e++) { pn0[e] = r[n0[e]]; pn1[e] = r[n1[e]]; }
    HostPattern p;
    kf_build_pattern(p, N, E, pn0.data(), pn1.data());
    if (nlev_lower) *nlev_lower = (unsigned int)p.lev_l_ptr.size() - 1;
    if (nlev_upper) *nlev_upper = (unsigned int)p.lev_u_ptr.size() - 1;
  }
  return 0;
}

// ----------------------------------------------------------------- additive Schwarz subdomains

// The nodes cut into `parts` subdomains by recursive coordinate bisection: a
// set of nodes going to p parts is split across the longest side of its
// bounding box into floor(p/2) and p - floor(p/2) parts, the first holding
// floor(n * floor(p/2) / p) of its n nodes (those lowest in that coordinate,
// ties by node index), so part sizes differ by at most one node per level of
// the recursion.  The reference partitions its mesh with METIS
// (matrix/matrix.cpp:99-135, src/subdomains.c:118-122) for its threads; a
// geometric cut serves the same purpose here without the library.
std::vector<uint32_t> kf_partition_rcb(const double *X, const double *Y, const double *Z, size_t N, uint32_t parts)
{
  std::vector<uint32_t> part(N, 0);
  if (parts <= 1 || N == 0) return part;
  std::vector<uint32_t> idx(N);
  for (size_t i = 0; i < N; i++) idx[i] = (uint32_t)i;
  const double *C[3] = {X, Y, Z};
  auto split = [&](auto &&self, size_t a, size_t b, uint32_t p0, uint32_t np) -> void {
    if (np <= 1 || b - a <= 1) {
      for (size_t q = a; q < b; q++) part[idx[q]] = p0;
      return;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (size_t q = a; q < b; q++)
      for (int d = 0; d < 3; d++) {
        lo[d] = std::min(lo[d], C[d][idx[q]]);
        hi[d] = std::max(hi[d], C[d][idx[q]]);
      }
    int ax = 0;
    for (int d = 1; d < 3; d++)
      if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
    const uint32_t nl = np / 2;
    const size_t cut = a + (size_t)((unsigned long long)(b - a) * nl / np);
    const double *c = C[ax];
    std::nth_element(idx.begin() + a, idx.begin() + cut, idx.begin() + b,
                     [c](uint32_t u, uint32_t v) { return c[u] < c[v] || (!(c[v] < c[u]) && u < v); });
    self(self, a, cut, p0, nl);
    self(self, cut, b, p0 + nl, np - nl);
  };
  split(split, 0, N, 0, parts);
  return part;
}

int kf_schwarz_select(DevMesh &m, const GEOMETRY *g, unsigned parts)
{
  if (parts <= 1) {
    if (m.sub_parts) m.factored = false;
    m.sub_parts = 0;
    return KFUN3D_OK;
  }
  if (parts == m.sub_parts) return KFUN3D_OK;
  if (!g || !g->n || !g->n->xyz) {
    kf_set_error(KFUN3D_ERR_ARG, "additive Schwarz: the GEOMETRY has no node coordinates");
    return KFUN3D_ERR_ARG;
  }
  const std::vector<uint32_t> part = kf_partition_rcb(g->n->xyz->x0, g->n->xyz->x1, g->n->xyz->x2, m.N, parts);
  if ((!m.sub_part && cudaMalloc(&m.sub_part, (size_t)m.N * sizeof(uint32_t)) != cudaSuccess) ||
      cudaMemcpy(m.sub_part, part.data(), (size_t)m.N * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) {
    kf_set_error(KFUN3D_ERR_CUDA, "additive Schwarz: uploading the subdomains failed");
    return KFUN3D_ERR_CUDA;
  }
  m.sub_parts = parts;
  m.factored = false;
  return KFUN3D_OK;
}

extern "C" int kfun3d_schwarz_partition(const GEOMETRY *g, unsigned int parts, unsigned int *part)
{
  if (!g || !g->n || !g->n->xyz || !part || parts < 1) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_schwarz_partition: bad arguments");
    return -1;
  }
  const std::vector<uint32_t> p = kf_partition_rcb(g->n->xyz->x0, g->n->xyz->x1, g->n->xyz->x2, g->n->sz, parts);
  std::copy(p.begin(), p.end(), part);
  return 0;
}
