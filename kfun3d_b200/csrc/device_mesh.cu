// kfun3d_b200: library state, the matrix handle, and the device mirror of a
// GEOMETRY (built once per GEOMETRY, on its first kernel call).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>

#include "internal.h"

// ----------------------------------------------------------------- settings and status

namespace {
std::atomic<int> g_status{KFUN3D_OK};
std::string g_error;
std::mutex g_mu;
int g_abort = 1;
double g_aoa = 3.0;
int g_mode = KFUN3D_MODE_EXACT;
int g_precision = 0;
int g_ilu_order = 0;
int g_first_order = 0;
unsigned g_schwarz = 0;
std::atomic<unsigned long long> g_launches{0};
}  // namespace

int g_kf_verbose = 1;

void kf_set_error(int code, const char *msg)
{
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_status = code;
    g_error = msg ? msg : "";
  }
  // a failed CUDA call, or no device at all, ends the process like the
  // reference's asserts (unless kfun3d_set_abort_on_error(0)): the reference's
  // void entry points have no other way to report that nothing was computed
  if ((code == KFUN3D_ERR_CUDA || code == KFUN3D_ERR_NO_DEVICE) && g_abort) {
    fprintf(stderr, "kfun3d_b200: %s\n", msg);
    abort();
  }
}

int kf_mode() { return g_mode; }
int kf_precision() { return g_precision; }
int kf_ilu_order() { return g_ilu_order; }
int kf_first_order() { return g_first_order; }
unsigned kf_schwarz() { return g_schwarz; }
void kf_count_launch(unsigned n) { g_launches += n; }
void kfun3d_reset_launch_count_by(unsigned long long n) { g_launches -= n; }

extern "C" {

int kfun3d_gpu_last_status(void) { return g_status; }
const char *kfun3d_gpu_last_error(void) { return g_error.c_str(); }
void kfun3d_clear_status(void)
{
  std::lock_guard<std::mutex> lk(g_mu);
  g_status = KFUN3D_OK;
  g_error.clear();
}
void kfun3d_set_abort_on_error(int on) { g_abort = on; }
void kfun3d_set_aoa(double deg) { g_aoa = deg; }
double kfun3d_get_aoa(void) { return g_aoa; }
// inc/phy.h:8-9
void kfun3d_get_freestream(double *u, double *v)
{
  *u = cos(g_aoa / (180 / M_PI));
  *v = sin(g_aoa / (180 / M_PI));
}
void kfun3d_set_mode(int mode) { g_mode = mode == KFUN3D_MODE_FAST ? KFUN3D_MODE_FAST : KFUN3D_MODE_EXACT; }
int kfun3d_get_mode(void) { return g_mode; }
void kfun3d_set_precision(int p) { g_precision = p ? 1 : 0; }
void kfun3d_set_ilu_order(int o) { g_ilu_order = o ? 1 : 0; }
int kfun3d_get_ilu_order(void) { return g_ilu_order; }
void kfun3d_set_first_order(int on) { g_first_order = on ? 1 : 0; }
void kfun3d_set_schwarz(unsigned int parts) { g_schwarz = parts > 1 ? parts : 0; }
unsigned int kfun3d_get_schwarz(void) { return g_schwarz; }
void kfun3d_set_verbose(int on) { g_kf_verbose = on; }
unsigned long long kfun3d_launch_count(void) { return g_launches; }
void kfun3d_reset_launch_count(void) { g_launches = 0; }

// src/utils.c:5-51
void fun3d_printf(const uint32_t c, const char *format, ...)
{
  static const int codes[6] = {31, 32, 33, 34, 35, 36};
  const int val = c < 6 ? codes[c] : 0;
  va_list ap;
  va_start(ap, format);
  fprintf(stdout, "\x1b[%dm", val);
  vfprintf(stdout, format, ap);
  fprintf(stdout, "\x1b[0m");
  va_end(ap);
}

}  // extern "C"

// ----------------------------------------------------------------- block pattern

// matrix/init.cpp:7-74 (pattern), 194-274 (level sets) and the reference's
// fill order (src/fill.c:496-511) for the persistent-L-slot rule.
// f(begin, end) over [0, n) split across the host's threads (sequential for
// small n); every index is handled by exactly one call.
template <class F> static void parallel_ranges(size_t n, F f)
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

void kf_build_pattern(HostPattern &p, size_t N, size_t E, const unsigned int *n0, const unsigned int *n1)
{
  p.n = N;
  p.ia.assign(N + 1, 0);
  for (size_t e = 0; e < E; e++) { p.ia[n0[e] + 1]++; p.ia[n1[e] + 1]++; }
  for (size_t i = 0; i < N; i++) p.ia[i + 1] += p.ia[i] + 1;
  p.nnz = p.ia[N];
  p.ja.assign(p.nnz, 0);
  // rows filled in parallel, each edge taking the next free slot of both of
  // its rows; a row's order is undone by the sort below
  std::vector<std::atomic<uint32_t>> fillp(N);
  parallel_ranges(N, [&](size_t r0, size_t r1) {
    for (size_t i = r0; i < r1; i++) {
      p.ja[p.ia[i]] = (uint32_t)i;
      fillp[i].store(p.ia[i] + 1, std::memory_order_relaxed);
    }
  });
  parallel_ranges(E, [&](size_t e0, size_t e1) {
    for (size_t e = e0; e < e1; e++) {
      p.ja[fillp[n0[e]].fetch_add(1, std::memory_order_relaxed)] = n1[e];
      p.ja[fillp[n1[e]].fetch_add(1, std::memory_order_relaxed)] = n0[e];
    }
  });
  p.diag.assign(N, 0);
  p.lpos.assign(N + 1, 0);
  parallel_ranges(N, [&](size_t r0, size_t r1) {
    for (size_t i = r0; i < r1; i++) {
      std::sort(p.ja.begin() + p.ia[i], p.ja.begin() + p.ia[i + 1]);
      for (uint32_t j = p.ia[i]; j < p.ia[i + 1]; j++)
        if (p.ja[j] == i) { p.diag[i] = j; break; }
    }
  });
  for (size_t i = 0; i < N; i++) p.lpos[i + 1] = p.lpos[i] + (p.diag[i] - p.ia[i]);
  auto find = [&](uint32_t row, uint32_t col) -> uint32_t {
    auto b = p.ja.begin() + p.ia[row], e = p.ja.begin() + p.ia[row + 1];
    auto it = std::lower_bound(b, e, col);
    return (it != e && *it == col) ? (uint32_t)(it - p.ja.begin()) : 0xffffffffu;
  };
  p.tblk.assign(p.nnz, 0);
  parallel_ranges(N, [&](size_t r0, size_t r1) {
    for (size_t i = r0; i < r1; i++)
      for (uint32_t j = p.ia[i]; j < p.ia[i + 1]; j++) p.tblk[j] = find(p.ja[j], (uint32_t)i);
  });
  p.last_lower.assign(N, 0xffffffffu);
  for (size_t e = 0; e < E; e++) {
    const uint32_t a = n0[e], b = n1[e];
    if (b < a) p.last_lower[a] = b;
    if (a < b) p.last_lower[b] = a;
  }
  for (size_t i = 0; i < N; i++)
    if (p.last_lower[i] != 0xffffffffu) p.last_lower[i] = find((uint32_t)i, p.last_lower[i]);
  // level sets: depth(i) = 1 + max depth over the lower (resp. upper) columns
  std::vector<uint32_t> depth(N);
  auto levels = [&](bool lower, std::vector<uint32_t> &rows, std::vector<uint32_t> &ptr) {
    uint32_t nlev = 1;
    for (size_t s = 0; s < N; s++) {
      const size_t i = lower ? s : N - 1 - s;
      uint32_t d = 1;
      const uint32_t jb = lower ? p.ia[i] : p.diag[i] + 1, je = lower ? p.diag[i] : p.ia[i + 1];
      for (uint32_t j = jb; j < je; j++) d = std::max(d, depth[p.ja[j]] + 1);
      depth[i] = d;
      nlev = std::max(nlev, d);
    }
    ptr.assign(nlev + 1, 0);
    for (size_t i = 0; i < N; i++) ptr[depth[i]]++;
    for (uint32_t l = 0; l < nlev; l++) ptr[l + 1] += ptr[l];
    rows.assign(N, 0);
    std::vector<uint32_t> top(ptr.begin(), ptr.end() - 1);
    for (size_t i = 0; i < N; i++) rows[top[depth[i] - 1]++] = (uint32_t)i;
  };
  levels(true, p.lev_l, p.lev_l_ptr);
  levels(false, p.lev_u, p.lev_u_ptr);
  // ILU(0) product lists: for block (i,k) merge row i's columns up to the
  // diagonal with row k's columns up to the diagonal (= U's column k)
  // (two passes over the rows in parallel: count, then fill in place)
  p.pair_ptr.assign(p.nnz + 1, 0);
  auto merge = [&](size_t i, uint32_t j, auto emit) {
    const uint32_t k = p.ja[j];
    uint32_t pl = p.ia[i], pu = p.ia[k];
    while (pl <= p.diag[i] && pu <= p.diag[k]) {
      const uint32_t cl = p.ja[pl], cu = p.ja[pu];
      if (cl == cu) emit(cl == i ? 0xffffffffu : p.lpos[i] + (pl - p.ia[i]), p.tblk[pu]);
      if (cl <= cu) pl++;
      if (cl >= cu) pu++;
    }
  };
  parallel_ranges(N, [&](size_t r0, size_t r1) {
    for (size_t i = r0; i < r1; i++)
      for (uint32_t j = p.ia[i]; j < p.ia[i + 1]; j++) {
        uint32_t c = 0;
        merge(i, j, [&](uint32_t, uint32_t) { c++; });
        p.pair_ptr[j + 1] = c;
      }
  });
  for (size_t j = 0; j < p.nnz; j++) p.pair_ptr[j + 1] += p.pair_ptr[j];
  p.pairs.resize(2 * (size_t)p.pair_ptr[p.nnz]);   // every element is written below
  parallel_ranges(N, [&](size_t r0, size_t r1) {
    for (size_t i = r0; i < r1; i++)
      for (uint32_t j = p.ia[i]; j < p.ia[i + 1]; j++) {
        size_t o = 2 * (size_t)p.pair_ptr[j];
        merge(i, j, [&](uint32_t a, uint32_t b) { p.pairs[o++] = a; p.pairs[o++] = b; });
      }
  });
}

// ----------------------------------------------------------------- matrix handle ABI

extern "C" void *CXX_Matrix_Init(const size_t nnodes, const size_t nedges, const unsigned int block_size,
                                 const unsigned int nthreads, const unsigned int *n0, const unsigned int *n1)
{
  (void)nthreads;
  if (block_size != 4) {
    kf_set_error(KFUN3D_ERR_ARG, "block size must be 4");
    return nullptr;
  }
  MatrixHandle *h = new MatrixHandle();
  h->e0.assign(n0, n0 + nedges);
  h->e1.assign(n1, n1 + nedges);
  h->pat.n = nnodes;   // the pattern itself: on the device with the mirror, or kf_host_pattern
  return h;
}

const HostPattern &kf_host_pattern(MatrixHandle *h)
{
  if (h->pat.ia.empty()) kf_build_pattern(h->pat, h->pat.n, h->e0.size(), h->e0.data(), h->e1.data());
  return h->pat;
}

static void release_device(MatrixHandle *h);

extern "C" void CXX_Matrix_Delete(void *ptr)
{
  MatrixHandle *h = (MatrixHandle *)ptr;
  if (!h || h->magic != 0x4B463344u) return;
  release_device(h);
  h->magic = 0;
  delete h;
}

extern "C" void CXX_METIS(const unsigned int nparts, unsigned int *parts, void *ptr)
{
  MatrixHandle *h = (MatrixHandle *)ptr;
  if (!h || nparts == 0) return;
  const size_t N = h->pat.n;
  for (size_t i = 0; i < N; i++) parts[i] = (unsigned int)((i * nparts) / (N ? N : 1));
}

MatrixHandle *kf_handle(const GEOMETRY *g)
{
  if (!g || !g->matrix) return nullptr;
  MatrixHandle *h = (MatrixHandle *)g->matrix;
  return h->magic == 0x4B463344u ? h : nullptr;
}

// ----------------------------------------------------------------- device mirror

#define KF_CUDA(call)                                                             \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      std::string m_ = std::string(#call) + ": " + cudaGetErrorString(e_);       \
      kf_set_error(KFUN3D_ERR_CUDA, m_.c_str());                                  \
      release_device(h);                                                          \
      return nullptr;                                                             \
    }                                                                             \
  } while (0)

// A copy from pageable host memory may return before its last DMA has
// landed; the wait makes the data safe for kernels on the mirror's own
// (non-blocking) stream.
template <class T> static cudaError_t upload(T **dst, const T *src, size_t n)
{
  cudaError_t e = cudaMalloc((void **)dst, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess || n == 0) return e;
  e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
}

void kf_ilu_release(DevMesh &m);

// ----------------------------------------------------------------- packed level schedule

void kf_free_packed(PackedSweep pk[2])
{
  for (int s = 0; s < 2; s++) {
    void *ptrs[] = {pk[s].row, pk[s].first, pk[s].col, pk[s].src, pk[s].chunk[0], pk[s].chunk[1]};
    for (void *q : ptrs)
      if (q) cudaFree(q);
    pk[s] = PackedSweep{};
  }
}

// Stream order = slot order of the level-ordered descriptors: slot s of the
// lower sweep contributes its lower blocks [d.y, d.z) (matrix/sptrsv.cpp:173-189
// reads them in this column order); slot s of the upper sweep its inverted
// diagonal block and then its upper blocks [d.y, d.z) (matrix/sptrsv.cpp:191-209).
// Each level's slots are cut into chunks, one CTA each, twice: at most 32 rows
// and 256 blocks, and at most 64 rows and 512 blocks.  KFUN3D_ERR_ARG (and
// nothing allocated) when a row has more than KF_PK_ROW_MAX blocks.
// (f(i) for every i in [0, n), interleaved over the host's threads: for
// items of uneven size, such as levels)
template <class F> static void parallel_items(size_t n, size_t work, F f)
{
  const unsigned T = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (work < 65536 || T == 1 || n < 2) {
    for (size_t i = 0; i < n; i++) f(i);
    return;
  }
  std::vector<std::thread> th;
  for (unsigned t = 0; t < T; t++)
    th.emplace_back([&, t] {
      for (size_t i = t; i < n; i += T) f(i);
    });
  for (auto &x : th) x.join();
}

void kf_level_descriptors(const HostPattern &p, std::vector<uint4> &dl, std::vector<uint4> &du)
{
  const size_t N = p.n;
  dl.resize(N);
  du.resize(N);
  parallel_ranges(N, [&](size_t a, size_t b) {
    for (size_t q = a; q < b; q++) {
      const uint32_t i = p.lev_l[q];
      dl[q] = make_uint4(i, p.ia[i], p.diag[i], 0);
      const uint32_t k = p.lev_u[q];
      du[q] = make_uint4(k, p.diag[k] + 1, p.ia[k + 1], 0);
    }
  });
  auto by_length = [N](std::vector<uint4> &d, const std::vector<uint32_t> &ptr) {
    parallel_items(ptr.size() - 1, N, [&](size_t l) {
      std::stable_sort(d.begin() + ptr[l], d.begin() + ptr[l + 1],
                       [](const uint4 &a, const uint4 &b) { return a.z - a.y > b.z - b.y; });
    });
  };
  by_length(dl, p.lev_l_ptr);
  by_length(du, p.lev_u_ptr);
}

int kf_build_packed(PackedSweep pk[2], const HostPattern &p, const std::vector<uint4> &desc_l,
                    const std::vector<uint4> &desc_u, const uint4 *ddesc_l, const uint4 *ddesc_u,
                    const uint32_t *ja, const uint32_t *diag, cudaStream_t st)
{
  const size_t N = p.n;
  for (int sw = 0; sw < 2; sw++) {
    const std::vector<uint4> &d = sw == 0 ? desc_l : desc_u;
    const std::vector<uint32_t> &lp = sw == 0 ? p.lev_l_ptr : p.lev_u_ptr;
    std::vector<uint32_t> first(N + 1);
    size_t nblk = 0;
    for (size_t s = 0; s < N; s++) {
      const size_t len = (d[s].z - d[s].y) + (sw == 1 ? 1u : 0u);
      if (len > KF_PK_ROW_MAX) { kf_free_packed(pk); return KFUN3D_ERR_ARG; }
      first[s] = (uint32_t)std::min<size_t>(nblk, 0xffffffffu);
      nblk += len;
    }
    if (nblk >= 0xffffffffu) { kf_free_packed(pk); return KFUN3D_ERR_ARG; }
    first[N] = (uint32_t)nblk;
    PackedSweep &o = pk[sw];
    o.nblk = (uint32_t)nblk;
    // the streams (slot rows, block columns, source blocks) written on the device
    bool ok = upload(&o.first, first.data(), N + 1) == cudaSuccess &&
              cudaMalloc(&o.row, std::max<size_t>(N, 1) * sizeof(uint32_t)) == cudaSuccess &&
              cudaMalloc(&o.col, std::max<size_t>(nblk, 1) * sizeof(uint32_t)) == cudaSuccess &&
              cudaMalloc(&o.src, std::max<size_t>(nblk, 1) * sizeof(uint32_t)) == cudaSuccess;
    ok = ok && kf_packed_streams_device((uint32_t)N, sw == 1, sw == 0 ? ddesc_l : ddesc_u, o.first, ja, diag, o.row,
                                        o.col, o.src, st) == KFUN3D_OK;
    for (int cut = 0; cut < 2 && ok; cut++) {
      const uint32_t rows = cut == 0 ? 32u : 64u, budget = 8u * rows;
      std::vector<uint4> chunk;
      std::vector<uint32_t> lev(1, 0);
      uint32_t maxblk = 0;
      for (size_t l = 0; l + 1 < lp.size(); l++) {
        uint32_t s = lp[l];
        while (s < lp[l + 1]) {
          uint32_t e = s + 1;   // a chunk holds at least one row, however long
          while (e < lp[l + 1] && e - s < rows && first[e + 1] - first[s] <= budget) e++;
          chunk.push_back(make_uint4(s, e, first[s], first[e]));
          maxblk = std::max(maxblk, first[e] - first[s]);
          s = e;
        }
        lev.push_back((uint32_t)chunk.size());
      }
      o.lev[cut] = lev;
      o.maxblk[cut] = maxblk;
      ok = upload(&o.chunk[cut], chunk.data(), chunk.size()) == cudaSuccess;
    }
    if (ok) ok = cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      kf_free_packed(pk);
      return KFUN3D_ERR_CUDA;
    }
  }
  return KFUN3D_OK;
}

static void release_device(MatrixHandle *h)
{
  DevMesh *m = h->dev;
  if (!m) return;
  kf_ilu_release(*m);   // the spatial ILU set's arrays; the reference set's fields are back in place
  kf_free_packed(m->iset[0].pk);
  if (m->pk_buf) cudaFree(m->pk_buf);
  void *ptrs[] = {m->col, m->egeo, m->xyz, m->inc_ptr, m->inc_oth, m->inc_edge, m->inc_blk, m->inc_w, m->wf_nodes,
                  m->wf_n, m->s_n, m->f_n, m->bnd_of, m->bnd_node, m->bnd_ptr, m->bnd_ent, m->ia, m->ja,
                  m->diag, m->tblk, m->lpos, m->last_lower, m->lev_l, m->lev_u, m->A, m->lslot, m->dinv,
                  m->Af, m->dinvf, m->q, m->r, m->gx, m->gy, m->gz, m->cdt, m->w, m->t, m->x, m->rhs, m->V,
                  m->red, m->scal, m->forces, m->dscr, m->status, m->flags, m->ticket, m->part, m->lsq_coef,
                  m->qv, m->xyzv, m->gxv, m->gyv, m->gzv, m->inc_othv, m->n0v, m->n1v, m->inc_geo, m->desc_l, m->desc_u, m->eoff, m->n1, m->in1_ptr, m->in1_edge, m->eres, m->n0s, m->pair_ptr, m->pairs, m->lev_ptr_d, m->bar, m->Z, m->qold, m->fy, m->fx, m->pscr, m->ord, m->rowof, m->egeo_s, m->sub_part};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (m->h_scal) cudaFreeHost(m->h_scal);
  if (m->mgraph) kfun3d_mpnn_graph_free(m->mgraph);
  for (auto &a : m->arnoldi)
    for (auto &b : a)
      for (auto &g : b)
        if (g) cudaGraphExecDestroy(g);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  h->dev = nullptr;
}

// The mirror's edge geometry, incidence lists, two-pass edge storage and
// visit-order copies rebuilt on the host threads from the GEOMETRY (in the
// visit order the mirror uses) and compared with the device-built arrays,
// element for element and bit for bit: 1 equal, 0 different, -1 CUDA error.
static int lists_match_host(const DevMesh &m, const GEOMETRY *g, const HostPattern &p)
{
  const uint32_t N = m.N, E = m.E;
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
  bool ok = true, same = true;
  auto down = [&](auto &vec, const void *src) {
    if (ok && !vec.empty() && cudaMemcpy(vec.data(), src, vec.size() * sizeof(vec[0]), cudaMemcpyDeviceToHost) != cudaSuccess)
      ok = false;
  };
  auto cmp = [&](const auto &host, const void *dev) {
    if (!ok || !same) return;
    auto d = host;
    down(d, dev);
    same = ok && memcmp(d.data(), host.data(), host.size() * sizeof(host[0])) == 0;
  };
  std::vector<uint32_t> ord(N), rowof(N);
  down(ord, m.ord);
  for (uint32_t q = 0; q < N; q++) rowof[ord[q]] = q;
  std::vector<double4> eg(E);
  for (uint32_t e = 0; e < E; e++)
    eg[e] = make_double4(g->e->xyzn->x0[e], g->e->xyzn->x1[e], g->e->xyzn->x2[e], g->e->xyzn->x3[e]);
  cmp(eg, m.egeo);
  cmp(rowof, m.rowof);
  // incidence: per visit position, the node's edges in edge order
  std::vector<uint32_t> deg(N, 0), ptr(N + 1, 0);
  for (uint32_t e = 0; e < E; e++) { deg[n0[e]]++; deg[n1[e]]++; }
  for (uint32_t q = 0; q < N; q++) ptr[q + 1] = ptr[q] + deg[ord[q]];
  const size_t ninc = 2 * (size_t)E, wst = m.wstride;
  std::vector<uint32_t> oth(wst + 4, 0), edg(ninc), blk(ninc), pos(N);
  std::vector<double> w(3 * wst + 4, 0.0);
  for (uint32_t i = 0; i < N; i++) pos[i] = ptr[rowof[i]];
  const double *w0[3] = {g->e->w->w0->x0, g->e->w->w0->x1, g->e->w->w0->x2};
  const double *w1[3] = {g->e->w->w1->x0, g->e->w->w1->x1, g->e->w->w1->x2};
  for (uint32_t e = 0; e < E; e++) {
    const uint32_t a = n0[e], b = n1[e];
    uint32_t k = pos[a]++;
    oth[k] = b; edg[k] = e;
    for (int c = 0; c < 3; c++) w[c * wst + k] = w0[c][e];
    k = pos[b]++;
    oth[k] = a; edg[k] = e | 0x80000000u;
    for (int c = 0; c < 3; c++) w[c * wst + k] = w1[c][e];
  }
  parallel_ranges(N, [&](size_t r0, size_t r1) {
    for (size_t row = r0; row < r1; row++)
      for (uint32_t k = ptr[row]; k < ptr[row + 1]; k++) {
        auto b = p.ja.begin() + p.ia[ord[row]], en = p.ja.begin() + p.ia[ord[row] + 1];
        blk[k] = (uint32_t)(std::lower_bound(b, en, oth[k]) - p.ja.begin());
      }
  });
  cmp(ptr, m.inc_ptr);
  cmp(oth, m.inc_oth);
  cmp(edg, m.inc_edge);
  cmp(blk, m.inc_blk);
  cmp(w, m.inc_w);
  if (m.two_pass) {
    // storage: groups by n0 in visit order, each in edge order
    std::vector<uint32_t> r0(N + 1, 0), c1(N, 0);
    for (uint32_t e = 0; e < E; e++) { r0[n0[e] + 1]++; c1[n1[e]]++; }
    for (uint32_t i = 0; i < N; i++) r0[i + 1] += r0[i];
    std::vector<uint32_t> eoff(N + 1, 0), spos(E), n0s(E), n1s(E), iptr(N + 1, 0), iedge(E);
    std::vector<double4> egs(E);
    uint32_t next = 0;
    for (uint32_t q = 0; q < N; q++) {
      const uint32_t nd = ord[q];
      eoff[q] = next;
      for (uint32_t e = r0[nd]; e < r0[nd + 1]; e++) {
        spos[e] = next;
        n0s[next] = nd;
        n1s[next] = n1[e];
        egs[next] = eg[e];
        next++;
      }
      iptr[q + 1] = iptr[q] + c1[nd];
    }
    eoff[N] = next;
    std::vector<uint32_t> ipos(N);
    for (uint32_t q = 0; q < N; q++) ipos[ord[q]] = iptr[q];
    for (uint32_t e = 0; e < E; e++) iedge[ipos[n1[e]]++] = spos[e];
    cmp(eoff, m.eoff);
    cmp(n0s, m.n0s);
    cmp(n1s, m.n1);
    cmp(egs, m.egeo_s);
    cmp(iptr, m.in1_ptr);
    cmp(iedge, m.in1_edge);
    if (m.visit) {
      std::vector<uint32_t> othv(ninc), e0v(E), e1v(E);
      std::vector<double4> xv(N), ig(ninc);
      for (uint32_t q = 0; q < N; q++) {
        const uint32_t nd = ord[q];
        xv[q] = make_double4(g->n->xyz->x0[nd], g->n->xyz->x1[nd], g->n->xyz->x2[nd], 0.0);
      }
      for (size_t k = 0; k < ninc; k++) {
        othv[k] = rowof[oth[k]];
        ig[k] = eg[edg[k] & 0x7fffffffu];
      }
      for (uint32_t e = 0; e < E; e++) { e0v[e] = rowof[n0s[e]]; e1v[e] = rowof[n1s[e]]; }
      cmp(othv, m.inc_othv);
      cmp(ig, m.inc_geo);
      cmp(e0v, m.n0v);
      cmp(e1v, m.n1v);
      cmp(xv, m.xyzv);
    }
  }
  if (!ok) {
    cudaGetLastError();
    kf_set_error(KFUN3D_ERR_CUDA, "mesh list check: a copy from the device failed");
    return -1;
  }
  return same ? 1 : 0;
}

extern "C" long kfun3d_device_query(const GEOMETRY *g, const char *key)
{
  DevMesh *m = key ? kf_device(g) : nullptr;
  if (!m) return -1;
  if (strcmp(key, "sptrsv_schedule") == 0) return m->trsv_mode;
  if (strcmp(key, "lsq_terms_match") == 0) return m->lsq_match ? 1 : 0;
  if (strcmp(key, "visit_order_copies") == 0) return m->visit ? 1 : 0;
  if (strcmp(key, "mgs_resident") == 0) return m->mgs_resident ? 1 : 0;
  if (strcmp(key, "setup_us") == 0) return m->setup_us;
  if (strcmp(key, "pattern_us") == 0) return m->pattern_us;
  if (strcmp(key, "spatial_setup_us") == 0) return m->spatial_us;
  if (strcmp(key, "host_pattern_us") == 0) return m->host_pattern_us;
  if (strcmp(key, "lists_match_host") == 0) return lists_match_host(*m, g, kf_host_pattern(kf_handle(g)));
  if (strcmp(key, "pattern_matches_host") == 0) {
    const MatrixHandle *h = kf_handle(g);
    return kf_pattern_matches(m->iset[0], m->N, m->E, h->e0.data(), h->e1.data(), m->stream, &m->host_pattern_us);
  }
  if (strcmp(key, "spatial_pattern_matches_host") == 0) {
    if (!m->iset[1].valid) return -1;
    std::vector<uint32_t> rank(m->N);
    if (cudaMemcpy(rank.data(), m->ilu_rank, m->N * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    const MatrixHandle *h = kf_handle(g);
    std::vector<uint32_t> pn0(m->E), pn1(m->E);
    for (size_t e = 0; e < m->E; e++) { pn0[e] = rank[h->e0[e]]; pn1[e] = rank[h->e1[e]]; }
    return kf_pattern_matches(m->iset[1], m->N, m->E, pn0.data(), pn1.data(), m->stream, nullptr);
  }
  return -1;
}

extern "C" void kfun3d_device_release(GEOMETRY *g)
{
  MatrixHandle *h = kf_handle(g);
  if (h) release_device(h);
}

DevMesh *kf_device(const GEOMETRY *g)
{
  MatrixHandle *h = kf_handle(g);
  if (!h) {
    kf_set_error(KFUN3D_ERR_ARG, "GEOMETRY::matrix is not a kfun3d_b200 handle (create it with CXX_Matrix_Init)");
    return nullptr;
  }
  if (h->dev) return h->dev;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    kf_set_error(KFUN3D_ERR_NO_DEVICE, "no CUDA device");
    return nullptr;
  }
  if (g->s && g->s->sz > 1) {
    kf_set_error(KFUN3D_ERR_ARG, "GEOMETRY built for more than one OpenMP thread: set it up with one thread");
    if (g_abort) {
      fprintf(stderr, "kfun3d_b200: GEOMETRY built for more than one OpenMP thread: set it up with one thread\n");
      abort();
    }
    return nullptr;
  }
  const auto t_start = std::chrono::steady_clock::now();
  auto us_since = [](std::chrono::steady_clock::time_point t) {
    return (long)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t).count();
  };
  const uint32_t N = (uint32_t)g->n->sz, E = (uint32_t)g->e->sz;
  if (h->pat.n != N || h->e0.size() != E) {
    kf_set_error(KFUN3D_ERR_ARG, "matrix handle does not match the GEOMETRY");
    return nullptr;
  }
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;

  SetupTrace tr("device mirror");
  DevMesh *m = new DevMesh();
  h->dev = m;
  h->owner = g;
  KF_CUDA(cudaGetDevice(&m->device));
  KF_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  tr.mark("CUDA context and stream");
  // the block pattern, persistent L slots and ILU(0) product lists, built on
  // the device; the host keeps the arrays its set-up code below reads
  {
    DevPattern dp;
    const auto t_pat = std::chrono::steady_clock::now();
    if (kf_build_pattern_device(h->pat, dp, N, E, h->e0.data(), h->e1.data(), m->stream) != KFUN3D_OK) {
      release_device(h);
      return nullptr;
    }
    m->ia = dp.ia; m->ja = dp.ja; m->diag = dp.diag; m->tblk = dp.tblk; m->lpos = dp.lpos;
    m->last_lower = dp.last_lower; m->pair_ptr = dp.pair_ptr; m->pairs = dp.pairs;
    m->pattern_us = us_since(t_pat);
  }
  tr.mark("block pattern on the device");
  const HostPattern &p = h->pat;
  m->N = N;
  m->E = E;
  m->Ns = (uint32_t)g->b->s->sz;
  m->Nf = (uint32_t)g->b->f->sz;
  m->F = (uint32_t)g->b->fc->sz;
  m->ncol = (uint32_t)g->t->sz;
  m->nnz = (uint32_t)p.nnz;
  m->nlower = p.lpos[N];

  // node coordinates
  {
    std::vector<double4> xyz(N);
    for (uint32_t i = 0; i < N; i++)
      xyz[i] = make_double4(g->n->xyz->x0[i], g->n->xyz->x1[i], g->n->xyz->x2[i], 0.0);
    KF_CUDA(upload(&m->xyz, xyz.data(), N));
  }
  // Order in which the node-centric kernels visit nodes: on meshes whose node
  // data (state, gradients, coordinates: 160 B a node) outgrows what L2 keeps
  // (from 500,000 nodes), Morton (Z-order) of the coordinates, so that a
  // warp's nodes and their neighbours are close in space and the gathers hit
  // in L2 even when the mesh's own numbering is random; below, the mesh's own
  // order.  A node's sums still run over its edges in edge order, so results
  // do not depend on this order.  KFUN3D_NODE_ORDER=natural|morton overrides.
  std::vector<uint32_t> ord(N);
  for (uint32_t i = 0; i < N; i++) ord[i] = i;
  {
    const char *env = getenv("KFUN3D_NODE_ORDER");
    bool morton = N >= 500000u;
    if (env && strcmp(env, "natural") == 0) morton = false;
    if (env && strcmp(env, "morton") == 0) morton = true;
    m->spatial_order = morton;
    if (morton && N > 0) {
      const double *X = g->n->xyz->x0, *Y = g->n->xyz->x1, *Z = g->n->xyz->x2;
      double lo[3] = {X[0], Y[0], Z[0]}, hi[3] = {X[0], Y[0], Z[0]};
      for (uint32_t i = 0; i < N; i++) {
        const double c[3] = {X[i], Y[i], Z[i]};
        for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], c[d]); hi[d] = std::max(hi[d], c[d]); }
      }
      auto spread = [](uint64_t v) {   // 21 bits -> every third bit
        v &= 0x1fffffull;
        v = (v | v << 32) & 0x1f00000000ffffull;
        v = (v | v << 16) & 0x1f0000ff0000ffull;
        v = (v | v << 8) & 0x100f00f00f00f00full;
        v = (v | v << 4) & 0x10c30c30c30c30c3ull;
        v = (v | v << 2) & 0x1249249249249249ull;
        return v;
      };
      std::vector<uint64_t> key(N);
      for (uint32_t i = 0; i < N; i++) {
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
    }
    KF_CUDA(upload(&m->ord, ord.data(), N));
    std::vector<uint32_t> rowof(N);
    for (uint32_t q = 0; q < N; q++) rowof[ord[q]] = q;
    KF_CUDA(upload(&m->rowof, rowof.data(), N));
  }
  tr.mark("visit order");
  // two-pass residual structure when the edges are sorted by n0 with n0 < n1
  // everywhere; visit-order copies of the node data when the visit order is
  // not the mesh's own (KFUN3D_VISIT_COPIES=0: not)
  {
    bool ok = true;
    for (uint32_t e = 0; e < E && ok; e++) {
      if (n0[e] >= n1[e]) ok = false;
      if (e && n0[e] < n0[e - 1]) ok = false;
    }
    const char *env = getenv("KFUN3D_RESIDUAL");
    m->two_pass = ok && !(env && strcmp(env, "gather") == 0);
    const char *venv = getenv("KFUN3D_VISIT_COPIES");
    m->visit = m->two_pass && m->spatial_order && !(venv && strcmp(venv, "0") == 0);
  }
  // edge geometry, node incidence in edge order (with the least-squares
  // terms seen from the node and the block of (node, other)), the two-pass
  // residual's edge storage and the visit-order copies, built on the device
  if (kf_build_mesh_lists_device(*m, g) != KFUN3D_OK) {
    release_device(h);
    return nullptr;
  }
  tr.mark("incidence lists, residual structure, visit-order copies");
  {
    std::vector<uint32_t> ptr(N + 1);
    KF_CUDA(cudaMemcpy(ptr.data(), m->inc_ptr, ((size_t)N + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    // shared memory of the staged gradient: the widest 128-node block range
    size_t maxcnt = 0;
    for (uint32_t nb = 0; nb < N; nb += 128) {
      const uint32_t ne = std::min<uint32_t>(nb + 128, N);
      const size_t ka = ptr[nb] & ~3u, kb = (ptr[ne] + 3u) & ~3u;
      maxcnt = std::max(maxcnt, kb - ka);
    }
    const size_t smem = 4 * ((maxcnt + 3) & ~(size_t)3) + 24 * maxcnt;
    const char *genv = getenv("KFUN3D_GRADIENT");
    // staged (TMA) gradient in the mesh's own order; in the spatial order
    // consecutive rows are already read in sequence and the plain gather is
    // the faster one.  KFUN3D_GRADIENT=plain|tma overrides.
    bool tma = smem <= 200 * 1024 && !m->spatial_order;
    if (genv && strcmp(genv, "plain") == 0) tma = false;
    if (genv && strcmp(genv, "tma") == 0) tma = smem <= 200 * 1024;
    m->grad_smem = tma ? (unsigned)smem : 0;
  }
  // wall faces (colour order) with normals -(1/6) a x b (src/flux.c:485-508)
  {
    const unsigned int *f0 = g->b->fc->fptr->n0, *f1 = g->b->fc->fptr->n1, *f2 = g->b->fc->fptr->n2;
    const double *X = g->n->xyz->x0, *Y = g->n->xyz->x1, *Z = g->n->xyz->x2;
    const double MAG0 = 0.5 / 3, MAG1 = -MAG0;
    std::vector<uint32_t> fn(3 * (size_t)m->F);
    std::vector<double> nn(3 * (size_t)m->F);
    for (uint32_t j = 0; j < m->F; j++) {
      const uint32_t a = f0[j], b = f1[j], d = f2[j];
      fn[3 * j] = a; fn[3 * j + 1] = b; fn[3 * j + 2] = d;
      const double ax = X[b] - X[a], ay = Y[b] - Y[a], az = Z[b] - Z[a];
      const double bx = X[d] - X[a], by = Y[d] - Y[a], bz = Z[d] - Z[a];
      double xn = ay * bz; xn -= az * by; xn *= MAG1;
      double yn = ax * bz; yn -= az * bx; yn *= MAG0;
      double zn = ax * by; zn -= ay * bx; zn *= MAG1;
      nn[3 * j] = xn; nn[3 * j + 1] = yn; nn[3 * j + 2] = zn;
    }
    KF_CUDA(upload(&m->wf_nodes, fn.data(), fn.size()));
    KF_CUDA(upload(&m->col, g->t->i, (size_t)m->ncol + 1));
    KF_CUDA(upload(&m->wf_n, nn.data(), nn.size()));
    std::vector<double> sn(3 * (size_t)m->Ns), fnn(3 * (size_t)m->Nf);
    for (uint32_t i = 0; i < m->Ns; i++) {
      sn[3 * i] = g->b->s->xyz->x0[i]; sn[3 * i + 1] = g->b->s->xyz->x1[i]; sn[3 * i + 2] = g->b->s->xyz->x2[i];
    }
    for (uint32_t i = 0; i < m->Nf; i++) {
      fnn[3 * i] = g->b->f->xyz->x0[i]; fnn[3 * i + 1] = g->b->f->xyz->x1[i]; fnn[3 * i + 2] = g->b->f->xyz->x2[i];
    }
    KF_CUDA(upload(&m->s_n, sn.data(), sn.size()));
    KF_CUDA(upload(&m->f_n, fnn.data(), fnn.size()));
    // per boundary node: wall-face corners (face order = colour order), then
    // wall-node entries, then far-field entries, each in list order
    std::vector<std::vector<uint32_t>> ent(N);
    for (uint32_t j = 0; j < m->F; j++) {
      ent[f0[j]].push_back(0u << 29 | (3 * j + 0));
      ent[f1[j]].push_back(0u << 29 | (3 * j + 1));
      ent[f2[j]].push_back(0u << 29 | (3 * j + 2));
    }
    for (uint32_t i = 0; i < m->Ns; i++) ent[g->b->s->nptr[i]].push_back(1u << 29 | i);
    for (uint32_t i = 0; i < m->Nf; i++) ent[g->b->f->nptr[i]].push_back(2u << 29 | i);
    std::vector<uint32_t> of(N, 0xffffffffu), nodes, bptr(1, 0), bent;
    for (uint32_t i = 0; i < N; i++) {
      if (ent[i].empty()) continue;
      of[i] = (uint32_t)nodes.size();
      nodes.push_back(i);
      bent.insert(bent.end(), ent[i].begin(), ent[i].end());
      bptr.push_back((uint32_t)bent.size());
    }
    m->nb = (uint32_t)nodes.size();
    KF_CUDA(upload(&m->bnd_of, of.data(), N));
    KF_CUDA(upload(&m->bnd_node, nodes.data(), nodes.size()));
    KF_CUDA(upload(&m->bnd_ptr, bptr.data(), bptr.size()));
    KF_CUDA(upload(&m->bnd_ent, bent.data(), bent.size()));
  }
  tr.mark("boundary lists");
  // level sets (the block pattern, persistent L slots and ILU(0) product
  // lists were built on the device above)
  const std::vector<uint32_t> &lev_l = p.lev_l, &lev_u = p.lev_u;
  KF_CUDA(upload(&m->lev_l, lev_l.data(), lev_l.size()));
  KF_CUDA(upload(&m->lev_u, lev_u.data(), lev_u.size()));
  m->lev_l_ptr = p.lev_l_ptr;
  m->lev_u_ptr = p.lev_u_ptr;
  m->nlev_l = (uint32_t)p.lev_l_ptr.size() - 1;
  m->nlev_u = (uint32_t)p.lev_u_ptr.size() - 1;
  const size_t nb16 = 16 * (size_t)m->nnz;
  KF_CUDA(cudaMalloc(&m->A, nb16 * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->Af, nb16 * sizeof(float)));
  KF_CUDA(cudaMalloc(&m->lslot, (16 * (size_t)m->nlower + 16) * sizeof(double)));
  KF_CUDA(cudaMemset(m->lslot, 0, (16 * (size_t)m->nlower + 16) * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->dinv, 16 * (size_t)N * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->dinvf, 16 * (size_t)N * sizeof(float)));
  KF_CUDA(cudaMalloc(&m->dscr, (16 * (size_t)m->nb + 16) * sizeof(double)));
  // vectors
  const size_t dofs = 4 * (size_t)N;
  double **vecs[] = {&m->q, &m->r, &m->gx, &m->gy, &m->gz, &m->w, &m->t, &m->x, &m->rhs};
  for (double **v : vecs) {
    KF_CUDA(cudaMalloc(v, dofs * sizeof(double)));
    KF_CUDA(cudaMemset(*v, 0, dofs * sizeof(double)));
  }
  KF_CUDA(cudaMalloc(&m->cdt, (size_t)N * sizeof(double)));
  KF_CUDA(cudaMemset(m->cdt, 0, (size_t)N * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->V, KF_NBASIS * dofs * sizeof(double)));
  KF_CUDA(cudaMemset(m->V, 0, KF_NBASIS * dofs * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->red, 4096 * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->scal, 256 * sizeof(double)));
  KF_CUDA(cudaMemset(m->scal, 0, 256 * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->forces, 4 * sizeof(double)));
  KF_CUDA(cudaMalloc(&m->status, 4 * sizeof(int)));
  KF_CUDA(cudaMemset(m->status, 0, 4 * sizeof(int)));
  KF_CUDA(cudaMalloc(&m->flags, (size_t)N * sizeof(uint32_t)));
  KF_CUDA(cudaMemset(m->flags, 0, (size_t)N * sizeof(uint32_t)));
  KF_CUDA(cudaMalloc(&m->ticket, sizeof(unsigned long long)));
  KF_CUDA(cudaMemset(m->ticket, 0, sizeof(unsigned long long)));
  {
    int nsm = 0;
    KF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device));
    // cooperative grid: 4 blocks of 256 threads per SM (the kernel's launch
    // bounds guarantee they fit); the runtime refuses the launch otherwise
    m->trsv_grid = (unsigned)nsm * 4;
    // mode 5: 1-3 CTAs of 512 threads per SM (the kernel's launch bounds
    // guarantee they fit); KFUN3D_SPTRSV_CTAS picks the count
    const char *cenv = getenv("KFUN3D_SPTRSV_CTAS");
    if (cenv && (atoi(cenv) >= 1 && atoi(cenv) <= 3)) m->trsv_mgrid_per = atoi(cenv);
    m->trsv_mgrid = (unsigned)nsm * (unsigned)m->trsv_mgrid_per;
    const char *lenv = getenv("KFUN3D_SPTRSV_LANES");   // lanes per row: 8 (default), 4 or 16
    if (lenv && (atoi(lenv) == 4 || atoi(lenv) == 8 || atoi(lenv) == 16)) m->trsv_lanes = atoi(lenv);
    std::vector<uint4> dl, du;
    kf_level_descriptors(p, dl, du);
    KF_CUDA(upload(&m->desc_l, dl.data(), N));
    KF_CUDA(upload(&m->desc_u, du.data(), N));
    // the packed factor (room for FP64 blocks, shared by both ILU orders) and
    // this pattern's packed level schedule
    KF_CUDA(cudaMalloc(&m->pk_buf, 16 * (size_t)m->nnz * sizeof(double)));
    // ERR_ARG: rows too long, no packed schedule
    const int pkrc = kf_build_packed(m->iset[0].pk, p, dl, du, m->desc_l, m->desc_u, m->ja, m->diag, m->stream);
    if (pkrc == KFUN3D_ERR_CUDA) {
      kf_set_error(KFUN3D_ERR_CUDA, "device mirror: building the packed triangular-solve schedule failed");
      return nullptr;
    }
    // chunk cut per factor precision (KFUN3D_PK_ROWS="<fp64 rows>,<fp32 rows>", 32 or 64 each)
    const char *fenv = getenv("KFUN3D_PK_FP64");
    m->pk_fp64 = fenv && strcmp(fenv, "1") == 0;
    const char *renv = getenv("KFUN3D_PK_ROWS");
    if (renv) {
      int r64 = 0, r32 = 0;
      if (sscanf(renv, "%d,%d", &r64, &r32) == 2) {
        m->pk_cut[0] = r64 == 32 ? 0 : 1;
        m->pk_cut[1] = r32 == 32 ? 0 : 1;
      }
    }
    // triangular-solve schedule (KFUN3D_SPTRSV): "packed" (default: one
    // launch per level with programmatic dependent launch, each CTA's rows
    // one contiguous run of the packed factor staged into shared memory by a
    // bulk copy), "pdl4" (one launch per level with programmatic dependent
    // launch, 4 lanes per row, blocks read in the matrix's order), "pdl"
    // (the same with 16 lanes per row), "persistent" / "mono" (one
    // cooperative launch, bounded grid barrier between levels), "syncfree"
    // (per-row flags, no level barriers; the allocation-free entry point's
    // sweep) or "levels" (one plain launch per level, 4 lanes per row)
    const char *env = getenv("KFUN3D_SPTRSV");
    m->trsv_mode = m->iset[0].pk[0].chunk[0] ? 8 : 7;
    if (env && strcmp(env, "pdl") == 0) m->trsv_mode = 4;
    if (env && strcmp(env, "persistent") == 0) m->trsv_mode = 3;
    if (env && strcmp(env, "syncfree") == 0) m->trsv_mode = 1;
    if (env && strcmp(env, "levels") == 0) m->trsv_mode = 0;
    if (env && strcmp(env, "mono") == 0) m->trsv_mode = 5;
    if (env && strcmp(env, "pdl4") == 0) m->trsv_mode = 7;
    if (env && strcmp(env, "packed") == 0 && m->iset[0].pk[0].chunk[0]) m->trsv_mode = 8;
    std::vector<uint32_t> lp(p.lev_l_ptr);
    lp.insert(lp.end(), p.lev_u_ptr.begin(), p.lev_u_ptr.end());
    KF_CUDA(upload(&m->lev_ptr_d, lp.data(), lp.size()));
    KF_CUDA(cudaMalloc(&m->bar, 8 * sizeof(unsigned)));
    KF_CUDA(cudaMemset(m->bar, 0, 8 * sizeof(unsigned)));
    m->syncfree = m->trsv_mode == 1;
    const char *genv = getenv("KFUN3D_GRAPHS");
    m->use_graphs = !(genv && strcmp(genv, "0") == 0);
  }
  tr.mark("matrix, vectors, level descriptors, packed schedule");
  KF_CUDA(cudaMallocHost(&m->h_scal, 256 * sizeof(double)));
  {
    IluSet &s0 = m->iset[0];
    s0.ia = m->ia; s0.ja = m->ja; s0.diag = m->diag; s0.tblk = m->tblk; s0.lpos = m->lpos;
    s0.last_lower = m->last_lower; s0.pair_ptr = m->pair_ptr; s0.pairs = m->pairs;
    s0.lev_l = m->lev_l; s0.lev_u = m->lev_u; s0.lev_ptr_d = m->lev_ptr_d;
    s0.lev_l_ptr = m->lev_l_ptr; s0.lev_u_ptr = m->lev_u_ptr;
    s0.nlev_l = m->nlev_l; s0.nlev_u = m->nlev_u;
    s0.desc_l = m->desc_l; s0.desc_u = m->desc_u;
    s0.trsv_mode = m->trsv_mode;
    m->pk[0] = s0.pk[0];
    m->pk[1] = s0.pk[1];
    s0.fill_blk = m->inc_blk; s0.fill_diag = m->diag; s0.fill_last = m->last_lower; s0.fill_lpos = m->lpos;
    s0.valid = true;
    m->fill_blk = m->inc_blk; m->fill_diag = m->diag; m->fill_last = m->last_lower; m->fill_lpos = m->lpos;
  }
  // least-squares coefficients on the device; the gradient's terms on the fly
  // when they reproduce the GEOMETRY's stored ones bit for bit
  if (kf_exact::lsq_setup(*m) != KFUN3D_OK) {
    kf_set_error(KFUN3D_ERR_CUDA, "device mirror: least-squares coefficients failed");
    release_device(h);
    return nullptr;
  }
  KF_CUDA(cudaDeviceSynchronize());
  tr.mark("least-squares coefficients");
  m->setup_us = us_since(t_start);
  return m;
}
