// kfun3d_b200: the block pattern of the edge graph built on the device.
//
// The same arrays kf_build_pattern makes on the host threads (device_mesh.cu;
// matrix/init.cpp:7-74 for the pattern and 194-274 for the level sets, the
// reference's fill order src/fill.c:496-511 for the persistent-L-slot rule,
// matrix/ilu.cpp:71-84 for the ILU(0) products), bit for bit:
//   ia/ja   rows of the diagonal and one block per incident edge, columns
//           sorted (edges append to their rows through atomic slots, then
//           each row is sorted, so the order of the appends does not matter);
//   diag    each row's diagonal slot, lpos the first persistent L slot of each
//           row (exclusive sum of the lower lengths);
//   tblk    block (i,j) -> index of block (j,i);
//   last_lower  the lower block of each row that the reference's fill touches
//           last: the lower neighbour through the row's last incident edge in
//           edge order (the largest such edge index, by atomicMax);
//   levels  depth(i) = 1 + max depth over the lower (upper) columns, the
//           longest-path fixpoint, reached by repeated sweeps (any visiting
//           order reaches the same fixpoint); rows are then listed by level in
//           row order on the host (a counting sort of N depths);
//   pairs   for block (i,k) the merge of row i's columns up to its diagonal
//           with row k's up to its diagonal: (L slot or ~0, block of U(m,k)),
//           counted, summed and written in place.
// The host keeps the arrays its own set-up code reads (ia, ja, diag, lpos,
// last_lower, level lists); tblk, pair_ptr and pairs stay on the device.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.h"

namespace {

inline unsigned nblk(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// Host-to-device copies of large pageable arrays through pinned staging
// buffers: the host's threads fill one buffer while the copies of the
// previous ones run.  A copy the driver makes from pageable memory goes
// through one thread's memcpy into its own staging area, which bounds it to
// a few GB/s.  The buffers live as long as the object (one set-up).
struct Stager {
  static constexpr int K = 4;
  static constexpr size_t CHUNK = 4u << 20;
  void *buf[K] = {};
  cudaEvent_t ev[K] = {};
  bool used[K] = {};
  int next = 0;
  bool ok = false;
  Stager()
  {
    ok = true;
    for (int b = 0; b < K && ok; b++)
      ok = cudaMallocHost(&buf[b], CHUNK) == cudaSuccess && cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) cudaGetLastError();
  }
  ~Stager()
  {
    for (int b = 0; b < K; b++) {
      if (ev[b]) { cudaEventSynchronize(ev[b]); cudaEventDestroy(ev[b]); }
      if (buf[b]) cudaFreeHost(buf[b]);
    }
  }
  // dst (device) = src (host), stream-ordered on st; false on a CUDA error
  bool copy(void *dst, const void *src, size_t bytes, cudaStream_t st)
  {
    if (!ok) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
    const unsigned T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (size_t off = 0; off < bytes; off += CHUNK) {
      const size_t len = std::min(CHUNK, bytes - off);
      const int b = next;
      next = (next + 1) % K;
      if (used[b] && cudaEventSynchronize(ev[b]) != cudaSuccess) return false;   // its previous copy has landed
      char *d = (char *)buf[b];
      const char *sp = (const char *)src + off;
      if (len < (1u << 20) || T == 1) {
        memcpy(d, sp, len);
      } else {
        std::vector<std::thread> th;
        const size_t part = (len + T - 1) / T;
        for (unsigned t = 0; t < T; t++) {
          const size_t a = t * part, e = std::min(len, a + part);
          if (a < e) th.emplace_back([=] { memcpy(d + a, sp + a, e - a); });
        }
        for (auto &x : th) x.join();
      }
      if (cudaMemcpyAsync((char *)dst + off, d, len, cudaMemcpyHostToDevice, st) != cudaSuccess) return false;
      if (cudaEventRecord(ev[b], st) != cudaSuccess) return false;
      used[b] = true;
    }
    return true;
  }
};

__global__ void k_pat_count(uint32_t E, const uint32_t *__restrict__ n0, const uint32_t *__restrict__ n1,
                            uint32_t *cnt)
{
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  atomicAdd(cnt + n0[e], 1u);
  atomicAdd(cnt + n1[e], 1u);
}

__global__ void k_pat_first(uint32_t N, const uint32_t *__restrict__ ia, uint32_t *ja, uint32_t *fillp)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  ja[ia[i]] = i;
  fillp[i] = ia[i] + 1;
}

__global__ void k_pat_fill(uint32_t E, const uint32_t *__restrict__ n0, const uint32_t *__restrict__ n1,
                           uint32_t *fillp, uint32_t *ja, uint32_t *lastE)
{
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const uint32_t a = n0[e], b = n1[e];
  ja[atomicAdd(fillp + a, 1u)] = b;
  ja[atomicAdd(fillp + b, 1u)] = a;
  // the edge's lower end point is a lower neighbour of the other
  if (b < a) atomicMax(lastE + a, e + 1);
  if (a < b) atomicMax(lastE + b, e + 1);
}

// row i sorted (insertion sort: rows hold about 15 entries), its diagonal
// slot, its lower length
__global__ void k_pat_sort(uint32_t N, const uint32_t *__restrict__ ia, uint32_t *ja, uint32_t *diag,
                           uint32_t *lcnt)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t b = ia[i], e = ia[i + 1];
  for (uint32_t k = b + 1; k < e; k++) {
    const uint32_t v = ja[k];
    uint32_t m = k;
    while (m > b && ja[m - 1] > v) {
      ja[m] = ja[m - 1];
      m--;
    }
    ja[m] = v;
  }
  uint32_t d = b;
  while (d < e && ja[d] != i) d++;
  diag[i] = d;
  lcnt[i] = d - b;
}

__device__ __forceinline__ uint32_t find_col(const uint32_t *__restrict__ ja, uint32_t b, uint32_t e, uint32_t c)
{
  while (b < e) {   // first position with ja >= c
    const uint32_t m = (b + e) >> 1;
    if (ja[m] < c) b = m + 1;
    else e = m;
  }
  return b;
}

__global__ void k_pat_tblk(uint32_t N, const uint32_t *__restrict__ ia, const uint32_t *__restrict__ ja,
                           uint32_t *tblk)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (uint32_t j = ia[i]; j < ia[i + 1]; j++) {
    const uint32_t k = ja[j];
    const uint32_t p = find_col(ja, ia[k], ia[k + 1], i);
    tblk[j] = (p < ia[k + 1] && ja[p] == i) ? p : 0xffffffffu;
  }
}

__global__ void k_pat_last_lower(uint32_t N, const uint32_t *__restrict__ n0, const uint32_t *__restrict__ n1,
                                 const uint32_t *__restrict__ lastE, const uint32_t *__restrict__ ia,
                                 const uint32_t *__restrict__ ja, uint32_t *last_lower)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t le = lastE[i];
  if (!le) {
    last_lower[i] = 0xffffffffu;
    return;
  }
  const uint32_t e = le - 1, o = n0[e] == i ? n1[e] : n0[e];
  const uint32_t p = find_col(ja, ia[i], ia[i + 1], o);
  last_lower[i] = (p < ia[i + 1] && ja[p] == o) ? p : 0xffffffffu;
}

// one relaxation sweep of depth(i) = 1 + max depth over the lower (LOWER) or
// upper columns; *changed set when any depth grew
template <bool LOWER>
__global__ void k_pat_levels(uint32_t N, const uint32_t *__restrict__ ia, const uint32_t *__restrict__ ja,
                             const uint32_t *__restrict__ diag, uint32_t *depth, uint32_t *changed)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t jb = LOWER ? ia[i] : diag[i] + 1, je = LOWER ? diag[i] : ia[i + 1];
  uint32_t d = 1;
  for (uint32_t j = jb; j < je; j++) d = max(d, ((volatile uint32_t *)depth)[ja[j]] + 1);
  if (d > depth[i]) {
    depth[i] = d;
    *changed = 1;
  }
}

// ILU(0) products of every block of row i (matrix/ilu.cpp:71-84): COUNT
// writes the number per block, otherwise the (L slot or ~0, U block) pairs
template <bool COUNT>
__global__ void k_pat_pairs(uint32_t N, const uint32_t *__restrict__ ia, const uint32_t *__restrict__ ja,
                            const uint32_t *__restrict__ diag, const uint32_t *__restrict__ lpos,
                            const uint32_t *__restrict__ tblk, uint32_t *cnt, const uint32_t *__restrict__ pair_ptr,
                            uint2 *pairs)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t di = diag[i], ai = ia[i];
  for (uint32_t j = ia[i]; j < ia[i + 1]; j++) {
    const uint32_t k = ja[j], dk = diag[k];
    uint32_t pl = ai, pu = ia[k], c = 0, o = COUNT ? 0 : pair_ptr[j];
    while (pl <= di && pu <= dk) {
      const uint32_t cl = ja[pl], cu = ja[pu];
      if (cl == cu) {
        if (!COUNT) pairs[o + c] = make_uint2(cl == i ? 0xffffffffu : lpos[i] + (pl - ai), tblk[pu]);
        c++;
      }
      if (cl <= cu) pl++;
      if (cl >= cu) pu++;
    }
    if (COUNT) cnt[j] = c;
  }
}

// ---------------------------------------------------------------- exclusive scan
// out[0..n] = exclusive prefix sums of in[0..n-1] (out[n] = the total), in
// blocks of 1024 with the block totals scanned recursively.

__global__ void k_scan_block(size_t n, const uint32_t *__restrict__ in, uint32_t *out, uint32_t *bsum)
{
  __shared__ uint32_t s[1024];
  const size_t i = (size_t)blockIdx.x * 1024 + threadIdx.x;
  const uint32_t v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (unsigned off = 1; off < 1024; off <<= 1) {
    const uint32_t t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) bsum[blockIdx.x] = s[1023];
}

__global__ void k_scan_add(size_t n, uint32_t *out, const uint32_t *__restrict__ boff)
{
  const size_t i = (size_t)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += boff[blockIdx.x];
}

__global__ void k_scan_total(size_t n, const uint32_t *__restrict__ in, uint32_t *out)
{
  out[n] = n ? out[n - 1] + in[n - 1] : 0;
}

cudaError_t scan(size_t n, const uint32_t *in, uint32_t *out, cudaStream_t st)
{
  if (n == 0) {
    k_scan_total<<<1, 1, 0, st>>>(0, in, out);
    return cudaGetLastError();
  }
  const size_t nb = (n + 1023) / 1024;
  uint32_t *bsum = nullptr, *boff = nullptr;
  cudaError_t e = cudaMallocAsync(&bsum, nb * sizeof(uint32_t), st);
  if (e == cudaSuccess) e = cudaMallocAsync(&boff, (nb + 1) * sizeof(uint32_t), st);
  if (e != cudaSuccess) {
    if (bsum) cudaFreeAsync(bsum, st);
    return e;
  }
  k_scan_block<<<(unsigned)nb, 1024, 0, st>>>(n, in, out, bsum);
  kf_count_launch();
  if (nb > 1) {
    e = scan(nb, bsum, boff, st);
    if (e == cudaSuccess) {
      k_scan_add<<<(unsigned)nb, 1024, 0, st>>>(n, out, boff);
      kf_count_launch();
    }
  }
  k_scan_total<<<1, 1, 0, st>>>(n, in, out);
  kf_count_launch();
  cudaFreeAsync(bsum, st);
  cudaFreeAsync(boff, st);
  return e == cudaSuccess ? cudaGetLastError() : e;
}

// ------------------------------------------------------- mesh lists of the mirror

__global__ void k_pack4(uint32_t n, const double *__restrict__ a, const double *__restrict__ b,
                        const double *__restrict__ c, const double *__restrict__ d, double4 *out)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_double4(a[i], b[i], c[i], d[i]);
}

// incident edges of node ord[p] (row p): 1 + their count is the node's
// pattern row length
__global__ void k_inc_count(uint32_t N, const uint32_t *__restrict__ ord, const uint32_t *__restrict__ ia,
                            uint32_t *cnt)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t i = ord[p];
  cnt[p] = ia[i + 1] - ia[i] - 1;
}

__global__ void k_inc_place(uint32_t E, const uint32_t *__restrict__ n0, const uint32_t *__restrict__ n1,
                            const uint32_t *__restrict__ rowof, const uint32_t *__restrict__ ptr, uint32_t *slot,
                            uint32_t *edg)
{
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const uint32_t a = n0[e], b = n1[e];
  edg[ptr[rowof[a]] + atomicAdd(slot + a, 1u)] = e;
  edg[ptr[rowof[b]] + atomicAdd(slot + b, 1u)] = e | 0x80000000u;
}

// each row back in edge order (an edge appears once per row), then its other
// end points, least-squares terms seen from the node and blocks of (node, other)
__global__ void k_inc_rows(uint32_t N, const uint32_t *__restrict__ ord, const uint32_t *__restrict__ ptr,
                           uint32_t *edg, const uint32_t *__restrict__ n0, const uint32_t *__restrict__ n1,
                           const double *__restrict__ w, size_t E, const uint32_t *__restrict__ ia,
                           const uint32_t *__restrict__ ja, uint32_t *oth, double *incw, size_t wst, uint32_t *blk)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t b = ptr[p], en = ptr[p + 1], node = ord[p];
  for (uint32_t k = b + 1; k < en; k++) {
    const uint32_t v = edg[k];
    uint32_t m = k;
    while (m > b && (edg[m - 1] & 0x7fffffffu) > (v & 0x7fffffffu)) {
      edg[m] = edg[m - 1];
      m--;
    }
    edg[m] = v;
  }
  for (uint32_t k = b; k < en; k++) {
    const uint32_t v = edg[k], e = v & 0x7fffffffu, side = v >> 31;
    const uint32_t o = side ? n0[e] : n1[e];
    oth[k] = o;
    for (int c = 0; c < 3; c++) incw[c * wst + k] = w[(3 * side + c) * E + e];
    blk[k] = find_col(ja, ia[node], ia[node + 1], o);
  }
}

// first edge with n0 >= i (edges sorted by n0)
__global__ void k_n0_start(uint32_t N, uint32_t E, const uint32_t *__restrict__ n0, uint32_t *r0)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > N) return;
  uint32_t lo = 0, hi = E;
  while (lo < hi) {
    const uint32_t m = (lo + hi) >> 1;
    if (n0[m] < i) lo = m + 1;
    else hi = m;
  }
  r0[i] = lo;
}

// per visit position: edges with n0 = ord[p] (storage group size) and the
// node's n1-side incidences
__global__ void k_group_counts(uint32_t N, const uint32_t *__restrict__ ord, const uint32_t *__restrict__ r0,
                               const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ edg, uint32_t *c0,
                               uint32_t *c1)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t i = ord[p];
  c0[p] = r0[i + 1] - r0[i];
  uint32_t c = 0;
  for (uint32_t k = ptr[p]; k < ptr[p + 1]; k++) c += edg[k] >> 31;
  c1[p] = c;
}

__global__ void k_store_edges(uint32_t E, const uint32_t *__restrict__ n0, const uint32_t *__restrict__ n1,
                              const uint32_t *__restrict__ rowof, const uint32_t *__restrict__ eoff,
                              const uint32_t *__restrict__ r0, const double4 *__restrict__ egeo, uint32_t *spos,
                              uint32_t *n0s, uint32_t *n1s, double4 *egs)
{
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const uint32_t a = n0[e], s = eoff[rowof[a]] + (e - r0[a]);
  spos[e] = s;
  n0s[s] = a;
  n1s[s] = n1[e];
  egs[s] = egeo[e];
}

__global__ void k_in1_edges(uint32_t N, const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ edg,
                            const uint32_t *__restrict__ iptr, const uint32_t *__restrict__ spos, uint32_t *iedge)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  uint32_t j = iptr[p];
  for (uint32_t k = ptr[p]; k < ptr[p + 1]; k++)
    if (edg[k] >> 31) iedge[j++] = spos[edg[k] & 0x7fffffffu];
}

__global__ void k_visit_incidence(size_t n, const uint32_t *__restrict__ oth, const uint32_t *__restrict__ edg,
                                  const uint32_t *__restrict__ rowof, const double4 *__restrict__ egeo,
                                  uint32_t *othv, double4 *geo)
{
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  othv[k] = rowof[oth[k]];
  geo[k] = egeo[edg[k] & 0x7fffffffu];
}

__global__ void k_visit_edges(uint32_t E, const uint32_t *__restrict__ n0s, const uint32_t *__restrict__ n1s,
                              const uint32_t *__restrict__ rowof, uint32_t *e0v, uint32_t *e1v)
{
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E) return;
  e0v[s] = rowof[n0s[s]];
  e1v[s] = rowof[n1s[s]];
}

__global__ void k_visit_nodes(uint32_t N, const uint32_t *__restrict__ ord, const double4 *__restrict__ xyz,
                              double4 *xv)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) xv[p] = xyz[ord[p]];
}

// packed level schedule: the stream positions of slot s are [first[s],
// first[s+1]): for the upper sweep the row's diagonal block first, then the
// row's blocks of its descriptor's range, in column order
__global__ void k_packed_streams(uint32_t N, bool upper, const uint4 *__restrict__ desc,
                                 const uint32_t *__restrict__ first, const uint32_t *__restrict__ ja,
                                 const uint32_t *__restrict__ diag, uint32_t *row, uint32_t *col, uint32_t *src)
{
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  const uint4 d = desc[q];
  uint32_t k = first[q];
  row[q] = d.x;
  if (upper) {
    col[k] = d.x;
    src[k++] = diag[d.x];
  }
  for (uint32_t j = d.y; j < d.z; j++) {
    col[k] = ja[j];
    src[k++] = j;
  }
}

// the fill's view of a renumbered pattern, per incidence (visit row p, node
// ord[p]) and per node of the mesh
__global__ void k_fill_targets(uint32_t N, const uint32_t *__restrict__ ord, const uint32_t *__restrict__ rank,
                               const uint32_t *__restrict__ inc_ptr, const uint32_t *__restrict__ inc_oth,
                               const uint32_t *__restrict__ ia, const uint32_t *__restrict__ ja,
                               const uint32_t *__restrict__ diag, const uint32_t *__restrict__ last_lower,
                               const uint32_t *__restrict__ lpos, uint32_t *blk, uint32_t *fd, uint32_t *fl,
                               uint32_t *fp, uint32_t *row_node)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t node = ord[p], r = rank[node];
  for (uint32_t k = inc_ptr[p]; k < inc_ptr[p + 1]; k++) blk[k] = find_col(ja, ia[r], ia[r + 1], rank[inc_oth[k]]);
  fd[node] = diag[r];
  fl[node] = last_lower[r];
  fp[node] = lpos[r];
  row_node[r] = node;
}

// rows listed by level in row order from their depths (counting sort)
void levels_from_depth(const std::vector<uint32_t> &depth, std::vector<uint32_t> &rows, std::vector<uint32_t> &ptr)
{
  const size_t N = depth.size();
  uint32_t nlev = 1;
  for (uint32_t d : depth) nlev = d > nlev ? d : nlev;
  ptr.assign(nlev + 1, 0);
  for (size_t i = 0; i < N; i++) ptr[depth[i]]++;
  for (uint32_t l = 0; l < nlev; l++) ptr[l + 1] += ptr[l];
  rows.assign(N, 0);
  std::vector<uint32_t> top(ptr.begin(), ptr.end() - 1);
  for (size_t i = 0; i < N; i++) rows[top[depth[i] - 1]++] = (uint32_t)i;
}

}  // namespace

int kf_pattern_matches(const IluSet &s, size_t N, size_t E, const unsigned int *n0, const unsigned int *n1,
                       cudaStream_t st, long *host_us)
{
  HostPattern r;
  const auto t0 = std::chrono::steady_clock::now();
  kf_build_pattern(r, N, E, n0, n1);
  if (host_us)
    *host_us = (long)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0)
                   .count();
  bool ok = true, same = true;
  auto cmp = [&](const uint32_t *dev, const uint32_t *host, size_t n) {
    if (!ok || !same) return;
    std::vector<uint32_t> v(n);
    if (n && (cudaMemcpyAsync(v.data(), dev, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
              cudaStreamSynchronize(st) != cudaSuccess)) {
      ok = false;
      return;
    }
    same = std::equal(v.begin(), v.end(), host);
  };
  cmp(s.ia, r.ia.data(), N + 1);
  cmp(s.ja, r.ja.data(), r.nnz);
  cmp(s.diag, r.diag.data(), N);
  cmp(s.tblk, r.tblk.data(), r.nnz);
  cmp(s.lpos, r.lpos.data(), N + 1);
  cmp(s.last_lower, r.last_lower.data(), N);
  cmp(s.pair_ptr, r.pair_ptr.data(), r.nnz + 1);
  cmp(reinterpret_cast<const uint32_t *>(s.pairs), r.pairs.data(), r.pairs.size());
  cmp(s.lev_l, r.lev_l.data(), N);
  cmp(s.lev_u, r.lev_u.data(), N);
  same = same && s.lev_l_ptr == r.lev_l_ptr && s.lev_u_ptr == r.lev_u_ptr;
  if (!ok) {
    cudaGetLastError();
    kf_set_error(KFUN3D_ERR_CUDA, "pattern check: a copy from the device failed");
    return -1;
  }
  return same ? 1 : 0;
}

void kf_free_device_pattern(DevPattern &d)
{
  void *ptrs[] = {d.ia, d.ja, d.diag, d.tblk, d.lpos, d.last_lower, d.pair_ptr, d.pairs};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  d = DevPattern{};
}

int kf_build_pattern_device(HostPattern &p, DevPattern &d, size_t N, size_t E, const unsigned int *n0,
                            const unsigned int *n1, cudaStream_t st)
{
  d = DevPattern{};
  // every end point a row of the matrix (the kernels below index by them)
  if (N == 0 || N >= 0xffffffffu || E >= 0x7fffffffu) {
    kf_set_error(KFUN3D_ERR_ARG, "block pattern: no nodes, or more nodes or edges than 32-bit indices hold");
    return KFUN3D_ERR_ARG;
  }
  for (size_t e = 0; e < E; e++)
    if (n0[e] >= N || n1[e] >= N) {
      kf_set_error(KFUN3D_ERR_ARG, "block pattern: an edge end point is not a node");
      return KFUN3D_ERR_ARG;
    }
  uint32_t *dn0 = nullptr, *dn1 = nullptr, *cnt = nullptr, *fillp = nullptr, *lastE = nullptr, *lcnt = nullptr;
  uint32_t *depth = nullptr, *changed = nullptr;
  bool ok = true;
  auto ck = [&](cudaError_t e) {
    if (e != cudaSuccess && ok) {
      ok = false;
      cudaGetLastError();
    }
  };
  const size_t N1 = N + 1;
  ck(cudaMalloc(&dn0, (E + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&dn1, (E + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&cnt, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&fillp, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&lastE, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&lcnt, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&depth, 2 * N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&changed, sizeof(uint32_t)));
  ck(cudaMalloc(&d.ia, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&d.diag, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&d.lpos, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&d.last_lower, N1 * sizeof(uint32_t)));
  if (ok && E) {
    ck(cudaMemcpyAsync(dn0, n0, E * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(dn1, n1, E * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  }
  size_t nnz = 0;
  const std::vector<uint32_t> ones(N, 1u);
  if (ok) {
    // row lengths: 1 (the diagonal) + incident edges
    ck(cudaMemcpyAsync(cnt, ones.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ck(cudaMemsetAsync(lastE, 0, N1 * sizeof(uint32_t), st));
    if (E) {
      k_pat_count<<<nblk(E, 256), 256, 0, st>>>((uint32_t)E, dn0, dn1, cnt);
      kf_count_launch();
    }
    ck(scan(N, cnt, d.ia, st));
    uint32_t nz = 0;
    ck(cudaMemcpyAsync(&nz, d.ia + N, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));
    nnz = nz;
  }
  if (ok) {
    ck(cudaMalloc(&d.ja, (nnz + 1) * sizeof(uint32_t)));
    ck(cudaMalloc(&d.tblk, (nnz + 1) * sizeof(uint32_t)));
    ck(cudaMalloc(&d.pair_ptr, (nnz + 1) * sizeof(uint32_t)));
  }
  if (ok) {
    k_pat_first<<<nblk(N, 256), 256, 0, st>>>((uint32_t)N, d.ia, d.ja, fillp);
    if (E) k_pat_fill<<<nblk(E, 256), 256, 0, st>>>((uint32_t)E, dn0, dn1, fillp, d.ja, lastE);
    k_pat_sort<<<nblk(N, 128), 128, 0, st>>>((uint32_t)N, d.ia, d.ja, d.diag, lcnt);
    kf_count_launch(E ? 3 : 2);
    ck(cudaGetLastError());
    ck(scan(N, lcnt, d.lpos, st));
    k_pat_tblk<<<nblk(N, 128), 128, 0, st>>>((uint32_t)N, d.ia, d.ja, d.tblk);
    k_pat_last_lower<<<nblk(N, 256), 256, 0, st>>>((uint32_t)N, dn0, dn1, lastE, d.ia, d.ja, d.last_lower);
    kf_count_launch(2);
    ck(cudaGetLastError());
  }
  // level sets: relax until no depth grows (at most one sweep more than levels)
  std::vector<uint32_t> hdepth[2];
  for (int lower = 1; lower >= 0 && ok; lower--) {
    uint32_t *dp = depth + (lower ? 0 : N1);
    ck(cudaMemcpyAsync(dp, ones.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    for (size_t it = 0; it <= N && ok; it++) {
      uint32_t h = 0;
      ck(cudaMemsetAsync(changed, 0, sizeof(uint32_t), st));
      if (lower) k_pat_levels<true><<<nblk(N, 256), 256, 0, st>>>((uint32_t)N, d.ia, d.ja, d.diag, dp, changed);
      else k_pat_levels<false><<<nblk(N, 256), 256, 0, st>>>((uint32_t)N, d.ia, d.ja, d.diag, dp, changed);
      kf_count_launch();
      ck(cudaGetLastError());
      ck(cudaMemcpyAsync(&h, changed, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      ck(cudaStreamSynchronize(st));
      if (!h) break;
    }
    hdepth[lower ? 0 : 1].resize(N);
    ck(cudaMemcpyAsync(hdepth[lower ? 0 : 1].data(), dp, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  }
  // ILU(0) product lists: counts per block (into a buffer of nnz entries),
  // their exclusive sums, then the pairs
  if (ok) {
    ck(cudaStreamSynchronize(st));
    cudaFree(fillp);   // the row slots are no longer needed
    fillp = nullptr;
    ck(cudaMalloc(&fillp, (nnz + 1) * sizeof(uint32_t)));
  }
  if (ok) {
    k_pat_pairs<true><<<nblk(N, 128), 128, 0, st>>>((uint32_t)N, d.ia, d.ja, d.diag, d.lpos, d.tblk, fillp, nullptr,
                                                   nullptr);
    kf_count_launch();
    ck(cudaGetLastError());
    ck(scan(nnz, fillp, d.pair_ptr, st));
    uint32_t np = 0;
    ck(cudaMemcpyAsync(&np, d.pair_ptr + nnz, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));
    d.npairs = np;
    if (ok) ck(cudaMalloc(&d.pairs, (size_t)std::max<uint32_t>(np, 1) * sizeof(uint2)));
    if (ok) {
      k_pat_pairs<false><<<nblk(N, 128), 128, 0, st>>>((uint32_t)N, d.ia, d.ja, d.diag, d.lpos, d.tblk, nullptr,
                                                      d.pair_ptr, d.pairs);
      kf_count_launch();
      ck(cudaGetLastError());
    }
  }
  // the host's copy of what its set-up code reads
  if (ok) {
    p = HostPattern{};
    p.n = N;
    p.nnz = nnz;
    p.ia.resize(N1);
    p.ja.resize(nnz);
    p.diag.resize(N);
    p.lpos.resize(N1);
    p.last_lower.resize(N);
    ck(cudaMemcpyAsync(p.ia.data(), d.ia, N1 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(cudaMemcpyAsync(p.ja.data(), d.ja, nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(cudaMemcpyAsync(p.diag.data(), d.diag, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(cudaMemcpyAsync(p.lpos.data(), d.lpos, N1 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(cudaMemcpyAsync(p.last_lower.data(), d.last_lower, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));
  }
  if (ok) {
    levels_from_depth(hdepth[0], p.lev_l, p.lev_l_ptr);
    levels_from_depth(hdepth[1], p.lev_u, p.lev_u_ptr);
    p.on_device = true;
  }
  void *tmp[] = {dn0, dn1, cnt, fillp, lastE, lcnt, depth, changed};
  for (void *t : tmp)
    if (t) cudaFree(t);
  if (!ok) {
    kf_free_device_pattern(d);
    kf_set_error(KFUN3D_ERR_CUDA, "block pattern on the device: a CUDA call failed");
    return KFUN3D_ERR_CUDA;
  }
  return KFUN3D_OK;
}

int kf_build_mesh_lists_device(DevMesh &m, const GEOMETRY *g)
{
  const uint32_t N = m.N, E = m.E;
  const cudaStream_t st = m.stream;
  const size_t ninc = 2 * (size_t)E, wst = (ninc + 3) & ~(size_t)3;
  m.wstride = (uint32_t)wst;
  uint32_t *dn0 = nullptr, *dn1 = nullptr, *cnt = nullptr, *slot = nullptr, *r0 = nullptr, *c1 = nullptr,
           *spos = nullptr;
  double *raw = nullptr;   // [4][E] edge geometry, then [6][E] least-squares terms (w0, w1)
  bool ok = true;
  auto ck = [&](cudaError_t e) {
    if (e != cudaSuccess && ok) {
      ok = false;
      cudaGetLastError();
    }
  };
  Stager sg;
  auto up = [&](void *dst, const void *src, size_t bytes) {
    if (ok && bytes && !sg.copy(dst, src, bytes, st)) ck(cudaErrorUnknown);
  };
  const size_t E1 = (size_t)E + 1, N1 = (size_t)N + 1;
  ck(cudaMalloc(&dn0, E1 * sizeof(uint32_t)));
  ck(cudaMalloc(&dn1, E1 * sizeof(uint32_t)));
  ck(cudaMalloc(&cnt, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&slot, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&raw, 6 * E1 * sizeof(double)));
  ck(cudaMalloc(&m.egeo, E1 * sizeof(double4)));
  ck(cudaMalloc(&m.inc_ptr, N1 * sizeof(uint32_t)));
  ck(cudaMalloc(&m.inc_oth, (wst + 4) * sizeof(uint32_t)));
  ck(cudaMalloc(&m.inc_edge, (ninc + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&m.inc_blk, (ninc + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&m.inc_w, (3 * wst + 4) * sizeof(double)));
  up(dn0, g->e->eptr->n0, (size_t)E * sizeof(uint32_t));
  up(dn1, g->e->eptr->n1, (size_t)E * sizeof(uint32_t));
  // edge geometry (unit normal, area) packed per edge
  {
    const double *src[4] = {g->e->xyzn->x0, g->e->xyzn->x1, g->e->xyzn->x2, g->e->xyzn->x3};
    for (int c = 0; c < 4; c++) up(raw + c * (size_t)E, src[c], (size_t)E * sizeof(double));
    if (ok && E) {
      k_pack4<<<nblk(E, 256), 256, 0, st>>>(E, raw, raw + E, raw + 2 * (size_t)E, raw + 3 * (size_t)E, m.egeo);
      kf_count_launch();
      ck(cudaGetLastError());
    }
  }
  // node incidence in edge order (row p belongs to node ord[p])
  if (ok) {
    const double *src[6] = {g->e->w->w0->x0, g->e->w->w0->x1, g->e->w->w0->x2,
                            g->e->w->w1->x0, g->e->w->w1->x1, g->e->w->w1->x2};
    for (int c = 0; c < 6; c++) up(raw + c * (size_t)E, src[c], (size_t)E * sizeof(double));
    ck(cudaMemsetAsync(slot, 0, N1 * sizeof(uint32_t), st));
    ck(cudaMemsetAsync(m.inc_oth, 0, (wst + 4) * sizeof(uint32_t), st));
    ck(cudaMemsetAsync(m.inc_w, 0, (3 * wst + 4) * sizeof(double), st));
  }
  if (ok) {
    k_inc_count<<<nblk(N, 256), 256, 0, st>>>(N, m.ord, m.ia, cnt);
    kf_count_launch();
    ck(cudaGetLastError());
    ck(scan(N, cnt, m.inc_ptr, st));
  }
  if (ok) {
    if (E) {
      k_inc_place<<<nblk(E, 256), 256, 0, st>>>(E, dn0, dn1, m.rowof, m.inc_ptr, slot, m.inc_edge);
      kf_count_launch();
    }
    k_inc_rows<<<nblk(N, 128), 128, 0, st>>>(N, m.ord, m.inc_ptr, m.inc_edge, dn0, dn1, raw, E, m.ia, m.ja,
                                            m.inc_oth, m.inc_w, wst, m.inc_blk);
    kf_count_launch();
    ck(cudaGetLastError());
  }
  // two-pass residual storage: groups by n0 in visit order, each in edge order
  if (ok && m.two_pass) {
    ck(cudaMalloc(&r0, N1 * sizeof(uint32_t)));
    ck(cudaMalloc(&c1, N1 * sizeof(uint32_t)));
    ck(cudaMalloc(&spos, E1 * sizeof(uint32_t)));
    ck(cudaMalloc(&m.eoff, N1 * sizeof(uint32_t)));
    ck(cudaMalloc(&m.n0s, E1 * sizeof(uint32_t)));
    ck(cudaMalloc(&m.n1, E1 * sizeof(uint32_t)));
    ck(cudaMalloc(&m.egeo_s, E1 * sizeof(double4)));
    ck(cudaMalloc(&m.in1_ptr, N1 * sizeof(uint32_t)));
    ck(cudaMalloc(&m.in1_edge, E1 * sizeof(uint32_t)));
    ck(cudaMalloc(&m.eres, E1 * sizeof(double4)));
    if (ok) {
      k_n0_start<<<nblk(N1, 256), 256, 0, st>>>(N, E, dn0, r0);
      k_group_counts<<<nblk(N, 256), 256, 0, st>>>(N, m.ord, r0, m.inc_ptr, m.inc_edge, cnt, c1);
      kf_count_launch(2);
      ck(cudaGetLastError());
      ck(scan(N, cnt, m.eoff, st));
      ck(scan(N, c1, m.in1_ptr, st));
    }
    if (ok) {
      if (E) {
        k_store_edges<<<nblk(E, 256), 256, 0, st>>>(E, dn0, dn1, m.rowof, m.eoff, r0, m.egeo, spos, m.n0s, m.n1,
                                                   m.egeo_s);
        kf_count_launch();
      }
      k_in1_edges<<<nblk(N, 256), 256, 0, st>>>(N, m.inc_ptr, m.inc_edge, m.in1_ptr, spos, m.in1_edge);
      kf_count_launch();
      ck(cudaGetLastError());
    }
    // visit-order copies: each incidence's other end as a visit position and
    // its edge geometry, the edges' end points as visit positions, the
    // coordinates in visit order, room for the state and the gradients
    if (ok && m.visit) {
      ck(cudaMalloc(&m.inc_othv, (ninc + 1) * sizeof(uint32_t)));
      ck(cudaMalloc(&m.inc_geo, (ninc + 1) * sizeof(double4)));
      ck(cudaMalloc(&m.n0v, E1 * sizeof(uint32_t)));
      ck(cudaMalloc(&m.n1v, E1 * sizeof(uint32_t)));
      ck(cudaMalloc(&m.xyzv, N1 * sizeof(double4)));
      double4 **vv[] = {&m.qv, &m.gxv, &m.gyv, &m.gzv};
      for (double4 **v : vv) ck(cudaMalloc(v, N1 * sizeof(double4)));
      if (ok) {
        if (E) {
          k_visit_incidence<<<nblk(ninc, 256), 256, 0, st>>>(ninc, m.inc_oth, m.inc_edge, m.rowof, m.egeo,
                                                             m.inc_othv, m.inc_geo);
          k_visit_edges<<<nblk(E, 256), 256, 0, st>>>(E, m.n0s, m.n1, m.rowof, m.n0v, m.n1v);
          kf_count_launch(2);
        }
        k_visit_nodes<<<nblk(N, 256), 256, 0, st>>>(N, m.ord, m.xyz, m.xyzv);
        kf_count_launch();
        ck(cudaGetLastError());
      }
    }
  }
  ck(cudaStreamSynchronize(st));
  void *tmp[] = {dn0, dn1, cnt, slot, raw, r0, c1, spos};
  for (void *t : tmp)
    if (t) cudaFree(t);
  if (!ok) {
    kf_set_error(KFUN3D_ERR_CUDA, "device mirror: building the incidence lists on the device failed");
    return KFUN3D_ERR_CUDA;
  }
  return KFUN3D_OK;
}

int kf_packed_streams_device(uint32_t N, bool upper, const uint4 *desc, const uint32_t *first, const uint32_t *ja,
                             const uint32_t *diag, uint32_t *row, uint32_t *col, uint32_t *src, cudaStream_t st)
{
  if (N) {
    k_packed_streams<<<nblk(N, 256), 256, 0, st>>>(N, upper, desc, first, ja, diag, row, col, src);
    kf_count_launch();
  }
  return cudaGetLastError() == cudaSuccess ? KFUN3D_OK : KFUN3D_ERR_CUDA;
}

int kf_fill_targets_device(const DevMesh &m, IluSet &s)
{
  const uint32_t N = m.N;
  const size_t ninc = 2 * (size_t)m.E;
  bool ok = true;
  auto ck = [&](cudaError_t e) {
    if (e != cudaSuccess && ok) {
      ok = false;
      cudaGetLastError();
    }
  };
  ck(cudaMalloc(&s.fill_blk, (ninc + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&s.fill_diag, ((size_t)N + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&s.fill_last, ((size_t)N + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&s.fill_lpos, ((size_t)N + 1) * sizeof(uint32_t)));
  ck(cudaMalloc(&s.row_node, ((size_t)N + 1) * sizeof(uint32_t)));
  if (ok && N) {
    k_fill_targets<<<nblk(N, 128), 128, 0, m.stream>>>(N, m.ord, m.ilu_rank, m.inc_ptr, m.inc_oth, s.ia, s.ja,
                                                       s.diag, s.last_lower, s.lpos, s.fill_blk, s.fill_diag,
                                                       s.fill_last, s.fill_lpos, s.row_node);
    kf_count_launch();
    ck(cudaGetLastError());
  }
  ck(cudaStreamSynchronize(m.stream));
  if (!ok) {
    kf_set_error(KFUN3D_ERR_CUDA, "spatial ILU(0) order: fill targets on the device failed");
    return KFUN3D_ERR_CUDA;
  }
  return KFUN3D_OK;
}
