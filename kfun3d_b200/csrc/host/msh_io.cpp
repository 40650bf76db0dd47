// kfun3d_b200 host side: uns3d .msh generator, reader and GEOMETRY set-up.
//
// The file format is the reference's (read by src/mesh.c:22-154 through
// matrix/fio.h:10-72): big-endian, 1-based indices.
//   header  13 x u32: tets, nodes, edges, wall groups, 0, far groups,
//                     wall triangles, 0, far triangles, wall nodes, 0, far nodes, 0
//   edges   u32 n0[E], u32 n1[E], f64 xn[E], yn[E], zn[E], area[E]
//   nodes   f64 x[N], y[N], z[N], vol[N]
//   per boundary kind (wall, then far field): 2 x groups u32 (skipped by the
//   reader), 4 x triangles u32 (three indices into the kind's node list and
//   the owning tet), node ids u32, normals f64 nx[], ny[], nz[].
//
// kfun3d_setup_load() builds the same GEOMETRY as the reference's Setup at
// one thread: the edge permutation of src/index.c:53-111 (merge sort with
// selection-sort leaves, which is not stable, so it is followed exactly), the
// greedy wall-face colouring of src/sbface_coloring.c:11-93 and the
// least-squares weights of src/weights.c:9-398 in the reference's operation
// order, so the result is bit-identical.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "kfun3d_b200.h"
#include "internal.h"

namespace {

// ----------------------------------------------------------------- byte order
inline uint32_t bswap32(uint32_t v) { return __builtin_bswap32(v); }
inline uint64_t bswap64(uint64_t v) { return __builtin_bswap64(v); }

struct Writer {
  FILE *f;
  bool ok = true;
  void u32(const uint32_t *a, size_t n) {
    std::vector<uint32_t> b(n);
    for (size_t i = 0; i < n; i++) b[i] = bswap32(a[i]);
    ok = ok && fwrite(b.data(), 4, n, f) == n;
  }
  void f64(const double *a, size_t n) {
    std::vector<uint64_t> b(n);
    for (size_t i = 0; i < n; i++) {
      uint64_t u;
      memcpy(&u, a + i, 8);
      b[i] = bswap64(u);
    }
    ok = ok && fwrite(b.data(), 8, n, f) == n;
  }
};

// f(begin, end) over [0, n) split across the host's threads (sequential for
// small n); every index is handled by exactly one call.
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

struct Reader {
  const unsigned char *p, *end;
  bool ok = true;
  void u32(uint32_t *a, size_t n) {
    if ((size_t)(end - p) < 4 * n) { ok = false; return; }
    const unsigned char *src = p;
    parallel_ranges(n, [&](size_t i0, size_t i1) {
      for (size_t i = i0; i < i1; i++) {
        uint32_t u;
        memcpy(&u, src + 4 * i, 4);
        a[i] = bswap32(u);
      }
    });
    p += 4 * n;
  }
  void f64(double *a, size_t n) {
    if ((size_t)(end - p) < 8 * n) { ok = false; return; }
    const unsigned char *src = p;
    parallel_ranges(n, [&](size_t i0, size_t i1) {
      for (size_t i = i0; i < i1; i++) {
        uint64_t u;
        memcpy(&u, src + 8 * i, 8);
        u = bswap64(u);
        memcpy(a + i, &u, 8);
      }
    });
    p += 8 * n;
  }
  void skip(size_t bytes) {
    if ((size_t)(end - p) < bytes) { ok = false; return; }
    p += bytes;
  }
};

// ----------------------------------------------------------------- generator
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct V3 { double x, y, z; };
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// The seven lattice directions of the Kuhn (Freudenthal) split: every edge of
// every tet joins p to p + d for one of these.
const int DIRS[7][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};

int dir_index(int dx, int dy, int dz) {
  for (int k = 0; k < 7; k++)
    if (DIRS[k][0] == dx && DIRS[k][1] == dy && DIRS[k][2] == dz) return k;
  return -1;
}

}  // namespace

extern "C" int kfun3d_mesh_generate(const char *path, const kfun3d_mesh_spec *spec)
{
  const long n = spec->n;
  if (n < 3 || n > 2000) return -1;
  const long N = n * n * n;
  const double h = 1.0 / (double)(n - 1);
  auto nid = [n](long i, long j, long k) { return i + n * (j + n * k); };

  // coordinates: jitter interior nodes, then the Gaussian bump on z = 0
  // decaying linearly to the top face.
  SplitMix rng{spec->seed * 0x2545F4914F6CDD1Dull + 12345};
  std::vector<V3> X(N);
  for (long k = 0; k < n; k++)
    for (long j = 0; j < n; j++)
      for (long i = 0; i < n; i++) {
        V3 p{i * h, j * h, k * h};
        bool interior = i > 0 && i < n - 1 && j > 0 && j < n - 1 && k > 0 && k < n - 1;
        if (interior && spec->jitter > 0) {
          p.x += (2 * rng.uniform() - 1) * spec->jitter * h;
          p.y += (2 * rng.uniform() - 1) * spec->jitter * h;
          p.z += (2 * rng.uniform() - 1) * spec->jitter * h;
        }
        const double s2 = 2 * spec->bump_sigma * spec->bump_sigma;
        p.z += spec->bump_height * std::exp(-((p.x - 0.5) * (p.x - 0.5) + (p.y - 0.5) * (p.y - 0.5)) / s2) * (1 - p.z);
        X[nid(i, j, k)] = p;
      }

  // node numbering: the lattice order (permute = 0), a seeded random
  // permutation (1, Fisher-Yates) or the Morton order of the lattice (2)
  std::vector<uint32_t> perm(N);
  for (long i = 0; i < N; i++) perm[i] = (uint32_t)i;
  if (spec->permute == 1)
    for (long i = N - 1; i > 0; i--) {
      long r = (long)(rng.next() % (uint64_t)(i + 1));
      std::swap(perm[i], perm[r]);
    }
  if (spec->permute == 2) {
    auto spread = [](uint64_t v) {
      uint64_t r = 0;
      for (int b = 0; b < 21; b++) r |= ((v >> b) & 1ull) << (3 * b);
      return r;
    };
    std::vector<std::pair<uint64_t, uint32_t>> key(N);
    for (long k = 0; k < n; k++)
      for (long j = 0; j < n; j++)
        for (long i = 0; i < n; i++)
          key[nid(i, j, k)] = {spread(i) | spread(j) << 1 | spread(k) << 2, (uint32_t)nid(i, j, k)};
    std::sort(key.begin(), key.end());
    for (long r = 0; r < N; r++) perm[key[r].second] = (uint32_t)r;
  }

  // median-dual face vectors, accumulated per (node, direction) slot
  std::vector<V3> S(7 * N, V3{0, 0, 0});
  std::vector<double> vol(N, 0.0);
  // tet edges (p,q) with the other two vertices (r,s) so that (p,q,r,s) is an
  // even permutation of a positively oriented tet (0,1,2,3)
  const int EDGE[6][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 2, 0, 3}, {1, 3, 2, 0}, {2, 3, 0, 1}};
  const int PERMS[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  long ntets = 0;
  for (long k = 0; k < n - 1; k++)
    for (long j = 0; j < n - 1; j++)
      for (long i = 0; i < n - 1; i++)
        for (int t = 0; t < 6; t++) {
          int L[4][3];
          L[0][0] = (int)i; L[0][1] = (int)j; L[0][2] = (int)k;
          for (int s = 1; s < 4; s++) {
            for (int c = 0; c < 3; c++) L[s][c] = L[s - 1][c];
            L[s][PERMS[t][s - 1]] += 1;
          }
          // orientation from the unperturbed lattice (consistent even if the
          // jitter inverts a tet)
          V3 a{(double)(L[1][0] - L[0][0]), (double)(L[1][1] - L[0][1]), (double)(L[1][2] - L[0][2])};
          V3 b{(double)(L[2][0] - L[0][0]), (double)(L[2][1] - L[0][1]), (double)(L[2][2] - L[0][2])};
          V3 c{(double)(L[3][0] - L[0][0]), (double)(L[3][1] - L[0][1]), (double)(L[3][2] - L[0][2])};
          if (dot(cross(a, b), c) < 0)
            for (int cc = 0; cc < 3; cc++) std::swap(L[1][cc], L[2][cc]);
          long v[4];
          V3 P[4];
          for (int s = 0; s < 4; s++) { v[s] = nid(L[s][0], L[s][1], L[s][2]); P[s] = X[v[s]]; }
          const V3 g = 0.25 * (P[0] + P[1] + P[2] + P[3]);
          const double tv = dot(cross(P[1] - P[0], P[2] - P[0]), P[3] - P[0]) / 6.0;
          for (int s = 0; s < 4; s++) vol[v[s]] += 0.25 * tv;
          for (int e = 0; e < 6; e++) {
            const int p = EDGE[e][0], q = EDGE[e][1], r = EDGE[e][2], s = EDGE[e][3];
            const V3 m = 0.5 * (P[p] + P[q]);
            const V3 fr = (1.0 / 3.0) * (P[p] + P[q] + P[r]);
            const V3 fs = (1.0 / 3.0) * (P[p] + P[q] + P[s]);
            V3 sv = 0.5 * (cross(fr - m, g - m) + cross(g - m, fs - m));
            int dx = L[q][0] - L[p][0], dy = L[q][1] - L[p][1], dz = L[q][2] - L[p][2];
            int di = dir_index(dx, dy, dz);
            long base = v[p];
            if (di < 0) {
              di = dir_index(-dx, -dy, -dz);
              base = v[q];
              sv = -1.0 * sv;
            }
            if (di < 0) return -2;
            S[7 * base + di] = S[7 * base + di] + sv;
          }
          ntets++;
        }

  // unique edges in slot order
  std::vector<uint32_t> e0, e1;
  std::vector<double> ex, ey, ez, ea;
  e0.reserve(7 * N); e1.reserve(7 * N);
  for (long k = 0; k < n; k++)
    for (long j = 0; j < n; j++)
      for (long i = 0; i < n; i++)
        for (int d = 0; d < 7; d++) {
          long i2 = i + DIRS[d][0], j2 = j + DIRS[d][1], k2 = k + DIRS[d][2];
          if (i2 >= n || j2 >= n || k2 >= n) continue;
          long a = nid(i, j, k), b = nid(i2, j2, k2);
          V3 sv = S[7 * a + d];
          uint32_t pa = perm[a], pb = perm[b];
          if (pb < pa) { std::swap(pa, pb); sv = -1.0 * sv; }
          double area = std::sqrt(dot(sv, sv));
          e0.push_back(pa + 1);
          e1.push_back(pb + 1);
          ex.push_back(sv.x / area);
          ey.push_back(sv.y / area);
          ez.push_back(sv.z / area);
          ea.push_back(area);
        }
  const size_t E = e0.size();

  // boundary triangles: bottom face (z = 0) is the slip wall, the other five
  // are far field.  Winding so that -(a x b) points out of the domain.
  struct Tri { long v[3]; long tet; };
  std::vector<Tri> wall, farf;
  auto add_face = [&](int axis, long fixed, int outward) {
    int u = (axis + 1) % 3, w = (axis + 2) % 3;
    for (long b = 0; b < n - 1; b++)
      for (long a = 0; a < n - 1; a++) {
        long c00[3], c10[3], c01[3], c11[3];
        c00[axis] = c10[axis] = c01[axis] = c11[axis] = fixed;
        c00[u] = a; c00[w] = b;
        c10[u] = a + 1; c10[w] = b;
        c01[u] = a; c01[w] = b + 1;
        c11[u] = a + 1; c11[w] = b + 1;
        long *tri[2][3] = {{c00, c10, c11}, {c00, c11, c01}};
        for (int t = 0; t < 2; t++) {
          V3 A{(double)(tri[t][1][0] - tri[t][0][0]), (double)(tri[t][1][1] - tri[t][0][1]), (double)(tri[t][1][2] - tri[t][0][2])};
          V3 B{(double)(tri[t][2][0] - tri[t][0][0]), (double)(tri[t][2][1] - tri[t][0][1]), (double)(tri[t][2][2] - tri[t][0][2])};
          V3 cr = cross(A, B);
          double comp = axis == 0 ? cr.x : (axis == 1 ? cr.y : cr.z);
          Tri T;
          for (int s = 0; s < 3; s++) T.v[s] = nid(tri[t][s][0], tri[t][s][1], tri[t][s][2]);
          if (comp * outward > 0) std::swap(T.v[1], T.v[2]);
          T.tet = 0;
          (axis == 2 && fixed == 0 ? wall : farf).push_back(T);
        }
      }
  };
  add_face(2, 0, -1);
  add_face(2, n - 1, +1);
  add_face(0, 0, -1);
  add_face(0, n - 1, +1);
  add_face(1, 0, -1);
  add_face(1, n - 1, +1);

  auto node_list = [&](const std::vector<Tri> &tris, std::vector<uint32_t> &ids,
                       std::vector<double> &nx, std::vector<double> &ny, std::vector<double> &nz,
                       std::vector<uint32_t> &fidx) {
    std::vector<int32_t> slot(N, -1);
    std::vector<V3> acc;
    std::vector<long> nodes;
    for (const Tri &t : tris)
      for (int s = 0; s < 3; s++)
        if (slot[t.v[s]] < 0) { slot[t.v[s]] = 0; nodes.push_back(t.v[s]); }
    // list ordered by permuted id
    std::vector<std::pair<uint32_t, long>> order;
    for (long v : nodes) order.push_back({perm[v], v});
    std::sort(order.begin(), order.end());
    for (size_t i = 0; i < order.size(); i++) slot[order[i].second] = (int32_t)i;
    acc.assign(order.size(), V3{0, 0, 0});
    fidx.resize(4 * tris.size());
    for (size_t f = 0; f < tris.size(); f++) {
      const Tri &t = tris[f];
      V3 a = X[t.v[1]] - X[t.v[0]], b = X[t.v[2]] - X[t.v[0]];
      V3 nv = (-1.0 / 6.0) * cross(a, b);
      for (int s = 0; s < 3; s++) {
        acc[slot[t.v[s]]] = acc[slot[t.v[s]]] + nv;
        fidx[s * tris.size() + f] = (uint32_t)slot[t.v[s]] + 1;
      }
      fidx[3 * tris.size() + f] = 1;   // owning tet: not used by the reader
    }
    ids.resize(order.size());
    nx.resize(order.size()); ny.resize(order.size()); nz.resize(order.size());
    for (size_t i = 0; i < order.size(); i++) {
      ids[i] = order[i].first + 1;
      nx[i] = acc[i].x; ny[i] = acc[i].y; nz[i] = acc[i].z;
    }
  };
  std::vector<uint32_t> sids, fids, sfac, ffac;
  std::vector<double> snx, sny, snz, fnx, fny, fnz;
  node_list(wall, sids, snx, sny, snz, sfac);
  node_list(farf, fids, fnx, fny, fnz, ffac);

  std::vector<double> xs(N), ys(N), zs(N), vs(N);
  for (long i = 0; i < N; i++) {
    xs[perm[i]] = X[i].x; ys[perm[i]] = X[i].y; zs[perm[i]] = X[i].z; vs[perm[i]] = vol[i];
  }

  FILE *f = fopen(path, "wb");
  if (!f) return -3;
  Writer w{f};
  uint32_t hdr[13] = {(uint32_t)ntets, (uint32_t)N, (uint32_t)E, 1, 0, 1,
                      (uint32_t)wall.size(), 0, (uint32_t)farf.size(),
                      (uint32_t)sids.size(), 0, (uint32_t)fids.size(), 0};
  w.u32(hdr, 13);
  w.u32(e0.data(), E); w.u32(e1.data(), E);
  w.f64(ex.data(), E); w.f64(ey.data(), E); w.f64(ez.data(), E); w.f64(ea.data(), E);
  w.f64(xs.data(), N); w.f64(ys.data(), N); w.f64(zs.data(), N); w.f64(vs.data(), N);
  uint32_t wg[2] = {(uint32_t)wall.size(), (uint32_t)sids.size()};
  w.u32(wg, 2);
  w.u32(sfac.data(), sfac.size());
  w.u32(sids.data(), sids.size());
  w.f64(snx.data(), snx.size()); w.f64(sny.data(), sny.size()); w.f64(snz.data(), snz.size());
  uint32_t fg[2] = {(uint32_t)farf.size(), (uint32_t)fids.size()};
  w.u32(fg, 2);
  w.u32(ffac.data(), ffac.size());
  w.u32(fids.data(), fids.size());
  w.f64(fnx.data(), fnx.size()); w.f64(fny.data(), fny.size()); w.f64(fnz.data(), fnz.size());
  bool ok = w.ok;
  ok = (fclose(f) == 0) && ok;
  return ok ? 0 : -4;
}

// ----------------------------------------------------------------- set-up

namespace {

// Index sort of src/index.c:53-111 (merge sort over halves, selection-sort
// leaves of at most 500 entries that swap in place), producing the same
// permutation for equal keys.
const long LEAF = 500;

void leaf_sort(const uint32_t *key, uint32_t *lo, uint32_t *hi)
{
  for (uint32_t *i = lo; i < hi; i++) {
    uint32_t ki = key[*i];
    for (uint32_t *j = i + 1; j < hi; j++)
      if (ki > key[*j]) {
        uint32_t t = *i; *i = *j; *j = t;
        ki = key[*i];
      }
  }
}

void merge_runs(const uint32_t *key, const uint32_t *a, const uint32_t *ae,
                const uint32_t *b, const uint32_t *be, uint32_t *out)
{
  while (a != ae && b != be) *out++ = (key[*b] < key[*a]) ? *b++ : *a++;
  while (a != ae) *out++ = *a++;
  while (b != be) *out++ = *b++;
}

// Sorts [lo,hi); the result lands in lo when in_place, else in tmp.  The two
// halves are disjoint, so the top `par` levels sort them on two threads:
// every leaf and every merge is the same as in the sequential recursion, so
// is the permutation.
void index_sort(const uint32_t *key, uint32_t *lo, uint32_t *hi, uint32_t *tmp, bool in_place, int par = 0)
{
  if (hi - lo <= LEAF) {
    leaf_sort(key, lo, hi);
    if (!in_place) memcpy(tmp, lo, (size_t)(hi - lo) * sizeof(uint32_t));
    return;
  }
  uint32_t *mid = lo + (hi - lo) / 2;
  uint32_t *tmid = tmp + (mid - lo), *thi = tmp + (hi - lo);
  if (par > 0) {
    std::thread left([=] { index_sort(key, lo, mid, tmp, !in_place, par - 1); });
    index_sort(key, mid, hi, tmid, !in_place, par - 1);
    left.join();
  } else {
    index_sort(key, lo, mid, tmp, !in_place);
    index_sort(key, mid, hi, tmid, !in_place);
  }
  if (in_place) merge_runs(key, tmp, tmid, tmid, thi, lo);
  else merge_runs(key, lo, mid, mid, hi, tmp);
}

int sort_levels()
{
  unsigned t = std::thread::hardware_concurrency();
  int lv = 0;
  while ((1u << (lv + 1)) <= t && lv < 6) lv++;
  return lv;
}

template <class T> T *alloc(size_t n) { return (T *)calloc(n ? n : 1, sizeof(T)); }

}  // namespace

extern "C" GEOMETRY *kfun3d_setup_load(const char *path)
{
  SetupTrace tr("load");
  FILE *fs = fopen(path, "rb");
  if (!fs) { kf_set_error(KFUN3D_ERR_IO, "cannot open mesh file"); return nullptr; }
  fseek(fs, 0, SEEK_END);
  long fsz = ftell(fs);
  rewind(fs);
  std::vector<unsigned char> buf((size_t)fsz);
  if (fread(buf.data(), 1, (size_t)fsz, fs) != (size_t)fsz) { fclose(fs); kf_set_error(KFUN3D_ERR_IO, "short read"); return nullptr; }
  fclose(fs);
  tr.mark("file read");
  Reader rd{buf.data(), buf.data() + fsz};
  uint32_t p[13];
  rd.u32(p, 13);
  const size_t N = p[1], E = p[2];

  GEOMETRY *g = alloc<GEOMETRY>(1);
  // edges (src/edges.c:22-87)
  std::vector<uint32_t> ebuf(2 * E);
  std::vector<double> nbuf(4 * E);
  rd.u32(ebuf.data(), 2 * E);
  rd.f64(nbuf.data(), 4 * E);
  std::vector<uint32_t> order(E), tmp(E);
  for (size_t i = 0; i < E; i++) order[i] = (uint32_t)i;
  tr.mark("edges decoded");
  if (E) index_sort(ebuf.data(), order.data(), order.data() + E, tmp.data(), true, E > 100000 ? sort_levels() : 0);
  tr.mark("index sort");
  g->e = alloc<struct etbl>(1);
  g->e->sz = E;
  g->e->eptr = alloc<struct edge>(1);
  g->e->eptr->n0 = alloc<unsigned int>(E);
  g->e->eptr->n1 = alloc<unsigned int>(E);
  g->e->xyzn = alloc<struct xyzn>(1);
  g->e->xyzn->x0 = alloc<double>(E); g->e->xyzn->x1 = alloc<double>(E);
  g->e->xyzn->x2 = alloc<double>(E); g->e->xyzn->x3 = alloc<double>(E);
  parallel_ranges(E, [&](size_t i0, size_t i1) {
    for (size_t i = i0; i < i1; i++) {
      const uint32_t s = order[i];
      g->e->eptr->n0[i] = ebuf[s] - 1;
      g->e->eptr->n1[i] = ebuf[s + E] - 1;
      g->e->xyzn->x0[i] = nbuf[s];
      g->e->xyzn->x1[i] = nbuf[s + E];
      g->e->xyzn->x2[i] = nbuf[s + 2 * E];
      g->e->xyzn->x3[i] = nbuf[s + 3 * E];
    }
  });
  tr.mark("edges permuted");
  // nodes (src/nodes.c:19-56); the dual volume is read and dropped
  g->n = alloc<struct ntbl>(1);
  g->n->sz = N;
  g->n->xyz = alloc<struct xyz>(1);
  g->n->xyz->x0 = alloc<double>(N); g->n->xyz->x1 = alloc<double>(N); g->n->xyz->x2 = alloc<double>(N);
  rd.f64(g->n->xyz->x0, N); rd.f64(g->n->xyz->x1, N); rd.f64(g->n->xyz->x2, N);
  rd.skip(8 * N);
  g->n->cdt = alloc<double>(N);
  g->n->part = alloc<unsigned int>(N);
  // boundaries (src/boundaries.c:143-204)
  auto read_kind = [&](size_t nfaces, size_t nnodes, size_t ngroups, std::vector<uint32_t> &fc,
                       struct bntbl *bn) {
    rd.skip(ngroups * 2 * 4);
    fc.resize(4 * nfaces);
    rd.u32(fc.data(), 4 * nfaces);
    bn->sz = nnodes;
    bn->nptr = alloc<unsigned int>(nnodes);
    rd.u32(bn->nptr, nnodes);
    for (size_t i = 0; i < nnodes; i++) bn->nptr[i] -= 1;
    bn->xyz = alloc<struct xyz>(1);
    bn->xyz->x0 = alloc<double>(nnodes); bn->xyz->x1 = alloc<double>(nnodes); bn->xyz->x2 = alloc<double>(nnodes);
    rd.f64(bn->xyz->x0, nnodes); rd.f64(bn->xyz->x1, nnodes); rd.f64(bn->xyz->x2, nnodes);
  };
  g->b = alloc<struct btbl>(1);
  g->b->s = alloc<struct bntbl>(1);
  g->b->f = alloc<struct bntbl>(1);
  std::vector<uint32_t> sfc, ffc;
  read_kind(p[6], p[9], p[3], sfc, g->b->s);
  read_kind(p[8], p[11], p[5], ffc, g->b->f);
  if (!rd.ok || rd.p != rd.end) {
    kfun3d_setup_free(g);
    kf_set_error(KFUN3D_ERR_IO, "mesh file size does not match its header");
    return nullptr;
  }
  const size_t F = p[6];
  g->b->fc = alloc<struct bftbl>(1);
  g->b->fc->sz = F;
  g->b->fc->fptr = alloc<struct face>(1);
  unsigned int *f0 = alloc<unsigned int>(F), *f1 = alloc<unsigned int>(F), *f2 = alloc<unsigned int>(F);
  for (size_t i = 0; i < F; i++) {
    f0[i] = g->b->s->nptr[sfc[i] - 1];
    f1[i] = g->b->s->nptr[sfc[i + F] - 1];
    f2[i] = g->b->s->nptr[sfc[i + 2 * F] - 1];
  }
  g->b->fc->fptr->n0 = f0; g->b->fc->fptr->n1 = f1; g->b->fc->fptr->n2 = f2;

  // block sizes (src/csr.c:123-128) and the matrix handle (src/mesh.c:121)
  g->c = alloc<struct ctbl>(1);
  g->c->b = 4;
  g->c->b2 = 16;
  g->c->sz = 4 * N;
  tr.mark("nodes and boundaries");
  g->matrix = CXX_Matrix_Init(N, E, 4, 1, g->e->eptr->n0, g->e->eptr->n1);
  tr.mark("matrix handle");

  // one thread owns every node and edge (src/subdomains.c:116-188 at T = 1)
  g->s = alloc<struct stbl>(1);
  g->s->sz = 1;
  g->s->i = alloc<unsigned int>(2);
  g->s->i[1] = (unsigned int)E;

  // greedy wall-face colouring (src/sbface_coloring.c:11-93)
  {
    std::vector<uint32_t> count(F + 1, 0);
    std::vector<uint8_t> mark(N);
    size_t k = 0, c = 0;
    for (size_t i = 0; i < F;) {
      std::fill(mark.begin(), mark.end(), 0);
      for (size_t j = i; j < F; j++) {
        if (mark[f0[j]] | mark[f1[j]] | mark[f2[j]]) continue;
        mark[f0[j]] = mark[f1[j]] = mark[f2[j]] = 1;
        std::swap(f0[j], f0[k]);
        std::swap(f1[j], f1[k]);
        std::swap(f2[j], f2[k]);
        k++;
        count[c]++;
      }
      c++;
      i = k;
    }
    g->t = alloc<struct stbl>(1);
    g->t->sz = c;
    g->t->i = alloc<unsigned int>(c + 1);
    unsigned int sum = 0;
    for (size_t i = 0; i < c; i++) { g->t->i[i] = sum; sum += count[i]; }
    g->t->i[c] = sum;
  }

  tr.mark("wall colouring");
  // least-squares weights (src/weights.c:299-398).  The reference's edge
  // loops add into both end points; here every node gathers over its edges in
  // edge order (the same additions in the same order) and the nodes run in
  // parallel.
  {
    const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
    const double *X = g->n->xyz->x0, *Y = g->n->xyz->x1, *Z = g->n->xyz->x2;
    std::vector<uint32_t> iptr(N + 1, 0), inc(2 * E);
    for (size_t e = 0; e < E; e++) { iptr[n0[e] + 1]++; iptr[n1[e] + 1]++; }
    for (size_t i = 0; i < N; i++) iptr[i + 1] += iptr[i];
    {
      std::vector<uint32_t> pos(iptr.begin(), iptr.end() - 1);
      for (size_t e = 0; e < E; e++) { inc[pos[n0[e]]++] = (uint32_t)e; inc[pos[n1[e]]++] = (uint32_t)e; }
    }
    std::vector<double> w(7 * N, 0.0);
    parallel_ranges(N, [&](size_t r0, size_t r1) {     // weights.c:237-297
      for (size_t i = r0; i < r1; i++)
        for (uint32_t k = iptr[i]; k < iptr[i + 1]; k++) {
          const size_t e = inc[k], a = n0[e], b = n1[e];
          double rx, ry, rz;
          if (a == i) { rx = X[b] - X[a]; ry = Y[b] - Y[a]; rz = Z[b] - Z[a]; }
          else { rx = X[a] - X[b]; ry = Y[a] - Y[b]; rz = Z[a] - Z[b]; }
          w[7 * i + 0] += rx * rx; w[7 * i + 1] += rx * ry; w[7 * i + 2] += rx * rz;
        }
    });
    parallel_ranges(N, [&](size_t r0, size_t r1) {
      for (size_t i = r0; i < r1; i++) {
        w[7 * i + 0] = std::sqrt(w[7 * i + 0]);
        w[7 * i + 1] /= w[7 * i + 0];
        w[7 * i + 2] /= w[7 * i + 0];
      }
    });
    parallel_ranges(N, [&](size_t r0, size_t r1) {     // weights.c:173-232
      for (size_t i = r0; i < r1; i++)
        for (uint32_t k = iptr[i]; k < iptr[i + 1]; k++) {
          const size_t e = inc[k], a = n0[e], b = n1[e];
          const double dx = X[b] - X[a], dy = Y[b] - Y[a], dz = Z[b] - Z[a];
          if (a == i) {
            const double d = w[7 * a + 1] / w[7 * a + 0];
            const double d_ = dy - dx * d;
            w[7 * a + 3] += d_ * d_;
            w[7 * a + 4] += d_ * dz;
          } else {
            const double d = w[7 * b + 1] / w[7 * b + 0];
            const double d_ = -dy + dx * d;
            w[7 * b + 3] += d_ * d_;
            w[7 * b + 4] -= d_ * dz;
          }
        }
    });
    parallel_ranges(N, [&](size_t r0, size_t r1) {
      for (size_t i = r0; i < r1; i++) {
        w[7 * i + 3] = std::sqrt(w[7 * i + 3]);
        w[7 * i + 4] /= w[7 * i + 3];
      }
    });
    parallel_ranges(N, [&](size_t r0, size_t r1) {     // weights.c:102-170
      for (size_t i = r0; i < r1; i++)
        for (uint32_t k = iptr[i]; k < iptr[i + 1]; k++) {
          const size_t e = inc[k], a = n0[e], b = n1[e];
          const double dx = X[b] - X[a], dy = Y[b] - Y[a], dz = Z[b] - Z[a];
          if (a == i) {
            const double d0 = w[7 * a + 1] / w[7 * a + 0];
            const double d0_ = dy - dx * d0;
            const double d1 = w[7 * a + 2] / w[7 * a + 0];
            const double d1_ = dz - dx * d1;
            const double d2 = w[7 * a + 4] / w[7 * a + 3];
            const double d2_ = d1_ - d2 * d0_;
            w[7 * a + 5] += d2_ * d2_;
          } else {
            const double d0 = w[7 * b + 1] / w[7 * b + 0];
            const double d0_ = -dy + dx * d0;
            const double d1 = w[7 * b + 2] / w[7 * b + 0];
            const double d1_ = -dz + dx * d1;
            const double d2 = w[7 * b + 4] / w[7 * b + 3];
            const double d2_ = d1_ - d2 * d0_;
            w[7 * b + 5] += d2_ * d2_;
          }
        }
    });
    parallel_ranges(N, [&](size_t r0, size_t r1) {     // weights.c:335-366
      for (size_t i = r0; i < r1; i++) {
        double *wi = &w[7 * i];
        wi[5] = std::sqrt(wi[5]);
        const double sw00 = wi[0] * wi[0], sw11 = wi[3] * wi[3], sw22 = wi[5] * wi[5];
        const double w00 = 1.0 / sw00, w11 = 1.0 / sw11, w22 = 1.0 / sw22;
        const double w01 = wi[1] / wi[0], w02 = wi[2] / wi[0], w12 = wi[4] / wi[3];
        double m0 = wi[1] * wi[4];
        m0 -= wi[2] * wi[3];
        const double m1 = wi[0] * wi[3] * sw22;
        const double w33 = m0 / m1;
        wi[0] = w00; wi[3] = w11; wi[5] = w22; wi[1] = w01; wi[2] = w02; wi[4] = w12; wi[6] = w33;
      }
    });
    g->e->w = alloc<struct weights>(1);
    g->e->w->w0 = alloc<struct xyz>(1);
    g->e->w->w1 = alloc<struct xyz>(1);
    double *t0x = alloc<double>(E), *t0y = alloc<double>(E), *t0z = alloc<double>(E);
    double *t1x = alloc<double>(E), *t1y = alloc<double>(E), *t1z = alloc<double>(E);
    parallel_ranges(E, [&](size_t r0, size_t r1) {     // weights.c:9-100
      for (size_t e = r0; e < r1; e++) {
        const size_t a = n0[e], b = n1[e];
        const double dx = X[b] - X[a], dy = Y[b] - Y[a], dz = Z[b] - Z[a];
        {
          const double *wa = &w[7 * a];
          double c0 = -dx * wa[1] + dy;
          double c1 = -dx * wa[2] + dz;
          c1 = -wa[4] * c0 + c1;
          double tx = wa[3] * wa[1] * c0;
          tx = dx * wa[0] - tx;
          tx += wa[6] * c1;
          double ty = wa[4] * wa[5] * c1;
          ty = wa[3] * c0 - ty;
          t0x[e] = tx; t0y[e] = ty; t0z[e] = wa[5] * c1;
        }
        {
          const double *wb = &w[7 * b];
          double c0 = dx * wb[1] - dy;
          double c1 = dx * wb[2] - dz;
          c1 = -wb[4] * c0 + c1;
          double tx = wb[3] * wb[1] * c0;
          tx = -dx * wb[0] - tx;
          tx += wb[6] * c1;
          double ty = wb[4] * wb[5] * c1;
          ty = wb[3] * c0 - ty;
          t1x[e] = tx; t1y[e] = ty; t1z[e] = wb[5] * c1;
        }
      }
    });
    g->e->w->w0->x0 = t0x; g->e->w->w0->x1 = t0y; g->e->w->w0->x2 = t0z;
    g->e->w->w1->x0 = t1x; g->e->w->w1->x1 = t1y; g->e->w->w1->x2 = t1z;
  }

  tr.mark("least-squares weights");
  // free-stream initial state (src/guess.c:8-20)
  g->q = alloc<struct qtbl>(1);
  g->q->q = alloc<double>(4 * N);
  kfun3d_initial_guess(g);
  return g;
}

extern "C" void kfun3d_initial_guess(GEOMETRY *g)
{
  double u, v;
  kfun3d_get_freestream(&u, &v);
  for (size_t i = 0; i < g->n->sz; i++) {
    g->q->q[4 * i + 0] = 1.0;
    g->q->q[4 * i + 1] = u;
    g->q->q[4 * i + 2] = v;
    g->q->q[4 * i + 3] = 0.0;
  }
}

extern "C" void kfun3d_setup_free(GEOMETRY *g)
{
  if (!g) return;
  if (g->e) {
    if (g->e->xyzn) { free(g->e->xyzn->x0); free(g->e->xyzn->x1); free(g->e->xyzn->x2); free(g->e->xyzn->x3); free(g->e->xyzn); }
    if (g->e->w) {
      if (g->e->w->w0) { free(g->e->w->w0->x0); free(g->e->w->w0->x1); free(g->e->w->w0->x2); free(g->e->w->w0); }
      if (g->e->w->w1) { free(g->e->w->w1->x0); free(g->e->w->w1->x1); free(g->e->w->w1->x2); free(g->e->w->w1); }
      free(g->e->w);
    }
    if (g->e->eptr) { free(g->e->eptr->n0); free(g->e->eptr->n1); free(g->e->eptr); }
    free(g->e);
  }
  if (g->s) { free(g->s->i); free(g->s); }
  if (g->t) { free(g->t->i); free(g->t); }
  free(g->c);
  if (g->b) {
    for (struct bntbl *bn : {g->b->s, g->b->f}) {
      if (!bn) continue;
      if (bn->xyz) { free(bn->xyz->x0); free(bn->xyz->x1); free(bn->xyz->x2); free(bn->xyz); }
      free(bn->nptr);
      free(bn);
    }
    if (g->b->fc) {
      if (g->b->fc->fptr) { free(g->b->fc->fptr->n0); free(g->b->fc->fptr->n1); free(g->b->fc->fptr->n2); free(g->b->fc->fptr); }
      free(g->b->fc);
    }
    free(g->b);
  }
  if (g->n) {
    if (g->n->xyz) { free(g->n->xyz->x0); free(g->n->xyz->x1); free(g->n->xyz->x2); free(g->n->xyz); }
    free(g->n->cdt); free(g->n->part); free(g->n);
  }
  if (g->q) { free(g->q->q); free(g->q); }
  if (g->matrix) CXX_Matrix_Delete(g->matrix);
  free(g);
}

// Big-endian walkers of matrix/fio.h:10-72, exported for a host driver that
// links the reference's own src/mesh.c.
extern "C" void CXX_Walk_Int(char *l, const char *h, const size_t sz, unsigned int *b)
{
  (void)h;
  Reader rd{(const unsigned char *)l, (const unsigned char *)l + 4 * sz};
  rd.u32(b, sz);
}

extern "C" void CXX_Walk_Double(char *l, const char *h, const size_t sz, double *b)
{
  (void)h;
  Reader rd{(const unsigned char *)l, (const unsigned char *)l + 8 * sz};
  rd.f64(b, sz);
}
