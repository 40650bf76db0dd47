// kfun3d_b200: BLAS-1 reductions, wall forces, the reference's C entry points
// and the device-resident pseudo-transient Newton / GMRES(30) driver.
//
// Compiled with -fmad=false: in exact mode every reduction sums in index
// order (as the reference at one OpenMP thread) and every scalar update keeps
// its operation order; fast mode uses explicit fma() and fixed-shape tree
// reductions (deterministic run to run).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

extern int g_kf_verbose;

namespace {

constexpr double JV_EPS = 1.490116119384766e-08;   // src/kernel.c:12
constexpr int RED_BLOCKS = 296;                    // 2 x 148 SMs
constexpr int S_XN = 40, S_H = 41, S_QN = 42, S_FN = 43, S_T0 = 44, S_CMP = 52;

inline unsigned nblk(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// ------------------------------------------------------------------ reductions

// Sum of a[i]*b[i] in index order (src/utils.c:53-67, src/kernel.c:131-134):
// one warp loads 32 products at a time and every lane adds them in order.
__global__ void k_dot_seq(size_t n, const double *__restrict__ a, const double *__restrict__ b,
                          double *__restrict__ out, int op)
{
  const int lane = threadIdx.x;
  double s = 0.0;
  for (size_t base = 0; base < n; base += 32) {
    const size_t i = base + lane;
    const double p = (i < n) ? a[i] * b[i] : 0.0;
    const int cnt = (n - base) < 32 ? (int)(n - base) : 32;
    for (int l = 0; l < cnt; l++) s += __shfl_sync(0xffffffffu, p, l);
  }
  if (lane == 0) {
    if (op == 0) *out = s;
    else if (op == 1) *out = sqrt(s);
    else *out = sqrt(1.0 + sqrt(s));   // src/kernel.c:95
  }
}

__device__ __forceinline__ double warp_sum(double v)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Fast form: fixed grid, fixed tree, so the result is run-to-run identical.
__global__ void __launch_bounds__(256) k_dot_partial(size_t n, const double *__restrict__ a,
                                                     const double *__restrict__ b, double *__restrict__ part)
{
  __shared__ double sm[8];
  double s = 0.0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t n2 = n / 2;
  const double2 *a2 = reinterpret_cast<const double2 *>(a), *b2 = reinterpret_cast<const double2 *>(b);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
    const double2 x = a2[i], y = b2[i];
    s = fma(x.x, y.x, s);
    s = fma(x.y, y.y, s);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) s = fma(a[n - 1], b[n - 1], s);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < 8 ? sm[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
  }
}

__global__ void k_dot_final(const double *__restrict__ part, int np, double *__restrict__ out, int op)
{
  __shared__ double sm[8];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sm[w];
    if (op == 0) *out = v;
    else if (op == 1) *out = sqrt(v);
    else *out = sqrt(1.0 + sqrt(v));
  }
}

// Fast-mode modified Gram-Schmidt of V[k+1] against V[0..k] and its
// normalisation (src/kernel.c:129-141) in one cooperative launch.  Pass v
// applies the previous projection, w -= h[v-1] V[v-1], and forms the block
// partial sums of w.V[v] in the same sweep; after a grid-wide barrier every
// block adds the partial sums in the same fixed order, so all blocks hold the
// identical h[v] (run-to-run deterministic).  Partial sums alternate between
// two buffers, so one barrier per projection suffices.
__device__ __forceinline__ double block_sum(double v, double *sm)
{
  v = warp_sum(v);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sm[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;   // valid in thread 0
}

__device__ __forceinline__ double grid_total(const double *part, int np, double *sm)
{
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) v += __ldcg(part + i);   // written by other blocks
  v = block_sum(v, sm);
  if (threadIdx.x == 0) sm[32] = v;
  __syncthreads();
  const double t = sm[32];
  __syncthreads();
  return t;
}

constexpr int KF_MGS_ELEMS = 8;   // double2 elements per thread kept in registers

__global__ void __launch_bounds__(256, 3) k_mgs_coop(size_t n, double *__restrict__ V, int k,
                                                     double *__restrict__ h, double *__restrict__ part,
                                                     unsigned *bar, int *err)
{
  __shared__ double sm[40];
  const int G = gridDim.x;
  const size_t n2 = n / 2;
  double2 *w = reinterpret_cast<double2 *>(V + (size_t)(k + 1) * n);
  const size_t stride = (size_t)G * blockDim.x;
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t iend_reg = i0 + KF_MGS_ELEMS * stride;   // elements beyond are re-read from memory
  double2 pv[KF_MGS_ELEMS];   // this thread's elements of the previous basis vector
  double hprev = 0.0;
  for (int v = 0; v <= k + 1; v++) {
    const double2 *prev = v > 0 ? reinterpret_cast<const double2 *>(V + (size_t)(v - 1) * n) : nullptr;
    const double2 *cur = v <= k ? reinterpret_cast<const double2 *>(V + (size_t)v * n) : nullptr;
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < KF_MGS_ELEMS; t++) {
      const size_t i = i0 + (size_t)t * stride;
      if (i < n2) {
        double2 a = w[i];
        if (v > 0) {
          a.x = fma(-hprev, pv[t].x, a.x);
          a.y = fma(-hprev, pv[t].y, a.y);
          w[i] = a;
        }
        if (cur) {
          const double2 c = __ldcs(cur + i);
          s = fma(a.x, c.x, s);
          s = fma(a.y, c.y, s);
          pv[t] = c;
        } else {
          s = fma(a.x, a.x, s);
          s = fma(a.y, a.y, s);
        }
      }
    }
    for (size_t i = iend_reg; i < n2; i += stride) {
      double2 a = w[i];
      if (prev) {
        const double2 p = prev[i];
        a.x = fma(-hprev, p.x, a.x);
        a.y = fma(-hprev, p.y, a.y);
        w[i] = a;
      }
      if (cur) {
        const double2 c = cur[i];
        s = fma(a.x, c.x, s);
        s = fma(a.y, c.y, s);
      } else {
        s = fma(a.x, a.x, s);
        s = fma(a.y, a.y, s);
      }
    }
    double *pb = part + (v & 1) * G;
    const double bs = block_sum(s, sm);
    if (threadIdx.x == 0) pb[blockIdx.x] = bs;
    __threadfence();
    if (!kf_grid_barrier(bar, err)) return;
    const double tot = grid_total(pb, G, sm);
    if (v <= k) {
      hprev = tot;
      if (blockIdx.x == 0 && threadIdx.x == 0) h[v] = tot;
    } else {
      const double nrm = sqrt(tot);
      if (blockIdx.x == 0 && threadIdx.x == 0) h[k + 1] = nrm;
      const double sc = 1.0 / nrm;
      for (size_t i = i0; i < n2; i += stride) {
        double2 a = w[i];
        a.x *= sc;
        a.y *= sc;
        w[i] = a;
      }
    }
  }
}

// The same modified Gram-Schmidt with the vector being orthogonalised, w,
// resident on chip for the whole launch: each thread keeps its first
// KF_MGS_REG double2 elements of w in registers and the next `ts` in shared
// memory (the rest, on meshes too large for that, stays in global memory).
// A sweep then reads only the previous basis vector (just read by the sweep
// before, so mostly an L2 hit) and the current one from memory, instead of
// reading and writing w as well.  One CTA of 512 threads per SM; element i of
// thread g (grid-wide) is g + t * stride for t = 0, 1, ...  The arithmetic is
// k_mgs_coop's: per thread the same fma chain in the same element order,
// block sums and the fixed-order grid total unchanged in form.
constexpr int KF_MGS_REG = 16;    // double2 elements per thread in registers
constexpr int KF_MGS_BATCH = 4;   // elements whose loads are in flight together

__global__ void __launch_bounds__(512, 1) k_mgs_resident(size_t n, double *__restrict__ V, int k,
                                                         double *__restrict__ h, double *__restrict__ part,
                                                         unsigned *bar, int *err, int ts)
{
  extern __shared__ double2 wsm[];   // [ts][blockDim.x]
  __shared__ double sm[40];
  const int G = gridDim.x;
  const size_t n2 = n / 2;
  double2 *w = reinterpret_cast<double2 *>(V + (size_t)(k + 1) * n);
  const size_t stride = (size_t)G * blockDim.x;
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tcache = (size_t)KF_MGS_REG + (size_t)ts;   // elements t below this are on chip
  double2 wr[KF_MGS_REG];
#pragma unroll
  for (int t = 0; t < KF_MGS_REG; t++) {
    const size_t i = i0 + (size_t)t * stride;
    wr[t] = i < n2 ? w[i] : make_double2(0.0, 0.0);
  }
  for (int t = 0; t < ts; t++) {
    const size_t i = i0 + (size_t)(KF_MGS_REG + t) * stride;
    wsm[(size_t)t * blockDim.x + threadIdx.x] = i < n2 ? w[i] : make_double2(0.0, 0.0);
  }
  double hprev = 0.0;
  for (int v = 0; v <= k + 1; v++) {
    const double2 *prev = v > 0 ? reinterpret_cast<const double2 *>(V + (size_t)(v - 1) * n) : nullptr;
    const double2 *cur = v <= k ? reinterpret_cast<const double2 *>(V + (size_t)v * n) : nullptr;
    double s = 0.0;
    // elements in batches of KF_MGS_BATCH: all their loads are issued before
    // any is used, so a thread keeps that many pairs of loads in flight
    double2 pv[KF_MGS_BATCH], cv[KF_MGS_BATCH];
    auto load = [&](int u, size_t i) {
      if (prev) pv[u] = prev[i];
      if (cur) cv[u] = cur[i];
    };
    auto step = [&](double2 &a, int u) {
      if (prev) {
        a.x = fma(-hprev, pv[u].x, a.x);
        a.y = fma(-hprev, pv[u].y, a.y);
      }
      if (cur) {
        s = fma(a.x, cv[u].x, s);
        s = fma(a.y, cv[u].y, s);
      } else {
        s = fma(a.x, a.x, s);
        s = fma(a.y, a.y, s);
      }
    };
#pragma unroll
    for (int t0 = 0; t0 < KF_MGS_REG; t0 += KF_MGS_BATCH) {
#pragma unroll
      for (int u = 0; u < KF_MGS_BATCH; u++) {
        const size_t i = i0 + (size_t)(t0 + u) * stride;
        if (i < n2) load(u, i);
      }
#pragma unroll
      for (int u = 0; u < KF_MGS_BATCH; u++) {
        const size_t i = i0 + (size_t)(t0 + u) * stride;
        if (i < n2) step(wr[t0 + u], u);
      }
    }
    for (int t0 = 0; t0 < ts; t0 += KF_MGS_BATCH) {
#pragma unroll
      for (int u = 0; u < KF_MGS_BATCH; u++) {
        const size_t i = i0 + (size_t)(KF_MGS_REG + t0 + u) * stride;
        if (t0 + u < ts && i < n2) load(u, i);
      }
#pragma unroll
      for (int u = 0; u < KF_MGS_BATCH; u++) {
        const size_t i = i0 + (size_t)(KF_MGS_REG + t0 + u) * stride;
        if (t0 + u < ts && i < n2) {
          double2 a = wsm[(size_t)(t0 + u) * blockDim.x + threadIdx.x];
          step(a, u);
          wsm[(size_t)(t0 + u) * blockDim.x + threadIdx.x] = a;
        }
      }
    }
    for (size_t i0g = i0 + tcache * stride; i0g < n2; i0g += KF_MGS_BATCH * stride) {
#pragma unroll
      for (int u = 0; u < KF_MGS_BATCH; u++) {
        const size_t i = i0g + (size_t)u * stride;
        if (i < n2) load(u, i);
      }
#pragma unroll
      for (int u = 0; u < KF_MGS_BATCH; u++) {
        const size_t i = i0g + (size_t)u * stride;
        if (i < n2) {
          double2 a = w[i];
          step(a, u);
          if (prev) w[i] = a;
        }
      }
    }
    double *pb = part + (v & 1) * G;
    const double bs = block_sum(s, sm);
    if (threadIdx.x == 0) pb[blockIdx.x] = bs;
    __threadfence();
    if (!kf_grid_barrier(bar, err)) return;
    const double tot = grid_total(pb, G, sm);
    if (v <= k) {
      hprev = tot;
      if (blockIdx.x == 0 && threadIdx.x == 0) h[v] = tot;
    } else {
      const double nrm = sqrt(tot);
      if (blockIdx.x == 0 && threadIdx.x == 0) h[k + 1] = nrm;
      const double sc = 1.0 / nrm;
#pragma unroll
      for (int t = 0; t < KF_MGS_REG; t++) {
        const size_t i = i0 + (size_t)t * stride;
        if (i < n2) w[i] = make_double2(wr[t].x * sc, wr[t].y * sc);
      }
      for (int t = 0; t < ts; t++) {
        const size_t i = i0 + (size_t)(KF_MGS_REG + t) * stride;
        if (i < n2) {
          const double2 a = wsm[(size_t)t * blockDim.x + threadIdx.x];
          w[i] = make_double2(a.x * sc, a.y * sc);
        }
      }
      for (size_t i = i0 + tcache * stride; i < n2; i += stride) {
        double2 a = w[i];
        a.x *= sc;
        a.y *= sc;
        w[i] = a;
      }
    }
  }
}

// y = (mult * coef[0]) * x + y with the coefficient on the device
__global__ void k_axpy_dev(size_t n, const double *__restrict__ coef, double mult, const double *__restrict__ x,
                           double *__restrict__ y, int fast)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = mult * coef[0];
  y[i] = fast ? fma(a, x[i], y[i]) : a * x[i] + y[i];
}

// y = a x + y (src/utils.c:69-87)
__global__ void k_axpy(size_t n, double a, const double *__restrict__ x, double *__restrict__ y, int fast)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = fast ? fma(a, x[i], y[i]) : a * x[i] + y[i];
}

// y = a[0] v[0] + y, then a[1] v[1] + y, ... (k_axpy's arithmetic, vector
// after vector in that order) in one pass: y and every v read once
struct AxpyList {
  const double *v[KF_NBASIS];
  double a[KF_NBASIS];
};
__global__ void k_axpy_multi(size_t n, int k, AxpyList L, double *__restrict__ y, int fast)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc = y[i];
  for (int v = 0; v < k; v++) acc = fast ? fma(L.a[v], L.v[v][i], acc) : L.a[v] * L.v[v][i] + acc;
  y[i] = acc;
}

// w = a x + y (src/utils.c:89-107)
__global__ void k_waxpy(size_t n, double a, const double *__restrict__ x, const double *__restrict__ y,
                        double *__restrict__ w, int fast)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  w[i] = fast ? fma(a, x[i], y[i]) : a * x[i] + y[i];
}

// x *= 1/|x| with |x| on the device (src/utils.c:109-122)
__global__ void k_scale_inv(size_t n, const double *__restrict__ nrm, double *__restrict__ x)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] *= (1.0 / nrm[0]);
}

// J.v set-up, src/kernel.c:27-30: h = eps * qnorm; w = (h/|x|) x + q
__global__ void k_jv_shift(size_t n, const double *__restrict__ scal, const double *__restrict__ x,
                           const double *__restrict__ q, double *__restrict__ w, int fast)
{
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double h = JV_EPS * scal[S_QN];
  const double a = h / scal[S_XN];
  w[i] = fast ? fma(a, x[i], q[i]) : a * x[i] + q[i];
}

// k_jv_shift with the visit-order copy of w written alongside: node i's w in
// the mesh's order (coalesced, like x and q) and at its visit position
// rowof[i] in qv (the same arithmetic)
__global__ void k_jv_shift_visit(uint32_t N, const uint32_t *__restrict__ rowof, const double *__restrict__ scal,
                                 const double *__restrict__ x, const double *__restrict__ q, double *__restrict__ w,
                                 double4 *__restrict__ qv, int fast)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double h = JV_EPS * scal[S_QN];
  const double a = h / scal[S_XN];
  const double4 xx = reinterpret_cast<const double4 *>(x)[i], qq = reinterpret_cast<const double4 *>(q)[i];
  double4 o;
  o.x = fast ? fma(a, xx.x, qq.x) : a * xx.x + qq.x;
  o.y = fast ? fma(a, xx.y, qq.y) : a * xx.y + qq.y;
  o.z = fast ? fma(a, xx.z, qq.z) : a * xx.z + qq.z;
  o.w = fast ? fma(a, xx.w, qq.w) : a * xx.w + qq.w;
  reinterpret_cast<double4 *>(w)[i] = o;
  qv[rowof[i]] = o;
}

__global__ void k_set_h(double *scal)
{
  scal[S_H] = JV_EPS * scal[S_QN];
}

// src/forces.c:8-120 in the reference's order: per colour an OpenMP
// reduction from zero over the colour's faces in face order, each colour's sum
// then added to the running total.  One warp per colour: the lanes form 32
// faces' products at once, then every lane applies them to the running sums
// in face order (lift = (lift - dcx V) + dcy U, drag = (drag + dcx U) + dcy V,
// momn = (momn + (xmid - 1/4) dcy) - ymid dcx), so the arithmetic is the
// reference's.  The colour sums are added in colour order by one thread.
__global__ void __launch_bounds__(1024) k_forces(uint32_t ncol, const uint32_t *__restrict__ col,
                                                 const uint32_t *__restrict__ wf, const double4 *__restrict__ xyz,
                                                 const double4 *__restrict__ q, double U, double V,
                                                 double *__restrict__ out)
{
  __shared__ double part[3 * 1024];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (uint32_t c = warp; c < ncol; c += nw) {
    double l = 0.0, d = 0.0, m = 0.0;
    for (uint32_t base = col[c]; base < col[c + 1]; base += 32) {
      const uint32_t j = base + lane;
      double a1 = 0, a2 = 0, b1 = 0, b2 = 0, c1 = 0, c2 = 0;
      if (j < col[c + 1]) {
        const uint32_t a = wf[3 * j], b = wf[3 * j + 1], e = wf[3 * j + 2];
        const double4 pa = xyz[a], pb = xyz[b], pe = xyz[e];
        const double ax = pb.x - pa.x, ay = pb.y - pa.y, az = pb.z - pa.z;
        const double bx = pe.x - pa.x, by = pe.y - pa.y, bz = pe.z - pa.z;
        double xnorm = ay * bz; xnorm -= az * by; xnorm = -0.5 * xnorm;
        double ynorm = ax * bz; ynorm -= az * bx; ynorm = 0.5 * ynorm;
        const double press = (q[a].x + q[b].x + q[e].x) / 3.0;
        const double cp = 2.0 * (press - 1.0);
        const double dcx = cp * xnorm, dcy = cp * ynorm;
        const double xmid = pa.x + pb.x + pe.x;
        const double ymid = pa.y + pb.y + pe.y;
        a1 = dcx * V; a2 = dcy * U;
        b1 = dcx * U; b2 = dcy * V;
        c1 = (xmid - 0.25) * dcy; c2 = ymid * dcx;
      }
      const uint32_t cnt = min(32u, col[c + 1] - base);
      for (uint32_t k = 0; k < cnt; k++) {
        l = l - __shfl_sync(0xffffffffu, a1, k);
        l = l + __shfl_sync(0xffffffffu, a2, k);
        d = d + __shfl_sync(0xffffffffu, b1, k);
        d = d + __shfl_sync(0xffffffffu, b2, k);
        m = m + __shfl_sync(0xffffffffu, c1, k);
        m = m - __shfl_sync(0xffffffffu, c2, k);
      }
    }
    if (lane == 0 && c < 1024) {
      part[3 * c] = l;
      part[3 * c + 1] = d;
      part[3 * c + 2] = m;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double lift = 0.0, drag = 0.0, momn = 0.0;
    for (uint32_t c = 0; c < ncol && c < 1024; c++) {
      lift += part[3 * c];
      drag += part[3 * c + 1];
      momn += part[3 * c + 2];
    }
    out[0] = lift;
    out[1] = drag;
    out[2] = momn;
  }
}

// ------------------------------------------------------------------ helpers

unsigned forces_threads(uint32_t ncol) { return 32u * std::min<uint32_t>(std::max<uint32_t>(ncol, 1u), 32u); }

bool check_cuda(const char *what)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::string s = std::string(what) + ": " + cudaGetErrorString(e);
    kf_set_error(KFUN3D_ERR_CUDA, s.c_str());
    return false;
  }
  return true;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      std::string s_ = std::string(#call) + ": " + cudaGetErrorString(e_);        \
      kf_set_error(KFUN3D_ERR_CUDA, s_.c_str());                                   \
    }                                                                              \
  } while (0)

// Rows between the mesh numbering and the spatial ILU numbering:
// to_spatial: dst[rank[i]] = src[i]; from_spatial: dst[i] = src[rank[i]].
__global__ void k_rows_permute(uint32_t N, const uint32_t *__restrict__ rank, const double4 *__restrict__ src,
                               double4 *__restrict__ dst, int to_spatial)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t r = rank[i];
  if (to_spatial) dst[r] = src[i];
  else dst[i] = src[r];
}

// Kernel set of the current arithmetic mode.
struct Ops {
  bool fast;
  void gradient(DevMesh &m, const double *q) const { fast ? kf_fast::gradient(m, q) : kf_exact::gradient(m, q); }
  void residual(DevMesh &m, const double *q, double *r, int fo, double u, double v) const
  {
    fast ? kf_fast::residual(m, q, r, fo, u, v) : kf_exact::residual(m, q, r, fo, u, v);
  }
  void timestep(DevMesh &m, const double *q, double cfl) const
  {
    fast ? kf_fast::timestep(m, q, cfl) : kf_exact::timestep(m, q, cfl);
  }
  void fill(DevMesh &m, const double *q, double u, double v, int p) const
  {
    fast ? kf_fast::fill(m, q, u, v, p) : kf_exact::fill(m, q, u, v, p);
  }
  void ilu(DevMesh &m, int p) const { fast ? kf_fast::ilu(m, p) : kf_exact::ilu(m, p); }
  void sptrsv(DevMesh &m, const double *b, double *x, int p) const
  {
    if (m.ilu_active) {
      // spatial ILU(0): x = P^T (LU)^-1 P b, the permutations folded into the
      // packed sweeps where that schedule runs
      if (fast ? kf_fast::sptrsv_permuted(m, b, x, p) : kf_exact::sptrsv_permuted(m, b, x, p)) return;
      const unsigned nb = (m.N + 255) / 256;
      k_rows_permute<<<nb, 256, 0, m.stream>>>(m.N, m.ilu_rank, (const double4 *)b, (double4 *)m.pb, 1);
      fast ? kf_fast::sptrsv(m, m.pb, m.px, p) : kf_exact::sptrsv(m, m.pb, m.px, p);
      k_rows_permute<<<nb, 256, 0, m.stream>>>(m.N, m.ilu_rank, (const double4 *)m.px, (double4 *)x, 0);
      kf_count_launch(2);
      return;
    }
    fast ? kf_fast::sptrsv(m, b, x, p) : kf_exact::sptrsv(m, b, x, p);
  }
  void jv_combine(DevMesh &m, double *y, const double *r, const double *w, const double *q) const
  {
    fast ? kf_fast::jv_combine(m, y, r, w, q, m.scal, S_XN) : kf_exact::jv_combine(m, y, r, w, q, m.scal, S_XN);
  }
};

Ops ops() { return Ops{kf_mode() == KFUN3D_MODE_FAST}; }

// dot / norm into a device scalar: op 0 = sum, 1 = sqrt(sum), 2 = sqrt(1 + sqrt(sum))
void dev_reduce(DevMesh &m, const double *a, const double *b, double *out, int op, bool fast)
{
  const size_t n = 4 * (size_t)m.N;
  if (fast) {
    k_dot_partial<<<RED_BLOCKS, 256, 0, m.stream>>>(n, a, b, m.red);
    k_dot_final<<<1, 256, 0, m.stream>>>(m.red, RED_BLOCKS, out, op);
    kf_count_launch(2);
  } else {
    k_dot_seq<<<1, 32, 0, m.stream>>>(n, a, b, out, op);
    kf_count_launch();
  }
}

void fetch(DevMesh &m, int first, int count)
{
  CK(cudaMemcpyAsync(m.h_scal + first, m.scal + first, count * sizeof(double), cudaMemcpyDeviceToHost, m.stream));
  CK(cudaStreamSynchronize(m.stream));
}

// Residual of state q into r (gradient first unless first order).
void dev_residual(DevMesh &m, const Ops &o, const double *q, double *r)
{
  double u, v;
  kfun3d_get_freestream(&u, &v);
  const int fo = kf_first_order();
  if (!fo) o.gradient(m, q);
  o.residual(m, q, r, fo, u, v);
}

// iJacVec, src/kernel.c:24-45: y = (F(q + h x/|x|) - r + cdt (w - q)) |x| / h
void dev_jacvec(DevMesh &m, const Ops &o, const double *x, double *y)
{
  const size_t n = 4 * (size_t)m.N;
  dev_reduce(m, x, x, m.scal + S_XN, 1, o.fast);
  k_set_h<<<1, 1, 0, m.stream>>>(m.scal);
  if (m.visit) {
    // the shifted state and its visit-order copy in one pass
    k_jv_shift_visit<<<nblk(m.N, 256), 256, 0, m.stream>>>(m.N, m.rowof, m.scal, x, m.q, m.w, m.qv, o.fast);
    m.qv_of = m.w;
  } else {
    k_jv_shift<<<nblk(n, 256), 256, 0, m.stream>>>(n, m.scal, x, m.q, m.w, o.fast);
  }
  kf_count_launch(2);
  dev_residual(m, o, m.w, y);
  o.jv_combine(m, y, m.r, m.w, m.q);
}

void dev_axpy(DevMesh &m, double a, const double *x, double *y, bool fast)
{
  const size_t n = 4 * (size_t)m.N;
  k_axpy<<<nblk(n, 256), 256, 0, m.stream>>>(n, a, x, y, fast);
  kf_count_launch();
}

double *Vb(DevMesh &m, int k) { return m.V + (size_t)k * 4 * m.N; }

// y += sum over v < k of a[v] x[v], one launch (the sum of k dev_axpy calls,
// in their order)
void dev_axpy_multi(DevMesh &m, int k, const double *a, const double *const *x, double *y, bool fast)
{
  if (k <= 0) return;
  const size_t n = 4 * (size_t)m.N;
  AxpyList L{};
  for (int v = 0; v < k && v < KF_NBASIS; v++) { L.v[v] = x[v]; L.a[v] = a[v]; }
  k_axpy_multi<<<nblk(n, 256), 256, 0, m.stream>>>(n, std::min(k, (int)KF_NBASIS), L, y, fast);
  kf_count_launch();
}

void dev_normalize(DevMesh &m, double *x, double *nrm, bool fast)
{
  const size_t n = 4 * (size_t)m.N;
  dev_reduce(m, x, x, nrm, 1, fast);
  k_scale_inv<<<nblk(n, 256), 256, 0, m.stream>>>(n, nrm, x);
  kf_count_launch();
}

// Gram-Schmidt kernel: k_mgs_resident (default, w kept on chip) or
// k_mgs_coop (KFUN3D_MGS=coop); grid and shared memory fixed per mesh.
void mgs_coop_prepare(DevMesh &m)
{
  if (!m.mgs_grid) {
    int nsm = 0, per = 0, smax = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m.device));
    const char *env = getenv("KFUN3D_MGS");
    m.mgs_resident = !(env && strcmp(env, "coop") == 0);
    if (m.mgs_resident) {
      CK(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, m.device));
      const size_t n2 = 2 * (size_t)m.N, stride = (size_t)nsm * 512;
      const size_t per_thread = (n2 + stride - 1) / stride;
      const size_t room = (size_t)std::max(smax - 1024, 0) / (512 * sizeof(double2));
      m.mgs_ts = (int)std::min(room, per_thread > (size_t)KF_MGS_REG ? per_thread - KF_MGS_REG : (size_t)0);
      CK(cudaFuncSetAttribute((const void *)k_mgs_resident, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(m.mgs_ts * 512 * sizeof(double2))));
      m.mgs_grid = (unsigned)nsm;
    } else {
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_mgs_coop, 256, 0));
      m.mgs_grid = (unsigned)nsm * (unsigned)std::min(std::max(per, 1), 3);
    }
    CK(cudaMalloc(&m.part, 2 * m.mgs_grid * sizeof(double)));
  }
}

void mgs_coop(DevMesh &m, int k)
{
  mgs_coop_prepare(m);
  size_t n = 4 * (size_t)m.N;
  double *V = m.V, *h = m.scal, *part = m.part;
  unsigned *bar = m.bar + 2;
  int *err = m.status + 1;
  int ts = m.mgs_ts;
  void *args[] = {&n, &V, &k, &h, &part, &bar, &err, &ts};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(m.mgs_grid);
  cfg.blockDim = dim3(m.mgs_resident ? 512 : 256);
  cfg.dynamicSmemBytes = m.mgs_resident ? (size_t)m.mgs_ts * 512 * sizeof(double2) : 0;
  cfg.stream = m.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelExC(&cfg, m.mgs_resident ? (const void *)k_mgs_resident : (const void *)k_mgs_coop, args));
  kf_count_launch();
}

// One Arnoldi step k (src/kernel.c:123-141): V[k+1] = M^-1 J V[k],
// modified Gram-Schmidt against V[0..k], normalised; h in scal[0..k+1].
// Modified Gram-Schmidt of V[k+1] against V[0..k], normalised; h in scal[0..k+1].
void orthogonalize(DevMesh &m, const Ops &o, int k)
{
  const size_t n = 4 * (size_t)m.N;
  if (o.fast && (n % 2) == 0) {
    mgs_coop(m, k);
    return;
  }
  for (int v = 0; v <= k; v++) {
    dev_reduce(m, Vb(m, k + 1), Vb(m, v), m.scal + v, 0, o.fast);
    k_axpy_dev<<<nblk(n, 256), 256, 0, m.stream>>>(n, m.scal + v, -1.0, Vb(m, v), Vb(m, k + 1), o.fast);
    kf_count_launch();
  }
  dev_normalize(m, Vb(m, k + 1), m.scal + k + 1, o.fast);
}

void arnoldi_step(DevMesh &m, const Ops &o, int k, int prec)
{
  const size_t n = 4 * (size_t)m.N;
  dev_jacvec(m, o, Vb(m, k), m.t);
  o.sptrsv(m, m.t, Vb(m, k + 1), prec);
  if (o.fast && (n % 2) == 0) {
    mgs_coop(m, k);
    return;
  }
  for (int v = 0; v <= k; v++) {
    dev_reduce(m, Vb(m, k + 1), Vb(m, v), m.scal + v, 0, o.fast);
    k_axpy_dev<<<nblk(n, 256), 256, 0, m.stream>>>(n, m.scal + v, -1.0, Vb(m, v), Vb(m, k + 1), o.fast);
    kf_count_launch();
  }
  dev_normalize(m, Vb(m, k + 1), m.scal + k + 1, o.fast);
}

// Fast mode: the Arnoldi step and the read-back of its Hessenberg column as
// one CUDA graph per (precision, first order, k), captured on first use.
void arnoldi_step_graph(DevMesh &m, const Ops &o, int k, int prec)
{
  const int fo = kf_first_order();
  double u, v;
  kfun3d_get_freestream(&u, &v);
  if (m.graph_aoa != kfun3d_get_aoa() || m.graph_ilu != m.ilu_active) {
    for (auto &a : m.arnoldi)
      for (auto &b : a)
        for (auto &g : b)
          if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    m.graph_aoa = kfun3d_get_aoa();
    m.graph_ilu = m.ilu_active;
  }
  cudaGraphExec_t &ge = m.arnoldi[prec][fo][k];
  if (!ge) {
    mgs_coop_prepare(m);
    const unsigned long long before = kfun3d_launch_count();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(m.stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      arnoldi_step(m, o, k, prec);
      cudaMemcpyAsync(m.h_scal, m.scal, (k + 2) * sizeof(double), cudaMemcpyDeviceToHost, m.stream);
      e = cudaStreamEndCapture(m.stream, &graph);
    }
    const unsigned nodes = (unsigned)(kfun3d_launch_count() - before);
    kfun3d_reset_launch_count_by(nodes);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      // capture not available: run this solve without graphs
      cudaGetLastError();
      ge = nullptr;
      m.use_graphs = false;
      arnoldi_step(m, o, k, prec);
      fetch(m, 0, k + 2);
      return;
    }
    m.arnoldi_nodes[prec][fo][k] = nodes;
  }
  CK(cudaGraphLaunch(ge, m.stream));
  kf_count_launch(m.arnoldi_nodes[prec][fo][k]);
  CK(cudaStreamSynchronize(m.stream));
}

// Device status words: [0] pivot failure in ILU(0), [1] a bounded wait gave up.
int device_status(DevMesh &m)
{
  int st[2] = {0, 0};
  CK(cudaMemcpyAsync(st, m.status, 2 * sizeof(int), cudaMemcpyDeviceToHost, m.stream));
  CK(cudaStreamSynchronize(m.stream));
  if (st[0] || st[1]) {
    CK(cudaMemsetAsync(m.status, 0, 2 * sizeof(int), m.stream));
    // a wait that gave up may leave a grid barrier half-counted
    if (st[1] && m.bar) CK(cudaMemsetAsync(m.bar, 0, 8 * sizeof(unsigned), m.stream));
  }
  if (st[1]) return KFUN3D_ERR_TIMEOUT;
  return st[0];
}

}  // namespace

// ------------------------------------------------------------------ solve

extern "C" void kfun3d_default_params(kfun3d_solver_params *p)
{
  p->ts_max = 15;
  p->stop_ratio = 10000000.0;
  p->gmres_rtol = 0.01;
  p->gmres_restart = 30;
  p->gmres_max_it = 10000;
  p->cfl_init = 50.0;
  p->cfl_max = 100000.0;
}

// The device-resident solve of src/kernel.c:47-232 (parameters as data).
// The state stays on the device; the host keeps the small GMRES scalars and
// reads one column of the Hessenberg matrix per Arnoldi step.
static int solve_device(DevMesh &m, const GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_step *hist,
                        int max_hist, bool print)
{
  const Ops o = ops();
  const int prec = kf_precision();
  const size_t n = 4 * (size_t)m.N;
  const int restart = std::min(std::max(p->gmres_restart, 1), 30);
  double u, v;
  kfun3d_get_freestream(&u, &v);
  double ghh[KF_NBASIS * (KF_NBASIS + 1)] = {0};
  double cs[KF_NBASIS], sn[KF_NBASIS], rs[KF_NBASIS];
  double fnorm0 = 0.0, cfl = p->cfl_init;
  int nrec = 0, steps = 0;
  cudaEvent_t ev0, ev1;
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  for (int its = 0; its < p->ts_max; its++) {
    CK(cudaEventRecord(ev0, m.stream));
    dev_residual(m, o, m.q, m.r);
    dev_reduce(m, m.r, m.r, m.scal + S_FN, 1, o.fast);
    fetch(m, S_FN, 1);
    const double fnorm = m.h_scal[S_FN];
    if (!std::isfinite(fnorm)) {
      kf_set_error(KFUN3D_ERR_NONFINITE, "residual norm is not finite");
      steps = -1;
      break;
    }
    if (its == 0) fnorm0 = fnorm;
    else {
      double cfl0 = 1.1 * p->cfl_init * fnorm0;   // src/kernel.c:86-88
      cfl0 /= fnorm;
      cfl = (cfl0 < p->cfl_max) ? cfl0 : p->cfl_max;
    }
    o.timestep(m, m.q, cfl);
    o.fill(m, m.q, u, v, prec);
    dev_reduce(m, m.q, m.q, m.scal + S_QN, 2, o.fast);
    CK(cudaMemsetAsync(m.x, 0, n * sizeof(double), m.stream));
    o.ilu(m, prec);
    o.sptrsv(m, m.r, Vb(m, 0), prec);
    {
      const int st = device_status(m);
      if (st == KFUN3D_ERR_PIVOT) {
        kf_set_error(KFUN3D_ERR_PIVOT, "singular or non-finite pivot block in ILU(0)");
        steps = -1;
        break;
      }
      if (st == KFUN3D_ERR_TIMEOUT) {
        kf_set_error(KFUN3D_ERR_TIMEOUT, "a triangular-solve wait exceeded its bound");
        steps = -1;
        break;
      }
    }

    double tol = 0.0;
    unsigned int total = 0;
    bool done = false;
    while (total <= (unsigned)p->gmres_max_it) {     // src/kernel.c:107-196
      if (total > 0) {
        dev_jacvec(m, o, m.x, m.t);
        k_waxpy<<<nblk(n, 256), 256, 0, m.stream>>>(n, -1.0, m.t, m.r, m.w, o.fast);
        kf_count_launch();
        o.sptrsv(m, m.w, Vb(m, 0), prec);
      }
      dev_normalize(m, Vb(m, 0), m.scal + S_T0, o.fast);
      fetch(m, S_T0, 1);
      rs[0] = m.h_scal[S_T0];
      if (!std::isfinite(rs[0])) {
        kf_set_error(KFUN3D_ERR_NONFINITE, "preconditioned residual is not finite");
        done = false;
        steps = -1;
        break;
      }
      if (total == 0) tol = p->gmres_rtol * rs[0];
      int k = 0;
      while (k < restart) {
        if (o.fast && m.use_graphs) {
          arnoldi_step_graph(m, o, k, prec);
        } else {
          arnoldi_step(m, o, k, prec);
          fetch(m, 0, k + 2);
        }
        double *hh = ghh + k * (KF_NBASIS + 1);
        for (int i = 0; i <= k + 1; i++) hh[i] = m.h_scal[i];
        for (int i = 0; i < k; i++) {               // src/kernel.c:143-149
          const double tt = hh[i];
          hh[i] = cs[i] * hh[i] + sn[i] * hh[i + 1];
          hh[i + 1] = cs[i] * hh[i + 1] - sn[i] * tt;
        }
        const double tt = sqrt(hh[k] * hh[k] + hh[k + 1] * hh[k + 1]);
        const double c = hh[k] / tt, s = hh[k + 1] / tt;
        cs[k] = c;
        sn[k] = s;
        rs[k + 1] = -(s * rs[k]);
        rs[k] = c * rs[k];
        hh[k] = c * hh[k] + s * hh[k + 1];
        const double res = fabs(rs[k + 1]);
        k++;
        if (res <= tol) { done = true; break; }
        if (!std::isfinite(res)) break;
      }
      total += k;
      rs[k - 1] /= ghh[(k - 1) * (KF_NBASIS + 1) + (k - 1)];   // src/kernel.c:178-188
      for (int i = 1; i <= k - 1; i++) {
        const int mm = (k - 1) - i;
        double tt = rs[mm];
        for (int j = mm + 1; j <= k - 1; j++) tt -= ghh[j * (KF_NBASIS + 1) + mm] * rs[j];
        rs[mm] = tt / ghh[mm * (KF_NBASIS + 1) + mm];
      }
      {
        const double *vs[KF_NBASIS];
        for (int vv = 0; vv < k; vv++) vs[vv] = Vb(m, vv);
        dev_axpy_multi(m, k, rs, vs, m.x, o.fast);
      }
      if (print && k == restart) fun3d_printf(5, ">> GMRES: COMPLETED ONE CYCLE\n");
      if (done) break;
    }
    if (steps < 0) break;
    if (print) fun3d_printf(5, ">> GMRES: TOTAL ITERATIONS %d\n", total);
    dev_axpy(m, -1.0, m.x, m.q, o.fast);                           // src/kernel.c:200
    k_forces<<<1, forces_threads(m.ncol), 0, m.stream>>>(m.ncol, m.col, m.wf_nodes, m.xyz, (const double4 *)m.q, u, v, m.forces);
    kf_count_launch();
    CK(cudaEventRecord(ev1, m.stream));
    CK(cudaMemcpyAsync(m.h_scal + 48, m.forces, 3 * sizeof(double), cudaMemcpyDeviceToHost, m.stream));
    CK(cudaStreamSynchronize(m.stream));
    if (!check_cuda("solve")) { steps = -1; break; }
    if (device_status(m) == KFUN3D_ERR_TIMEOUT) {
      kf_set_error(KFUN3D_ERR_TIMEOUT, "a triangular-solve wait exceeded its bound");
      steps = -1;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    const double lift = m.h_scal[48], drag = m.h_scal[49], momn = m.h_scal[50];
    if (print) {
      printf("STEP: %d ", its);
      printf("CFL: %g ", cfl);
      printf("NORM: %g\n", fnorm);
      printf("LIFT: %g DRAG: %g MOMN: %g\n", lift, drag, momn);
    }
    if (hist && nrec < max_hist) {
      hist[nrec] = kfun3d_step{its, (int)total, cfl, fnorm, lift, drag, momn, ms * 1e-3};
      nrec++;
    }
    steps = its + 1;
    if (round(fnorm0 / fnorm) >= p->stop_ratio) break;   // src/kernel.c:214
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  return steps < 0 ? -1 : nrec;
}

// ------------------------------------------------------------------ flexible GMRES

namespace {

// Training pairs written by the ILU(0)-FGMRES solve: slot i holds x0 at
// x0 + i * 16N bytes (BF16 [N x 8]) and the target at tgt + i * 4N floats.
struct PairSink {
  int stride = 0;
  unsigned char *x0 = nullptr;
  float *tgt = nullptr;
  int cap = 0;
  int count = 0;
};

// Givens update of Hessenberg column k (host, src/kernel.c:143-160 arithmetic);
// returns |rs[k+1]|.
double givens(double *hh, double *cs, double *sn, double *rs, int k)
{
  for (int i = 0; i < k; i++) {
    const double tt = hh[i];
    hh[i] = cs[i] * hh[i] + sn[i] * hh[i + 1];
    hh[i + 1] = cs[i] * hh[i + 1] - sn[i] * tt;
  }
  const double tt = sqrt(hh[k] * hh[k] + hh[k + 1] * hh[k + 1]);
  const double c = hh[k] / tt, s = hh[k + 1] / tt;
  cs[k] = c;
  sn[k] = s;
  rs[k + 1] = -(s * rs[k]);
  rs[k] = c * rs[k];
  hh[k] = c * hh[k] + s * hh[k + 1];
  return fabs(rs[k + 1]);
}

// y[0..k-1] from the rotated Hessenberg columns and right-hand side
void back_substitute(const double *ghh, const double *rs, int k, double *y)
{
  for (int i = 0; i < k; i++) y[i] = rs[i];
  y[k - 1] /= ghh[(k - 1) * (KF_NBASIS + 1) + (k - 1)];
  for (int i = 1; i <= k - 1; i++) {
    const int mm = (k - 1) - i;
    double tt = y[mm];
    for (int j = mm + 1; j <= k - 1; j++) tt -= ghh[j * (KF_NBASIS + 1) + mm] * y[j];
    y[mm] = tt / ghh[mm * (KF_NBASIS + 1) + mm];
  }
}

double *Zb(DevMesh &m, int k) { return m.Z + (size_t)k * 4 * m.N; }

bool ensure_flex(DevMesh &m)
{
  const size_t n = 4 * (size_t)m.N;
  if (!m.Z && cudaMalloc(&m.Z, 30 * n * sizeof(double)) != cudaSuccess) return false;
  if (!m.qold && cudaMalloc(&m.qold, n * sizeof(double)) != cudaSuccess) return false;
  if (!m.fy && cudaMalloc(&m.fy, n * sizeof(double)) != cudaSuccess) return false;
  if (!m.fx && cudaMalloc(&m.fx, n * sizeof(double)) != cudaSuccess) return false;
  if (!m.pscr && cudaMalloc(&m.pscr, 264 * sizeof(double)) != cudaSuccess) return false;
  return true;
}

// Pair of the correction x (device, 4N): v = J x, y = ILU(0)^-1 v,
// x0 = BF16([y/s, q]), target = (x - y)/s.
void write_pair(DevMesh &m, const Ops &o, int prec, const double *x, PairSink &ps)
{
  if (ps.count >= ps.cap) return;
  dev_jacvec(m, o, x, m.t);
  o.sptrsv(m, m.t, m.fy, prec);
  kf_mpnn_pair_async(m.N, m.fy, m.q, x, ps.x0 + (size_t)ps.count * 16 * m.N,
                     ps.tgt + (size_t)ps.count * 4 * m.N, m.pscr, m.stream);
  ps.count++;
}

}  // namespace

// The pseudo-transient Newton loop of src/kernel.c:47-232 with its linear
// solves done by flexible GMRES on the reference's left-preconditioned
// system: Arnoldi on ILU(0)^-1 J, residual measured as |ILU(0)^-1 (b - J x)|
// exactly as the reference does, and a right preconditioner allowed to
// change from one iteration to the next,
//   z_k = N_k(v_k),  w = ILU(0)^-1 J z_k orthogonalised against v_0..v_k,
//   x = Z y after each cycle.
// N_k is the identity -- the reference's GMRES, iteration for iteration -- or
// the network's correction v + s N([v/s, q]), which maps an ILU(0)-
// preconditioned residual to an approximation of the correction x with
// ILU(0)^-1 J x = v.  The network is a guest: each linear solve starts with
// both candidate first directions and keeps the network only if its image
// under ILU(0)^-1 J lies closer to v0 (one extra product per Newton step);
// it keeps its place only while the residual falls at least half as fast
// (per iteration, in log) as in the previous step's solve, and for at most
// 1.5x that solve's iterations, after which the solve goes on without it;
// Newton step 0 runs without it to set the pace; three fallbacks in a row
// switch it off for good; and an update after which
// the FP64 nonlinear residual is non-finite or grows tenfold is undone and
// redone without it.
static int solve_flexible(DevMesh &m, const GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_mpnn *net,
                          PairSink *ps, kfun3d_step *hist, int max_hist, kfun3d_flex_stats *st)
{
  const Ops o = ops();
  const int prec = kf_precision();
  const size_t n = 4 * (size_t)m.N;
  const int restart = std::min(std::max(p->gmres_restart, 1), 30);
  double u, v;
  kfun3d_get_freestream(&u, &v);
  kfun3d_flex_stats S{};
  if (!ensure_flex(m)) {
    kf_set_error(KFUN3D_ERR_CUDA, "flexible solve: out of device memory");
    return -1;
  }
  if (net) {
    if (!m.mgraph) m.mgraph = kfun3d_mpnn_graph_create(g);
    if (!m.mgraph || kf_mpnn_prepare(net, m.mgraph) != KFUN3D_OK) return -1;
  }
  double ghh[KF_NBASIS * (KF_NBASIS + 1)] = {0};
  double cs[KF_NBASIS], sn[KF_NBASIS], rs[KF_NBASIS], yk[KF_NBASIS];
  double fnorm0 = 0.0, fnorm_prev = 0.0, cfl = p->cfl_init;
  bool use_net = net != nullptr, last_used_net = false;
  int misses = 0, prev_total = -1;
  double rate_prev = 0.0;   // log residual reduction per iteration of the previous linear solve
  int nrec = 0, steps = 0;
  cudaEvent_t ev0, ev1, es0, es1;
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  CK(cudaEventCreate(&es0));
  CK(cudaEventCreate(&es1));
  CK(cudaEventRecord(es0, m.stream));
  for (int its = 0; its < p->ts_max; its++) {
    CK(cudaEventRecord(ev0, m.stream));
    dev_residual(m, o, m.q, m.r);
    dev_reduce(m, m.r, m.r, m.scal + S_FN, 1, o.fast);
    fetch(m, S_FN, 1);
    double fnorm = m.h_scal[S_FN];
    if (last_used_net && (!std::isfinite(fnorm) || fnorm > 10.0 * fnorm_prev)) {
      // the nonlinear residual rejects the learned update: undo it, go on without the network
      CK(cudaMemcpyAsync(m.q, m.qold, n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
      dev_residual(m, o, m.q, m.r);
      dev_reduce(m, m.r, m.r, m.scal + S_FN, 1, o.fast);
      fetch(m, S_FN, 1);
      fnorm = m.h_scal[S_FN];
      use_net = false;
      S.disabled = 1;
      S.rejected_steps++;
    }
    if (!std::isfinite(fnorm)) {
      kf_set_error(KFUN3D_ERR_NONFINITE, "residual norm is not finite");
      steps = -1;
      break;
    }
    if (its == 0) fnorm0 = fnorm;
    else {
      double cfl0 = 1.1 * p->cfl_init * fnorm0;   // src/kernel.c:86-88
      cfl0 /= fnorm;
      cfl = (cfl0 < p->cfl_max) ? cfl0 : p->cfl_max;
    }
    fnorm_prev = fnorm;
    o.timestep(m, m.q, cfl);
    o.fill(m, m.q, u, v, prec);
    dev_reduce(m, m.q, m.q, m.scal + S_QN, 2, o.fast);
    CK(cudaMemsetAsync(m.x, 0, n * sizeof(double), m.stream));
    o.ilu(m, prec);
    o.sptrsv(m, m.r, Vb(m, 0), prec);                            // src/kernel.c:103
    {
      const int sd = device_status(m);
      if (sd == KFUN3D_ERR_PIVOT) {
        kf_set_error(KFUN3D_ERR_PIVOT, "singular or non-finite pivot block in ILU(0)");
        steps = -1;
        break;
      }
    }
    // Newton step 0 runs without the network: it measures the rate the
    // network then has to beat
    bool step_net = use_net && prev_total > 0;
    // iterations the network may use in this solve: 1.5 x the previous step's
    const int budget = prev_total > 0 ? (3 * prev_total + 1) / 2 : 2 * restart;
    double rs_first = 0.0, res_last = 0.0;
    bool usez[KF_NBASIS] = {false};
    double tol = 0.0;
    unsigned int total = 0;
    bool done = false, failed = false;
    for (int cycle = 0; total <= (unsigned)p->gmres_max_it; cycle++) {   // src/kernel.c:107-196
      if (total > 0) {
        dev_jacvec(m, o, m.x, m.t);
        k_waxpy<<<nblk(n, 256), 256, 0, m.stream>>>(n, -1.0, m.t, m.r, m.w, o.fast);
        kf_count_launch();
        o.sptrsv(m, m.w, Vb(m, 0), prec);
      }
      dev_normalize(m, Vb(m, 0), m.scal + S_T0, o.fast);
      fetch(m, S_T0, 1);
      rs[0] = m.h_scal[S_T0];
      if (!std::isfinite(rs[0])) { failed = true; break; }
      if (total == 0) {
        tol = p->gmres_rtol * rs[0];
        rs_first = rs[0];
        if (rs[0] == 0.0) { done = true; break; }
      }
      int k = 0;
      while (k < restart) {
        bool stepped = false;   // the step ran as a captured graph (its Gram-Schmidt and read-back too)
        if (step_net && cycle == 0 && k == 0) {
          // the network earns this solve on its first direction: both
          // candidates, z = v0 and the network's z, are mapped by
          // ILU(0)^-1 J; the one whose image comes closer to v0
          // (1 - (v0.w)^2 / w.w, the least-squares residual along w) is kept
          if (kf_mpnn_apply_async(net, m.mgraph, Vb(m, 0), m.q, Zb(m, 0), m.stream) != KFUN3D_OK) {
            failed = true;
            break;
          }
          dev_jacvec(m, o, Zb(m, 0), m.t);
          o.sptrsv(m, m.t, Vb(m, 1), prec);
          dev_jacvec(m, o, Vb(m, 0), m.t);
          o.sptrsv(m, m.t, m.fy, prec);
          dev_reduce(m, Vb(m, 0), Vb(m, 1), m.scal + S_CMP, 0, o.fast);
          dev_reduce(m, Vb(m, 1), Vb(m, 1), m.scal + S_CMP + 1, 0, o.fast);
          dev_reduce(m, Vb(m, 0), m.fy, m.scal + S_CMP + 2, 0, o.fast);
          dev_reduce(m, m.fy, m.fy, m.scal + S_CMP + 3, 0, o.fast);
          fetch(m, S_CMP, 4);
          const double *c = m.h_scal + S_CMP;
          const double rho_net = 1.0 - c[0] * c[0] / c[1], rho_plain = 1.0 - c[2] * c[2] / c[3];
          if (!(rho_net < rho_plain)) {
            CK(cudaMemcpyAsync(Vb(m, 1), m.fy, n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
            step_net = false;
            usez[0] = false;
            S.fallback_solves++;
            if (++misses >= 3) {   // three solves in a row: off for the rest of the solve
              use_net = false;
              S.disabled = 1;
            }
          } else {
            misses = 0;
            usez[0] = true;
            S.learned_its++;
          }
        } else if (step_net) {
          if (kf_mpnn_apply_async(net, m.mgraph, Vb(m, k), m.q, Zb(m, k), m.stream) != KFUN3D_OK) {
            failed = true;
            break;
          }
          dev_jacvec(m, o, Zb(m, k), m.t);
          o.sptrsv(m, m.t, Vb(m, k + 1), prec);
          usez[k] = true;
          S.learned_its++;
        } else {
          const bool pair = ps && ps->stride < 0 && (k % -ps->stride) == 0 && ps->count < ps->cap;
          usez[k] = false;
          if (o.fast && m.use_graphs && !pair) {
            // without the network the step is the plain Arnoldi step: its
            // captured graph (Gram-Schmidt and the column's read-back included)
            arnoldi_step_graph(m, o, k, prec);
            stepped = true;
          } else {
            dev_jacvec(m, o, Vb(m, k), m.t);                             // src/kernel.c:123-130
            o.sptrsv(m, m.t, Vb(m, k + 1), prec);
            if (pair) {
              // basis pair: x = v_k, y = ILU(0)^-1 J v_k (before Gram-Schmidt)
              kf_mpnn_pair_async(m.N, Vb(m, k + 1), m.q, Vb(m, k), ps->x0 + (size_t)ps->count * 16 * m.N,
                                 ps->tgt + (size_t)ps->count * 4 * m.N, m.pscr, m.stream);
              ps->count++;
            }
          }
        }
        if (!stepped) {
          orthogonalize(m, o, k);
          fetch(m, 0, k + 2);
        }
        double *hh = ghh + k * (KF_NBASIS + 1);
        for (int i = 0; i <= k + 1; i++) hh[i] = m.h_scal[i];
        const double res = givens(hh, cs, sn, rs, k);
        k++;
        if (res <= tol) { done = true; break; }
        if (!std::isfinite(res)) { failed = true; break; }
        res_last = res;
        // the network must keep at least half the previous solve's rate (log
        // residual per iteration) and stay within its iteration budget
        if (step_net && (((int)total + k >= 6 && rate_prev < 0.0 &&
                          log(res / rs_first) > 0.5 * ((int)total + k) * rate_prev) ||
                         (int)total + k > budget)) {
          step_net = false;
          S.fallback_solves++;
          if (++misses >= 3) {
            use_net = false;
            S.disabled = 1;
          }
        }
        if (ps && ps->stride > 0 && cycle == 0 && k < restart && (k % ps->stride) == 0 && ps->count < ps->cap) {
          back_substitute(ghh, rs, k, yk);
          CK(cudaMemsetAsync(m.fx, 0, n * sizeof(double), m.stream));
          {
            const double *vs[KF_NBASIS];
            for (int vv = 0; vv < k; vv++) vs[vv] = Vb(m, vv);
            dev_axpy_multi(m, k, yk, vs, m.fx, o.fast);
          }
          write_pair(m, o, prec, m.fx, *ps);
        }
      }
      if (failed || k == 0) break;
      total += k;
      back_substitute(ghh, rs, k, yk);                                  // src/kernel.c:178-190
      {
        const double *vs[KF_NBASIS];
        for (int vv = 0; vv < k; vv++) vs[vv] = usez[vv] ? Zb(m, vv) : Vb(m, vv);
        dev_axpy_multi(m, k, yk, vs, m.x, o.fast);
      }
      if (done) break;
    }
    if (failed || !done) {
      if (!failed && total > (unsigned)p->gmres_max_it) {
        // iteration limit: keep the iterate, as the reference does
      } else {
        kf_set_error(KFUN3D_ERR_NONFINITE, "flexible GMRES: non-finite residual");
        steps = -1;
        break;
      }
    }
    if (net && kf_mpnn_status(net, m.stream) != KFUN3D_OK) { steps = -1; break; }
    S.gmres_its += (int)total;
    prev_total = (int)total;
    if (total > 0 && rs_first > 0.0 && res_last > 0.0) rate_prev = log(res_last / rs_first) / total;
    if (ps && ps->count < ps->cap) write_pair(m, o, prec, m.x, *ps);
    if (step_net) CK(cudaMemcpyAsync(m.qold, m.q, n * sizeof(double), cudaMemcpyDeviceToDevice, m.stream));
    last_used_net = step_net;
    dev_axpy(m, -1.0, m.x, m.q, o.fast);                           // src/kernel.c:200
    k_forces<<<1, forces_threads(m.ncol), 0, m.stream>>>(m.ncol, m.col, m.wf_nodes, m.xyz, (const double4 *)m.q, u, v,
                                                         m.forces);
    kf_count_launch();
    CK(cudaEventRecord(ev1, m.stream));
    CK(cudaMemcpyAsync(m.h_scal + 48, m.forces, 3 * sizeof(double), cudaMemcpyDeviceToHost, m.stream));
    CK(cudaStreamSynchronize(m.stream));
    if (!check_cuda("flexible solve")) { steps = -1; break; }
    if (device_status(m) == KFUN3D_ERR_TIMEOUT) {
      kf_set_error(KFUN3D_ERR_TIMEOUT, "a triangular-solve wait exceeded its bound");
      steps = -1;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (hist && nrec < max_hist) {
      hist[nrec] = kfun3d_step{its, (int)total, cfl, fnorm, m.h_scal[48], m.h_scal[49], m.h_scal[50], ms * 1e-3};
      nrec++;
    }
    steps = its + 1;
    if (round(fnorm0 / fnorm) >= p->stop_ratio) break;   // src/kernel.c:214
  }
  CK(cudaEventRecord(es1, m.stream));
  CK(cudaEventSynchronize(es1));
  float tot = 0.f;
  cudaEventElapsedTime(&tot, es0, es1);
  S.newton_steps = steps < 0 ? 0 : steps;
  S.seconds = tot * 1e-3;
  S.pairs = ps ? ps->count : 0;
  if (st) *st = S;
  for (cudaEvent_t e : {ev0, ev1, es0, es1}) cudaEventDestroy(e);
  return steps < 0 ? -1 : nrec;
}

// ------------------------------------------------------------------ entry points

namespace {

DevMesh *dev_or_fail(const GEOMETRY *g)
{
  DevMesh *m = kf_device(g);
  if (m && kf_ilu_select(*m, g, kf_ilu_order()) != KFUN3D_OK) return nullptr;
  if (m && kf_schwarz_select(*m, g, kf_schwarz()) != KFUN3D_OK) return nullptr;
  return m;
}

void h2d(DevMesh &m, double *dst, const double *src, size_t n)
{
  CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, m.stream));
}

void d2h(DevMesh &m, double *dst, const double *src, size_t n)
{
  CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, m.stream));
}

bool finish(DevMesh &m, const char *what)
{
  CK(cudaStreamSynchronize(m.stream));
  return check_cuda(what);
}

}  // namespace

extern "C" void ComputeFlux(const GEOMETRY *g, const double *q, GRADIENT *grad, double *r)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return;
  const size_t n = 4 * (size_t)m->N;
  h2d(*m, m->w, q, n);
  const Ops o = ops();
  if (kf_first_order()) {
    CK(cudaMemsetAsync(m->gx, 0, n * sizeof(double), m->stream));
    CK(cudaMemsetAsync(m->gy, 0, n * sizeof(double), m->stream));
    CK(cudaMemsetAsync(m->gz, 0, n * sizeof(double), m->stream));
  }
  dev_residual(*m, o, m->w, m->t);
  if (!kf_first_order()) {
    if (o.fast) kf_fast::gradient_to_mesh_order(*m);
    else kf_exact::gradient_to_mesh_order(*m);
  }
  d2h(*m, grad->x0, m->gx, n);
  d2h(*m, grad->x1, m->gy, n);
  d2h(*m, grad->x2, m->gz, n);
  d2h(*m, r, m->t, n);
  finish(*m, "ComputeFlux");
}

extern "C" void ComputeTimeStep(const double cfl, GEOMETRY *g)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return;
  h2d(*m, m->q, g->q->q, 4 * (size_t)m->N);
  ops().timestep(*m, m->q, cfl);
  d2h(*m, g->n->cdt, m->cdt, m->N);
  finish(*m, "ComputeTimeStep");
}

extern "C" void ComputeA(GEOMETRY *g)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return;
  double u, v;
  kfun3d_get_freestream(&u, &v);
  h2d(*m, m->q, g->q->q, 4 * (size_t)m->N);
  h2d(*m, m->cdt, g->n->cdt, m->N);
  ops().fill(*m, m->q, u, v, kf_precision());
  m->a_valid = true;
  m->factored = false;
  finish(*m, "ComputeA");
}

extern "C" void ComputeNumericalILU(GEOMETRY *g)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return;
  ops().ilu(*m, kf_precision());
  m->factored = true;
  m->factor_precision = kf_precision();
  if (!finish(*m, "ComputeNumericalILU")) return;
  if (device_status(*m) == KFUN3D_ERR_PIVOT)
    kf_set_error(KFUN3D_ERR_PIVOT, "singular or non-finite pivot block in ILU(0)");
}

extern "C" void ComputeSparseTriangularSolve(const GEOMETRY *g, const double *b, double *x)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return;
  const size_t n = 4 * (size_t)m->N;
  h2d(*m, m->rhs, b, n);
  ops().sptrsv(*m, m->rhs, m->t, kf_precision());
  d2h(*m, x, m->t, n);
  if (!finish(*m, "ComputeSparseTriangularSolve")) return;
  if (device_status(*m) == KFUN3D_ERR_TIMEOUT)
    kf_set_error(KFUN3D_ERR_TIMEOUT, "a triangular-solve wait exceeded its bound");
}

extern "C" void ComputeForces(const GEOMETRY *g, double *forces)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return;
  double u, v;
  kfun3d_get_freestream(&u, &v);
  h2d(*m, m->q, g->q->q, 4 * (size_t)m->N);
  k_forces<<<1, forces_threads(m->ncol), 0, m->stream>>>(m->ncol, m->col, m->wf_nodes, m->xyz, (const double4 *)m->q, u, v, m->forces);
  kf_count_launch();
  d2h(*m, forces, m->forces, 3);
  finish(*m, "ComputeForces");
}

// ---- BLAS-1 on host arrays (inc/utils.h): staged through a device buffer

namespace {

struct Scratch {
  double *buf = nullptr;
  size_t cap = 0;
  cudaStream_t stream = nullptr;
  double *ensure(size_t n)
  {
    if (!stream) CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    if (n > cap) {
      if (buf) cudaFree(buf);
      cap = std::max(n, (size_t)1 << 16);
      CK(cudaMalloc(&buf, (3 * cap + 4096) * sizeof(double)));
    }
    return buf;
  }
} g_scr;

double blas_reduce(size_t sz, const double *hv, int op)
{
  double *d = g_scr.ensure(sz);
  if (!d) return NAN;
  cudaStream_t s = g_scr.stream;
  double *red = d + 3 * g_scr.cap, out = 0.0;
  CK(cudaMemcpyAsync(d, hv, sz * sizeof(double), cudaMemcpyHostToDevice, s));
  if (kf_mode() == KFUN3D_MODE_FAST) {
    k_dot_partial<<<RED_BLOCKS, 256, 0, s>>>(sz, d, d, red + 8);
    k_dot_final<<<1, 256, 0, s>>>(red + 8, RED_BLOCKS, red, op);
    kf_count_launch(2);
  } else {
    k_dot_seq<<<1, 32, 0, s>>>(sz, d, d, red, op);
    kf_count_launch();
  }
  CK(cudaMemcpyAsync(&out, red, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  check_cuda("Compute2ndNorm");
  return out;
}

}  // namespace

extern "C" double Compute2ndNorm(const size_t sz, const double *v) { return blas_reduce(sz, v, 1); }

extern "C" void ComputeAXPY(const size_t sz, const double a, const double *x, double *y)
{
  double *d = g_scr.ensure(sz);
  if (!d) return;
  cudaStream_t s = g_scr.stream;
  CK(cudaMemcpyAsync(d, x, sz * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d + g_scr.cap, y, sz * sizeof(double), cudaMemcpyHostToDevice, s));
  k_axpy<<<nblk(sz, 256), 256, 0, s>>>(sz, a, d, d + g_scr.cap, kf_mode() == KFUN3D_MODE_FAST);
  kf_count_launch();
  CK(cudaMemcpyAsync(y, d + g_scr.cap, sz * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  check_cuda("ComputeAXPY");
}

extern "C" void ComputeNewAXPY(const size_t sz, const double a, const double *x, const double *y, double *w)
{
  double *d = g_scr.ensure(sz);
  if (!d) return;
  cudaStream_t s = g_scr.stream;
  CK(cudaMemcpyAsync(d, x, sz * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d + g_scr.cap, y, sz * sizeof(double), cudaMemcpyHostToDevice, s));
  k_waxpy<<<nblk(sz, 256), 256, 0, s>>>(sz, a, d, d + g_scr.cap, d + 2 * g_scr.cap, kf_mode() == KFUN3D_MODE_FAST);
  kf_count_launch();
  CK(cudaMemcpyAsync(w, d + 2 * g_scr.cap, sz * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  check_cuda("ComputeNewAXPY");
}

extern "C" double Normalize(const size_t sz, double *x)
{
  double *d = g_scr.ensure(sz);
  if (!d) return NAN;
  cudaStream_t s = g_scr.stream;
  double *red = d + 3 * g_scr.cap, nrm = 0.0;
  CK(cudaMemcpyAsync(d, x, sz * sizeof(double), cudaMemcpyHostToDevice, s));
  if (kf_mode() == KFUN3D_MODE_FAST) {
    k_dot_partial<<<RED_BLOCKS, 256, 0, s>>>(sz, d, d, red + 8);
    k_dot_final<<<1, 256, 0, s>>>(red + 8, RED_BLOCKS, red, 1);
    kf_count_launch(2);
  } else {
    k_dot_seq<<<1, 32, 0, s>>>(sz, d, d, red, 1);
    kf_count_launch();
  }
  k_scale_inv<<<nblk(sz, 256), 256, 0, s>>>(sz, red, d);
  kf_count_launch();
  CK(cudaMemcpyAsync(x, d, sz * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&nrm, red, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  check_cuda("Normalize");
  return nrm;
}

// ---- whole solves

extern "C" int kfun3d_solve(GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_step *hist, int max_hist)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return -1;
  kfun3d_solver_params def;
  if (!p) { kfun3d_default_params(&def); p = &def; }
  h2d(*m, m->q, g->q->q, 4 * (size_t)m->N);
  CK(cudaMemsetAsync(m->lslot, 0, (16 * (size_t)m->nlower + 16) * sizeof(double), m->stream));
  const int n = solve_device(*m, g, p, hist, max_hist, false);
  d2h(*m, g->q->q, m->q, 4 * (size_t)m->N);
  d2h(*m, g->n->cdt, m->cdt, m->N);
  finish(*m, "kfun3d_solve");
  return n;
}

extern "C" void Kernel(GEOMETRY *g)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return;
  kfun3d_solver_params p;
  kfun3d_default_params(&p);
  h2d(*m, m->q, g->q->q, 4 * (size_t)m->N);
  solve_device(*m, g, &p, nullptr, 0, g_kf_verbose != 0);
  d2h(*m, g->q->q, m->q, 4 * (size_t)m->N);
  d2h(*m, g->n->cdt, m->cdt, m->N);
  finish(*m, "Kernel");
}

// ---- device-resident timing

extern "C" double kfun3d_time_kernel(GEOMETRY *g, int which, int reps)
{
  DevMesh *m = dev_or_fail(g);
  if (!m || reps < 1) return -1.0;
  const Ops o = ops();
  const int prec = kf_precision();
  const size_t n = 4 * (size_t)m->N;
  double u, v;
  kfun3d_get_freestream(&u, &v);
  h2d(*m, m->q, g->q->q, n);
  // a consistent state for the preconditioner and the Krylov vectors
  dev_residual(*m, o, m->q, m->r);
  o.timestep(*m, m->q, 50.0);
  o.fill(*m, m->q, u, v, prec);
  o.ilu(*m, prec);
  dev_reduce(*m, m->q, m->q, m->scal + S_QN, 2, o.fast);
  for (int k = 0; k <= 16; k++) {
    CK(cudaMemcpyAsync(Vb(*m, k), m->r, n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
    dev_normalize(*m, Vb(*m, k), m->scal + S_T0, o.fast);
  }
  auto run = [&]() {
    switch (which) {
      case 0: dev_residual(*m, o, m->q, m->r); break;
      case 1: o.timestep(*m, m->q, 50.0); break;
      case 2: o.fill(*m, m->q, u, v, prec); break;
      case 3: o.fill(*m, m->q, u, v, prec); o.ilu(*m, prec); break;
      case 4: o.sptrsv(*m, m->r, m->t, prec); break;
      case 5: arnoldi_step(*m, o, 15, prec); break;
      case 6:
        if (o.fast) {
          mgs_coop(*m, 15);
          break;
        }
        for (int vv = 0; vv <= 15; vv++) {
          dev_reduce(*m, Vb(*m, 16), Vb(*m, vv), m->scal + vv, 0, o.fast);
          k_axpy_dev<<<nblk(n, 256), 256, 0, m->stream>>>(n, m->scal + vv, -1.0, Vb(*m, vv), Vb(*m, 16), o.fast);
          kf_count_launch();
        }
        dev_normalize(*m, Vb(*m, 16), m->scal + 16, o.fast);
        break;
      case 7: o.gradient(*m, m->q); break;
      case 8: o.residual(*m, m->q, m->r, kf_first_order(), u, v); break;
      default: break;
    }
  };
  for (int i = 0; i < 2; i++) run();
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, m->stream));
  for (int i = 0; i < reps; i++) run();
  CK(cudaEventRecord(e1, m->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!finish(*m, "kfun3d_time_kernel")) return -1.0;
  return (double)ms / reps;
}

extern "C" int kfun3d_check_bounded_wait(void)
{
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    kf_set_error(KFUN3D_ERR_NO_DEVICE, "no CUDA device");
    return KFUN3D_ERR_NO_DEVICE;
  }
  return kf_fast::bounded_wait_check(0);
}

extern "C" long kfun3d_matrix_read(const GEOMETRY *g, unsigned int *ia, unsigned int *ja, double *blocks)
{
  MatrixHandle *h = kf_handle(g);
  if (!h) {
    kf_set_error(KFUN3D_ERR_ARG, "GEOMETRY::matrix is not a kfun3d_b200 handle");
    return -1;
  }
  const HostPattern &p = kf_host_pattern(h);
  if (ia) memcpy(ia, p.ia.data(), p.ia.size() * sizeof(unsigned int));
  if (ja) memcpy(ja, p.ja.data(), p.ja.size() * sizeof(unsigned int));
  if (blocks) {
    DevMesh *m = dev_or_fail(g);
    if (!m) return -1;
    if (m->ilu_active) {
      kf_set_error(KFUN3D_ERR_ARG, "kfun3d_matrix_read: the blocks are stored in the spatial ILU order; "
                                   "select the mesh order (kfun3d_set_ilu_order(0)) first");
      return -1;
    }
    const size_t nv = 16 * p.nnz;
    if (kf_precision() == 0) {
      d2h(*m, blocks, m->A, nv);
    } else {
      std::vector<float> tmp(nv);
      CK(cudaMemcpyAsync(tmp.data(), m->Af, nv * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
      CK(cudaStreamSynchronize(m->stream));
      for (size_t i = 0; i < nv; i++) blocks[i] = tmp[i];
    }
    if (!finish(*m, "kfun3d_matrix_read")) return -1;
  }
  return (long)p.nnz;
}

extern "C" double kfun3d_time_solve(GEOMETRY *g, const kfun3d_solver_params *p, int reps, kfun3d_step *hist,
                                    int max_hist, int *nsteps)
{
  DevMesh *m = dev_or_fail(g);
  if (!m || reps < 1) return -1.0;
  kfun3d_solver_params def;
  if (!p) { kfun3d_default_params(&def); p = &def; }
  const size_t n = 4 * (size_t)m->N;
  double *q0 = nullptr;
  CK(cudaMalloc(&q0, n * sizeof(double)));
  if (!q0) return -1.0;
  h2d(*m, q0, g->q->q, n);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double total = 0.0;
  int ns = 0;
  for (int r = 0; r < reps; r++) {
    CK(cudaMemcpyAsync(m->q, q0, n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
    CK(cudaMemsetAsync(m->lslot, 0, (16 * (size_t)m->nlower + 16) * sizeof(double), m->stream));
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaEventRecord(e0, m->stream));
    ns = solve_device(*m, g, p, hist, max_hist, false);
    CK(cudaEventRecord(e1, m->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    total += ms * 1e-3;
    if (ns < 0) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(q0);
  if (nsteps) *nsteps = ns;
  if (!finish(*m, "kfun3d_time_solve") || ns < 0) return -1.0;
  return total / reps;
}

// ---- flexible GMRES and the learned preconditioner

extern "C" int kfun3d_solve_flexible(GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_mpnn *net,
                                     kfun3d_step *hist, int max_hist, kfun3d_flex_stats *stats)
{
  DevMesh *m = dev_or_fail(g);
  if (!m) return -1;
  kfun3d_solver_params def;
  if (!p) { kfun3d_default_params(&def); p = &def; }
  h2d(*m, m->q, g->q->q, 4 * (size_t)m->N);
  const int n = solve_flexible(*m, g, p, net, nullptr, hist, max_hist, stats);
  d2h(*m, g->q->q, m->q, 4 * (size_t)m->N);
  d2h(*m, g->n->cdt, m->cdt, m->N);
  if (!finish(*m, "kfun3d_solve_flexible")) return -1;
  return n;
}

extern "C" int kfun3d_collect_pairs(GEOMETRY *g, const kfun3d_solver_params *p, int stride, void *d_x0,
                                    float *d_target, int cap, kfun3d_flex_stats *stats)
{
  if (!d_x0 || !d_target || cap < 0) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_collect_pairs: bad arguments");
    return -1;
  }
  DevMesh *m = dev_or_fail(g);
  if (!m) return -1;
  kfun3d_solver_params def;
  if (!p) { kfun3d_default_params(&def); p = &def; }
  PairSink ps;
  ps.stride = stride;
  ps.x0 = (unsigned char *)d_x0;
  ps.tgt = d_target;
  ps.cap = cap;
  h2d(*m, m->q, g->q->q, 4 * (size_t)m->N);
  const int n = solve_flexible(*m, g, p, nullptr, &ps, nullptr, 0, stats);
  d2h(*m, g->q->q, m->q, 4 * (size_t)m->N);
  d2h(*m, g->n->cdt, m->cdt, m->N);
  if (!finish(*m, "kfun3d_collect_pairs")) return -1;
  return n < 0 ? -1 : ps.count;
}

extern "C" double kfun3d_time_solve_flexible(GEOMETRY *g, const kfun3d_solver_params *p, kfun3d_mpnn *net,
                                             int reps, kfun3d_step *hist, int max_hist, int *nsteps,
                                             kfun3d_flex_stats *stats)
{
  DevMesh *m = dev_or_fail(g);
  if (!m || reps < 1) return -1.0;
  kfun3d_solver_params def;
  if (!p) { kfun3d_default_params(&def); p = &def; }
  const size_t n = 4 * (size_t)m->N;
  double *q0 = nullptr;
  CK(cudaMalloc(&q0, n * sizeof(double)));
  if (!q0) return -1.0;
  h2d(*m, q0, g->q->q, n);
  double total = 0.0;
  int ns = 0;
  for (int r = 0; r < reps; r++) {
    CK(cudaMemcpyAsync(m->q, q0, n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    kfun3d_flex_stats st{};
    ns = solve_flexible(*m, g, p, net, nullptr, hist, max_hist, &st);
    total += st.seconds;
    if (stats) *stats = st;
    if (ns < 0) break;
  }
  cudaFree(q0);
  if (nsteps) *nsteps = ns;
  if (!finish(*m, "kfun3d_time_solve_flexible") || ns < 0) return -1.0;
  return total / reps;
}

extern "C" double kfun3d_time_learned_apply(GEOMETRY *g, kfun3d_mpnn *net, int reps)
{
  DevMesh *m = dev_or_fail(g);
  if (!m || !net || reps < 1) return -1.0;
  if (!ensure_flex(*m)) return -1.0;
  if (!m->mgraph) m->mgraph = kfun3d_mpnn_graph_create(g);
  if (!m->mgraph || kf_mpnn_prepare(net, m->mgraph) != KFUN3D_OK) return -1.0;
  const Ops o = ops();
  const size_t n = 4 * (size_t)m->N;
  h2d(*m, m->q, g->q->q, n);
  dev_residual(*m, o, m->q, m->fy);   // a residual-like input
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  kf_mpnn_apply_async(net, m->mgraph, m->fy, m->q, m->t, m->stream);   // warm-up
  CK(cudaEventRecord(e0, m->stream));
  for (int r = 0; r < reps; r++) kf_mpnn_apply_async(net, m->mgraph, m->fy, m->q, m->t, m->stream);
  CK(cudaEventRecord(e1, m->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (kf_mpnn_status(net, m->stream) != KFUN3D_OK || !finish(*m, "kfun3d_time_learned_apply")) return -1.0;
  return ms / reps;
}
