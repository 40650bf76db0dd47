// kfun3d_b200 device kernels for the residual, time step, Jacobian fill,
// ILU(0) and triangular solves.
//
// Included twice: kernels_exact.cu (KF_FAST 0, compiled with -fmad=false) and
// kernels_fast.cu (KF_FAST 1, fused multiply-add allowed).  In the exact build
// every expression keeps the reference's operation order, and every per-node
// sum is taken in the reference's order (edges by index, then wall faces by
// colour, then far-field nodes), which makes the results bit-identical to the
// reference at one OpenMP thread.  No kernel uses floating-point atomics: each
// node (or matrix row) is owned by one thread, which gathers its incident
// edges and recomputes the edge terms it needs, so every run is deterministic.
//
// Layout in HBM (DevMesh): node state q, residual r and the three gradient
// arrays are double4 per node (the reference's q[4*node+var] AoS, one 32-byte
// sector per gather); edge geometry is a double4 (unit normal, area) per edge;
// each node's incident edges are a contiguous run of the incidence arrays.
#include <cstdint>
#include <type_traits>

#include "internal.h"

#ifndef KF_FAST
#error "define KF_FAST"
#endif

namespace KF_NS {

constexpr double KB = 15.0;                  // inc/phy.h:6 (beta)
constexpr double KP = 1.0;                   // inc/phy.h:7
constexpr double KW = 0.0;                   // inc/phy.h:10
constexpr double SWITCH = (double)0.95f;     // src/flux.c:181 (a float literal)
constexpr double MAG0 = 0.5 / 3;             // src/flux.c:11
constexpr double MAG1 = -MAG0;
constexpr double INV_B = 1.0 / 15.0;

__device__ __forceinline__ double div_b(double x)
{
#if KF_FAST
  return x * INV_B;
#else
  return x / KB;
#endif
}

struct Frame { double x1, y1, z1, x2, y2, z2; };

// src/flux.c:173-217: unit tangents completing the unit normal.
__device__ __forceinline__ Frame tangents(double xn, double yn, double zn)
{
  Frame f;
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
#if KF_FAST
  const double is = rsqrt(s);
  f.x1 *= is;
  f.y1 *= is;
  f.z1 *= is;
#else
  s = sqrt(s);
  f.x1 /= s;
  f.y1 /= s;
  f.z1 /= s;
#endif
  f.x2 = yn * f.z1;
  f.x2 -= zn * f.y1;
  f.y2 = zn * f.x1;
  f.y2 -= xn * f.z1;
  f.z2 = xn * f.y1;
  f.z2 -= yn * f.x1;
  return f;
}

struct Phi { double p4, p5, p6, p7, p8, p9; };

// src/flux.c:299-324
__device__ __forceinline__ Phi phis(double xn, double yn, double zn, double u, double v,
                                    double w, double ubar, const Frame &f)
{
  double p1 = xn * KB; p1 += u * ubar;
  double p2 = yn * KB; p2 += v * ubar;
  double p3 = zn * KB; p3 += w * ubar;
  Phi ph;
  ph.p4 = f.y2 * p3; ph.p4 -= f.z2 * p2;
  ph.p5 = f.z2 * p1; ph.p5 -= f.x2 * p3;
  ph.p6 = f.x2 * p2; ph.p6 -= f.y2 * p1;
  ph.p7 = f.z1 * p2; ph.p7 -= f.y1 * p3;
  ph.p8 = f.x1 * p3; ph.p8 -= f.z1 * p1;
  ph.p9 = f.y1 * p1; ph.p9 -= f.x1 * p2;
  return ph;
}

__device__ __forceinline__ double4 add4(double4 a, double4 b) { return make_double4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ double4 sub4(double4 a, double4 b) { return make_double4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }

// Reconstructed state at the edge midpoint, src/flux.c:222-251.
__device__ __forceinline__ double4 recon(double4 q, double4 gx, double4 gy, double4 gz,
                                         double rx, double ry, double rz)
{
  double4 s;
  s.x = q.x + gx.x * rx; s.x += gy.x * ry; s.x += gz.x * rz;
  s.y = q.y + gx.y * rx; s.y += gy.y * ry; s.y += gz.y * rz;
  s.z = q.z + gx.z * rx; s.z += gy.z * ry; s.z += gz.z * rz;
  s.w = q.w + gx.w * rx; s.w += gy.w * ry; s.w += gz.w * rz;
  return s;
}

// Dissipative edge flux of src/flux.c:159-448 between end points a = n0 and
// b = n1 (states already reconstructed, sL/sR = p,u,v,w).
__device__ __forceinline__ double4 edge_flux(double4 geo, double4 sL, double4 sR)
{
  const double xn = geo.x, yn = geo.y, zn = geo.z, ln = geo.w;
  const Frame f = tangents(xn, yn, zn);
  double ubarL = xn * sL.y; ubarL += yn * sL.z; ubarL += zn * sL.w;
  double ubarR = xn * sR.y; ubarR += yn * sR.z; ubarR += zn * sR.w;
  const double u = 0.5 * (sL.y + sR.y);
  const double v = 0.5 * (sL.z + sR.z);
  const double w = 0.5 * (sL.w + sR.w);
  double ubar = xn * u; ubar += yn * v; ubar += zn * w;
  const Phi ph = phis(xn, yn, zn, u, v, w, ubar, f);
  const double c2 = ubar * ubar + KB;
  const double c = sqrt(c2);
  const double e12 = fabs(ubar), e3 = fabs(ubar + c), e4 = fabs(ubar - c);
  const double dp = sR.x - sL.x, du = sR.y - sL.y, dv = sR.z - sL.z, dw = sR.w - sL.w;

  double ti11 = u * ph.p4; ti11 += v * ph.p5; ti11 += w * ph.p6; ti11 = div_b(-ti11);
  double ti21 = u * ph.p7; ti21 += v * ph.p8; ti21 += w * ph.p9; ti21 = div_b(-ti21);
  double ti31 = 0.5 * (c - ubar); ti31 = div_b(ti31);
  double ti41 = -0.5 * (c + ubar); ti41 = div_b(ti41);

  double dv1 = ti11 * dp; dv1 += ph.p4 * du; dv1 += ph.p5 * dv; dv1 += ph.p6 * dw;
  double dv2 = ti21 * dp; dv2 += ph.p7 * du; dv2 += ph.p8 * dv; dv2 += ph.p9 * dw;
  double dv3 = 2.0 * ti31 * dp; dv3 += xn * du; dv3 += yn * dv; dv3 += zn * dw;
  double dv4 = 2.0 * ti41 * dp; dv4 += xn * du; dv4 += yn * dv; dv4 += zn * dw;
#if KF_FAST
  const double ic2 = 1.0 / c2;
  dv1 *= ic2;
  dv2 *= ic2;
  dv3 *= 0.5 * ic2;
  dv4 *= 0.5 * ic2;
#else
  dv1 /= c2;
  dv2 /= c2;
  const double hc2 = 0.5 / c2;
  dv3 *= hc2;
  dv4 *= hc2;
#endif
  const double r13 = c * KB;
  double r23 = u * (ubar + c); r23 += xn * KB;
  double r33 = v * (ubar + c); r33 += yn * KB;
  double r43 = w * (ubar + c); r43 += zn * KB;
  const double r14 = -c * KB;
  double r24 = u * (ubar - c); r24 += xn * KB;
  double r34 = v * (ubar - c); r34 += yn * KB;
  double r44 = w * (ubar - c); r44 += zn * KB;

  const double t1 = e3 * r13 * dv3 + e4 * r14 * dv4;
  double t2 = e12 * f.x1 * dv1 + e12 * f.x2 * dv2;
  t2 += e3 * r23 * dv3 + e4 * r24 * dv4;
  double t3 = e12 * f.y1 * dv1 + e12 * f.y2 * dv2;
  t3 += e3 * r33 * dv3 + e4 * r34 * dv4;
  double t4 = e12 * f.z1 * dv1 + e12 * f.z2 * dv2;
  t4 += e3 * r43 * dv3 + e4 * r44 * dv4;

  const double fp1 = ln * KB * ubarL;
  const double fp2 = ln * (sL.y * ubarL + xn * sL.x);
  const double fp3 = ln * (sL.z * ubarL + yn * sL.x);
  const double fp4 = ln * (sL.w * ubarL + zn * sL.x);
  const double fm1 = ln * KB * ubarR;
  const double fm2 = ln * (sR.y * ubarR + xn * sR.x);
  const double fm3 = ln * (sR.z * ubarR + yn * sR.x);
  const double fm4 = ln * (sR.w * ubarR + zn * sR.x);
  double4 res;
  res.x = 0.5 * (fp1 + fm1 - ln * t1);
  res.y = 0.5 * (fp2 + fm2 - ln * t2);
  res.z = 0.5 * (fp3 + fm3 - ln * t3);
  res.w = 0.5 * (fp4 + fm4 - ln * t4);
  return res;
}

// Characteristic far-field flux at one node, src/flux.c:552-778.
__device__ __forceinline__ double4 farfield_flux(double U, double V, double fx, double fy,
                                                 double fz, double4 qi)
{
  double area = fx * fx; area += fy * fy; area += fz * fz; area = sqrt(area);
  const double xn = fx / area, yn = fy / area, zn = fz / area;
  const Frame f = tangents(xn, yn, zn);
  double ubar0 = xn * U; ubar0 += yn * V; ubar0 += zn * KW;
  const double c20 = ubar0 * ubar0 + KB;
  const double c0 = sqrt(c20);
  const Phi ph = phis(xn, yn, zn, U, V, KW, ubar0, f);
  const double t13 = c0 * KB;
  double t23 = U * (ubar0 + c0); t23 += xn * KB;
  double t33 = V * (ubar0 + c0); t33 += yn * KB;
  double t43 = KW * (ubar0 + c0); t43 += zn * KB;
  const double t14 = -c0 * KB;
  double t24 = U * (ubar0 - c0); t24 += xn * KB;
  double t34 = V * (ubar0 - c0); t34 += yn * KB;
  double t44 = KW * (ubar0 - c0); t44 += zn * KB;
  double ti11 = U * ph.p4; ti11 += V * ph.p5; ti11 += KW * ph.p6; ti11 = -ti11 / KB;
  double ti21 = U * ph.p7; ti21 += V * ph.p8; ti21 += KW * ph.p9; ti21 = -ti21 / KB;
  double ti31 = 0.5 * (c0 - ubar0); ti31 /= KB;
  double ti41 = -0.5 * (c0 + ubar0); ti41 /= KB;
  const double pi = qi.x, ui = qi.y, vi = qi.z, wi = qi.w;
  double un = xn * ui; un += yn * vi; un += zn * wi;
  double pr, ur, vr, wr;
  if (un > 0.0) { pr = pi; ur = ui; vr = vi; wr = wi; }
  else { pr = KP; ur = U; vr = V; wr = KW; }
  double rhs1 = ti11 * pr; rhs1 += ph.p4 * ur; rhs1 += ph.p5 * vr; rhs1 += ph.p6 * wr; rhs1 /= c20;
  double rhs2 = ti21 * pr; rhs2 += ph.p7 * ur; rhs2 += ph.p8 * vr; rhs2 += ph.p9 * wr; rhs2 /= c20;
  double rhs3 = 2.0 * ti31 * pi; rhs3 += xn * ui; rhs3 += yn * vi; rhs3 += zn * wi;
  rhs3 = 0.5 * rhs3 / c20;
  double rhs4 = 2.0 * ti41 * KP; rhs4 += xn * U; rhs4 += yn * V; rhs4 += zn * KW;
  rhs4 = 0.5 * rhs4 / c20;
  double pb = t13 * rhs3; pb += t14 * rhs4;
  double ub = f.x1 * rhs1; ub += f.x2 * rhs2; ub += t23 * rhs3; ub += t24 * rhs4;
  double vb = f.y1 * rhs1; vb += f.y2 * rhs2; vb += t33 * rhs3; vb += t34 * rhs4;
  double wb = f.z1 * rhs1; wb += f.z2 * rhs2; wb += t43 * rhs3; wb += t44 * rhs4;
  double ubar = xn * ub; ubar += yn * vb; ubar += zn * wb;
  double4 o;
  o.x = area * KB * ubar;
  o.y = area * (ub * ubar + xn * pb);
  o.z = area * (vb * ubar + yn * pb);
  o.w = area * (wb * ubar + zn * pb);
  return o;
}

// ------------------------------------------------------------------ TMA bulk staging

// 1-D bulk copies (cp.async.bulk, the TMA engine's untiled path) into shared
// memory, completed on an mbarrier.  Source and destination addresses and the
// size must be multiples of 16 bytes; callers guarantee it.
__device__ __forceinline__ unsigned smem_addr(const void *p)
{
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *mbar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(mbar))
               : "memory");
}

constexpr uint32_t KF_MBAR_LIMIT = 1u << 24;

// Bounded wait for phase `phase` of the mbarrier; false (and *err set) if it
// gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, unsigned phase, int *err)
{
  const unsigned a = smem_addr(mbar);
  for (uint32_t spins = 0; spins < KF_MBAR_LIMIT; spins++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  atomicExch(err, 1);
  return false;
}

// ------------------------------------------------------------------ gradient

// Same sum as k_gradient, with the block's contiguous incidence range (other
// end points and least-squares terms) staged into shared memory by four bulk
// copies.  The range is widened to 4-entry boundaries so every copy starts and
// ends on 16 bytes (the arrays are padded to a multiple of 4 entries).
__global__ void __launch_bounds__(128) k_gradient_tma(uint32_t N, const uint32_t *__restrict__ ord,
                                                      const uint32_t *__restrict__ inc_ptr,
                                                      const uint32_t *__restrict__ inc_oth,
                                                      const double *__restrict__ inc_w, uint32_t wstride,
                                                      const double4 *__restrict__ q, double4 *__restrict__ gx,
                                                      double4 *__restrict__ gy, double4 *__restrict__ gz, int *err)
{
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  const uint32_t nb = blockIdx.x * blockDim.x;
  const uint32_t ne = min(nb + blockDim.x, N);
  const uint32_t k0 = inc_ptr[nb], k1 = inc_ptr[ne];
  const uint32_t ka = k0 & ~3u, kb = (k1 + 3u) & ~3u, cnt = kb - ka;
  uint32_t *s_oth = reinterpret_cast<uint32_t *>(smem);
  double *s_w = reinterpret_cast<double *>(smem + 4 * (size_t)((cnt + 3u) & ~3u));
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_expect_tx(&mbar, cnt * 28u);
    if (cnt) {
      bulk_g2s(s_oth, inc_oth + ka, cnt * 4u, &mbar);
      bulk_g2s(s_w, inc_w + ka, cnt * 8u, &mbar);
      bulk_g2s(s_w + cnt, inc_w + wstride + ka, cnt * 8u, &mbar);
      bulk_g2s(s_w + 2 * (size_t)cnt, inc_w + 2 * (size_t)wstride + ka, cnt * 8u, &mbar);
    }
  }
  __syncthreads();
  if (!mbar_wait(&mbar, 0, err)) return;
  const uint32_t p = nb + threadIdx.x;
  if (p >= N) return;
  const uint32_t n = ord[p];
  const double4 qn = q[n];
  double4 ax = make_double4(0, 0, 0, 0), ay = ax, az = ax;
  const uint32_t e1 = inc_ptr[p + 1] - ka;
  for (uint32_t k = inc_ptr[p] - ka; k < e1; k++) {
    const double4 qo = q[s_oth[k]];
    const double wx = s_w[k], wy = s_w[cnt + k], wz = s_w[2 * (size_t)cnt + k];
    double dq;
    dq = qo.x - qn.x; ax.x += wx * dq; ay.x += wy * dq; az.x += wz * dq;
    dq = qo.y - qn.y; ax.y += wx * dq; ay.y += wy * dq; az.y += wz * dq;
    dq = qo.z - qn.z; ax.z += wx * dq; ay.z += wy * dq; az.z += wz * dq;
    dq = qo.w - qn.w; ax.w += wx * dq; ay.w += wy * dq; az.w += wz * dq;
  }
  gx[n] = ax;
  gy[n] = ay;
  gz[n] = az;
}



// src/flux.c:60-145 as a gather: node n sums w.(q[other]-q[n]) over its
// incident edges in edge order.
__global__ void __launch_bounds__(256) k_gradient(uint32_t N, const uint32_t *__restrict__ ord,
                                                  const uint32_t *__restrict__ inc_ptr,
                                                  const uint32_t *__restrict__ inc_oth,
                                                  const double *__restrict__ inc_w, uint32_t ninc,
                                                  const double4 *__restrict__ q, double4 *__restrict__ gx,
                                                  double4 *__restrict__ gy, double4 *__restrict__ gz)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t n = ord[p];
  const double4 qn = q[n];
  double4 ax = make_double4(0, 0, 0, 0), ay = ax, az = ax;
  const uint32_t k1 = inc_ptr[p + 1];
  for (uint32_t k = inc_ptr[p]; k < k1; k++) {
    const double4 qo = q[inc_oth[k]];
    const double wx = inc_w[k], wy = inc_w[ninc + k], wz = inc_w[2 * (size_t)ninc + k];
    double dq;
    dq = qo.x - qn.x; ax.x += wx * dq; ay.x += wy * dq; az.x += wz * dq;
    dq = qo.y - qn.y; ax.y += wx * dq; ay.y += wy * dq; az.y += wz * dq;
    dq = qo.z - qn.z; ax.z += wx * dq; ay.z += wy * dq; az.z += wz * dq;
    dq = qo.w - qn.w; ax.w += wx * dq; ay.w += wy * dq; az.w += wz * dq;
  }
  gx[n] = ax;
  gy[n] = ay;
  gz[n] = az;
}

// ------------------------------------------------------------------ least-squares weights on the device

// The seven least-squares coefficients of node n (src/weights.c:237-297,
// 173-232, 102-170 and 335-366): three passes over the node's incident edges
// in edge order, each followed by the node's own normalisation, exactly the
// reference's operations (its edge loops add into both end points; here each
// node gathers its own terms in the same order).  Output per node: w00, w01,
// w02, w11, w12, w22, w33 and a zero, as two double4.
__global__ void __launch_bounds__(128) k_lsq_coef(uint32_t N, const uint32_t *__restrict__ ord,
                                                  const uint32_t *__restrict__ inc_ptr,
                                                  const uint32_t *__restrict__ inc_oth,
                                                  const uint32_t *__restrict__ inc_edge,
                                                  const double4 *__restrict__ xyz, double4 *__restrict__ coef)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t n = ord[p];
  const double4 xn = xyz[n];
  const uint32_t k0 = inc_ptr[p], k1 = inc_ptr[p + 1];
  double w0 = 0.0, w1 = 0.0, w2 = 0.0;
  for (uint32_t k = k0; k < k1; k++) {
    const double4 xo = xyz[inc_oth[k]];
    const double rx = xo.x - xn.x, ry = xo.y - xn.y, rz = xo.z - xn.z;
    w0 += rx * rx;
    w1 += rx * ry;
    w2 += rx * rz;
  }
  w0 = sqrt(w0);
  w1 /= w0;
  w2 /= w0;
  double w3 = 0.0, w4 = 0.0;
  for (uint32_t k = k0; k < k1; k++) {
    const double4 xo = xyz[inc_oth[k]];
    const double d = w1 / w0;
    if (!(inc_edge[k] >> 31)) {   // n is n0: edge vector from n to the other end
      const double dx = xo.x - xn.x, dy = xo.y - xn.y, dz = xo.z - xn.z;
      const double d_ = dy - dx * d;
      w3 += d_ * d_;
      w4 += d_ * dz;
    } else {
      const double dx = xn.x - xo.x, dy = xn.y - xo.y, dz = xn.z - xo.z;
      const double d_ = -dy + dx * d;
      w3 += d_ * d_;
      w4 -= d_ * dz;
    }
  }
  w3 = sqrt(w3);
  w4 /= w3;
  double w5 = 0.0;
  for (uint32_t k = k0; k < k1; k++) {
    const double4 xo = xyz[inc_oth[k]];
    const double d0 = w1 / w0, d1 = w2 / w0, d2 = w4 / w3;
    double d0_, d1_;
    if (!(inc_edge[k] >> 31)) {
      const double dx = xo.x - xn.x, dy = xo.y - xn.y, dz = xo.z - xn.z;
      d0_ = dy - dx * d0;
      d1_ = dz - dx * d1;
    } else {
      const double dx = xn.x - xo.x, dy = xn.y - xo.y, dz = xn.z - xo.z;
      d0_ = -dy + dx * d0;
      d1_ = -dz + dx * d1;
    }
    const double d2_ = d1_ - d2 * d0_;
    w5 += d2_ * d2_;
  }
  w5 = sqrt(w5);
  const double sw00 = w0 * w0, sw11 = w3 * w3, sw22 = w5 * w5;
  const double w00 = 1.0 / sw00, w11 = 1.0 / sw11, w22 = 1.0 / sw22;
  const double w01 = w1 / w0, w02 = w2 / w0, w12 = w4 / w3;
  double m0 = w1 * w4;
  m0 -= w2 * w3;
  const double m1 = w0 * w3 * sw22;
  const double w33 = m0 / m1;
  coef[2 * (size_t)n] = make_double4(w00, w01, w02, w11);
  coef[2 * (size_t)n + 1] = make_double4(w12, w22, w33, 0.0);
}

// The least-squares term of one incidence seen from node n (src/weights.c:
// 9-100): (dx, dy, dz) is the edge vector from n0 to n1, c = n's coefficients
// (w00, w01, w02, w11 | w12, w22, w33), n0side = n is the edge's n0.
__device__ __forceinline__ void lsq_term(bool n0side, double dx, double dy, double dz, const double4 ca,
                                         const double4 cb, double &tx, double &ty, double &tz)
{
  double c0, c1;
  if (n0side) {
    c0 = -dx * ca.y + dy;
    c1 = -dx * ca.z + dz;
  } else {
    c0 = dx * ca.y - dy;
    c1 = dx * ca.z - dz;
  }
  c1 = -cb.x * c0 + c1;
  tx = ca.w * ca.y * c0;
  tx = (n0side ? dx : -dx) * ca.x - tx;
  tx += cb.z * c1;
  ty = cb.x * cb.y * c1;
  ty = ca.w * c0 - ty;
  tz = cb.y * c1;
}

// Counts the incidences whose term, recomputed from the coefficients, differs
// in any bit from the stored one (inc_w): zero means the gradient may compute
// its terms on the fly.
__global__ void __launch_bounds__(128) k_lsq_check(uint32_t N, const uint32_t *__restrict__ ord,
                                                   const uint32_t *__restrict__ inc_ptr,
                                                   const uint32_t *__restrict__ inc_oth,
                                                   const uint32_t *__restrict__ inc_edge,
                                                   const double *__restrict__ inc_w, uint32_t wstride,
                                                   const double4 *__restrict__ xyz,
                                                   const double4 *__restrict__ coef, unsigned *bad)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t n = ord[p];
  const double4 xn = xyz[n], ca = coef[2 * (size_t)n], cb = coef[2 * (size_t)n + 1];
  unsigned nbad = 0;
  for (uint32_t k = inc_ptr[p]; k < inc_ptr[p + 1]; k++) {
    const double4 xo = xyz[inc_oth[k]];
    const bool n0side = !(inc_edge[k] >> 31);
    const double dx = n0side ? xo.x - xn.x : xn.x - xo.x;
    const double dy = n0side ? xo.y - xn.y : xn.y - xo.y;
    const double dz = n0side ? xo.z - xn.z : xn.z - xo.z;
    double tx, ty, tz;
    lsq_term(n0side, dx, dy, dz, ca, cb, tx, ty, tz);
    if (__double_as_longlong(tx) != __double_as_longlong(inc_w[k]) ||
        __double_as_longlong(ty) != __double_as_longlong(inc_w[wstride + k]) ||
        __double_as_longlong(tz) != __double_as_longlong(inc_w[2 * (size_t)wstride + k]))
      nbad++;
  }
  if (nbad) atomicAdd(bad, nbad);
}

// The gradient with four lanes per node, lane r owning state component r:
// each lane sums its component's three gradient entries over the node's
// incident edges in edge order (the same additions as one thread doing all
// four components, so the same result).  A quad of lanes reads one 32-byte
// state record per edge and shares the index and term loads; a lane keeps 3
// accumulators instead of 12, so four times as many nodes are in flight.
// ord == nullptr: node data in visit order (row p of the incidence is node p
// of q and of the outputs).
__global__ void __launch_bounds__(256, 4) k_gradient4(uint32_t N, const uint32_t *__restrict__ ord,
                                                      const uint32_t *__restrict__ inc_ptr,
                                                      const uint32_t *__restrict__ inc_oth,
                                                      const double *__restrict__ inc_w, uint32_t ninc,
                                                      const double *__restrict__ q, double *__restrict__ gx,
                                                      double *__restrict__ gy, double *__restrict__ gz)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t p = gid >> 2, r = gid & 3;
  if (p >= N) return;
  const uint32_t n = ord ? ord[p] : p;
  const double qn = q[4 * (size_t)n + r];
  double ax = 0.0, ay = 0.0, az = 0.0;
  const uint32_t k1 = inc_ptr[p + 1];
  for (uint32_t k = inc_ptr[p]; k < k1; k++) {
    const double dq = q[4 * (size_t)inc_oth[k] + r] - qn;
    ax += inc_w[k] * dq;
    ay += inc_w[ninc + k] * dq;
    az += inc_w[2 * (size_t)ninc + k] * dq;
  }
  gx[4 * (size_t)n + r] = ax;
  gy[4 * (size_t)n + r] = ay;
  gz[4 * (size_t)n + r] = az;
}

// Node data in the visit order of the node-centric passes: dst[p] =
// src[ord[p]] (gather) and back (scatter).  On large meshes the residual
// passes work on visit-ordered copies of the state, coordinates and
// gradients, so that a node's neighbours -- close to it in space, hence in
// the Morton visit order -- are close to it in memory too.
__global__ void __launch_bounds__(256) k_visit_gather(uint32_t N, const uint32_t *__restrict__ ord,
                                                      const double4 *__restrict__ src, double4 *__restrict__ dst)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) dst[p] = src[ord[p]];
}

__global__ void __launch_bounds__(256) k_visit_scatter(uint32_t N, const uint32_t *__restrict__ ord,
                                                       const double4 *__restrict__ src, double4 *__restrict__ dst)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) dst[ord[p]] = src[p];
}

// ------------------------------------------------------------------ residual

// src/flux.c:151-465 as a gather: node n recomputes the flux of each incident
// edge (end points in the reference's n0/n1 roles) and adds it (n = n0) or
// subtracts it (n = n1) in edge order.
template <bool FIRST_ORDER>
__global__ void __launch_bounds__(128) k_residual(uint32_t N, const uint32_t *__restrict__ ord,
                                                  const uint32_t *__restrict__ inc_ptr,
                                                  const uint32_t *__restrict__ inc_oth,
                                                  const uint32_t *__restrict__ inc_edge,
                                                  const double4 *__restrict__ egeo,
                                                  const double4 *__restrict__ xyz,
                                                  const double4 *__restrict__ q,
                                                  const double4 *__restrict__ gx,
                                                  const double4 *__restrict__ gy,
                                                  const double4 *__restrict__ gz, double4 *__restrict__ r)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t n = ord[p];
  const double4 qs = q[n], xs = xyz[n];
  double4 gxs, gys, gzs;
  if (!FIRST_ORDER) { gxs = gx[n]; gys = gy[n]; gzs = gz[n]; }
  double4 acc = make_double4(0, 0, 0, 0);
  const uint32_t k1 = inc_ptr[p + 1];
  for (uint32_t k = inc_ptr[p]; k < k1; k++) {
    const uint32_t o = inc_oth[k], ev = inc_edge[k];
    const bool is_n1 = ev >> 31;
    const double4 geo = egeo[ev & 0x7fffffffu];
    const double4 qo = q[o], xo = xyz[o];
    const double4 xa = is_n1 ? xo : xs, xb = is_n1 ? xs : xo;
    const double4 qa = is_n1 ? qo : qs, qb = is_n1 ? qs : qo;
    const double xm = 0.5 * (xa.x + xb.x), ym = 0.5 * (xa.y + xb.y), zm = 0.5 * (xa.z + xb.z);
    double4 sL, sR;
    if (FIRST_ORDER) {
      const double4 z = make_double4(0, 0, 0, 0);
      sL = recon(qa, z, z, z, xm - xa.x, ym - xa.y, zm - xa.z);
      sR = recon(qb, z, z, z, xm - xb.x, ym - xb.y, zm - xb.z);
    } else {
      const double4 gxo = gx[o], gyo = gy[o], gzo = gz[o];
      sL = is_n1 ? recon(qa, gxo, gyo, gzo, xm - xa.x, ym - xa.y, zm - xa.z)
                 : recon(qa, gxs, gys, gzs, xm - xa.x, ym - xa.y, zm - xa.z);
      sR = is_n1 ? recon(qb, gxs, gys, gzs, xm - xb.x, ym - xb.y, zm - xb.z)
                 : recon(qb, gxo, gyo, gzo, xm - xb.x, ym - xb.y, zm - xb.z);
    }
    const double4 res = edge_flux(geo, sL, sR);
    acc = is_n1 ? sub4(acc, res) : add4(acc, res);
  }
  r[n] = acc;
}

// Two-pass residual, used when every edge has n0 < n1 (edges sorted by n0).
// Then a node's edges as n1 all precede its edges as n0 in edge order, so the
// reference's per-node sum in edge order is: subtract the n1-side fluxes in
// edge order, then add the n0-side fluxes in edge order.  Pass 1 evaluates
// each edge's flux once, one thread per edge, and stores it; pass 2 gathers
// per node.  The edge arrays (end points, geometry, flux) are stored grouped
// by n0 in the nodes' visit order ord, each group in edge order: a warp's
// edges are then close in space (their end points' data is shared in L2 and
// L1), and eoff / in1_ptr are indexed by visit position, in1_edge holds
// storage positions.
template <bool FIRST_ORDER>
__global__ void __launch_bounds__(128) k_flux_edges(uint32_t E, const uint32_t *__restrict__ n0,
                                                    const uint32_t *__restrict__ n1,
                                                    const double4 *__restrict__ egeo,
                                                    const double4 *__restrict__ xyz,
                                                    const double4 *__restrict__ q,
                                                    const double4 *__restrict__ gx,
                                                    const double4 *__restrict__ gy,
                                                    const double4 *__restrict__ gz, double4 *__restrict__ res)
{
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const uint32_t a = n0[e], o = n1[e];
  const double4 geo = egeo[e];
  const double4 qa = q[a], xa = xyz[a], qb = q[o], xb = xyz[o];
  const double xm = 0.5 * (xa.x + xb.x), ym = 0.5 * (xa.y + xb.y), zm = 0.5 * (xa.z + xb.z);
  double4 sL, sR;
  if (FIRST_ORDER) {
    const double4 z = make_double4(0, 0, 0, 0);
    sL = recon(qa, z, z, z, xm - xa.x, ym - xa.y, zm - xa.z);
    sR = recon(qb, z, z, z, xm - xb.x, ym - xb.y, zm - xb.z);
  } else {
    sL = recon(qa, gx[a], gy[a], gz[a], xm - xa.x, ym - xa.y, zm - xa.z);
    sR = recon(qb, gx[o], gy[o], gz[o], xm - xb.x, ym - xb.y, zm - xb.z);
  }
  res[e] = edge_flux(geo, sL, sR);
}

__global__ void __launch_bounds__(256) k_flux_nodes(uint32_t N, const uint32_t *__restrict__ ord,
                                                    const uint32_t *__restrict__ in1_ptr,
                                                    const uint32_t *__restrict__ in1_edge,
                                                    const uint32_t *__restrict__ eoff,
                                                    const double4 *__restrict__ res, double4 *__restrict__ r)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t n = ord[p];
  double4 acc = make_double4(0, 0, 0, 0);
  const uint32_t k1 = in1_ptr[p + 1];
  for (uint32_t k = in1_ptr[p]; k < k1; k++) acc = sub4(acc, res[in1_edge[k]]);
  const uint32_t e1 = eoff[p + 1];
  for (uint32_t e = eoff[p]; e < e1; e++) acc = add4(acc, res[e]);
  r[n] = acc;
}

// k_flux_nodes with four lanes per node, lane r summing flux component r in
// the same order (so the same result): a quad reads each edge flux as one
// 32-byte sector, and four times as many nodes' gathers are in flight.
__global__ void __launch_bounds__(256) k_flux_nodes4(uint32_t N, const uint32_t *__restrict__ ord,
                                                     const uint32_t *__restrict__ in1_ptr,
                                                     const uint32_t *__restrict__ in1_edge,
                                                     const uint32_t *__restrict__ eoff,
                                                     const double *__restrict__ res, double *__restrict__ r)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t p = gid >> 2, c = gid & 3;
  if (p >= N) return;
  const uint32_t n = ord[p];
  double acc = 0.0;
  const uint32_t k1 = in1_ptr[p + 1];
  for (uint32_t k = in1_ptr[p]; k < k1; k++) acc = acc - res[4 * (size_t)in1_edge[k] + c];
  const uint32_t e1 = eoff[p + 1];
  for (uint32_t e = eoff[p]; e < e1; e++) acc = acc + res[4 * (size_t)e + c];
  r[4 * (size_t)n + c] = acc;
}

// Boundary terms, after all edges: wall faces by colour (src/flux.c:467-539),
// then far-field nodes (src/flux.c:541-779), each node in list order.
__global__ void k_residual_boundary(uint32_t nb, const uint32_t *__restrict__ bnd_node,
                                    const uint32_t *__restrict__ bnd_ptr,
                                    const uint32_t *__restrict__ bnd_ent,
                                    const uint32_t *__restrict__ wf_nodes,
                                    const double *__restrict__ wf_n, const double *__restrict__ f_n,
                                    const double4 *__restrict__ q, double4 *__restrict__ r,
                                    double U, double V)
{
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const uint32_t n = bnd_node[b];
  double4 acc = r[n];
  for (uint32_t k = bnd_ptr[b]; k < bnd_ptr[b + 1]; k++) {
    const uint32_t ent = bnd_ent[k], kind = ent >> 29, idx = ent & 0x1fffffffu;
    if (kind == 0) {
      const uint32_t f = idx / 3, corner = idx % 3;
      const double p1 = q[wf_nodes[3 * f]].x, p2 = q[wf_nodes[3 * f + 1]].x, p3 = q[wf_nodes[3 * f + 2]].x;
      double p;
      if (corner == 0) { p = 0.125 * (p2 + p3); p += 0.75 * p1; }
      else if (corner == 1) { p = 0.125 * (p3 + p1); p += 0.75 * p2; }
      else { p = 0.125 * (p1 + p2); p += 0.75 * p3; }
      acc.y += wf_n[3 * f] * p;
      acc.z += wf_n[3 * f + 1] * p;
      acc.w += wf_n[3 * f + 2] * p;
    } else if (kind == 2) {
      const double4 o = farfield_flux(U, V, f_n[3 * idx], f_n[3 * idx + 1], f_n[3 * idx + 2], q[n]);
      acc.x += o.x;
      acc.y += o.y;
      acc.z += o.z;
      acc.w += o.w;
    }
  }
  r[n] = acc;
}

// ------------------------------------------------------------------ time step

// src/timestep.c:58-91 as a gather; nodes without boundary terms are divided
// by the CFL number here, boundary nodes in k_timestep_boundary.
// VISIT: q and the incidences' other ends in visit order (row p of the
// incidence is node p of q), and the geometry per incidence (inc_geo[k])
// instead of per edge.
template <bool VISIT>
__global__ void __launch_bounds__(256) k_timestep(uint32_t N, const uint32_t *__restrict__ ord,
                                                  const uint32_t *__restrict__ inc_ptr,
                                                  const uint32_t *__restrict__ inc_oth,
                                                  const uint32_t *__restrict__ inc_edge,
                                                  const double4 *__restrict__ egeo,
                                                  const double4 *__restrict__ q,
                                                  const uint32_t *__restrict__ bnd_of, double cfl,
                                                  double *__restrict__ cdt)
{
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const uint32_t n = ord[p];
  const double4 qs = q[VISIT ? p : n];
  double acc = 0.0;
  const uint32_t k1 = inc_ptr[p + 1];
  for (uint32_t k = inc_ptr[p]; k < k1; k++) {
    const uint32_t ev = inc_edge[k];
    const bool is_n1 = ev >> 31;
    const double4 geo = egeo[VISIT ? k : (ev & 0x7fffffffu)];
    const double4 qo = q[inc_oth[k]];
    const double4 qa = is_n1 ? qo : qs, qb = is_n1 ? qs : qo;
    const double xnorm = geo.x * geo.w, ynorm = geo.y * geo.w, znorm = geo.z * geo.w;
    const double u = 0.5 * (qa.y + qb.y), v = 0.5 * (qa.z + qb.z), w = 0.5 * (qa.w + qb.w);
    const double ubar = geo.x * u + geo.y * v + geo.z * w;
    const double c = sqrt(ubar * ubar + KB);
    double term = u * xnorm;
    term += v * ynorm;
    term += w * znorm;
    term = fabs(term) + c * geo.w;
    acc = acc + term;
  }
  cdt[n] = (bnd_of[n] == 0xffffffffu) ? acc / cfl : acc;
}

__device__ __forceinline__ double boundary_rate(double xn, double yn, double zn, double4 qi)
{
  // src/timestep.c:98-118 and 126-146
  const double ln = sqrt(xn * xn + yn * yn + zn * zn);
  const double ubar = qi.y * xn + qi.z * yn + qi.w * zn;
  const double ub = ubar / ln;
  const double c = sqrt(ub * ub + KB);
  return fabs(ubar) + c * ln;
}

__global__ void k_timestep_boundary(uint32_t nb, const uint32_t *__restrict__ bnd_node,
                                    const uint32_t *__restrict__ bnd_ptr,
                                    const uint32_t *__restrict__ bnd_ent,
                                    const double *__restrict__ s_n, const double *__restrict__ f_n,
                                    const double4 *__restrict__ q, double cfl, double *__restrict__ cdt)
{
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const uint32_t n = bnd_node[b];
  double acc = cdt[n];
  const double4 qi = q[n];
  for (uint32_t k = bnd_ptr[b]; k < bnd_ptr[b + 1]; k++) {
    const uint32_t ent = bnd_ent[k], kind = ent >> 29, idx = ent & 0x1fffffffu;
    if (kind == 1) acc += boundary_rate(s_n[3 * idx], s_n[3 * idx + 1], s_n[3 * idx + 2], qi);
    else if (kind == 2) acc += boundary_rate(f_n[3 * idx], f_n[3 * idx + 1], f_n[3 * idx + 2], qi);
  }
  cdt[n] = acc / cfl;
}

// ------------------------------------------------------------------ Jacobian

// First-order edge Jacobians v0 = (A_L + |A|)/2 and v1 = (A_R - |A|)/2 of
// src/fill.c:171-494 (row-major 4x4, row = flux component).
__device__ __forceinline__ void edge_jacobians(double4 geo, double4 qa, double4 qb, double *v0, double *v1)
{
  const double xn = geo.x, yn = geo.y, zn = geo.z, ln = geo.w;
  const Frame f = tangents(xn, yn, zn);
  const double uL = qa.y, vL = qa.z, wL = qa.w;
  double ubarL = xn * uL; ubarL += yn * vL; ubarL += zn * wL;
  const double uR = qb.y, vR = qb.z, wR = qb.w;
  double ubarR = xn * uR; ubarR += yn * vR; ubarR += zn * wR;
  const double u = 0.5 * (uL + uR), v = 0.5 * (vL + vR), w = 0.5 * (wL + wR);
  double ubar = xn * u; ubar += yn * v; ubar += zn * w;
  const double c2 = ubar * ubar + KB;
  const double c = sqrt(c2);
  const double e12 = ln * fabs(ubar), e3 = ln * fabs(ubar + c), e4 = ln * fabs(ubar - c);
  const Phi ph = phis(xn, yn, zn, u, v, w, ubar, f);
  const double c2inv = 1.0 / c2;
  double y1[4], y2[4], y3[4], y4[4];   // rows of T^-1, columns p,u,v,w
  double t;
  t = u * ph.p4; t += v * ph.p5; t += w * ph.p6; y1[0] = div_b(-c2inv * t);
  t = u * ph.p7; t += v * ph.p8; t += w * ph.p9; y2[0] = div_b(-c2inv * t);
  t = c2inv * (c - ubar); y3[0] = div_b(0.5 * t);
  t = c2inv * (c + ubar); y4[0] = div_b(-0.5 * t);
  y1[1] = c2inv * ph.p4; y2[1] = c2inv * ph.p7; y3[1] = c2inv * 0.5 * xn; y4[1] = c2inv * 0.5 * xn;
  y1[2] = c2inv * ph.p5; y2[2] = c2inv * ph.p8; y3[2] = c2inv * 0.5 * yn; y4[2] = c2inv * 0.5 * yn;
  y1[3] = c2inv * ph.p6; y2[3] = c2inv * ph.p9; y3[3] = c2inv * 0.5 * zn; y4[3] = c2inv * 0.5 * zn;
  const double t13 = c * KB;
  double t23 = u * (ubar + c); t23 += xn * KB;
  double t33 = v * (ubar + c); t33 += yn * KB;
  double t43 = w * (ubar + c); t43 += zn * KB;
  const double t14 = -c * KB;
  double t24 = u * (ubar - c); t24 += xn * KB;
  double t34 = v * (ubar - c); t34 += yn * KB;
  double t44 = w * (ubar - c); t44 += zn * KB;
  double a[4][4];   // |A| = T |Lambda| T^-1, src/fill.c:367-439
#pragma unroll
  for (int j = 0; j < 4; j++) {
    double s = e3 * t13 * y3[j];
    s += e4 * t14 * y4[j];
    a[0][j] = s;
    s = e12 * f.x1 * y1[j]; s += e12 * f.x2 * y2[j]; s += e3 * t23 * y3[j]; s += e4 * t24 * y4[j];
    a[1][j] = s;
    s = e12 * f.y1 * y1[j]; s += e12 * f.y2 * y2[j]; s += e3 * t33 * y3[j]; s += e4 * t34 * y4[j];
    a[2][j] = s;
    s = e12 * f.z1 * y1[j]; s += e12 * f.z2 * y2[j]; s += e3 * t43 * y3[j]; s += e4 * t44 * y4[j];
    a[3][j] = s;
  }
  const double lb = ln * KB, lx = ln * xn, ly = ln * yn, lz = ln * zn;
  v0[0] = 0.5 * a[0][0];
  v0[4] = 0.5 * (lx + a[1][0]);
  v0[8] = 0.5 * (ly + a[2][0]);
  v0[12] = 0.5 * (lz + a[3][0]);
  v0[1] = 0.5 * ((lb * xn) + a[0][1]);
  v0[5] = 0.5 * ((ln * (ubarL + xn * uL)) + a[1][1]);
  v0[9] = 0.5 * ((lx * vL) + a[2][1]);
  v0[13] = 0.5 * ((lx * wL) + a[3][1]);
  v0[2] = 0.5 * ((lb * yn) + a[0][2]);
  v0[6] = 0.5 * ((ly * uL) + a[1][2]);
  v0[10] = 0.5 * ((ln * (ubarL + yn * vL)) + a[2][2]);
  v0[14] = 0.5 * ((ly * wL) + a[3][2]);
  v0[3] = 0.5 * ((lb * zn) + a[0][3]);
  v0[7] = 0.5 * ((lz * uL) + a[1][3]);
  v0[11] = 0.5 * ((lz * vL) + a[2][3]);
  v0[15] = 0.5 * ((ln * (ubarL + zn * wL)) + a[3][3]);
  v1[0] = 0.5 * -a[0][0];
  v1[4] = 0.5 * (lx - a[1][0]);
  v1[8] = 0.5 * (ly - a[2][0]);
  v1[12] = 0.5 * (lz - a[3][0]);
  v1[1] = 0.5 * ((lb * xn) - a[0][1]);
  v1[5] = 0.5 * ((ln * (ubarR + xn * uR)) - a[1][1]);
  v1[9] = 0.5 * ((lx * vR) - a[2][1]);
  v1[13] = 0.5 * ((lx * wR) - a[3][1]);
  v1[2] = 0.5 * ((lb * yn) - a[0][2]);
  v1[6] = 0.5 * ((ly * uR) - a[1][2]);
  v1[10] = 0.5 * ((ln * (ubarR + yn * vR)) - a[2][2]);
  v1[14] = 0.5 * ((ly * wR) - a[3][2]);
  v1[3] = 0.5 * ((lb * zn) - a[0][3]);
  v1[7] = 0.5 * ((lz * uR) - a[1][3]);
  v1[11] = 0.5 * ((lz * vR) - a[2][3]);
  v1[15] = 0.5 * ((ln * (ubarR + zn * wR)) - a[3][3]);
}

// Far-field diagonal block (frozen free-stream T), src/fill.c:527-877.
__device__ __forceinline__ void farfield_jacobian(double U, double V, double fx, double fy, double fz,
                                                  double4 qi, double *vb)
{
  const double ln = sqrt(fx * fx + fy * fy + fz * fz);
  const double xn = fx / ln, yn = fy / ln, zn = fz / ln;
  const Frame f = tangents(xn, yn, zn);
  double ubar0 = xn * U; ubar0 += yn * V; ubar0 += zn * KW;
  const double c20 = ubar0 * ubar0 + KB;
  const double c0 = sqrt(c20);
  const Phi ph = phis(xn, yn, zn, U, V, KW, ubar0, f);
  const double t13 = c0 * KB;
  double t23 = U * (ubar0 + c0); t23 += xn * KB;
  double t33 = V * (ubar0 + c0); t33 += yn * KB;
  double t43 = KW * (ubar0 + c0); t43 += zn * KB;
  const double t14 = -c0 * KB;
  double t24 = U * (ubar0 - c0); t24 += xn * KB;
  double t34 = V * (ubar0 - c0); t34 += yn * KB;
  double t44 = KW * (ubar0 - c0); t44 += zn * KB;
  double ti11 = U * ph.p4; ti11 += V * ph.p5; ti11 += KW * ph.p6; ti11 = -ti11 / KB / c20;
  double ti21 = U * ph.p7; ti21 += V * ph.p8; ti21 += KW * ph.p9; ti21 = -ti21 / KB / c20;
  const double ti31 = (c0 - ubar0) / (2.0 * KB * c20);
  const double ti41 = -(c0 + ubar0) / (2.0 * KB * c20);
  const double ti12 = ph.p4 / c20, ti22 = ph.p7 / c20, ti32 = 0.5 * xn / c20, ti42 = 0.5 * xn / c20;
  const double ti13 = ph.p5 / c20, ti23 = ph.p8 / c20, ti33 = 0.5 * yn / c20, ti43 = 0.5 * yn / c20;
  const double ti14 = ph.p6 / c20, ti24 = ph.p9 / c20, ti34 = 0.5 * zn / c20, ti44 = 0.5 * zn / c20;
  const double pi = qi.x, ui = qi.y, vi = qi.z, wi = qi.w;
  double un = xn * ui; un += yn * vi; un += zn * wi;
  double pr, prp, ur, uru, vr, vrv, wr, wrw;
  if (un > 0.0) { pr = pi; prp = 1.0; ur = ui; uru = 1.0; vr = vi; vrv = 1.0; wr = wi; wrw = 1.0; }
  else { pr = KP; prp = 0.0; ur = U; uru = 0.0; vr = V; vrv = 0.0; wr = KW; wrw = 0.0; }
  double rhs1 = ti11 * pr; rhs1 += ti12 * ur; rhs1 += ti13 * vr; rhs1 += ti14 * wr;
  const double r1d[4] = {ti11 * prp, ti12 * uru, ti13 * vrv, ti14 * wrw};
  double rhs2 = ti21 * pr; rhs2 += ti22 * ur; rhs2 += ti23 * vr; rhs2 += ti24 * wr;
  const double r2d[4] = {ti21 * prp, ti22 * uru, ti23 * vrv, ti24 * wrw};
  double rhs3 = ti31 * pi; rhs3 += ti32 * ui; rhs3 += ti33 * vi; rhs3 += ti34 * wi;
  double rhs4 = ti41 * KP; rhs4 += ti42 * U; rhs4 += ti43 * V; rhs4 += ti44 * KW;
  double pb = t13 * rhs3; pb += t14 * rhs4;
  const double tid[4] = {ti31, ti32, ti33, ti34};
  double ub = f.x1 * rhs1; ub += f.x2 * rhs2; ub += t23 * rhs3; ub += t24 * rhs4;
  double vb_ = f.y1 * rhs1; vb_ += f.y2 * rhs2; vb_ += t33 * rhs3; vb_ += t34 * rhs4;
  double wb = f.z1 * rhs1; wb += f.z2 * rhs2; wb += t43 * rhs3; wb += t44 * rhs4;
  double unb = xn * ub; unb += yn * vb_; unb += zn * wb;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const double pbd = t13 * tid[k];
    double ubd = f.x1 * r1d[k]; ubd += f.x2 * r2d[k]; ubd += t23 * tid[k];
    double vbd = f.y1 * r1d[k]; vbd += f.y2 * r2d[k]; vbd += t33 * tid[k];
    double wbd = f.z1 * r1d[k]; wbd += f.z2 * r2d[k]; wbd += t43 * tid[k];
    double unbd = xn * ubd; unbd += yn * vbd; unbd += zn * wbd;
    vb[k] = ln * KB * unbd;
    vb[4 + k] = ln * (ub * unbd + unb * ubd + xn * pbd);
    vb[8 + k] = ln * (vb_ * unbd + unb * vbd + yn * pbd);
    vb[12 + k] = ln * (wb * unbd + unb * wbd + zn * pbd);
  }
}

template <typename T> __device__ __forceinline__ void store_block(T *dst, const double *v);
template <> __device__ __forceinline__ void store_block<double>(double *dst, const double *v)
{
  double2 *d2 = reinterpret_cast<double2 *>(dst);
#pragma unroll
  for (int i = 0; i < 8; i++) d2[i] = make_double2(v[2 * i], v[2 * i + 1]);
}
template <> __device__ __forceinline__ void store_block<float>(float *dst, const double *v)
{
  float4 *d4 = reinterpret_cast<float4 *>(dst);
#pragma unroll
  for (int i = 0; i < 4; i++)
    d4[i] = make_float4((float)v[4 * i], (float)v[4 * i + 1], (float)v[4 * i + 2], (float)v[4 * i + 3]);
}

// One matrix row per thread (src/fill.c:150-512): the diagonal block starts
// at cdt*I and takes v0 (row = n0) or -v1 (row = n1) of every incident edge
// in edge order; the off-diagonal block of each edge, v1 in row n0 and -v0 in
// row n1, is written once.  The row's first persistent L slot receives the
// last lower block the reference's fill would touch (matrix/matrix.cpp:239).
// Threads run in the active pattern's row order (row_node maps a row to its
// node; null: the identity, the mesh's own pattern), so consecutive threads
// write consecutive rows in both ILU(0) orders.
template <typename T, bool VISIT>
__global__ void __launch_bounds__(128) k_fill(uint32_t N, const uint32_t *__restrict__ row_node,
                                              const uint32_t *__restrict__ rowof,
                                              const uint32_t *__restrict__ inc_ptr,
                                              const uint32_t *__restrict__ inc_oth,
                                              const uint32_t *__restrict__ inc_edge,
                                              const uint32_t *__restrict__ inc_blk,
                                              const double4 *__restrict__ egeo,
                                              const double4 *__restrict__ q,
                                              const double *__restrict__ cdt,
                                              const uint32_t *__restrict__ diag,
                                              const uint32_t *__restrict__ last_lower,
                                              const uint32_t *__restrict__ lpos, T *__restrict__ A,
                                              double *__restrict__ lslot,
                                              const uint32_t *__restrict__ bnd_of, double *__restrict__ dscr)
{
  const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= N) return;
  const uint32_t n = row_node ? row_node[row] : row;
  const uint32_t p = rowof[n];
  const double4 qs = q[VISIT ? p : n];
  double D[16];
#pragma unroll
  for (int i = 0; i < 16; i++) D[i] = 0.0;
  const double c = cdt[n];
  D[0] += c; D[5] += c; D[10] += c; D[15] += c;
  const uint32_t ll = last_lower[n];
  const uint32_t k1 = inc_ptr[p + 1];
  for (uint32_t k = inc_ptr[p]; k < k1; k++) {
    const uint32_t ev = inc_edge[k];
    const bool is_n1 = ev >> 31;
    const double4 geo = egeo[VISIT ? k : (ev & 0x7fffffffu)];
    const double4 qo = q[inc_oth[k]];
    double v0[16], v1[16], off[16];
    edge_jacobians(geo, is_n1 ? qo : qs, is_n1 ? qs : qo, v0, v1);
    if (is_n1) {
#pragma unroll
      for (int i = 0; i < 16; i++) { D[i] += -1.0 * v1[i]; off[i] = 0.0 + -1.0 * v0[i]; }
    } else {
#pragma unroll
      for (int i = 0; i < 16; i++) { D[i] += v0[i]; off[i] = 0.0 + v1[i]; }
    }
    const uint32_t blk = inc_blk[k];
    store_block<T>(A + 16 * (size_t)blk, off);
    if (lslot != nullptr && blk == ll) store_block<double>(lslot + 16 * (size_t)lpos[n], off);
  }
  // FP32 form: boundary rows keep their diagonal in double until the wall and
  // far-field terms are added, so the block is rounded once.
  const uint32_t bo = bnd_of[n];
  if (dscr != nullptr && bo != 0xffffffffu) store_block<double>(dscr + 16 * (size_t)bo, D);
  else store_block<T>(A + 16 * (size_t)diag[n], D);
}

// Wall (matrix/matrix.cpp:282-296) and far-field (src/fill.c:527-877) terms
// on the diagonal blocks of boundary nodes, in list order.
template <typename T>
__global__ void k_fill_boundary(uint32_t nb, const uint32_t *__restrict__ bnd_node,
                                const uint32_t *__restrict__ bnd_ptr, const uint32_t *__restrict__ bnd_ent,
                                const double *__restrict__ s_n, const double *__restrict__ f_n,
                                const double4 *__restrict__ q, const uint32_t *__restrict__ diag,
                                T *__restrict__ A, double U, double V, const double *__restrict__ Dsrc)
{
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const uint32_t n = bnd_node[b];
  T *dst = A + 16 * (size_t)diag[n];
  double D[16];
  // The FP32 form keeps the double diagonal of the row kernel in Dsrc.
#pragma unroll
  for (int i = 0; i < 16; i++) D[i] = Dsrc ? Dsrc[16 * (size_t)b + i] : (double)dst[i];
  for (uint32_t k = bnd_ptr[b]; k < bnd_ptr[b + 1]; k++) {
    const uint32_t ent = bnd_ent[k], kind = ent >> 29, idx = ent & 0x1fffffffu;
    if (kind == 1) {
      D[4] += s_n[3 * idx];
      D[8] += s_n[3 * idx + 1];
      D[12] += s_n[3 * idx + 2];
    } else if (kind == 2) {
      double v[16];
      farfield_jacobian(U, V, f_n[3 * idx], f_n[3 * idx + 1], f_n[3 * idx + 2], q[n], v);
#pragma unroll
      for (int i = 0; i < 16; i++) D[i] += v[i];
    }
  }
  store_block<T>(dst, D);
}

// ------------------------------------------------------------------ ILU(0)


// 4x4 inverse of matrix/inverse.cpp:195-355 by the 16 lanes of a row group
// (lane l = 4*row + col holds entry l of the block s): lane l forms the
// cofactor d[l] as that file does, six triple products in its order and with
// its signs, summed left to right (one table word each: sign bit 15, the
// three entries in bits 0-3, 4-7 and 8-11, multiplied left to right), then
// det = s0 d0 + s1 d4 + s2 d8 + s3 d12, det = 1 / det, entry l = d[l] det.
__device__ const uint16_t kInv4Terms[96] = {0x0fa5u, 0x8eb5u, 0x8f69u, 0x0e79u, 0x0b6du, 0x8a7du, 0x8fa1u, 0x0eb1u, 0x0f29u, 0x8e39u, 0x8b2du, 0x0a3du, 0x0f61u, 0x8e71u, 0x8f25u, 0x0e35u, 0x072du, 0x863du, 0x8b61u, 0x0a71u, 0x0b25u, 0x8a35u, 0x8729u, 0x0639u, 0x8fa4u, 0x0eb4u, 0x0f68u, 0x8e78u, 0x8b6cu, 0x0a7cu, 0x0fa0u, 0x8eb0u, 0x8f28u, 0x0e38u, 0x0b2cu, 0x8a3cu, 0x8f60u, 0x0e70u, 0x0f24u, 0x8e34u, 0x872cu, 0x063cu, 0x0b60u, 0x8a70u, 0x8b24u, 0x0a34u, 0x0728u, 0x8638u, 0x0f94u, 0x8db4u, 0x8f58u, 0x0d78u, 0x0b5cu, 0x897cu, 0x8f90u, 0x0db0u, 0x0f18u, 0x8d38u, 0x8b1cu, 0x093cu, 0x0f50u, 0x8d70u, 0x8f14u, 0x0d34u, 0x071cu, 0x853cu, 0x8b50u, 0x0970u, 0x0b14u, 0x8934u, 0x8718u, 0x0538u, 0x8e94u, 0x0da4u, 0x0e58u, 0x8d68u, 0x8a5cu, 0x096cu, 0x0e90u, 0x8da0u, 0x8e18u, 0x0d28u, 0x0a1cu, 0x892cu, 0x8e50u, 0x0d60u, 0x0e14u, 0x8d24u, 0x861cu, 0x052cu, 0x0a50u, 0x8960u, 0x8a14u, 0x0924u, 0x0618u, 0x8528u};

__device__ __forceinline__ double inv4_lane(double v, int lane16, unsigned mask, int base)
{
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const uint32_t w = kInv4Terms[6 * lane16 + k];
    const double x = __shfl_sync(mask, v, base + (int)(w & 15u));
    const double y = __shfl_sync(mask, v, base + (int)((w >> 4) & 15u));
    const double z = __shfl_sync(mask, v, base + (int)((w >> 8) & 15u));
    const bool neg = (w >> 15) != 0;
    if (k == 0) {
      acc = ((neg ? -x : x) * y) * z;
    } else {
      const double p = (x * y) * z;
      acc = neg ? acc - p : acc + p;
    }
  }
  const double s0 = __shfl_sync(mask, v, base + 0), s1 = __shfl_sync(mask, v, base + 1);
  const double s2 = __shfl_sync(mask, v, base + 2), s3 = __shfl_sync(mask, v, base + 3);
  const double d0 = __shfl_sync(mask, acc, base + 0), d4 = __shfl_sync(mask, acc, base + 4);
  const double d8 = __shfl_sync(mask, acc, base + 8), d12 = __shfl_sync(mask, acc, base + 12);
  double det = s0 * d0 + s1 * d4 + s2 * d8 + s3 * d12;
  det = 1.0 / det;
  return acc * det;
}

// Product of two 4x4 blocks held one entry per lane of a 16-lane group
// (lane l = 4*row + col); entry (r,c) = sum over t of a(r,t) b(t,c), summed
// from zero in t order (matrix/init.cpp:105-116).
__device__ __forceinline__ double gemm_lane(double a, double b, int lane16, unsigned mask, int base)
{
  const int r = lane16 >> 2, c = lane16 & 3;
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < 4; t++) {
    const double at = __shfl_sync(mask, a, base + 4 * r + t);
    const double bt = __shfl_sync(mask, b, base + 4 * t + c);
    s += at * bt;
  }
  return s;
}

// One level of the ILU(0) sweep of matrix/ilu.cpp:49-97, 16 lanes per row.
// For block (i,k) the lanes walk row i's lower columns plus the diagonal
// against column k of U (row k's lower columns plus k, through tblk),
// subtracting L(i,m) U(m,k) for every common m; the last product is added back
// (ilu.cpp:86).  Its L(i,k) factor is the row's persistent slot, the U(i,k)
// factor the not yet updated block, as in the reference.  Lower blocks are
// then multiplied by inv(U(k,k)) and stored in lslot; upper blocks are
// updated in place; the diagonal's inverse goes to dinv.
__global__ void __launch_bounds__(128) k_ilu_level(uint32_t nrows, const uint32_t *__restrict__ rows,
                                                   const uint32_t *__restrict__ ia,
                                                   const uint32_t *__restrict__ ja,
                                                   const uint32_t *__restrict__ diag,
                                                   const uint32_t *__restrict__ tblk,
                                                   const uint32_t *__restrict__ lpos, double *__restrict__ A,
                                                   double *__restrict__ lslot, double *__restrict__ dinv,
                                                   int *__restrict__ status)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t grp = gid >> 4;
  const int lane = threadIdx.x & 31, l16 = lane & 15, base = lane & 16;
  const unsigned mask = 0xffffu << base;
  if (grp >= nrows) return;   // both halves of a warp exit together or stay
  const uint32_t i = rows[grp];
  const uint32_t j0 = ia[i], jd = diag[i], j1 = ia[i + 1];
  const double ident = ((l16 >> 2) == (l16 & 3)) ? 1.0 : 0.0;
  for (uint32_t j = j0; j < j1; j++) {
    const uint32_t k = ja[j];
    double a = A[16 * (size_t)j + l16];
    double d = 0.0;
    // merge L row i (columns ja[j0..jd]) with U column k (rows ja[ia[k]..diag[k]])
    uint32_t pl = j0, pu = ia[k];
    const uint32_t pu_end = diag[k];
    while (pl <= jd && pu <= pu_end) {
      const uint32_t cl = ja[pl], cu = ja[pu];
      if (cl == cu) {
        const double lv = (cl == i) ? ident : lslot[16 * (size_t)(lpos[i] + (pl - j0)) + l16];
        const double uv = A[16 * (size_t)tblk[pu] + l16];
        d = gemm_lane(lv, uv, l16, mask, base);
        a = -1.0 * d + a;
      }
      if (cl <= cu) pl++;
      if (cl >= cu) pu++;
    }
    a = 1.0 * d + a;
    if (k < i) {
      const double dk = dinv[16 * (size_t)k + l16];
      const double lv = gemm_lane(a, dk, l16, mask, base);
      lslot[16 * (size_t)(lpos[i] + (j - j0)) + l16] = lv;
    } else {
      A[16 * (size_t)j + l16] = a;
      if (k == i) {
        // the inverse of the row's diagonal block, entry l on lane l
        const double inv = inv4_lane((double)a, l16, mask, base);
        dinv[16 * (size_t)i + l16] = inv;
        if (__any_sync(mask, !isfinite(inv)) && l16 == 0) atomicExch(status, KFUN3D_ERR_PIVOT);
      }
    }
  }
}

// Same sweep with the merge precomputed: the products of block (i,k) come from
// its pair list (L slot or identity, U block) in merge order, so all loads of
// a product are issued at once instead of walking two index lists.  Lane l16
// owns entry l16 of every block, so the L slots this row wrote earlier are
// read back by the lane that wrote them.
__global__ void __launch_bounds__(128) k_ilu_level_pairs(uint32_t nrows, const uint32_t *__restrict__ rows,
                                                         const uint32_t *__restrict__ ia,
                                                         const uint32_t *__restrict__ ja,
                                                         const uint32_t *__restrict__ diag,
                                                         const uint32_t *__restrict__ pair_ptr,
                                                         const uint2 *__restrict__ pairs,
                                                         const uint32_t *__restrict__ lpos, double *__restrict__ A,
                                                         double *__restrict__ lslot, double *__restrict__ dinv,
                                                         int *__restrict__ status)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t grp = gid >> 4;
  const int lane = threadIdx.x & 31, l16 = lane & 15, base = lane & 16;
  const unsigned mask = 0xffffu << base;
  if (grp >= nrows) return;
  const uint32_t i = rows[grp];
  const uint32_t j0 = ia[i], j1 = ia[i + 1];
  const double ident = ((l16 >> 2) == (l16 & 3)) ? 1.0 : 0.0;
  for (uint32_t j = j0; j < j1; j++) {
    const uint32_t k = ja[j];
    double a = A[16 * (size_t)j + l16];
    double d = 0.0;
    const uint32_t p0 = pair_ptr[j], p1 = pair_ptr[j + 1];
    for (uint32_t pb = p0; pb < p1; pb += 8) {
      double lv[8], uv[8];
      const uint32_t cnt = (p1 - pb) < 8 ? (p1 - pb) : 8;
#pragma unroll
      for (int t = 0; t < 8; t++) {
        lv[t] = 0.0;
        uv[t] = 0.0;
        if ((uint32_t)t < cnt) {
          const uint2 pr = pairs[pb + t];
          lv[t] = pr.x == 0xffffffffu ? ident : lslot[16 * (size_t)pr.x + l16];
          uv[t] = A[16 * (size_t)pr.y + l16];
        }
      }
#pragma unroll
      for (int t = 0; t < 8; t++) {
        if ((uint32_t)t >= cnt) break;
        d = gemm_lane(lv[t], uv[t], l16, mask, base);
        a = -1.0 * d + a;
      }
    }
    a = 1.0 * d + a;
    if (k < i) {
      const double dk = dinv[16 * (size_t)k + l16];
      lslot[16 * (size_t)(lpos[i] + (j - j0)) + l16] = gemm_lane(a, dk, l16, mask, base);
    } else {
      A[16 * (size_t)j + l16] = a;
      if (k == i) {
        // the inverse of the row's diagonal block, entry l on lane l
        const double inv = inv4_lane((double)a, l16, mask, base);
        dinv[16 * (size_t)i + l16] = inv;
        if (__any_sync(mask, !isfinite(inv)) && l16 == 0) atomicExch(status, KFUN3D_ERR_PIVOT);
      }
    }
  }
}

// matrix/ilu.cpp:115-136: the factor over A, lower blocks from the L slots,
// diagonal blocks inverted.
__global__ void k_ilu_finish(uint32_t N, const uint32_t *__restrict__ ia, const uint32_t *__restrict__ diag,
                             const uint32_t *__restrict__ lpos, const double *__restrict__ lslot,
                             const double *__restrict__ dinv, double *__restrict__ A)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t i = gid >> 4, l = gid & 15;
  if (i >= N) return;
  const uint32_t j0 = ia[i], jd = diag[i];
  for (uint32_t j = j0; j < jd; j++) A[16 * (size_t)j + l] = lslot[16 * (size_t)(lpos[i] + (j - j0)) + l];
  A[16 * (size_t)jd + l] = dinv[16 * (size_t)i + l];
}

// FP32 form: plain block ILU(0) in natural order on float blocks (no
// persistent slots); L(i,k) = (A(i,k) - sum L(i,m) U(m,k)) inv(U(k,k)),
// U(i,k) = A(i,k) - sum L(i,m) U(m,k), inverses formed in double and rounded.
__device__ __forceinline__ float gemm_lane_f(float a, float b, int lane16, unsigned mask, int base)
{
  const int r = lane16 >> 2, c = lane16 & 3;
  float s = 0.0f;
#pragma unroll
  for (int t = 0; t < 4; t++) s += __shfl_sync(mask, a, base + 4 * r + t) * __shfl_sync(mask, b, base + 4 * t + c);
  return s;
}

__global__ void __launch_bounds__(128) k_ilu_level_f32(uint32_t nrows, const uint32_t *__restrict__ rows,
                                                       const uint32_t *__restrict__ ia,
                                                       const uint32_t *__restrict__ ja,
                                                       const uint32_t *__restrict__ diag,
                                                       const uint32_t *__restrict__ tblk, float *__restrict__ A,
                                                       float *__restrict__ dinv, int *__restrict__ status)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t grp = gid >> 4;
  const int lane = threadIdx.x & 31, l16 = lane & 15, base = lane & 16;
  const unsigned mask = 0xffffu << base;
  if (grp >= nrows) return;
  const uint32_t i = rows[grp];
  const uint32_t j0 = ia[i], jd = diag[i], j1 = ia[i + 1];
  for (uint32_t j = j0; j < j1; j++) {
    const uint32_t k = ja[j];
    float a = A[16 * (size_t)j + l16];
    // sum over m < min(i,k): row i's lower columns against U(m,k)
    uint32_t pl = j0, pu = ia[k];
    const uint32_t pu_end = diag[k];
    while (pl < jd && pu < pu_end) {
      const uint32_t cl = ja[pl], cu = ja[pu];
      if (cl == cu) {
        const float lv = A[16 * (size_t)pl + l16];
        const float uv = A[16 * (size_t)tblk[pu] + l16];
        a -= gemm_lane_f(lv, uv, l16, mask, base);
      }
      if (cl <= cu) pl++;
      if (cl >= cu) pu++;
    }
    if (k < i) {
      A[16 * (size_t)j + l16] = gemm_lane_f(a, dinv[16 * (size_t)k + l16], l16, mask, base);
    } else {
      A[16 * (size_t)j + l16] = a;
      if (k == i) {
        // the inverse of the row's diagonal block, entry l on lane l
        const double inv = inv4_lane((double)a, l16, mask, base);
        dinv[16 * (size_t)i + l16] = (float)inv;
        if (__any_sync(mask, !isfinite(inv)) && l16 == 0) atomicExch(status, KFUN3D_ERR_PIVOT);
      }
    }
  }
}

// FP32 sweep on the precomputed pair lists: the products of m < min(i,k) are
// the list without its last entry (which is m = min(i,k)); the L factor lives in
// place in the lower blocks, so the L operand of a pair is block
// ia[i] + (slot - lpos[i]).
__global__ void __launch_bounds__(128) k_ilu_level_pairs_f32(uint32_t nrows, const uint32_t *__restrict__ rows,
                                                             const uint32_t *__restrict__ ia,
                                                             const uint32_t *__restrict__ ja,
                                                             const uint32_t *__restrict__ pair_ptr,
                                                             const uint2 *__restrict__ pairs,
                                                             const uint32_t *__restrict__ lpos, float *__restrict__ A,
                                                             float *__restrict__ dinv, int *__restrict__ status)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t grp = gid >> 4;
  const int lane = threadIdx.x & 31, l16 = lane & 15, base = lane & 16;
  const unsigned mask = 0xffffu << base;
  if (grp >= nrows) return;
  const uint32_t i = rows[grp];
  const uint32_t j0 = ia[i], j1 = ia[i + 1], lp = lpos[i];
  for (uint32_t j = j0; j < j1; j++) {
    const uint32_t k = ja[j];
    float a = A[16 * (size_t)j + l16];
    const uint32_t p0 = pair_ptr[j], p1 = pair_ptr[j + 1] - 1;   // without the last product
    for (uint32_t pb = p0; pb < p1; pb += 8) {
      float lv[8], uv[8];
      const uint32_t cnt = (p1 - pb) < 8 ? (p1 - pb) : 8;
#pragma unroll
      for (int t = 0; t < 8; t++) {
        lv[t] = 0.0f;
        uv[t] = 0.0f;
        if ((uint32_t)t < cnt) {
          const uint2 pr = pairs[pb + t];
          lv[t] = A[16 * (size_t)(j0 + (pr.x - lp)) + l16];
          uv[t] = A[16 * (size_t)pr.y + l16];
        }
      }
#pragma unroll
      for (int t = 0; t < 8; t++) {
        if ((uint32_t)t >= cnt) break;
        a -= gemm_lane_f(lv[t], uv[t], l16, mask, base);
      }
    }
    if (k < i) {
      A[16 * (size_t)j + l16] = gemm_lane_f(a, dinv[16 * (size_t)k + l16], l16, mask, base);
    } else {
      A[16 * (size_t)j + l16] = a;
      if (k == i) {
        // the inverse of the row's diagonal block, entry l on lane l
        const double inv = inv4_lane((double)a, l16, mask, base);
        dinv[16 * (size_t)i + l16] = (float)inv;
        if (__any_sync(mask, !isfinite(inv)) && l16 == 0) atomicExch(status, KFUN3D_ERR_PIVOT);
      }
    }
  }
}

// Additive Schwarz without overlap on one device: every block that couples
// two subdomains (row and column nodes in different parts) is set to zero
// before the factorisation.  ILU(0) then keeps those blocks exactly zero
// (each of their products has a factor in another such block, and the
// reference's last product is subtracted and added back: (0 - d) + d = 0),
// so the factor is block-Jacobi ILU(0), one independent factor per
// subdomain in the active elimination order, and the triangular solves are
// the subdomains' own.  One thread per row; row_node maps a row of the
// active numbering to its mesh node (null: the identity).
template <typename T>
__global__ void k_drop_coupling(uint32_t N, const uint32_t *__restrict__ ia, const uint32_t *__restrict__ ja,
                                const uint32_t *__restrict__ row_node, const uint32_t *__restrict__ part,
                                T *__restrict__ A)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const uint32_t pi = part[row_node ? row_node[i] : i];
  for (uint32_t j = ia[i]; j < ia[i + 1]; j++) {
    const uint32_t k = ja[j];
    if (part[row_node ? row_node[k] : k] == pi) continue;
    T *blk = A + 16 * (size_t)j;
#pragma unroll
    for (int e = 0; e < 16; e++) blk[e] = T(0);
  }
}

__global__ void k_ilu_finish_f32(uint32_t N, const uint32_t *__restrict__ diag, const float *__restrict__ dinv,
                                 float *__restrict__ A)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t i = gid >> 4, l = gid & 15;
  if (i >= N) return;
  A[16 * (size_t)diag[i] + l] = dinv[16 * (size_t)i + l];
}

// ------------------------------------------------------------------ SpTRSV

// Forward level of matrix/sptrsv.cpp:173-189, 4 lanes per row (lane = block
// row): x_r = b_r - sum over lower blocks of A x, each block product summed
// from zero in column order, then subtracted, in column order.
template <typename T>
__global__ void __launch_bounds__(128) k_trsv_lower(uint32_t nrows, const uint32_t *__restrict__ rows,
                                                    const uint32_t *__restrict__ ia,
                                                    const uint32_t *__restrict__ ja,
                                                    const uint32_t *__restrict__ diag, const T *__restrict__ A,
                                                    const double *__restrict__ b, double *__restrict__ x)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t g = gid >> 2, rr = gid & 3;
  if (g >= nrows) return;
  const uint32_t i = rows[g];
  double xi = b[4 * (size_t)i + rr];
  const uint32_t jd = diag[i];
  for (uint32_t j = ia[i]; j < jd; j++) {
    const T *blk = A + 16 * (size_t)j + 4 * rr;
    const double4 xc = reinterpret_cast<const double4 *>(x)[ja[j]];
    double t = 0.0;
    t += (double)blk[0] * xc.x;
    t += (double)blk[1] * xc.y;
    t += (double)blk[2] * xc.z;
    t += (double)blk[3] * xc.w;
    xi = -1.0 * t + xi;
  }
  x[4 * (size_t)i + rr] = xi;
}

// Backward level of matrix/sptrsv.cpp:191-209: x_r -= sum over upper blocks,
// then x_r = inv(U_rr) x_r.
template <typename T>
__global__ void __launch_bounds__(128) k_trsv_upper(uint32_t nrows, const uint32_t *__restrict__ rows,
                                                    const uint32_t *__restrict__ ia,
                                                    const uint32_t *__restrict__ ja,
                                                    const uint32_t *__restrict__ diag, const T *__restrict__ A,
                                                    double *__restrict__ x)
{
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t g = gid >> 2, rr = gid & 3;
  const unsigned mask = 0xfu << (threadIdx.x & 28);
  if (g >= nrows) return;
  const uint32_t i = rows[g];
  double xi = x[4 * (size_t)i + rr];
  const uint32_t jd = diag[i], j1 = ia[i + 1];
  for (uint32_t j = jd + 1; j < j1; j++) {
    const T *blk = A + 16 * (size_t)j + 4 * rr;
    const double4 xc = reinterpret_cast<const double4 *>(x)[ja[j]];
    double t = 0.0;
    t += (double)blk[0] * xc.x;
    t += (double)blk[1] * xc.y;
    t += (double)blk[2] * xc.z;
    t += (double)blk[3] * xc.w;
    xi = -1.0 * t + xi;
  }
  const int b4 = threadIdx.x & 28;
  const double x0 = __shfl_sync(mask, xi, b4 + 0), x1 = __shfl_sync(mask, xi, b4 + 1);
  const double x2 = __shfl_sync(mask, xi, b4 + 2), x3 = __shfl_sync(mask, xi, b4 + 3);
  const T *dblk = A + 16 * (size_t)jd + 4 * rr;
  double t = 0.0;
  t += (double)dblk[0] * x0;
  t += (double)dblk[1] * x1;
  t += (double)dblk[2] * x2;
  t += (double)dblk[3] * x3;
  x[4 * (size_t)i + rr] = t;
}

// One row of a triangular sweep for a 16-lane group (lane = 4*block +
// component): every load of the row (its blocks, their columns, and the
// already final x of those columns) is issued at once, then the products are
// subtracted in column order exactly as in matrix/sptrsv.cpp:173-209.
template <typename T, bool UPPER>
__device__ __forceinline__ void trsv_row16(const uint4 d, const uint32_t *__restrict__ ja, const T *__restrict__ A,
                                           const double *__restrict__ b, double *x, int half, int jj, int r,
                                           int l16, unsigned hmask)
{
  const uint32_t i = d.x, jb = d.y, je = d.z;
  double xi = UPPER ? __ldcg(x + 4 * (size_t)i + r) : b[4 * (size_t)i + r];
  for (uint32_t c0 = jb; c0 < je; c0 += 16) {
    double t[4];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const uint32_t j = c0 + 4 * p + jj;
      t[p] = 0.0;
      if (j < je) {
        const uint32_t col = ja[j];
        const T *blk = A + 16 * (size_t)j + 4 * r;
        const double2 x01 = __ldcg(reinterpret_cast<const double2 *>(x) + 2 * (size_t)col);
        const double2 x23 = __ldcg(reinterpret_cast<const double2 *>(x) + 2 * (size_t)col + 1);
        double s = 0.0;
        s += (double)blk[0] * x01.x;
        s += (double)blk[1] * x01.y;
        s += (double)blk[2] * x23.x;
        s += (double)blk[3] * x23.y;
        t[p] = s;
      }
    }
    const uint32_t cnt = (je - c0) < 16u ? (je - c0) : 16u;
#pragma unroll
    for (int p = 0; p < 4; p++)
      for (uint32_t q = 0; q < 4; q++) {
        if (4 * p + q >= cnt) break;
        xi = -1.0 * __shfl_sync(hmask, t[p], 16 * half + 4 * q + r) + xi;
      }
  }
  if (UPPER) {
    const int b4 = 16 * half;
    const double x0 = __shfl_sync(hmask, xi, b4 + 0), x1 = __shfl_sync(hmask, xi, b4 + 1);
    const double x2 = __shfl_sync(hmask, xi, b4 + 2), x3 = __shfl_sync(hmask, xi, b4 + 3);
    const T *dg = A + 16 * (size_t)(jb - 1) + 4 * r;
    double y = 0.0;
    y += (double)dg[0] * x0;
    y += (double)dg[1] * x1;
    y += (double)dg[2] * x2;
    y += (double)dg[3] * x3;
    xi = y;
  }
  if (l16 < 4) __stcg(x + 4 * (size_t)i + r, xi);
}

// One row of a triangular sweep for a group of G lanes (G = 8 or 16): lane
// (jj, r) takes blocks c0 + (G/4) p + jj, row r of each; the partial products
// are subtracted in column order, so the arithmetic is trsv_row16's.
template <typename T, bool UPPER, int G>
__device__ __forceinline__ void trsv_row_g(const uint4 d, const uint32_t *__restrict__ ja, const T *__restrict__ A,
                                           const double *__restrict__ b, double *x, int base, int gl,
                                           unsigned gmask)
{
  constexpr int S = G / 4;   // block slots per step
  const int jj = gl >> 2, r = gl & 3;
  const uint32_t i = d.x, jb = d.y, je = d.z;
  double xi = UPPER ? __ldcg(x + 4 * (size_t)i + r) : b[4 * (size_t)i + r];
  for (uint32_t c0 = jb; c0 < je; c0 += 4 * S) {
    double t[4];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const uint32_t j = c0 + S * p + jj;
      t[p] = 0.0;
      if (j < je) {
        const uint32_t col = ja[j];
        const T *blk = A + 16 * (size_t)j + 4 * r;
        const double2 x01 = __ldcg(reinterpret_cast<const double2 *>(x) + 2 * (size_t)col);
        const double2 x23 = __ldcg(reinterpret_cast<const double2 *>(x) + 2 * (size_t)col + 1);
        double s = 0.0;
        s += (double)blk[0] * x01.x;
        s += (double)blk[1] * x01.y;
        s += (double)blk[2] * x23.x;
        s += (double)blk[3] * x23.y;
        t[p] = s;
      }
    }
    const uint32_t cnt = (je - c0) < (uint32_t)(4 * S) ? (je - c0) : (uint32_t)(4 * S);
#pragma unroll
    for (int p = 0; p < 4; p++)
      for (int q = 0; q < S; q++) {
        if ((uint32_t)(S * p + q) >= cnt) break;
        xi = -1.0 * __shfl_sync(gmask, t[p], base + 4 * q + r) + xi;
      }
  }
  if (UPPER) {
    const double x0 = __shfl_sync(gmask, xi, base + 0), x1 = __shfl_sync(gmask, xi, base + 1);
    const double x2 = __shfl_sync(gmask, xi, base + 2), x3 = __shfl_sync(gmask, xi, base + 3);
    const T *dg = A + 16 * (size_t)(jb - 1) + 4 * r;
    double y = 0.0;
    y += (double)dg[0] * x0;
    y += (double)dg[1] * x1;
    y += (double)dg[2] * x2;
    y += (double)dg[3] * x3;
    xi = y;
  }
  if (gl < 4) __stcg(x + 4 * (size_t)i + r, xi);
}

// Both sweeps in one cooperative launch: the rows of each level are spread
// over every half-warp of the grid, and a grid barrier (kf_grid_barrier,
// bounded) separates consecutive levels.  Arithmetic as in trsv_row16.
template <typename T>
__global__ void __launch_bounds__(256, 4) k_trsv_persistent(const uint32_t *__restrict__ lev_l, uint32_t nl,
                                                            const uint32_t *__restrict__ lev_u, uint32_t nu,
                                                            const uint4 *__restrict__ desc_l,
                                                            const uint4 *__restrict__ desc_u,
                                                            const uint32_t *__restrict__ ja, const T *__restrict__ A,
                                                            const double *__restrict__ b, double *x, unsigned *bar,
                                                            int *err)
{
  const int lane = threadIdx.x & 31, half = lane >> 4, l16 = lane & 15, jj = l16 >> 2, r = l16 & 3;
  const unsigned hmask = 0xffffu << (16 * half);
  const uint32_t H = gridDim.x * (blockDim.x >> 4);
  const uint32_t h = blockIdx.x * (blockDim.x >> 4) + (threadIdx.x >> 4);
  for (uint32_t l = 0; l < nl; l++) {
    const uint32_t s1 = lev_l[l + 1];
    for (uint32_t s = lev_l[l] + h; s < s1; s += H)
      trsv_row16<T, false>(desc_l[s], ja, A, b, x, half, jj, r, l16, hmask);
    __threadfence();
    if (!kf_grid_barrier(bar, err)) return;
  }
  for (uint32_t l = 0; l < nu; l++) {
    const uint32_t s1 = lev_u[l + 1];
    for (uint32_t s = lev_u[l] + h; s < s1; s += H)
      trsv_row16<T, true>(desc_u[s], ja, A, b, x, half, jj, r, l16, hmask);
    __threadfence();
    if (l + 1 < nu && !kf_grid_barrier(bar, err)) return;
  }
}

// Grid barrier on a counter that only grows within one launch (cleared before
// it): every CTA adds one on arrival and waits, bounded, until the counter
// reaches target = (barriers passed so far) x (CTAs).  One atomic per CTA, no
// generation word to flip.  The CTA barrier before the arrival and thread 0's
// fences order every thread's earlier stores before the arrival and every
// later load after the wait (the cumulative fence pattern of a grid sync), so
// the threads themselves need no fence.
__device__ __forceinline__ bool kf_mono_barrier(unsigned *cnt, unsigned target, int *err)
{
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    atomicAdd(cnt, 1u);
    unsigned spins = 0, v = 0;
    while (true) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
      if (v >= target) break;
      if (++spins > KF_BARRIER_LIMIT) { atomicExch(err, 1); ok = 0; break; }
      if ((spins & 255) == 0 && *(volatile int *)err) { ok = 0; break; }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// Both sweeps in one cooperative launch of MINB 512-thread CTAs per SM;
// levels separated by kf_mono_barrier.  Arithmetic as in trsv_row16.
template <typename T, int MINB, int G>
__global__ void __launch_bounds__(512, MINB) k_trsv_persistent_mono(const uint32_t *__restrict__ lev_l, uint32_t nl,
                                                                 const uint32_t *__restrict__ lev_u, uint32_t nu,
                                                                 const uint4 *__restrict__ desc_l,
                                                                 const uint4 *__restrict__ desc_u,
                                                                 const uint32_t *__restrict__ ja,
                                                                 const T *__restrict__ A,
                                                                 const double *__restrict__ b, double *x,
                                                                 unsigned *cnt, int *err)
{
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), base = lane - gl;
  const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << base;
  const uint32_t H = gridDim.x * (blockDim.x / G);
  const uint32_t h = blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
  unsigned passed = 0;
  for (uint32_t l = 0; l < nl; l++) {
    const uint32_t s1 = lev_l[l + 1];
    uint32_t s = lev_l[l] + h;
    for (; s < s1; s += H) trsv_row_g<T, false, G>(desc_l[s], ja, A, b, x, base, gl, gmask);
    if (!kf_mono_barrier(cnt, ++passed * gridDim.x, err)) return;
  }
  for (uint32_t l = 0; l < nu; l++) {
    const uint32_t s1 = lev_u[l + 1];
    uint32_t s = lev_u[l] + h;
    for (; s < s1; s += H) trsv_row_g<T, true, G>(desc_u[s], ja, A, b, x, base, gl, gmask);
    if (l + 1 < nu && !kf_mono_barrier(cnt, ++passed * gridDim.x, err)) return;
  }
}

// Level-synchronous sweep with programmatic dependent launch: each level's
// kernel lets the next one start at once (griddepcontrol.launch_dependents);
// the next kernel loads everything that does not depend on earlier levels --
// its row descriptor, the columns and the factor blocks (final since the
// factorisation, which completed before this solve began) -- and only then
// waits for the previous level's grid (griddepcontrol.wait) before reading x.
// Arithmetic as in trsv_row16.  Rows with more than 16 blocks take a second
// pass after the wait.
template <typename T, bool UPPER>
__global__ void __launch_bounds__(256) k_trsv_level_pdl(uint32_t s0, uint32_t s1, const uint4 *__restrict__ desc,
                                                        const uint32_t *__restrict__ ja, const T *__restrict__ A,
                                                        const double *__restrict__ b, double *x)
{
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t slot = s0 + (gid >> 4);
  const int lane = threadIdx.x & 31, half = lane >> 4, l16 = lane & 15, jj = l16 >> 2, r = l16 & 3;
  const unsigned hmask = 0xffffu << (16 * half);
  const bool active = slot < s1;
  uint4 d = make_uint4(0, 0, 0, 0);
  uint32_t col[4];
  double a[4][4];
  if (active) {
    d = desc[slot];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const uint32_t j = d.y + 4 * p + jj;
      col[p] = 0xffffffffu;
      a[p][0] = a[p][1] = a[p][2] = a[p][3] = 0.0;
      if (j < d.z) {
        col[p] = ja[j];
        const T *blk = A + 16 * (size_t)j + 4 * r;
        a[p][0] = (double)blk[0]; a[p][1] = (double)blk[1];
        a[p][2] = (double)blk[2]; a[p][3] = (double)blk[3];
      }
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (!active) return;
  const uint32_t i = d.x, jb = d.y, je = d.z;
  double xi = UPPER ? x[4 * (size_t)i + r] : b[4 * (size_t)i + r];
  for (uint32_t c0 = jb; c0 < je; c0 += 16) {
    double t[4];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const uint32_t j = c0 + 4 * p + jj;
      t[p] = 0.0;
      if (j < je) {
        uint32_t cc = col[p];
        double a0 = a[p][0], a1 = a[p][1], a2 = a[p][2], a3 = a[p][3];
        if (c0 != jb) {   // second pass (rows with more than 16 blocks)
          cc = ja[j];
          const T *blk = A + 16 * (size_t)j + 4 * r;
          a0 = (double)blk[0]; a1 = (double)blk[1]; a2 = (double)blk[2]; a3 = (double)blk[3];
        }
        const double4 xc = reinterpret_cast<const double4 *>(x)[cc];
        double s = 0.0;
        s += a0 * xc.x;
        s += a1 * xc.y;
        s += a2 * xc.z;
        s += a3 * xc.w;
        t[p] = s;
      }
    }
    const uint32_t cnt = (je - c0) < 16u ? (je - c0) : 16u;
#pragma unroll
    for (int p = 0; p < 4; p++)
      for (uint32_t q = 0; q < 4; q++) {
        if (4 * p + q >= cnt) break;
        xi = -1.0 * __shfl_sync(hmask, t[p], 16 * half + 4 * q + r) + xi;
      }
  }
  if (UPPER) {
    const int b4 = 16 * half;
    const double x0 = __shfl_sync(hmask, xi, b4 + 0), x1 = __shfl_sync(hmask, xi, b4 + 1);
    const double x2 = __shfl_sync(hmask, xi, b4 + 2), x3 = __shfl_sync(hmask, xi, b4 + 3);
    const T *dg = A + 16 * (size_t)(jb - 1) + 4 * r;
    double y = 0.0;
    y += (double)dg[0] * x0;
    y += (double)dg[1] * x1;
    y += (double)dg[2] * x2;
    y += (double)dg[3] * x3;
    xi = y;
  }
  if (l16 < 4) x[4 * (size_t)i + r] = xi;
}

// One launch per level with programmatic dependent launch, four lanes per
// row: lane r keeps component r and subtracts the row's block products one
// block at a time (each summed from zero, in block order: the arithmetic of
// trsv_row16), so there is no reduction across lanes and a level needs a
// quarter of the threads of k_trsv_level_pdl.  Before waiting for the
// previous level (griddepcontrol.wait) a row loads everything that does not
// depend on x: its descriptor, the columns and rows of its first 8 blocks,
// and its diagonal block (upper sweep) or right-hand side (lower sweep).
template <typename T, bool UPPER>
__global__ void __launch_bounds__(256) k_trsv_level_pdl4(uint32_t s0, uint32_t s1, const uint4 *__restrict__ desc,
                                                         const uint32_t *__restrict__ ja, const T *__restrict__ A,
                                                         const double *__restrict__ b, double *x)
{
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t slot = s0 + (gid >> 2);
  const int r = threadIdx.x & 3, base = (threadIdx.x & 31) & ~3;
  const unsigned gmask = 0xfu << base;
  const bool active = slot < s1;
  uint4 d = make_uint4(0, 0, 0, 0);
  uint32_t nb = 0;
  uint32_t col[8];
  T a[8][4], dg[4];
  double xi = 0.0;
  if (active) {
    d = desc[slot];
    nb = d.z - d.y < 8u ? d.z - d.y : 8u;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      col[c] = 0;
#pragma unroll
      for (int e = 0; e < 4; e++) a[c][e] = (T)0;
      if ((uint32_t)c < nb) {
        col[c] = ja[d.y + c];
        const T *blk = A + 16 * (size_t)(d.y + c) + 4 * r;
#pragma unroll
        for (int e = 0; e < 4; e++) a[c][e] = blk[e];
      }
    }
    if (UPPER) {
      const T *blk = A + 16 * (size_t)(d.y - 1) + 4 * r;
#pragma unroll
      for (int e = 0; e < 4; e++) dg[e] = blk[e];
    } else {
      xi = b[4 * (size_t)d.x + r];
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (!active) return;
  if (UPPER) xi = x[4 * (size_t)d.x + r];
#pragma unroll
  for (int c = 0; c < 8; c++) {
    if ((uint32_t)c < nb) {
      const double4 xc = reinterpret_cast<const double4 *>(x)[col[c]];
      double sum = 0.0;
      sum += (double)a[c][0] * xc.x;
      sum += (double)a[c][1] * xc.y;
      sum += (double)a[c][2] * xc.z;
      sum += (double)a[c][3] * xc.w;
      xi = -1.0 * sum + xi;
    }
  }
  for (uint32_t j = d.y + 8; j < d.z; j++) {
    const double4 xc = reinterpret_cast<const double4 *>(x)[ja[j]];
    const T *blk = A + 16 * (size_t)j + 4 * r;
    double sum = 0.0;
    sum += (double)blk[0] * xc.x;
    sum += (double)blk[1] * xc.y;
    sum += (double)blk[2] * xc.z;
    sum += (double)blk[3] * xc.w;
    xi = -1.0 * sum + xi;
  }
  if (UPPER) {
    const double x0 = __shfl_sync(gmask, xi, base + 0), x1 = __shfl_sync(gmask, xi, base + 1);
    const double x2 = __shfl_sync(gmask, xi, base + 2), x3 = __shfl_sync(gmask, xi, base + 3);
    double y = 0.0;
    y += (double)dg[0] * x0;
    y += (double)dg[1] * x1;
    y += (double)dg[2] * x2;
    y += (double)dg[3] * x3;
    xi = y;
  }
  x[4 * (size_t)d.x + r] = xi;
}

// ------------------------------------------------------------------ packed level schedule

// Copies the factor's blocks into the packed stream of one sweep: stream
// position k takes matrix block src[k] (16-byte words, one per thread).
template <typename T>
__global__ void __launch_bounds__(256) k_trsv_pack(uint32_t nblk, const uint32_t *__restrict__ src,
                                                   const T *__restrict__ A, T *__restrict__ P)
{
  constexpr uint32_t V = 16 * sizeof(T) / 16;   // 16-byte words per block
  const size_t gid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (gid >= (size_t)nblk * V) return;
  const uint32_t k = (uint32_t)(gid / V), w = (uint32_t)(gid % V);
  const uint4 v = __ldcs(reinterpret_cast<const uint4 *>(A + 16 * (size_t)__ldg(src + k)) + w);
  reinterpret_cast<uint4 *>(P + 16 * (size_t)k)[w] = v;
}

// Row r (0..3) of a 4x4 block in shared memory, widened to double.
__device__ __forceinline__ void block_row(const float *a, double &a0, double &a1, double &a2, double &a3)
{
  const float4 v = *reinterpret_cast<const float4 *>(a);
  a0 = v.x; a1 = v.y; a2 = v.z; a3 = v.w;
}
__device__ __forceinline__ void block_row(const double *a, double &a0, double &a1, double &a2, double &a3)
{
  const double2 u = reinterpret_cast<const double2 *>(a)[0], v = reinterpret_cast<const double2 *>(a)[1];
  a0 = u.x; a1 = u.y; a2 = v.x; a3 = v.y;
}

#ifndef KF_PK_GATHER
#define KF_PK_GATHER 4   // column states gathered at once per row (8 measured slower: fewer rows in flight)
#endif

// One level of the packed schedule (matrix/sptrsv.cpp:173-209), one CTA per
// chunk (up to ROWS rows of the level, four lanes per row, lane r = component
// r).  Before the previous level has finished (griddepcontrol.wait) the CTA
// stages its chunk of the packed factor -- one contiguous run -- into shared
// memory with a single bulk copy, and loads the chunk's columns, rows and
// (lower sweep) right-hand side; after it, it gathers the final x of the
// columns (KF_PK_GATHER at a time) and subtracts the block products in column order,
// each product summed from zero in component order as the reference does.
// The upper sweep then applies the inverted diagonal block (the first block
// of the row's run).  The chunk's blocks in shared memory: 16 T each, then
// their columns.  With perm (matrix row -> mesh node, a renumbered pattern)
// the lower sweep reads b at the row's node and the upper sweep also writes
// the row's result at its node into xout: the permutations of the right-hand
// side and of the solution without passes of their own.
template <typename T, bool UPPER, int ROWS>
__global__ void __launch_bounds__(4 * ROWS, 256 / ROWS) k_trsv_packed(uint32_t c0, const uint4 *__restrict__ chunk,
                                                        const uint32_t *__restrict__ prow,
                                                        const uint32_t *__restrict__ pfirst,
                                                        const uint32_t *__restrict__ pcol, const T *__restrict__ pk,
                                                        const double *__restrict__ b, double *x,
                                                        const uint32_t *__restrict__ perm, double *xout, int *err)
{
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const uint4 ch = chunk[c0 + blockIdx.x];
  const uint32_t nblk = ch.w - ch.z;
  T *sa = reinterpret_cast<T *>(smem);
  uint32_t *sc = reinterpret_cast<uint32_t *>(smem + (size_t)nblk * 16 * sizeof(T));
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_expect_tx(&mbar, nblk * 16u * (unsigned)sizeof(T));
    if (nblk) bulk_g2s(sa, pk + 16 * (size_t)ch.z, nblk * 16u * (unsigned)sizeof(T), &mbar);
  }
  for (uint32_t k = threadIdx.x; k < nblk; k += blockDim.x) sc[k] = __ldg(pcol + ch.z + k);
  const uint32_t s = ch.x + (threadIdx.x >> 2);
  const int r = threadIdx.x & 3, base = (threadIdx.x & 31) & ~3;
  const bool active = s < ch.y;
  uint32_t row = 0, k0 = 0, k1 = 0, node = 0;
  double xi = 0.0;
  if (active) {
    row = __ldg(prow + s);
    k0 = __ldg(pfirst + s) - ch.z;
    k1 = __ldg(pfirst + s + 1) - ch.z;
    node = perm ? __ldg(perm + row) : row;
    if (!UPPER) xi = b[4 * (size_t)node + r];
  }
  __syncthreads();   // the columns and the barrier's initialisation, for every thread
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (!mbar_wait(&mbar, 0, err)) return;
  if (!active) return;
  uint32_t k = k0;
  if (UPPER) {
    xi = __ldcg(x + 4 * (size_t)row + r);
    k = k0 + 1;
  }
  const double2 *x2 = reinterpret_cast<const double2 *>(x);
  for (; k < k1; k += KF_PK_GATHER) {
    double2 lo[KF_PK_GATHER], hi[KF_PK_GATHER];
#pragma unroll
    for (int c = 0; c < KF_PK_GATHER; c++) {
      if (k + c < k1) {
        const size_t col = sc[k + c];
        lo[c] = __ldcg(x2 + 2 * col);
        hi[c] = __ldcg(x2 + 2 * col + 1);
      }
    }
#pragma unroll
    for (int c = 0; c < KF_PK_GATHER; c++) {
      if (k + c < k1) {
        double a0, a1, a2, a3;
        block_row(sa + 16 * (size_t)(k + c) + 4 * r, a0, a1, a2, a3);
        double sum = 0.0;
        sum += a0 * lo[c].x;
        sum += a1 * lo[c].y;
        sum += a2 * hi[c].x;
        sum += a3 * hi[c].y;
        xi = -1.0 * sum + xi;
      }
    }
  }
  if (UPPER) {
    const unsigned gmask = 0xfu << base;
    const double x0 = __shfl_sync(gmask, xi, base + 0), x1 = __shfl_sync(gmask, xi, base + 1);
    const double x2v = __shfl_sync(gmask, xi, base + 2), x3 = __shfl_sync(gmask, xi, base + 3);
    double a0, a1, a2, a3;
    block_row(sa + 16 * (size_t)k0 + 4 * r, a0, a1, a2, a3);
    double y = 0.0;
    y += a0 * x0;
    y += a1 * x1;
    y += a2 * x2v;
    y += a3 * x3;
    xi = y;
  }
  x[4 * (size_t)row + r] = xi;
  if (UPPER && xout) xout[4 * (size_t)node + r] = xi;
}

// ------------------------------------------------------------------ sync-free SpTRSV

// Bounded wait for a row's completion flag (device scope, acquire).
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p)
{
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v)
{
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr uint32_t KF_SPIN_LIMIT = 1u << 20;   // polls (about 0.1-0.5 s) before a wait is declared failed

// One triangular sweep without level barriers (matrix/sptrsv.cpp:34-73).
// Launched cooperatively, so every block of the grid is resident at once.
// Half-warp h (of H) owns the rows at level-order positions h, h+H, h+2H, ...
// and works them in that order.  desc[slot] = (row, first block, end block)
// in level order.  For a row, the 16 lanes (lane = 4*block + component) first
// load all of the row's blocks (up to KF_TRSV_MAXB, four per pass), then wait
// until each block's column row has published its result (flag == epoch),
// form the block-vector products, and subtract them from x_i in column order;
// every row's arithmetic is the reference's (products summed from zero in
// column order, subtracted in block order), only the schedule differs.
// Deadlock-free: the unfinished row with the smallest position has all its
// dependencies done, and its owner, being resident and having finished its
// earlier rows, is working on it.  A wait that exceeds KF_SPIN_LIMIT polls
// records an error in *err, after which every other wait gives up too.
constexpr int KF_TRSV_MAXB = 16;   // blocks per row held in registers (longer rows loop)

template <typename T, bool UPPER>
__global__ void __launch_bounds__(256, 4) k_trsv_syncfree(uint32_t N, const uint4 *__restrict__ desc,
                                                          const uint32_t *__restrict__ ja,
                                                          const T *__restrict__ A, const double *__restrict__ b,
                                                          double *x, uint32_t *flags, uint32_t epoch, int *err)
{
  const int lane = threadIdx.x & 31, half = lane >> 4, l16 = lane & 15, jj = l16 >> 2, r = l16 & 3;
  const unsigned hmask = 0xffffu << (16 * half);
  const uint32_t H = gridDim.x * (blockDim.x >> 4);
  const uint32_t h = blockIdx.x * (blockDim.x >> 4) + (threadIdx.x >> 4);
  for (uint32_t slot = h; slot < N; slot += H) {
    const uint4 d = desc[slot];
    const uint32_t i = d.x, jb = d.y, je = d.z;
    double xi = UPPER ? __ldcg(x + 4 * (size_t)i + r) : b[4 * (size_t)i + r];
    for (uint32_t c0 = jb; c0 < je; c0 += KF_TRSV_MAXB) {
      // 1. all loads that do not depend on other rows
      double a[4][4];
      uint32_t col[4];
#pragma unroll
      for (int p = 0; p < 4; p++) {
        const uint32_t j = c0 + 4 * p + jj;
        col[p] = 0xffffffffu;
        a[p][0] = a[p][1] = a[p][2] = a[p][3] = 0.0;
        if (j < je) {
          col[p] = ja[j];
          const T *blk = A + 16 * (size_t)j + 4 * r;
          a[p][0] = (double)blk[0]; a[p][1] = (double)blk[1];
          a[p][2] = (double)blk[2]; a[p][3] = (double)blk[3];
        }
      }
      // 2. wait for the column rows, then the products
      double t[4];
#pragma unroll
      for (int p = 0; p < 4; p++) {
        t[p] = 0.0;
        if (col[p] != 0xffffffffu) {
          uint32_t spins = 0;
          while (ld_acquire(flags + col[p]) != epoch) {
            if (++spins > KF_SPIN_LIMIT) { atomicExch(err, 1); break; }
            if ((spins & 63) == 0 && *(volatile int *)err) break;
          }
          const double2 x01 = __ldcg(reinterpret_cast<const double2 *>(x) + 2 * (size_t)col[p]);
          const double2 x23 = __ldcg(reinterpret_cast<const double2 *>(x) + 2 * (size_t)col[p] + 1);
          double s = 0.0;
          s += a[p][0] * x01.x;
          s += a[p][1] * x01.y;
          s += a[p][2] * x23.x;
          s += a[p][3] * x23.y;
          t[p] = s;
        }
      }
      // 3. subtract in column order
      const uint32_t cnt = (je - c0) < (uint32_t)KF_TRSV_MAXB ? (je - c0) : (uint32_t)KF_TRSV_MAXB;
#pragma unroll
      for (int p = 0; p < 4; p++)
        for (uint32_t q = 0; q < 4; q++) {
          if (4 * p + q >= cnt) break;
          const double tq = __shfl_sync(hmask, t[p], 16 * half + 4 * q + r);
          xi = -1.0 * tq + xi;
        }
    }
    if (UPPER) {
      const int b4 = 16 * half;
      const double x0 = __shfl_sync(hmask, xi, b4 + 0), x1 = __shfl_sync(hmask, xi, b4 + 1);
      const double x2 = __shfl_sync(hmask, xi, b4 + 2), x3 = __shfl_sync(hmask, xi, b4 + 3);
      const T *dg = A + 16 * (size_t)(jb - 1) + 4 * r;
      double y = 0.0;
      y += (double)dg[0] * x0;
      y += (double)dg[1] * x1;
      y += (double)dg[2] * x2;
      y += (double)dg[3] * x3;
      xi = y;
    }
    if (l16 < 4) {
      __stcg(x + 4 * (size_t)i + r, xi);
      __threadfence();
    }
    __syncwarp(hmask);
    if (l16 == 0) st_release(flags + i, epoch);
  }
}

// ------------------------------------------------------------------ J.v

// src/kernel.c:35-44: y = (y - r + cdt (w - q)) * a, a = |x| / h from the
// device scalars (scal[ia] = |x|, scal[ia+1] = h).
__global__ void k_jv_combine(uint32_t N, double *__restrict__ y, const double *__restrict__ r,
                             const double *__restrict__ w, const double *__restrict__ q,
                             const double *__restrict__ cdt, const double *__restrict__ scal, int ia)
{
  const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const double a = scal[ia] / scal[ia + 1];
  const double c = cdt[n];
  const double4 yy = reinterpret_cast<double4 *>(y)[n];
  const double4 rr = reinterpret_cast<const double4 *>(r)[n];
  const double4 ww = reinterpret_cast<const double4 *>(w)[n];
  const double4 qq = reinterpret_cast<const double4 *>(q)[n];
  double4 o;
  o.x = (yy.x - rr.x + c * (ww.x - qq.x)) * a;
  o.y = (yy.y - rr.y + c * (ww.y - qq.y)) * a;
  o.z = (yy.z - rr.z + c * (ww.z - qq.z)) * a;
  o.w = (yy.w - rr.w + c * (ww.w - qq.w)) * a;
  reinterpret_cast<double4 *>(y)[n] = o;
}

// ------------------------------------------------------------------ launchers

inline unsigned blocks(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// The least-squares coefficients of every node on the device (k_lsq_coef),
// and whether the terms recomputed from them equal the GEOMETRY's stored
// terms bit for bit (k_lsq_check).
int lsq_setup(DevMesh &m)
{
  if (!m.lsq_coef && cudaMalloc(&m.lsq_coef, 2 * (size_t)m.N * sizeof(double4)) != cudaSuccess) {
    cudaGetLastError();
    m.lsq_coef = nullptr;
    return KFUN3D_ERR_CUDA;
  }
  unsigned *bad = reinterpret_cast<unsigned *>(m.status + 2);
  if (cudaMemsetAsync(bad, 0, sizeof(unsigned), m.stream) != cudaSuccess) return KFUN3D_ERR_CUDA;
  k_lsq_coef<<<blocks(m.N, 128), 128, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_edge,
                                                     (const double4 *)m.xyz, m.lsq_coef);
  k_lsq_check<<<blocks(m.N, 128), 128, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_edge, m.inc_w,
                                                      m.wstride, (const double4 *)m.xyz, m.lsq_coef, bad);
  kf_count_launch(2);
  unsigned nbad = 1;
  if (cudaMemcpyAsync(&nbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, m.stream) != cudaSuccess ||
      cudaStreamSynchronize(m.stream) != cudaSuccess || cudaMemsetAsync(bad, 0, sizeof(unsigned), m.stream) != cudaSuccess)
    return KFUN3D_ERR_CUDA;
  m.lsq_match = nbad == 0;
  return KFUN3D_OK;
}

// The state's visit-order copy (when the residual passes use one).
static void visit_state(DevMesh &m, const double *q)
{
  if (!m.visit) return;
  const bool held = m.qv_of == q;
  m.qv_of = nullptr;
  if (held) return;
  k_visit_gather<<<blocks(m.N, 256), 256, 0, m.stream>>>(m.N, m.ord, (const double4 *)q, m.qv);
  kf_count_launch();
}

// Gradients of q (src/flux.c:60-145) into gx/gy/gz, or into their visit-order
// copies (m.visit; the residual reads those).  Kernel (KFUN3D_GRADIENT):
// four lanes per node (default on large meshes), one thread per node with
// the incidence staged into shared memory by bulk copies (default in the
// mesh's own order), "plain" one thread per node.
void gradient(DevMesh &m, const double *q)
{
  if (m.visit) {
    visit_state(m, q);
    k_gradient4<<<blocks(4 * (size_t)m.N, 256), 256, 0, m.stream>>>(m.N, nullptr, m.inc_ptr, m.inc_othv, m.inc_w,
                                                                     m.wstride, (const double *)m.qv,
                                                                     (double *)m.gxv, (double *)m.gyv,
                                                                     (double *)m.gzv);
    kf_count_launch();
    return;
  }
  if (m.grad_lanes == 4) {
    k_gradient4<<<blocks(4 * (size_t)m.N, 256), 256, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_w,
                                                                     m.wstride, q, m.gx, m.gy, m.gz);
    kf_count_launch();
    return;
  }
  if (m.grad_smem) {
    static bool attr_set = false;
    if (!attr_set) {
      cudaFuncSetAttribute(k_gradient_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      attr_set = true;
    }
    k_gradient_tma<<<blocks(m.N, 128), 128, m.grad_smem, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_w, m.wstride,
                                                                    (const double4 *)q, (double4 *)m.gx,
                                                                    (double4 *)m.gy, (double4 *)m.gz, m.status + 1);
  } else {
    k_gradient<<<blocks(m.N, 256), 256, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_w, m.wstride,
                                                        (const double4 *)q, (double4 *)m.gx,
                                                        (double4 *)m.gy, (double4 *)m.gz);
  }
  kf_count_launch();
}

// The gradients in the mesh's numbering (after gradient() wrote visit-order
// copies), for callers that read them back.
void gradient_to_mesh_order(DevMesh &m)
{
  if (!m.visit) return;
  const unsigned nb = blocks(m.N, 256);
  k_visit_scatter<<<nb, 256, 0, m.stream>>>(m.N, m.ord, m.gxv, (double4 *)m.gx);
  k_visit_scatter<<<nb, 256, 0, m.stream>>>(m.N, m.ord, m.gyv, (double4 *)m.gy);
  k_visit_scatter<<<nb, 256, 0, m.stream>>>(m.N, m.ord, m.gzv, (double4 *)m.gz);
  kf_count_launch(3);
}

// Residual of q into r.  With visit-order copies (m.visit) the edge pass
// reads the state, coordinates and gradients from them: the copy of q made
// by gradient() for the second-order flux, made here for the first order.
void residual(DevMesh &m, const double *q, double *r, int first_order, double u, double v)
{
  if (m.two_pass) {
    if (first_order) visit_state(m, q);
    const double4 *G[3] = {m.visit ? m.gxv : (const double4 *)m.gx, m.visit ? m.gyv : (const double4 *)m.gy,
                           m.visit ? m.gzv : (const double4 *)m.gz};
    const double4 *Q = m.visit ? m.qv : (const double4 *)q;
    const double4 *X = m.visit ? m.xyzv : m.xyz;
    const uint32_t *E0 = m.visit ? m.n0v : m.n0s, *E1 = m.visit ? m.n1v : m.n1;
    {
      if (first_order)
        k_flux_edges<true><<<blocks(m.E, 128), 128, 0, m.stream>>>(m.E, E0, E1, m.egeo_s, X, Q, nullptr, nullptr,
                                                                    nullptr, m.eres);
      else
        k_flux_edges<false><<<blocks(m.E, 128), 128, 0, m.stream>>>(m.E, E0, E1, m.egeo_s, X, Q, G[0], G[1], G[2],
                                                                     m.eres);
      k_flux_nodes4<<<blocks(4 * (size_t)m.N, 256), 256, 0, m.stream>>>(m.N, m.ord, m.in1_ptr, m.in1_edge, m.eoff,
                                                                         (const double *)m.eres, r);
      kf_count_launch(2);
    }
  } else if (first_order)
    k_residual<true><<<blocks(m.N, 128), 128, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_edge, m.egeo, m.xyz,
                                                            (const double4 *)q, nullptr, nullptr, nullptr,
                                                            (double4 *)r);
  else
    k_residual<false><<<blocks(m.N, 128), 128, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_edge, m.egeo, m.xyz,
                                                             (const double4 *)q, (const double4 *)m.gx,
                                                             (const double4 *)m.gy, (const double4 *)m.gz,
                                                             (double4 *)r);
  if (!m.two_pass) kf_count_launch();
  if (m.nb) {
    k_residual_boundary<<<blocks(m.nb, 64), 64, 0, m.stream>>>(m.nb, m.bnd_node, m.bnd_ptr, m.bnd_ent, m.wf_nodes,
                                                               m.wf_n, m.f_n, (const double4 *)q, (double4 *)r, u, v);
    kf_count_launch();
  }
}

void timestep(DevMesh &m, const double *q, double cfl)
{
  if (m.visit && m.inc_geo) {
    visit_state(m, q);
    k_timestep<true><<<blocks(m.N, 256), 256, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_othv, m.inc_edge,
                                                              m.inc_geo, m.qv, m.bnd_of, cfl, m.cdt);
  } else {
    k_timestep<false><<<blocks(m.N, 256), 256, 0, m.stream>>>(m.N, m.ord, m.inc_ptr, m.inc_oth, m.inc_edge, m.egeo,
                                                               (const double4 *)q, m.bnd_of, cfl, m.cdt);
  }
  kf_count_launch();
  if (m.nb) {
    k_timestep_boundary<<<blocks(m.nb, 64), 64, 0, m.stream>>>(m.nb, m.bnd_node, m.bnd_ptr, m.bnd_ent, m.s_n,
                                                               m.f_n, (const double4 *)q, cfl, m.cdt);
    kf_count_launch();
  }
}

void fill(DevMesh &m, const double *q, double u, double v, int precision)
{
  const bool vis = m.visit && m.inc_geo;
  if (vis) visit_state(m, q);
  const uint32_t *oth = vis ? m.inc_othv : m.inc_oth;
  const double4 *geo = vis ? m.inc_geo : m.egeo, *qq = vis ? m.qv : (const double4 *)q;
  auto fill_fn = [&](auto *A, double *lslot, double *dscr) {
    using T = std::remove_pointer_t<decltype(A)>;
    if (vis)
      k_fill<T, true><<<blocks(m.N, 128), 128, 0, m.stream>>>(m.N, m.row_node, m.rowof, m.inc_ptr, oth, m.inc_edge,
                                                              m.fill_blk, geo, qq, m.cdt, m.fill_diag, m.fill_last,
                                                              m.fill_lpos, A, lslot, m.bnd_of, dscr);
    else
      k_fill<T, false><<<blocks(m.N, 128), 128, 0, m.stream>>>(m.N, m.row_node, m.rowof, m.inc_ptr, oth, m.inc_edge,
                                                               m.fill_blk, geo, qq, m.cdt, m.fill_diag, m.fill_last,
                                                               m.fill_lpos, A, lslot, m.bnd_of, dscr);
  };
  if (precision == 0) {
    fill_fn(m.A, m.lslot, nullptr);
    kf_count_launch();
    if (m.nb) {
      k_fill_boundary<double><<<blocks(m.nb, 64), 64, 0, m.stream>>>(m.nb, m.bnd_node, m.bnd_ptr, m.bnd_ent, m.s_n,
                                                                     m.f_n, (const double4 *)q, m.fill_diag, m.A, u, v,
                                                                     nullptr);
      kf_count_launch();
    }
  } else {
    fill_fn(m.Af, nullptr, m.dscr);
    kf_count_launch();
    if (m.nb) {
      k_fill_boundary<float><<<blocks(m.nb, 64), 64, 0, m.stream>>>(m.nb, m.bnd_node, m.bnd_ptr, m.bnd_ent, m.s_n,
                                                                    m.f_n, (const double4 *)q, m.fill_diag, m.Af, u, v,
                                                                    m.dscr);
      kf_count_launch();
    }
  }
}

static void packed_setup();

void ilu(DevMesh &m, int precision)
{
  int *status = m.status;
  if (m.sub_parts > 1 && m.sub_part) {
    if (precision == 0)
      k_drop_coupling<double><<<blocks(m.N, 256), 256, 0, m.stream>>>(m.N, m.ia, m.ja, m.row_node, m.sub_part, m.A);
    else
      k_drop_coupling<float><<<blocks(m.N, 256), 256, 0, m.stream>>>(m.N, m.ia, m.ja, m.row_node, m.sub_part, m.Af);
    kf_count_launch();
  }
  for (uint32_t l = 0; l < m.nlev_l; l++) {
    const uint32_t r0 = m.lev_l_ptr[l], nr = m.lev_l_ptr[l + 1] - r0;
    if (precision == 0 && m.pairs)
      k_ilu_level_pairs<<<blocks((size_t)nr * 16, 128), 128, 0, m.stream>>>(nr, m.lev_l + r0, m.ia, m.ja, m.diag,
                                                                            m.pair_ptr, m.pairs, m.lpos, m.A,
                                                                            m.lslot, m.dinv, status);
    else if (precision == 0)
      k_ilu_level<<<blocks((size_t)nr * 16, 128), 128, 0, m.stream>>>(nr, m.lev_l + r0, m.ia, m.ja, m.diag, m.tblk,
                                                                      m.lpos, m.A, m.lslot, m.dinv, status);
    else if (m.pairs)
      k_ilu_level_pairs_f32<<<blocks((size_t)nr * 16, 128), 128, 0, m.stream>>>(nr, m.lev_l + r0, m.ia, m.ja,
                                                                                m.pair_ptr, m.pairs, m.lpos, m.Af,
                                                                                m.dinvf, status);
    else
      k_ilu_level_f32<<<blocks((size_t)nr * 16, 128), 128, 0, m.stream>>>(nr, m.lev_l + r0, m.ia, m.ja, m.diag,
                                                                          m.tblk, m.Af, m.dinvf, status);
    kf_count_launch();
  }
  if (precision == 0)
    k_ilu_finish<<<blocks((size_t)m.N * 16, 256), 256, 0, m.stream>>>(m.N, m.ia, m.diag, m.lpos, m.lslot, m.dinv, m.A);
  else
    k_ilu_finish_f32<<<blocks((size_t)m.N * 16, 256), 256, 0, m.stream>>>(m.N, m.diag, m.dinvf, m.Af);
  kf_count_launch();
  if (m.trsv_mode == 8 && m.pk[0].chunk[0] && (precision == 1 || m.pk_fp64)) {
    packed_setup();
    for (int pass = 0; pass < 2; pass++) {
      const uint32_t nb = m.pk[pass].nblk, off = pass == 0 ? 0u : m.pk[0].nblk;
      if (precision == 0)
        k_trsv_pack<double><<<blocks((size_t)nb * 8, 256), 256, 0, m.stream>>>(
            nb, m.pk[pass].src, m.A, reinterpret_cast<double *>(m.pk_buf) + 16 * (size_t)off);
      else
        k_trsv_pack<float><<<blocks((size_t)nb * 4, 256), 256, 0, m.stream>>>(
            nb, m.pk[pass].src, m.Af, reinterpret_cast<float *>(m.pk_buf) + 16 * (size_t)off);
      kf_count_launch();
    }
  }
}

// Dynamic shared memory of k_trsv_packed for a chunk of `blocks` blocks.
template <typename T> static size_t packed_smem(uint32_t blocks)
{
  return (size_t)blocks * (16 * sizeof(T) + 4);
}

// The kernels' shared-memory limit, raised once to the largest chunk the
// schedule allows (a single row of KF_PK_ROW_MAX blocks).
static void packed_setup()
{
  static bool done = false;
  if (done) return;
  const int f32 = (int)packed_smem<float>(KF_PK_ROW_MAX), f64 = (int)packed_smem<double>(KF_PK_ROW_MAX);
  const void *fns32[] = {(const void *)k_trsv_packed<float, false, 32>, (const void *)k_trsv_packed<float, true, 32>,
                         (const void *)k_trsv_packed<float, false, 64>, (const void *)k_trsv_packed<float, true, 64>};
  const void *fns64[] = {(const void *)k_trsv_packed<double, false, 32>, (const void *)k_trsv_packed<double, true, 32>,
                         (const void *)k_trsv_packed<double, false, 64>, (const void *)k_trsv_packed<double, true, 64>};
  for (const void *f : fns32) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, f32);
  for (const void *f : fns64) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, f64);
  done = true;
}

// The bounded wait of the sync-free sweep on a flag nothing sets: gives up
// after KF_SPIN_LIMIT polls and records that in *err (bounded_wait_check).
__global__ void k_wait_on_flag(const uint32_t *flag, uint32_t value, int *err)
{
  if (threadIdx.x != 0) return;
  uint32_t spins = 0;
  while (ld_acquire(flag) != value) {
    if (++spins > KF_SPIN_LIMIT) { atomicExch(err, 1); return; }
  }
}

// Both sweeps of the packed schedule: one launch per level, chained by
// programmatic dependent launch (the first level of the lower sweep waits for
// the right-hand side normally).  The chunk cut (32 or 64 rows a CTA) is the
// one chosen for the factor's precision.
template <typename T>
static void sptrsv_packed(DevMesh &m, const double *b, double *x, const uint32_t *perm = nullptr,
                          double *xout = nullptr)
{
  packed_setup();
  int *err = m.status + 1;
  const T *base = reinterpret_cast<const T *>(m.pk_buf);
  const int cut = m.pk_cut[sizeof(T) == 8 ? 0 : 1];
  for (int pass = 0; pass < 2; pass++) {
    const PackedSweep &pk = m.pk[pass];
    const T *P = pass == 0 ? base : base + 16 * (size_t)m.pk[0].nblk;
    const void *fn = cut == 0 ? (pass == 0 ? (const void *)k_trsv_packed<T, false, 32> : (const void *)k_trsv_packed<T, true, 32>)
                              : (pass == 0 ? (const void *)k_trsv_packed<T, false, 64> : (const void *)k_trsv_packed<T, true, 64>);
    const size_t smem = packed_smem<T>(pk.maxblk[cut]);
    const uint4 *chunk = pk.chunk[cut];
    const std::vector<uint32_t> &lev = pk.lev[cut];
    for (size_t l = 0; l + 1 < lev.size(); l++) {
      uint32_t c0 = lev[l];
      const uint32_t nc = lev[l + 1] - c0;
      if (nc == 0) continue;
      const double *bb = b;
      double *xx = x;
      const uint32_t *pp = perm;
      double *xo = xout;
      void *args[] = {&c0,         (void *)&chunk, (void *)&pk.row, (void *)&pk.first, (void *)&pk.col, (void *)&P,
                      (void *)&bb, (void *)&xx,    (void *)&pp,     (void *)&xo,       (void *)&err};
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(nc);
      cfg.blockDim = dim3(cut == 0 ? 128 : 256);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = m.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = (pass == 0 && l == 0) ? 0 : 1;
      const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
      if (e != cudaSuccess) kf_set_error(KFUN3D_ERR_CUDA, cudaGetErrorString(e));
      kf_count_launch();
    }
  }
}

// x = P^T (LU)^-1 P b for a renumbered pattern (m.row_node) through the
// packed schedule, the permutations folded into its first and last sweeps;
// false (nothing done) when the active schedule is not the packed one.
bool sptrsv_permuted(DevMesh &m, const double *b, double *x, int precision)
{
  const int mode = (m.trsv_mode == 8 && precision == 0 && !m.pk_fp64) ? 7 : m.trsv_mode;
  if (mode != 8 || !m.pk[0].chunk[0] || !m.row_node) return false;
  if (precision == 0) sptrsv_packed<double>(m, b, m.px, m.row_node, x);
  else sptrsv_packed<float>(m, b, m.px, m.row_node, x);
  return true;
}

// The device-side bounded waits at work without a fault: a wait on a flag
// that nothing sets must give up (KFUN3D_ERR_TIMEOUT), and the same wait on a
// set flag must return at once, in the same context.  Anything else is an
// error code (KFUN3D_ERR_CUDA for a CUDA failure, KFUN3D_ERR_ARG if either
// wait behaved otherwise).
int bounded_wait_check(cudaStream_t st)
{
  uint32_t *flag = nullptr;
  int *err = nullptr;
  int h[2] = {0, 0};
  bool ok = cudaMalloc(&flag, sizeof(uint32_t)) == cudaSuccess && cudaMalloc(&err, 2 * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMemsetAsync(flag, 0, sizeof(uint32_t), st) == cudaSuccess &&
       cudaMemsetAsync(err, 0, 2 * sizeof(int), st) == cudaSuccess;
  if (ok) {
    k_wait_on_flag<<<1, 32, 0, st>>>(flag, 1u, err);       // nothing sets it: gives up
    k_wait_on_flag<<<1, 32, 0, st>>>(flag, 0u, err + 1);   // already set: returns at once
    kf_count_launch(2);
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(h, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
  }
  if (flag) cudaFree(flag);
  if (err) cudaFree(err);
  if (!ok) {
    cudaGetLastError();
    return KFUN3D_ERR_CUDA;
  }
  return (h[0] == 1 && h[1] == 0) ? KFUN3D_ERR_TIMEOUT : KFUN3D_ERR_ARG;
}

void sptrsv(DevMesh &m, const double *b, double *x, int precision)
{
  // the packed schedule serves FP32 factors; FP64 factors take the four-lane
  // level launches unless m.pk_fp64 (measured faster at 120^3 in both orders)
  const int mode = (m.trsv_mode == 8 && precision == 0 && !m.pk_fp64) ? 7 : m.trsv_mode;
  if (mode == 8 && m.pk[0].chunk[0]) {
    if (precision == 0) sptrsv_packed<double>(m, b, x);
    else sptrsv_packed<float>(m, b, x);
    return;
  }
  if (mode == 4 || mode == 7) {
    const bool four = mode == 7;   // four lanes per row (k_trsv_level_pdl4), else sixteen
    for (int pass = 0; pass < 2; pass++) {
      const std::vector<uint32_t> &ptr = pass == 0 ? m.lev_l_ptr : m.lev_u_ptr;
      const uint4 *desc = pass == 0 ? m.desc_l : m.desc_u;
      const void *Ap = precision == 0 ? (const void *)m.A : (const void *)m.Af;
      const void *fn;
      if (four && precision == 0)
        fn = pass == 0 ? (const void *)k_trsv_level_pdl4<double, false> : (const void *)k_trsv_level_pdl4<double, true>;
      else if (four)
        fn = pass == 0 ? (const void *)k_trsv_level_pdl4<float, false> : (const void *)k_trsv_level_pdl4<float, true>;
      else if (precision == 0)
        fn = pass == 0 ? (const void *)k_trsv_level_pdl<double, false> : (const void *)k_trsv_level_pdl<double, true>;
      else
        fn = pass == 0 ? (const void *)k_trsv_level_pdl<float, false> : (const void *)k_trsv_level_pdl<float, true>;
      for (size_t l = 0; l + 1 < ptr.size(); l++) {
        uint32_t s0 = ptr[l], s1 = ptr[l + 1];
        const double *bb = b;
        double *xx = x;
        void *args[] = {&s0, &s1, (void *)&desc, (void *)&m.ja, (void *)&Ap, (void *)&bb, (void *)&xx};
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(blocks((size_t)(s1 - s0) * (four ? 4 : 16), 256));
        cfg.blockDim = dim3(256);
        cfg.stream = m.stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        // the first level of the lower sweep waits normally for its right-hand side
        cfg.numAttrs = (pass == 0 && l == 0) ? 0 : 1;
        const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
        if (e != cudaSuccess) kf_set_error(KFUN3D_ERR_CUDA, cudaGetErrorString(e));
        kf_count_launch();
      }
    }
    return;
  }
  if (m.trsv_mode == 5) {
    const uint32_t *levl = m.lev_ptr_d, *levu = m.lev_ptr_d + m.nlev_l + 1;
    uint32_t nl = m.nlev_l, nu = m.nlev_u;
    const double *bb = b;
    unsigned *cnt = m.bar + 4;
    int *err = m.status + 1;
    cudaMemsetAsync(cnt, 0, sizeof(unsigned), m.stream);
    const void *Ap = precision == 0 ? (const void *)m.A : (const void *)m.Af;
    void *args[] = {(void *)&levl, &nl, (void *)&levu, &nu, (void *)&m.desc_l, (void *)&m.desc_u,
                    (void *)&m.ja, (void *)&Ap, (void *)&bb, (void *)&x, (void *)&cnt, (void *)&err};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(m.trsv_mgrid);
    cfg.blockDim = dim3(512);
    cfg.stream = m.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // instance for (precision, CTAs per SM, lanes per row)
    auto pick = [&](auto ctas) -> const void * {
      constexpr int C = decltype(ctas)::value;
      switch (m.trsv_lanes) {
        case 4: return precision == 0 ? (const void *)k_trsv_persistent_mono<double, C, 4>
                                      : (const void *)k_trsv_persistent_mono<float, C, 4>;
        case 16: return precision == 0 ? (const void *)k_trsv_persistent_mono<double, C, 16>
                                       : (const void *)k_trsv_persistent_mono<float, C, 16>;
        default: return precision == 0 ? (const void *)k_trsv_persistent_mono<double, C, 8>
                                       : (const void *)k_trsv_persistent_mono<float, C, 8>;
      }
    };
    const void *fn = m.trsv_mgrid_per == 1 ? pick(std::integral_constant<int, 1>())
                   : m.trsv_mgrid_per == 3 ? pick(std::integral_constant<int, 3>())
                                           : pick(std::integral_constant<int, 2>());
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    if (e != cudaSuccess) kf_set_error(KFUN3D_ERR_CUDA, cudaGetErrorString(e));
    kf_count_launch();
    return;
  }
  if (m.trsv_mode == 3) {
    const uint32_t *levl = m.lev_ptr_d, *levu = m.lev_ptr_d + m.nlev_l + 1;
    uint32_t nl = m.nlev_l, nu = m.nlev_u;
    const double *bb = b;
    unsigned *bar = m.bar;
    int *err = m.status + 1;
    const void *Ap = precision == 0 ? (const void *)m.A : (const void *)m.Af;
    void *args[] = {(void *)&levl, &nl, (void *)&levu, &nu, (void *)&m.desc_l, (void *)&m.desc_u,
                    (void *)&m.ja, (void *)&Ap, (void *)&bb, (void *)&x, (void *)&bar, (void *)&err};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(m.trsv_grid);
    cfg.blockDim = dim3(256);
    cfg.stream = m.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const void *fn = precision == 0 ? (const void *)k_trsv_persistent<double> : (const void *)k_trsv_persistent<float>;
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    if (e != cudaSuccess) kf_set_error(KFUN3D_ERR_CUDA, cudaGetErrorString(e));
    kf_count_launch();
    return;
  }
  if (m.syncfree) {
    // flags restart from zero on every solve (graph-capturable); epoch 1
    // marks rows done in the lower sweep, 2 in the upper sweep
    cudaMemsetAsync(m.flags, 0, (size_t)m.N * sizeof(uint32_t), m.stream);
    const double *bb = b;
    uint32_t N = m.N, eL = 1, eU = 2;
    int *err = m.status + 1;
    auto launch = [&](const void *fn, const uint4 *desc, uint32_t *e) {
      const void *Ap = precision == 0 ? (const void *)m.A : (const void *)m.Af;
      void *args[] = {&N, (void *)&desc, (void *)&m.ja, (void *)&Ap, (void *)&bb, (void *)&x, (void *)&m.flags,
                      e, (void *)&err};
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(m.trsv_grid);
      cfg.blockDim = dim3(256);
      cfg.stream = m.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeCooperative;
      attr[0].val.cooperative = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      const cudaError_t e2 = cudaLaunchKernelExC(&cfg, fn, args);
      if (e2 != cudaSuccess) kf_set_error(KFUN3D_ERR_CUDA, cudaGetErrorString(e2));
    };
    if (precision == 0) {
      launch((const void *)k_trsv_syncfree<double, false>, m.desc_l, &eL);
      launch((const void *)k_trsv_syncfree<double, true>, m.desc_u, &eU);
    } else {
      launch((const void *)k_trsv_syncfree<float, false>, m.desc_l, &eL);
      launch((const void *)k_trsv_syncfree<float, true>, m.desc_u, &eU);
    }
    kf_count_launch(2);
    return;
  }
  for (uint32_t l = 0; l < m.nlev_l; l++) {
    const uint32_t r0 = m.lev_l_ptr[l], nr = m.lev_l_ptr[l + 1] - r0;
    if (precision == 0)
      k_trsv_lower<double><<<blocks((size_t)nr * 4, 128), 128, 0, m.stream>>>(nr, m.lev_l + r0, m.ia, m.ja, m.diag,
                                                                             m.A, b, x);
    else
      k_trsv_lower<float><<<blocks((size_t)nr * 4, 128), 128, 0, m.stream>>>(nr, m.lev_l + r0, m.ia, m.ja, m.diag,
                                                                            m.Af, b, x);
    kf_count_launch();
  }
  for (uint32_t l = 0; l < m.nlev_u; l++) {
    const uint32_t r0 = m.lev_u_ptr[l], nr = m.lev_u_ptr[l + 1] - r0;
    if (precision == 0)
      k_trsv_upper<double><<<blocks((size_t)nr * 4, 128), 128, 0, m.stream>>>(nr, m.lev_u + r0, m.ia, m.ja, m.diag,
                                                                             m.A, x);
    else
      k_trsv_upper<float><<<blocks((size_t)nr * 4, 128), 128, 0, m.stream>>>(nr, m.lev_u + r0, m.ia, m.ja, m.diag,
                                                                            m.Af, x);
    kf_count_launch();
  }
}

// The sync-free sweep with caller-supplied completion flags (N words, cleared
// here), for the allocation-free entry point in noalloc.cu.
void sptrsv_flags(DevMesh &m, const double *b, double *x, int precision, uint32_t *flags)
{
  cudaMemsetAsync(flags, 0, (size_t)m.N * sizeof(uint32_t), m.stream);
  const double *bb = b;
  uint32_t N = m.N, eL = 1, eU = 2;
  int *err = m.status + 1;
  auto launch = [&](const void *fn, const uint4 *desc, uint32_t *e) {
    const void *Ap = precision == 0 ? (const void *)m.A : (const void *)m.Af;
    void *args[] = {&N, (void *)&desc, (void *)&m.ja, (void *)&Ap, (void *)&bb, (void *)&x, (void *)&flags,
                    e, (void *)&err};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(m.trsv_grid);
    cfg.blockDim = dim3(256);
    cfg.stream = m.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e2 = cudaLaunchKernelExC(&cfg, fn, args);
    if (e2 != cudaSuccess) kf_set_error(KFUN3D_ERR_CUDA, cudaGetErrorString(e2));
  };
  if (precision == 0) {
    launch((const void *)k_trsv_syncfree<double, false>, m.desc_l, &eL);
    launch((const void *)k_trsv_syncfree<double, true>, m.desc_u, &eU);
  } else {
    launch((const void *)k_trsv_syncfree<float, false>, m.desc_l, &eL);
    launch((const void *)k_trsv_syncfree<float, true>, m.desc_u, &eU);
  }
  kf_count_launch(2);
}

void jv_combine(DevMesh &m, double *y, const double *r, const double *w, const double *q, const double *scal, int ia)
{
  k_jv_combine<<<blocks(m.N, 256), 256, 0, m.stream>>>(m.N, y, r, w, q, m.cdt, scal, ia);
  kf_count_launch();
}

}  // namespace KF_NS
