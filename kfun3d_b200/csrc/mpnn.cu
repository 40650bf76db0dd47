// kfun3d_b200: the learned right preconditioner -- an edge-based
// message-passing network (MPNN) evaluated and trained on fifth-generation
// tensor cores (tcgen05, BF16 operands, FP32 accumulators in tensor memory).
//
// Network, hidden width 32, every MLP two linear layers with a ReLU between:
//   h0  = enc([y/s, q])                                      nodes
//   for l = 1..3
//     m_r = edge_l([h_i, h_j, n_r, a_r])                     directed edges r = (i <- j)
//     h_l = h_{l-1} + node_l([h_{l-1,i}, sum_{r at i} m_r])  nodes
//   out = dec(h3)                                            nodes, 4 outputs
// y is the ILU(0)-preconditioned vector, s its RMS, q the flow state; n_r is
// the unit edge normal seen from i and a_r the dual-face area over the mesh's
// mean.  Every linear map is X~ W~^T with X~ = [X, 1, 0...]: the bias is the
// column of W~ at the ones feature, so a layer is one GEMM.
//
// Directed edges are the node-incidence (CSR) rows of the mesh: the rows of
// node i are contiguous, so the sum of messages is a segment sum (no atomics,
// deterministic), and the adjoint of "gather h_j" is a segment sum over the
// reverse rows.  Weight gradients are per-CTA tensor-memory accumulators
// summed over CTAs in a fixed order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_bf16.h>

#include "internal.h"
#include "umma.cuh"

using bf16 = __nv_bfloat16;
using namespace kf_umma;

namespace {

constexpr uint32_t BF16_ONE = 0x3F80u;

// ------------------------------------------------------------ parameters

// W~ matrices [out x kin], FP32 master copy in one vector.
enum {
  L_ENC1 = 0, L_ENC2 = 1,
  // layer l (0..2): edge1 2+4l, edge2 3+4l, node1 4+4l, node2 5+4l
  L_DEC1 = 14, L_DEC2 = 15, NLAYERS = 16
};
struct LayerShape { int out, kin, nreal; };   // nreal: inputs before the ones feature
constexpr LayerShape kShape[NLAYERS] = {
    {32, 16, 8}, {32, 48, 32},
    {32, 80, 68}, {32, 48, 32}, {32, 80, 64}, {32, 48, 32},
    {32, 80, 68}, {32, 48, 32}, {32, 80, 64}, {32, 48, 32},
    {32, 80, 68}, {32, 48, 32}, {32, 80, 64}, {32, 48, 32},
    {32, 48, 32}, {16, 48, 32}};

struct Offsets {
  int off[NLAYERS + 1];
  constexpr Offsets() : off()
  {
    int o = 0;
    for (int i = 0; i < NLAYERS; i++) { off[i] = o; o += kShape[i].out * kShape[i].kin; }
    off[NLAYERS] = o;
  }
};
constexpr Offsets kOff{};
constexpr int NPARAM = kOff.off[NLAYERS];
constexpr int L_EDGE1(int l) { return 2 + 4 * l; }
constexpr int L_NODE1(int l) { return 4 + 4 * l; }

__constant__ int c_off[NLAYERS + 1];
__constant__ int c_out[NLAYERS];
__constant__ int c_kin[NLAYERS];

// ------------------------------------------------------------ small helpers

__device__ __forceinline__ uint32_t pack2(float a, float b)
{
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}
__device__ __forceinline__ float lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

__device__ __forceinline__ void unpack8(uint4 c, float *f)
{
  f[0] = lo(c.x); f[1] = hi(c.x); f[2] = lo(c.y); f[3] = hi(c.y);
  f[4] = lo(c.z); f[5] = hi(c.z); f[6] = lo(c.w); f[7] = hi(c.w);
}
__device__ __forceinline__ uint4 pack8(const float *f)
{
  return make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
}

__device__ __forceinline__ void st_chunk(unsigned char *tile, int row, int c, int K, uint4 v)
{
  *reinterpret_cast<uint4 *>(tile + kmajor_offset(row, 8 * c, K)) = v;
}
// element (f, r) of a transposed 128 x 128 tile (features x rows)
__device__ __forceinline__ void st_t(unsigned char *tile, int f, int r, uint16_t bits)
{
  *reinterpret_cast<uint16_t *>(tile + kmajor_offset(f, r, 128)) = bits;
}
__device__ __forceinline__ void st_t_chunk(unsigned char *tile, int f0, int r, uint4 v)
{
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    st_t(tile, f0 + 2 * i, r, (uint16_t)(w[i] & 0xFFFFu));
    st_t(tile, f0 + 2 * i + 1, r, (uint16_t)(w[i] >> 16));
  }
}

__device__ __forceinline__ void sync_tc()
{
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
}

// ------------------------------------------------------------ graph

struct GraphDev {
  uint32_t N = 0, R = 0;
  uint32_t *seg = nullptr;     // [N+1] rows of each node
  uint32_t *rnode = nullptr;   // [R] receiving node i
  uint32_t *oth = nullptr;     // [R] sending node j
  uint32_t *rev = nullptr;     // [R] row of (j <- i)
  uint2 *efeat = nullptr;      // [R] BF16 (n_x, n_y, n_z, a / mean a) seen from i
  // tiles of whole nodes for the edge MLP with the message sum in its
  // epilogue: (first row, rows <= 128, first node, nodes); null when a node
  // has more than 128 rows
  uint4 *plan = nullptr;
  uint32_t nplan = 0;
};

// ------------------------------------------------------------ gathers (X rows)

struct GatherEnc {   // [x0 (8), 1, 0 x 7]
  const uint4 *x0;
  __device__ void load(uint32_t i, uint4 *c) const
  {
    c[0] = x0[i];
    c[1] = make_uint4(BF16_ONE, 0, 0, 0);
  }
};

struct GatherEdge {   // [h_i (32), h_j (32), n (3), a, 1, 0 x 11]
  const uint4 *h;
  const uint32_t *rnode, *oth;
  const uint2 *efeat;
  __device__ void load(uint32_t r, uint4 *c) const
  {
    const uint32_t i = rnode[r], j = oth[r];
#pragma unroll
    for (int k = 0; k < 4; k++) c[k] = h[4 * (size_t)i + k];
#pragma unroll
    for (int k = 0; k < 4; k++) c[4 + k] = h[4 * (size_t)j + k];
    const uint2 e = efeat[r];
    c[8] = make_uint4(e.x, e.y, BF16_ONE, 0);
    c[9] = make_uint4(0, 0, 0, 0);
  }
};

// [h_i (32), sum of messages (32, rounded to BF16), 1, 0 x 15].  With agg_out
// the rounded sums are saved; with agg_in they are read instead of summed.
struct GatherNode {
  const uint4 *h;
  const uint32_t *seg;
  const uint4 *msg;
  uint4 *agg_out;
  const uint4 *agg_in;
  __device__ void load(uint32_t i, uint4 *c) const
  {
#pragma unroll
    for (int k = 0; k < 4; k++) c[k] = h[4 * (size_t)i + k];
    if (agg_in) {
#pragma unroll
      for (int k = 0; k < 4; k++) c[4 + k] = agg_in[4 * (size_t)i + k];
    } else {
      float s[32];
#pragma unroll
      for (int k = 0; k < 32; k++) s[k] = 0.f;
      const uint32_t r0 = seg[i], r1 = seg[i + 1];
      for (uint32_t r = r0; r < r1; r++) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          float f[8];
          unpack8(msg[4 * (size_t)r + k], f);
#pragma unroll
          for (int u = 0; u < 8; u++) s[8 * k + u] += f[u];
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) c[4 + k] = pack8(s + 8 * k);
      if (agg_out) {
#pragma unroll
        for (int k = 0; k < 4; k++) agg_out[4 * (size_t)i + k] = c[4 + k];
      }
    }
    c[8] = make_uint4(BF16_ONE, 0, 0, 0);
    c[9] = make_uint4(0, 0, 0, 0);
  }
};

struct GatherDec {   // [h (32), 1, 0 x 15]
  const uint4 *h;
  __device__ void load(uint32_t i, uint4 *c) const
  {
#pragma unroll
    for (int k = 0; k < 4; k++) c[k] = h[4 * (size_t)i + k];
    c[4] = make_uint4(BF16_ONE, 0, 0, 0);
    c[5] = make_uint4(0, 0, 0, 0);
  }
};

// ------------------------------------------------------------ forward outputs

struct OutBf16 {   // rows of 32 BF16
  uint4 *dst;
  __device__ void store(uint32_t r, const float *v) const
  {
#pragma unroll
    for (int k = 0; k < 4; k++) dst[4 * (size_t)r + k] = pack8(v + 8 * k);
  }
};

// The edge MLP's messages summed per receiving node inside the tile (tiles of
// whole nodes, OutSegSum::plan): each row's message rounded to BF16, then per
// node and component the FP32 sum over the node's rows in row order from
// zero, rounded to BF16 -- what GatherNode forms from stored messages, so the
// node MLP reads the sums (agg_in) and the messages never reach memory.
struct OutSegSum {
  const uint4 *plan;        // per tile: (first row, rows, first node, nodes)
  const uint32_t *seg;      // [N+1] first row of each node
  uint16_t *agg;            // [N][32] BF16
  uint32_t ntiles;
};
template <class O> struct SegSum { static constexpr bool value = false; };
template <> struct SegSum<OutSegSum> { static constexpr bool value = true; };

struct OutResidual {   // dst = BF16(src + v)
  const uint4 *src;
  uint4 *dst;
  __device__ void store(uint32_t r, const float *v) const
  {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float f[8];
      unpack8(src[4 * (size_t)r + k], f);
#pragma unroll
      for (int u = 0; u < 8; u++) f[u] += v[8 * k + u];
      dst[4 * (size_t)r + k] = pack8(f);
    }
  }
};

struct OutDecTrain {   // out[4i + c] = v[c]
  float4 *out;
  __device__ void store(uint32_t i, const float *v) const { out[i] = make_float4(v[0], v[1], v[2], v[3]); }
};

struct OutDecApply {   // z = y + s out (FP64), s = scal[0]
  const double *y;
  double *z;
  const double *scal;
  __device__ void store(uint32_t i, const float *v) const
  {
    const double s = scal[0];
#pragma unroll
    for (int c = 0; c < 4; c++) z[4 * (size_t)i + c] = y[4 * (size_t)i + c] + s * (double)v[c];
  }
};

// ------------------------------------------------------------ forward kernel

// Y = MLP(X) for `rows` rows: H = ReLU(X~ W1~^T) (32 wide), Y = H~ W2~^T (N2 wide).
// One 128-row tile at a time per CTA (persistent); thread t owns row t of the
// tile and TMEM lane t.  a1_save (optional) keeps H for the backward pass.
template <int K1, int N2>
constexpr size_t fwd_smem() { return (size_t)128 * K1 * 2 + 128 * 48 * 2 + 32 * K1 * 2 + N2 * 48 * 2; }

template <int K1, int N2, class G, class O>
__global__ void __launch_bounds__(128) k_mlp_fwd(G gat, O out, uint32_t rows, const uint4 *__restrict__ W1,
                                                 const uint4 *__restrict__ W2, uint4 *__restrict__ a1_save,
                                                 int *__restrict__ err)
{
  static_assert(K1 % 16 == 0 && K1 <= 128 && (N2 == 16 || N2 == 32), "shape");
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *Xs = smem;                    // 128 x K1
  unsigned char *Hs = Xs + 128 * K1 * 2;       // 128 x 48
  unsigned char *W1s = Hs + 128 * 48 * 2;      // 32 x K1
  unsigned char *W2s = W1s + 32 * K1 * 2;      // N2 x 48
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int s_abort;
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) tmem_alloc(&tslot, 64);
  if (t == 0) {
    mbar_init1(&mbar);
    s_abort = 0;
  }
  for (int idx = t; idx < 32 * K1 / 8; idx += 128) st_chunk(W1s, idx / (K1 / 8), idx % (K1 / 8), K1, W1[idx]);
  for (int idx = t; idx < N2 * 6; idx += 128) st_chunk(W2s, idx / 6, idx % 6, 48, W2[idx]);
  st_chunk(Hs, t, 4, 48, make_uint4(BF16_ONE, 0, 0, 0));
  st_chunk(Hs, t, 5, 48, make_uint4(0, 0, 0, 0));
  fence_proxy_async();
  sync_tc();
  const uint32_t tm = tslot;
  const uint32_t lane = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  constexpr bool SEG = SegSum<O>::value;
  uint32_t ntiles = (rows + 127) / 128;
  if constexpr (SEG) ntiles = out.ntiles;
  // a tile's first row and row count (SEG: the plan's tiles of whole nodes)
  auto span = [&](uint32_t tile) -> uint2 {
    if constexpr (SEG) {
      const uint4 pl = out.plan[tile];
      return make_uint2(pl.x, pl.y);
    }
    const uint32_t r0 = tile * 128;
    return make_uint2(r0, rows - r0 < 128u ? rows - r0 : 128u);
  };
  // the next tile's rows are gathered into registers while this tile's GEMMs
  // and epilogues run (software pipeline of depth one)
  uint4 c[K1 / 8];
  auto gather = [&](uint32_t tile) {
    const uint2 sp = tile < ntiles ? span(tile) : make_uint2(0, 0);
    if ((uint32_t)t < sp.y) gat.load(sp.x + t, c);
    else {
#pragma unroll
      for (int k = 0; k < K1 / 8; k++) c[k] = make_uint4(0, 0, 0, 0);
    }
  };
  gather(blockIdx.x);
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint2 sp = span(tile);
    const uint32_t row = sp.x + t;
    const bool valid = (uint32_t)t < sp.y;
#pragma unroll
    for (int k = 0; k < K1 / 8; k++) st_chunk(Xs, t, k, K1, c[k]);
    fence_proxy_async();
    sync_tc();
    if (t == 0) gemm_issue(tm, Xs, W1s, K1, 32, &mbar, false);
    gather(tile + gridDim.x);
    if (!mbar_try(&mbar, phase)) { atomicExch(err, 1); s_abort = 1; }
    phase ^= 1;
    fence_after_sync();
    {
      float v[32];
      tmem_ld32(tm + lane, v);
#pragma unroll
      for (int k = 0; k < 32; k++) v[k] = fmaxf(v[k], 0.f);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint4 p = pack8(v + 8 * k);
        st_chunk(Hs, t, k, 48, p);
        if (a1_save && valid) a1_save[4 * (size_t)row + k] = p;
      }
    }
    fence_proxy_async();
    sync_tc();
    if (t == 0) gemm_issue(tm + 32, Hs, W2s, 48, N2, &mbar, false);
    if (!mbar_try(&mbar, phase)) { atomicExch(err, 1); s_abort = 1; }
    phase ^= 1;
    fence_after_sync();
    {
      float v[32];
      if (N2 == 32) tmem_ld32(tm + lane + 32, v);
      else tmem_ld16(tm + lane + 32, v);
      if constexpr (SEG) {
        // the row's message rounded to BF16, staged in the X tile (free: the
        // first GEMM has completed and the next tile's rows are in registers)
        float *S = reinterpret_cast<float *>(Xs);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          float f[8];
          unpack8(pack8(v + 8 * k), f);
#pragma unroll
          for (int u = 0; u < 8; u++) S[32 * t + 8 * k + u] = f[u];
        }
        __syncthreads();
        const uint4 pl = out.plan[tile];
        const int l32 = t & 31;
        for (uint32_t j = (uint32_t)warp; j < pl.w; j += 4) {   // warp per node, lane per component
          const uint32_t node = pl.z + j;
          const uint32_t r0 = out.seg[node] - pl.x, r1 = out.seg[node + 1] - pl.x;
          float sum = 0.f;
          for (uint32_t r = r0; r < r1; r++) sum += S[32 * r + l32];
          const __nv_bfloat16 bsum = __float2bfloat16_rn(sum);
          out.agg[32 * (size_t)node + l32] = *reinterpret_cast<const uint16_t *>(&bsum);
        }
      } else {
        if (valid) out.store(row, v);
      }
    }
    sync_tc();
    if (s_abort) break;
  }
  sync_tc();
  if (warp == 0) tmem_dealloc(tm, 64);
}

// ------------------------------------------------------------ backward: dY sources

struct DYDense32 {   // dY row from an FP32 [rows x 32] array
  const float4 *g;
  __device__ void load(uint32_t r, float *d) const
  {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const float4 v = g[8 * (size_t)r + k];
      d[4 * k] = v.x; d[4 * k + 1] = v.y; d[4 * k + 2] = v.z; d[4 * k + 3] = v.w;
    }
  }
};

struct DYEdge {   // dY_r = dagg[rnode[r]]
  const float4 *dagg;
  const uint32_t *rnode;
  __device__ void load(uint32_t r, float *d) const
  {
    const uint32_t i = rnode[r];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const float4 v = dagg[8 * (size_t)i + k];
      d[4 * k] = v.x; d[4 * k + 1] = v.y; d[4 * k + 2] = v.z; d[4 * k + 3] = v.w;
    }
  }
};

struct DYLoss {   // d/d out of w * sum (out - target)^2
  const float4 *out, *tgt;
  float w;
  __device__ void load(uint32_t i, float *d) const
  {
    const float4 o = out[i], g = tgt[i];
    d[0] = 2.f * w * (o.x - g.x); d[1] = 2.f * w * (o.y - g.y);
    d[2] = 2.f * w * (o.z - g.z); d[3] = 2.f * w * (o.w - g.w);
#pragma unroll
    for (int k = 4; k < 16; k++) d[k] = 0.f;
  }
};

// ------------------------------------------------------------ backward: dX sinks (16 columns per call)

struct SinkNone {
  __device__ void store(uint32_t, int, const float *) const {}
};

struct SinkDense {   // columns 0..31 -> FP32 [rows x 32]
  float4 *dst;
  __device__ void store(uint32_t r, int c, const float *v) const
  {
    if (c >= 2) return;
#pragma unroll
    for (int k = 0; k < 4; k++)
      dst[8 * (size_t)r + 4 * c + k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
  }
};

struct SinkNode {   // columns 0..31 -> dh_prev = dX + dh_next; 32..63 -> dagg
  float4 *dh_prev;
  const float4 *dh_next;
  float4 *dagg;
  __device__ void store(uint32_t r, int c, const float *v) const
  {
    if (c >= 4) return;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float4 o = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
      if (c < 2) {
        const float4 a = dh_next[8 * (size_t)r + 4 * c + k];
        o.x += a.x; o.y += a.y; o.z += a.z; o.w += a.w;
        dh_prev[8 * (size_t)r + 4 * c + k] = o;
      } else {
        dagg[8 * (size_t)r + 4 * (c - 2) + k] = o;
      }
    }
  }
};

struct SinkEdge {   // columns 0..31 -> part_i[r], 32..63 -> part_j[r]
  float4 *pi, *pj;
  __device__ void store(uint32_t r, int c, const float *v) const
  {
    if (c >= 4) return;
    float4 *d = c < 2 ? pi + 8 * (size_t)r + 4 * c : pj + 8 * (size_t)r + 4 * (c - 2);
#pragma unroll
    for (int k = 0; k < 4; k++) d[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
  }
};

// ------------------------------------------------------------ backward kernel

// For Y = MLP(X) with the forward's saved hidden activations H (a1_save):
//   G1: dH  = dY W2~[:, :32]           (TMEM cols   0..31)
//       dP  = dH * (H > 0)
//   G2: dX  = dP W1~                   (TMEM cols  32..32+K1)
//   G3: dW2~^T += H~^T dY  (over rows) (TMEM cols 128..128+N2, lanes = features)
//   G4: dW1~^T += X~^T dP              (TMEM cols 160..191)
// W1t = W1~^T [K1 x 32], W2t = W2~^T [48 x N2] (rows 0..31 used by G1).  Each
// CTA writes its weight-gradient sums to part[blockIdx] ([K1 x 32] then [48 x N2]).
template <int K1, int N2>
constexpr size_t bwd_smem()
{
  return (size_t)128 * N2 * 2 * 2 + 128 * 32 * 2 * 2 + 128 * 128 * 2 * 2 + 32 * N2 * 2 + K1 * 32 * 2;
}

template <int K1, int N2, bool DX, class G, class DY, class S>
__global__ void __launch_bounds__(128) k_mlp_bwd(G gat, DY dyf, S sink, uint32_t rows, const uint4 *__restrict__ W1t,
                                                 const uint4 *__restrict__ W2t, const uint4 *__restrict__ a1_save,
                                                 float *__restrict__ part, int *__restrict__ err)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *dYs = smem;                     // A: 128 x N2
  unsigned char *dYt = dYs + 128 * N2 * 2;       // B: N2 x 128
  unsigned char *Ps = dYt + 128 * N2 * 2;        // A: 128 x 32
  unsigned char *Pt = Ps + 128 * 32 * 2;         // B: 32 x 128
  unsigned char *Ht = Pt + 128 * 32 * 2;         // A: 128 features x 128 rows
  unsigned char *Xt = Ht + 128 * 128 * 2;        // A: 128 features x 128 rows
  unsigned char *W2s = Xt + 128 * 128 * 2;       // B: 32 x N2
  unsigned char *W1s = W2s + 32 * N2 * 2;        // B: K1 x 32
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int s_abort;
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) tmem_alloc(&tslot, 256);
  if (t == 0) {
    mbar_init1(&mbar);
    s_abort = 0;
  }
  for (int idx = t; idx < 32 * N2 / 8; idx += 128)   // rows 0..31 of W2t
    st_chunk(W2s, idx / (N2 / 8), idx % (N2 / 8), N2, W2t[idx]);
  for (int idx = t; idx < K1 * 4; idx += 128) st_chunk(W1s, idx / 4, idx % 4, 32, W1t[idx]);
  {
    uint4 *z0 = reinterpret_cast<uint4 *>(Ht), *z1 = reinterpret_cast<uint4 *>(Xt);
    for (int idx = t; idx < 128 * 128 * 2 / 16; idx += 128) {
      z0[idx] = make_uint4(0, 0, 0, 0);
      z1[idx] = make_uint4(0, 0, 0, 0);
    }
  }
  fence_proxy_async();
  sync_tc();
  const uint32_t tm = tslot;
  const uint32_t lane = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  bool first = true;
  const uint32_t ntiles = (rows + 127) / 128;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t row = tile * 128 + t;
    const bool valid = row < rows;
    // dY (both layouts)
    {
      float d[32];
      if (valid) dyf.load(row, d);
      else {
#pragma unroll
        for (int k = 0; k < N2; k++) d[k] = 0.f;
      }
#pragma unroll
      for (int k = 0; k < N2 / 8; k++) {
        const uint4 p = pack8(d + 8 * k);
        st_chunk(dYs, t, k, N2, p);
        st_t_chunk(dYt, 8 * k, t, p);
      }
    }
    // H~^T from the saved activations (ones feature at 32 for valid rows)
    uint4 h[4];
#pragma unroll
    for (int k = 0; k < 4; k++) h[k] = valid ? a1_save[4 * (size_t)row + k] : make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int k = 0; k < 4; k++) st_t_chunk(Ht, 8 * k, t, h[k]);
    st_t(Ht, 32, t, valid ? (uint16_t)BF16_ONE : (uint16_t)0);
    // X~^T regathered
    {
      uint4 c[K1 / 8];
      if (valid) gat.load(row, c);
      else {
#pragma unroll
        for (int k = 0; k < K1 / 8; k++) c[k] = make_uint4(0, 0, 0, 0);
      }
#pragma unroll
      for (int k = 0; k < K1 / 8; k++) st_t_chunk(Xt, 8 * k, t, c[k]);
    }
    fence_proxy_async();
    sync_tc();
    if (t == 0) {
      gemm_issue_nc(tm, dYs, W2s, N2, 32, false);            // G1
      gemm_issue_nc(tm + 128, Ht, dYt, 128, N2, !first);     // G3
      mma_commit(&mbar);
    }
    if (!mbar_try(&mbar, phase)) { atomicExch(err, 1); s_abort = 1; }
    phase ^= 1;
    fence_after_sync();
    {
      float v[32], hf[32];
      tmem_ld32(tm + lane, v);
#pragma unroll
      for (int k = 0; k < 4; k++) unpack8(h[k], hf + 8 * k);
#pragma unroll
      for (int k = 0; k < 32; k++) v[k] = hf[k] > 0.f ? v[k] : 0.f;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint4 p = pack8(v + 8 * k);
        st_chunk(Ps, t, k, 32, p);
        st_t_chunk(Pt, 8 * k, t, p);
      }
    }
    fence_proxy_async();
    sync_tc();
    if (t == 0) {
      if (DX) gemm_issue_nc(tm + 32, Ps, W1s, 32, K1, false);   // G2
      gemm_issue_nc(tm + 160, Xt, Pt, 128, 32, !first);         // G4
      mma_commit(&mbar);
    }
    if (!mbar_try(&mbar, phase)) { atomicExch(err, 1); s_abort = 1; }
    phase ^= 1;
    fence_after_sync();
    if (DX) {
#pragma unroll
      for (int c = 0; c < K1 / 16; c++) {
        float v[16];
        tmem_ld16(tm + lane + 32 + 16 * c, v);
        if (valid) sink.store(row, c, v);
      }
    }
    first = false;
    sync_tc();
    if (s_abort) break;
  }
  // per-CTA weight-gradient sums; lanes are features
  float *p1 = part + (size_t)blockIdx.x * (K1 * 32 + 48 * N2);
  float *p2 = p1 + K1 * 32;
  {
    float v[32];
    tmem_ld32(tm + lane + 160, v);
    if (t < K1)
      for (int o = 0; o < 32; o++) p1[t * 32 + o] = first ? 0.f : v[o];
    if (N2 == 32) tmem_ld32(tm + lane + 128, v);
    else tmem_ld16(tm + lane + 128, v);
    if (t < 48)
      for (int o = 0; o < N2; o++) p2[t * N2 + o] = first ? 0.f : v[o];
  }
  sync_tc();
  if (warp == 0) tmem_dealloc(tm, 256);
}

// grad(W1~)[o][f] += sum_b part[b][f][o]; grad(W2~)[o][f] += sum_b part[b][K1*32 + f*N2 + o]
__global__ void k_wgrad_reduce(const float *__restrict__ part, int nblk, int K1, int N2, float *__restrict__ g1,
                               float *__restrict__ g2)
{
  const int n1 = 32 * K1, n2 = N2 * 48, stride = K1 * 32 + 48 * N2;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < n1) {
    const int o = idx / K1, f = idx % K1;
    float s = 0.f;
    for (int b = 0; b < nblk; b++) s += part[(size_t)b * stride + f * 32 + o];
    g1[idx] += s;
  } else if (idx < n1 + n2) {
    const int j = idx - n1, o = j / 48, f = j % 48;
    float s = 0.f;
    for (int b = 0; b < nblk; b++) s += part[(size_t)b * stride + K1 * 32 + f * N2 + o];
    g2[j] += s;
  }
}

// dh[i] += sum_{r at i} part_i[r] + part_j[rev[r]]; one warp per node, lane = feature
__global__ void k_edge_adjoint(uint32_t N, const uint32_t *__restrict__ seg, const uint32_t *__restrict__ rev,
                               const float *__restrict__ pi, const float *__restrict__ pj, float *__restrict__ dh)
{
  const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int f = threadIdx.x & 31;
  if (i >= N) return;
  float s = dh[32 * (size_t)i + f];
  for (uint32_t r = seg[i]; r < seg[i + 1]; r++) s += pi[32 * (size_t)r + f] + pj[32 * (size_t)rev[r] + f];
  dh[32 * (size_t)i + f] = s;
}

// block sums of (out - target)^2 in FP64
__global__ void k_loss_partial(uint32_t N, const float4 *__restrict__ out, const float4 *__restrict__ tgt,
                               double *__restrict__ part)
{
  __shared__ double sh[256];
  double s = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float4 o = out[i], g = tgt[i];
    const double a = (double)o.x - g.x, b = (double)o.y - g.y, c = (double)o.z - g.z, d = (double)o.w - g.w;
    s += a * a + b * b + c * c + d * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_loss_final(const double *__restrict__ part, int n, double w, double *__restrict__ loss)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < n; b++) s += part[b];
    loss[0] += w * s;
  }
}

// Adam on the FP32 master copy; refreshes the BF16 W~ and W~^T copies.
__global__ void k_adam(int n, float *__restrict__ theta, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, float lr, float b1, float b2, float eps, float c1, float c2,
                       bf16 *__restrict__ W, bf16 *__restrict__ Wt)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  // every operation rounded on its own (no contraction), in this order
  const float gi = g[idx];
  const float mi = __fadd_rn(__fmul_rn(b1, m[idx]), __fmul_rn(__fsub_rn(1.f, b1), gi));
  const float vi = __fadd_rn(__fmul_rn(b2, v[idx]), __fmul_rn(__fmul_rn(__fsub_rn(1.f, b2), gi), gi));
  m[idx] = mi;
  v[idx] = vi;
  const float mh = __fdiv_rn(mi, c1), vh = __fdiv_rn(vi, c2);
  const float th = __fsub_rn(theta[idx], __fdiv_rn(__fmul_rn(lr, mh), __fadd_rn(__fsqrt_rn(vh), eps)));
  theta[idx] = th;
  int L = 0;
  while (idx >= c_off[L + 1]) L++;
  const int j = idx - c_off[L], o = j / c_kin[L], f = j % c_kin[L];
  const bf16 b = __float2bfloat16_rn(th);
  W[idx] = b;
  Wt[c_off[L] + f * c_out[L] + o] = b;
}

// BF16 copies of the master weights
__global__ void k_refresh(int n, const float *__restrict__ theta, bf16 *__restrict__ W, bf16 *__restrict__ Wt)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int L = 0;
  while (idx >= c_off[L + 1]) L++;
  const int j = idx - c_off[L], o = j / c_kin[L], f = j % c_kin[L];
  const bf16 b = __float2bfloat16_rn(theta[idx]);
  W[idx] = b;
  Wt[c_off[L] + f * c_out[L] + o] = b;
}

// block sums of y^2
__global__ void k_sumsq(size_t n, const double *__restrict__ y, double *__restrict__ part)
{
  __shared__ double sh[256];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    s += y[i] * y[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// scal[0] = RMS = sqrt(sum of part / n), or 1 when that is zero
__global__ void k_rms(const double *__restrict__ part, int nb, double n, double *__restrict__ scal)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += part[b];
    const double r = sqrt(s / n);
    scal[0] = r > 0.0 ? r : 1.0;
  }
}

// x0[i] = BF16([y_i / s, q_i]) with s = scal[0]
__global__ void k_features(uint32_t N, const double *__restrict__ y, const double *__restrict__ q,
                           const double *__restrict__ scal, uint4 *__restrict__ x0)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float inv = (float)(1.0 / scal[0]);
  float f[8];
  for (int c = 0; c < 4; c++) f[c] = (float)y[4 * (size_t)i + c] * inv;
  for (int c = 0; c < 4; c++) f[4 + c] = (float)q[4 * (size_t)i + c];
  x0[i] = pack8(f);
}

// target[i] = (x_i - y_i) / s  (FP32)
__global__ void k_target(uint32_t N, const double *__restrict__ x, const double *__restrict__ y,
                         const double *__restrict__ scal, float4 *__restrict__ tgt)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double inv = 1.0 / scal[0];
  const double *a = x + 4 * (size_t)i, *b = y + 4 * (size_t)i;
  tgt[i] = make_float4((float)((a[0] - b[0]) * inv), (float)((a[1] - b[1]) * inv), (float)((a[2] - b[2]) * inv),
                       (float)((a[3] - b[3]) * inv));
}

// ------------------------------------------------------------ self-test kernel (one GEMM tile)

__global__ void __launch_bounds__(128) k_umma_selftest(const bf16 *__restrict__ X, const bf16 *__restrict__ Wt,
                                                       float *__restrict__ Y, int rows, int K, int N, int *err)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  unsigned char *As = smem;
  unsigned char *Bs = smem + 128 * K * 2;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int row0 = blockIdx.x * 128;
  if (warp == 0) tmem_alloc(&tslot, 128);
  for (int k = 0; k < K; k++) {
    const int r = row0 + t;
    const bf16 v = r < rows ? X[(size_t)r * K + k] : __float2bfloat16(0.f);
    *reinterpret_cast<bf16 *>(As + kmajor_offset(t, k, K)) = v;
  }
  for (int idx = t; idx < N * K; idx += 128) {
    const int n = idx / K, k = idx % K;
    *reinterpret_cast<bf16 *>(Bs + kmajor_offset(n, k, K)) = Wt[idx];
  }
  fence_proxy_async();
  sync_tc();
  const uint32_t taddr = tslot;
  if (t == 0) {
    mbar_init1(&mbar);
    gemm_issue(taddr, As, Bs, K, N, &mbar, false);
  }
  __syncthreads();
  const bool ok = mbar_try(&mbar, 0);
  if (!ok && lane == 0) atomicExch(err, 1);
  fence_after_sync();
  if (ok) {
    const int r = row0 + warp * 32 + lane;
    for (int c = 0; c < N; c += 16) {
      float v[16];
      tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      if (r < rows)
        for (int i = 0; i < 16; i++) Y[(size_t)r * N + c + i] = v[i];
    }
  }
  sync_tc();
  if (warp == 0) tmem_dealloc(taddr, 128);
}

}  // namespace

// ============================================================ host side

struct kfun3d_mpnn_graph {
  GraphDev d;
  int device = 0;
};

namespace {

#define MP_CK(call)                                                                         \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      std::string s_ = std::string("mpnn: ") + #call + ": " + cudaGetErrorString(e_);       \
      kf_set_error(KFUN3D_ERR_CUDA, s_.c_str());                                            \
      return KFUN3D_ERR_CUDA;                                                               \
    }                                                                                       \
  } while (0)

struct Buf {
  void *p = nullptr;
  size_t cap = 0;
  cudaError_t need(size_t bytes)
  {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace

struct kfun3d_mpnn {
  int device = 0;
  float *theta = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
  bf16 *W = nullptr, *Wt = nullptr;
  int *err = nullptr;
  double *dscal = nullptr;   // [0] scale, [2] loss
  double *red = nullptr;     // [256] partial sums
  long steps = 0;
  // workspace
  Buf h[4], agg[3], a1_enc, a1_dec, a1_node[3], a1_edge[3], msg, out, dh[2], dagg, pi, pj, wpart, x0;
  int nsm = 0;
};

namespace {

constexpr int NRED = 256;

int mp_error(int code, const char *msg)
{
  kf_set_error(code, msg);
  return code;
}

uint64_t splitmix(uint64_t &s)
{
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// He-uniform for layers followed by a ReLU, Glorot-uniform for the others;
// messages scaled by 1/4 (a node sums about 14 of them) and the output layer
// by 1/100 (the untrained network starts close to plain ILU(0)); biases and
// padding zero.
void init_params(std::vector<float> &th, unsigned long long seed)
{
  th.assign(NPARAM, 0.f);
  uint64_t s = seed;
  for (int L = 0; L < NLAYERS; L++) {
    const LayerShape sh = kShape[L];
    const bool relu_after = (L % 2) == 0;   // first layer of every MLP
    double bound = relu_after ? std::sqrt(6.0 / sh.nreal) : std::sqrt(6.0 / (sh.nreal + sh.out));
    if (L == L_DEC2) bound *= 0.01;
    if (L >= 2 && L < 14 && (L - 2) % 4 == 1) bound *= 0.25;   // edge2 of each layer
    const int nout = (L == L_DEC2) ? 4 : sh.out;
    for (int o = 0; o < nout; o++)
      for (int f = 0; f < sh.nreal; f++) {
        const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
        th[kOff.off[L] + o * sh.kin + f] = (float)((2.0 * u - 1.0) * bound);
      }
  }
}

int upload_tables(int device)
{
  static bool done[64] = {false};
  if (device >= 0 && device < 64 && done[device]) return KFUN3D_OK;
  int outs[NLAYERS], kins[NLAYERS];
  for (int L = 0; L < NLAYERS; L++) { outs[L] = kShape[L].out; kins[L] = kShape[L].kin; }
  MP_CK(cudaMemcpyToSymbol(c_off, kOff.off, sizeof(kOff.off)));
  MP_CK(cudaMemcpyToSymbol(c_out, outs, sizeof(outs)));
  MP_CK(cudaMemcpyToSymbol(c_kin, kins, sizeof(kins)));
  if (device >= 0 && device < 64) done[device] = true;
  return KFUN3D_OK;
}

template <class K>
unsigned persistent_grid(K kernel, size_t smem, int nsm, int cap)
{
  // CTAs of 128 threads an SM holds, from the kernel's registers (allocated
  // in units of 8 a thread) and shared memory (with the per-CTA reserve),
  // at most `cap` (the SM's 512 TMEM columns).  The occupancy query answers
  // one CTA an SM for these kernels, so the count is formed here; a grid
  // larger than what is resident would still be correct (every CTA loops
  // over its tiles on its own, and a TMEM allocation waits for a free one).
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncAttributes fa{};
  int dev = 0, regs_sm = 65536, smem_sm = 0, reserve = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&reserve, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  int per = 1;
  if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess && fa.numRegs > 0) {
    const int by_regs = regs_sm / (((fa.numRegs + 7) / 8) * 8 * 128);
    const int by_smem = smem_sm / (int)(smem + fa.sharedSizeBytes + (size_t)reserve);
    per = std::min(by_regs, by_smem);
  }
  cudaGetLastError();
  per = std::max(1, std::min(per, cap));
  return (unsigned)(nsm * per);
}

template <int K1, int N2, class G, class O>
int launch_fwd(kfun3d_mpnn *net, G g, O o, uint32_t rows, int layer, uint4 *a1_save, cudaStream_t st)
{
  if (rows == 0) return KFUN3D_OK;
  constexpr size_t smem = fwd_smem<K1, N2>();
  auto kern = k_mlp_fwd<K1, N2, G, O>;
  static unsigned grid_cache[64] = {0};
  unsigned &gc = grid_cache[net->device & 63];
  if (!gc) gc = persistent_grid(kern, smem, net->nsm, 8);   // 64 TMEM columns per CTA: 8 fill the SM's 512
  unsigned ntiles = (rows + 127) / 128;
  if constexpr (SegSum<O>::value) ntiles = o.ntiles;
  const unsigned grid = std::min(gc, ntiles);
  const uint4 *W1 = reinterpret_cast<const uint4 *>(net->W + kOff.off[layer]);
  const uint4 *W2 = reinterpret_cast<const uint4 *>(net->W + kOff.off[layer + 1]);
  kern<<<grid, 128, smem, st>>>(g, o, rows, W1, W2, a1_save, net->err);
  kf_count_launch();
  MP_CK(cudaGetLastError());
  return KFUN3D_OK;
}

template <int K1, int N2, bool DX, class G, class DY, class S>
int launch_bwd(kfun3d_mpnn *net, G g, DY dy, S sink, uint32_t rows, int layer, const uint4 *a1_save, cudaStream_t st)
{
  constexpr size_t smem = bwd_smem<K1, N2>();
  auto kern = k_mlp_bwd<K1, N2, DX, G, DY, S>;
  static unsigned grid_cache[64] = {0};
  unsigned &gc = grid_cache[net->device & 63];
  if (!gc) gc = persistent_grid(kern, smem, net->nsm, 2);   // 256 TMEM columns per CTA
  const unsigned ntiles = std::max(1u, (rows + 127) / 128);
  const unsigned grid = std::min(gc, ntiles);
  const size_t stride = K1 * 32 + 48 * N2;
  if (net->wpart.need((size_t)grid * stride * sizeof(float)) != cudaSuccess)
    return mp_error(KFUN3D_ERR_CUDA, "mpnn: out of device memory (weight-gradient partials)");
  const uint4 *W1t = reinterpret_cast<const uint4 *>(net->Wt + kOff.off[layer]);
  const uint4 *W2t = reinterpret_cast<const uint4 *>(net->Wt + kOff.off[layer + 1]);
  kern<<<grid, 128, smem, st>>>(g, dy, sink, rows, W1t, W2t, a1_save, net->wpart.as<float>(), net->err);
  const int n = 32 * K1 + N2 * 48;
  k_wgrad_reduce<<<(n + 255) / 256, 256, 0, st>>>(net->wpart.as<float>(), (int)grid, K1, N2,
                                                   net->grad + kOff.off[layer], net->grad + kOff.off[layer + 1]);
  kf_count_launch(2);
  MP_CK(cudaGetLastError());
  return KFUN3D_OK;
}

int check_err(kfun3d_mpnn *net, cudaStream_t st)
{
  int h = 0;
  MP_CK(cudaMemcpyAsync(&h, net->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MP_CK(cudaStreamSynchronize(st));
  if (h) {
    cudaMemsetAsync(net->err, 0, sizeof(int), st);
    return mp_error(KFUN3D_ERR_TIMEOUT, "mpnn: a tensor-core completion wait gave up");
  }
  return KFUN3D_OK;
}

// Workspace for a graph; `train` adds what the backward pass needs.
int ensure_workspace(kfun3d_mpnn *net, const GraphDev &g, bool train)
{
  const size_t N = g.N, R = g.R;
  bool ok = true;
  for (int k = 0; k < 4; k++) ok &= net->h[k].need(N * 64) == cudaSuccess;
  ok &= net->msg.need(R * 64) == cudaSuccess;
  ok &= net->agg[0].need(N * 64) == cudaSuccess;   // the fused edge MLP's sums
  ok &= net->x0.need(N * 16) == cudaSuccess;
  ok &= net->out.need(N * 16) == cudaSuccess;
  if (train) {
    for (int k = 0; k < 3; k++) {
      ok &= net->agg[k].need(N * 64) == cudaSuccess;
      ok &= net->a1_node[k].need(N * 64) == cudaSuccess;
      ok &= net->a1_edge[k].need(R * 64) == cudaSuccess;
    }
    ok &= net->a1_enc.need(N * 64) == cudaSuccess;
    ok &= net->a1_dec.need(N * 64) == cudaSuccess;
    for (int k = 0; k < 2; k++) ok &= net->dh[k].need(N * 128) == cudaSuccess;
    ok &= net->dagg.need(N * 128) == cudaSuccess;
    ok &= net->pi.need(R * 128) == cudaSuccess;
    ok &= net->pj.need(R * 128) == cudaSuccess;
  }
  if (!ok) return mp_error(KFUN3D_ERR_CUDA, "mpnn: out of device memory (workspace)");
  return KFUN3D_OK;
}

// Forward pass.  train: keep every activation the backward pass reads.
// With z the decoder writes z = y + s out instead of out.
int forward(kfun3d_mpnn *net, const GraphDev &g, const uint4 *x0, bool train, const double *y, double *z,
            const double *scal, cudaStream_t st)
{
  int rc = ensure_workspace(net, g, train);
  if (rc) return rc;
  uint4 *h[4];
  for (int k = 0; k < 4; k++) h[k] = net->h[k].as<uint4>();
  // inference ping-pongs between h[0] and h[1]
  auto H = [&](int l) { return train ? h[l] : h[l & 1]; };
  rc = launch_fwd<16, 32>(net, GatherEnc{x0}, OutBf16{H(0)}, g.N, L_ENC1, train ? net->a1_enc.as<uint4>() : nullptr,
                          st);
  // inference with a tile plan: the message sums formed in the edge MLP
  const bool fused = !train && g.plan && g.nplan;
  for (int l = 0; l < 3 && !rc; l++) {
    if (fused)
      rc = launch_fwd<80, 32>(net, GatherEdge{H(l), g.rnode, g.oth, g.efeat},
                              OutSegSum{g.plan, g.seg, net->agg[0].as<uint16_t>(), g.nplan}, g.R, L_EDGE1(l),
                              nullptr, st);
    else
      rc = launch_fwd<80, 32>(net, GatherEdge{H(l), g.rnode, g.oth, g.efeat}, OutBf16{net->msg.as<uint4>()}, g.R,
                              L_EDGE1(l), train ? net->a1_edge[l].as<uint4>() : nullptr, st);
    if (rc) break;
    GatherNode gn{H(l), g.seg, fused ? nullptr : net->msg.as<uint4>(), train ? net->agg[l].as<uint4>() : nullptr,
                  fused ? net->agg[0].as<uint4>() : nullptr};
    rc = launch_fwd<80, 32>(net, gn, OutResidual{H(l), H(l + 1)}, g.N, L_NODE1(l),
                            train ? net->a1_node[l].as<uint4>() : nullptr, st);
  }
  if (rc) return rc;
  if (z)
    rc = launch_fwd<48, 16>(net, GatherDec{H(3)}, OutDecApply{y, z, scal}, g.N, L_DEC1, nullptr, st);
  else
    rc = launch_fwd<48, 16>(net, GatherDec{H(3)}, OutDecTrain{net->out.as<float4>()}, g.N, L_DEC1,
                            train ? net->a1_dec.as<uint4>() : nullptr, st);
  return rc;
}

// Backward pass of w * sum (out - target)^2 after forward(train = true).
int backward(kfun3d_mpnn *net, const GraphDev &g, const uint4 *x0, const float4 *tgt, float w, cudaStream_t st)
{
  uint4 *h[4];
  for (int k = 0; k < 4; k++) h[k] = net->h[k].as<uint4>();
  float4 *dA = net->dh[0].as<float4>(), *dB = net->dh[1].as<float4>();
  float4 *dagg = net->dagg.as<float4>();
  float4 *pi = net->pi.as<float4>(), *pj = net->pj.as<float4>();
  // decoder: dh3 -> dA
  int rc = launch_bwd<48, 16, true>(net, GatherDec{h[3]}, DYLoss{net->out.as<float4>(), tgt, w}, SinkDense{dA}, g.N,
                                    L_DEC1, net->a1_dec.as<uint4>(), st);
  for (int l = 2; l >= 0 && !rc; l--) {
    // node layer: dY = dh_{l+1} (dA); dX -> dh_l (dB, with the residual path) and dagg
    GatherNode gn{h[l], g.seg, nullptr, nullptr, net->agg[l].as<uint4>()};
    rc = launch_bwd<80, 32, true>(net, gn, DYDense32{dA}, SinkNode{dB, dA, dagg}, g.N, L_NODE1(l),
                                  net->a1_node[l].as<uint4>(), st);
    if (rc) break;
    rc = launch_bwd<80, 32, true>(net, GatherEdge{h[l], g.rnode, g.oth, g.efeat}, DYEdge{dagg, g.rnode},
                                  SinkEdge{pi, pj}, g.R, L_EDGE1(l), net->a1_edge[l].as<uint4>(), st);
    if (rc) break;
    k_edge_adjoint<<<(unsigned)((g.N * 32ull + 255) / 256), 256, 0, st>>>(g.N, g.seg, g.rev, (const float *)pi,
                                                                          (const float *)pj, (float *)dB);
    kf_count_launch();
    std::swap(dA, dB);
  }
  if (rc) return rc;
  rc = launch_bwd<16, 32, false>(net, GatherEnc{x0}, DYDense32{dA}, SinkNone{}, g.N, L_ENC1,
                                 net->a1_enc.as<uint4>(), st);
  MP_CK(cudaGetLastError());
  return rc;
}

int set_device_of(kfun3d_mpnn *net)
{
  MP_CK(cudaSetDevice(net->device));
  return KFUN3D_OK;
}

// x0 (and target) of a pair on stream st; scr: >= NRED + 1 doubles
void pair_async(uint32_t N, const double *y, const double *q, const double *x, uint4 *x0, float4 *tgt, double *scr,
                cudaStream_t st)
{
  k_sumsq<<<NRED, 256, 0, st>>>(4 * (size_t)N, y, scr + 1);
  k_rms<<<1, 32, 0, st>>>(scr + 1, NRED, 4.0 * N, scr);
  k_features<<<(N + 255) / 256, 256, 0, st>>>(N, y, q, scr, x0);
  kf_count_launch(3);
  if (x && tgt) {
    k_target<<<(N + 255) / 256, 256, 0, st>>>(N, x, y, scr, tgt);
    kf_count_launch();
  }
}

}  // namespace

// ------------------------------------------------------------ solver-facing (internal)

int kf_mpnn_prepare(kfun3d_mpnn *net, kfun3d_mpnn_graph *G)
{
  if (!net || !G) return mp_error(KFUN3D_ERR_ARG, "mpnn: no network or graph");
  return ensure_workspace(net, G->d, false);
}

int kf_mpnn_apply_async(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const double *y, const double *q, double *z,
                        cudaStream_t st)
{
  const GraphDev &g = G->d;
  pair_async(g.N, y, q, nullptr, net->x0.as<uint4>(), nullptr, net->red, st);
  // scale lands in red[0]
  return forward(net, g, net->x0.as<uint4>(), false, y, z, net->red, st);
}

int kf_mpnn_status(kfun3d_mpnn *net, cudaStream_t st) { return check_err(net, st); }

int kf_mpnn_pair_async(size_t nnodes, const double *y, const double *q, const double *x, void *x0, float *tgt,
                       double *scr, cudaStream_t st)
{
  pair_async((uint32_t)nnodes, y, q, x, (uint4 *)x0, (float4 *)tgt, scr, st);
  MP_CK(cudaGetLastError());
  return KFUN3D_OK;
}

// ------------------------------------------------------------ C ABI

extern "C" size_t kfun3d_mpnn_param_count(void) { return (size_t)NPARAM; }

extern "C" int kfun3d_mpnn_layer_shape(int layer, int *out, int *kin, int *nreal, int *offset)
{
  if (layer < 0 || layer >= NLAYERS) return KFUN3D_ERR_ARG;
  if (out) *out = kShape[layer].out;
  if (kin) *kin = kShape[layer].kin;
  if (nreal) *nreal = kShape[layer].nreal;
  if (offset) *offset = kOff.off[layer];
  return KFUN3D_OK;
}

extern "C" kfun3d_mpnn *kfun3d_mpnn_create(unsigned long long seed)
{
  int dev = 0, count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    kf_set_error(KFUN3D_ERR_NO_DEVICE, "no CUDA device");
    return nullptr;
  }
  cudaGetDevice(&dev);
  if (upload_tables(dev)) return nullptr;
  kfun3d_mpnn *net = new kfun3d_mpnn();
  net->device = dev;
  cudaDeviceGetAttribute(&net->nsm, cudaDevAttrMultiProcessorCount, dev);
  bool ok = true;
  ok &= cudaMalloc(&net->theta, NPARAM * sizeof(float)) == cudaSuccess;
  ok &= cudaMalloc(&net->m, NPARAM * sizeof(float)) == cudaSuccess;
  ok &= cudaMalloc(&net->v, NPARAM * sizeof(float)) == cudaSuccess;
  ok &= cudaMalloc(&net->grad, NPARAM * sizeof(float)) == cudaSuccess;
  ok &= cudaMalloc(&net->W, NPARAM * sizeof(bf16)) == cudaSuccess;
  ok &= cudaMalloc(&net->Wt, NPARAM * sizeof(bf16)) == cudaSuccess;
  ok &= cudaMalloc(&net->err, sizeof(int)) == cudaSuccess;
  ok &= cudaMalloc(&net->dscal, 8 * sizeof(double)) == cudaSuccess;
  ok &= cudaMalloc(&net->red, (NRED + 8) * sizeof(double)) == cudaSuccess;
  if (!ok) {
    kf_set_error(KFUN3D_ERR_CUDA, "mpnn: out of device memory");
    kfun3d_mpnn_free(net);
    return nullptr;
  }
  cudaMemset(net->err, 0, sizeof(int));
  cudaMemset(net->dscal, 0, 8 * sizeof(double));
  std::vector<float> th;
  init_params(th, seed);
  if (kfun3d_mpnn_set_params(net, th.data(), th.size()) != KFUN3D_OK) {
    kfun3d_mpnn_free(net);
    return nullptr;
  }
  return net;
}

extern "C" void kfun3d_mpnn_free(kfun3d_mpnn *net)
{
  if (!net) return;
  cudaSetDevice(net->device);
  for (void *p : {(void *)net->theta, (void *)net->m, (void *)net->v, (void *)net->grad, (void *)net->W,
                  (void *)net->Wt, (void *)net->err, (void *)net->dscal, (void *)net->red})
    if (p) cudaFree(p);
  for (Buf *b : {&net->a1_enc, &net->a1_dec, &net->msg, &net->out, &net->dagg, &net->pi, &net->pj, &net->wpart,
                 &net->x0})
    b->release();
  for (int k = 0; k < 4; k++) net->h[k].release();
  for (int k = 0; k < 3; k++) {
    net->agg[k].release();
    net->a1_node[k].release();
    net->a1_edge[k].release();
  }
  for (int k = 0; k < 2; k++) net->dh[k].release();
  delete net;
}

extern "C" int kfun3d_mpnn_set_params(kfun3d_mpnn *net, const float *host, size_t n)
{
  if (!net || !host || n != (size_t)NPARAM) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_set_params: bad arguments");
  if (set_device_of(net)) return KFUN3D_ERR_CUDA;
  MP_CK(cudaMemcpy(net->theta, host, NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  MP_CK(cudaMemset(net->m, 0, NPARAM * sizeof(float)));
  MP_CK(cudaMemset(net->v, 0, NPARAM * sizeof(float)));
  MP_CK(cudaMemset(net->grad, 0, NPARAM * sizeof(float)));
  k_refresh<<<(NPARAM + 255) / 256, 256>>>(NPARAM, net->theta, net->W, net->Wt);
  kf_count_launch();
  MP_CK(cudaDeviceSynchronize());
  net->steps = 0;
  return KFUN3D_OK;
}

extern "C" int kfun3d_mpnn_get_params(const kfun3d_mpnn *net, float *host, size_t n)
{
  if (!net || !host || n != (size_t)NPARAM) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_get_params: bad arguments");
  MP_CK(cudaSetDevice(net->device));
  MP_CK(cudaMemcpy(host, net->theta, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  return KFUN3D_OK;
}

extern "C" int kfun3d_mpnn_get_grad(const kfun3d_mpnn *net, float *host, size_t n)
{
  if (!net || !host || n != (size_t)NPARAM) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_get_grad: bad arguments");
  MP_CK(cudaSetDevice(net->device));
  MP_CK(cudaMemcpy(host, net->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  return KFUN3D_OK;
}

extern "C" int kfun3d_mpnn_zero_grad(kfun3d_mpnn *net)
{
  if (!net) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_zero_grad: null network");
  MP_CK(cudaSetDevice(net->device));
  MP_CK(cudaMemset(net->grad, 0, NPARAM * sizeof(float)));
  return KFUN3D_OK;
}

extern "C" kfun3d_mpnn_graph *kfun3d_mpnn_graph_create(const GEOMETRY *g)
{
  if (!g || !g->e || !g->n || !g->e->eptr || !g->e->xyzn) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_graph_create: incomplete GEOMETRY");
    return nullptr;
  }
  const uint32_t N = (uint32_t)g->n->sz, E = (uint32_t)g->e->sz;
  const unsigned int *n0 = g->e->eptr->n0, *n1 = g->e->eptr->n1;
  for (uint32_t e = 0; e < E; e++)
    if (n0[e] >= N || n1[e] >= N) {
      kf_set_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_graph_create: edge end point out of range");
      return nullptr;
    }
  const size_t R = 2 * (size_t)E;
  std::vector<uint32_t> seg(N + 1, 0), rnode(R), oth(R), rev(R);
  std::vector<uint2> ef(R);
  for (uint32_t e = 0; e < E; e++) { seg[n0[e] + 1]++; seg[n1[e] + 1]++; }
  for (uint32_t i = 0; i < N; i++) seg[i + 1] += seg[i];
  std::vector<uint32_t> pos(seg.begin(), seg.end() - 1);
  double amean = 0.0;
  for (uint32_t e = 0; e < E; e++) amean += g->e->xyzn->x3[e];
  amean = E ? amean / E : 1.0;
  if (!(amean > 0.0)) amean = 1.0;
  auto bf = [](double x) -> uint32_t {
    const bf16 b = __float2bfloat16_rn((float)x);
    return (uint32_t)*reinterpret_cast<const uint16_t *>(&b);
  };
  for (uint32_t e = 0; e < E; e++) {
    const uint32_t a = n0[e], b = n1[e];
    const uint32_t ka = pos[a]++, kb = pos[b]++;
    const double nx = g->e->xyzn->x0[e], ny = g->e->xyzn->x1[e], nz = g->e->xyzn->x2[e];
    const double ar = g->e->xyzn->x3[e] / amean;
    rnode[ka] = a; oth[ka] = b; rev[ka] = kb;
    rnode[kb] = b; oth[kb] = a; rev[kb] = ka;
    ef[ka] = make_uint2(bf(nx) | (bf(ny) << 16), bf(nz) | (bf(ar) << 16));
    ef[kb] = make_uint2(bf(-nx) | (bf(-ny) << 16), bf(-nz) | (bf(ar) << 16));
  }
  kfun3d_mpnn_graph *G = new kfun3d_mpnn_graph();
  cudaGetDevice(&G->device);
  G->d.N = N;
  G->d.R = (uint32_t)R;
  bool ok = true;
  auto up = [&](auto *&dst, const auto &vec) {
    using T = typename std::decay<decltype(vec[0])>::type;
    if (cudaMalloc(&dst, std::max<size_t>(vec.size(), 1) * sizeof(T)) != cudaSuccess) { ok = false; return; }
    if (cudaMemcpy(dst, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
  };
  up(G->d.seg, seg);
  up(G->d.rnode, rnode);
  up(G->d.oth, oth);
  up(G->d.rev, rev);
  up(G->d.efeat, ef);
  // tiles of whole nodes, at most 128 rows each, in node order
  // (KFUN3D_MPNN_FUSED=0: none, the messages go through memory)
  const char *fenv = getenv("KFUN3D_MPNN_FUSED");
  if (!(fenv && strcmp(fenv, "0") == 0)) {
    std::vector<uint4> plan;
    bool fits = true;
    for (uint32_t i = 0; i < N && fits; ) {
      if (seg[i + 1] - seg[i] > 128u) fits = false;
      uint32_t j = i;
      while (j < N && seg[j + 1] - seg[i] <= 128u) j++;
      if (fits) plan.push_back(make_uint4(seg[i], seg[j] - seg[i], i, j - i));
      i = j;
    }
    if (fits && !plan.empty()) {
      up(G->d.plan, plan);
      G->d.nplan = (uint32_t)plan.size();
    }
  }
  if (!ok) {
    kf_set_error(KFUN3D_ERR_CUDA, "kfun3d_mpnn_graph_create: out of device memory");
    kfun3d_mpnn_graph_free(G);
    return nullptr;
  }
  return G;
}

extern "C" void kfun3d_mpnn_graph_free(kfun3d_mpnn_graph *G)
{
  if (!G) return;
  cudaSetDevice(G->device);
  for (void *p : {(void *)G->d.seg, (void *)G->d.rnode, (void *)G->d.oth, (void *)G->d.rev, (void *)G->d.efeat,
                  (void *)G->d.plan})
    if (p) cudaFree(p);
  delete G;
}

extern "C" int kfun3d_mpnn_forward(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const void *d_x0, float *d_out)
{
  if (!net || !G || !d_x0 || !d_out) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_forward: bad arguments");
  if (set_device_of(net)) return KFUN3D_ERR_CUDA;
  int rc = forward(net, G->d, (const uint4 *)d_x0, false, nullptr, nullptr, nullptr, 0);
  if (rc) return rc;
  MP_CK(cudaMemcpyAsync(d_out, net->out.p, (size_t)G->d.N * 16, cudaMemcpyDeviceToDevice, 0));
  return check_err(net, 0);
}

extern "C" int kfun3d_mpnn_accumulate(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const void *d_x0,
                                      const float *d_target, double weight, double *loss)
{
  if (!net || !G || !d_x0 || !d_target) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_accumulate: bad arguments");
  if (set_device_of(net)) return KFUN3D_ERR_CUDA;
  const GraphDev &g = G->d;
  int rc = forward(net, g, (const uint4 *)d_x0, true, nullptr, nullptr, nullptr, 0);
  if (rc) return rc;
  MP_CK(cudaMemsetAsync(net->dscal + 2, 0, sizeof(double), 0));
  k_loss_partial<<<NRED, 256>>>(g.N, net->out.as<float4>(), (const float4 *)d_target, net->red);
  k_loss_final<<<1, 32>>>(net->red, NRED, weight, net->dscal + 2);
  kf_count_launch(2);
  rc = backward(net, g, (const uint4 *)d_x0, (const float4 *)d_target, (float)weight, 0);
  if (rc) return rc;
  rc = check_err(net, 0);
  if (rc) return rc;
  if (loss) MP_CK(cudaMemcpy(loss, net->dscal + 2, sizeof(double), cudaMemcpyDeviceToHost));
  return KFUN3D_OK;
}

extern "C" int kfun3d_mpnn_adam_step(kfun3d_mpnn *net, double lr, double beta1, double beta2, double eps)
{
  if (!net) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_adam_step: null network");
  if (set_device_of(net)) return KFUN3D_ERR_CUDA;
  net->steps++;
  const double c1 = 1.0 - std::pow(beta1, (double)net->steps), c2 = 1.0 - std::pow(beta2, (double)net->steps);
  k_adam<<<(NPARAM + 255) / 256, 256>>>(NPARAM, net->theta, net->m, net->v, net->grad, (float)lr, (float)beta1,
                                        (float)beta2, (float)eps, (float)c1, (float)c2, net->W, net->Wt);
  kf_count_launch();
  MP_CK(cudaGetLastError());
  MP_CK(cudaMemsetAsync(net->grad, 0, NPARAM * sizeof(float), 0));
  MP_CK(cudaDeviceSynchronize());
  return KFUN3D_OK;
}

extern "C" int kfun3d_mpnn_make_pair(size_t nnodes, const double *d_y, const double *d_q, const double *d_x,
                                     void *d_x0, float *d_target)
{
  if (!d_y || !d_q || !d_x0) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_make_pair: bad arguments");
  double *scr = nullptr;
  MP_CK(cudaMalloc(&scr, (NRED + 8) * sizeof(double)));
  pair_async((uint32_t)nnodes, d_y, d_q, d_x, (uint4 *)d_x0, (float4 *)d_target, scr, 0);
  cudaError_t e = cudaDeviceSynchronize();
  cudaFree(scr);
  MP_CK(e);
  return KFUN3D_OK;
}

extern "C" int kfun3d_mpnn_apply(kfun3d_mpnn *net, kfun3d_mpnn_graph *G, const double *d_y, const double *d_q,
                                 double *d_z)
{
  if (!net || !G || !d_y || !d_q || !d_z) return mp_error(KFUN3D_ERR_ARG, "kfun3d_mpnn_apply: bad arguments");
  if (set_device_of(net)) return KFUN3D_ERR_CUDA;
  int rc = ensure_workspace(net, G->d, false);
  if (!rc) rc = kf_mpnn_apply_async(net, G, d_y, d_q, d_z, 0);
  if (rc) return rc;
  return check_err(net, 0);
}

extern "C" int kfun3d_umma_selftest(const void *X, const void *Wt, float *Y, int rows, int K, int N)
{
  if (rows <= 0 || K <= 0 || N <= 0 || K % 16 || N % 16 || K > 128 || N > 128) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_umma_selftest: K and N must be multiples of 16 up to 128");
    return KFUN3D_ERR_ARG;
  }
  int *err = nullptr;
  cudaError_t e = cudaMalloc(&err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(err, 0, sizeof(int));
  const size_t smem = (size_t)(128 + N) * K * 2;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    k_umma_selftest<<<(rows + 127) / 128, 128, smem>>>((const bf16 *)X, (const bf16 *)Wt, Y, rows, K, N, err);
    kf_count_launch();
    e = cudaDeviceSynchronize();
  }
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
  if (err) cudaFree(err);
  if (e != cudaSuccess) {
    std::string s = std::string("kfun3d_umma_selftest: ") + cudaGetErrorString(e);
    kf_set_error(KFUN3D_ERR_CUDA, s.c_str());
    return KFUN3D_ERR_CUDA;
  }
  if (h) {
    kf_set_error(KFUN3D_ERR_TIMEOUT, "kfun3d_umma_selftest: MMA completion wait gave up");
    return KFUN3D_ERR_TIMEOUT;
  }
  return KFUN3D_OK;
}
