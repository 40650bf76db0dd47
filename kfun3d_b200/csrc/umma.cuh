// kfun3d_b200: fifth-generation tensor-core (tcgen05, sm_100a) building blocks
// for the learned preconditioner.
//
// One CTA of 128 threads computes D[128 x N] (+)= A[128 x K] . B[N x K]^T in
// BF16 with FP32 accumulators in tensor memory (TMEM):
//   * A and B are staged in shared memory in the canonical K-major layout
//     without swizzle: 8-row x 16-byte core matrices, core matrices of one
//     8-row group adjacent along K (leading byte offset 128 B), 8-row groups
//     K * 16 bytes apart (stride byte offset);
//   * one thread issues K/16 tcgen05.mma instructions and commits them to an
//     mbarrier; every thread waits on it (bounded);
//   * warp w reads TMEM lanes 32w..32w+31 (rows of D) with tcgen05.ld.
// Descriptor bit layouts follow the PTX ISA's tcgen05 shared-memory matrix
// descriptor and instruction descriptor (kind::f16).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace kf_umma {

// ---------------------------------------------------------------- descriptors

// Shared-memory matrix descriptor, SWIZZLE_NONE, K-major.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);                // start address, bits [0,14)
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;      // leading byte offset, bits [16,30)
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;      // stride byte offset, bits [32,46)
  d |= (uint64_t)1 << 46;                                 // descriptor version (sm100), bits [46,48)
  // base offset 0, lbo mode 0, layout type 0 (SWIZZLE_NONE)
  return d;
}

// Instruction descriptor: BF16 x BF16 -> F32, A and B K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
  return (1u << 4)                      // D format F32
         | (1u << 7)                    // A format BF16
         | (1u << 10)                   // B format BF16
         | ((uint32_t)(N >> 3) << 17)   // N >> 3
         | ((uint32_t)(M >> 4) << 24);  // M >> 4
}

// Byte offset of element (row, k) of a K-major operand in the canonical
// no-swizzle layout: 8-row groups of (K/8) core matrices of 8 x 8 BF16.
__host__ __device__ __forceinline__ uint32_t kmajor_offset(uint32_t row, uint32_t k, uint32_t K)
{
  return (row >> 3) * (K * 16u) + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// ---------------------------------------------------------------- TMEM

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(dst_smem);
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---------------------------------------------------------------- MMA

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
  const uint32_t z = 0;   // disable-output-lane mask: every lane written
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(a) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init1(uint64_t *mbar)
{
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait on an mbarrier phase; false if it gave up.
__device__ __forceinline__ bool mbar_try(uint64_t *mbar, uint32_t phase)
{
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
  for (uint32_t spins = 0; spins < (1u << 24); spins++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 lanes x 32 columns of FP32 from TMEM (this warp's lanes).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 16 columns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// D (TMEM, N columns) (+)= A (smem, 128 x K) . B (smem, N x K)^T, both K-major
// in the canonical layout; issued by one thread, no commit.
__device__ __forceinline__ void gemm_issue_nc(uint32_t d_tmem, const void *A_smem, const void *B_smem, int K, int N,
                                              bool accumulate)
{
  const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(A_smem);
  const uint32_t b0 = (uint32_t)__cvta_generic_to_shared(B_smem);
  const uint32_t idesc = idesc_bf16(128, N);
  for (int ks = 0; ks < K / 16; ks++) {
    // K step ks covers core-matrix columns 2ks, 2ks+1 (128 B apart)
    const uint64_t ad = smem_desc(a0 + ks * 256u, 128u, (uint32_t)K * 16u);
    const uint64_t bd = smem_desc(b0 + ks * 256u, 128u, (uint32_t)K * 16u);
    mma_bf16(d_tmem, ad, bd, idesc, (accumulate || ks > 0) ? 1u : 0u);
  }
}

// The same, followed by a commit of every MMA issued so far to mbar.
__device__ __forceinline__ void gemm_issue(uint32_t d_tmem, const void *A_smem, const void *B_smem, int K, int N,
                                           uint64_t *mbar, bool accumulate)
{
  gemm_issue_nc(d_tmem, A_smem, B_smem, K, N, accumulate);
  mma_commit(mbar);
}

}  // namespace kf_umma
