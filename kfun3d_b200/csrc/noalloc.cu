// kfun3d_b200: an allocation-free triangular solve for callers that cannot
// allocate device memory.
//
// Who needs it: a host framework that owns every device allocation (a
// solver framework with its own pooled allocator, or an application that
// sizes all device memory at start-up and forbids libraries from calling
// cudaMalloc afterwards).  ComputeSparseTriangularSolve takes host arrays and
// stages them through buffers of the GEOMETRY's device mirror;
// kfun3d_sptrsv_device_noalloc instead takes the caller's device arrays and
// keeps its only working memory -- the per-row completion flags of the
// sync-free sweep -- in a fixed, file-scope device array, so the call itself
// allocates nothing.
//
// Ordering: the call first waits for all work already queued on the device
// (so the caller's writes of b, on any stream, are complete), runs the sweep
// on the library's stream and waits for it before returning (so x is final
// when the call returns).
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.h"

namespace {

// Per-row completion flags of the sync-free sweep: one word per matrix row.
// Every GPU that loads the library holds this array until the process exits.
constexpr uint32_t KF_NOALLOC_MAX_ROWS = 1u << 21;   // 2,097,152 rows (8 MiB)
static __device__ __align__(256) uint32_t kf_noalloc_flags[KF_NOALLOC_MAX_ROWS];

// Device address of the array, looked up once per device with that device
// current.  In host code kf_noalloc_flags names a host-side stand-in, not the
// device array, so it is never passed to a kernel directly.  The cache is
// guarded, so first calls from several host threads are safe.
constexpr int KF_MAX_DEVICES = 64;
uint32_t *g_flags_addr[KF_MAX_DEVICES] = {};
std::mutex g_flags_mutex;

uint32_t *flags_address(int dev)
{
  if (dev < 0 || dev >= KF_MAX_DEVICES) return nullptr;
  std::lock_guard<std::mutex> lock(g_flags_mutex);
  if (!g_flags_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, kf_noalloc_flags);
    if (e != cudaSuccess) {
      std::string s = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      kf_set_error(KFUN3D_ERR_CUDA, s.c_str());
      return nullptr;
    }
    g_flags_addr[dev] = (uint32_t *)p;
  }
  return g_flags_addr[dev];
}

}  // namespace

extern "C" int kfun3d_sptrsv_device_noalloc(const GEOMETRY *g, const double *d_b, double *d_x)
{
  MatrixHandle *h = kf_handle(g);
  if (h && h->pat.n > KF_NOALLOC_MAX_ROWS) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: more than 2,097,152 rows; "
                                 "use ComputeSparseTriangularSolve");
    return KFUN3D_ERR_ARG;
  }
  if (!h || !h->dev) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: no device factor for this GEOMETRY; "
                                 "call ComputeA and ComputeNumericalILU first");
    return KFUN3D_ERR_ARG;
  }
  DevMesh &m = *h->dev;
  if (m.N > KF_NOALLOC_MAX_ROWS) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: more than 2,097,152 rows; "
                                 "use ComputeSparseTriangularSolve");
    return KFUN3D_ERR_ARG;
  }
  if (m.ilu_active) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: the factor is in the spatial ILU order; "
                                 "use ComputeSparseTriangularSolve or the mesh order");
    return KFUN3D_ERR_ARG;
  }
  if (!m.factored) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: the matrix has not been factored "
                                 "(call ComputeNumericalILU)");
    return KFUN3D_ERR_ARG;
  }
  if (m.factor_precision != kf_precision()) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: the factor was computed in another "
                                 "precision than the one now set (kfun3d_set_precision); refactor first");
    return KFUN3D_ERR_ARG;
  }
  if (!d_b || !d_x || ((uintptr_t)d_b & 15) || ((uintptr_t)d_x & 15) || d_b == d_x) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: b and x must be distinct, 16-byte aligned "
                                 "device arrays of 4*nnodes doubles");
    return KFUN3D_ERR_ARG;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != m.device) {
    kf_set_error(KFUN3D_ERR_ARG, "kfun3d_sptrsv_device_noalloc: the current device is not the one "
                                 "holding this GEOMETRY's factor");
    return KFUN3D_ERR_ARG;
  }
  uint32_t *flags = flags_address(dev);
  if (!flags) return KFUN3D_ERR_CUDA;
  // the caller's pending work (b written on any stream, an earlier read of x)
  // completes first; an error it left is reported here, not blamed on the sweep
  cudaError_t e0 = cudaDeviceSynchronize();
  if (e0 == cudaSuccess) e0 = cudaGetLastError();
  if (e0 != cudaSuccess) {
    std::string s = std::string("kfun3d_sptrsv_device_noalloc: earlier device work failed: ") +
                    cudaGetErrorString(e0);
    kf_set_error(KFUN3D_ERR_CUDA, s.c_str());
    return KFUN3D_ERR_CUDA;
  }
  if (kf_mode() == KFUN3D_MODE_FAST) kf_fast::sptrsv_flags(m, d_b, d_x, kf_precision(), flags);
  else kf_exact::sptrsv_flags(m, d_b, d_x, kf_precision(), flags);
  cudaError_t e = cudaStreamSynchronize(m.stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::string s = std::string("kfun3d_sptrsv_device_noalloc: ") + cudaGetErrorString(e);
    kf_set_error(KFUN3D_ERR_CUDA, s.c_str());
    return KFUN3D_ERR_CUDA;
  }
  int st[2] = {0, 0};
  e = cudaMemcpy(st, m.status, sizeof(st), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && st[1]) {
    cudaMemset(m.status + 1, 0, sizeof(int));
    kf_set_error(KFUN3D_ERR_TIMEOUT, "kfun3d_sptrsv_device_noalloc: a triangular-solve wait exceeded its bound");
    return KFUN3D_ERR_TIMEOUT;
  }
  return KFUN3D_OK;
}
