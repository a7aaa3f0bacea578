// knn_noalloc.cu -- the exact 5-NN search (the same grid search as tgmm_knn) for callers
// that must not allocate device memory.  Some callers cannot call cudaMalloc: code that
// runs while its process's device memory is owned by another allocator (a framework's
// caching pool, a fixed-size arena handed out by a host application), code on a real-time
// path where an allocation's latency or failure is unacceptable, and code inside a region
// where the driver is not to be asked for memory.  Their scratch here is one file-scope
// device array, created when the library is loaded on a device and kept until the process
// exits.  Its device address is looked up once per device and kept; cudaDeviceReset on a
// device ends the context that held the array, so a process that resets a device must not
// call this entry point on that device again.
#include <cuda_runtime.h>

#include <mutex>

#include "tgmm_internal.cuh"

namespace {

// Scratch for TGMM_KNN_NOALLOC_MAX_REF reference points (about 2.8 MB on each device that
// loads the library).
constexpr size_t kScratchBytes = (256 + 4 * (2 * (size_t)TGMM_KNN_NOALLOC_MAX_REF + 2) * 3 + 4 +
                                  4 * (size_t)TGMM_KNN_NOALLOC_MAX_REF + 255) / 256 * 256 +
                                 16 * (size_t)TGMM_KNN_NOALLOC_MAX_REF;

static __device__ __align__(256) unsigned char g_knn_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

extern "C" int tgmm_knn_noalloc(const float* query, int64_t nq, const float* ref, int32_t nref, const float scale[3],
                                int32_t* ind, void* stream) {
  if (!query || !ref || !scale || !ind || nq < 0 || nref < 0)
    return tgmm::report_error(TGMM_ERR_INVALID_ARG, "tgmm_knn_noalloc: null pointer or negative size", cudaSuccess);
  if (nref < TGMM_J)
    return tgmm::report_error(TGMM_ERR_BAD_SIZE, "tgmm_knn_noalloc needs at least 5 reference points", cudaSuccess);
  if (nref > TGMM_KNN_NOALLOC_MAX_REF)
    return tgmm::report_error(TGMM_ERR_BAD_SIZE,
                              "tgmm_knn_noalloc: more reference points than its fixed scratch holds "
                              "(TGMM_KNN_NOALLOC_MAX_REF = 65535); use tgmm_knn",
                              cudaSuccess);
  if (tgmm::knn_grid_scratch_bytes(nref) > kScratchBytes)
    return tgmm::report_error(TGMM_ERR_BAD_SIZE, "tgmm_knn_noalloc: scratch too small", cudaSuccess);
  if (nq == 0) return TGMM_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return tgmm::report_error(TGMM_ERR_CUDA, "tgmm_knn_noalloc: cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices)
    return tgmm::report_error(TGMM_ERR_INVALID_ARG, "tgmm_knn_noalloc: device ordinal out of range", cudaSuccess);
  void* scratch = nullptr;
  {
    // Host code sees g_knn_scratch only as a host-side stand-in: the array's device address
    // is looked up once per device, with that device current, on the first call there.
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_knn_scratch);
      if (e != cudaSuccess) return tgmm::report_error(TGMM_ERR_CUDA, "tgmm_knn_noalloc: cudaGetSymbolAddress", e);
      g_scratch_ptr[dev] = p;
    }
    scratch = g_scratch_ptr[dev];
  }
  e = tgmm::knn_grid_in_scratch(query, nq, ref, nref, scale, ind, (cudaStream_t)stream, scratch);
  if (e != cudaSuccess) return tgmm::report_error(TGMM_ERR_CUDA, "tgmm_knn_noalloc", e);
  return TGMM_OK;
}
