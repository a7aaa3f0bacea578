// local_ll.cu -- the local log-likelihood of supervoxel lists: the likelihood the split
// round compares before and after a proposed cell division (calculateLocalLikelihood,
// UtilsCUDA/GMEMupdateCUDA.h:120, body GMEMupdateCUDA.cu:2952-3055, over
// addLocalLikelihoodWithSupervoxels :2876-2949 and the kernel
// GMEMcomputeLocalLikelihoodKernelWithSupervoxels :1989-2103).
//
// For each list and each supervoxel s in it (a supervoxel listed twice counts twice), with
// s's five candidates ind[j*n_sv+s] and the given Gaussians, each voxel's density is
//   sum_j sqrt(det W_j nu_j^3)/(2 pi)^{3/2} exp(-nu_j d'W_j d/2) alpha_j/A,  d = x - m_j,
// A the sum of alpha over every Gaussian, all in FP64 as the reference evaluates it.  The
// supervoxel's value keeps the reference's per-thread overwrite: of the voxels v = t + 1024 i
// (t < 1024, relative to s's first voxel) only the last one with a positive density adds
// I_v ln(density_v).  The reference then sums in float (a block tree per supervoxel, a
// power-of-two pass over the list, a double sum of the blocks on the host); here every sum
// is FP64 in a fixed order: a warp's lanes, then the supervoxels in list order.
//
// Launches: k_local_alpha (one block: A), k_local_items (a warp per listed supervoxel),
// k_local_lists (a thread per list).
#include <cuda_runtime.h>

#include <vector>

#include "tgmm_internal.cuh"

namespace tgmm {
namespace {

constexpr double kTwoPi15 = 15.749609945722419;  // (2 pi)^(3/2)
constexpr int kLocalWarps = 8;                   // warps per block of k_local_items

__device__ __forceinline__ double det_sym3(const double* w) {
  return w[0] * (w[3] * w[5] - w[4] * w[4]) - w[1] * (w[1] * w[5] - w[2] * w[4]) +
         w[2] * (w[1] * w[4] - w[2] * w[3]);
}

// A = sum of alpha_k in FP64: thread-strided partials in index order, then a fixed tree.
__global__ void __launch_bounds__(1024) k_local_alpha(const TgmmGaussian* gm, int n, double* out) {
  __shared__ double sh[1024];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += 1024) s += gm[k].alpha_k;
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int h = 512; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

struct LocalCand {
  double m[3];
  double W[6];
  double nu, c;  // c = sqrt(det W nu^3)/(2 pi)^{3/2} * alpha/A
};

__device__ __forceinline__ double local_density(const LocalCand* C, float x0, float x1, float x2) {
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < kJ; j++) {
    const double* W = C[j].W;
    const double d0 = (double)x0 - C[j].m[0], d1 = (double)x1 - C[j].m[1], d2 = (double)x2 - C[j].m[2];
    const double maha = C[j].nu * (W[0] * d0 * d0 + W[3] * d1 * d1 + W[5] * d2 * d2 + 2.0 * W[1] * d0 * d1 +
                                   2.0 * W[2] * d0 * d2 + 2.0 * W[4] * d1 * d2);
    acc += C[j].c * exp(-0.5 * maha);
  }
  return acc;
}

// Warp per listed supervoxel (item p of the flattened lists): its local log-likelihood into
// item_ll[p].  Lane t handles the reference's threads t, t + 32, ... < min(n, 1024): the last
// voxel of each thread's stride, walking back a stride at a time past zero densities.
__global__ void __launch_bounds__(kLocalWarps * 32) k_local_items(const float* query, const float* img,
                                                                   const int64_t* lptr, int64_t n_vox, int n_sv,
                                                                   const int32_t* ind, const TgmmGaussian* gm,
                                                                   int n_gauss, const int32_t* list_idx, int n_items,
                                                                   const double* alpha_total, double* item_ll,
                                                                   int* bad) {
  __shared__ LocalCand cand[kLocalWarps][kJ];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * kLocalWarps + warp;
  if (p >= n_items) return;  // whole warps leave; no block-wide barrier follows
  const int s = list_idx[p];
  LocalCand* C = cand[warp];
  int ok = 1;
  if (lane < kJ) {
    const int k = ind[(int64_t)lane * n_sv + s];
    if (k < 0 || k >= n_gauss) {
      ok = 0;
      for (int d = 0; d < 3; d++) C[lane].m[d] = 0.0;
      for (int e = 0; e < 6; e++) C[lane].W[e] = 0.0;
      C[lane].nu = 0.0;
      C[lane].c = 0.0;
    } else {
      const TgmmGaussian& g = gm[k];
      for (int d = 0; d < 3; d++) C[lane].m[d] = g.m_k[d];
      for (int e = 0; e < 6; e++) C[lane].W[e] = g.W_k[e];
      C[lane].nu = g.nu_k;
      double c = sqrt(det_sym3(g.W_k) * pow(g.nu_k, 3.0)) / kTwoPi15;
      C[lane].c = c * (g.alpha_k / *alpha_total);
    }
  }
  if (!__all_sync(0xffffffffu, ok)) {
    if (lane == 0) {
      atomicOr(bad, 1);
      item_ll[p] = 0.0;
    }
    return;
  }
  __syncwarp();
  const int64_t a = lptr[s], b = lptr[s + 1];
  const int64_t n = b - a;
  double acc = 0.0;
  for (int64_t t = lane; t < (n < 1024 ? n : 1024); t += 32) {
    for (int64_t v = a + t + ((n - 1 - t) / 1024) * 1024; v >= a; v -= 1024) {
      const double dens = local_density(C, query[v], query[n_vox + v], query[2 * n_vox + v]);
      if (dens > 0.0) {
        acc += (double)img[v] * log(dens);
        break;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) item_ll[p] = acc;
}

__global__ void k_local_lists(const int32_t* list_ptr, int n_lists, const double* item_ll, double* ll) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_lists) return;
  double s = 0.0;
  for (int p = list_ptr[i]; p < list_ptr[i + 1]; p++) s += item_ll[p];
  ll[i] = s;
}

}  // namespace
}  // namespace tgmm

extern "C" int tgmm_local_likelihood(const TgmmFrame* frame, const int32_t* ind_dev, const TgmmGaussian* gm_dev,
                                     int32_t n_gauss, const int32_t* list_ptr, const int32_t* list_idx,
                                     int32_t n_lists, double* ll_out, void* stream) {
  using namespace tgmm;
  if (!frame || !ind_dev || !gm_dev || !list_ptr || !ll_out || n_lists < 0 || n_gauss < TGMM_J)
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_local_likelihood: null argument or fewer than 5 Gaussians",
                        cudaSuccess);
  if (!frame->query || !frame->img || !frame->label_ptr || frame->n_sv < 1 || frame->n_vox < 0)
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_local_likelihood: bad frame", cudaSuccess);
  if (n_lists == 0) return TGMM_OK;
  if (list_ptr[0] != 0) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_local_likelihood: list_ptr[0] != 0", cudaSuccess);
  for (int32_t i = 0; i < n_lists; i++)
    if (list_ptr[i + 1] < list_ptr[i])
      return report_error(TGMM_ERR_INVALID_ARG, "tgmm_local_likelihood: list_ptr not monotone", cudaSuccess);
  const int32_t n_items = list_ptr[n_lists];
  if (n_items > 0 && !list_idx) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_local_likelihood: null list_idx", cudaSuccess);
  for (int32_t p = 0; p < n_items; p++)
    if (list_idx[p] < 0 || list_idx[p] >= frame->n_sv)
      return report_error(TGMM_ERR_INVALID_ARG, "tgmm_local_likelihood: supervoxel index out of range", cudaSuccess);
  cudaStream_t st = (cudaStream_t)stream;
  // one stream-ordered scratch: lists (ptr, idx), per-item values, per-list values, A, a flag
  const size_t o_ptr = 0, o_idx = o_ptr + 4 * ((size_t)n_lists + 1);
  const size_t o_item = (o_idx + 4 * (size_t)(n_items > 0 ? n_items : 1) + 7) / 8 * 8;
  const size_t o_ll = o_item + 8 * (size_t)(n_items > 0 ? n_items : 1);
  const size_t o_a = o_ll + 8 * (size_t)n_lists, o_bad = o_a + 8, total = o_bad + 8;
  char* buf = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&buf, total, st);
  if (e != cudaSuccess) return report_error(TGMM_ERR_OOM, "tgmm_local_likelihood: scratch", e);
  int32_t* d_ptr = (int32_t*)(buf + o_ptr);
  int32_t* d_idx = (int32_t*)(buf + o_idx);
  double* d_item = (double*)(buf + o_item);
  double* d_ll = (double*)(buf + o_ll);
  double* d_a = (double*)(buf + o_a);
  int* d_bad = (int*)(buf + o_bad);
  std::vector<double> host_ll(n_lists);
  int bad = 0;
  e = cudaMemcpyAsync(d_ptr, list_ptr, 4 * ((size_t)n_lists + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && n_items > 0) e = cudaMemcpyAsync(d_idx, list_idx, 4 * (size_t)n_items, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, 4, st);
  if (e == cudaSuccess) {
    k_local_alpha<<<1, 1024, 0, st>>>(gm_dev, n_gauss, d_a);
    if (n_items > 0)
      k_local_items<<<(n_items + kLocalWarps - 1) / kLocalWarps, kLocalWarps * 32, 0, st>>>(
          frame->query, frame->img, frame->label_ptr, frame->n_vox, frame->n_sv, ind_dev, gm_dev, n_gauss, d_idx,
          n_items, d_a, d_item, d_bad);
    k_local_lists<<<(n_lists + 255) / 256, 256, 0, st>>>(d_ptr, n_lists, d_item, d_ll);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(host_ll.data(), d_ll, 8 * (size_t)n_lists, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, st);
  cudaError_t ef = cudaFreeAsync(buf, st);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return report_error(TGMM_ERR_CUDA, "tgmm_local_likelihood", e);
  if (bad) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_local_likelihood: a candidate index is out of range", cudaSuccess);
  for (int32_t i = 0; i < n_lists; i++) ll_out[i] = host_ll[i];
  return TGMM_OK;
}
