// ref_harness.cu -- TEST INFRASTRUCTURE ONLY.  A C entry point over the reference's own
// GPU path (UtilsCUDA/GMEMupdateCUDA.cu + knnCuda.cu, compiled from the reference
// sources by oracle/build_ref.sh into oracle/_ref/libtgmm_ref.so), so that tests can run
// the unmodified reference on the same seeded inputs and pin the CPU oracle to it.
#include <cuda_runtime.h>
#include <stdio.h>

#include <fstream>
#include <string>
#include <vector>

#include "GMEMupdateCUDA.h"
#include "knnCuda.h"

extern "C" int ref_em_run(float* query, float* img, float* cent, long long* lptr, long long N, int S, void* gauss,
                          int K, int max_iter, double tol, int w4dof, double lmin, double lmax, double maxexc,
                          float* scale, float* rnk_out, int* ind_out) {
  if (S < 1 || S > 65535 || K < 5) return 1;
  regularizePrecisionMatrixConstants::setConstants(lmin, lmax, maxexc);
  float *qc = 0, *ic = 0, *rc = 0, *cc = 0;
  int *indc = 0, *indtr = 0;
  long long* lc = 0;
  GMEMinitializeMemoryWithSupervoxels(&qc, query, &ic, img, scale, N, &rc, &indc, &indtr, (unsigned short)S, &cc,
                                      cent, &lc, lptr);
  copyScaleToDvice(scale);
  GMEMvariationalInferenceCUDAWithSupervoxels(qc, ic, rc, NULL, indc, indtr, cc, lc, (GaussianMixtureModelCUDA*)gauss,
                                              N, K, (unsigned short)S, max_iter, tol, 0, 0, w4dof != 0,
                                              std::string(""));
  cudaError_t e = cudaMemcpy(rnk_out, rc, sizeof(float) * 5 * (size_t)S, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(ind_out, indc, sizeof(int) * 5 * (size_t)S, cudaMemcpyDeviceToHost);
  GMEMreleaseMemoryWithSupervoxels(&qc, &ic, &rc, &indc, &indtr, &cc, &lc);
  fflush(stdout);
  return e == cudaSuccess ? 0 : 2;
}

// kNN only: query SoA (host, nq points), refs AoS xyz (host).
extern "C" int ref_knn(float* query, long long nq, float* ref, int nref, float* scale, int* ind_out) {
  float *qd = 0, *rd = 0;
  int* id = 0;
  cudaMalloc(&qd, sizeof(float) * 3 * nq);
  cudaMalloc(&rd, sizeof(float) * 3 * nref);
  cudaMalloc(&id, sizeof(int) * 5 * nq);
  cudaMemcpy(qd, query, sizeof(float) * 3 * nq, cudaMemcpyHostToDevice);
  cudaMemcpy(rd, ref, sizeof(float) * 3 * nref, cudaMemcpyHostToDevice);
  uploadScaleCUDA(scale);
  knnCUDAinPlace(id, qd, rd, nq, nref);
  cudaError_t e = cudaMemcpy(ind_out, id, sizeof(int) * 5 * nq, cudaMemcpyDeviceToHost);
  cudaFree(qd);
  cudaFree(rd);
  cudaFree(id);
  return e == cudaSuccess ? 0 : 2;
}

// The reference's GMM XML document of n Gaussians (its writeXMLheader, writeXML(os, i) per
// record, writeXMLfooter), to compare the library's writer with byte for byte.
extern "C" int ref_write_gmm_xml(const char* path, void* gauss, int n) {
  std::ofstream os(path);
  if (!os) return 1;
  GaussianMixtureModelCUDA* g = (GaussianMixtureModelCUDA*)gauss;
  GaussianMixtureModelCUDA::writeXMLheader(os);
  for (int i = 0; i < n; i++) g[i].writeXML(os, i);
  GaussianMixtureModelCUDA::writeXMLfooter(os);
  return os.good() ? 0 : 2;
}

// The reference's calculateLocalLikelihood: frame arrays, candidates (ind, slot-major 5*S)
// and Gaussians on the host; the supervoxel lists as CSR (list_ptr[n+1], list_idx); one
// double per list out.
extern "C" int ref_local_likelihood(float* query, float* img, long long* lptr, long long N, int S, int* ind,
                                    void* gauss, int K, int* list_ptr, int* list_idx, int n_lists, double* out) {
  float *qd = 0, *id = 0;
  long long* ld = 0;
  int* indd = 0;
  cudaMalloc(&qd, sizeof(float) * 3 * N);
  cudaMalloc(&id, sizeof(float) * N);
  cudaMalloc(&ld, sizeof(long long) * (S + 1));
  cudaMalloc(&indd, sizeof(int) * 5 * (size_t)S);
  cudaMemcpy(qd, query, sizeof(float) * 3 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(id, img, sizeof(float) * N, cudaMemcpyHostToDevice);
  cudaMemcpy(ld, lptr, sizeof(long long) * (S + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(indd, ind, sizeof(int) * 5 * (size_t)S, cudaMemcpyHostToDevice);
  std::vector<std::vector<int> > lists(n_lists);
  for (int i = 0; i < n_lists; i++) lists[i].assign(list_idx + list_ptr[i], list_idx + list_ptr[i + 1]);
  std::vector<double> ll;
  calculateLocalLikelihood(ll, lists, qd, id, NULL, indd, (GaussianMixtureModelCUDA*)gauss, ld, N, K, S);
  for (int i = 0; i < n_lists; i++) out[i] = ll[i];
  cudaError_t e = cudaDeviceSynchronize();
  cudaFree(qd);
  cudaFree(id);
  cudaFree(ld);
  cudaFree(indd);
  return e == cudaSuccess ? 0 : 2;
}
