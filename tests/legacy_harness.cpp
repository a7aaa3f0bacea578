// legacy_harness.cpp -- a minimal program written against the reference's C++ interface
// (the calls of mainTrackingGaussianMixtureModel.cpp:1065-1107), linked against
// libtgmm_gmem.so.  Usage: legacy_harness <dir> <maxIterEM> <tol>
// Reads <dir>/{query,img,cent,lptr,gauss}.bin, writes <dir>/{gauss_out,rnk,ind,local}.bin.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "tgmm_legacy.h"

static std::vector<char> slurp(const std::string& p) {
  FILE* f = fopen(p.c_str(), "rb");
  if (!f) {
    printf("cannot open %s\n", p.c_str());
    exit(2);
  }
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<char> b(n);
  if (fread(b.data(), 1, n, f) != (size_t)n) exit(2);
  fclose(f);
  return b;
}

static void spill(const std::string& p, const void* d, size_t n) {
  FILE* f = fopen(p.c_str(), "wb");
  if (!f || fwrite(d, 1, n, f) != n) exit(2);
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 4) return 1;
  const std::string dir = argv[1];
  const int max_iter = atoi(argv[2]);
  const double tol = atof(argv[3]);
  std::vector<char> q = slurp(dir + "/query.bin"), im = slurp(dir + "/img.bin"), ce = slurp(dir + "/cent.bin"),
                    lp = slurp(dir + "/lptr.bin"), gm = slurp(dir + "/gauss.bin");
  const long long N = (long long)(im.size() / 4);
  const int S = (int)(lp.size() / 8) - 1;
  const int K = (int)(gm.size() / sizeof(GaussianMixtureModelCUDA));
  float scale[3] = {1.0f, 1.0f, 2.0f};
  regularizePrecisionMatrixConstants::setConstants(0.02, 0.2222, 9.0);
  setDeviceCUDA(selectCUDAdeviceMaxMemory() >= 0 ? 0 : 0);
  float *queryCUDA, *imgCUDA, *rnkCUDA, *centCUDA;
  int *indCUDA, *indTrCUDA;
  long long* lptrCUDA;
  GMEMinitializeMemoryWithSupervoxels(&queryCUDA, (float*)q.data(), &imgCUDA, (float*)im.data(), scale, N, &rnkCUDA,
                                      &indCUDA, &indTrCUDA, (unsigned short)S, &centCUDA, (float*)ce.data(), &lptrCUDA,
                                      (long long*)lp.data());
  copyScaleToDvice(scale);
  GaussianMixtureModelCUDA* g = (GaussianMixtureModelCUDA*)gm.data();
  GMEMvariationalInferenceCUDAWithSupervoxels(queryCUDA, imgCUDA, rnkCUDA, NULL, indCUDA, indTrCUDA, centCUDA, lptrCUDA,
                                              g, N, K, (unsigned short)S, max_iter, tol, 0, 0, true, std::string(""));
  std::vector<float> rnk(5 * (size_t)S);
  std::vector<int> ind(5 * (size_t)S);
  cudaMemcpy(rnk.data(), rnkCUDA, rnk.size() * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(ind.data(), indCUDA, ind.size() * 4, cudaMemcpyDeviceToHost);
  // the split round's local likelihood around every Gaussian (main:1303-1331): its
  // supervoxels after the EM, under the EM's mixture and candidates
  std::vector<std::vector<int> > lists(K);
  for (int k = 0; k < K; k++) lists[k].assign(g[k].supervoxelIdx, g[k].supervoxelIdx + g[k].supervoxelNum);
  std::vector<double> local;
  calculateLocalLikelihood(local, lists, queryCUDA, imgCUDA, rnkCUDA, indCUDA, g, lptrCUDA, N, K, S);
  GMEMreleaseMemoryWithSupervoxels(&queryCUDA, &imgCUDA, &rnkCUDA, &indCUDA, &indTrCUDA, &centCUDA, &lptrCUDA);
  spill(dir + "/gauss_out.bin", gm.data(), gm.size());
  spill(dir + "/rnk.bin", rnk.data(), rnk.size() * 4);
  spill(dir + "/ind.bin", ind.data(), ind.size() * 4);
  spill(dir + "/local.bin", local.data(), local.size() * 8);
  return 0;
}
