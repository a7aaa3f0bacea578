// legacy_api.cu -- the reference's C++ entry points (UtilsCUDA/GMEMupdateCUDA.h,
// UtilsCUDA/knnCuda.h) over the C ABI.  Keeps one cached plan per process, grown on
// demand, and the two scale settings of the reference (kNN scale and regularisation
// scale).  Failures print and exit like the reference's HANDLE_ERROR.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tgmm_legacy.h"

// Weak definitions: a program that defines these statics (constants.cpp) overrides them.
__attribute__((weak)) double regularizePrecisionMatrixConstants::lambdaMin = -1.0;
__attribute__((weak)) double regularizePrecisionMatrixConstants::lambdaMax = -1.0;
__attribute__((weak)) double regularizePrecisionMatrixConstants::maxExcentricity = -1.0;

namespace {

struct LegacyState {
  std::mutex mu;
  TgmmPlan* plan = nullptr;
  TgmmPlanDesc desc{};
  float knn_scale[3] = {1.0f, 1.0f, 1.0f};
  float reg_scale[3] = {1.0f, 1.0f, 1.0f};
};

LegacyState& state() {
  static LegacyState s;
  return s;
}

void die(const char* what, int code = EXIT_FAILURE) {
  printf("ERROR: %s: %s\n", what, tgmm_last_error());
  exit(code);
}

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    printf("%s in %s\n", cudaGetErrorString(e), what);
    exit(EXIT_FAILURE);
  }
}

TgmmPlan* plan_for(int64_t n_vox, int32_t n_sv, int32_t n_gauss, int device) {
  LegacyState& S = state();
  const TgmmPlanDesc& d = S.desc;
  if (S.plan && d.max_vox >= n_vox && d.max_sv >= n_sv && d.max_gauss >= n_gauss && d.device == device) return S.plan;
  if (S.plan) tgmm_plan_destroy(S.plan);
  S.plan = nullptr;
  TgmmPlanDesc nd{};
  nd.max_vox = std::max<int64_t>(n_vox, d.max_vox);
  nd.max_sv = std::max(n_sv, d.max_sv);
  nd.max_gauss = std::max(n_gauss, std::max(d.max_gauss, TGMM_J));
  nd.max_frames = 1;
  nd.device = device;
  if (tgmm_plan_create(&nd, &S.plan) != TGMM_OK) die("allocating the EM workspace");
  S.desc = nd;
  return S.plan;
}

}  // namespace

std::ostream& GaussianMixtureModelCUDA::writeXML(std::ostream& os, int id) {
  os << "<GaussianMixtureModel ";
  os << "id=\"" << id << "\" lineage=\"" << 0 << "\" parent=\"" << 0 << "\" dims=\"" << 3 << "\" splitScore=\""
     << splitScore << "\"";
  os << " scale=\"";
  for (int ii = 0; ii < 3; ii++) os << 1.0f << " ";
  os << "\"" << std::endl;
  os << "nu=\"" << nu_k << "\" beta=\"" << beta_k << "\" alpha=\"" << alpha_k << "\"";
  os << " m=\"";
  for (int ii = 0; ii < 3; ii++) os << m_k[ii] << " ";
  os << "\" W=\"" << W_k[0] << " " << W_k[1] << " " << W_k[2] << " " << W_k[1] << " " << W_k[3] << " " << W_k[4]
     << " " << W_k[2] << " " << W_k[4] << " " << W_k[5];
  os << "\"" << std::endl;
  os << "nuPrior=\"" << nu_o << "\" betaPrior=\"" << beta_o << "\" alphaPrior=\"" << alpha_o
     << "\" distMRFPrior=\"" << 0.0 << "\"";
  os << " mPrior=\"";
  for (int ii = 0; ii < 3; ii++) os << m_o[ii] << " ";
  os << "\" WPrior=\"" << W_o[0] << " " << W_o[1] << " " << W_o[2] << " " << W_o[1] << " " << W_o[3] << " "
     << W_o[4] << " " << W_o[2] << " " << W_o[4] << " " << W_o[5];
  os << "\">" << std::endl;
  os << "</GaussianMixtureModel>" << std::endl;
  return os;
}

void GMEMinitializeMemoryWithSupervoxels(float** queryCUDA, float* query, float** imgDataCUDA, float* imgData,
                                         float* scale, long long int query_nb, float** rnkCUDA, int** indCUDA,
                                         int** indCUDAtr, unsigned short int numLabels,
                                         float** centroidLabelPositionCUDA, float* centroidLabelPosition,
                                         long long int** labelListPtrCUDA, long long int* labelListPtrHOST) {
  TgmmFrame f;
  if (tgmm_frame_upload(query, imgData, centroidLabelPosition, (const int64_t*)labelListPtrHOST, query_nb,
                        (int32_t)numLabels, &f) != TGMM_OK)
    die("GMEMinitializeMemoryWithSupervoxels");
  *queryCUDA = (float*)f.query;
  *imgDataCUDA = (float*)f.img;
  *centroidLabelPositionCUDA = (float*)f.centroids;
  *labelListPtrCUDA = (long long int*)f.label_ptr;
  const size_t n = (size_t)numLabels * TGMM_J;
  check_cuda(cudaMalloc((void**)rnkCUDA, n * sizeof(float)), "cudaMalloc rnk");
  check_cuda(cudaMalloc((void**)indCUDA, n * sizeof(int)), "cudaMalloc ind");
  check_cuda(cudaMalloc((void**)indCUDAtr, n * sizeof(int)), "cudaMalloc indTr");
  uploadScaleCUDA(scale);
}

void GMEMreleaseMemoryWithSupervoxels(float** queryCUDA, float** imgDataCUDA, float** rnkCUDA, int** indCUDA,
                                      int** indCUDAtr, float** centroidLabelPositionCUDA,
                                      long long int** labelListPtrCUDA) {
  void** ptrs[] = {(void**)queryCUDA, (void**)imgDataCUDA, (void**)rnkCUDA, (void**)indCUDA,
                   (void**)indCUDAtr, (void**)centroidLabelPositionCUDA, (void**)labelListPtrCUDA};
  for (void** p : ptrs) {
    check_cuda(cudaFree(*p), "cudaFree");
    *p = nullptr;
  }
}

void GMEMvariationalInferenceCUDAWithSupervoxels(float* queryCUDA, float* imgDataCUDA, float* rnkCUDA,
                                                 float* /*rnkCUDAtr*/, int* indCUDA, int* indCUDAtr,
                                                 float* centroidLabelPositionCUDA, long long int* labelListPtrCUDA,
                                                 GaussianMixtureModelCUDA* vecGMtemp, long long int query_nb,
                                                 int ref_nb, unsigned short int numLabels, int maxIterEM,
                                                 double tolLikelihood, int devCUDA, int frame, bool W4DOF,
                                                 std::string debugPath) {
  // the reference's size guards (GMEMupdateCUDA.cu:3992-4007)
  if (query_nb > 1024LL * 65535LL) {
    printf("ERROR: Too many query points for the GPU resources\n");
    exit(0);
  }
  if (ref_nb > 65535) {
    printf("ERROR: Too many reference points for the GPU resources\n");
    exit(0);
  }
  if (regularizePrecisionMatrixConstants::lambdaMin < 0) {
    printf("ERROR: before GMEMregularizeWkKernel: regularizePrecisionMatrixConstants were not set\n");
    exit(3);
  }
  LegacyState& S = state();
  std::lock_guard<std::mutex> lock(S.mu);
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  (void)devCUDA;  // the reference only uses it for a memory printout
  cudaEvent_t t0, t1;
  check_cuda(cudaEventCreate(&t0), "cudaEventCreate");
  check_cuda(cudaEventCreate(&t1), "cudaEventCreate");
  check_cuda(cudaEventRecord(t0, 0), "cudaEventRecord");
  TgmmPlan* plan = plan_for(query_nb, numLabels, ref_nb, dev);
  TgmmEmParams p;
  tgmm_default_params(&p);
  p.max_iter_em = maxIterEM;
  p.tol_likelihood = tolLikelihood;
  p.w4dof = W4DOF ? 1 : 0;
  p.lambda_min = regularizePrecisionMatrixConstants::lambdaMin;
  p.lambda_max = regularizePrecisionMatrixConstants::lambdaMax;
  p.max_excentricity = regularizePrecisionMatrixConstants::maxExcentricity;
  for (int d = 0; d < 3; d++) {
    p.scale[d] = S.knn_scale[d];
    p.reg_scale[d] = S.reg_scale[d];
  }
  p.frame = frame;
  TgmmFrame f;
  f.query = queryCUDA;
  f.img = imgDataCUDA;
  f.centroids = centroidLabelPositionCUDA;
  f.label_ptr = (const int64_t*)labelListPtrCUDA;
  f.n_vox = query_nb;
  f.n_sv = numLabels;
  f.n_gauss = ref_nb;
  TgmmEmStats st;
  if (maxIterEM < 1) {
    // the reference runs no iteration and only re-derives the supervoxel lists from rnk
    for (int k = 0; k < ref_nb; k++) vecGMtemp[k].supervoxelNum = 0;
  } else {
    int rc = tgmm_em_run(plan, &f, (TgmmGaussian*)vecGMtemp, rnkCUDA, indCUDA, indCUDAtr, &p, &st, nullptr);
    if (rc != TGMM_OK) die("GMEMvariationalInferenceCUDAWithSupervoxels", rc == TGMM_ERR_BAD_CSR ? 3 : EXIT_FAILURE);
    printf("Frame=%d;iter=%d;Log-likelihood =%16.12f\n", frame, st.iterations + 1, st.ll);
  }
  if (!debugPath.empty()) {
    const size_t n = (size_t)numLabels * TGMM_J;
    std::vector<float> r(n);
    std::vector<int32_t> ind(n);
    check_cuda(cudaMemcpy(r.data(), rnkCUDA, n * 4, cudaMemcpyDeviceToHost), "read rnk");
    check_cuda(cudaMemcpy(ind.data(), indCUDA, n * 4, cudaMemcpyDeviceToHost), "read ind");
    if (tgmm_write_rnk_file(debugPath.c_str(), r.data(), ind.data(), numLabels) != TGMM_OK) {
      printf("ERROR: opening file %s to save rnk values from variational inference\n", debugPath.c_str());
      exit(2);
    }
  }
  check_cuda(cudaEventRecord(t1, 0), "cudaEventRecord");
  check_cuda(cudaEventSynchronize(t1), "cudaEventSynchronize");
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  const int iters = maxIterEM < 1 ? 0 : st.iterations;
  printf(" done in %f secs for %d EM iterations (%f secs per iteration)\n", ms / 1000, iters,
         iters > 0 ? ms / (iters * 1000.0) : 0.0);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
}

void calculateLocalLikelihood(std::vector<double>& localLikelihood, const std::vector<std::vector<int> >& lists,
                              float* queryCUDA, float* imgDataCUDA, float* rnkCUDA, int* indCUDA,
                              GaussianMixtureModelCUDA* vecGMtemp, long long int* labelListPtrCUDA,
                              long long int query_nb, int ref_nb, int numLabels) {
  (void)rnkCUDA;  // the reference's signature carries it; the local likelihood does not read it
  localLikelihood.resize(lists.size());
  std::vector<int32_t> ptr(lists.size() + 1, 0), idx, which;
  for (size_t i = 0; i < lists.size(); i++) {
    if (!lists[i].empty()) which.push_back((int32_t)i);  // the reference skips empty lists
  }
  if (which.empty()) return;
  ptr.assign(which.size() + 1, 0);
  for (size_t w = 0; w < which.size(); w++) {
    const std::vector<int>& l = lists[which[w]];
    idx.insert(idx.end(), l.begin(), l.end());
    ptr[w + 1] = (int32_t)idx.size();
  }
  TgmmGaussian* gd = nullptr;
  check_cuda(cudaMalloc((void**)&gd, sizeof(TgmmGaussian) * (size_t)ref_nb), "calculateLocalLikelihood: cudaMalloc");
  check_cuda(cudaMemcpy(gd, vecGMtemp, sizeof(TgmmGaussian) * (size_t)ref_nb, cudaMemcpyHostToDevice),
             "calculateLocalLikelihood: upload");
  TgmmFrame f{};
  f.query = queryCUDA;
  f.img = imgDataCUDA;
  f.label_ptr = reinterpret_cast<const int64_t*>(labelListPtrCUDA);
  f.centroids = nullptr;
  f.n_vox = query_nb;
  f.n_sv = numLabels;
  f.n_gauss = ref_nb;
  std::vector<double> out(which.size());
  const int rc = tgmm_local_likelihood(&f, indCUDA, gd, ref_nb, ptr.data(), idx.data(), (int32_t)which.size(),
                                       out.data(), nullptr);
  cudaFree(gd);
  if (rc != TGMM_OK) die("calculateLocalLikelihood");
  for (size_t w = 0; w < which.size(); w++) localLikelihood[which[w]] = out[w];
}

void copyScaleToDvice(float* scale) {
  LegacyState& S = state();
  for (int d = 0; d < 3; d++) S.reg_scale[d] = scale[d];
}

void uploadScaleCUDA(float* scale) {
  LegacyState& S = state();
  for (int d = 0; d < 3; d++) S.knn_scale[d] = scale[d];
}

void setDeviceCUDA(int devCUDA) { check_cuda(cudaSetDevice(devCUDA), "cudaSetDevice"); }

void knnCUDAinPlace(int* indCUDA, float* queryCUDA, float* refTemp, long long int query_nb, int ref_nb) {
  LegacyState& S = state();
  if (tgmm_knn(queryCUDA, query_nb, refTemp, ref_nb, S.knn_scale, indCUDA, nullptr) != TGMM_OK) die("knnCUDAinPlace");
}

// Host arrays in and out, like the reference's (which allocates and copies per call too);
// failures print and exit as the reference's HANDLE_ERROR does.
int knnCUDA_(int* ind, float* dist, float* query, float* ref, long long int query_nb, int ref_nb, int KNN,
             float* scale, int devCUDA) {
  if (KNN < 1 || KNN > 11) die("knnCUDA_: KNN must be 1..11");
  if (ref_nb <= 0) {  // nothing to assign (the reference's early return)
    if (dist)
      for (long long i = 0; i < query_nb * KNN; i++) dist[i] = 1e32f;
    return 0;
  }
  check_cuda(cudaSetDevice(devCUDA), "knnCUDA_: cudaSetDevice");
  float *qd = nullptr, *rd = nullptr, *dd = nullptr;
  int* id = nullptr;
  const size_t nq = (size_t)query_nb, nr = (size_t)ref_nb, no = nq * (size_t)KNN;
  check_cuda(cudaMalloc((void**)&qd, 3 * nq * sizeof(float)), "knnCUDA_: cudaMalloc");
  check_cuda(cudaMalloc((void**)&rd, 3 * nr * sizeof(float)), "knnCUDA_: cudaMalloc");
  check_cuda(cudaMalloc((void**)&id, no * sizeof(int)), "knnCUDA_: cudaMalloc");
  if (dist) check_cuda(cudaMalloc((void**)&dd, no * sizeof(float)), "knnCUDA_: cudaMalloc");
  check_cuda(cudaMemcpy(qd, query, 3 * nq * sizeof(float), cudaMemcpyHostToDevice), "knnCUDA_: copy");
  check_cuda(cudaMemcpy(rd, ref, 3 * nr * sizeof(float), cudaMemcpyHostToDevice), "knnCUDA_: copy");
  if (tgmm_knn_k(qd, query_nb, rd, ref_nb, KNN, scale, id, dd, nullptr) != TGMM_OK) die("knnCUDA_");
  check_cuda(cudaMemcpy(ind, id, no * sizeof(int), cudaMemcpyDeviceToHost), "knnCUDA_: copy");
  if (dist) check_cuda(cudaMemcpy(dist, dd, no * sizeof(float), cudaMemcpyDeviceToHost), "knnCUDA_: copy");
  cudaFree(qd);
  cudaFree(rd);
  cudaFree(id);
  if (dd) cudaFree(dd);
  return 0;
}

int selectCUDAdeviceMaxMemory() {
  int count = 0, device = -1;
  size_t best = 0;
  check_cuda(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
  for (int i = 0; i < count; i++) {
    cudaDeviceProp prop;
    check_cuda(cudaGetDeviceProperties(&prop, i), "cudaGetDeviceProperties");
    if (prop.totalGlobalMem > best) {
      best = prop.totalGlobalMem;
      device = i;
    }
  }
  return device;
}

extern "C" int tgmm_write_gmm_xml(const char* path, const TgmmGaussian* gm, int32_t n) {
  static_assert(sizeof(TgmmGaussian) == sizeof(GaussianMixtureModelCUDA), "one 288-byte record layout");
  if (!path || (!gm && n > 0) || n < 0) return TGMM_ERR_INVALID_ARG;
  std::ofstream os(path);
  if (!os) return TGMM_ERR_INVALID_ARG;
  GaussianMixtureModelCUDA::writeXMLheader(os);
  for (int32_t i = 0; i < n; i++) {
    GaussianMixtureModelCUDA g;
    memcpy((void*)&g, gm + i, sizeof(g));
    g.writeXML(os, i);
  }
  GaussianMixtureModelCUDA::writeXMLfooter(os);
  return os.good() ? TGMM_OK : TGMM_ERR_INVALID_ARG;
}
