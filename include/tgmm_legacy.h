/*
 * tgmm_legacy.h -- the reference's own C++ entry points for the supervoxel EM, with
 * identical (mangled) signatures, implemented over the C ABI of tgmm_gmem.h.  A
 * program written against UtilsCUDA/GMEMupdateCUDA.h and UtilsCUDA/knnCuda.h links
 * against libtgmm_gmem.so unchanged.  Error behaviour follows the reference: failures
 * print a message and exit (EXIT_FAILURE; exit(0) for the size guards, exit(3) when the
 * regularisation constants were never set).
 *
 *   GaussianMixtureModelCUDA                       <- UtilsCUDA/GMEMupdateCUDA.h:22-57
 *   GMEMinitializeMemoryWithSupervoxels            <- UtilsCUDA/GMEMupdateCUDA.h:132-137
 *   GMEMreleaseMemoryWithSupervoxels               <- UtilsCUDA/GMEMupdateCUDA.h:140-144
 *   GMEMvariationalInferenceCUDAWithSupervoxels    <- UtilsCUDA/GMEMupdateCUDA.h:92-98
 *   copyScaleToDvice                               <- UtilsCUDA/GMEMupdateCUDA.h:82
 *   calculateLocalLikelihood                       <- UtilsCUDA/GMEMupdateCUDA.h:120-127
 *   knnCUDAinPlace, setDeviceCUDA, uploadScaleCUDA, knnCUDA_ (temporalLogicalRules/knnCUDA),
 *   selectCUDAdeviceMaxMemory                      <- UtilsCUDA/knnCuda.h:225-231
 *   regularizePrecisionMatrixConstants             <- constants.h:19-45 (the library carries
 *       weak definitions of the three statics; a program's own definitions take precedence)
 */
#ifndef TGMM_LEGACY_H_
#define TGMM_LEGACY_H_

#ifdef __cplusplus
#include <ostream>
#include <string>
#include <vector>

#include "tgmm_gmem.h"

#ifndef CONSTANTS_H_
struct regularizePrecisionMatrixConstants {
  static double lambdaMin;
  static double lambdaMax;
  static double maxExcentricity;
  static void setConstants(double lambdaMin_, double lambdaMax_, double maxExcentricity_) {
    lambdaMin = lambdaMin_;
    lambdaMax = lambdaMax_;
    maxExcentricity = maxExcentricity_;
  }
};
#endif

struct GaussianMixtureModelCUDA {
  double beta_k, nu_k, alpha_k;
  double m_k[3];
  double W_k[6];
  double expectedLogDetCovarianceCUDA;
  double expectedLogResponsivityCUDA;
  double splitScore;
  double beta_o, nu_o, alpha_o;
  double m_o[3];
  double W_o[6];
  bool fixed;
  int supervoxelIdx[TGMM_MAX_SV_PER_GAUSSIAN];
  int supervoxelNum;

  std::ostream& writeXML(std::ostream& os, int id);
  static std::ostream& writeXMLheader(std::ostream& os) {
    os << "<?xml version=\"1.0\" encoding=\"utf-8\"?>" << std::endl << "<document>" << std::endl;
    return os;
  }
  static std::ostream& writeXMLfooter(std::ostream& os) {
    os << "</document>" << std::endl;
    return os;
  }
};
static_assert(sizeof(GaussianMixtureModelCUDA) == 288, "reference layout is 288 bytes");
static_assert(sizeof(TgmmGaussian) == 288, "C ABI record is 288 bytes");

void GMEMinitializeMemoryWithSupervoxels(float** queryCUDA, float* query, float** imgDataCUDA, float* imgData,
                                         float* scale, long long int query_nb, float** rnkCUDA, int** indCUDA,
                                         int** indCUDAtr, unsigned short int numLabels,
                                         float** centroidLabelPositionCUDA, float* centroidLabelPositionlong,
                                         long long int** labelListPtrCUDA, long long int* labelListPtrHOST);
void GMEMreleaseMemoryWithSupervoxels(float** queryCUDA, float** imgDataCUDA, float** rnkCUDA, int** indCUDA,
                                      int** indCUDAtr, float** centroidLabelPositionCUDA,
                                      long long int** labelListPtrCUDA);
void GMEMvariationalInferenceCUDAWithSupervoxels(float* queryCUDA, float* imgDataCUDA, float* rnkCUDA,
                                                 float* rnkCUDAtr, int* indCUDA, int* indCUDAtr,
                                                 float* centroidLabelPositionCUDA, long long int* labelListPtrCUDA,
                                                 GaussianMixtureModelCUDA* vecGMtemp, long long int query_nb,
                                                 int ref_nb, unsigned short int maxLabels, int maxIterEM,
                                                 double tolLikelihood, int devCUDA, int frame, bool W4DOF,
                                                 std::string debugPath = "");
void copyScaleToDvice(float* scale);
/* The local log-likelihood of supervoxel lists (UtilsCUDA/GMEMupdateCUDA.h:120-127): the
 * frame and the candidates (indCUDA) on the device, the Gaussians (vecGMtemp, ref_nb records)
 * on the host, one value per list into localLikelihood (resized to the list count; an empty
 * list leaves its entry as it was); rnkCUDA is not read.  Over tgmm_local_likelihood. */
void calculateLocalLikelihood(std::vector<double>& localLikelihood,
                              const std::vector<std::vector<int> >& listSupervoxels, float* queryCUDA,
                              float* imgDataCUDA, float* rnkCUDA, int* indCUDA, GaussianMixtureModelCUDA* vecGMtemp,
                              long long int* labelListPtrCUDA, long long int query_nb, int ref_nb, int numLabels);
void knnCUDAinPlace(int* indCUDA, float* queryCUDA, float* refTemp, long long int query_nb, int ref_nb);
/* The tracking graph's supervoxel kNN (temporalLogicalRules/knnCUDA/knnCuda.h:48-58): host
 * query (SoA) and ref (SoA) in, ind (and dist, if not NULL) out, KNN <= 11; over tgmm_knn_k. */
int knnCUDA_(int* ind, float* dist, float* query, float* ref, long long int query_nb, int ref_nb, int KNN,
             float* scale, int devCUDA);
void setDeviceCUDA(int devCUDA);
void uploadScaleCUDA(float* scale);
int selectCUDAdeviceMaxMemory();

#endif /* __cplusplus */
#endif /* TGMM_LEGACY_H_ */
