// TEST INFRASTRUCTURE ONLY.  Runs the reference's own supervoxel trimming and weighted
// statistics (temporalLogicalRules/supervoxel.cpp) and its erase of small supervoxels
// (nucleiChSvWshedPBC/hierarchicalSegmentation.cpp), compiled from their sources by
// oracle/build_ref.sh, for the frame preparation of mainTrackingGaussianMixtureModel.cpp:
// 557-634: per supervoxel (given as an ascending voxel list) the threshold
// trimSupervoxel<uint16>() returns, the voxels it keeps, the centroid and intensity
// weightedGaussianStatistics<uint16>(true) computes from the raw image; and the order
// eraseSupervoxelFromCurrentSegmentation leaves the survivors in.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "constants.h"
#include "hierarchicalSegmentation.h"
#include "supervoxel.h"

// supervoxel.cpp references the tracking graph's kNN; trimming and statistics never call it
int knnCUDA_(int*, float*, float*, float*, long long, int, int, float*, int) { abort(); }

extern "C" int ref_trim_stats(const uint16_t* raw, const int32_t* dims, const int64_t* lptr, const uint64_t* lin,
                              int32_t n_sv, int32_t max_size, float max_pct, int32_t conn, uint16_t* thr_out,
                              int64_t* cnt_out, uint64_t* lin_out, float* cent_out, float* intensity_out) {
  uint64 dd[3] = {(uint64)dims[0], (uint64)dims[1], (uint64)dims[2]};
  supervoxel::setDataDims(dd);
  supervoxel::dataSizeInBytes = sizeof(uint16_t) * dd[0] * dd[1] * dd[2];
  float scale[3] = {1.f, 1.f, 2.f};
  supervoxel::setScale(scale);
  regularizePrecisionMatrixConstants::setConstants(0.02, 0.2222, 9.0);
  supervoxel::setTrimParameters(max_size, max_pct, conn);
  const size_t nvol = (size_t)dims[0] * dims[1] * dims[2];
  std::vector<uint16_t> img(raw, raw + nvol);  // the reference writes nothing here, but holds a non-const pointer
  for (int32_t s = 0; s < n_sv; s++) {
    supervoxel sv;
    sv.PixelIdxList.assign(lin + lptr[s], lin + lptr[s + 1]);
    sv.dataPtr = img.data();
    thr_out[s] = sv.trimSupervoxel<unsigned short int>();
    cnt_out[s] = (int64_t)sv.PixelIdxList.size();
    for (size_t i = 0; i < sv.PixelIdxList.size(); i++) lin_out[lptr[s] + i] = sv.PixelIdxList[i];
    sv.weightedGaussianStatistics<unsigned short int>(true);
    for (int d = 0; d < 3; d++) cent_out[3 * s + d] = sv.centroid[d];
    intensity_out[s] = sv.intensity;
  }
  supervoxel::freeTrimParameters();
  return 0;
}

// order[0..n-m) = the original index of each supervoxel left after erasing those flagged
// (eraseIdx ascending, as main:598-600 builds it); returns n - m.
extern "C" int ref_erase_order(const uint8_t* erased, int32_t n, int32_t* order) {
  hierarchicalSegmentation hs;
  hs.currentSegmentatioSupervoxel.resize(n);
  hs.currentSegmentationNodes.assign(n, nullptr);
  std::vector<int> erase_idx;
  for (int32_t i = 0; i < n; i++) {
    hs.currentSegmentatioSupervoxel[i].PixelIdxList.assign(1, (uint64)i);  // the supervoxel's tag
    if (erased[i]) erase_idx.push_back(i);
  }
  hs.eraseSupervoxelFromCurrentSegmentation(erase_idx);
  const int32_t left = (int32_t)hs.currentSegmentatioSupervoxel.size();
  for (int32_t i = 0; i < left; i++) order[i] = (int32_t)hs.currentSegmentatioSupervoxel[i].PixelIdxList[0];
  return left;
}
