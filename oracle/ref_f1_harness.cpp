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

// The reference's host frame build (mainTrackingGaussianMixtureModel.cpp:553-651, 664-669,
// 774-870) with its own trimming, statistics and erase: the loop around them is main's, kept
// step for step (trim; erase below min_size, else statistics, subtract the threshold and mark
// the voxels; erase; zero every unmarked voxel; to float; Scale_Array_To_Range(0, 1) over the
// whole volume as mylib/array.p:2798-2822 computes it; the SoA/CSR arrays).  The deltaZ split
// (main:566-592) needs the segmentation hierarchy and is not run.  The arrays hold the kept
// voxels only (stride = their count; the reference's stride also counts the erased ones'
// voxels).  Returns 0, 5 (every supervoxel erased: the reference's exit(5)) or 2 (max_vox too
// small; *n_vox set).
extern "C" int ref_frame_build(const uint16_t* raw, const int32_t* dims, const int64_t* lptr, const uint64_t* lin,
                               int32_t n, int32_t max_size, float max_pct, int32_t conn, int32_t min_size,
                               float* query, float* img_out, float* cent, int64_t* lptr_out, int64_t max_vox,
                               int64_t* n_vox, int32_t* n_sv) {
  uint64 dd[3] = {(uint64)dims[0], (uint64)dims[1], (uint64)dims[2]};
  supervoxel::setDataDims(dd);
  const size_t nvol = (size_t)dd[0] * dd[1] * dd[2];
  supervoxel::dataSizeInBytes = sizeof(uint16_t) * nvol;
  float scale[3] = {1.f, 1.f, 2.f};
  supervoxel::setScale(scale);
  regularizePrecisionMatrixConstants::setConstants(0.02, 0.2222, 9.0);
  supervoxel::setTrimParameters(max_size, max_pct, conn);
  std::vector<uint16_t> img(raw, raw + nvol);
  hierarchicalSegmentation hs;
  hs.currentSegmentatioSupervoxel.resize(n);
  hs.currentSegmentationNodes.assign(n, nullptr);
  for (int32_t s = 0; s < n; s++) {
    hs.currentSegmentatioSupervoxel[s].PixelIdxList.assign(lin + lptr[s], lin + lptr[s + 1]);
    hs.currentSegmentatioSupervoxel[s].dataPtr = img.data();
  }
  std::vector<char> visited(nvol, 0);
  std::vector<int> erase_idx;
  for (size_t ii = 0; ii < hs.currentSegmentatioSupervoxel.size(); ii++) {
    supervoxel& sv = hs.currentSegmentatioSupervoxel[ii];
    const uint16_t thr = sv.trimSupervoxel<unsigned short int>();
    if ((int)sv.PixelIdxList.size() < min_size) {
      erase_idx.push_back((int)ii);
    } else {
      sv.weightedGaussianStatistics<unsigned short int>(true);
      for (uint64 v : sv.PixelIdxList) {
        img[v] -= thr;
        visited[v] = 1;
      }
    }
    sv.localBackgroundSubtracted = true;
  }
  supervoxel::freeTrimParameters();
  if (erase_idx.size() >= hs.currentSegmentatioSupervoxel.size()) return 5;
  hs.eraseSupervoxelFromCurrentSegmentation(erase_idx);
  for (size_t v = 0; v < nvol; v++)
    if (!visited[v]) img[v] = 0;
  // to float, then Scale_Array_To_Range(img, 0, 1)
  std::vector<float> f(nvol);
  for (size_t v = 0; v < nvol; v++) f[v] = (float)img[v];
  float mn = f[0], mx = f[0];
  for (size_t v = nvol; v-- > 1;) {
    const float x = f[v];
    if (x < mn)
      mn = x;
    else if (x > mx)
      mx = x;
  }
  if (mx != mn) {
    double fct = 1.0;
    fct /= (double)mx - (double)mn;
    const double off = 0.0 / fct - (double)mn;
    for (size_t v = 0; v < nvol; v++) f[v] = (float)(fct * (f[v] + off));
  }
  const int32_t S = (int32_t)hs.currentSegmentatioSupervoxel.size();
  int64_t N = 0;
  for (int32_t s = 0; s < S; s++) N += (int64_t)hs.currentSegmentatioSupervoxel[s].PixelIdxList.size();
  *n_vox = N;
  *n_sv = S;
  if (N > max_vox) return 2;
  int64_t at = 0;
  lptr_out[0] = 0;
  for (int32_t s = 0; s < S; s++) {
    const supervoxel& sv = hs.currentSegmentatioSupervoxel[s];
    for (uint64 v : sv.PixelIdxList) {
      img_out[at] = f[v];
      query[at] = (float)(v % dd[0]);
      query[N + at] = (float)((v / dd[0]) % dd[1]);
      query[2 * N + at] = (float)(v / (dd[0] * dd[1]));
      at++;
    }
    lptr_out[s + 1] = at;
    for (int d = 0; d < 3; d++) cent[(int64_t)d * S + s] = sv.centroid[d];
  }
  return 0;
}
