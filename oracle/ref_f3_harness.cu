// ref_f3_harness.cu -- TEST INFRASTRUCTURE ONLY.  A C entry point over the reference's
// supervoxel kNN of the tracking graph (temporalLogicalRules/knnCUDA/knnCuda.cu, compiled
// from the reference sources by oracle/build_ref.sh into oracle/_ref/libtgmm_ref_f3.so), so
// that tests can compare tgmm_knn_k with it.  Its kernel returns early for surplus threads
// of a block before a __syncthreads(): callers keep n_query <= 1024 (one full block).
#include "knnCuda.h"

extern "C" int ref_knn_k(int* ind, float* dist, float* query, float* ref, long long nq, int nref, int k,
                         float* scale) {
  if (nq < 1 || nq > 1024 || k < 1 || k > 11) return 1;
  return knnCUDA_(ind, dist, query, ref, nq, nref, k, scale, 0);
}
