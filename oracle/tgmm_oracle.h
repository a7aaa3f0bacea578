/*
 * tgmm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of TGMM's per-time-point variational-inference EM over
 * supervoxels (reference: nmeth.3036-S2/src/UtilsCUDA/GMEMupdateCUDA.cu and
 * knnCuda.cu).  It is the checker for the CUDA path and the CPU baseline of the
 * benchmark; it is never linked into, called by, or shipped with the product.
 *
 * Two arithmetic modes:
 *   OR_MODE_FP64  -- every accumulation and every formula in FP64 (the "truth"
 *                    the CUDA path is measured against);
 *   OR_MODE_REF32 -- the reference kernels' own arithmetic: FP32 per-thread
 *                    accumulators over a 1024-thread stride, FP32 shared-memory
 *                    tree reductions, float temporaries in the mean update, the
 *                    reference's kNN replacement rule and slot order.  It pins this
 *                    oracle to the reference compiled from source (oracle/_ref) and
 *                    is the faithful OpenMP transcription timed as the CPU baseline.
 * Parity is pinned by running the reference's own GPU code (built from source by
 * oracle/build_ref.sh) on the seeded fixtures under tests/golden/.
 */
#ifndef TGMM_ORACLE_H_
#define TGMM_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_J 5
#define OR_MAX_SV 16

/* Same 288-byte layout as GaussianMixtureModelCUDA (GMEMupdateCUDA.h:22-57). */
typedef struct OrGaussian {
  double beta_k, nu_k, alpha_k;
  double m_k[3];
  double W_k[6];
  double eLD;   /* expectedLogDetCovarianceCUDA */
  double eLR;   /* expectedLogResponsivityCUDA */
  double splitScore;
  double beta_o, nu_o, alpha_o;
  double m_o[3];
  double W_o[6];
  unsigned char fixed;
  int32_t supervoxelIdx[OR_MAX_SV];
  int32_t supervoxelNum;
} OrGaussian;

enum { OR_MODE_FP64 = 0, OR_MODE_REF32 = 1 };
enum { OR_LL_AS_REFERENCE = 0, OR_LL_TRUE = 1 };

typedef struct OrParams {
  int32_t max_iter;
  int32_t w4dof;
  double tol;
  double lambda_min, lambda_max, max_exc;
  float scale[3];
  int32_t ll_mode;
  int32_t mode;
} OrParams;

typedef struct OrStats {
  int32_t iterations;
  int32_t converged;
  double ll;            /* value used by the convergence test */
  double ll_true;
  double ll_as_reference;
  double total_alpha;
  int32_t n_dead;
} OrStats;

/* ---- building blocks (each cites the reference lines it restates) ---- */
double or_digamma(double x);
double or_det3(const double* w);
void or_inv3(const double* w, double* out);
void or_eig3(const double* w, double* d, double* v);
/* knn: canonical = top-5 by (float distance, index), NaN as +inf; reference = the
 * reference kernel's replace-the-current-maximum rule and slot order. */
void or_knn_canonical(const float* query, int64_t nq, const float* ref_xyz, int32_t nref,
                      const float scale[3], int32_t* ind);
#define OR_MAXK 11
void or_knn_topk(const float* query, int64_t nq, const float* ref, int32_t nref, int32_t k,
                 const float scale[3], int32_t* ind, float* dist);
void or_knn_reference(const float* query, int64_t nq, const float* ref_xyz, int32_t nref,
                      const float scale[3], int32_t* ind);
double or_total_alpha(const OrGaussian* g, int32_t K, int32_t mode);
void or_prior_constants(OrGaussian* g, int32_t K, double total_alpha);
void or_estep(const OrGaussian* g, const float* query, int64_t N, const int64_t* lptr,
              int32_t S, const int32_t* ind, int32_t mode, float* rnk, double* L_out);
void or_mstep(const float* query, const float* img, int64_t N, const int64_t* lptr,
              int32_t S, int32_t K, const int32_t* ind, const float* rnk, int32_t mode,
              double* Nk, double* Xk, double* Sk);
void or_update(OrGaussian* g, int32_t K, const double* Nk, const double* Xk,
               const double* Sk, int32_t mode);
void or_regularize(OrGaussian* g, int32_t K, const float scale[3], int32_t w4dof,
                   double lmin, double lmax, double maxexc);
void or_kill(OrGaussian* g, int32_t K, double* Nk, double total_alpha);
void or_loglik(const OrGaussian* g, const float* query, const float* img, int64_t N,
               const int64_t* lptr, int32_t S, const int32_t* ind, double total_alpha,
               int32_t mode, double* ll_true, double* ll_as_ref);
void or_split_proposal(const OrGaussian* g, const float scale[3], OrGaussian* a, OrGaussian* b);
int or_local_likelihood(const OrGaussian* g, int32_t K, const float* query, const float* img, int64_t N,
                        const int64_t* lptr, int32_t S, const int32_t* ind, const int32_t* list_ptr,
                        const int32_t* list_idx, int32_t n_lists, int32_t mode, double* out);
void or_update_priors(OrGaussian* g, int32_t K, double beta_pct, double nu_pct,
                      double alpha_pct, double alpha_total);
void or_assign_supervoxels(const float* rnk, const int32_t* ind, int32_t S, OrGaussian* g,
                           int32_t K);

/* Whole EM for one time point (GMEMvariationalInferenceCUDAWithSupervoxels).
 * rnk/ind: 5*S outputs of the last iteration; ll_hist (optional): max_iter values. */
int or_em_run(const float* query, const float* img, const float* centroids,
              const int64_t* lptr, int64_t N, int32_t S, OrGaussian* g, int32_t K,
              const OrParams* p, float* rnk, int32_t* ind, double* ll_hist, OrStats* st);

/* Frame preparation from a supervoxel label volume (frame_oracle.c): trimming, size
 * filter, centroids, background subtraction, [0,1] rescale, SoA/CSR arrays. */
typedef struct OrFrameParams {
  int32_t max_size;  /* maxNucleiSize (3000) */
  float max_pct;     /* maxPercentileTrimSV (0.4) */
  int32_t conn;      /* conn3DsvTrim (6) */
  int32_t min_size;  /* minNucleiSize (50) */
} OrFrameParams;
int or_conn_offsets(int32_t conn, const int32_t dims[3], int64_t* off);
float or_otsu(const float* v, int32_t n);
uint16_t or_trim_threshold(const uint16_t* val, int32_t n, int32_t max_size, float max_pct, int32_t* seed);
int64_t or_trim_flood(const uint32_t* lin, const uint16_t* val, int64_t n, int32_t seed, uint16_t thr,
                      const int64_t* off, int32_t noff, int64_t nvol, uint8_t* keep);
void or_erase_order(const uint8_t* erased, int32_t n, int32_t* order);
/* 0 ok, 1 bad argument (label above n_labels, unknown neighbourhood), 2 outputs too small
 * (n_vox/n_sv still set), 5 every supervoxel erased. */
int or_frame_build(const uint16_t* raw, const uint32_t* label, const int32_t dims[3], int32_t n_labels,
                   const OrFrameParams* p, float* query, float* img, float* cent, int64_t* lptr, uint16_t* thr_out,
                   int64_t max_vox, int32_t max_sv, int64_t* n_vox, int32_t* n_sv);

int or_num_threads(void);
void or_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
