/*
 * tgmm_gmem.h -- C ABI of the B200 variational-inference Gaussian-mixture EM
 * over foreground supervoxels (one TGMM time point, or a batch of them).
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (TGMM_OK == 0).  Device pointers are marked "dev", host pointers "host".
 * Nothing here allocates implicitly except tgmm_plan_create (and the legacy
 * C++ shims declared in tgmm_legacy.h, which keep a cached plan).
 *
 * Reference interface each entry point replaces (paths inside the reference
 * project nmeth.3036-S2/src):
 *   struct TgmmGaussian      <- GaussianMixtureModelCUDA, UtilsCUDA/GMEMupdateCUDA.h:22-57
 *   tgmm_em_run              <- GMEMvariationalInferenceCUDAWithSupervoxels,
 *                               UtilsCUDA/GMEMupdateCUDA.h:92-98 (body GMEMupdateCUDA.cu:3985-4421)
 *   tgmm_knn                 <- knnCUDAinPlace, UtilsCUDA/knnCuda.h:225-226 (knnCuda.cu:781-817)
 *   tgmm_knn_k               <- knnCUDA_, temporalLogicalRules/knnCUDA/knnCuda.h:48-58
 *   tgmm_local_likelihood    <- calculateLocalLikelihood, UtilsCUDA/GMEMupdateCUDA.h:120-127
 *   tgmm_split_proposal      <- GaussianMixtureModel::splitGaussian(GM, id) + updatePriorsAfterSplitProposal,
 *                               GaussianMixtureModel.cpp:514-557, 912-922
 *   tgmm_split_round         <- the split round, mainTrackingGaussianMixtureModel.cpp:1233-1507
 *   tgmm_update_priors       <- GaussianMixtureModel::updatePriors, GaussianMixtureModel.cpp:892-910,
 *                               plus the nu_k*=2, W_k/=2 step of mainTrackingGaussianMixtureModel.cpp:961-969
 *   tgmm_frame_upload        <- GMEMinitializeMemoryWithSupervoxels, UtilsCUDA/GMEMupdateCUDA.h:132-137
 *   tgmm_frame_release       <- GMEMreleaseMemoryWithSupervoxels, UtilsCUDA/GMEMupdateCUDA.h:140-144
 *   tgmm_assign_supervoxels  <- post-loop rnk>0.5 assignment, GMEMupdateCUDA.cu:4310-4350
 *   tgmm_write_rnk_file      <- rnk/ind debug dump, GMEMupdateCUDA.cu:4364-4384
 *   tgmm_write_gmm_xml       <- GMM XML document, GMEMupdateCUDA.cu:4679-4716 (+ :3841-3844)
 */
#ifndef TGMM_GMEM_H_
#define TGMM_GMEM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- constants of the reference (constants.h:11-17, GMEMupdateCUDA.h:20) ---- */
#define TGMM_DIMS 3
#define TGMM_J 5                      /* maxGaussiansPerVoxel */
#define TGMM_MAX_SV_PER_GAUSSIAN 16   /* MAX_SUPERVOXELS_PER_GAUSSIAN */
#define TGMM_MIN_PI_FOR_DEAD 1e-5     /* minPi_kForDead */
#define TGMM_DEAD_SENTINEL (-1e32)    /* m_o[0] < -1e31 marks a dead Gaussian */

/* ---- status codes ---- */
enum {
  TGMM_OK = 0,
  TGMM_ERR_INVALID_ARG = 1,   /* null pointer, negative size, bad parameter */
  TGMM_ERR_BAD_SIZE = 2,      /* sizes beyond the plan capacity or the ABI limits */
  TGMM_ERR_BAD_CSR = 3,       /* labelListPtr not monotone / out of range */
  TGMM_ERR_NAN_INPUT = 4,     /* NaN/Inf in coordinates or Gaussian parameters */
  TGMM_ERR_CUDA = 5,          /* a CUDA runtime call failed */
  TGMM_ERR_OOM = 6,           /* device allocation failed */
  TGMM_ERR_DEVICE_FLAG = 7,   /* a kernel reported an internal inconsistency */
  TGMM_ERR_NOT_SET = 8,       /* regularisation constants not set (reference exit(3)) */
  TGMM_ERR_ADMISSION = 9,     /* served form: request does not fit in free HBM */
  TGMM_ERR_NO_SUPERVOXEL = 10 /* frame preparation erased every supervoxel (reference exit(5)) */
};

/* Per-Gaussian record.  Byte-for-byte the reference's 288-byte
 * GaussianMixtureModelCUDA (offsets: beta_k 0, m_k 24, W_k 48, eLD 96, beta_o 120,
 * m_o 144, W_o 168, fixed 216, supervoxelIdx 220, supervoxelNum 284).
 * W is the upper triangle, row major: 00,01,02,11,12,22. */
typedef struct TgmmGaussian {
  double beta_k, nu_k, alpha_k;
  double m_k[3];
  double W_k[6];
  double expectedLogDetCovarianceCUDA;
  double expectedLogResponsivityCUDA;
  double splitScore;
  double beta_o, nu_o, alpha_o;
  double m_o[3];
  double W_o[6];
  unsigned char fixed; /* C++ bool */
  int32_t supervoxelIdx[TGMM_MAX_SV_PER_GAUSSIAN];
  int32_t supervoxelNum;
} TgmmGaussian;

/* Log-likelihood flavour used by the convergence test. */
enum {
  TGMM_LL_AS_REFERENCE = 0, /* the reference's per-thread overwrite for supervoxels with
                               more than 1024 voxels (GMEMupdateCUDA.cu:1961-1962) */
  TGMM_LL_TRUE = 1          /* every foreground voxel counted */
};

/* Precision of the per-voxel log-likelihood terms (accumulation is always FP64). */
enum {
  TGMM_LLPREC_MIXED = 0, /* dominant component in FP64, log1p correction of the others in FP32 */
  TGMM_LLPREC_FP64 = 1   /* every component in FP64 */
};

typedef struct TgmmEmParams {
  int32_t max_iter_em;      /* maxIterEM (reference default 400) */
  int32_t w4dof;            /* regularize_W4DOF (reference main sets true) */
  double tol_likelihood;    /* tolLikelihood (default 1e-6; 0 = run max_iter_em unless ll repeats) */
  double lambda_min;        /* regularizePrecisionMatrixConstants::lambdaMin (0.02) */
  double lambda_max;        /* lambdaMax (0.2222) */
  double max_excentricity;  /* maxExcentricity (9) */
  float scale[3];           /* anisotropy scale of the kNN distance, e.g. {1,1,2}
                               (the reference's scaleCUDA, uploadScaleCUDA) */
  float reg_scale[3];       /* scale of the regularisation (scaleGMEMCUDA, copyScaleToDvice);
                               all zero = same as scale */
  int32_t ll_mode;          /* TGMM_LL_AS_REFERENCE or TGMM_LL_TRUE */
  int32_t ll_precision;     /* TGMM_LLPREC_MIXED or TGMM_LLPREC_FP64 */
  int32_t frame;            /* only echoed in logs */
} TgmmEmParams;

/* Fill *p with the reference defaults (parseConfigFile.h:152-195, main:124). */
void tgmm_default_params(TgmmEmParams* p);

/* One time point on the device.  Layout is the reference's:
 *   query[d*n_vox + v]      voxel coordinates, SoA (x block, y block, z block), float
 *   img[v]                  intensity in [0,1]
 *   centroids[d*n_sv + s]   supervoxel centroids, SoA
 *   label_ptr[0..n_sv]      CSR: voxels of supervoxel s are [label_ptr[s], label_ptr[s+1]) */
typedef struct TgmmFrame {
  const float* query;        /* dev */
  const float* img;          /* dev */
  const float* centroids;    /* dev */
  const int64_t* label_ptr;  /* dev */
  int64_t n_vox;
  int32_t n_sv;
  int32_t n_gauss;
} TgmmFrame;

/* Bits of TgmmEmStats.device_flags: what the kernels met during the call.  The overflow
 * bits name the exact slower branch a frame took (results are the same either way); the
 * others make the call return an error status. */
#define TGMM_FLAG_BAD_CSR 1         /* labelListPtr not a CSR over the voxels (TGMM_ERR_BAD_CSR) */
#define TGMM_FLAG_NAN_INPUT 2       /* NaN coordinate or intensity (TGMM_ERR_NAN_INPUT) */
#define TGMM_FLAG_FEW_GAUSS 4       /* fewer than 5 Gaussians in a frame (TGMM_ERR_BAD_SIZE) */
#define TGMM_FLAG_BUCKET_OVERFLOW 8 /* a Gaussian was a candidate of more than 32 (slot, supervoxel)
                                       pairs: its M-step sums came from an ordered scan of the frame */
#define TGMM_FLAG_ASSIGN_OVERFLOW 16 /* more than 32 supervoxels with rnk > 0.5 on one Gaussian: its
                                        supervoxelIdx came from an ordered scan of the frame */
#define TGMM_FLAG_CELL_OVERFLOW 32  /* more than 32 Gaussian centres in one kNN grid cell: the
                                       frame's kNN scanned every Gaussian */
#define TGMM_FLAG_STAGE_TIMEOUT 64  /* a voxel tile copy missed the plan's wait limit
                                       (TGMM_ERR_DEVICE_FLAG; the outputs are not valid) */

typedef struct TgmmEmStats {
  int32_t iterations;       /* EM iterations executed (numIterEM-1 in the reference) */
  int32_t converged;        /* 1 if stopped by the tolerance test */
  double ll;                /* log-likelihood used by the convergence test (last iteration) */
  double ll_true;           /* every-voxel log-likelihood (last iteration) */
  double ll_as_reference;   /* overwrite-quirk log-likelihood (last iteration) */
  double total_alpha;       /* sum of alpha_k after the last kill step */
  int32_t n_dead;           /* dead Gaussians after the call */
  int32_t device_flags;     /* bit mask of device-side anomaly flags (0 = none) */
  int32_t knn_searches;     /* supervoxel kNN grid searches after the first iteration: the
                               later iterations take each supervoxel's five candidates from
                               its list of 8 nearest unless its Gaussians moved too far */
  int32_t reserved;
} TgmmEmStats;

/* ---- plans: all device workspace, sized once, reused by every call ---- */
typedef struct TgmmPlan TgmmPlan;

/* Capacity of one plan.  A batch may hold up to max_frames frames whose totals fit. */
typedef struct TgmmPlanDesc {
  int64_t max_vox;     /* total voxels over the batch */
  int32_t max_sv;      /* total supervoxels */
  int32_t max_gauss;   /* total Gaussians */
  int32_t max_frames;  /* frames per batch */
  int32_t device;      /* CUDA device ordinal */
} TgmmPlanDesc;

int tgmm_plan_create(const TgmmPlanDesc* desc, TgmmPlan** out);
int tgmm_plan_destroy(TgmmPlan* plan);
/* Bytes of device memory tgmm_plan_create would allocate for desc. */
int64_t tgmm_plan_bytes(const TgmmPlanDesc* desc);

/* Single time point, Gaussians in HOST memory (read, updated in place, including
 * supervoxelIdx/supervoxelNum), rnk/ind written to DEVICE buffers of n_sv*5
 * (slot-major: rnk[j*n_sv+s]); ind_tr_dev (optional, may be NULL) receives the
 * Gaussian-sorted keys like the reference's indCUDAtr.  stream: cudaStream_t or NULL. */
int tgmm_em_run(TgmmPlan* plan, const TgmmFrame* frame, TgmmGaussian* gm_host,
                float* rnk_dev, int32_t* ind_dev, int32_t* ind_tr_dev,
                const TgmmEmParams* params, TgmmEmStats* stats, void* stream);

/* Same with the Gaussians already on the device (gm_dev, n_gauss records), updated in
 * place on the device; supervoxelIdx/Num are filled on the device.  No host sync
 * unless stats != NULL. */
int tgmm_em_run_device(TgmmPlan* plan, const TgmmFrame* frame, TgmmGaussian* gm_dev,
                       float* rnk_dev, int32_t* ind_dev, const TgmmEmParams* params,
                       TgmmEmStats* stats, void* stream);

/* Batched form: n_frames independent time points, each with its own frame and its own
 * Gaussian array (device), run together, one launch per EM phase over all frames.
 * rnk_dev[f]/ind_dev[f] are per-frame outputs.  stats may be NULL or an array of n_frames.
 * Results are bit-identical to running each frame alone through tgmm_em_run_device. */
int tgmm_em_run_batch(TgmmPlan* plan, int32_t n_frames, const TgmmFrame* frames,
                      TgmmGaussian* const* gm_dev, float* const* rnk_dev,
                      int32_t* const* ind_dev, const TgmmEmParams* params,
                      TgmmEmStats* stats, void* stream);

/* kNN of n_query points (SoA, dev) against n_ref points (AoS xyz float, dev), ordered by
 * (scaled squared distance, index); ind_dev[j*n_query+q].  Exact. */
int tgmm_knn(const float* query_dev, int64_t n_query, const float* ref_xyz_dev,
             int32_t n_ref, const float scale[3], int32_t* ind_dev, void* stream);

/* The tracking graph's supervoxel kNN (knnCUDA_, temporalLogicalRules/knnCUDA/knnCuda.h:48-58,
 * body knnCuda.cu:56-140): the k nearest (1 <= k <= 11) of n_query points (SoA, dev) among
 * n_ref points (SoA: x block, y block, z block, dev) by the same scaled squared distance, with
 * the distances: ind_dev[j*n_query+q] and, if dist_dev is not NULL, dist_dev[j*n_query+q],
 * ordered by (distance, index).  A slot with no point closer than 1e32 holds index -1 and
 * distance 1e32 (the reference leaves such indices unset).  Exact; ties go to the lower
 * index (the reference's replacement rule lets the later one win and leaves the slots
 * unsorted). */
int tgmm_knn_k(const float* query_dev, int64_t n_query, const float* ref_dev, int32_t n_ref,
               int32_t k, const float scale[3], int32_t* ind_dev, float* dist_dev, void* stream);

/* No counterpart in the reference.  The same exact kNN as tgmm_knn for callers that may not
 * allocate device memory -- code whose device memory belongs to another allocator (a
 * framework's caching pool, a host application's fixed arena) or that runs on a path where
 * an allocation's latency or failure is not acceptable.  It calls no cudaMalloc, cudaFree or
 * allocating library routine; its scratch is a file-scope device array of about 2.8 MB that
 * every GPU which loads the library holds until the process exits.  At most
 * TGMM_KNN_NOALLOC_MAX_REF reference points (TGMM_ERR_BAD_SIZE beyond).  The first call on a
 * device looks the array's device address up with that device current; make that first call
 * before any stream capture.  All calls share the one array: calls that overlap on the GPU
 * (different streams, or different host threads) race and must be serialised by the caller.
 * The looked-up address is kept for the life of the process: after cudaDeviceReset on a
 * device, do not call this entry point on that device again. */
#define TGMM_KNN_NOALLOC_MAX_REF 65535
int tgmm_knn_noalloc(const float* query_dev, int64_t n_query, const float* ref_xyz_dev,
                     int32_t n_ref, const float scale[3], int32_t* ind_dev, void* stream);

/* Local log-likelihood of supervoxel lists, the likelihood the split round compares before
 * and after a proposed division (calculateLocalLikelihood, UtilsCUDA/GMEMupdateCUDA.h:120-127;
 * body GMEMupdateCUDA.cu:2952-3055, kernel :1989-2103).  For list i (supervoxel indices
 * list_idx[list_ptr[i] .. list_ptr[i+1]), host arrays; a supervoxel listed twice counts twice)
 * ll_out[i] (host) = the sum over its supervoxels s of the reference's as-reference
 * log-likelihood of s's voxels under s's five candidates ind_dev[j*n_sv+s] and the Gaussians
 * gm_dev (n_gauss records, device): each voxel's density is
 * sum_j sqrt(det W_j nu_j^3)/(2 pi)^{3/2} exp(-nu_j d'W_j d/2) alpha_j/A, A the sum of alpha
 * over all n_gauss records, and of the voxels t, t + 1024, ... of s only the last with a
 * positive density adds I ln(density).  Every step in FP64 (the reference sums in float).  An
 * empty list gives 0.  The frame needs query, img, label_ptr, n_vox and n_sv (centroids are not
 * read).  Synchronises `stream`. */
int tgmm_local_likelihood(const TgmmFrame* frame, const int32_t* ind_dev, const TgmmGaussian* gm_dev,
                          int32_t n_gauss, const int32_t* list_ptr, const int32_t* list_idx, int32_t n_lists,
                          double* ll_out, void* stream);

/* The split proposal of one Gaussian (GaussianMixtureModel::splitGaussian(GM, id),
 * GaussianMixtureModel.cpp:514-557, then updatePriorsAfterSplitProposal, :912-922, on both
 * halves), on host records: S = nu W / (s_i s_j); lmin, v its smallest eigenvalue and
 * eigenvector, lmax its largest; sigma = 1/sqrt(max(lmin, 1e-3)); both halves take
 * W = (lmax/nu) I with W_ii *= s_i s_i and N_k/2 (N_k = nu_k - nu_o); *a (the split Gaussian)
 * at m + sigma v, *b (the new one) at m - sigma v; then m_o = m_k, beta_o = max(N_k/2, 1e-5),
 * nu_o = max(N_k/2, 3), W_o = W_k nu_k / nu_o.  v's sign makes its largest-magnitude
 * component positive (the reference takes its Eigen solver's sign, so a and b can trade
 * places against it).  Host only; no device work. */
int tgmm_split_proposal(const TgmmGaussian* g, const float scale[3], TgmmGaussian* a, TgmmGaussian* b);

/* The split round of one time point (mainTrackingGaussianMixtureModel.cpp:1233-1507) with the
 * candidates chosen by the caller (the reference's 3D Haar classifier picks them) and the
 * accept/reject decision left to the caller (the reference's likelihoodRatioTestSplitMerge,
 * called at main:1373, is not defined in its sources).  gm_host holds the n_gauss records of
 * the first EM (with its supervoxelIdx/Num) and room for n_split more; ind_dev that EM's
 * candidates (5*n_sv).  For each candidate cand[i] (distinct, alive):
 *   ll_before[i] = tgmm_local_likelihood of its supervoxels under the first EM's mixture;
 *   it is split by tgmm_split_proposal (scale: params->reg_scale, or scale when that is all
 *   zero), the new Gaussian stored at gm_host[n_gauss + i]; every other Gaussian gets
 *   fixed = 1, as the reference fixes them for this EM (clear them before the next frame; a
 *   candidate keeps its own flag);
 * then the EM on the n_gauss + n_split records (tgmm_em_run: gm_host updated, rnk_dev and
 * ind_out_dev written, stats if not NULL), and ll_after[i] = the local log-likelihood of the
 * same supervoxels under the new mixture and candidates.  The plan must hold
 * n_gauss + n_split Gaussians.  Synchronises `stream`. */
int tgmm_split_round(TgmmPlan* plan, const TgmmFrame* frame, TgmmGaussian* gm_host, int32_t n_gauss,
                     const int32_t* ind_dev, const int32_t* cand, int32_t n_split, float* rnk_dev,
                     int32_t* ind_out_dev, const TgmmEmParams* params, double* ll_before, double* ll_after,
                     TgmmEmStats* stats, void* stream);

/* Posterior -> prior for the next time point, on the device (served form):
 * N_k = nu_k - nu_o; m_o = m_k; beta_o = max(beta_pct*N_k, 1e-5);
 * nu_o = max(nu_pct*N_k, 3); W_o = W_k*nu_k/nu_o; alpha_o = alpha_total*1e-5*alpha_pct
 * (unchanged when alpha_total < 0); then nu_k *= 2, W_k /= 2.  alpha_total < 0 and
 * compute_alpha_total != 0 means "use the sum of alpha_k of this array". */
int tgmm_update_priors(TgmmGaussian* gm_dev, int32_t n_gauss, double beta_pct,
                       double nu_pct, double alpha_pct, double alpha_total,
                       int32_t compute_alpha_total, void* stream);

/* Frame preparation on the device: the EM's input arrays from the raw 16-bit image and the
 * label volume of the segmentation at tau (mainTrackingGaussianMixtureModel.cpp:553-651 and
 * 774-870; supervoxel.cpp:1410-1450, 1556-1747).  Each supervoxel is trimmed as the
 * reference's trimSupervoxel does -- threshold = the largest of its (n - max_nuclei_size)-th
 * value, its (1 - max_percentile) percentile and Otsu's threshold, then the voxels above it
 * connected to its brightest voxel through the conn3d neighbourhood (linear-index offsets, as
 * the reference builds them) -- supervoxels left with fewer than min_nuclei_size voxels are
 * erased in the reference's order (each erased index trades places with the current last
 * supervoxel), the centroids are the FP32 raw-intensity-weighted means of the kept voxels,
 * each kept supervoxel's threshold is subtracted from its voxels (16-bit), every other voxel
 * counts as 0, and the volume is rescaled to [0,1] as mylib's Scale_Array_To_Range does.
 *
 * raw, label: X*Y*Z device arrays (x fastest; label 16-byte aligned); label l in
 * 1..n_labels puts a voxel in supervoxel l-1 (0: none); X*Y*Z < 2^32.  workspace: device memory of at least
 * tgmm_frame_build_bytes(dims, n_labels) bytes (no other allocation is made).  Outputs
 * (device): query[3*max_vox] (SoA with stride *n_vox), img[max_vox],
 * centroids[3*max_sv] (SoA with stride *n_sv), label_ptr[max_sv+1], and, if thr is not
 * NULL, thr[max_sv] (each output supervoxel's threshold).  *n_vox and *n_sv are set on
 * TGMM_OK and on TGMM_ERR_BAD_SIZE (outputs too small; nothing written).  Synchronises
 * `stream`.  The reference's deltaZ split of tall supervoxels (main:566-592) needs the
 * segmentation hierarchy and is not part of this step. */
typedef struct TgmmFrameBuildParams {
  int32_t max_nuclei_size; /* 3000 */
  float max_percentile;    /* 0.4 */
  int32_t conn3d;          /* 4, 6, 8, 26 or 74 (6) */
  int32_t min_nuclei_size; /* 50 */
} TgmmFrameBuildParams;
void tgmm_frame_build_default_params(TgmmFrameBuildParams* p);
/* Measurement hook (no reference counterpart): tgmm_frame_build with CUDA events between its
 * steps; stage_ms[TGMM_FRAME_BUILD_STAGES] receives each step's milliseconds: clear + init,
 * volume scan, supervoxel CSR, grouping, trimming, erase order, output CSR, emission. */
#define TGMM_FRAME_BUILD_STAGES 8
int64_t tgmm_frame_build_bytes(const int32_t dims[3], int32_t n_labels);
int tgmm_frame_build(const uint16_t* raw_dev, const uint32_t* label_dev, const int32_t dims[3],
                     int32_t n_labels, const TgmmFrameBuildParams* p, void* workspace_dev,
                     int64_t workspace_bytes, float* query_dev, float* img_dev,
                     float* centroids_dev, int64_t* label_ptr_dev, uint16_t* thr_dev,
                     int64_t max_vox, int32_t max_sv, int64_t* n_vox, int32_t* n_sv,
                     void* stream);
int tgmm_frame_build_timed(const uint16_t* raw_dev, const uint32_t* label_dev,
                           const int32_t dims[3], int32_t n_labels, const TgmmFrameBuildParams* p,
                           void* workspace_dev, int64_t workspace_bytes, float* query_dev,
                           float* img_dev, float* centroids_dev, int64_t* label_ptr_dev,
                           uint16_t* thr_dev, int64_t max_vox, int32_t max_sv, int64_t* n_vox,
                           int32_t* n_sv, void* stream, float* stage_ms);

/* The same build from the segmentation as per-supervoxel pixel lists, the form the tracking
 * program holds it in (supervoxel::PixelIdxList, temporalLogicalRules/supervoxel.h:72; the
 * lists main:553-651 trims), so that no volume crosses to the device: supervoxel s
 * (label s+1 of tgmm_frame_build) is lin[lists_ptr[s] .. lists_ptr[s+1]) (uint32 linear
 * indices, x fastest, strictly ascending, inside the volume; the lists disjoint) with the raw
 * values val[...] of those voxels (uint16).  lists_ptr: n_labels + 1 int64 on the device, 0 ..
 * n_list.  Outputs, their sizes and the status codes as tgmm_frame_build, bit for bit the same
 * arrays for the same segmentation; a list that is not ascending, leaves the volume or a CSR
 * outside 0 .. n_list gives TGMM_ERR_DEVICE_FLAG.  A flood that leaves shared memory (box above
 * 65536 voxels) finds a neighbour in the supervoxel's own list by binary search, as the
 * reference's lower_bound does.  workspace: tgmm_frame_build_lists_bytes(dims, n_labels,
 * n_list) bytes.  stage_ms (optional, host): TGMM_FRAME_BUILD_STAGES step times as
 * tgmm_frame_build_timed's (the scan's place holds the lists' check and boxes; no CSR or
 * grouping step).  Synchronous on `stream` (the sizes are read back). */
int64_t tgmm_frame_build_lists_bytes(const int32_t dims[3], int32_t n_labels, int64_t n_list);
int tgmm_frame_build_lists(const uint32_t* lin_dev, const uint16_t* val_dev, const int64_t* lists_ptr_dev,
                           int64_t n_list, const int32_t dims[3], int32_t n_labels,
                           const TgmmFrameBuildParams* p, void* workspace_dev, int64_t workspace_bytes,
                           float* query_dev, float* img_dev, float* centroids_dev, int64_t* label_ptr_dev,
                           uint16_t* thr_dev, int64_t max_vox, int32_t max_sv, int64_t* n_vox, int32_t* n_sv,
                           void* stream, float* stage_ms);

/* A frame's voxels in compact form (6 bytes a voxel instead of 16) expanded on the device into
 * the float arrays the EM reads: lin[v] = x + X (y + Y z) (uint32) gives query (x block, y
 * block, z block; query[3*n_vox]) and raw[v] (uint16) gives img[v] =
 * (float)(((double)raw[v] - raw_offset) / raw_denom) -- the reference's per-supervoxel
 * background subtraction and [0,1] rescale (mainTrackingGaussianMixtureModel.cpp:616, 664-669)
 * when raw_offset is the threshold and raw_denom the range, bit for bit the arrays the host
 * builds.  dims = X, Y, Z (X*Y*Z <= 2^32).  No reference counterpart: it cuts the
 * host-to-device bytes of a frame to 6 per voxel.  Asynchronous on `stream`. */
int tgmm_frame_expand(const uint32_t* lin_dev, const uint16_t* raw_dev, int64_t n_vox, const int32_t dims[3],
                      double raw_offset, double raw_denom, float* query_dev, float* img_dev, void* stream);

/* The same float arrays from runs, about 3 bytes a voxel for nuclei volumes (a supervoxel's
 * voxels, ascending in linear index, fall into runs of consecutive indices, ~6 voxels each in
 * the synthetic frames): the voxels of supervoxel s (label_ptr[s] .. label_ptr[s+1]) are the
 * runs run_ptr[s] .. run_ptr[s+1] in order, run r being the run_len[r] linear indices
 * run_start[r], run_start[r] + 1, ...; raw[v] (uint16, voxel order) as tgmm_frame_expand.  The
 * runs of a supervoxel must cover exactly its voxel range: nothing is written outside that
 * range whatever the tables say, and voxels they leave out keep what the arrays held.  A
 * supervoxel with an invalid range is skipped (the EM flags the CSR), and no run outside
 * 0 .. n_runs is read.  No reference
 * counterpart: it halves the host-to-device bytes of tgmm_frame_expand's codes.
 * Asynchronous on `stream`; every array on the device. */
int tgmm_frame_expand_runs(const int32_t* run_ptr_dev, const uint32_t* run_start_dev, const uint16_t* run_len_dev,
                           const uint16_t* raw_dev, const int64_t* label_ptr_dev, int32_t n_sv, int64_t n_runs,
                           int64_t n_vox, const int32_t dims[3], double raw_offset, double raw_denom, float* query_dev,
                           float* img_dev, void* stream);

/* Allocate device buffers and upload one frame from host arrays (legacy ownership model). */
int tgmm_frame_upload(const float* query_host, const float* img_host,
                      const float* centroids_host, const int64_t* label_ptr_host,
                      int64_t n_vox, int32_t n_sv, TgmmFrame* out_frame);
int tgmm_frame_release(TgmmFrame* frame);

/* Reference post-loop assignment on host arrays: for j in 0..4, s in 0..n_sv-1, if
 * rnk[j*n_sv+s] > 0.5, append s to gm[ind].supervoxelIdx (at most 16). */
int tgmm_assign_supervoxels(const float* rnk_host, const int32_t* ind_host, int32_t n_sv,
                            TgmmGaussian* gm_host, int32_t n_gauss);

/* Reference GMM XML document of n Gaussians (host records): the header, one
 * <GaussianMixtureModel> element per Gaussian with its index as id, the footer -- the text
 * the reference's writeXMLheader / writeXML / writeXMLfooter produce
 * (GMEMupdateCUDA.h:43-52, GMEMupdateCUDA.cu:4679-4716, as called at :3841-3844). */
int tgmm_write_gmm_xml(const char* path, const TgmmGaussian* gm_host, int32_t n);

/* Reference rnk dump: int n_sv, int 5, float rnk[5*n_sv], int ind[5*n_sv]. */
int tgmm_write_rnk_file(const char* path, const float* rnk_host, const int32_t* ind_host,
                        int32_t n_sv);

/* Measurement hook (no reference counterpart): launch one kernel of the EM `reps` times
 * back to back on `stream` between two CUDA events, on the batch last run through this
 * plan, and return the average milliseconds per launch.  The plan's per-frame EM state
 * is restored afterwards; the results of the last call stay as they were returned. */
enum {
  TGMM_KERNEL_MOMENTS = 0,    /* per-supervoxel moment pass (once per call) */
  TGMM_KERNEL_LL_PASS = 2,    /* log-likelihood voxel pass alone */
  TGMM_KERNEL_LL_PASS_KNN = 3 /* the voxel pass running the next iteration's kNN/E-step */
};
int tgmm_plan_time_kernel(TgmmPlan* plan, int32_t kernel, int32_t reps, float* ms_per_launch, void* stream);

/* Lanes per supervoxel of the kNN/E-step kernel (4, 8, 16 or 32; default 8; with 4 lanes a
 * lane holds two list members and lane 0 two candidates, and the kNN/E-step always runs in
 * its own kernel).  Every width computes the same bits; only the speed differs with the
 * batch (supervoxel count, cells per ring, candidates per cell).  No reference counterpart: the reference runs one fixed
 * launch shape (knnCuda.cu:781-817, GMEMupdateCUDA.cu:3120-3141). */
int tgmm_plan_set_knn_group(TgmmPlan* plan, int32_t lanes);

/* Whether the log-likelihood voxel pass of each iteration also runs the next iteration's
 * kNN/E-step (1) or that kernel follows the pass (0, the default).  Both give the same
 * bits; running them together pays off when the voxel pass leaves the SMs idle (small
 * frames), apart when the batch is large.  No reference counterpart. */
int tgmm_plan_set_knn_fusion(TgmmPlan* plan, int32_t on);
/* Wait limit, in nanoseconds, of each voxel tile copy of the voxel passes (default 1 s;
 * 1 ns .. 60 s).  No reference counterpart.  A copy that misses it flags its frame with
 * TGMM_FLAG_STAGE_TIMEOUT and the call returns TGMM_ERR_DEVICE_FLAG; the warp that met it
 * still waits for its own copies in flight (bounded by 1 s) before it leaves, and the next
 * call on the plan starts from a clean state.  A short limit exercises that path. */
int tgmm_plan_set_stage_wait(TgmmPlan* plan, int64_t wait_ns);

/* The plan's current kNN/E-step width and arrangement (either pointer may be NULL). */
int tgmm_plan_tuning(TgmmPlan* plan, int32_t* lanes, int32_t* fused);

/* Autotuner (no reference counterpart): runs the whole EM call of the batch (the
 * arguments of tgmm_em_run_batch; at most 20 iterations) `reps` times for every kNN/E-step
 * width and arrangement, after a first run that warms up, and keeps the fastest pair in
 * the plan (the width is returned in *lanes_out, tgmm_plan_tuning reads both).  The runs
 * work on a copy of the Gaussians in the plan: gm_dev is only read.  rnk_dev and ind_dev
 * are overwritten; the results of later calls do not depend on the choices. */
int tgmm_plan_autotune(TgmmPlan* plan, int32_t n_frames, const TgmmFrame* frames,
                       TgmmGaussian* const* gm_dev, float* const* rnk_dev, int32_t* const* ind_dev,
                       const TgmmEmParams* params, int32_t reps, int32_t* lanes_out, void* stream);

/* Last CUDA error string recorded by this library on the calling thread. */
const char* tgmm_last_error(void);
/* Library version string. */
const char* tgmm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TGMM_GMEM_H_ */
