/*
 * tgmm_serve.h -- served form of the B200 EM: a request loop over batched EM calls.
 *
 * The reference runs one time point at a time from its tracking loop
 * (mainTrackingGaussianMixtureModel.cpp:1065-1107) and carries each lineage's Gaussians
 * from frame to frame on the host: the posterior of frame t becomes the prior of frame
 * t+1 through GaussianMixtureModel::updatePriors (GaussianMixtureModel.cpp:892-910) with
 * alphaTotal = sum of alpha_k, followed by nu_k *= 2, W_k /= 2 (main:946-969).  A server
 * keeps that chain on the device: a lineage's Gaussians stay resident, each frame of the
 * lineage runs with the current Gaussians as posterior-and-prior, and after it the update
 * above runs on the device (tgmm_update_priors).
 *
 * Frames of different lineages are independent.  A worker thread admits submitted frames
 * against the server's HBM budget (their input and output buffers) in arrival order and
 * uploads each on a copy stream as soon as it is admitted; it packs the ready frames whose
 * lineage has no frame in flight into a batch and runs the batch through
 * tgmm_em_run_batch -- one launch per EM phase for all its frames -- on one of `lanes`
 * streams, each with its own plan.  Uploads, batches and downloads of different frames
 * overlap.  Results are bit-identical to running each frame alone.
 *
 * Every entry point returns an int status (tgmm_gmem.h); results carry their own status.
 */
#ifndef TGMM_SERVE_H_
#define TGMM_SERVE_H_

#include "tgmm_gmem.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct TgmmServer TgmmServer;

typedef struct TgmmServerDesc {
  int32_t device;            /* CUDA device ordinal */
  int64_t hbm_budget;        /* device bytes for frame buffers and resident lineages;
                                0 = 80% of the free memory left after the plans */
  int32_t lanes;             /* batches in flight (one stream and one plan each), >= 1 */
  int32_t max_batch_frames;  /* frames per batch */
  int64_t max_batch_vox;     /* voxels per batch */
  int32_t max_batch_sv;      /* supervoxels per batch */
  int32_t max_batch_gauss;   /* Gaussians per batch */
  TgmmEmParams params;       /* EM parameters of every frame */
  double beta_pct;           /* posterior -> prior after each frame (betaPercentageOfN_k, 0.01) */
  double nu_pct;             /* nuPercentageOfN_k (1.0) */
  double alpha_pct;          /* alphaPercentage (0.8) */
} TgmmServerDesc;

/* Fill *d with defaults: device 0, automatic budget, 2 lanes, 64 frames / 2^25 voxels /
 * 2^17 supervoxels / 2^17 Gaussians per batch, tgmm_default_params, the reference's
 * prior percentages (parseConfigFile.h:155-157). */
void tgmm_server_default_desc(TgmmServerDesc* d);

int tgmm_server_create(const TgmmServerDesc* d, TgmmServer** out);
/* Completes every submitted frame, then stops the worker and frees the server. */
int tgmm_server_destroy(TgmmServer* s);

/* A lineage: n_gauss Gaussians (copied from host memory) that stay on the device. */
int tgmm_server_open_lineage(TgmmServer* s, const TgmmGaussian* gm_host, int32_t n_gauss,
                             int32_t* lineage);
/* Frees a lineage that has no frame queued or in flight. */
int tgmm_server_close_lineage(TgmmServer* s, int32_t lineage);
/* Copies a lineage's current Gaussians (the prior of its next frame) to host memory; waits
 * for its frames in flight. */
int tgmm_server_read_lineage(TgmmServer* s, int32_t lineage, TgmmGaussian* gm_host);

/* One frame of a lineage, in host memory with the layout of TgmmFrame, or with its voxels
 * in the compact form below.  The arrays must stay valid and unchanged until the frame's
 * result has been polled; page-locked host memory makes the upload asynchronous.  A frame
 * is admitted -- its device buffers taken from the HBM budget and its upload started --
 * as soon as the budget allows, before its lineage is ready to run it.  Outputs (each
 * optional, NULL to skip): rnk_out, ind_out (5*n_sv, slot-major like tgmm_em_run) and
 * gm_out (n_gauss records: the frame's posterior, before the prior update), written before
 * the result is returned; outputs in page-locked memory are downloaded in place, others
 * through page-locked staging and a host copy.
 *
 * Compact voxels (used when query and img are NULL): lin[v] = x + X (y + Y z) and the raw
 * intensity raw[v]; the device expands them into query (float x, y, z) and
 * img = (float)(((double)raw - raw_offset) / raw_denom), the rescale of the reference's
 * input build (mainTrackingGaussianMixtureModel.cpp:664-669).  6 bytes a voxel cross the
 * host link instead of 16, and the expanded frame is bit-identical to the float one. */
typedef struct TgmmServeRequest {
  int32_t lineage;
  uint64_t tag;                 /* echoed in the result */
  const float* query;           /* host, 3*n_vox, SoA */
  const float* img;             /* host, n_vox */
  const float* centroids;       /* host, 3*n_sv, SoA */
  const int64_t* label_ptr;     /* host, n_sv + 1 */
  int64_t n_vox;
  int32_t n_sv;
  float* rnk_out;               /* host or NULL */
  int32_t* ind_out;             /* host or NULL */
  TgmmGaussian* gm_out;         /* host or NULL */
  const uint32_t* lin;          /* host, n_vox (compact form) */
  const uint16_t* raw;          /* host, n_vox (compact form) */
  int32_t dims[3];              /* X, Y, Z of the volume (compact form) */
  double raw_offset;            /* compact form: intensity offset (the foreground threshold) */
  double raw_denom;             /* compact form: intensity denominator (max - threshold) */
  /* Run form (query, img and lin NULL; raw, dims, raw_offset, raw_denom as the compact form):
   * the voxels of supervoxel s are the runs run_ptr[s] .. run_ptr[s+1], run r the run_len[r]
   * consecutive linear indices from run_start[r] (see tgmm_frame_expand_runs). */
  const int32_t* run_ptr;       /* host, n_sv + 1 */
  const uint32_t* run_start;    /* host, n_runs */
  const uint16_t* run_len;      /* host, n_runs */
  int64_t n_runs;
} TgmmServeRequest;

int tgmm_server_submit(TgmmServer* s, const TgmmServeRequest* r);

typedef struct TgmmServeResult {
  uint64_t tag;
  int32_t lineage;
  int32_t status;               /* TGMM_OK, or why the frame did not run / ran with flags */
  TgmmEmStats stats;
  double submit_ms;             /* server clock (ms since creation) */
  double start_ms;              /* batch launch */
  double done_ms;               /* result available */
  int32_t batch_id;
  int32_t batch_frames;
} TgmmServeResult;

/* Up to max results, oldest first; waits up to wait_ms milliseconds for the first one
 * (0: no wait, negative: until one arrives or nothing is pending). */
int tgmm_server_poll(TgmmServer* s, TgmmServeResult* out, int32_t max, int32_t wait_ms,
                     int32_t* n_out);

typedef struct TgmmServerStats {
  int64_t submitted, completed, rejected, batches;
  int64_t frames_in_batches;    /* sum of batch sizes */
  int64_t hbm_budget, hbm_in_use, hbm_peak;
  int64_t h2d_bytes;            /* bytes uploaded from host memory */
  int32_t queued, in_flight;
} TgmmServerStats;

int tgmm_server_stats(TgmmServer* s, TgmmServerStats* out);

/* Host-only self-test of the server's admission arena (first-fit allocation, coalescing,
 * budget): returns 0 when every check holds.  Runs without a GPU. */
int tgmm_server_selftest(void);

#ifdef __cplusplus
}
#endif
#endif /* TGMM_SERVE_H_ */
