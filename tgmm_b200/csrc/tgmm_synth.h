/*
 * tgmm_synth.h -- seeded synthetic nuclei volumes, supervoxels and first-frame
 * Gaussians (host library libtgmm_synth.so).  Used by the benchmark and the tests to
 * stand in for TGMM's image reading and segmentation.
 */
#ifndef TGMM_SYNTH_H_
#define TGMM_SYNTH_H_

#include <stdint.h>

#include "../../include/tgmm_gmem.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct TgmmSynthConfig {
  int32_t dims[3];        /* X, Y, Z in voxels */
  float axis_min, axis_max; /* semi-axis range (x, y); z is divided by anisotropy */
  float anisotropy;       /* z scale of the sampling grid (2.0) */
  float peak_min, peak_max; /* nucleus peak above background */
  float background;       /* 100 */
  float threshold;        /* foreground: value > threshold (150) */
  float jitter;           /* sigma of the initial-mean jitter, voxels (1.5) */
  int32_t min_size;       /* minimum supervoxel size (50) */
} TgmmSynthConfig;

typedef struct TgmmSynthFrame TgmmSynthFrame;

/* n random nuclei: centre[3n], axes[3n] (semi-axes, z already divided), rot[9n]
 * (row-major rotation), peak[n]. */
void tgmm_synth_nuclei(const TgmmSynthConfig* c, int32_t n, uint64_t seed, float* centre, float* axes, float* rot,
                       float* peak);
/* One frame from an explicit nucleus list (noise seeded by `seed`). */
TgmmSynthFrame* tgmm_synth_frame(const TgmmSynthConfig* c, int32_t n, const float* centre, const float* axes,
                                 const float* rot, const float* peak, uint64_t seed);
int64_t tgmm_synth_n_vox(const TgmmSynthFrame* f);
int32_t tgmm_synth_n_sv(const TgmmSynthFrame* f);
float tgmm_synth_max_fg(const TgmmSynthFrame* f);
/* Copy out: query[3N] SoA, img[N], cent[3S] SoA, lptr[S+1], sv_nucleus[S] (any may be NULL). */
void tgmm_synth_copy(const TgmmSynthFrame* f, float* query, float* img, float* cent, int64_t* lptr,
                     int32_t* sv_nucleus);
/* Raw uint16 foreground values in the order of query (img = (raw - threshold) / (max_fg -
 * threshold), evaluated in double and rounded to float). */
void tgmm_synth_copy_raw(const TgmmSynthFrame* f, uint16_t* raw);
void tgmm_synth_free(TgmmSynthFrame* f);
/* First-frame Gaussians; returns K (out may be NULL to count). */
int32_t tgmm_synth_init_gaussians(const TgmmSynthFrame* f, const TgmmSynthConfig* c, int32_t n_nuclei,
                                  const float* centre, uint64_t seed, const TgmmEmParams* prm, TgmmGaussian* out,
                                  int32_t* nucleus_of_gaussian);

#ifdef __cplusplus
}
#endif
#endif
