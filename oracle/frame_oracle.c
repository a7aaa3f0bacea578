/*
 * frame_oracle.c -- TEST INFRASTRUCTURE ONLY (see tgmm_oracle.h).
 *
 * Plain-C restatement of the tracking program's frame preparation, the step between the
 * segmentation at tau and the EM's input arrays (nmeth.3036-S2/src/...):
 *   trimming       temporalLogicalRules/supervoxel.cpp:1556-1590 (intensityThreshold),
 *                  :1597-1664 (otsuThreshold), :1667-1747 (trimSupervoxel), with the
 *                  neighbourhoods of buildNeighboorhoodConnectivity (:474-609);
 *   size filter    mainTrackingGaussianMixtureModel.cpp:598-600, 626-634, and the
 *                  swap-to-the-back erase of hierarchicalSegmentation.cpp:1064-1092;
 *   centroids      supervoxel.cpp:1410-1450 (weightedGaussianStatistics, FP32, raw image);
 *   background     main:610-618 (raw -= thr per kept supervoxel, 16-bit), 643-648 (the
 *                  other voxels to 0), 664-669 (to float, Scale_Array_To_Range to [0,1]:
 *                  mylib/array.p:2769-2822);
 *   arrays         main:822-866 (coordinates SoA, intensities, CSR, centroids SoA).
 * Built with -ffp-contract=off: FP32 and FP64 expressions round as written.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "tgmm_oracle.h"

/* neighbour offsets in linear-index space (supervoxel.cpp:474-609); returns their count */
int or_conn_offsets(int32_t conn, const int32_t dims[3], int64_t* off) {
  const int64_t X = dims[0], XY = (int64_t)dims[0] * dims[1];
  int n = 0;
  switch (conn) {
    case 4:
      off[0] = -X, off[1] = -1, off[2] = 1, off[3] = X;
      return 4;
    case 6:
      off[0] = -XY, off[1] = -X, off[2] = -1, off[3] = 1, off[4] = X, off[5] = XY;
      return 6;
    case 8:
      for (int y = -1; y <= 1; y++)
        for (int x = -1; x <= 1; x++)
          if (x || y) off[n++] = x + X * y;
      return n;
    case 26:
      for (int z = -1; z <= 1; z++)
        for (int y = -1; y <= 1; y++)
          for (int x = -1; x <= 1; x++)
            if (x || y || z) off[n++] = x + X * y + XY * z;
      return n;
    case 74:
      for (int z = -1; z <= 1; z++)
        for (int y = -2; y <= 2; y++)
          for (int x = -2; x <= 2; x++)
            if (x || y || z) off[n++] = x + X * y + XY * z;
      return n;
    default:
      return 0;
  }
}

/* otsuThreshold (supervoxel.cpp:1597-1664): 256-bin histogram of the values mapped onto
 * [0,255], the bin with the largest between-class variance, back in value units. */
float or_otsu(const float* v, int32_t n) {
  float mn = FLT_MAX, mx = -FLT_MAX;
  for (int32_t i = 0; i < n; i++) {
    if (v[i] < mn) mn = v[i];
    if (v[i] > mx) mx = v[i];
  }
  const float mm = 255.0f / (mx - mn);
  if (!isfinite(mm)) return -FLT_MAX;
  int32_t hist[256] = {0};
  for (int32_t i = 0; i < n; i++) {
    int b = (int)((v[i] - mn) * mm);
    hist[b > 255 ? 255 : b]++;
  }
  float sum = 0.0f;
  for (int t = 0; t < 256; t++) sum += (float)(t * hist[t]);
  float sum_b = 0.0f, var_max = 0.0f;
  int32_t w_b = 0, best = 0;
  for (int t = 0; t < 256; t++) {
    w_b += hist[t];
    if (w_b == 0) continue;
    const int32_t w_f = n - w_b;
    if (w_f == 0) break;
    sum_b += (float)(t * hist[t]);
    const float m_b = sum_b / (float)w_b, m_f = (sum - sum_b) / (float)w_f;
    const float d = m_b - m_f;
    const float var = (float)w_b * (float)w_f * d * d;
    if (var > var_max) {
      var_max = var;
      best = t;
    }
  }
  return (float)best / mm + mn;
}

static int cmp_f(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* intensityThreshold for a supervoxel that has not been background-subtracted: the largest
 * of the (n - max_size)-th value, the (1 - max_pct) percentile and Otsu's threshold, cut to
 * 16 bits; *seed = first voxel (list order) holding the maximum. */
uint16_t or_trim_threshold(const uint16_t* val, int32_t n, int32_t max_size, float max_pct, int32_t* seed) {
  *seed = 0;
  if (n == 0) return 0;
  float* s = (float*)malloc(sizeof(float) * n);
  float best = (float)val[0];
  for (int32_t i = 0; i < n; i++) {
    s[i] = (float)val[i];
    if (s[i] > best) {
      best = s[i];
      *seed = i;
    }
  }
  qsort(s, n, sizeof(float), cmp_f);
  float thr = s[n - max_size > 0 ? n - max_size : 0];
  int32_t i2 = (int32_t)((1.0f - max_pct) * (float)n);
  if (i2 > n - 1) i2 = n - 1; /* the reference reads one past the end only for max_pct < 1/n */
  if (i2 < 0) i2 = 0;
  if (s[i2] > thr) thr = s[i2];
  const float t3 = or_otsu(s, n);
  if (t3 > thr) thr = t3;
  free(s);
  return (uint16_t)thr;
}

static int64_t find_sorted(const uint32_t* a, int64_t n, int64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if ((int64_t)a[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo < n && (int64_t)a[lo] == key ? lo : -1;
}

/* trimSupervoxel's flood: from the seed, the voxels of the list brighter than thr that
 * connect to it through the neighbourhood; keep[i] = 1 for those. Returns their count. */
int64_t or_trim_flood(const uint32_t* lin, const uint16_t* val, int64_t n, int32_t seed, uint16_t thr,
                      const int64_t* off, int32_t noff, int64_t nvol, uint8_t* keep) {
  memset(keep, 0, (size_t)n);
  if (n == 0 || val[seed] <= thr) return 0;
  int64_t* queue = (int64_t*)malloc(sizeof(int64_t) * n);
  int64_t head = 0, tail = 0, kept = 0;
  queue[tail++] = seed;
  keep[seed] = 1;
  while (head < tail) {
    const int64_t i = queue[head++];
    kept++;
    for (int32_t j = 0; j < noff; j++) {
      const int64_t nb = (int64_t)lin[i] + off[j];
      if (nb < 0 || nb >= nvol) continue;
      const int64_t k = find_sorted(lin, n, nb);
      if (k < 0 || keep[k] || val[k] <= thr) continue;
      keep[k] = 1;
      queue[tail++] = k;
    }
  }
  free(queue);
  return kept;
}

/* eraseSupervoxelFromCurrentSegmentation: each erased index, from the last, trades places
 * with the current last supervoxel; order[0..n-m) is what remains. */
void or_erase_order(const uint8_t* erased, int32_t n, int32_t* order) {
  for (int32_t i = 0; i < n; i++) order[i] = i;
  int32_t pos = n - 1;
  for (int32_t i = n - 1; i >= 0; i--) {
    if (!erased[i]) continue;
    const int32_t t = order[i];
    order[i] = order[pos];
    order[pos] = t;
    pos--;
  }
}

int or_frame_build(const uint16_t* raw, const uint32_t* label, const int32_t dims[3], int32_t n_labels,
                   const OrFrameParams* p, float* query, float* img, float* cent, int64_t* lptr, uint16_t* thr_out,
                   int64_t max_vox, int32_t max_sv, int64_t* n_vox, int32_t* n_sv) {
  const int64_t X = dims[0], Y = dims[1], nvol = (int64_t)dims[0] * dims[1] * dims[2];
  int64_t off[74];
  const int32_t noff = or_conn_offsets(p->conn, dims, off);
  if (noff == 0 || n_labels < 1) return 1;
  /* supervoxel lists, each in ascending linear index */
  int64_t* ptr = (int64_t*)calloc((size_t)n_labels + 1, sizeof(int64_t));
  for (int64_t v = 0; v < nvol; v++) {
    if (label[v] > (uint32_t)n_labels) {
      free(ptr);
      return 1;
    }
    if (label[v]) ptr[label[v]]++;
  }
  for (int32_t s = 0; s < n_labels; s++) ptr[s + 1] += ptr[s];
  const int64_t nfg = ptr[n_labels];
  uint32_t* lin = (uint32_t*)malloc(sizeof(uint32_t) * (nfg ? nfg : 1));
  uint16_t* val = (uint16_t*)malloc(sizeof(uint16_t) * (nfg ? nfg : 1));
  uint8_t* keep = (uint8_t*)malloc(nfg ? nfg : 1);
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * n_labels);
  for (int32_t s = 0; s < n_labels; s++) fill[s] = ptr[s];
  for (int64_t v = 0; v < nvol; v++)
    if (label[v]) {
      const int64_t at = fill[label[v] - 1]++;
      lin[at] = (uint32_t)v;
      val[at] = raw[v];
    }
  free(fill);
  /* trim, size filter */
  uint16_t* thr = (uint16_t*)malloc(sizeof(uint16_t) * n_labels);
  int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * n_labels);
  uint8_t* erased = (uint8_t*)malloc(n_labels);
  int32_t n_erased = 0;
  for (int32_t s = 0; s < n_labels; s++) {
    const int64_t a = ptr[s], n = ptr[s + 1] - a;
    int32_t seed;
    thr[s] = or_trim_threshold(val + a, (int32_t)n, p->max_size, p->max_pct, &seed);
    cnt[s] = or_trim_flood(lin + a, val + a, n, seed, thr[s], off, noff, nvol, keep + a);
    erased[s] = cnt[s] < p->min_size;
    n_erased += erased[s];
  }
  int rc = 0;
  if (n_erased >= n_labels) rc = 5;
  const int32_t S = n_labels - n_erased;
  int32_t* order = (int32_t*)malloc(sizeof(int32_t) * n_labels);
  or_erase_order(erased, n_labels, order);
  int64_t N = 0;
  for (int32_t q = 0; q < S; q++) N += cnt[order[q]];
  *n_vox = N;
  *n_sv = S;
  if (!rc && (N > max_vox || S > max_sv)) rc = 2;
  if (!rc) {
    /* the image after background subtraction: its range over the whole volume */
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int32_t q = 0; q < S; q++) {
      const int32_t s = order[q];
      for (int64_t i = ptr[s]; i < ptr[s + 1]; i++)
        if (keep[i]) {
          const float f = (float)(uint16_t)(val[i] - thr[s]);
          if (f < mn) mn = f;
          if (f > mx) mx = f;
        }
    }
    if (N < nvol) {
      if (0.0f < mn) mn = 0.0f;
      if (0.0f > mx) mx = 0.0f;
    }
    const int scaled = mx != mn;
    double fct = 1.0;
    fct /= (double)mx - (double)mn;
    const double shift = 0.0 / fct - (double)mn;
    int64_t at = 0;
    lptr[0] = 0;
    for (int32_t q = 0; q < S; q++) {
      const int32_t s = order[q];
      float w = 0.0f, c[3] = {0.0f, 0.0f, 0.0f};
      for (int64_t i = ptr[s]; i < ptr[s + 1]; i++) {
        if (!keep[i]) continue;
        const int64_t v = lin[i];
        const int64_t xyz[3] = {v % X, (v / X) % Y, v / (X * Y)};
        const float I = (float)val[i];
        w += I;
        for (int d = 0; d < 3; d++) c[d] += I * (float)xyz[d];
        const float sub = (float)(uint16_t)(val[i] - thr[s]);
        img[at] = scaled ? (float)(fct * ((double)sub + shift)) : sub;
        for (int d = 0; d < 3; d++) query[d * N + at] = (float)xyz[d];
        at++;
      }
      lptr[q + 1] = at;
      for (int d = 0; d < 3; d++) cent[d * S + q] = w < 1e-5 ? 0.0f : c[d] / w;
      if (thr_out) thr_out[q] = thr[s];
    }
  }
  free(order);
  free(erased);
  free(cnt);
  free(thr);
  free(keep);
  free(val);
  free(lin);
  free(ptr);
  return rc;
}
