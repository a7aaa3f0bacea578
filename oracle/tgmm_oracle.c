/*
 * tgmm_oracle.c -- TEST INFRASTRUCTURE ONLY (see tgmm_oracle.h).
 *
 * Plain-C restatement of the reference path.  Each function names the reference
 * lines (nmeth.3036-S2/src/...) whose behaviour it restates.  Build with
 * -ffp-contract=off so that the only fused multiply-adds are the explicit fmaf()
 * calls (the FP32 kNN distance is specified as mul, fma, fma).
 */
#include "tgmm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

_Static_assert(sizeof(OrGaussian) == 288, "OrGaussian must match the 288-byte reference struct");

#define OR_LN2 0.69314718055994530942
#define OR_TWO_PI_POW_1_5 15.74960994572241901324 /* (2*pi)^(3/2) */
#define OR_PI 3.14159265358979323846
#define OR_BLK 1024 /* MAX_THREADS of the reference kernels (GMEMcommonCUDA.h) */

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void or_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

static int is_dead(const OrGaussian* g) { return g->m_o[0] < -1e31; }

/* ---------------------------------------------------------------------------
 * Digamma: Bernardo, Algorithm AS 103 (Applied Statistics 25(3), 1976) with the
 * small-argument shortcut and the x>=12 asymptotic series used by the reference
 * (GMEMupdateCUDA.cu:494-525); reflection for negative arguments.
 * ------------------------------------------------------------------------- */
static double psi_positive(double x) {
  const double euler = -0.57721566490153286;     /* psi(1) */
  const double zeta2 = 1.6449340668482264365;    /* pi^2/6 */
  if (x <= 1e-6) return euler - 1.0 / x + zeta2 * x;
  double acc = 0.0;
  while (x < 12.0) {
    acc -= 1.0 / x;
    x += 1.0;
  }
  double inv = 1.0 / x;
  acc += log(x) - 0.5 * inv;
  double t = inv * inv;
  /* Bernoulli terms B_2n/(2n): 1/12, 1/120, 1/252, 1/240, 1/132 */
  acc -= t * (1.0 / 12 - t * (1.0 / 120 - t * (1.0 / 252 - t * (1.0 / 240 - t * (1.0 / 132)))));
  return acc;
}

double or_digamma(double x) {
  if (x <= 0 && floor(x) == x) return -1e300;
  if (x < 0) return psi_positive(1.0 - x) + OR_PI / tan(-OR_PI * x);
  return psi_positive(x);
}

/* 3x3 symmetric determinant and adjugate inverse, singular below |det|<1e-16
 * (GMEMupdateCUDA.cu:163-192). */
double or_det3(const double* w) {
  return w[0] * (w[3] * w[5] - w[4] * w[4]) - w[1] * (w[1] * w[5] - w[2] * w[4]) +
         w[2] * (w[1] * w[4] - w[2] * w[3]);
}

void or_inv3(const double* w, double* o) {
  double det = or_det3(w);
  if (fabs(det) < 1e-16) {
    for (int i = 0; i < 6; i++) o[i] = 1e300;
    return;
  }
  o[0] = (w[3] * w[5] - w[4] * w[4]) / det;
  o[1] = (w[4] * w[2] - w[1] * w[5]) / det;
  o[2] = (w[1] * w[4] - w[3] * w[2]) / det;
  o[3] = (w[0] * w[5] - w[2] * w[2]) / det;
  o[4] = (w[1] * w[2] - w[0] * w[4]) / det;
  o[5] = (w[0] * w[3] - w[1] * w[1]) / det;
}

/* ---------------------------------------------------------------------------
 * Closed-form eigen-decomposition of a symmetric 3x3 matrix (trigonometric
 * method for the characteristic cubic; eigenvectors from cross products of the
 * rows of W - d I), with the reference's singular/degenerate branches and sign
 * conventions (GMEMupdateCUDA.cu:198-422).  Eigenvalue order: d0 = largest,
 * d1 = smallest, d2 = middle.  v holds three row vectors v[3i..3i+2].
 * ------------------------------------------------------------------------- */
static int normalise3(double* a) {
  double n = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  if (n > 1e-12) {
    a[0] /= n;
    a[1] /= n;
    a[2] /= n;
    return 1;
  }
  return 0;
}

void or_eig3(const double* w, double* d, double* v) {
  double det = or_det3(w);
  if (fabs(det) < 1e-24) {
    /* one zero eigenvalue: the other two solve a quadratic */
    double b = -w[0] - w[3] - w[5];
    double c = w[0] * w[3] + w[0] * w[5] + w[3] * w[5] - w[1] * w[1] - w[2] * w[2] - w[4] * w[4];
    double disc = b * b - 4.0 * c;
    disc = disc < 0 ? 0.0 : sqrt(disc);
    d[0] = 0.0;
    d[1] = 0.5 * (-b + disc);
    d[2] = 0.5 * (-b - disc);
  } else {
    double mean = (w[0] + w[3] + w[5]) / 3.0;
    double a0 = w[0] - mean, a3 = w[3] - mean, a5 = w[5] - mean;
    double halfdet = 0.5 * (a0 * (a3 * a5 - w[4] * w[4]) - w[1] * (w[1] * a5 - w[2] * w[4]) +
                            w[2] * (w[1] * w[4] - w[2] * a3));
    double p = (2.0 * (w[1] * w[1] + w[2] * w[2] + w[4] * w[4]) + a0 * a0 + a3 * a3 + a5 * a5) / 6.0;
    double ratio = halfdet / pow(p, 1.5);
    double phi;
    if (ratio <= -1)
      phi = 3.14159265358979311600 / 3.0;
    else if (ratio >= 1)
      phi = 0;
    else
      phi = acos(ratio) / 3.0;
    double c = cos(phi), s = sin(phi), r = sqrt(p);
    const double sqrt3 = 1.73205080756887719318;
    d[0] = mean + 2.0 * r * c;
    d[1] = mean - r * (c + sqrt3 * s);
    d[2] = mean - r * (c - sqrt3 * s);
  }

  int missing = 0;
  for (int i = 0; i < 3; i++) {
    double di = d[i];
    double* e = v + 3 * i;
    /* rows 0 and 1 of (W - di I) */
    e[0] = w[1] * w[4] - w[2] * (w[3] - di);
    e[1] = w[2] * w[1] - w[4] * (w[0] - di);
    e[2] = (w[0] - di) * (w[3] - di) - w[1] * w[1];
    if (!normalise3(e)) {
      /* rows 0 and 2 */
      e[0] = w[1] * (w[5] - di) - w[2] * w[4];
      e[1] = w[2] * w[2] - (w[5] - di) * (w[0] - di);
      e[2] = (w[0] - di) * w[4] - w[1] * w[2];
      if (!normalise3(e)) missing |= (1 << i);
    }
  }

  double n;
  switch (missing) {
    case 1:
      v[0] = v[4] * v[8] - v[5] * v[7];
      v[1] = v[5] * v[6] - v[3] * v[8];
      v[2] = v[4] * v[6] - v[3] * v[7];
      break;
    case 2:
      v[3] = v[1] * v[8] - v[2] * v[7];
      v[4] = v[2] * v[6] - v[0] * v[8];
      v[5] = v[1] * v[6] - v[0] * v[7];
      break;
    case 4:
      v[6] = v[4] * v[2] - v[5] * v[1];
      v[7] = v[5] * v[0] - v[3] * v[2];
      v[8] = v[4] * v[0] - v[3] * v[1];
      break;
    case 3:
      n = sqrt(v[7] * v[7] + v[6] * v[6]);
      if (n < 1e-12) {
        v[3] = 1.0;
        v[4] = 0.0;
        v[5] = 0.0;
      } else {
        v[3] = -v[7] / n;
        v[4] = v[6] / n;
        v[5] = 0.0;
      }
      v[0] = v[4] * v[8] - v[5] * v[7];
      v[1] = v[5] * v[6] - v[3] * v[8];
      v[2] = v[3] * v[7] - v[4] * v[6];
      break;
    case 6:
      n = sqrt(v[1] * v[1] + v[0] * v[0]);
      if (n < 1e-12) {
        v[6] = 1.0;
        v[7] = 0.0;
        v[8] = 0.0;
      } else {
        v[6] = -v[1] / n;
        v[7] = v[0] / n;
        v[8] = 0.0;
      }
      v[3] = v[1] * v[8] - v[2] * v[7];
      v[4] = v[2] * v[6] - v[0] * v[8];
      v[5] = v[0] * v[7] - v[1] * v[6];
      break;
    case 5:
      n = sqrt(v[4] * v[4] + v[5] * v[5]);
      if (n < 1e-12) {
        v[0] = 1.0;
        v[1] = 0.0;
        v[2] = 0.0;
      } else {
        v[0] = -v[4] / n;
        v[1] = v[5] / n;
        v[2] = 0.0;
      }
      v[6] = v[4] * v[2] - v[5] * v[1];
      v[7] = v[5] * v[0] - v[3] * v[2];
      v[8] = v[1] * v[3] - v[4] * v[0];
      break;
    case 7:
      v[1] = v[2] = v[3] = v[5] = v[6] = v[7] = 0.0;
      v[0] = v[4] = v[8] = 1.0;
      break;
    default:
      break;
  }
  double s = v[0] * (v[4] * v[8] - v[5] * v[7]) - v[1] * (v[3] * v[8] - v[5] * v[6]) +
             v[2] * (v[3] * v[7] - v[4] * v[6]);
  if (s < 0) {
    v[0] = -v[0];
    v[1] = -v[1];
    v[2] = -v[2];
  }
}

/* ---------------------------------------------------------------------------
 * kNN of supervoxel centroids against Gaussian means (knnCuda.cu:61-246).
 * Distance in FP32: a=(q0-r0)*s0; d=a*a; b=(q1-r1)*s1; d=fma(b,b,d); c=...; d=fma(c,c,d).
 * ------------------------------------------------------------------------- */
static inline float knn_dist(const float* q, const float* r, const float* s) {
  float a = (q[0] - r[0]) * s[0];
  float d = a * a;
  float b = (q[1] - r[1]) * s[1];
  d = fmaf(b, b, d);
  float c = (q[2] - r[2]) * s[2];
  d = fmaf(c, c, d);
  return d;
}

void or_knn_canonical(const float* query, int64_t nq, const float* ref, int32_t nref,
                      const float scale[3], int32_t* ind) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nq; i++) {
    float q[3] = {query[i], query[nq + i], query[2 * nq + i]};
    float bd[OR_J];
    int32_t bi[OR_J];
    int cnt = 0;
    for (int32_t r = 0; r < nref; r++) {
      float d = knn_dist(q, ref + 3 * (int64_t)r, scale);
      if (isnan(d)) d = INFINITY;
      if (cnt == OR_J && !(d < bd[OR_J - 1])) continue; /* ties keep the lower index */
      int pos = (cnt < OR_J) ? cnt++ : OR_J - 1;
      while (pos > 0 && d < bd[pos - 1]) {
        bd[pos] = bd[pos - 1];
        bi[pos] = bi[pos - 1];
        pos--;
      }
      bd[pos] = d;
      bi[pos] = r;
    }
    for (int j = 0; j < OR_J; j++) ind[(int64_t)j * nq + i] = (j < cnt) ? bi[j] : -1;
  }
}

/* The tracking graph's supervoxel kNN (knnCUDA_, temporalLogicalRules/knnCUDA/knnCuda.cu:
 * 56-140) restated canonically: the k nearest (k <= OR_MAXK) of each query (SoA) among the
 * reference points (SoA), the same scaled squared FP32 distance, (distance, index) order;
 * slots with no point closer than 1e32 get index -1 and distance 1e32. */
void or_knn_topk(const float* query, int64_t nq, const float* ref, int32_t nref, int32_t k,
                 const float scale[3], int32_t* ind, float* dist) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nq; i++) {
    float q[3] = {query[i], query[nq + i], query[2 * nq + i]};
    float bd[OR_MAXK];
    int32_t bi[OR_MAXK];
    int cnt = 0;
    for (int32_t r = 0; r < nref; r++) {
      float rp[3] = {ref[r], ref[(int64_t)nref + r], ref[2 * (int64_t)nref + r]};
      float d = knn_dist(q, rp, scale);
      if (isnan(d)) d = INFINITY;
      if (!(d < 1e32f)) continue; /* never assigned, as in the reference */
      if (cnt == k && !(d < bd[k - 1])) continue; /* ties keep the lower index */
      int pos = (cnt < k) ? cnt++ : k - 1;
      while (pos > 0 && d < bd[pos - 1]) {
        bd[pos] = bd[pos - 1];
        bi[pos] = bi[pos - 1];
        pos--;
      }
      bd[pos] = d;
      bi[pos] = r;
    }
    for (int j = 0; j < k; j++) {
      ind[(int64_t)j * nq + i] = (j < cnt) ? bi[j] : -1;
      if (dist) dist[(int64_t)j * nq + i] = (j < cnt) ? bd[j] : 1e32f;
    }
  }
}

void or_knn_reference(const float* query, int64_t nq, const float* ref, int32_t nref,
                      const float scale[3], int32_t* ind) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nq; i++) {
    float q[3] = {query[i], query[nq + i], query[2 * nq + i]};
    float dist[OR_J];
    int32_t idx[OR_J];
    for (int j = 0; j < OR_J; j++) {
      dist[j] = 1e32f;
      idx[j] = -1; /* the reference leaves these uninitialised */
    }
    float thr = 1e32f;
    int slot = 0;
    for (int32_t r = 0; r < nref; r++) {
      const float* rr = ref + 3 * (int64_t)r;
      float a = (q[0] - rr[0]) * scale[0];
      float d = a * a;
      if (d > thr) continue;
      float b = (q[1] - rr[1]) * scale[1];
      d = fmaf(b, b, d);
      if (d > thr) continue;
      float c = (q[2] - rr[2]) * scale[2];
      d = fmaf(c, c, d);
      if (d > thr) continue;
      dist[slot] = d;
      idx[slot] = r;
      thr = dist[0];
      slot = 0;
      for (int j = 1; j < OR_J; j++)
        if (thr < dist[j]) {
          thr = dist[j];
          slot = j;
        }
    }
    for (int j = 0; j < OR_J; j++) ind[(int64_t)j * nq + i] = idx[j];
  }
}

/* Sum of alpha_k (GMEMupdateCUDA.cu:579-604 + 2765-2799): FP64 sequential, or the
 * reference's per-block shared-memory tree followed by a host sum. */
double or_total_alpha(const OrGaussian* g, int32_t K, int32_t mode) {
  if (mode == OR_MODE_FP64) {
    double s = 0;
    for (int32_t k = 0; k < K; k++) s += g[k].alpha_k;
    return s;
  }
  int threads = K < OR_BLK ? K : OR_BLK;
  int grids = (K + threads - 1) / threads;
  if (grids == 1) {
    int p = 1;
    while (p < threads) p <<= 1;
    threads = p;
  }
  double total = 0;
  double* cache = (double*)malloc(sizeof(double) * threads);
  for (int b = 0; b < grids; b++) {
    for (int t = 0; t < threads; t++) {
      int64_t k = (int64_t)b * threads + t;
      cache[t] = k < K ? g[k].alpha_k : 0.0;
    }
    for (int h = threads / 2; h > 0; h /= 2)
      for (int t = 0; t < h; t++) cache[t] += cache[t + h];
    total = (b == 0) ? cache[0] : total + cache[0];
  }
  free(cache);
  return total;
}

/* E[ln|Lambda|] and E[ln pi] (GMEMupdateCUDA.cu:553-576, 607-628; driver :4167-4170).
 * Note the psi index runs i = 0..2: psi((nu+1-i)/2). */
void or_prior_constants(OrGaussian* g, int32_t K, double total_alpha) {
  double psi_total = or_digamma(total_alpha);
#pragma omp parallel for schedule(static)
  for (int32_t k = 0; k < K; k++) {
    OrGaussian* G = &g[k];
    if (is_dead(G)) {
      G->eLD = -1e32;
      G->eLR = -1e32;
      continue;
    }
    double out = 3 * OR_LN2 + log(or_det3(G->W_k));
    for (int i = 0; i < 3; i++) out += or_digamma(0.5 * (G->nu_k + 1.0 - i));
    G->eLD = out;
    G->eLR = or_digamma(G->alpha_k) - psi_total;
  }
}

/* Per-voxel E-step term (GMEMupdateCUDA.cu:96-110 and 2291-2299):
 * -0.5*(3/beta + nu*d'Wd) + E[ln pi] + 0.5*E[ln|Lambda|], d = x - m in FP64. */
static inline double estep_term(const OrGaussian* G, double x0, double x1, double x2) {
  double d0 = x0 - G->m_k[0], d1 = x1 - G->m_k[1], d2 = x2 - G->m_k[2];
  const double* W = G->W_k;
  double maha = 3.0 / G->beta_k +
                G->nu_k * (W[0] * d0 * d0 + W[3] * d1 * d1 + W[5] * d2 * d2 + 2.0 * W[1] * d0 * d1 +
                           2.0 * W[2] * d0 * d2 + 2.0 * W[4] * d1 * d2);
  double aux = -0.5 * maha;
  aux += G->eLR;
  aux += 0.5 * G->eLD;
  return aux;
}

/* rnk_j = 1 / sum_i exp(L_i - L_j)  (GMEMupdateCUDA.cu:2327-2335). */
static void normalise_rnk(const double* L, float* out) {
  for (int j = 0; j < OR_J; j++) {
    double acc = 0.0;
    for (int i = 0; i < OR_J; i++) acc += exp(L[i] - L[j]);
    out[j] = (float)(1.0 / acc);
  }
}

/* E-step over supervoxels (GMEMcomputeRnkKernelWithSupervoxels, GMEMupdateCUDA.cu:2244-2336).
 * FP64 mode: exact sum in FP64, then the reference's float storage semantics for L:
 * an empty supervoxel gives L=0; a dead candidate (or any L beyond float range)
 * gives -inf, exactly what the reference's float accumulator holds. */
void or_estep(const OrGaussian* g, const float* query, int64_t N, const int64_t* lptr,
              int32_t S, const int32_t* ind, int32_t mode, float* rnk, double* L_out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int32_t s = 0; s < S; s++) {
    int64_t p0 = lptr[s], p1 = lptr[s + 1];
    double L[OR_J];
    for (int j = 0; j < OR_J; j++) {
      const OrGaussian* G = &g[ind[(int64_t)j * S + s]];
      if (mode == OR_MODE_FP64) {
        double acc = 0.0;
        for (int64_t v = p0; v < p1; v++)
          acc += estep_term(G, query[v], query[N + v], query[2 * N + v]);
        if (p1 > p0 && (is_dead(G) || acc < -FLT_MAX)) acc = -INFINITY;
        if (acc > FLT_MAX) acc = INFINITY;
        L[j] = acc;
      } else {
        float cache[OR_BLK];
        for (int t = 0; t < OR_BLK; t++) {
          float a = 0.0f;
          for (int64_t v = p0 + t; v < p1; v += OR_BLK)
            a = (float)((double)a + estep_term(G, query[v], query[N + v], query[2 * N + v]));
          cache[t] = a;
        }
        for (int h = OR_BLK / 2; h > 0; h /= 2)
          for (int t = 0; t < h; t++) cache[t] += cache[t + h];
        L[j] = (double)cache[0];
      }
    }
    float tmp[OR_J];
    normalise_rnk(L, tmp);
    for (int j = 0; j < OR_J; j++) {
      rnk[(int64_t)j * S + s] = tmp[j];
      if (L_out) L_out[(int64_t)j * S + s] = L[j];
    }
  }
}

/* Gaussian-major order of the (supervoxel, slot) pairs: a stable sort of the flat
 * position p = j*S + s by Gaussian id, as thrust::sort_by_key gives the reference
 * (GMEMupdateCUDA.cu:4181-4198). Returns CSR offsets (K+1) and the sorted positions. */
static void gaussian_major(const int32_t* ind, int32_t S, int32_t K, int64_t* off, int64_t* pos) {
  int64_t P = (int64_t)OR_J * S;
  memset(off, 0, sizeof(int64_t) * (K + 1));
  for (int64_t p = 0; p < P; p++) off[ind[p] + 1]++;
  for (int32_t k = 0; k < K; k++) off[k + 1] += off[k];
  int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (K + 1));
  memcpy(cur, off, sizeof(int64_t) * (K + 1));
  for (int64_t p = 0; p < P; p++) pos[cur[ind[p]]++] = p;
  free(cur);
}

/* M-step sufficient statistics (GMEMcomputeXkNkSkKernelTrWithSupervoxels,
 * GMEMupdateCUDA.cu:1286-1455).  Pairs with rnk <= 1e-3 are skipped; w = rnk*I.
 * Outputs: Nk[k], Xk[3k+d] = weighted mean, Sk[6k+e] = unnormalised scatter
 * sum w (x-mean)(x-mean)' (00,01,02,11,12,22).  Nk==0 leaves Xk=Sk=0. */
void or_mstep(const float* query, const float* img, int64_t N, const int64_t* lptr,
              int32_t S, int32_t K, const int32_t* ind, const float* rnk, int32_t mode,
              double* Nk, double* Xk, double* Sk) {
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (K + 1));
  int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * (int64_t)OR_J * (S > 0 ? S : 1));
  gaussian_major(ind, S, K, off, pos);
#pragma omp parallel for schedule(dynamic, 8)
  for (int32_t k = 0; k < K; k++) {
    Nk[k] = 0;
    for (int d = 0; d < 3; d++) Xk[3 * k + d] = 0;
    for (int e = 0; e < 6; e++) Sk[6 * k + e] = 0;
    if (mode == OR_MODE_FP64) {
      double n = 0, sx[3] = {0, 0, 0};
      for (int64_t e = off[k]; e < off[k + 1]; e++) {
        int64_t p = pos[e];
        float r = rnk[p];
        if (!((double)r > 1e-3)) continue;
        int32_t s = (int32_t)(p % S);
        for (int64_t v = lptr[s]; v < lptr[s + 1]; v++) {
          double w = (double)r * (double)img[v];
          n += w;
          sx[0] += w * query[v];
          sx[1] += w * query[N + v];
          sx[2] += w * query[2 * N + v];
        }
      }
      if (!(n > 0)) {
        Nk[k] = n > 0 ? n : 0.0;
        continue;
      }
      double mu[3] = {sx[0] / n, sx[1] / n, sx[2] / n};
      double sc[6] = {0, 0, 0, 0, 0, 0};
      for (int64_t e = off[k]; e < off[k + 1]; e++) {
        int64_t p = pos[e];
        float r = rnk[p];
        if (!((double)r > 1e-3)) continue;
        int32_t s = (int32_t)(p % S);
        for (int64_t v = lptr[s]; v < lptr[s + 1]; v++) {
          double w = (double)r * (double)img[v];
          double a = query[v] - mu[0], b = query[N + v] - mu[1], c = query[2 * N + v] - mu[2];
          sc[0] += w * a * a;
          sc[1] += w * a * b;
          sc[2] += w * a * c;
          sc[3] += w * b * b;
          sc[4] += w * b * c;
          sc[5] += w * c * c;
        }
      }
      Nk[k] = n;
      for (int d = 0; d < 3; d++) Xk[3 * k + d] = mu[d];
      for (int e = 0; e < 6; e++) Sk[6 * k + e] = sc[e];
    } else {
      /* 1024 emulated threads, float shared-memory accumulators, tree reduction */
      float* acc = (float*)calloc((size_t)10 * OR_BLK, sizeof(float));
      float *aN = acc, *aX0 = acc + OR_BLK, *aX1 = acc + 2 * OR_BLK, *aX2 = acc + 3 * OR_BLK;
      float *aS0 = acc + 4 * OR_BLK, *aS1 = acc + 5 * OR_BLK, *aS2 = acc + 6 * OR_BLK;
      float *aS3 = acc + 7 * OR_BLK, *aS4 = acc + 8 * OR_BLK, *aS5 = acc + 9 * OR_BLK;
      int any = off[k + 1] > off[k];
      for (int t = 0; t < OR_BLK && any; t++) {
        for (int64_t e = off[k]; e < off[k + 1]; e++) {
          int64_t p = pos[e];
          float r = rnk[p];
          if (!((double)r > 1e-3)) continue;
          int32_t s = (int32_t)(p % S);
          for (int64_t v = lptr[s] + t; v < lptr[s + 1]; v += OR_BLK) {
            float w = r * img[v];
            float x0 = query[v], x1 = query[N + v], x2 = query[2 * N + v];
            aN[t] += w;
            float w0 = w * x0;
            aX0[t] += w0;
            aS0[t] = fmaf(w0, x0, aS0[t]);
            aS1[t] = fmaf(w0, x1, aS1[t]);
            aS2[t] = fmaf(w0, x2, aS2[t]);
            float w1 = w * x1;
            aX1[t] += w1;
            aS3[t] = fmaf(w1, x1, aS3[t]);
            aS4[t] = fmaf(w1, x2, aS4[t]);
            float w2 = w * x2;
            aX2[t] += w2;
            aS5[t] = fmaf(w2, x2, aS5[t]);
          }
        }
      }
      if (any) {
        for (int h = OR_BLK / 2; h > 0; h /= 2)
          for (int t = 0; t < h; t++)
            for (int a = 0; a < 10; a++) acc[a * OR_BLK + t] += acc[a * OR_BLK + t + h];
        float n = aN[0];
        Nk[k] = n;
        if (n > 0.0f) {
          float m0 = aX0[0] / n, m1 = aX1[0] / n, m2 = aX2[0] / n;
          Xk[3 * k + 0] = m0;
          Xk[3 * k + 1] = m1;
          Xk[3 * k + 2] = m2;
          Sk[6 * k + 0] = fmaf(-m0, aX0[0], aS0[0]);
          Sk[6 * k + 1] = fmaf(-m1, aX0[0], aS1[0]);
          Sk[6 * k + 2] = fmaf(-m2, aX0[0], aS2[0]);
          Sk[6 * k + 3] = aS3[0] - aX1[0] * aX1[0] / n;
          Sk[6 * k + 4] = aS4[0] - aX1[0] * aX2[0] / n;
          Sk[6 * k + 5] = aS5[0] - aX2[0] * aX2[0] / n;
        }
      }
      free(acc);
    }
  }
  free(off);
  free(pos);
}

/* Dirichlet / Normal-Wishart update (GMEMupdateGaussianParametersKernel,
 * GMEMupdateCUDA.cu:1601-1677; CPU twin GaussianMixtureModel.h:252-272).
 * Skipped for dead or fixed Gaussians.  The W_o[5]<1e-8 fix is written into the prior. */
void or_update(OrGaussian* g, int32_t K, const double* Nk, const double* Xk, const double* Sk,
               int32_t mode) {
#pragma omp parallel for schedule(static)
  for (int32_t k = 0; k < K; k++) {
    OrGaussian* G = &g[k];
    if (!(G->m_o[0] > -1e31 && !G->fixed)) continue;
    double winv[6];
    if (mode == OR_MODE_FP64) {
      double n = Nk[k], bo = G->beta_o;
      const double* x = Xk + 3 * k;
      G->beta_k = bo + n;
      G->nu_k = G->nu_o + n;
      G->alpha_k = fmax(G->alpha_o + n, 0.0);
      for (int d = 0; d < 3; d++) G->m_k[d] = (bo * G->m_o[d] + n * x[d]) / G->beta_k;
      if (G->W_o[5] < 1e-8) G->W_o[5] = 0.5 * (G->W_o[0] + G->W_o[3]);
      or_inv3(G->W_o, winv);
      double dx[3] = {x[0] - G->m_o[0], x[1] - G->m_o[1], x[2] - G->m_o[2]};
      double f = n * bo / (bo + n);
      const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
      for (int e = 0; e < 6; e++) winv[e] += Sk[6 * k + e] + f * dx[ia[e]] * dx[ib[e]];
      or_inv3(winv, G->W_k);
    } else {
      float n = (float)Nk[k];
      float bo = (float)G->beta_o;
      float x[3] = {(float)Xk[3 * k], (float)Xk[3 * k + 1], (float)Xk[3 * k + 2]};
      float mo[3] = {(float)G->m_o[0], (float)G->m_o[1], (float)G->m_o[2]};
      G->beta_k = bo + n;
      float bk = (float)G->beta_k;
      G->nu_k = G->nu_o + n;
      G->alpha_k = fmax(G->alpha_o + n, 0.0);
      for (int d = 0; d < 3; d++) G->m_k[d] = fmaf(n, x[d], bo * mo[d]) / bk;
      if (G->W_o[5] < 1e-8) G->W_o[5] = 0.5 * (G->W_o[0] + G->W_o[3]);
      or_inv3(G->W_o, winv);
      for (int d = 0; d < 3; d++) x[d] -= mo[d];
      bo /= (bo + n);
      float f = n * bo;
      winv[0] += fmaf(f * x[0], x[0], (float)Sk[6 * k + 0]);
      winv[1] += fmaf(f * x[0], x[1], (float)Sk[6 * k + 1]);
      winv[2] += fmaf(f * x[0], x[2], (float)Sk[6 * k + 2]);
      winv[3] += fmaf(f * x[1], x[1], (float)Sk[6 * k + 3]);
      winv[4] += fmaf(f * x[1], x[2], (float)Sk[6 * k + 4]);
      winv[5] += fmaf(f * x[2], x[2], (float)Sk[6 * k + 5]);
      or_inv3(winv, G->W_k);
    }
  }
}

/* Precision-matrix regularisation (GMEMregularizeWkKernel, GMEMupdateCUDA.cu:1693-1809):
 * divide by s_i*s_j (float products), optional 4-DOF zeroing, eigenvalue clamp to
 * [lambda_min/nu, lambda_max/nu], pairwise eccentricity cap in the order (0,1),(0,2),(1,2),
 * rebuild, multiply back. */
void or_regularize(OrGaussian* g, int32_t K, const float scale[3], int32_t w4dof, double lmin,
                   double lmax, double maxexc) {
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma omp parallel for schedule(static)
  for (int32_t k = 0; k < K; k++) {
    OrGaussian* G = &g[k];
    if (G->m_o[0] < -1e31 || G->fixed) continue;
    double hi = lmax / G->nu_k, lo = lmin / G->nu_k;
    double W[6];
    for (int e = 0; e < 6; e++) W[e] = G->W_k[e] / (double)(scale[ia[e]] * scale[ib[e]]);
    if (w4dof) {
      W[2] = 0.0;
      W[4] = 0.0;
    }
    double d[3], v[9];
    or_eig3(W, d, v);
    for (int i = 0; i < 3; i++)
      if (d[i] > hi) d[i] = hi;
    for (int i = 0; i < 3; i++)
      if (d[i] < lo) d[i] = lo;
    const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
    for (int q = 0; q < 3; q++) {
      double r = d[pa[q]] / d[pb[q]];
      if (r > maxexc)
        d[pa[q]] = maxexc * d[pb[q]];
      else if (1. / r > maxexc)
        d[pb[q]] = maxexc * d[pa[q]];
    }
    W[0] = d[0] * v[0] * v[0] + d[1] * v[3] * v[3] + d[2] * v[6] * v[6];
    W[3] = d[0] * v[1] * v[1] + d[1] * v[4] * v[4] + d[2] * v[7] * v[7];
    W[5] = d[0] * v[2] * v[2] + d[1] * v[5] * v[5] + d[2] * v[8] * v[8];
    W[1] = d[0] * v[0] * v[1] + d[1] * v[3] * v[4] + d[2] * v[6] * v[7];
    if (!w4dof) {
      W[2] = d[0] * v[0] * v[2] + d[1] * v[3] * v[5] + d[2] * v[6] * v[8];
      W[4] = d[0] * v[1] * v[2] + d[1] * v[4] * v[5] + d[2] * v[7] * v[8];
    }
    for (int e = 0; e < 6; e++) G->W_k[e] = W[e] * (double)(scale[ia[e]] * scale[ib[e]]);
  }
}

/* Dead-Gaussian rule (GMEMcheckDeadCellsKernel, GMEMupdateCUDA.cu:1813-1843).  The
 * reference's NaN scan reads 7 doubles from W_k, the 7th being E[ln|Lambda|]. */
void or_kill(OrGaussian* g, int32_t K, double* Nk, double total_alpha) {
#pragma omp parallel for schedule(static)
  for (int32_t k = 0; k < K; k++) {
    OrGaussian* G = &g[k];
    int nanw = 0;
    for (int e = 0; e < 6; e++) nanw |= isnan(G->W_k[e]);
    nanw |= isnan(G->eLD);
    if (nanw || (G->alpha_k / total_alpha < 1e-5 && G->m_o[0] > -1e31 && !G->fixed)) {
      if (Nk) Nk[k] = 0.0;
      G->alpha_k = 0.0;
      for (int d = 0; d < 3; d++) {
        G->m_o[d] = -1e32;
        G->m_k[d] = -1e32;
      }
      G->W_k[0] = 1;
      G->W_k[1] = 0;
      G->W_k[2] = 0;
      G->W_k[3] = 1;
      G->W_k[4] = 0;
      G->W_k[5] = 1;
    }
  }
}

/* Mixture density of one voxel over its supervoxel's five candidates
 * (GMEMupdateCUDA.cu:1955-1960): sum_j (alpha_j/A) sqrt(det W_j nu_j^3)/(2 pi)^1.5
 * exp(-0.5 nu_j d'W_j d). */
static inline double voxel_density(const OrGaussian* const* c, double x0, double x1, double x2,
                                   double total_alpha) {
  double acc = 0.0;
  for (int j = 0; j < OR_J; j++) {
    const OrGaussian* G = c[j];
    const double* W = G->W_k;
    double d0 = x0 - G->m_k[0], d1 = x1 - G->m_k[1], d2 = x2 - G->m_k[2];
    double maha = G->nu_k * (W[0] * d0 * d0 + W[3] * d1 * d1 + W[5] * d2 * d2 +
                             2.0 * W[1] * d0 * d1 + 2.0 * W[2] * d0 * d2 + 2.0 * W[4] * d1 * d2);
    double a = sqrt(or_det3(W) * pow(G->nu_k, 3)) / OR_TWO_PI_POW_1_5;
    a *= exp(-0.5 * maha);
    a *= (G->alpha_k / total_alpha);
    acc += a;
  }
  return acc;
}

/* Split proposal of one Gaussian record (GaussianMixtureModel::splitGaussian(GM, id),
 * GaussianMixtureModel.cpp:514-557, then updatePriorsAfterSplitProposal :912-922 on both halves),
 * with N_k = nu_k - nu_o as copyFromGMEM_CUDA derives it (variationalInference.cpp:1008):
 * S = nu W / (s_i s_j) (float products of the scale); lmin, v = its smallest eigenvalue and
 * eigenvector, lmax its largest; sigma = 1/sqrt(max(lmin, 1e-3)); both halves get
 * W = (lmax / nu) I with W_ii *= s_i s_i and N_k / 2; a = m + sigma v, b = a - 2 sigma v; then
 * m_o = m_k, beta_o = max(N_k/2, 1e-5), nu_o = max(N_k/2, 3), W_o = W_k nu_k / nu_o.  The sign of
 * v is fixed by making its largest-magnitude component positive (the reference takes Eigen's
 * solver's sign, so a and b may trade places against it). */
void or_split_proposal(const OrGaussian* g, const float scale[3], OrGaussian* a, OrGaussian* b) {
  static const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  double w[6], d[3], v[9];
  for (int e = 0; e < 6; e++)
    w[e] = (g->W_k[e] * g->nu_k) / (double)(scale[ij[e][0]] * scale[ij[e][1]]);
  or_eig3(w, d, v);
  int imin = 0, imax = 0;
  for (int i = 1; i < 3; i++) {
    if (d[i] < d[imin]) imin = i;
    if (d[i] > d[imax]) imax = i;
  }
  double u[3] = {v[3 * imin], v[3 * imin + 1], v[3 * imin + 2]};
  int big = 0;
  for (int i = 1; i < 3; i++)
    if (fabs(u[i]) > fabs(u[big])) big = i;
  if (u[big] < 0)
    for (int i = 0; i < 3; i++) u[i] = -u[i];
  double smax = d[imin];
  if (smax < 1e-3) smax = 1e-3;
  const double sm2 = 1.0 / sqrt(smax);
  const double smin = d[imax];
  const double nk = 0.5 * (g->nu_k - g->nu_o);
  *a = *g;
  for (int e = 0; e < 6; e++) a->W_k[e] = 0.0;
  a->W_k[0] = smin / g->nu_k * (double)(scale[0] * scale[0]);
  a->W_k[3] = smin / g->nu_k * (double)(scale[1] * scale[1]);
  a->W_k[5] = smin / g->nu_k * (double)(scale[2] * scale[2]);
  for (int i = 0; i < 3; i++) a->m_k[i] = g->m_k[i] + sm2 * u[i];
  *b = *a;
  for (int i = 0; i < 3; i++) b->m_k[i] = a->m_k[i] - 2.0 * sm2 * u[i];
  OrGaussian* h[2] = {a, b};
  for (int q = 0; q < 2; q++) {
    OrGaussian* x = h[q];
    for (int i = 0; i < 3; i++) x->m_o[i] = x->m_k[i];
    x->beta_o = 0.5 * nk > 1e-5 ? 0.5 * nk : 1e-5;
    x->nu_o = 0.5 * nk > 3.0 ? 0.5 * nk : 3.0;
    for (int e = 0; e < 6; e++) x->W_o[e] = x->W_k[e] * x->nu_k / x->nu_o;
  }
}

/* Local log-likelihood of supervoxel lists (calculateLocalLikelihood, GMEMupdateCUDA.cu:2952-3055,
 * over addLocalLikelihoodWithSupervoxels :2876-2949 and GMEMcomputeLocalLikelihoodKernelWithSupervoxels
 * :1989-2103).  total alpha = sum of alpha_k over all K records (calculateTotalAlpha).  For list i and
 * each supervoxel s in it (duplicates count again), its five candidates ind[j*S+s]: thread t of 1024
 * keeps I*ln(density) of the last voxel of its stride with a positive density (the cache overwrite,
 * :2083-2084); the supervoxel's value is the sum of the 1024 slots.  FP64 mode sums in FP64 in list
 * order; REF32 mode reproduces the float cache, the per-block tree, the power-of-two sumVector pass
 * over the list's values and the host double sum (:2899-2944).  An empty list gives 0 (the reference
 * skips it and leaves the zero of its resize, :3037).  Returns -1 on an index out of range. */
int or_local_likelihood(const OrGaussian* g, int32_t K, const float* query, const float* img, int64_t N,
                        const int64_t* lptr, int32_t S, const int32_t* ind, const int32_t* list_ptr,
                        const int32_t* list_idx, int32_t n_lists, int32_t mode, double* out) {
  const double total_alpha = or_total_alpha(g, K, mode);
  int bad = 0;
  for (int32_t i = 0; i < n_lists; i++)
    for (int32_t p = list_ptr[i]; p < list_ptr[i + 1]; p++) {
      if (list_idx[p] < 0 || list_idx[p] >= S) bad = 1;
      else
        for (int j = 0; j < OR_J; j++) {
          const int32_t k = ind[(int64_t)j * S + list_idx[p]];
          if (k < 0 || k >= K) bad = 1;
        }
    }
  if (bad) return -1;
#pragma omp parallel for schedule(dynamic, 1)
  for (int32_t i = 0; i < n_lists; i++) {
    const int32_t n = list_ptr[i + 1] - list_ptr[i];
    if (n == 0) {
      out[i] = 0.0;
      continue;
    }
    double sum64 = 0.0;
    int size = 1;
    while (size < n) size <<= 1;
    float* vec32 = (float*)calloc(size, sizeof(float));
    for (int32_t q = 0; q < n; q++) {
      const int32_t s = list_idx[list_ptr[i] + q];
      const OrGaussian* c[OR_J];
      for (int j = 0; j < OR_J; j++) c[j] = &g[ind[(int64_t)j * S + s]];
      double cache64[OR_BLK];
      float cache[OR_BLK];
      for (int t = 0; t < OR_BLK; t++) {
        cache64[t] = 0.0;
        cache[t] = 0.0f;
      }
      for (int64_t v = lptr[s]; v < lptr[s + 1]; v++) {
        const double dens = voxel_density(c, query[v], query[N + v], query[2 * N + v], total_alpha);
        if (dens > 0.0) {
          const double term = (double)img[v] * log(dens);
          const int t = (int)((v - lptr[s]) % OR_BLK);
          cache64[t] = term;
          cache[t] = (float)term;
        }
      }
      double r64 = 0.0;
      for (int t = 0; t < OR_BLK; t++) r64 += cache64[t];
      sum64 += r64;
      for (int h = OR_BLK / 2; h > 0; h /= 2)
        for (int t = 0; t < h; t++) cache[t] += cache[t + h];
      vec32[q] = cache[0];
    }
    if (mode == OR_MODE_FP64) {
      out[i] = sum64;
    } else {
      const int threads = size < OR_BLK ? size : OR_BLK;
      const int grids = (size + threads - 1) / threads;
      double ll = 0.0;
      float* cache = (float*)malloc(sizeof(float) * threads);
      for (int b = 0; b < grids; b++) {
        for (int t = 0; t < threads; t++) cache[t] = vec32[(int64_t)b * threads + t];
        for (int h = threads / 2; h > 0; h /= 2)
          for (int t = 0; t < h; t++) cache[t] += cache[t + h];
        ll = (b == 0) ? (double)cache[0] : ll + (double)cache[0];
      }
      free(cache);
      out[i] = ll;
    }
    free(vec32);
  }
  return 0;
}

/* Log-likelihood (GMEMcomputeLikelihoodKernelWithSupervoxels, GMEMupdateCUDA.cu:1913-1978,
 * addTotalLikelihoodWithSupervoxels :2834-2873).
 * ll_true  = sum over every voxel of I*ln(density), densities <= 0 skipped;
 * ll_as_ref = the reference's value: per supervoxel, thread t (of 1024) keeps only the
 * last voxel of its stride with a positive density (the cache overwrite).
 * FP64 mode sums in FP64; REF32 mode reproduces the float cache, the per-block tree,
 * the power-of-two sumVector pass and the host double sum. */
void or_loglik(const OrGaussian* g, const float* query, const float* img, int64_t N,
               const int64_t* lptr, int32_t S, const int32_t* ind, double total_alpha,
               int32_t mode, double* ll_true, double* ll_as_ref) {
  double* part_true = (double*)calloc(S > 0 ? S : 1, sizeof(double));
  double* part_ref = (double*)calloc(S > 0 ? S : 1, sizeof(double));
  float* part_ref32 = (float*)calloc(S > 0 ? S : 1, sizeof(float));
#pragma omp parallel for schedule(dynamic, 16)
  for (int32_t s = 0; s < S; s++) {
    const OrGaussian* c[OR_J];
    for (int j = 0; j < OR_J; j++) c[j] = &g[ind[(int64_t)j * S + s]];
    int64_t p0 = lptr[s], p1 = lptr[s + 1];
    double acc_true = 0.0;
    float cache[OR_BLK];
    double cache64[OR_BLK];
    for (int t = 0; t < OR_BLK; t++) {
      cache[t] = 0.0f;
      cache64[t] = 0.0;
    }
    for (int64_t v = p0; v < p1; v++) {
      double dens = voxel_density(c, query[v], query[N + v], query[2 * N + v], total_alpha);
      if (dens > 0.0) {
        double term = (double)img[v] * log(dens);
        acc_true += term;
        int t = (int)((v - p0) % OR_BLK);
        cache[t] = (float)term;
        cache64[t] = term;
      }
    }
    part_true[s] = acc_true;
    double r64 = 0.0;
    for (int t = 0; t < OR_BLK; t++) r64 += cache64[t];
    part_ref[s] = r64;
    for (int h = OR_BLK / 2; h > 0; h /= 2)
      for (int t = 0; t < h; t++) cache[t] += cache[t + h];
    part_ref32[s] = cache[0];
  }
  double lt = 0.0, lr = 0.0;
  for (int32_t s = 0; s < S; s++) lt += part_true[s];
  if (mode == OR_MODE_FP64) {
    for (int32_t s = 0; s < S; s++) lr += part_ref[s];
  } else {
    /* sumVector over a power-of-two padded vector, blocks of min(1024, size) */
    int size = 1;
    while (size < S) size <<= 1;
    int threads = size < OR_BLK ? size : OR_BLK;
    int grids = (size + threads - 1) / threads;
    float* cache = (float*)malloc(sizeof(float) * threads);
    for (int b = 0; b < grids; b++) {
      for (int t = 0; t < threads; t++) {
        int64_t i = (int64_t)b * threads + t;
        cache[t] = i < S ? part_ref32[i] : 0.0f;
      }
      for (int h = threads / 2; h > 0; h /= 2)
        for (int t = 0; t < h; t++) cache[t] += cache[t + h];
      lr = (b == 0) ? (double)cache[0] : lr + (double)cache[0];
    }
    free(cache);
  }
  *ll_true = lt;
  *ll_as_ref = lr;
  free(part_true);
  free(part_ref);
  free(part_ref32);
}

/* Posterior -> prior (GaussianMixtureModel::updatePriors, GaussianMixtureModel.cpp:892-910,
 * with N_k = nu_k - nu_o from copyFromGMEM_CUDA/updateNk, GaussianMixtureModel.h:169, and
 * the nu_k*=2, W_k/=2 step of mainTrackingGaussianMixtureModel.cpp:961-969). */
void or_update_priors(OrGaussian* g, int32_t K, double beta_pct, double nu_pct, double alpha_pct,
                      double alpha_total) {
  for (int32_t k = 0; k < K; k++) {
    OrGaussian* G = &g[k];
    double n = G->nu_k - G->nu_o;
    for (int d = 0; d < 3; d++) G->m_o[d] = G->m_k[d];
    G->beta_o = fmax(beta_pct * n, 1e-5);
    G->nu_o = fmax(nu_pct * n, 3.0);
    for (int e = 0; e < 6; e++) G->W_o[e] = G->W_k[e] * G->nu_k / G->nu_o;
    if (alpha_total >= 0.0) G->alpha_o = alpha_total * 1e-5 * alpha_pct;
    G->nu_k *= 2.0;
    for (int e = 0; e < 6; e++) G->W_k[e] /= 2.0;
  }
}

/* Post-loop assignment (GMEMupdateCUDA.cu:4310-4350). */
void or_assign_supervoxels(const float* rnk, const int32_t* ind, int32_t S, OrGaussian* g,
                           int32_t K) {
  for (int32_t k = 0; k < K; k++) g[k].supervoxelNum = 0;
  int64_t p = 0;
  for (int j = 0; j < OR_J; j++)
    for (int32_t s = 0; s < S; s++, p++) {
      if (rnk[p] > 0.5f) {
        OrGaussian* G = &g[ind[p]];
        if (G->supervoxelNum < OR_MAX_SV) G->supervoxelIdx[G->supervoxelNum++] = s;
      }
    }
}

/* The EM driver (GMEMvariationalInferenceCUDAWithSupervoxels, GMEMupdateCUDA.cu:3985-4350). */
int or_em_run(const float* query, const float* img, const float* centroids, const int64_t* lptr,
              int64_t N, int32_t S, OrGaussian* g, int32_t K, const OrParams* p, float* rnk,
              int32_t* ind, double* ll_hist, OrStats* st) {
  if (K < OR_J || S < 0 || N < 0) return 1;
  float* ref = (float*)malloc(sizeof(float) * 3 * (size_t)K);
  double* Nk = (double*)malloc(sizeof(double) * K);
  double* Xk = (double*)malloc(sizeof(double) * 3 * (size_t)K);
  double* Sk = (double*)malloc(sizeof(double) * 6 * (size_t)K);
  double ll = -1.0, ll1 = -10.0, ll2 = -100.0, ll3 = -1000.0;
  double ll_true = 0, ll_ref = 0, total = 0;
  int iter = 1;
  int converged = 0;
  for (;;) {
    int go = fabs(ll - ll1) / fabs(ll1) > p->tol && fabs(ll - ll2) / fabs(ll2) > p->tol &&
             fabs(ll - ll3) / fabs(ll3) > p->tol;
    if (!go) {
      converged = 1;
      break;
    }
    if (iter > p->max_iter) break;
    for (int32_t k = 0; k < K; k++)
      for (int d = 0; d < 3; d++) ref[3 * k + d] = (float)g[k].m_k[d];
    if (p->mode == OR_MODE_FP64)
      or_knn_canonical(centroids, S, ref, K, p->scale, ind);
    else
      or_knn_reference(centroids, S, ref, K, p->scale, ind);
    total = or_total_alpha(g, K, p->mode);
    or_prior_constants(g, K, total);
    or_estep(g, query, N, lptr, S, ind, p->mode, rnk, NULL);
    or_mstep(query, img, N, lptr, S, K, ind, rnk, p->mode, Nk, Xk, Sk);
    or_update(g, K, Nk, Xk, Sk, p->mode);
    or_regularize(g, K, p->scale, p->w4dof, p->lambda_min, p->lambda_max, p->max_exc);
    total = or_total_alpha(g, K, p->mode);
    or_kill(g, K, Nk, total);
    ll3 = ll2;
    ll2 = ll1;
    ll1 = ll;
    total = or_total_alpha(g, K, p->mode);
    or_loglik(g, query, img, N, lptr, S, ind, total, p->mode, &ll_true, &ll_ref);
    ll = (p->ll_mode == OR_LL_TRUE) ? ll_true : ll_ref;
    if (ll_hist) ll_hist[iter - 1] = ll;
    iter++;
  }
  or_assign_supervoxels(rnk, ind, S, g, K);
  if (st) {
    st->iterations = iter - 1;
    st->converged = converged;
    st->ll = ll;
    st->ll_true = ll_true;
    st->ll_as_reference = ll_ref;
    st->total_alpha = total;
    int dead = 0;
    for (int32_t k = 0; k < K; k++) dead += g[k].m_o[0] < -1e31;
    st->n_dead = dead;
  }
  free(ref);
  free(Nk);
  free(Xk);
  free(Sk);
  return 0;
}
