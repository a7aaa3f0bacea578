/*
 * synth.cpp -- seeded synthetic nuclei volumes and their supervoxels (host, OpenMP).
 *
 * Stands in for TGMM's image reading + hierarchical segmentation (which produce the
 * supervoxels the EM consumes).  A nucleus is an anisotropic Gaussian blob
 * I(x) = P exp(-1/2 (x-c)' Sigma^-1 (x-c)) with semi-axes a (the 2-sigma contour),
 * a uniform random rotation and a peak P; the volume is background + sum of blobs with
 * Poisson noise, stored as uint16.  Foreground = value > threshold.  Each foreground
 * voxel belongs to the nearest nucleus centre (anisotropy-scaled distance) among the
 * nuclei whose blob reaches it; supervoxels are the 26-connected components of each
 * nucleus's foreground with at least min_size voxels, ordered by nucleus then by
 * first voxel, each a contiguous ascending run of linear indices (x fastest).
 * Intensities are rescaled to (0,1] as I = (v - thr)/(max_fg - thr); centroids are
 * intensity-weighted.  Voxels farther than the blob extent of every nucleus are not
 * sampled (they are background; an isolated noise voxel there would be dropped by the
 * minimum-size rule anyway).
 *
 * Also builds the first-frame Gaussian initialisation of TGMM
 * (mainTrackingGaussianMixtureModel.cpp:897-931 and supportFunctionsMain.cpp:18-121):
 * one Gaussian per nucleus with supervoxels, m = centre + N(0, jitter^2) per axis,
 * N_k = sum of I over its supervoxels, alpha = beta = nu = N_k, W = Id/(nu r^2),
 * regularised, nu_o = 4, W_o = W nu/nu_o, alpha_o = 0.1 N_k, then
 * updatePriors(0.1, 0.1, 0.1, -1) and nu *= 2, W /= 2.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../../include/tgmm_gmem.h"
#include "tgmm_math.cuh"
#include "tgmm_synth.h"

extern "C" {

/* ---------------- counter-based random numbers ---------------- */
static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

typedef struct {
  uint64_t key, ctr;
} Stream;

static inline double unif(Stream* s) {
  uint64_t r = mix64(s->key ^ mix64(s->ctr++));
  return ((r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static inline double normal(Stream* s) {
  double u1 = unif(s), u2 = unif(s);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* Poisson sample: transformed rejection with squeeze (Hoermann, "The transformed
 * rejection method for generating Poisson random variables", 1993) for lam >= 10,
 * multiplication of uniforms below. */
static int64_t poisson(Stream* s, double lam) {
  if (lam < 10.0) {
    double L = exp(-lam), p = 1.0;
    int64_t k = 0;
    do {
      k++;
      p *= unif(s);
    } while (p > L);
    return k - 1;
  }
  const double slam = sqrt(lam), loglam = log(lam);
  const double b = 0.931 + 2.53 * slam;
  const double a = -0.059 + 0.02483 * b;
  const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
  const double vr = 0.9277 - 3.6224 / (b - 2.0);
  for (;;) {
    double U = unif(s) - 0.5, V = unif(s);
    double us = 0.5 - fabs(U);
    int64_t k = (int64_t)floor((2.0 * a / us + b) * U + lam + 0.43);
    if (us >= 0.07 && V <= vr) return k;
    if (k < 0 || (us < 0.013 && V > us)) continue;
    if (log(V) + log(inv_alpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma((double)k + 1.0)) return k;
  }
}

/* ---------------- nuclei ---------------- */
void tgmm_synth_nuclei(const TgmmSynthConfig* c, int32_t n, uint64_t seed, float* centre, float* axes, float* rot,
                       float* peak) {
  for (int32_t i = 0; i < n; i++) {
    Stream s = {mix64(seed * 0x100000001B3ull + 17) ^ (uint64_t)i * 0xD6E8FEB86659FD93ull, 0};
    for (int d = 0; d < 3; d++) centre[3 * i + d] = (float)(unif(&s) * c->dims[d]);
    axes[3 * i + 0] = (float)(c->axis_min + unif(&s) * (c->axis_max - c->axis_min));
    axes[3 * i + 1] = (float)(c->axis_min + unif(&s) * (c->axis_max - c->axis_min));
    axes[3 * i + 2] = (float)((c->axis_min + unif(&s) * (c->axis_max - c->axis_min)) / c->anisotropy);
    /* uniform rotation from a uniform unit quaternion (Shoemake) */
    double u1 = unif(&s), u2 = unif(&s), u3 = unif(&s);
    double q0 = sqrt(1 - u1) * sin(6.283185307179586 * u2), q1 = sqrt(1 - u1) * cos(6.283185307179586 * u2);
    double q2 = sqrt(u1) * sin(6.283185307179586 * u3), q3 = sqrt(u1) * cos(6.283185307179586 * u3);
    double R[9] = {1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3),     2 * (q1 * q3 + q0 * q2),
                   2 * (q1 * q2 + q0 * q3),     1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1),
                   2 * (q1 * q3 - q0 * q2),     2 * (q2 * q3 + q0 * q1),     1 - 2 * (q1 * q1 + q2 * q2)};
    for (int e = 0; e < 9; e++) rot[9 * i + e] = (float)R[e];
    peak[i] = (float)(c->peak_min + unif(&s) * (c->peak_max - c->peak_min));
  }
}

/* ---------------- frame ---------------- */
typedef struct {
  double Q[6];  /* precision (upper triangle 00,01,02,11,12,22) */
  double c[3];
  double P;
  int32_t lo[3], hi[3]; /* inclusive voxel box */
} Blob;

struct TgmmSynthFrame {
  int64_t n_vox;
  int32_t n_sv;
  float* query;
  float* img;
  float* cent;
  int64_t* lptr;
  int32_t* sv_nucleus;
  uint16_t* raw;       /* raw foreground values, same order as query */
  float max_fg;
};

typedef struct {
  int64_t* v;
  int32_t* owner;
  uint16_t* val;
  int64_t n, cap;
} Emit;

static void emit_push(Emit* e, int64_t v, int32_t o, uint16_t val) {
  if (e->n == e->cap) {
    e->cap = e->cap ? 2 * e->cap : 4096;
    e->v = (int64_t*)realloc(e->v, sizeof(int64_t) * e->cap);
    e->owner = (int32_t*)realloc(e->owner, sizeof(int32_t) * e->cap);
    e->val = (uint16_t*)realloc(e->val, sizeof(uint16_t) * e->cap);
  }
  e->v[e->n] = v;
  e->owner[e->n] = o;
  e->val[e->n] = val;
  e->n++;
}

static int cmp_i64(const void* a, const void* b) {
  int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

static inline int in_box(const Blob* b, int x, int y, int z) {
  return x >= b->lo[0] && x <= b->hi[0] && y >= b->lo[1] && y <= b->hi[1] && z >= b->lo[2] && z <= b->hi[2];
}

TgmmSynthFrame* tgmm_synth_frame(const TgmmSynthConfig* c, int32_t n, const float* centre, const float* axes,
                                 const float* rot, const float* peak, uint64_t seed) {
  const int X = c->dims[0], Y = c->dims[1], Z = c->dims[2];
  const double bg = c->background, thr = c->threshold;
  const float sc[3] = {1.0f, 1.0f, c->anisotropy};
  Blob* B = (Blob*)calloc(n > 0 ? n : 1, sizeof(Blob));
  double maxh = 1.0;
  for (int32_t i = 0; i < n; i++) {
    const float* R = rot + 9 * i;
    double sg[3];
    for (int d = 0; d < 3; d++) sg[d] = 0.5 * axes[3 * i + d];
    /* Sigma = R diag(sg^2) R', Q = R diag(1/sg^2) R' */
    double S[9], Q[9];
    for (int r = 0; r < 3; r++)
      for (int q = 0; q < 3; q++) {
        double a = 0, b = 0;
        for (int k = 0; k < 3; k++) {
          a += R[3 * r + k] * sg[k] * sg[k] * R[3 * q + k];
          b += R[3 * r + k] / (sg[k] * sg[k]) * R[3 * q + k];
        }
        S[3 * r + q] = a;
        Q[3 * r + q] = b;
      }
    Blob* bl = &B[i];
    bl->Q[0] = Q[0];
    bl->Q[1] = Q[1];
    bl->Q[2] = Q[2];
    bl->Q[3] = Q[4];
    bl->Q[4] = Q[5];
    bl->Q[5] = Q[8];
    for (int d = 0; d < 3; d++) bl->c[d] = centre[3 * i + d];
    bl->P = peak[i];
    /* blob reaches 10 counts above background inside q <= 2 ln(P/10) */
    double qmax = bl->P > 10.0 ? 2.0 * log(bl->P / 10.0) : 0.0;
    for (int d = 0; d < 3; d++) {
      double h = sqrt(qmax * S[4 * d]) + 1.0;
      if (h > maxh) maxh = h;
      int lo = (int)floor(bl->c[d] - h), hi = (int)ceil(bl->c[d] + h);
      int dim = c->dims[d];
      bl->lo[d] = lo < 0 ? 0 : lo;
      bl->hi[d] = hi > dim - 1 ? dim - 1 : hi;
      if (qmax <= 0.0) bl->hi[d] = bl->lo[d] - 1; /* empty */
    }
  }
  /* neighbour lists through a uniform hash of the centres (cell = 2*max half extent) */
  const double cs = 2.0 * maxh + 2.0;
  const int gx = (int)ceil(X / cs) + 1, gy = (int)ceil(Y / cs) + 1, gz = (int)ceil(Z / cs) + 1;
  const int64_t ng = (int64_t)gx * gy * gz;
  int32_t* gcnt = (int32_t*)calloc(ng + 1, sizeof(int32_t));
  int32_t* gidx = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
  int32_t* gcell = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
  for (int32_t i = 0; i < n; i++) {
    int cx = (int)(B[i].c[0] / cs), cy = (int)(B[i].c[1] / cs), cz = (int)(B[i].c[2] / cs);
    cx = cx < 0 ? 0 : (cx >= gx ? gx - 1 : cx);
    cy = cy < 0 ? 0 : (cy >= gy ? gy - 1 : cy);
    cz = cz < 0 ? 0 : (cz >= gz ? gz - 1 : cz);
    gcell[i] = (int32_t)(((int64_t)cz * gy + cy) * gx + cx);
    gcnt[gcell[i] + 1]++;
  }
  for (int64_t g = 0; g < ng; g++) gcnt[g + 1] += gcnt[g];
  {
    int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (ng + 1));
    memcpy(cur, gcnt, sizeof(int32_t) * (ng + 1));
    for (int32_t i = 0; i < n; i++) gidx[cur[gcell[i]]++] = i; /* ascending i within a cell */
    free(cur);
  }
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  Emit* em = (Emit*)calloc(nthreads, sizeof(Emit));
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    Emit* E = &em[tid];
    int32_t* nb = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 4)
    for (int32_t i = 0; i < n; i++) {
      const Blob* bi = &B[i];
      if (bi->hi[0] < bi->lo[0]) continue;
      /* neighbours whose box overlaps box i */
      int nn = 0;
      int cx = gcell[i] % gx, cy = (gcell[i] / gx) % gy, cz = gcell[i] / (gx * gy);
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            int ux = cx + dx, uy = cy + dy, uz = cz + dz;
            if (ux < 0 || uy < 0 || uz < 0 || ux >= gx || uy >= gy || uz >= gz) continue;
            int64_t g = ((int64_t)uz * gy + uy) * gx + ux;
            for (int32_t q = gcnt[g]; q < gcnt[g + 1]; q++) {
              int32_t j = gidx[q];
              const Blob* bj = &B[j];
              if (bj->hi[0] < bj->lo[0]) continue;
              int ov = 1;
              for (int d = 0; d < 3; d++) ov &= !(bj->hi[d] < bi->lo[d] || bj->lo[d] > bi->hi[d]);
              if (ov) nb[nn++] = j;
            }
          }
      for (int z = bi->lo[2]; z <= bi->hi[2]; z++)
        for (int y = bi->lo[1]; y <= bi->hi[1]; y++)
          for (int x = bi->lo[0]; x <= bi->hi[0]; x++) {
            /* evaluated once: by the lowest-index nucleus whose box holds the voxel */
            int skip = 0;
            for (int q = 0; q < nn && !skip; q++)
              if (nb[q] < i && in_box(&B[nb[q]], x, y, z)) skip = 1;
            if (skip) continue;
            double lam = bg;
            double best = 1e300;
            int32_t owner = -1;
            for (int q = 0; q < nn; q++) {
              const Blob* b = &B[nb[q]];
              if (!in_box(b, x, y, z)) continue;
              double d0 = x - b->c[0], d1 = y - b->c[1], d2 = z - b->c[2];
              double qf = b->Q[0] * d0 * d0 + b->Q[3] * d1 * d1 + b->Q[5] * d2 * d2 +
                          2.0 * (b->Q[1] * d0 * d1 + b->Q[2] * d0 * d2 + b->Q[4] * d1 * d2);
              lam += b->P * exp(-0.5 * qf);
              double e0 = d0 * sc[0], e1 = d1 * sc[1], e2 = d2 * sc[2];
              double dist = e0 * e0 + e1 * e1 + e2 * e2;
              if (dist < best || (dist == best && nb[q] < owner)) {
                best = dist;
                owner = nb[q];
              }
            }
            int64_t v = ((int64_t)z * Y + y) * X + x;
            Stream st = {mix64(seed ^ 0xA0761D6478BD642Full) ^ mix64((uint64_t)v), 0};
            int64_t val = poisson(&st, lam);
            if (val > 65535) val = 65535;
            if ((double)val > thr && owner >= 0) emit_push(E, v, owner, (uint16_t)val);
          }
    }
    free(nb);
  }
  /* group by owner (counting sort), voxels ascending within an owner */
  int64_t total = 0;
  for (int t = 0; t < nthreads; t++) total += em[t].n;
  int64_t* ocnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  for (int t = 0; t < nthreads; t++)
    for (int64_t q = 0; q < em[t].n; q++) ocnt[em[t].owner[q] + 1]++;
  for (int32_t i = 0; i < n; i++) ocnt[i + 1] += ocnt[i];
  int64_t* pv = (int64_t*)malloc(sizeof(int64_t) * (total > 0 ? total : 1));
  uint16_t* pval = (uint16_t*)malloc(sizeof(uint16_t) * (total > 0 ? total : 1));
  {
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * ((size_t)n + 1));
    memcpy(cur, ocnt, sizeof(int64_t) * ((size_t)n + 1));
    for (int t = 0; t < nthreads; t++)
      for (int64_t q = 0; q < em[t].n; q++) {
        int64_t at = cur[em[t].owner[q]]++;
        pv[at] = em[t].v[q];
        pval[at] = em[t].val[q];
      }
    free(cur);
  }
  for (int t = 0; t < nthreads; t++) {
    free(em[t].v);
    free(em[t].owner);
    free(em[t].val);
  }
  free(em);
  /* per owner: sort by linear index (values travel with the index), components */
  int32_t* label = (int32_t*)malloc(sizeof(int32_t) * (total > 0 ? total : 1));
  int32_t* ncomp_kept = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
  int64_t* kept_vox = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 4)
  for (int32_t i = 0; i < n; i++) {
    int64_t b0 = ocnt[i], b1 = ocnt[i + 1], m = b1 - b0;
    if (m == 0) continue;
    /* sort (index, value) pairs by index */
    int64_t* key = (int64_t*)malloc(sizeof(int64_t) * m * 2);
    for (int64_t q = 0; q < m; q++) {
      key[2 * q] = pv[b0 + q];
      key[2 * q + 1] = pval[b0 + q];
    }
    qsort(key, m, 2 * sizeof(int64_t), cmp_i64);
    for (int64_t q = 0; q < m; q++) {
      pv[b0 + q] = key[2 * q];
      pval[b0 + q] = (uint16_t)key[2 * q + 1];
    }
    free(key);
    /* local bitmap over the owner's bounding box */
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-1, -1, -1};
    for (int64_t q = b0; q < b1; q++) {
      int64_t v = pv[q];
      int co[3] = {(int)(v % X), (int)((v / X) % Y), (int)(v / ((int64_t)X * Y))};
      for (int d = 0; d < 3; d++) {
        if (co[d] < lo[d]) lo[d] = co[d];
        if (co[d] > hi[d]) hi[d] = co[d];
      }
    }
    int bx = hi[0] - lo[0] + 1, by = hi[1] - lo[1] + 1, bz = hi[2] - lo[2] + 1;
    int64_t nb = (int64_t)bx * by * bz;
    int32_t* grid = (int32_t*)malloc(sizeof(int32_t) * nb);
    for (int64_t q = 0; q < nb; q++) grid[q] = -1;
    for (int64_t q = b0; q < b1; q++) {
      int64_t v = pv[q];
      int x = (int)(v % X) - lo[0], y = (int)((v / X) % Y) - lo[1], z = (int)(v / ((int64_t)X * Y)) - lo[2];
      grid[((int64_t)z * by + y) * bx + x] = (int32_t)(q - b0);
    }
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * m);
    int32_t* lab = label + b0;
    for (int64_t q = 0; q < m; q++) lab[q] = -1;
    int32_t ncomp = 0;
    for (int64_t q = 0; q < m; q++) {
      if (lab[q] >= 0) continue;
      int32_t sp = 0;
      stack[sp++] = (int32_t)q;
      lab[q] = ncomp;
      while (sp > 0) {
        int32_t u = stack[--sp];
        int64_t v = pv[b0 + u];
        int x = (int)(v % X) - lo[0], y = (int)((v / X) % Y) - lo[1], z = (int)(v / ((int64_t)X * Y)) - lo[2];
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              int xx = x + dx, yy = y + dy, zz = z + dz;
              if (xx < 0 || yy < 0 || zz < 0 || xx >= bx || yy >= by || zz >= bz) continue;
              int32_t w = grid[((int64_t)zz * by + yy) * bx + xx];
              if (w >= 0 && lab[w] < 0) {
                lab[w] = ncomp;
                stack[sp++] = w;
              }
            }
      }
      ncomp++;
    }
    /* component sizes; drop the small ones (label -1) and renumber in first-voxel order */
    int32_t* size = (int32_t*)calloc(ncomp, sizeof(int32_t));
    for (int64_t q = 0; q < m; q++) size[lab[q]]++;
    int32_t* remap = (int32_t*)malloc(sizeof(int32_t) * ncomp);
    int32_t kept = 0;
    for (int32_t k = 0; k < ncomp; k++) remap[k] = size[k] >= c->min_size ? kept++ : -1;
    int64_t kv = 0;
    for (int64_t q = 0; q < m; q++) {
      lab[q] = remap[lab[q]];
      if (lab[q] >= 0) kv++;
    }
    ncomp_kept[i + 1] = kept;
    kept_vox[i + 1] = kv;
    free(size);
    free(remap);
    free(stack);
    free(grid);
  }
  for (int32_t i = 0; i < n; i++) {
    ncomp_kept[i + 1] += ncomp_kept[i];
    kept_vox[i + 1] += kept_vox[i];
  }
  TgmmSynthFrame* F = (TgmmSynthFrame*)calloc(1, sizeof(TgmmSynthFrame));
  const int64_t N = kept_vox[n];
  const int32_t S = ncomp_kept[n];
  F->n_vox = N;
  F->n_sv = S;
  F->query = (float*)malloc(sizeof(float) * 3 * (N > 0 ? N : 1));
  F->img = (float*)malloc(sizeof(float) * (N > 0 ? N : 1));
  F->raw = (uint16_t*)malloc(sizeof(uint16_t) * (N > 0 ? N : 1));
  F->cent = (float*)malloc(sizeof(float) * 3 * (S > 0 ? S : 1));
  F->lptr = (int64_t*)calloc((size_t)S + 1, sizeof(int64_t));
  F->sv_nucleus = (int32_t*)malloc(sizeof(int32_t) * (S > 0 ? S : 1));
  /* supervoxel sizes -> CSR */
  for (int32_t i = 0; i < n; i++) {
    int64_t b0 = ocnt[i], b1 = ocnt[i + 1];
    int32_t s0 = ncomp_kept[i];
    for (int32_t k = s0; k < ncomp_kept[i + 1]; k++) F->sv_nucleus[k] = i;
    for (int64_t q = b0; q < b1; q++)
      if (label[q] >= 0) F->lptr[s0 + label[q] + 1]++;
  }
  for (int32_t s = 0; s < S; s++) F->lptr[s + 1] += F->lptr[s];
  uint16_t mx = 0;
  for (int64_t q = 0; q < total; q++)
    if (label[q] >= 0 && pval[q] > mx) mx = pval[q];
  F->max_fg = mx;
  const double denom = (double)mx - thr > 0 ? (double)mx - thr : 1.0;
#pragma omp parallel for schedule(dynamic, 8)
  for (int32_t i = 0; i < n; i++) {
    int64_t b0 = ocnt[i], b1 = ocnt[i + 1];
    int32_t s0 = ncomp_kept[i], ns = ncomp_kept[i + 1] - s0;
    if (ns == 0) continue;
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * ns);
    for (int32_t k = 0; k < ns; k++) fill[k] = F->lptr[s0 + k];
    for (int64_t q = b0; q < b1; q++) {
      int32_t l = label[q];
      if (l < 0) continue;
      int64_t at = fill[l]++;
      int64_t v = pv[q];
      F->query[at] = (float)(v % X);
      F->query[N + at] = (float)((v / X) % Y);
      F->query[2 * N + at] = (float)(v / ((int64_t)X * Y));
      F->raw[at] = pval[q];
      F->img[at] = (float)(((double)pval[q] - thr) / denom);
    }
    free(fill);
    for (int32_t k = 0; k < ns; k++) {
      int32_t s = s0 + k;
      double w = 0, a0 = 0, a1 = 0, a2 = 0;
      for (int64_t at = F->lptr[s]; at < F->lptr[s + 1]; at++) {
        double I = F->img[at];
        w += I;
        a0 += I * F->query[at];
        a1 += I * F->query[N + at];
        a2 += I * F->query[2 * N + at];
      }
      if (w <= 0) w = 1;
      F->cent[s] = (float)(a0 / w);
      F->cent[S + s] = (float)(a1 / w);
      F->cent[2 * S + s] = (float)(a2 / w);
    }
  }
  free(label);
  free(ncomp_kept);
  free(kept_vox);
  free(ocnt);
  free(pv);
  free(pval);
  free(gcnt);
  free(gidx);
  free(gcell);
  free(B);
  return F;
}

int64_t tgmm_synth_n_vox(const TgmmSynthFrame* F) { return F ? F->n_vox : 0; }
int32_t tgmm_synth_n_sv(const TgmmSynthFrame* F) { return F ? F->n_sv : 0; }
float tgmm_synth_max_fg(const TgmmSynthFrame* F) { return F ? F->max_fg : 0.0f; }

void tgmm_synth_copy(const TgmmSynthFrame* F, float* query, float* img, float* cent, int64_t* lptr,
                     int32_t* sv_nucleus) {
  if (!F) return;
  if (query) memcpy(query, F->query, sizeof(float) * 3 * F->n_vox);
  if (img) memcpy(img, F->img, sizeof(float) * F->n_vox);
  if (cent) memcpy(cent, F->cent, sizeof(float) * 3 * F->n_sv);
  if (lptr) memcpy(lptr, F->lptr, sizeof(int64_t) * (F->n_sv + 1));
  if (sv_nucleus) memcpy(sv_nucleus, F->sv_nucleus, sizeof(int32_t) * F->n_sv);
}

void tgmm_synth_copy_raw(const TgmmSynthFrame* F, uint16_t* raw) {
  if (F && raw) memcpy(raw, F->raw, sizeof(uint16_t) * F->n_vox);
}

void tgmm_synth_free(TgmmSynthFrame* F) {
  if (!F) return;
  free(F->query);
  free(F->img);
  free(F->cent);
  free(F->lptr);
  free(F->sv_nucleus);
  free(F->raw);
  free(F);
}

/* ---------------- first-frame Gaussians ---------------- */

int32_t tgmm_synth_init_gaussians(const TgmmSynthFrame* F, const TgmmSynthConfig* c, int32_t n_nuclei,
                                  const float* centre, uint64_t seed, const TgmmEmParams* prm, TgmmGaussian* out,
                                  int32_t* nucleus_of_gaussian) {
  if (!F || !c || !centre || !prm) return -1;
  double* Nk = (double*)calloc((size_t)n_nuclei + 1, sizeof(double));
  int32_t* nsv = (int32_t*)calloc((size_t)n_nuclei + 1, sizeof(int32_t));
  for (int32_t s = 0; s < F->n_sv; s++) {
    int32_t i = F->sv_nucleus[s];
    nsv[i]++;
    for (int64_t at = F->lptr[s]; at < F->lptr[s + 1]; at++) Nk[i] += F->img[at];
  }
  const double r = 0.5 * (c->axis_min + c->axis_max);
  tgmm::RegConst rc;
  const bool reg_zero = prm->reg_scale[0] == 0.0f && prm->reg_scale[1] == 0.0f && prm->reg_scale[2] == 0.0f;
  for (int d = 0; d < 3; d++) rc.scale[d] = reg_zero ? prm->scale[d] : prm->reg_scale[d];
  rc.w4dof = prm->w4dof;
  rc.lambda_min = prm->lambda_min;
  rc.lambda_max = prm->lambda_max;
  rc.max_exc = prm->max_excentricity;
  int32_t K = 0;
  for (int32_t i = 0; i < n_nuclei; i++) {
    if (nsv[i] == 0 || !(Nk[i] > 0)) continue;
    if (out) {
      TgmmGaussian* g = &out[K];
      memset(g, 0, sizeof(*g));
      Stream st = {mix64(seed * 0x9E3779B97F4A7C15ull + 99) ^ mix64((uint64_t)i + 1), 0};
      const double n = Nk[i];
      for (int d = 0; d < 3; d++) g->m_k[d] = centre[3 * i + d] + c->jitter * normal(&st);
      g->alpha_k = g->beta_k = g->nu_k = n;
      double W[6] = {1.0 / (n * r * r), 0, 0, 1.0 / (n * r * r), 0, 1.0 / (n * r * r)};
      tgmm::regularize_W(W, g->nu_k, rc);
      for (int e = 0; e < 6; e++) g->W_k[e] = W[e];
      g->nu_o = 4.0;
      for (int e = 0; e < 6; e++) g->W_o[e] = g->W_k[e] * g->nu_k / g->nu_o;
      g->alpha_o = 0.1 * n;
      /* updatePriors(0.1, 0.1, 0.1, -1): N_k is the intensity sum here */
      for (int d = 0; d < 3; d++) g->m_o[d] = g->m_k[d];
      g->beta_o = fmax(0.1 * n, 1e-5);
      g->nu_o = fmax(0.1 * n, 3.0);
      for (int e = 0; e < 6; e++) g->W_o[e] = g->W_k[e] * g->nu_k / g->nu_o;
      g->nu_k *= 2.0;
      for (int e = 0; e < 6; e++) g->W_k[e] /= 2.0;
      g->fixed = 0;
      g->splitScore = 0.0;
      int32_t m = 0;
      for (int32_t s = 0; s < F->n_sv && m < TGMM_MAX_SV_PER_GAUSSIAN; s++)
        if (F->sv_nucleus[s] == i) g->supervoxelIdx[m++] = s;
      g->supervoxelNum = m;
    }
    if (nucleus_of_gaussian) nucleus_of_gaussian[K] = i;
    K++;
  }
  free(Nk);
  free(nsv);
  return K;
}

}  /* extern "C" */
