// em_kernels.cu -- the sm_100a kernels of the supervoxel VI-EM.
//
// One EM call is:  build_maps, import (+ frame tail), moments,
//                  then per iteration: knn_estep, mstep_update, kill_prep (+ frame tail),
//                  ll_pass (+ convergence test);  finally assign, export.
// Every kernel loops over the whole batch (one or many frames); frames that have
// converged are skipped through their FrameState::done flag, so a captured graph of
// max_iter iterations serves any batch.  No kernel uses float atomics: per-frame sums
// are fixed-order sums of frame-aligned chunk partials, the M-step visits each
// Gaussian's (supervoxel, slot) pairs in ascending position order, and results are
// bit-identical whether a frame runs alone or inside a batch.
#include <float.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "tgmm_internal.cuh"

namespace tgmm {

namespace {

constexpr float kInfF = __builtin_huge_valf();
constexpr double kInf = __builtin_huge_val();

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;  // identical in every lane: each butterfly level adds commutative pairs
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order sum of the partials [base, base+n) by one warp: lane l adds l, l+32, ...
// in order, then a butterfly.  Every warp that calls it with the same data gets the
// same bits.
__device__ __forceinline__ double warp_sum_range(const double* a, int base, int n) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  int i = lane;
  for (; i + 96 < n; i += 128) {  // four loads in flight, added in the same order
    const double a0 = a[base + i], a1 = a[base + i + 32], a2 = a[base + i + 64], a3 = a[base + i + 96];
    s += a0;
    s += a1;
    s += a2;
    s += a3;
  }
  for (; i < n; i += 32) s += a[base + i];
  return warp_sum(s);
}

// Block (kN threads) fixed-order sum; result valid in thread 0.
template <int kN>
__device__ __forceinline__ double block_sum_n(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < kN / 32; i++) t += sh[i];
  return t;
}

// A chunk's alpha (fixed-order sum, kGChunk threads) and dead count, in one reduction,
// written to the chunk's partials by thread 0.
__device__ __forceinline__ void chunk_partials(double alpha, int dead, double* shd, int* shi, double* alpha_part,
                                               int32_t* dead_part, int c) {
  const double wa = warp_sum(alpha);
  const int wd = warp_sum_i(dead);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    shd[w] = wa;
    shi[w] = wd;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double at = 0.0;
    int nd = 0;
    for (int i = 0; i < kGChunk / 32; i++) {
      at += shd[i];
      nd += shi[i];
    }
    alpha_part[c] = at;
    dead_part[c] = nd;
  }
}

// ---------------------------------------------------------------------------
// kNN primitives.  Distance (FP32, the reference's formula and rounding):
//   a = (q0 - r0) * s0;  d = a*a;  b = (q1 - r1) * s1;  d = fma(b, b, d);  c = ...; d = fma(c, c, d)
// Order: (d, index) ascending, NaN as +inf -> ties go to the lower index.
// ---------------------------------------------------------------------------
// The N nearest found so far, sorted in (d, index) order; unused slots hold (+inf, INT_MAX).
template <int N>
struct TopN {
  float d[N];
  int i[N];
};
using Top5 = TopN<kJ>;

template <int N>
__device__ __forceinline__ void topn_init(TopN<N>& t) {
#pragma unroll
  for (int j = 0; j < N; j++) {
    t.d[j] = kInfF;
    t.i[j] = 0x7fffffff;
  }
}
__device__ __forceinline__ void top5_init(Top5& t) { topn_init<kJ>(t); }

__device__ __forceinline__ bool before(float da, int ia, float db, int ib) {
  return da < db || (da == db && ia < ib);
}

template <int N>
__device__ __forceinline__ void topn_insert(TopN<N>& t, float d, int idx) {
  if (!before(d, idx, t.d[N - 1], t.i[N - 1])) return;
  t.d[N - 1] = d;
  t.i[N - 1] = idx;
#pragma unroll
  for (int p = N - 1; p > 0; --p) {
    if (before(t.d[p], t.i[p], t.d[p - 1], t.i[p - 1])) {
      float td = t.d[p];
      t.d[p] = t.d[p - 1];
      t.d[p - 1] = td;
      int ti = t.i[p];
      t.i[p] = t.i[p - 1];
      t.i[p - 1] = ti;
    }
  }
}
__device__ __forceinline__ void top5_insert(Top5& t, float d, int idx) { topn_insert<kJ>(t, d, idx); }

__device__ __forceinline__ float knn_dist(float q0, float q1, float q2, float r0, float r1,
                                          float r2, const float* s) {
  float a = __fmul_rn(__fsub_rn(q0, r0), s[0]);
  float d = __fmul_rn(a, a);
  float b = __fmul_rn(__fsub_rn(q1, r1), s[1]);
  d = __fmaf_rn(b, b, d);
  float c = __fmul_rn(__fsub_rn(q2, r2), s[2]);
  d = __fmaf_rn(c, c, d);
  return isnan(d) ? kInfF : d;
}

// Grid geometry of one point set (the queries' bounding box in scaled space).
struct GridGeom {
  float lo[3];
  float h, inv_h;
  int dims[3];
};

__device__ __forceinline__ int cell_coord(float y, float lo, float inv_h, int dim) {
  float u = (y - lo) * inv_h;
  int c = (u > 0.0f) ? (u < (float)dim ? (int)u : dim - 1) : 0;  // NaN -> 0 (not used)
  return c;
}

// Exact grid search: rings of cells at growing Chebyshev distance r around the query's
// cell; stop after ring r once the fifth distance is strictly below the squared lower
// bound (r*h + delta - eps)^2 of every unvisited cell.  eps absorbs float rounding of
// the scaled coordinates and of the distance itself.  Refs outside the box sit in the
// boundary cells, which keeps the bound valid for queries inside the box.
template <int N>
__device__ void knn_grid_search(float q0, float q1, float q2, const float* s, const GridGeom& g,
                                const int32_t* __restrict__ cstart, const float4* __restrict__ refs,
                                TopN<N>& t) {
  const float y[3] = {q0 * s[0], q1 * s[1], q2 * s[2]};
  int c[3];
  float delta = kInfF;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    c[a] = cell_coord(y[a], g.lo[a], g.inv_h, g.dims[a]);
    float f0 = y[a] - (g.lo[a] + c[a] * g.h);
    float f1 = (g.lo[a] + (c[a] + 1) * g.h) - y[a];
    delta = fminf(delta, fminf(f0, f1));
  }
  delta = fmaxf(delta, 0.0f);
  const int maxr = max(g.dims[0], max(g.dims[1], g.dims[2]));
  for (int r = 0; r <= maxr; ++r) {
    const int z0 = max(c[2] - r, 0), z1 = min(c[2] + r, g.dims[2] - 1);
    const int y0 = max(c[1] - r, 0), y1 = min(c[1] + r, g.dims[1] - 1);
    for (int z = z0; z <= z1; ++z) {
      const bool zedge = (z == c[2] - r) || (z == c[2] + r);
      for (int yy = y0; yy <= y1; ++yy) {
        const bool edge = zedge || (yy == c[1] - r) || (yy == c[1] + r);
        const int row = (z * g.dims[1] + yy) * g.dims[0];
        int xa, xb, step;
        if (edge) {
          xa = max(c[0] - r, 0);
          xb = min(c[0] + r, g.dims[0] - 1);
          step = 1;
        } else {
          xa = c[0] - r;
          xb = c[0] + r;
          step = 2 * r;
        }
        for (int x = xa; x <= xb; x += step) {
          if (x < 0 || x >= g.dims[0]) continue;
          const int cell = row + x;
          const int b = cstart[cell], e = cstart[cell + 1];
          for (int k = b; k < e; ++k) {
            const float4 rr = refs[k];
            topn_insert<N>(t, knn_dist(q0, q1, q2, rr.x, rr.y, rr.z, s), __float_as_int(rr.w));
          }
        }
      }
    }
    const float lb = r * g.h + delta;
    const float eps = 4e-3f + 1e-6f * lb;
    if (lb > eps) {
      const float bound = (lb - eps) * (lb - eps);
      if (t.d[N - 1] < bound) break;
    }
  }
}

__device__ __forceinline__ FrameDesc load_desc(const DevPlan& P, int f) { return P.frames[f]; }

}  // namespace


// Grid geometry over the bounding box [lo, hi] (scaled space): cubic cells of side h,
// about one reference per cell, at most budget-1 cells in total.
__device__ void set_geometry(FrameState* S, const float* lo, const float* hi, int n_ref, int cell_budget) {
  float ext[3];
  double vol = 1.0;
  for (int d = 0; d < 3; d++) {
    ext[d] = fmaxf(hi[d] - lo[d], 1.0f);
    vol *= ext[d];
  }
  // about kRefsPerCell references per cell: the neighbours a supervoxel keeps then usually
  // lie within the first ring of cells around the query
  const int budget = max(cell_budget - 1, 1);
  const int target = max(1, min(budget, n_ref / kRefsPerCell));
  float h = (float)cbrt(vol / target);
  int dims[3] = {1, 1, 1};
  for (int guard = 0; guard < 400; guard++) {
    long long tot = 1;
    for (int d = 0; d < 3; d++) {
      dims[d] = max(1, min(1024, (int)ceilf(ext[d] / h)));
      tot *= dims[d];
    }
    if (tot <= budget) break;
    h *= 1.1f;
  }
  for (int d = 0; d < 3; d++) {
    S->lo[d] = lo[d];
    S->dims[d] = dims[d];
  }
  S->h = h;
  S->inv_h = 1.0f / h;
  S->n_cells = dims[0] * dims[1] * dims[2];
}

// The stream record (SvRec) of supervoxel s (frame-local sl) for the voxel pass.
__device__ void write_sv_rec(const DevPlan& P, const FrameDesc& D, int f, int s, int sl) {
  const int64_t a = D.lptr[sl], b = D.lptr[sl + 1];
  const bool ok = !(a < 0 || b < a || b > D.n_vox || b - a >= (1 << 30));
  const int nv = ok ? (int)(b - a) : 0;
  const int nt = (nv + kVoxTile - 1) / kVoxTile;
  const int r0 = nt ? nv - (nt - 1) * kVoxTile : 0;
  SvRec r;
  const float* comp[4] = {D.query, D.query + D.n_vox, D.query + 2 * D.n_vox, D.img};
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const uintptr_t a0 = nt ? (uintptr_t)(comp[c] + a) : 0;
    const uintptr_t a1 = a0 + 4u * (unsigned)r0;  // first voxel of tile 1
    r.lo0[c] = a0 & ~(uintptr_t)15;
    r.lo1[c] = a1 & ~(uintptr_t)15;
    r.n0[c] = nt ? (unsigned)(((a1 + 15) & ~(uintptr_t)15) - r.lo0[c]) : 0u;
    r.nf[c] = (4u * kVoxTile + ((a1 & 15) ? 16u : 0u)) | ((unsigned)((a0 & 15) >> 2) << 16) |
              ((unsigned)((a1 & 15) >> 2) << 20);
  }
  r.ntiles = nt;
  r.nv = nv;
  r.frame = f;
  r.frame_nsv = D.n_sv;
  r.c0 = D.cent[sl];
  r.c1 = D.cent[(int64_t)D.n_sv + sl];
  r.c2 = D.cent[2 * (int64_t)D.n_sv + sl];
  r.r0 = r0;
  P.sv_rec[s] = r;
  SvLL l;
  l.v0 = D.vox_base + (nt ? a : 0);
  l.nv = nv;
  l.ntiles = nt;
  l.r0 = r0;
  l.frame = f;
  l.frame_nsv = D.n_sv;
  l.c0 = r.c0;
  l.c1 = r.c1;
  l.c2 = r.c2;
  l.pad[0] = l.pad[1] = 0;
  P.sv_ll[s] = l;
}

// ===========================================================================
// build_maps: per frame -- supervoxel/Gaussian -> frame maps, CSR validation,
// centroid bounding box and grid geometry, EM state reset.
// ===========================================================================
__global__ void __launch_bounds__(kFrameThreads) k_build_maps(DevPlan P) {
  // block (f, y): the frame's map stores split over kMapSlices blocks; block (f, 0) also
  // checks the CSR, takes the centroids' bounding box and starts the frame's state
  const int f = blockIdx.x;
  if (f >= P.info->n_frames) return;
  const FrameDesc D = load_desc(P, f);
  const int first = blockIdx.y * blockDim.x + threadIdx.x, stride = kMapSlices * blockDim.x;
  for (int i = first; i < D.n_sv; i += stride) P.sv_frame[D.sv_base + i] = f;
#pragma unroll 4
  for (int i = first; i < D.n_gauss; i += stride) {
    P.g_frame[D.g_base + i] = f;
    P.bcnt[D.g_base + i] = 0;  // M-step and assignment buckets start empty
    P.acnt[D.g_base + i] = 0;
  }
  for (int i = first; i < D.cell_budget; i += stride) P.cell_cnt[D.cell_base + i] = 0;
  if (blockIdx.y != 0) return;
  FrameState* S = &P.state[f];
  __shared__ float smin[3][32], smax[3][32];
  __shared__ int sbad;
  if (threadIdx.x == 0) sbad = 0;
  __syncthreads();
  if (threadIdx.x < kOrderBuckets) {  // the supervoxel order's bucket counts and cursors
    P.ord_hist[f * kOrderBuckets + threadIdx.x] = 0;
    P.ord_cur[f * kOrderBuckets + threadIdx.x] = 0;
  }
  int bad = 0;
  float lo[3] = {kInfF, kInfF, kInfF}, hi[3] = {-kInfF, -kInfF, -kInfF};
  // unrolled so that several supervoxels' loads are in flight at once
#pragma unroll 4
  for (int i = threadIdx.x; i < D.n_sv; i += blockDim.x) {
    const int64_t a = D.lptr[i], b = D.lptr[i + 1];
    if (a < 0 || b < a || b > D.n_vox) bad = 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float y = D.cent[(int64_t)d * D.n_sv + i] * D.scale[d];
      if (!isfinite(y)) {
        bad |= 2;
        continue;
      }
      lo[d] = fminf(lo[d], y);
      hi[d] = fmaxf(hi[d], y);
    }
  }
  if (bad) atomicOr(&sbad, bad);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int d = 0; d < 3; d++) {
      smin[d][w] = lo[d];
      smax[d][w] = hi[d];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int d = 0; d < 3; d++) {
      lo[d] = smin[d][0];
      hi[d] = smax[d][0];
      for (int i = 1; i < (int)(blockDim.x >> 5); i++) {
        lo[d] = fminf(lo[d], smin[d][i]);
        hi[d] = fmaxf(hi[d], smax[d][i]);
      }
      if (!(lo[d] <= hi[d])) {
        lo[d] = 0.0f;
        hi[d] = 0.0f;
      }
    }
    int flags = 0;
    if (sbad & 1) flags |= F_BAD_CSR;
    if (sbad & 2) flags |= F_NAN_INPUT;
    if (D.n_gauss < kJ) flags |= F_FEW_GAUSS;
    set_geometry(S, lo, hi, D.n_gauss, D.cell_budget);
    S->iter = 1;
    S->disp_cum = 0.0;
    S->disp_max = 0u;
    S->knn_searches = 0;
    S->done = (flags & (F_BAD_CSR | F_FEW_GAUSS)) ? 1 : 0;
    S->converged = 0;
    S->flags = flags;
    S->n_dead = 0;
    S->ll = -1.0;
    S->ll1 = -10.0;
    S->ll2 = -100.0;
    S->ll3 = -1000.0;
    S->ll_true = 0.0;
    S->ll_ref = 0.0;
    S->total_alpha = 0.0;
    S->ln_alpha = 0.0;
    S->psi_total[0] = S->psi_total[1] = 0.0;
    S->ll_int[0] = S->ll_int[1] = 0;
    S->ll_frac[0] = S->ll_frac[1] = 0;
    S->sv_done = 0;
    S->blk_done = 0;
  }
}

// Gaussian -> grid cell (or -1 when its float centre is unusable for pruning).
__device__ __forceinline__ int ref_cell_of(const FrameState& S, const FrameDesc& D, float x, float y,
                                           float z) {
  const float ys[3] = {x * D.scale[0], y * D.scale[1], z * D.scale[2]};
#pragma unroll
  for (int d = 0; d < 3; d++)
    if (!isfinite(ys[d]) || fabsf(ys[d]) >= 1e25f) return -1;
  const int cx = cell_coord(ys[0], S.lo[0], S.inv_h, S.dims[0]);
  const int cy = cell_coord(ys[1], S.lo[1], S.inv_h, S.dims[1]);
  const int cz = cell_coord(ys[2], S.lo[2], S.inv_h, S.dims[2]);
  return (cz * S.dims[1] + cy) * S.dims[0] + cx;
}

// The next iteration's records of Gaussian k from its parameters: psi(alpha) and
// E[ln|Lambda|] (in the parity slot), the E-step record (nu W, m, 3/beta, psi(alpha) +
// E[ln|Lambda|]/2, or -inf for a dead Gaussian), the log-likelihood record (-nu W/2 with
// doubled off-diagonals, the log weight 1/2 ln(det W nu^3) - 3/2 ln(2 pi) + ln(alpha), the
// mean) and the float centre the kNN sees (kpos).  With `track`, returns how far that
// centre moved since the previous record (scaled distance, 0 unless live both times),
// which bounds the kNN neighbour lists.
__device__ __forceinline__ double write_records(const DevPlan& P, const FrameDesc& D, int k, int parity, bool dead,
                                                const double* W, double nu, double alpha, double beta,
                                                const double* m, bool track, float4 o = float4{}) {
  const double psa = digamma(alpha);
  const double eld = dead ? -1e32 : expected_log_det(W, nu);
  gcomp(P, G_PSIA0 + parity, k) = psa;
  gcomp(P, G_ELD0 + parity, k) = eld;
  double* E = P.ec + (int64_t)k * kEcStride;
#pragma unroll
  for (int e = 0; e < 6; e++) E[e] = nu * W[e];
  E[6] = m[0];
  E[7] = m[1];
  E[8] = m[2];
  E[9] = 3.0 / beta;
  E[10] = dead ? -(double)kInfF : psa + 0.5 * eld;
  double* L = P.llc + (int64_t)k * 10;
  L[0] = -0.5 * nu * W[0];
  L[1] = -nu * W[1];
  L[2] = -nu * W[2];
  L[3] = -0.5 * nu * W[3];
  L[4] = -nu * W[4];
  L[5] = -0.5 * nu * W[5];
  L[6] = 0.5 * log(det3(W) * nu * nu * nu) - 1.5 * kLnTwoPi + log(alpha);
  L[7] = m[0];
  L[8] = m[1];
  L[9] = m[2];
  const float x = __double2float_rn(m[0]);
  const float y = __double2float_rn(m[1]);
  const float z = __double2float_rn(m[2]);
  double move = 0.0;
  if (track && !dead) {  // o: the centre kpos held before (loaded by the caller)
    if (o.w != 0.0f) {
      const double a = ((double)x - (double)o.x) * (double)D.scale[0];
      const double b = ((double)y - (double)o.y) * (double)D.scale[1];
      const double c = ((double)z - (double)o.z) * (double)D.scale[2];
      move = sqrt(a * a + b * b + c * c);
    }
  }
  P.kpos[k] = make_float4(x, y, z, dead ? 0.0f : 1.0f);
  return move;
}

// A live Gaussian's float centre (kpos) into its grid cell (capacity kCellCap; a full cell
// flags the frame, whose kNN then scans every Gaussian).
// `cell`: ref_cell_of the centre, or -1 (outside every cell: not inserted).
__device__ __forceinline__ void grid_insert_at(const DevPlan& P, const FrameDesc& D, int cell, int k, float4 c4) {
  if (cell >= 0) {
    const int g = D.cell_base + cell;
    const int pos = atomicAdd(&P.cell_cnt[g], 1);
    if (pos < kCellCap)
      P.cell_refs[(int64_t)g * kCellCap + pos] = make_float4(c4.x, c4.y, c4.z, __int_as_float(k - D.g_base));
    else
      atomicOr(&P.state[D.frame_id].flags, F_CELL_OVERFLOW);
  }
}
__device__ __forceinline__ void grid_insert(const DevPlan& P, const FrameDesc& D, const FrameState& S, int k,
                                            float4 c4) {
  grid_insert_at(P, D, ref_cell_of(S, D, c4.x, c4.y, c4.z), k, c4);
}


// Run by the last Gaussian chunk of a frame to finish (import or kill step): the alpha
// total as a fixed-order sum of the chunk partials, psi and ln of it for the next
// iteration, and the dead count.
__device__ void frame_tail(const DevPlan& P, int f, int next_parity) {
  const FrameDesc D = load_desc(P, f);
  FrameState* S = &P.state[f];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w == 0) {
    const double a = warp_sum_range(P.alpha_part_f, D.gchunk_base, D.n_gchunks);
    int nd = 0;
    for (int i = lane; i < D.n_gchunks; i += 32) nd += P.dead_part[D.gchunk_base + i];
    nd = warp_sum_i(nd);
    if (lane == 0) {
      S->total_alpha = a;
      S->ln_alpha = log(a);
      S->psi_total[next_parity] = digamma(a);
      S->n_dead = nd;
      S->blk_done = 0;
      S->disp_cum += (double)__uint_as_float(S->disp_max);
      S->disp_max = 0u;
    }
  }
}

// The last-arriving chunk of frame f runs frame_tail.  Every chunk calls this after its
// own writes; no thread waits on another.
__device__ __forceinline__ void chunk_done(const DevPlan& P, int f, int n_chunks, int next_parity) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&P.state[f].blk_done, 1) == n_chunks - 1) ? 1 : 0;
  __syncthreads();
  if (s_last) {
    __threadfence();
    frame_tail(P, f, next_parity);
  }
}

// ===========================================================================
// import: AoS (288-byte records) -> SoA, validation, preparation of iteration 1.
// ===========================================================================
__global__ void __launch_bounds__(kGChunk) k_import(DevPlan P) {
  const int c = blockIdx.x;
  if (c >= P.info->n_gchunks) return;
  const GChunk ch = P.gchunks[c];
  const FrameDesc D = load_desc(P, ch.frame);
  const FrameState& S = P.state[ch.frame];
  __shared__ double shd[kGChunk / 32];
  __shared__ int shi[kGChunk / 32];
  const int k = ch.g_begin + threadIdx.x;
  double alpha = 0.0;
  int dead = 0;
  if (k < ch.g_end) {
    const TgmmGaussian& g = D.gm[k - D.g_base];
    bool bad = false;
    gcomp(P, G_BETA, k) = g.beta_k;
    gcomp(P, G_NU, k) = g.nu_k;
    gcomp(P, G_ALPHA, k) = g.alpha_k;
    for (int d = 0; d < 3; d++) gcomp(P, G_M0 + d, k) = g.m_k[d];
    for (int e = 0; e < 6; e++) gcomp(P, G_W0 + e, k) = g.W_k[e];
    gcomp(P, G_BETAO, k) = g.beta_o;
    gcomp(P, G_NUO, k) = g.nu_o;
    gcomp(P, G_ALPHAO, k) = g.alpha_o;
    for (int d = 0; d < 3; d++) gcomp(P, G_MO0 + d, k) = g.m_o[d];
    for (int e = 0; e < 6; e++) gcomp(P, G_WO0 + e, k) = g.W_o[e];
    P.fixed[k] = g.fixed ? 1 : 0;
    bad = isnan(g.beta_k) || isnan(g.nu_k) || isnan(g.alpha_k);
    for (int d = 0; d < 3; d++) bad = bad || isnan(g.m_k[d]);
    for (int e = 0; e < 6; e++) bad = bad || isnan(g.W_k[e]);
    if (bad) atomicOr(&P.state[ch.frame].flags, F_NAN_INPUT);
    // the first iteration's records and grid entry from the values just read
    const bool is_dead = is_dead_prior(g.m_o[0]);
    write_records(P, D, k, 1, is_dead, g.W_k, g.nu_k, g.alpha_k, g.beta_k, g.m_k, false);
    if (!is_dead) grid_insert(P, D, S, k, P.kpos[k]);
    alpha = g.alpha_k;
    dead = is_dead ? 1 : 0;
  }
  chunk_partials(alpha, dead, shd, shi, P.alpha_part_f, P.dead_part, c);
  chunk_done(P, ch.frame, D.n_gchunks, 1);
}

// ===========================================================================
// order: once per call.  The supervoxels' stream records, and the supervoxels of each
// frame by descending tile count (counting sort, ties in any order), frames in batch order.
// The voxel passes take supervoxels in this order, so a frame's last supervoxels are its
// smallest and no warp is left with a large one after the others ran out of work.  Their
// sums do not depend on the order.
// ===========================================================================

__device__ __forceinline__ int order_bucket(const FrameDesc& D, int sl) {
  const int64_t a = D.lptr[sl], b = D.lptr[sl + 1];
  const int64_t nv = (a < 0 || b < a || b > D.n_vox) ? 0 : b - a;
  const int64_t nt = (nv + kVoxTile - 1) / kVoxTile;
  return nt < kOrderBuckets - 1 ? (int)nt : kOrderBuckets - 1;
}

// k_sv_records: thread per supervoxel -- its stream record, and its bucket counted in its
// frame's histogram (lanes of a warp with the same frame and bucket add once).
__global__ void __launch_bounds__(256) k_sv_records(DevPlan P) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = s < P.info->total_sv;
  int key = -1;
  if (in) {
    const int f = P.sv_frame[s];
    const FrameDesc D = load_desc(P, f);
    const int sl = s - D.sv_base;
    write_sv_rec(P, D, f, s, sl);
    key = f * kOrderBuckets + order_bucket(D, sl);
  }
  const unsigned m = __match_any_sync(0xffffffffu, key);
  if (in && (m & ((1u << (threadIdx.x & 31)) - 1u)) == 0) atomicAdd(&P.ord_hist[key], __popc(m));
}

// k_order_base: one warp per frame -- the buckets' first places, largest tile counts first.
__global__ void __launch_bounds__(32) k_order_base(DevPlan P) {
  const int f = blockIdx.x;
  if (f >= P.info->n_frames || threadIdx.x != 0) return;
  int run = 0;
  for (int b = kOrderBuckets - 1; b >= 0; b--) {
    const int c = P.ord_hist[f * kOrderBuckets + b];
    P.ord_hist[f * kOrderBuckets + b] = run;  // from here on: the bucket's base
    run += c;
  }
}

// k_order_scatter: thread per supervoxel -- its place, its bucket's base plus a cursor
// (one atomic per warp and bucket).  Places within a bucket depend on the run; the voxel
// pass's sums do not.
__global__ void __launch_bounds__(256) k_order_scatter(DevPlan P) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = s < P.info->total_sv;
  int key = -1, base = 0;
  if (in) {
    const int f = P.sv_frame[s];
    const FrameDesc D = load_desc(P, f);
    key = f * kOrderBuckets + order_bucket(D, s - D.sv_base);
    base = D.sv_base + P.ord_hist[key];
  }
  const unsigned m = __match_any_sync(0xffffffffu, key);
  const int lane = threadIdx.x & 31, lead = __ffs(m) - 1;
  int start = 0;
  if (in && lane == lead) start = atomicAdd(&P.ord_cur[key], __popc(m));
  start = __shfl_sync(m, start, lead);
  if (in) P.sv_order[base + start + __popc(m & ((1u << lane) - 1u))] = s;
}


// ===========================================================================
// knn_estep: a group of G lanes per supervoxel (32 / G supervoxels per warp; G = 4, 8, 16
// or 32, chosen per plan, by tgmm_plan_autotune or tgmm_plan_set_knn_group; every G gives
// the same bits).
// Exact 5-NN of the centroid among the frame's Gaussian centres: the group's lanes split
// each ring of grid cells, keep private top-5 lists pruned by the group's current fifth
// distance, and after each ring the lists are merged by five rounds of a group-wide
// (distance, index) arg-min.  Then the E-step from the supervoxel's moments, candidate j
// on lane j mod G of the group (lane 0 also takes candidate 4 when G = 4):
//   L_j = sum_v [-1/2 (3/beta + nu d'Wd) + E ln pi + 1/2 E ln|Lambda|]
//       = -1/2 (3 n/beta + nu tr(W D)) + n (psi(alpha) - psi(sum alpha) + 1/2 E ln|Lambda|),
//   D = sum_v (x_v - m)(x_v - m)' = G2 - G1 u' - u G1' + n u u',  u = m - c_s,
// in FP64; then the reference's float-storage semantics (empty supervoxel -> 0, dead
// candidate or |L| beyond float range -> -inf) and rnk_j = 1 / sum_i exp(L_i - L_j).
// Pairs with rnk > 1e-3 go to the Gaussian's M-step bucket.
// ===========================================================================
constexpr int kKnnWarps = 4;  // warps per block; the lanes per supervoxel (G) come from the plan
#ifndef TGMM_KNN_BLOCKS
#define TGMM_KNN_BLOCKS 5  // 96 registers: the list path fits more warps; the rare grid search spills a little
#endif
constexpr int kKnnBlocks = TGMM_KNN_BLOCKS;  // resident blocks per SM the kNN/E-step is compiled for

// group-wide lexicographic arg-min of (d, i); every lane of the group gets the winner
template <int G>
__device__ __forceinline__ void group_min_pair(float& d, int& i, unsigned gmask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    const float od = __shfl_xor_sync(gmask, d, o);
    const int oi = __shfl_xor_sync(gmask, i, o);
    if (before(od, oi, d, i)) {
      d = od;
      i = oi;
    }
  }
}

// merge the group's sorted lists into its top-N (identical in every lane of the group)
template <int G, int N>
__device__ __forceinline__ void group_merge_topn(TopN<N>& mine, TopN<N>& out, unsigned gmask) {
#pragma unroll
  for (int r = 0; r < N; r++) {
    float d = mine.d[0];
    int i = mine.i[0];
    group_min_pair<G>(d, i, gmask);
    out.d[r] = d;
    out.i[r] = i;
    if (mine.i[0] == i && mine.d[0] == d && i != 0x7fffffff) {  // pop the front of the winner
#pragma unroll
      for (int q = 0; q < N - 1; q++) {
        mine.d[q] = mine.d[q + 1];
        mine.i[q] = mine.i[q + 1];
      }
      mine.d[N - 1] = kInfF;
      mine.i[N - 1] = 0x7fffffff;
    }
  }
}

// group-wide lexicographic arg-max of (d, i)
template <int G>
__device__ __forceinline__ void group_max_pair(float& d, int& i, unsigned gmask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    const float od = __shfl_xor_sync(gmask, d, o);
    const int oi = __shfl_xor_sync(gmask, i, o);
    if (before(d, i, od, oi)) {
      d = od;
      i = oi;
    }
  }
}

// Exact N nearest over the grid rings.  (td0, ti0): a (distance, index) no smaller than
// the true N-th neighbour's (the N-th of N known Gaussians), or +inf; refs after it in
// (distance, index) order cannot be among the N and are rejected without an insertion.
template <int G, int N>
__device__ void knn_group_search(float q0, float q1, float q2, const float* s, const GridGeom& g,
                                 const int32_t* __restrict__ ccnt, const float4* __restrict__ refs, TopN<N>& best,
                                 unsigned gmask, int gl, float td0, int ti0) {
  const float y[3] = {q0 * s[0], q1 * s[1], q2 * s[2]};
  int c[3];
  float delta = kInfF;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    c[a] = cell_coord(y[a], g.lo[a], g.inv_h, g.dims[a]);
    const float f0 = y[a] - (g.lo[a] + c[a] * g.h);
    const float f1 = (g.lo[a] + (c[a] + 1) * g.h) - y[a];
    delta = fminf(delta, fminf(f0, f1));
  }
  delta = fmaxf(delta, 0.0f);
  topn_init<N>(best);
  const int maxr = max(1, max(g.dims[0], max(g.dims[1], g.dims[2])));
  // the first pass covers rings 0 and 1 (27 cells), later passes one ring
  for (int r = 1; r <= maxr; ++r) {
    TopN<N> t;
    topn_init<N>(t);
    // prune with the group's current N-th (or the starting bound): a ref must not come
    // after it to matter
    const bool use_best = before(best.d[N - 1], best.i[N - 1], td0, ti0);
    const float td = use_best ? best.d[N - 1] : td0;
    const int ti = use_best ? best.i[N - 1] : ti0;
    auto scan_refs = [&](int cell, int e) {
      const float4* cr = refs + (int64_t)cell * kCellCap;
      for (int k = 0; k < e; ++k) {
        const float4 rr = cr[k];
        const float d = knn_dist(q0, q1, q2, rr.x, rr.y, rr.z, s);
        const int id = __float_as_int(rr.w);
        if (!before(td, ti, d, id)) topn_insert<N>(t, d, id);
      }
    };
    auto scan_cell = [&](int dx, int dy, int dz) {
      const int x = c[0] + dx, yy = c[1] + dy, z = c[2] + dz;
      if (x < 0 || yy < 0 || z < 0 || x >= g.dims[0] || yy >= g.dims[1] || z >= g.dims[2]) return;
      const int cell = (z * g.dims[1] + yy) * g.dims[0] + x;
      scan_refs(cell, min(ccnt[cell], kCellCap));
    };
    // the cells of ring r (the whole cube for r = 1), with constant divisors for the
    // rings a search usually needs
    if (r == 1) {
      // the lane's cells of the 3x3x3 cube: their counts first, as independent loads
      constexpr int kPer = (27 + G - 1) / G;
      int cq[kPer], eq[kPer];
#pragma unroll
      for (int q = 0; q < kPer; q++) {
        const int idx = gl + G * q;
        const int x = c[0] + idx % 3 - 1, yy = c[1] + (idx / 3) % 3 - 1, z = c[2] + idx / 9 - 1;
        const bool in = idx < 27 && x >= 0 && yy >= 0 && z >= 0 && x < g.dims[0] && yy < g.dims[1] && z < g.dims[2];
        cq[q] = in ? (z * g.dims[1] + yy) * g.dims[0] + x : 0;
        eq[q] = in ? min(ccnt[cq[q]], kCellCap) : 0;
      }
#pragma unroll
      for (int q = 0; q < kPer; q++) scan_refs(cq[q], eq[q]);
    } else if (r == 2) {
      for (int idx = gl; idx < 125; idx += G) {
        const int dx = idx % 5 - 2, dy = (idx / 5) % 5 - 2, dz = idx / 25 - 2;
        if (max(abs(dx), max(abs(dy), abs(dz))) == 2) scan_cell(dx, dy, dz);
      }
    } else if (r == 3) {
      for (int idx = gl; idx < 343; idx += G) {
        const int dx = idx % 7 - 3, dy = (idx / 7) % 7 - 3, dz = idx / 49 - 3;
        if (max(abs(dx), max(abs(dy), abs(dz))) == 3) scan_cell(dx, dy, dz);
      }
    } else {
      const int side = 2 * r + 1;
      const int cube = side * side * side;
      for (int idx = gl; idx < cube; idx += G) {
        const int dx = idx % side - r, dy = (idx / side) % side - r, dz = idx / (side * side) - r;
        if (max(abs(dx), max(abs(dy), abs(dz))) == r) scan_cell(dx, dy, dz);
      }
    }
    // lane 0 of the group also carries the previous best (disjoint from this ring's refs)
    if (gl == 0) {
#pragma unroll
      for (int q = 0; q < N; q++) topn_insert<N>(t, best.d[q], best.i[q]);
    }
    TopN<N> merged;
    group_merge_topn<G, N>(t, merged, gmask);
    best = merged;
    const float lb = r * g.h + delta;
    const float eps = 4e-3f + 1e-6f * lb;
    if (lb > eps) {
      const float bound = (lb - eps) * (lb - eps);
      if (best.d[N - 1] < bound) break;
    }
  }
}

// The kNN/E-step of supervoxel s for iteration `it` by the G lanes of one group (lane gl
// of the group whose first lane is gbase).  Its candidates and responsibilities go to the
// buffers of the iteration's parity.  It reads the frame state the kill step of iteration
// it - 1 left (grid, neighbour-list bound, psi of the alpha total) and the done flag:
// when it runs inside the voxel pass of iteration it - 1 (k_ll_pass), that pass may end
// the frame meanwhile, and the results of an iteration that does not run are never read.
template <int G>
__device__ __forceinline__ void knn_estep_sv(const DevPlan& P, int s, int it, int gl, int gbase, unsigned gmask) {
  static_assert(G >= 4 && G <= 32 && (G & (G - 1)) == 0, "groups of 4 to 32 lanes");
  // per lane: list members gl + G q (q < kM) and candidates gl + G q (q < kC); one of each
  // for groups of 8 or more lanes
  constexpr int kM = (kNbr + G - 1) / G, kC = (kJ + G - 1) / G;
  // whole groups leave together; every shuffle below names only the group's lanes
  if (s >= P.info->total_sv) return;
  // what needs only s goes out first, ahead of the frame's state and descriptor: the
  // supervoxel's stream record (frame, centroid, voxel count), the list member of this lane
  // (a global Gaussian index, so that its centre loads beside the frame's state) and the
  // list's bound, and (into L1) the moments the E-step reads
  const SvLL R = P.sv_ll[s];
  int lk[kM];
  double nbr_bound = 0.0;
#pragma unroll
  for (int q = 0; q < kM; q++) lk[q] = 0x7fffffff;
  if (it > 1) {
#pragma unroll
    for (int q = 0; q < kM; q++)
      if (gl + G * q < kNbr) lk[q] = P.nbr[(int64_t)s * kNbr + gl + G * q];
    nbr_bound = P.nbr_b[s];
  }
#pragma unroll
  for (int q = 0; q < (9 + G - 1) / G; q++)  // the nine moment rows M_E0 .. M_EE22 over the group
    if (gl + G * q < 9)
      asm volatile("prefetch.global.L1 [%0];" ::"l"(P.mom + (int64_t)(M_E0 + gl + G * q) * P.max_sv + s));
  const int f = R.frame;
  float4 lpos[kM];
#pragma unroll
  for (int q = 0; q < kM; q++) {
    lpos[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (it > 1 && gl + G * q < kNbr && lk[q] != 0x7fffffff) lpos[q] = P.kpos[lk[q]];
  }
  const FrameState& S = P.state[f];
  if (*(volatile const int32_t*)&S.done) return;
  const FrameDesc D = load_desc(P, f);
  const double psi_tot = S.psi_total[it & 1];  // loaded beside the frame's other scalars
  const int sl = s - D.sv_base;
  const int Sf = D.n_sv;
  const float q0 = R.c0, q1 = R.c1, q2 = R.c2;  // the frame's centroid of s, as the E-step reads it
  GridGeom g;
  for (int d = 0; d < 3; d++) {
    g.lo[d] = S.lo[d];
    g.dims[d] = S.dims[d];
  }
  g.h = S.h;
  g.inv_h = S.inv_h;
  const bool grid_ok = !(S.flags & F_CELL_OVERFLOW);
  const double disp = S.disp_cum;
  Top5 t;
  // After the first iteration: the supervoxel's neighbour list, the kNbr nearest Gaussians
  // when it was last searched (at displacement bound disp_b), member i on lane i mod G.  A
  // Gaussian outside the list was then at scaled distance >= rho from the centroid and has
  // since moved at most disp - disp_b, so the five nearest members (current centres, the
  // same FP32 distances and (distance, index) order) are the exact five nearest whenever
  //   sqrt(d5) (1 + 1e-6) + disp < nbr_b = rho (1 - 1e-6) - 4e-3 + disp_b;
  // the margins cover the FP32 rounding of the distances.  Otherwise the supervoxel runs
  // the exact search for the kNbr nearest and keeps them as its new list.
  float ld[kM];
  bool have = false;
#pragma unroll
  for (int q = 0; q < kM; q++) ld[q] = kInfF;
  if (it > 1) {
    Top5 mine;
    top5_init(mine);
#pragma unroll
    for (int q = 0; q < kM; q++) {
      if (gl + G * q < kNbr && lk[q] != 0x7fffffff)
        ld[q] = knn_dist(q0, q1, q2, lpos[q].x, lpos[q].y, lpos[q].z, D.scale);
      if (kM == 1) {
        mine.d[0] = ld[q];
        mine.i[0] = lk[q];
      } else {
        topn_insert<kJ>(mine, ld[q], lk[q]);
      }
    }
    group_merge_topn<G, kJ>(mine, t, gmask);
    have = t.d[kJ - 1] < kInfF && sqrt((double)t.d[kJ - 1]) * (1.0 + 1e-6) + disp < nbr_bound;
  }
  if (!have) {
    // starting bound: the kNbr-th of the list members at their current centres
    float td0 = kInfF;
    int ti0 = 0x7fffffff;
    if (it > 1) {
      float dj = -1.0f;  // lanes without a member never win the arg-max
      int ij = -1;
#pragma unroll
      for (int q = 0; q < kM; q++)
        if (gl + G * q < kNbr && before(dj, ij, ld[q], lk[q])) {
          dj = ld[q];
          ij = lk[q];
        }
      group_max_pair<G>(dj, ij, gmask);
      td0 = dj;
      ti0 = ij >= 0 && ij != 0x7fffffff ? ij - D.g_base : ij;  // the search's frame-local order
      if (gl == 0) atomicAdd(&P.state[f].knn_searches, 1);
    }
    TopN<kNbr> nb;
    topn_init<kNbr>(nb);
    if (grid_ok)
      knn_group_search<G, kNbr>(q0, q1, q2, D.scale, g, P.cell_cnt + D.cell_base,
                                P.cell_refs + (int64_t)D.cell_base * kCellCap, nb, gmask, gl, td0, ti0);
    if (!grid_ok || !(nb.d[kJ - 1] < kInfF)) {
      // fewer than five finite distances: exact scan of every Gaussian of the frame
      TopN<kNbr> m;
      topn_init<kNbr>(m);
      for (int kl = gl; kl < D.n_gauss; kl += G) {
        const int k = D.g_base + kl;
        const float x = __double2float_rn(gcomp(P, G_M0, k));
        const float y = __double2float_rn(gcomp(P, G_M1, k));
        const float z = __double2float_rn(gcomp(P, G_M2, k));
        topn_insert<kNbr>(m, knn_dist(q0, q1, q2, x, y, z, D.scale), kl);
      }
      group_merge_topn<G, kNbr>(m, nb, gmask);
    }
    // (frame-local indices from the search; global ones from here on)
#pragma unroll
    for (int j = 0; j < kJ; j++) {
      t.d[j] = nb.d[j];
      t.i[j] = nb.i[j] == 0x7fffffff ? nb.i[j] : D.g_base + nb.i[j];
    }
#pragma unroll
    for (int m = 0; m < kM; m++) {
      int mi = 0x7fffffff;
#pragma unroll
      for (int q = 0; q < kNbr; q++)
        if (gl + G * m == q) mi = nb.i[q];
      if (gl + G * m < kNbr) P.nbr[(int64_t)s * kNbr + gl + G * m] = mi == 0x7fffffff ? mi : D.g_base + mi;
    }
    if (gl == 0)
      P.nbr_b[s] = nb.d[kNbr - 1] < kInfF ? sqrt((double)nb.d[kNbr - 1]) * (1.0 - 1e-6) - 4e-3 + disp : (double)kInfF;
  }
  // E-step: candidate j = gl + G q on its lane (its voxel count: 0 for an invalid range, which
  // flags the frame)
  const double n = (double)R.nv;
  int kc[kC];
  double Lc[kC];
#pragma unroll
  for (int q = 0; q < kC; q++) {
    const int jj = gl + G * q;
    int k = 0;
#pragma unroll
    for (int j = 0; j < kJ; j++)
      if (jj == j) k = t.i[j];
    kc[q] = k;
    double Lj = 0.0;
    if (jj < kJ && n != 0.0) {
      const double* E = P.ec + (int64_t)k * kEcStride;
      const double2 e01 = *(const double2*)(E), e23 = *(const double2*)(E + 2), e45 = *(const double2*)(E + 4);
      const double2 e67 = *(const double2*)(E + 6), e89 = *(const double2*)(E + 8), e10 = *(const double2*)(E + 10);
      const double cst = e10.x;  // psi(alpha) + E[ln|Lambda|]/2, -inf when dead
      if (cst == -(double)kInfF) {
        Lj = -(double)kInfF;
      } else {
        double G1[3], G2[6];
#pragma unroll
        for (int i = 0; i < 3; i++) G1[i] = P.mom[(int64_t)(M_E0 + i) * P.max_sv + s];
#pragma unroll
        for (int i = 0; i < 6; i++) G2[i] = P.mom[(int64_t)(M_EE00 + i) * P.max_sv + s];
        const double u0 = e67.x - (double)q0, u1 = e67.y - (double)q1, u2 = e89.x - (double)q2;
        const double D00 = G2[0] - 2.0 * G1[0] * u0 + n * u0 * u0;
        const double D01 = G2[1] - (G1[0] * u1 + u0 * G1[1]) + n * u0 * u1;
        const double D02 = G2[2] - (G1[0] * u2 + u0 * G1[2]) + n * u0 * u2;
        const double D11 = G2[3] - 2.0 * G1[1] * u1 + n * u1 * u1;
        const double D12 = G2[4] - (G1[1] * u2 + u1 * G1[2]) + n * u1 * u2;
        const double D22 = G2[5] - 2.0 * G1[2] * u2 + n * u2 * u2;
        // nu * tr(W D) with nu*W from the record: W00 D00 + W11 D11 + W22 D22 + 2 (W01 D01 + W02 D02 + W12 D12)
        const double tr = e01.x * D00 + e23.y * D11 + e45.y * D22 + 2.0 * (e01.y * D01 + e23.x * D02 + e45.x * D12);
        Lj = -0.5 * (n * e89.y + tr) + n * (cst - psi_tot);
        if (Lj < -(double)FLT_MAX) Lj = -(double)kInfF;
        if (Lj > (double)FLT_MAX) Lj = (double)kInfF;
      }
    }
    Lc[q] = Lj;
  }
  // rnk_j = 1 / sum_i exp(L_i - L_j), the sum over i in increasing order
  double Li[kJ];
#pragma unroll
  for (int i = 0; i < kJ; i++) Li[i] = __shfl_sync(gmask, Lc[i / G], gbase + i % G);
#pragma unroll
  for (int q = 0; q < kC; q++) {
    const int j = gl + G * q;
    if (j < kJ) {
      const double Lj = Lc[q];
      const int k = kc[q];
      double acc = 0.0;
#pragma unroll
      for (int i = 0; i < kJ; i++) acc += exp(Li[i] - Lj);
      const float r = __double2float_rn(1.0 / acc);
      const int64_t pos = (int64_t)j * Sf + sl;
      cand_buf(P, it)[(int64_t)s * kJ + j] = k;
      rnk_buf(P, it)[(int64_t)s * kJ + j] = r;
      if ((double)r > 1e-3) {
        const int b = atomicAdd(&P.bcnt[k], 1);
        if (b < kBucketCap) P.bucket[(int64_t)k * kBucketCap + b] = (int)pos;
      }
    }
  }
}

template <int G>
__global__ void __launch_bounds__(kKnnWarps * 32, kKnnBlocks) k_knn_estep(DevPlan P) {
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1), gbase = lane - gl;
  const unsigned gmask = G == 32 ? 0xffffffffu : ((1u << G) - 1u) << gbase;
  const int s = blockIdx.x * (kKnnWarps * 32 / G) + (threadIdx.x >> 5) * (32 / G) + gbase / G;
  knn_estep_sv<G>(P, s, P.iter, gl, gbase, gmask);
}

// M-step contribution of one (supervoxel, slot) pair to Gaussian k, moments re-centred
// from the supervoxel centroid to m_ref, the Gaussian's prior mean m_o.  m_o stays fixed
// during a call, so responsibilities that repeat bit for bit give parameters that repeat
// bit for bit -- the exact fixed point the reference's tol = 0 stopping rule looks for:
//   A0 += r H0;  A1 += r (H1 + H0 d);  A2 += r (H2 + H1 d' + d H1' + H0 d d'),  d = c_s - m_ref.
// The inputs of one (supervoxel, slot) pair, loaded apart from their use so that the loads
// of several pairs can be in flight together.
struct MEntry {
  float r, c[3];
  double h0, h1[3], h2[6];
};

__device__ __forceinline__ MEntry mentry_load(const DevPlan& P, const FrameDesc& D, int p) {
  const int Sf = D.n_sv;
  const int j = p / Sf, sl = p - j * Sf;
  const int s = D.sv_base + sl;
  MEntry e;
  e.r = rnk_buf(P, P.iter)[(int64_t)s * kJ + j];
  e.c[0] = D.cent[sl];
  e.c[1] = D.cent[(int64_t)Sf + sl];
  e.c[2] = D.cent[2 * (int64_t)Sf + sl];
  e.h0 = P.mom[(int64_t)M_I * P.max_sv + s];
#pragma unroll
  for (int i = 0; i < 3; i++) e.h1[i] = P.mom[(int64_t)(M_IE0 + i) * P.max_sv + s];
#pragma unroll
  for (int i = 0; i < 6; i++) e.h2[i] = P.mom[(int64_t)(M_IEE00 + i) * P.max_sv + s];
  return e;
}

__device__ __forceinline__ void mentry_add(const MEntry& e, const double* mref, double* A) {
  const double r = (double)e.r;
  const double d0 = (double)e.c[0] - mref[0];
  const double d1 = (double)e.c[1] - mref[1];
  const double d2 = (double)e.c[2] - mref[2];
  const double h0 = e.h0;
  const double* h1 = e.h1;
  const double* h2 = e.h2;
  const double d[3] = {d0, d1, d2};
  A[0] += r * h0;
  A[1] += r * (h1[0] + h0 * d0);
  A[2] += r * (h1[1] + h0 * d1);
  A[3] += r * (h1[2] + h0 * d2);
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int e = 0; e < 6; e++)
    A[4 + e] += r * (h2[e] + h1[ia[e]] * d[ib[e]] + d[ia[e]] * h1[ib[e]] + h0 * d[ia[e]] * d[ib[e]]);
}

__device__ __forceinline__ void mstep_add(const DevPlan& P, const FrameDesc& D, int p, const double* mref,
                                          double* A) {
  mentry_add(mentry_load(P, D, p), mref, A);
}

// Block-cooperative ordered scan for Gaussians whose bucket overflowed: visit every
// position p = j*S + s of the frame in increasing order, keep those whose candidate is k
// and whose rnk exceeds `thr`; `visit(p)` is called by thread 0 in increasing p order.
template <typename F>
__device__ void ordered_scan(const DevPlan& P, const FrameDesc& D, int it, int k, double thr, int* sh_list,
                             int* sh_cnt, F visit) {
  const int32_t* cand = cand_buf(P, it);
  const float* rnk = rnk_buf(P, it);
  const int64_t total = (int64_t)kJ * D.n_sv;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t base = 0; base < total; base += blockDim.x) {
    const int64_t p = base + threadIdx.x;
    bool pred = false;
    if (p < total) {
      const int j = (int)(p / D.n_sv), sl = (int)(p - (int64_t)j * D.n_sv);
      const int64_t idx = (int64_t)(D.sv_base + sl) * kJ + j;
      pred = (cand[idx] == k) && ((double)rnk[idx] > thr);
    }
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (lane == 0) sh_cnt[w] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      int run = 0;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
        const int c = sh_cnt[i];
        sh_cnt[i] = run;
        run += c;
      }
      sh_cnt[blockDim.x >> 5] = run;
    }
    __syncthreads();
    if (pred) sh_list[sh_cnt[w] + __popc(m & ((1u << lane) - 1u))] = (int)p;
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < sh_cnt[blockDim.x >> 5]; i++) visit(sh_list[i]);
    __syncthreads();
  }
}

// ===========================================================================
// mstep_update: thread per Gaussian.  Sorted bucket -> FP64 sufficient statistics ->
// Dirichlet / Normal-Wishart update (GMEMupdateCUDA.cu:1601-1677) -> regularisation
// (:1693-1809).  Writes the chunk's alpha sum for the kill step.
// ===========================================================================
__global__ void __launch_bounds__(kMChunk) k_mstep_update(DevPlan P) {
  // two blocks per Gaussian chunk (twice the SMs busy): block b covers half b%2 of chunk b/2
  const int c = blockIdx.x >> 1, half = blockIdx.x & 1;
  if (c >= P.info->n_gchunks) return;
  const GChunk ch = P.gchunks[c];
  if (P.state[ch.frame].done) return;
  const FrameDesc D = load_desc(P, ch.frame);
  __shared__ int s_ovf[kMChunk];
  __shared__ int s_novf;
  __shared__ double s_ovf_acc[kMChunk][10];
  __shared__ int s_list[kMChunk];
  __shared__ int s_cnt[kMChunk / 32 + 1];
  __shared__ double shd[kMChunk / 32];
  __shared__ int s_bk[kBucketCap][kMChunk];  // each thread's bucket, one column per thread
  if (threadIdx.x == 0) s_novf = 0;
  __syncthreads();
  {
    // the grid of this frame was read by this iteration's kNN and is refilled by the kill
    // step: its 2*n_gchunks M-step blocks clear it
    const int nb = 2 * D.n_gchunks, rank = 2 * (c - D.gchunk_base) + half;
    const int ncell = P.state[ch.frame].n_cells;
    for (int i = rank * kMChunk + threadIdx.x; i < ncell; i += nb * kMChunk) P.cell_cnt[D.cell_base + i] = 0;
  }
  const int k = ch.g_begin + half * kMChunk + threadIdx.x;
  const bool valid = k < ch.g_end;
  double A[10];
#pragma unroll
  for (int i = 0; i < 10; i++) A[i] = 0.0;
  double mref[3] = {0, 0, 0};
  bool ovf = false;
  // the Gaussian's own inputs of the update, loaded ahead of the bucket work so that they
  // arrive beside it: the prior (m_o also re-centres the pairs), its fixed flag, this
  // iteration's E[ln|Lambda|] (the kill step's NaN test) and the centre the kNN saw
  const int cur = P.iter & 1, nxt = cur ^ 1;
  double bo = 0.0, nuo = 0.0, alo = 0.0, Wo[6] = {0, 0, 0, 0, 0, 0}, eld_cur = 0.0, alpha_old = 0.0;
  bool fixed_k = false;
  float4 kp_old = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (valid) {
    for (int d = 0; d < 3; d++) mref[d] = gcomp(P, G_MO0 + d, k);
    bo = gcomp(P, G_BETAO, k);
    nuo = gcomp(P, G_NUO, k);
    alo = gcomp(P, G_ALPHAO, k);
    for (int e = 0; e < 6; e++) Wo[e] = gcomp(P, G_WO0 + e, k);
    eld_cur = gcomp(P, G_ELD0 + cur, k);
    alpha_old = gcomp(P, G_ALPHA, k);
    fixed_k = P.fixed[k] != 0;
    kp_old = P.kpos[k];
    // the bucket's first eight entries load beside its count (entries past the count are
    // stale and unused; the bucket rows are 128-byte aligned)
    const int* bk = P.bucket + (int64_t)k * kBucketCap;
    const int4 b0 = *reinterpret_cast<const int4*>(bk), b1 = *reinterpret_cast<const int4*>(bk + 4);
    const int n = P.bcnt[k];
    P.bcnt[k] = 0;
    const int t = threadIdx.x;
    if (n > kBucketCap) {
      ovf = true;
      const int o = atomicAdd(&s_novf, 1);
      s_ovf[o] = threadIdx.x;
      atomicOr(&P.state[ch.frame].flags, F_BUCKET_OVERFLOW);
    } else if (n <= 8) {
      // up to eight positions (distinct, non-negative): sorted in registers by a 19-comparator
      // network, the unused slots padded with INT_MAX, then into shared memory
      int v[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (i >= n) v[i] = INT_MAX;
      constexpr int kNet[19][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {1, 2}, {5, 6},
                                   {0, 4}, {3, 7}, {1, 5}, {2, 6}, {1, 4}, {3, 6}, {2, 4}, {3, 5}, {3, 4}};
#pragma unroll
      for (int c2 = 0; c2 < 19; c2++) {
        const int lo = min(v[kNet[c2][0]], v[kNet[c2][1]]), hi = max(v[kNet[c2][0]], v[kNet[c2][1]]);
        v[kNet[c2][0]] = lo;
        v[kNet[c2][1]] = hi;
      }
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (i < n) s_bk[i][t] = v[i];
    } else {
      // this Gaussian's bucket into shared memory, sorted there by position
#pragma unroll 4
      for (int i = 0; i < n; i++) s_bk[i][t] = bk[i];
      for (int i = 1; i < n; i++) {
        const int v = s_bk[i][t];
        int q = i;
        while (q > 0 && s_bk[q - 1][t] > v) {
          s_bk[q][t] = s_bk[q - 1][t];
          q--;
        }
        s_bk[q][t] = v;
      }
    }
    if (!ovf) {
      // in that order, two pairs' inputs in flight at a time
      int i = 0;
      for (; i + 1 < n; i += 2) {
        const MEntry e0 = mentry_load(P, D, s_bk[i][t]);
        const MEntry e1 = mentry_load(P, D, s_bk[i + 1][t]);
        mentry_add(e0, mref, A);
        mentry_add(e1, mref, A);
      }
      if (i < n) mstep_add(P, D, s_bk[i][t], mref, A);
    }
  }
  __syncthreads();
  const int novf = s_novf;
  for (int o = 0; o < novf; o++) {
    const int tk = s_ovf[o];
    const int kk = ch.g_begin + half * kMChunk + tk;
    double mr[3] = {gcomp(P, G_MO0, kk), gcomp(P, G_MO1, kk), gcomp(P, G_MO2, kk)};
    double acc[10];
    for (int i = 0; i < 10; i++) acc[i] = 0.0;
    ordered_scan(P, D, P.iter, kk, 1e-3, s_list, s_cnt, [&](int p) { mstep_add(P, D, p, mr, acc); });
    if (threadIdx.x == 0)
      for (int i = 0; i < 10; i++) s_ovf_acc[tk][i] = acc[i];
    __syncthreads();
  }
  if (ovf)
    for (int i = 0; i < 10; i++) A[i] = s_ovf_acc[threadIdx.x][i];
  double alpha = 0.0, move = 0.0;
  // what the kill step tests: this Gaussian's alpha if it is live and not fixed, and whether
  // its W or this iteration's E[ln|Lambda|] holds a NaN
  double amin = kInf;
  bool nanw = false;
  if (valid) {
    const bool alive = !is_dead_prior(mref[0]) && !fixed_k;
    nanw = isnan(eld_cur);
    if (!alive)
      for (int e = 0; e < 6; e++) nanw = nanw || isnan(gcomp(P, G_W0 + e, k));
    if (alive) {
      const double N = A[0];
      double xb[3] = {0, 0, 0}, Sk[6] = {0, 0, 0, 0, 0, 0};
      if (N > 0.0) {
        const double iN = 1.0 / N;
        for (int d = 0; d < 3; d++) xb[d] = mref[d] + A[1 + d] * iN;
        const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
        for (int e = 0; e < 6; e++) Sk[e] = A[4 + e] - A[1 + ia[e]] * A[1 + ib[e]] * iN;
      }
      const double beta = bo + N;
      const double ib_ = 1.0 / beta;
      const double nu = nuo + N;
      const double alpha_n = fmax(alo + N, 0.0);
      gcomp(P, G_BETA, k) = beta;
      gcomp(P, G_NU, k) = nu;
      gcomp(P, G_ALPHA, k) = alpha_n;
      const double* mo = mref;
      double mn[3];
      for (int d = 0; d < 3; d++) {
        mn[d] = (bo * mo[d] + N * xb[d]) * ib_;
        gcomp(P, G_M0 + d, k) = mn[d];
      }
      if (Wo[5] < 1e-8) {
        Wo[5] = 0.5 * (Wo[0] + Wo[3]);
        gcomp(P, G_WO5, k) = Wo[5];
      }
      double Winv[6];
      inv3(Wo, Winv);
      const double dx[3] = {xb[0] - mo[0], xb[1] - mo[1], xb[2] - mo[2]};
      const double fct = N * (bo * ib_);
      const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
      for (int e = 0; e < 6; e++) Winv[e] += Sk[e] + fct * dx[ia[e]] * dx[ib[e]];
      double W[6];
      inv3(Winv, W);
      RegConst rc;
      for (int d = 0; d < 3; d++) rc.scale[d] = D.reg_scale[d];
      rc.w4dof = D.w4dof;
      rc.lambda_min = D.lambda_min;
      rc.lambda_max = D.lambda_max;
      rc.max_exc = D.max_exc;
      regularize_W(W, nu, rc);
      for (int e = 0; e < 6; e++) gcomp(P, G_W0 + e, k) = W[e];
      for (int e = 0; e < 6; e++) nanw = nanw || isnan(W[e]);
      amin = alpha_n;
      alpha = alpha_n;
      // the next iteration's records, as if the Gaussian survives the kill step (which
      // rewrites them for the Gaussians it kills)
      move = write_records(P, D, k, nxt, false, W, nu, alpha_n, beta, mn, true, kp_old);
    } else {
      // fixed or dead: unchanged parameters, unchanged records; psi and E[ln|Lambda|] go
      // on to the next iteration's slot
      gcomp(P, G_PSIA0 + nxt, k) = gcomp(P, G_PSIA0 + cur, k);
      gcomp(P, G_ELD0 + nxt, k) = eld_cur;
      alpha = alpha_old;
    }
  }
  const double a = block_sum_n<kMChunk>(alpha, shd);
  if (threadIdx.x == 0) P.alpha_part_e[blockIdx.x] = a;
  {
    __shared__ double s_amin[kMChunk / 32];
    __shared__ int s_nan[kMChunk / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, o));
    const int wn = __any_sync(0xffffffffu, nanw) ? 1 : 0;
    if ((threadIdx.x & 31) == 0) {
      s_amin[threadIdx.x >> 5] = amin;
      s_nan[threadIdx.x >> 5] = wn;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = kInf;
      int nn = 0;
      for (int i = 0; i < kMChunk / 32; i++) {
        m = fmin(m, s_amin[i]);
        nn |= s_nan[i];
      }
      P.alpha_min_e[blockIdx.x] = m;
      P.nan_e[blockIdx.x] = nn;
    }
  }
  // the block's largest move of a kNN centre, rounded up to a float (non-negative floats
  // order as their bits)
  float mv = __double2float_ru(move);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mv = fmaxf(mv, __shfl_xor_sync(0xffffffffu, mv, o));
  if ((threadIdx.x & 31) == 0 && mv > 0.0f) atomicMax(&P.state[ch.frame].disp_max, __float_as_uint(mv));
}

// ===========================================================================
// kill_prep: dead-Gaussian rule (GMEMcheckDeadCellsKernel, GMEMupdateCUDA.cu:1813-1843)
// with the post-update alpha total, then the preparation of the next iteration.
// ===========================================================================
__global__ void __launch_bounds__(kGChunk) k_kill_prep(DevPlan P) {
  const int c = blockIdx.x;
  if (c >= P.info->n_gchunks) return;
  const GChunk ch = P.gchunks[c];
  const FrameState& S = P.state[ch.frame];
  if (S.done) return;
  const FrameDesc D = load_desc(P, ch.frame);
  __shared__ double s_total;
  __shared__ double shd[kGChunk / 32];
  __shared__ int shi[kGChunk / 32];
  const int cur = P.iter & 1, nxt = cur ^ 1;
  const int k = ch.g_begin + threadIdx.x;
  const bool valid = k < ch.g_end;
  // this Gaussian's inputs are on their way while warp 0 sums the frame's alpha partials
  bool nanw = false, was_dead = true, fixed = true;
  double a = 0.0;
  float4 centre = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (valid) {
    centre = P.kpos[k];
    nanw = isnan(gcomp(P, G_ELD0 + cur, k));
    for (int e = 0; e < 6; e++) nanw = nanw || isnan(gcomp(P, G_W0 + e, k));
    a = gcomp(P, G_ALPHA, k);
    was_dead = is_dead_prior(gcomp(P, G_MO0, k));
    fixed = P.fixed[k] != 0;
  }
  __shared__ int s_fast;
  int cell = -1;
  {
    // the frame's M-step block partials, spread over the whole block so that their loads are
    // in flight together: the alpha total (a fixed order: each thread's partials in order, a
    // butterfly per warp, the warps in order -- the same bits in every block of the frame),
    // the smallest live alpha and the NaN flags.  No Gaussian of the frame can die this
    // iteration when none has a NaN and the smallest live alpha passes the rule.
    __shared__ double s_wt[kGChunk / 32], s_wm[kGChunk / 32];
    __shared__ int s_wn[kGChunk / 32];
    const int nb = 2 * D.n_gchunks, base = 2 * D.gchunk_base;
    double tp = 0.0, mp = kInf;
    int np = 0;
    for (int i = threadIdx.x; i < nb; i += kGChunk) {
      tp += P.alpha_part_e[base + i];
      mp = fmin(mp, P.alpha_min_e[base + i]);
      np |= P.nan_e[base + i];
    }
    tp = warp_sum(tp);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mp = fmin(mp, __shfl_xor_sync(0xffffffffu, mp, o));
    np = __any_sync(0xffffffffu, np != 0);
    // the grid cell of a live centre, from the frame's grid geometry, ahead of the barrier
    if (valid && !was_dead) cell = ref_cell_of(S, D, centre.x, centre.y, centre.z);
    if ((threadIdx.x & 31) == 0) {
      s_wt[threadIdx.x >> 5] = tp;
      s_wm[threadIdx.x >> 5] = mp;
      s_wn[threadIdx.x >> 5] = np;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0.0, amin = kInf;
      int nn = 0;
#pragma unroll
      for (int w = 0; w < kGChunk / 32; w++) {
        tot += s_wt[w];
        amin = fmin(amin, s_wm[w]);
        nn |= s_wn[w];
      }
      s_total = tot;
      s_fast = !nn && !(amin / tot < TGMM_MIN_PI_FOR_DEAD);
    }
  }
  __syncthreads();
  const double total = s_total;
  if (s_fast) {
    // nothing dies: the live Gaussians go into the grid, and the frame's first chunk writes
    // its totals (the post-kill total is the M-step's; the dead count stays)
    if (valid && !was_dead) grid_insert_at(P, D, cell, k, centre);
    if (c == D.gchunk_base && threadIdx.x == 0) {
      FrameState* Sw = &P.state[ch.frame];
      Sw->total_alpha = total;
      Sw->ln_alpha = log(total);
      Sw->psi_total[nxt] = digamma(total);
      Sw->blk_done = 0;
      Sw->disp_cum += (double)__uint_as_float(Sw->disp_max);
      Sw->disp_max = 0u;
    }
    return;
  }
  double alpha = 0.0;
  int dead = 0;
  if (valid) {
    if (nanw || (a / total < TGMM_MIN_PI_FOR_DEAD && !was_dead && !fixed)) {
      gcomp(P, G_ALPHA, k) = 0.0;
      const double mdead[3] = {-1e32, -1e32, -1e32};
      for (int d = 0; d < 3; d++) {
        gcomp(P, G_MO0 + d, k) = -1e32;
        gcomp(P, G_M0 + d, k) = -1e32;
      }
      const double I6[6] = {1, 0, 0, 1, 0, 1};
      for (int e = 0; e < 6; e++) gcomp(P, G_W0 + e, k) = I6[e];
      write_records(P, D, k, nxt, true, I6, gcomp(P, G_NU, k), 0.0, gcomp(P, G_BETA, k), mdead, false);
      dead = 1;
    } else {
      alpha = a;
      dead = was_dead ? 1 : 0;
      if (!was_dead) grid_insert_at(P, D, cell, k, centre);
    }
  }
  chunk_partials(alpha, dead, shd, shi, P.alpha_part_f, P.dead_part, c);
  chunk_done(P, ch.frame, D.n_gchunks, nxt);
}

// ===========================================================================
// ll_pass: the per-iteration voxel stream.  Warp per supervoxel:
//   ll_v = ln sum_j (alpha_j/A) sqrt(det(W_j) nu_j^3) (2 pi)^-3/2 exp(-nu_j d'W_j d / 2)
// over the supervoxel's five candidates (GMEMcomputeLikelihoodKernelWithSupervoxels,
// GMEMupdateCUDA.cu:1913-1978), I_v * ll_v summed when the density is positive.  Two
// sums: every voxel (true) and the reference's per-thread overwrite for supervoxels
// above 1024 voxels (as reference).
// Voxels are centred at the supervoxel centroid c (e = x - c is exact in FP32 for voxels
// near c) and candidate j enters through u_j = m_j - c, formed in FP64 and rounded once.
// With a_j = ln weight_j - nu_j d'W_j d/2 (d = e - u_j) each voxel's term
//   ll_v = a_max + ln sum_j exp(a_j - a_max)
// is evaluated in FP32, the five candidates in packed FP32x2 pairs (absolute error of a
// term about 1e-6); a lane adds its voxels of a tile in FP32 and the tile sums in FP64.
// The FP64 mode evaluates every component in FP64 with the reference's formula.
// Voxel tiles reach shared memory through TMA bulk copies (cp.async.bulk, one per
// component and tile, issued by one lane) that complete on a per-slot mbarrier:
// kLLStages tiles of kLLTile voxels are in flight per warp while it computes.  A copy
// covers the 16-byte aligned span around its tile and the lanes index it from the
// component's offset.
// Per-supervoxel results are added into per-frame 64-bit integer accumulators (integer
// part and 2^-40 fraction), so the frame total does not depend on the order in which
// warps finish; the warp that finishes a frame's last supervoxel runs the reference's
// convergence test for that frame.
// ===========================================================================
constexpr float kL2E = 1.4426950408889634f;  // log2(e)
constexpr float kLN2F = 0.6931471805599453f;
constexpr double kFracScale = 1099511627776.0;  // 2^40

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// FP32 constants of the five candidates: two packed pairs and one single.
struct CandF {
  float2 u[2][3];
  float2 A[2][6];
  float2 b[2];
  float u4[3], A4[6], b4;
};

// The candidates' constants from shared memory into a register copy; the 4-DOF form leaves the
// W02 and W12 entries (zero there) out, so that they are not kept live.
template <bool kW4>
__device__ __forceinline__ CandF load_cand(const CandF& S) {
  CandF C;
#pragma unroll
  for (int q = 0; q < 2; q++) {
#pragma unroll
    for (int d = 0; d < 3; d++) C.u[q][d] = S.u[q][d];
#pragma unroll
    for (int e = 0; e < 6; e++) C.A[q][e] = (kW4 && (e == 2 || e == 4)) ? make_float2(0.0f, 0.0f) : S.A[q][e];
    C.b[q] = S.b[q];
  }
#pragma unroll
  for (int d = 0; d < 3; d++) C.u4[d] = S.u4[d];
#pragma unroll
  for (int e = 0; e < 6; e++) C.A4[e] = (kW4 && (e == 2 || e == 4)) ? 0.0f : S.A4[e];
  C.b4 = S.b4;
  return C;
}

template <bool kW4>
__device__ __forceinline__ float2 eval_pair(const CandF& C, int q, float2 E0, float2 E1, float2 E2) {
  const float2 d0 = __fadd2_rn(E0, C.u[q][0]);  // u stored negated
  const float2 d1 = __fadd2_rn(E1, C.u[q][1]);
  const float2 d2 = __fadd2_rn(E2, C.u[q][2]);
  const float2* A = C.A[q];
  if (kW4) {
    const float2 t0 = __ffma2_rn(A[1], d1, __fmul2_rn(A[0], d0));
    return __ffma2_rn(d0, t0, __ffma2_rn(d1, __fmul2_rn(A[3], d1), __ffma2_rn(d2, __fmul2_rn(A[5], d2), C.b[q])));
  } else {
    const float2 t0 = __ffma2_rn(A[0], d0, __ffma2_rn(A[1], d1, __fmul2_rn(A[2], d2)));
    const float2 t1 = __ffma2_rn(A[3], d1, __fmul2_rn(A[4], d2));
    return __ffma2_rn(d0, t0, __ffma2_rn(d1, t1, __ffma2_rn(d2, __fmul2_rn(A[5], d2), C.b[q])));
  }
}

template <bool kW4>
__device__ __forceinline__ float eval_single(const CandF& C, float e0, float e1, float e2) {
  const float d0 = e0 + C.u4[0], d1 = e1 + C.u4[1], d2 = e2 + C.u4[2];
  const float* A = C.A4;
  if (kW4) {
    const float t0 = fmaf(A[1], d1, A[0] * d0);
    return fmaf(d0, t0, fmaf(d1, A[3] * d1, fmaf(d2, A[5] * d2, C.b4)));
  } else {
    const float t0 = fmaf(A[0], d0, fmaf(A[1], d1, A[2] * d2));
    const float t1 = fmaf(A[3], d1, A[4] * d2);
    return fmaf(d0, t0, fmaf(d1, t1, fmaf(d2, A[5] * d2, C.b4)));
  }
}

// max of three (one instruction on sm_100; the NaN rule of fmaxf: a NaN operand is ignored)
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

template <bool kW4>
__device__ __forceinline__ float voxel_ll_f32(const CandF& C, float e0, float e1, float e2) {
  const float2 E0 = make_float2(e0, e0), E1 = make_float2(e1, e1), E2 = make_float2(e2, e2);
  const float2 a01 = eval_pair<kW4>(C, 0, E0, E1, E2);
  const float2 a23 = eval_pair<kW4>(C, 1, E0, E1, E2);
  const float a4 = eval_single<kW4>(C, e0, e1, e2);
  const float am = fmax3(fmax3(a01.x, a01.y, a23.x), a23.y, a4);
  const float nm = -am * kL2E;
  const float2 t01 = __ffma2_rn(a01, make_float2(kL2E, kL2E), make_float2(nm, nm));
  const float2 t23 = __ffma2_rn(a23, make_float2(kL2E, kL2E), make_float2(nm, nm));
  const float s = (ex2_approx(t01.x) + ex2_approx(t01.y)) + (ex2_approx(t23.x) + ex2_approx(t23.y)) +
                  ex2_approx(fmaf(a4, kL2E, nm));
  return fmaf(lg2_approx(s), kLN2F, am);
}

// FP64 verification mode: the reference's formula, every component in FP64.
struct LLShared64 {
  double u[kJ][3];
  double A[kJ][6];  // nu * W
  double w[kJ];     // c_j * alpha_j / A
};

__device__ __forceinline__ double voxel_ll_fp64(const LLShared64& C, float x0, float x1, float x2, float c0, float c1,
                                                float c2, bool& ok) {
  const double e0 = (double)x0 - (double)c0, e1 = (double)x1 - (double)c1, e2 = (double)x2 - (double)c2;
  double dens = 0.0;
#pragma unroll
  for (int j = 0; j < kJ; j++) {
    const double d0 = e0 - C.u[j][0], d1 = e1 - C.u[j][1], d2 = e2 - C.u[j][2];
    const double* A = C.A[j];
    const double q = A[0] * d0 * d0 + A[3] * d1 * d1 + A[5] * d2 * d2 + 2.0 * A[1] * d0 * d1 +
                     2.0 * A[2] * d0 * d2 + 2.0 * A[4] * d1 * d2;
    dens += C.w[j] * exp(-0.5 * q);
  }
  ok = dens > 0.0;
  return ok ? log(dens) : 0.0;
}

// --- TMA bulk staging --------------------------------------------------------
#ifndef TGMM_LL_STAGES
#define TGMM_LL_STAGES 3
#endif
#ifndef TGMM_LL_BLOCKS
#define TGMM_LL_BLOCKS 2
#endif
#ifndef TGMM_LL_WARPS
#define TGMM_LL_WARPS 8
#endif
constexpr int kLLWarps = TGMM_LL_WARPS;       // warps per block of the voxel pass
constexpr int kLLTile = kVoxTile;             // voxels per tile (kVoxTile / 32 per lane)
constexpr int kLLStages = TGMM_LL_STAGES;     // tile slots per warp
constexpr int kLLBlocks = TGMM_LL_BLOCKS;     // resident blocks per SM the pass is compiled for
constexpr int kLLSpan = kLLTile + 4;          // floats per component in a slot (16-byte slack)
constexpr int kLLSlotFloats = 4 * kLLSpan;    // x, y, z, I
constexpr unsigned long long kLLWaitNs = 1000000000ull;  // default wait limit of a slot, and the drain's bound

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_test_wait(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
// Waits for the phase with the given parity; false after limit_ns without it.  try_wait
// suspends the thread for a while until the phase completes, so at the default limit the
// clock is read only between its returns; a limit below 1 ms polls with the non-blocking
// test_wait, so that the limit is kept to the clock's resolution.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned long long limit_ns) {
  if (limit_ns < 1000000ull) {
    if (mbar_test_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_test_wait(bar, parity))
      if (global_ns() - t0 > limit_ns) return false;
    return true;
  }
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
// Global -> shared bulk copy (non-multicast) completing on the mbarrier at `bar`.
__device__ __forceinline__ void bulk_g2s(unsigned dst, unsigned long long src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Small global -> shared copies (cp.async) for the look-ahead records.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Tile t of a supervoxel (SvRec): one bulk copy per component of the 16-byte chunks
// holding its voxels.  Every chunk copied holds a voxel of the tile, so no byte outside
// its array's pages is read.
__device__ __forceinline__ void ll_issue(const SvRec& R, int t, float* slot, unsigned bar) {
  unsigned n[4], total = 0;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    n[c] = t == 0 ? R.n0[c] : (R.nf[c] & 0xffffu);
    total += n[c];
  }
  mbar_expect_tx(bar, total);
#pragma unroll
  for (int c = 0; c < 4; c++)
    bulk_g2s(smem_addr(slot + c * kLLSpan),
             t == 0 ? R.lo0[c] : R.lo1[c] + (unsigned long long)(4 * kLLTile) * (unsigned)(t - 1), n[c], bar);
}

// Look-ahead records, fetched with cp.async ahead of use: a supervoxel's stream record and
// candidate ids (stage A, two supervoxels ahead) and its candidates' constants (10
// doubles each) with its frame's ln(sum alpha) and done flag (stage B, one ahead).
struct LLRec {
  SvRec rec;  // the moment pass and the FP64 pass: the SoA spans of the input arrays
  SvLL ll;    // the moment pass and the FP32 pass: the place in the centred voxel stream
  int32_t cand[8];
};
struct LLConst {
  double llc[kJ][10];
  double ln_alpha;
  int32_t done, pad;
};
static_assert(sizeof(LLRec) % 16 == 0 && sizeof(LLConst) % 16 == 0, "look-ahead records stay 16-byte aligned");

// Per-warp shared region: slots, one mbarrier per slot, three stage-A and two stage-B
// records, and the current supervoxel's FP32 candidate constants.
constexpr int kLLBarOff = kLLStages * kLLSlotFloats * 4;
constexpr int kLLRecOff = (kLLBarOff + kLLStages * 8 + 15) / 16 * 16;
constexpr int kLLConstOff = kLLRecOff + 3 * (int)sizeof(LLRec);
constexpr int kLLCandOff = kLLConstOff + 2 * (int)sizeof(LLConst);
constexpr int kLLWarpBytes = (kLLCandOff + (int)sizeof(CandF) + 15) / 16 * 16;
constexpr size_t kLLSmemBytes = (size_t)kLLWarpBytes * kLLWarps;
static_assert((kLLSlotFloats * 4) % 16 == 0 && kLLRecOff % 16 == 0 && kLLConstOff % 16 == 0 && kLLCandOff % 16 == 0,
              "slots and records stay 16-byte aligned");
// the FP32 forms keep kLLBlocks blocks on an SM (228 KB of shared memory, 1 KB reserved per
// block, the FP32 forms' one static LLShared64); the FP64 form sizes its own grid
static_assert(kLLBlocks * (kLLSmemBytes + 1024 + sizeof(LLShared64)) <= 233472, "the voxel pass's blocks fit an SM");

// Stage A: the records (SoA spans: kRec; centred-stream place: kLL) and candidate ids
// (kCand) of supervoxel s, one lane per 16-byte chunk or id.
template <bool kRec, bool kLL, bool kCand>
__device__ __forceinline__ void ll_fetch_a(const DevPlan& P, LLRec& X, int s) {
  const int lane = threadIdx.x & 31;
  constexpr int kRecChunks = kRec ? (int)sizeof(SvRec) / 16 : 0;
  constexpr int kLLChunks = kLL ? (int)sizeof(SvLL) / 16 : 0;
  static_assert(kRecChunks + kLLChunks + kJ <= 32, "one lane per chunk");
  if (lane < kRecChunks) {
    cp_async16(reinterpret_cast<char*>(&X.rec) + 16 * lane, reinterpret_cast<const char*>(P.sv_rec + s) + 16 * lane);
  } else if (lane < kRecChunks + kLLChunks) {
    const int c = lane - kRecChunks;
    cp_async16(reinterpret_cast<char*>(&X.ll) + 16 * c, reinterpret_cast<const char*>(P.sv_ll + s) + 16 * c);
  } else if (kCand && lane < kRecChunks + kLLChunks + kJ) {
    const int j = lane - kRecChunks - kLLChunks;
    cp_async4(&X.cand[j], cand_buf(P, P.iter) + (int64_t)s * kJ + j);
  }
}
// Stage B (after A landed): the candidates' constants and the frame scalars.
__device__ __forceinline__ void ll_fetch_b(const DevPlan& P, const LLRec& A, int frame, LLConst& X) {
  const int lane = threadIdx.x & 31;
  if (lane < 5 * kJ) {
    const int j = lane / 5, c = lane % 5;
    cp_async16(&X.llc[j][2 * c], P.llc + (int64_t)A.cand[j] * 10 + 2 * c);
  } else if (lane == 5 * kJ) {
    cp_async8(&X.ln_alpha, &P.state[frame].ln_alpha);
  } else if (lane == 5 * kJ + 1) {
    cp_async4(&X.done, &P.state[frame].done);
  }
}

// Tile t of a supervoxel from the centred voxel stream: one bulk copy of its float4 voxels
// (16 bytes each, so every tile starts and ends on a 16-byte boundary).
__device__ __forceinline__ void ll_issue4(const float4* vox4, const SvLL& R, int t, float* slot, unsigned bar) {
  const int off = t == 0 ? 0 : R.r0 + kLLTile * (t - 1);
  const unsigned bytes = 16u * (unsigned)(t == 0 ? R.r0 : kLLTile);
  mbar_expect_tx(bar, bytes);
  bulk_g2s(smem_addr(slot), (unsigned long long)(vox4 + R.v0 + off), bytes, bar);
}

// Evaluation of one voxel in the three modes: 0 FP32 4-DOF, 1 FP32 general, 2 FP64.
template <int kMode>
struct VoxelEval {
  using T = float;
  const CandF& C;
  __device__ __forceinline__ float operator()(float x, float y, float z, float c0, float c1, float c2) const {
    return voxel_ll_f32<kMode == 0>(C, x - c0, y - c1, z - c2);
  }
  // from e = x - c as the moment pass stored it (the same FP32 value as x - c0 above)
  __device__ __forceinline__ float e(float e0, float e1, float e2) const { return voxel_ll_f32<kMode == 0>(C, e0, e1, e2); }
  __device__ __forceinline__ static bool ok(float l) { return l > -745.13f; }  // exp(l) is a positive double
};
template <>
struct VoxelEval<2> {
  using T = double;
  const LLShared64& C;
  __device__ __forceinline__ double operator()(float x, float y, float z, float c0, float c1, float c2) const {
    bool ok;
    const double l = voxel_ll_fp64(C, x, y, z, c0, c1, c2, ok);
    return ok ? l : -kInf;
  }
  __device__ __forceinline__ static bool ok(double l) { return l > -kInf; }
};

// One staged tile: lane voxels o = u*32 + lane, sht[c] the offset of component c in the
// slot.  kFull: all kLLTile voxels present (else the first rem).  allok turns false when
// a present voxel has a zero density.
template <class Eval, bool kFull>
__device__ __forceinline__ void ll_tile(const Eval& eval, const float* __restrict__ slot, const int* sht, int rem,
                                        float c0, float c1, float c2, typename Eval::T& tsum, bool& allok) {
  using T = typename Eval::T;
  const int lane = threadIdx.x & 31;
  const float* bx = slot + sht[0] + lane;
  const float* by = slot + kLLSpan + sht[1] + lane;
  const float* bz = slot + 2 * kLLSpan + sht[2] + lane;
  const float* bi = slot + 3 * kLLSpan + sht[3] + lane;
#pragma unroll
  for (int u = 0; u < kLLTile / 32; u++) {
    if (!kFull && u * 32 >= rem) break;
    const T l = eval(bx[32 * u], by[32 * u], bz[32 * u], c0, c1, c2);
    const bool ok = Eval::ok(l);
    const bool in = kFull || u * 32 + lane < rem;
    allok = allok && (ok || !in);
    tsum += (in && ok) ? (T)bi[32 * u] * l : (T)0;
  }
}

// The same tile from the centred voxel stream: lane voxels o = u*32 + lane, each one float4
// (e0, e1, e2, I) read with one shared-memory load.
template <class Eval, bool kFull>
__device__ __forceinline__ void ll_tile4(const Eval& eval, const float4* __restrict__ slot, int rem, float& tsum,
                                         bool& allok) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int u = 0; u < kLLTile / 32; u++) {
    if (!kFull && u * 32 >= rem) break;
    const float4 v = slot[32 * u + lane];
    const float l = eval.e(v.x, v.y, v.z);
    const bool ok = Eval::ok(l);
    const bool in = kFull || u * 32 + lane < rem;
    allok = allok && (ok || !in);
    tsum += (in && ok) ? v.w * l : 0.0f;
  }
}

// A kept voxel (one of the last 1024 of a supervoxel above 1024 voxels) with a zero
// density: the reference thread of its stride still holds the last voxel of the stride
// with a positive density (GMEMupdateCUDA.cu:1961-1962).  Rare; reads global memory.
template <class Eval>
__device__ __forceinline__ double ll_walk_back(const Eval& eval, const SvRec& R, int i, float c0, float c1, float c2) {
  const float* v[4];
#pragma unroll
  for (int c = 0; c < 4; c++) v[c] = reinterpret_cast<const float*>(R.lo0[c]) + ((R.nf[c] >> 16) & 3);
  for (int i2 = i - 1024; i2 >= 0; i2 -= 1024) {
    const typename Eval::T l2 = eval(v[0][i2], v[1][i2], v[2][i2], c0, c1, c2);
    if (Eval::ok(l2)) return (double)v[3][i2] * (double)l2;
  }
  return 0.0;
}

// The kept tiles (bit t - (nt - kKeptTiles) of `mask`) that hold voxels of zero density, after the
// supervoxel's tiles: their voxels are read again from global memory and each one of zero
// density adds the walk-back value.  Rare.
template <class Eval>
__device__ __forceinline__ double ll_fixup(const Eval& eval, const SvRec& R, unsigned mask, float c0, float c1,
                                           float c2) {
  const int lane = threadIdx.x & 31;
  const float* v[4];
#pragma unroll
  for (int c = 0; c < 4; c++) v[c] = reinterpret_cast<const float*>(R.lo0[c]) + ((R.nf[c] >> 16) & 3);
  double add = 0.0;
  for (int k = 0; k < kKeptTiles; k++) {
    if (!(mask & (1u << k))) continue;
    const int t = R.ntiles - kKeptTiles + k;
    const int start = t == 0 ? 0 : R.r0 + (t - 1) * kLLTile;
    const int rem = t == 0 ? R.r0 : kLLTile;
    for (int o = lane; o < rem; o += 32) {
      const int i = start + o;
      const typename Eval::T l = eval(v[0][i], v[1][i], v[2][i], c0, c1, c2);
      if (!Eval::ok(l)) add += ll_walk_back(eval, R, i, c0, c1, c2);
    }
  }
  return add;
}

// The centred-stream forms of ll_walk_back and ll_fixup: v = the supervoxel's voxels in vox4.
template <class Eval>
__device__ __forceinline__ double ll_walk_back4(const Eval& eval, const float4* v, int i) {
  for (int i2 = i - 1024; i2 >= 0; i2 -= 1024) {
    const float4 x = v[i2];
    const float l2 = eval.e(x.x, x.y, x.z);
    if (Eval::ok(l2)) return (double)x.w * (double)l2;
  }
  return 0.0;
}

template <class Eval>
__device__ __forceinline__ double ll_fixup4(const Eval& eval, const float4* v, int nt, int r0, unsigned mask) {
  const int lane = threadIdx.x & 31;
  double add = 0.0;
  for (int k = 0; k < kKeptTiles; k++) {
    if (!(mask & (1u << k))) continue;
    const int t = nt - kKeptTiles + k;
    const int start = t == 0 ? 0 : r0 + (t - 1) * kLLTile;
    const int rem = t == 0 ? r0 : kLLTile;
    for (int o = lane; o < rem; o += 32) {
      const int i = start + o;
      const float4 x = v[i];
      if (!Eval::ok(eval.e(x.x, x.y, x.z))) add += ll_walk_back4(eval, v, i);
    }
  }
  return add;
}

// The moment pass's tile t (landed in `slot`): the 19 sums e, ee', I, Ie, Iee' (e = x - c in
// FP32, FP64 accumulation) of the lane's voxels o = u*32 + lane, each voxel also written to
// the centred voxel stream (out: the tile's first voxel there) as (e0, e1, e2, I); nan_seen
// turns true on a NaN coordinate or intensity.
template <bool kFull>
__device__ __forceinline__ void mom_tile(const float* __restrict__ slot, const int* sht, int rem, float c0, float c1,
                                         float c2, double* m, bool& nan_seen, float4* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const float* bx = slot + sht[0] + lane;
  const float* by = slot + kLLSpan + sht[1] + lane;
  const float* bz = slot + 2 * kLLSpan + sht[2] + lane;
  const float* bi = slot + 3 * kLLSpan + sht[3] + lane;
#pragma unroll
  for (int u = 0; u < kLLTile / 32; u++) {
    if (!kFull && u * 32 >= rem) break;
    if (!kFull && u * 32 + lane >= rem) continue;
    const float x = bx[32 * u], y = by[32 * u], z = bz[32 * u], I = bi[32 * u];
    nan_seen |= isnan(x) || isnan(y) || isnan(z) || isnan(I);
    const float e0f = x - c0, e1f = y - c1, e2f = z - c2;
    out[32 * u + lane] = make_float4(e0f, e1f, e2f, I);
    const double e0 = (double)e0f, e1 = (double)e1f, e2 = (double)e2f;
    const double wI = (double)I;
    m[M_E0] += e0;
    m[M_E1] += e1;
    m[M_E2] += e2;
    m[M_EE00] = fma(e0, e0, m[M_EE00]);
    m[M_EE01] = fma(e0, e1, m[M_EE01]);
    m[M_EE02] = fma(e0, e2, m[M_EE02]);
    m[M_EE11] = fma(e1, e1, m[M_EE11]);
    m[M_EE12] = fma(e1, e2, m[M_EE12]);
    m[M_EE22] = fma(e2, e2, m[M_EE22]);
    m[M_I] += wI;
    const double i0 = wI * e0, i1 = wI * e1, i2 = wI * e2;
    m[M_IE0] += i0;
    m[M_IE1] += i1;
    m[M_IE2] += i2;
    m[M_IEE00] = fma(i0, e0, m[M_IEE00]);
    m[M_IEE01] = fma(i0, e1, m[M_IEE01]);
    m[M_IEE02] = fma(i0, e2, m[M_IEE02]);
    m[M_IEE11] = fma(i1, e1, m[M_IEE11]);
    m[M_IEE12] = fma(i1, e2, m[M_IEE12]);
    m[M_IEE22] = fma(i2, e2, m[M_IEE22]);
  }
}

__device__ __forceinline__ void mom_consume(const float* slot, const int* pk, int t, int r0, float c0, float c1,
                                            float c2, double* m, bool& nan_seen, float4* sv_out) {
  const int sft = t == 0 ? 0 : 4;
  const int sht[4] = {(pk[0] >> sft) & 3, (pk[1] >> sft) & 3, (pk[2] >> sft) & 3, (pk[3] >> sft) & 3};
  const int rem = t == 0 ? r0 : kLLTile;
  float4* out = sv_out + (t == 0 ? 0 : r0 + kLLTile * (t - 1));
  if (rem == kLLTile)
    mom_tile<true>(slot, sht, rem, c0, c1, c2, m, nan_seen, out);
  else
    mom_tile<false>(slot, sht, rem, c0, c1, c2, m, nan_seen, out);
}

// Tile t (landed in `slot`) of the current supervoxel: its sum goes to lt, and to lr when
// the tile is one of the last kKeptTiles (the reference's kept window of 1024 voxels).  A kept
// tile of a supervoxel above 1024 voxels with a voxel of zero density is marked in fix.
template <class Eval>
__device__ __forceinline__ void ll_consume(const Eval& eval, const float* slot, const int* pk, int t, int nt, int nv,
                                           int r0, float c0, float c1, float c2, double& lt, double& lr,
                                           unsigned& fix) {
  using T = typename Eval::T;
  const int sft = t == 0 ? 0 : 4;
  const int sht[4] = {(pk[0] >> sft) & 3, (pk[1] >> sft) & 3, (pk[2] >> sft) & 3, (pk[3] >> sft) & 3};
  const int rem = t == 0 ? r0 : kLLTile;
  T tsum = (T)0;
  bool allok = true;
  if (rem == kLLTile)
    ll_tile<Eval, true>(eval, slot, sht, rem, c0, c1, c2, tsum, allok);
  else
    ll_tile<Eval, false>(eval, slot, sht, rem, c0, c1, c2, tsum, allok);
  lt += (double)tsum;
  if (t >= nt - kKeptTiles) {
    lr += (double)tsum;
    if (nv > 1024 && __any_sync(0xffffffffu, !allok)) fix |= 1u << (t - (nt - kKeptTiles));
  }
}

// A full tile without the per-voxel zero-density test: every voxel's term is added and the
// smallest term kept; a density is zero (the reference skips such a voxel) only when a term
// is at or below ln of the smallest double (-745.13) or NaN, and then -- rarely -- the tile
// is evaluated again with the per-voxel test.
template <class Eval>
__device__ __forceinline__ void ll_tile4_full(const Eval& eval, const float4* __restrict__ slot, float& tsum,
                                              bool& allok) {
  const int lane = threadIdx.x & 31;
  float s = 0.0f, lmin = kInfF;
#pragma unroll
  for (int u = 0; u < kLLTile / 32; u++) {
    const float4 v = slot[32 * u + lane];
    const float l = eval.e(v.x, v.y, v.z);
    lmin = fminf(lmin, l);
    s = fmaf(v.w, l, s);
  }
  if (__any_sync(0xffffffffu, !(lmin > -745.13f) || isnan(s))) {
    float t = 0.0f;
    bool ok = true;
    ll_tile4<Eval, true>(eval, slot, kLLTile, t, ok);
    tsum += t;
    allok = allok && ok;
  } else {
    tsum += s;
  }
}

// The centred-stream form of ll_consume (FP32 terms).
template <class Eval>
__device__ __forceinline__ void ll_consume4(const Eval& eval, const float* slot, int t, int nt, int nv, int r0,
                                            double& lt, double& lr, unsigned& fix) {
  const float4* s4 = reinterpret_cast<const float4*>(slot);
  const int rem = t == 0 ? r0 : kLLTile;
  float tsum = 0.0f;
  bool allok = true;
  if (rem == kLLTile)
    ll_tile4_full<Eval>(eval, s4, tsum, allok);
  else
    ll_tile4<Eval, false>(eval, s4, rem, tsum, allok);
  lt += (double)tsum;
  if (t >= nt - kKeptTiles) {
    lr += (double)tsum;
    if (nv > 1024 && __any_sync(0xffffffffu, !allok)) fix |= 1u << (t - (nt - kKeptTiles));
  }
}

// Order-free accumulation: a double becomes an (integer, 2^-40 fraction) pair, and pairs
// add as integers, so a total does not depend on the order of its parts.
__device__ __forceinline__ void fixed_acc(long long& ip, unsigned long long& fp, double v) {
  const double fl = floor(v);
  ip += (long long)fl;
  fp += (unsigned long long)((v - fl) * kFracScale);
}

__device__ __forceinline__ double fixed_read(const long long* ip, const unsigned long long* fp) {
  const long long i = *(volatile const long long*)ip;
  const unsigned long long f = *(volatile const unsigned long long*)fp;
  return (double)i + (double)f / kFracScale;
}

// The reference's convergence test after iteration t (GMEMupdateCUDA.cu:4145-4148), run
// by the warp that finished the frame's last supervoxel.
__device__ void frame_converge(const DevPlan& P, int f) {
  FrameState* S = &P.state[f];
  const FrameDesc D = load_desc(P, f);
  const double lt = fixed_read(&S->ll_int[0], &S->ll_frac[0]);
  const double lr = fixed_read(&S->ll_int[1], &S->ll_frac[1]);
  S->ll_int[0] = S->ll_int[1] = 0;
  S->ll_frac[0] = S->ll_frac[1] = 0;
  S->sv_done = 0;
  S->ll3 = S->ll2;
  S->ll2 = S->ll1;
  S->ll1 = S->ll;
  S->ll_true = lt;
  S->ll_ref = lr;
  S->ll = (D.ll_mode == TGMM_LL_TRUE) ? lt : lr;
  const int next = S->iter + 1;
  S->iter = next;
  const double ll = S->ll;
  const bool go = fabs(ll - S->ll1) / fabs(S->ll1) > D.tol && fabs(ll - S->ll2) / fabs(S->ll2) > D.tol &&
                  fabs(ll - S->ll3) / fabs(S->ll3) > D.tol;
  if (!go) S->converged = 1;
  S->done = (!go || next > D.max_iter) ? 1 : 0;
}

// Each warp streams the supervoxels it takes from the work counter through a ring of
// kLLStages tile slots; the ring runs on from one supervoxel into the next.  Tickets are
// taken two supervoxels ahead: while the warp computes its i-th supervoxel, the stream
// record and candidate ids of the (i+2)-th (stage A) and the candidates' constants of the
// (i+1)-th (stage B) are on their way, so every wait is for copies issued a supervoxel
// earlier.  A warp adds its supervoxels' sums into fixed-point registers and publishes
// them (with the count of supervoxels) when its frame changes and when it leaves; the
// warp that completes a frame's count runs the convergence test.
// With G > 0 the warps also run the kNN/E-step of the next iteration (G lanes per
// supervoxel, 32/G supervoxels an item, from a second work counter): one item after each
// supervoxel's look-ahead copies are issued, and the rest once the voxel work has run out.
// It needs only what the kill step left, and its results go to the next iteration's
// buffers, so it runs ahead of the convergence test; a frame that converges here never
// reads them.
template <bool kFp64, int G, bool kMom>
__global__ void __launch_bounds__(kLLWarps * 32, kLLBlocks) k_ll_pass(DevPlan P) {
  // the FP32 log-likelihood streams the centred voxel stream (one float4 per voxel, one bulk
  // copy per tile); the moment pass reads the input arrays (and writes that stream), the FP64
  // log-likelihood reads the input arrays too (its terms start from the exact x - c)
  constexpr bool kAos = !kFp64 && !kMom;
  constexpr bool kRec = !kAos, kLLr = kAos || kMom, kCand = !kMom;
  const int total = P.info->total_sv;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ LLShared64 sh64[kFp64 ? kLLWarps : 1];
  extern __shared__ __align__(128) unsigned char ll_smem[];
  unsigned char* wbase = ll_smem + (size_t)warp * kLLWarpBytes;
  float* wbuf = reinterpret_cast<float*>(wbase);
  const unsigned bar0 = smem_addr(wbase + kLLBarOff);
  LLRec* RA = reinterpret_cast<LLRec*>(wbase + kLLRecOff);
  LLConst* RB = reinterpret_cast<LLConst*>(wbase + kLLConstOff);
  CandF* cs = reinterpret_cast<CandF*>(wbase + kLLCandOff);
  if (lane == 0)
    for (int q = 0; q < kLLStages; q++) mbar_init(bar0 + 8 * q, 1);
  mbar_fence_init();
  __syncwarp();
  // lane 0: the fixed-point sums (true, as reference) of the warp's current frame run
  int acc_f = -1, acc_nsv = 0, acc_n = 0;
  long long acc_i0 = 0, acc_i1 = 0;
  unsigned long long acc_r0 = 0, acc_r1 = 0;
  auto publish = [&]() {
    if (lane == 0 && acc_n > 0) {
      FrameState* Sp = &P.state[acc_f];
      atomicAdd((unsigned long long*)&Sp->ll_int[0], (unsigned long long)acc_i0);
      atomicAdd((unsigned long long*)&Sp->ll_int[1], (unsigned long long)acc_i1);
      atomicAdd(&Sp->ll_frac[0], acc_r0);
      atomicAdd(&Sp->ll_frac[1], acc_r1);
      __threadfence();
      if (atomicAdd(&Sp->sv_done, acc_n) == acc_nsv - acc_n) {
        __threadfence();
        frame_converge(P, acc_f);
      }
    }
    acc_n = 0;
    acc_i0 = acc_i1 = 0;
    acc_r0 = acc_r1 = 0;
  };
  // tiles issued / consumed by this warp in this launch (slot = count mod kLLStages,
  // mbarrier phase = count / kLLStages), and tiles of the current and the next supervoxel
  // already issued; every lane keeps the same counts
  unsigned gi = 0, gc = 0;
  int ic = 0;
  FrameState* S = nullptr;
  bool failed = false;
  // tickets: the current, the next, and (lane 0) the one after
  // a ticket t is the supervoxel sv_order[t] (each frame's largest first), total at the end
  auto take = [&]() {
    const int t = atomicAdd(&P.work[0], 1);
    return t < total ? P.sv_order[t] : total;
  };
  int tk = 0;
  if (lane == 0) tk = take();
  int sc = __shfl_sync(0xffffffffu, tk, 0);
  if (lane == 0 && sc < total) tk = take();
  int sn = sc < total ? __shfl_sync(0xffffffffu, tk, 0) : total;
  if (lane == 0 && sn < total) tk = take();
  auto frame_of = [](const LLRec& A) { return kAos ? A.ll.frame : A.rec.frame; };
  if (sc < total) {
    ll_fetch_a<kRec, kLLr, kCand>(P, RA[0], sc);
    if (sn < total) ll_fetch_a<kRec, kLLr, kCand>(P, RA[1], sn);
    cp_commit();
    cp_wait_all();
    __syncwarp();
    if (!kMom) ll_fetch_b(P, RA[0], frame_of(RA[0]), RB[0]);
    cp_commit();
  }
  // the next iteration's kNN/E-step items
  constexpr int kPerItem = G > 0 ? 32 / G : 1;
  const int knn_items = G > 0 ? (total + kPerItem - 1) / kPerItem : 0;
  bool knn_more = G > 0;
  auto knn_step = [&]() {
    if constexpr (G > 0) {
      int item = 0;
      if (lane == 0) item = atomicAdd(&P.work[2], 1);
      item = __shfl_sync(0xffffffffu, item, 0);
      if (item < knn_items) {
        const int gl = lane & (G - 1), gbase = lane - gl;
        const unsigned gmask = G == 32 ? 0xffffffffu : ((1u << G) - 1u) << gbase;
        knn_estep_sv<G>(P, item * kPerItem + gbase / G, P.iter + 1, gl, gbase, gmask);
        __syncwarp();
      } else {
        knn_more = false;
      }
    }
  };
  for (unsigned i = 0; sc < total; i++) {
    // everything fetched so far was issued at least a supervoxel ago
    cp_wait_all();
    __syncwarp();
    const LLRec& CA = RA[i % 3];
    const LLConst& CB = RB[i & 1];
    const LLRec& NA = RA[(i + 1) % 3];
    const int s2 = __shfl_sync(0xffffffffu, tk, 0);
    if (lane == 0 && s2 < total) tk = take();
    if (!kMom && sn < total) ll_fetch_b(P, NA, frame_of(NA), RB[(i + 1) & 1]);
    if (s2 < total) ll_fetch_a<kRec, kLLr, kCand>(P, RA[(i + 2) % 3], s2);
    cp_commit();
    if (knn_more) knn_step();  // while this supervoxel's tiles and records land
    int in = 0;
    const int n_nt = sn < total ? (kAos ? NA.ll.ntiles : NA.rec.ntiles) : 0;  // the next one's tiles may start early
    const int nv = kAos ? CA.ll.nv : CA.rec.nv, nt = kAos ? CA.ll.ntiles : CA.rec.ntiles;
    const int f = frame_of(CA), nsv = kAos ? CA.ll.frame_nsv : CA.rec.frame_nsv;
    const float c0 = kAos ? CA.ll.c0 : CA.rec.c0, c1 = kAos ? CA.ll.c1 : CA.rec.c1, c2 = kAos ? CA.ll.c2 : CA.rec.c2;
    S = &P.state[f];
    int pk[4] = {0, 0, 0, 0};  // SoA slot offsets of the components: tile 0 in bits 0-1, later tiles in bits 4-5
    if constexpr (kRec) {
#pragma unroll
      for (int c = 0; c < 4; c++) pk[c] = (int)(CA.rec.nf[c] >> 16);
    }
    const int r0 = kAos ? CA.ll.r0 : CA.rec.r0;
    // the next staged tile of the supervoxel (of ntr): the ring is refilled first, with the
    // current supervoxel's tiles and then the next one's; nullptr if the tile never arrived
    auto ring_next = [&](int ntr) -> const float* {
      __syncwarp();  // every lane is done with the slots refilled below
      while (gi < gc + kLLStages) {
        const bool mine = ic < ntr;
        if (!mine && in >= n_nt) break;
        const int tt = mine ? ic++ : in++;
        if (lane == 0) {
          const unsigned q = gi % kLLStages;
          if constexpr (kAos)
            ll_issue4(P.vox4, mine ? CA.ll : NA.ll, tt, wbuf + q * kLLSlotFloats, bar0 + 8 * q);
          else
            ll_issue(mine ? CA.rec : NA.rec, tt, wbuf + q * kLLSlotFloats, bar0 + 8 * q);
        }
        gi++;
      }
      const unsigned q = gc % kLLStages;
      if (!__all_sync(0xffffffffu, mbar_wait(bar0 + 8 * q, (gc / kLLStages) & 1, P.stage_wait_ns))) return nullptr;
      return wbuf + q * kLLSlotFloats;
    };
    if constexpr (kMom) {
      // the moment pass: 19 sums per lane over its voxels of every tile, then per supervoxel
      double m[kNumMoments];
#pragma unroll
      for (int j = 0; j < kNumMoments; j++) m[j] = 0.0;
      bool nan_seen = false;
      for (int t = 0; t < nt; t++) {
        const float* slot = ring_next(nt);
        if (!slot) {
          failed = true;
          break;
        }
        mom_consume(slot, pk, t, r0, c0, c1, c2, m, nan_seen, P.vox4 + CA.ll.v0);
        gc++;
      }
      if (failed) break;
      if (__any_sync(0xffffffffu, nan_seen) && lane == 0) atomicOr(&S->flags, F_NAN_INPUT);
#pragma unroll
      for (int j = 0; j < kNumMoments; j++) m[j] = warp_sum(m[j]);
#pragma unroll
      for (int j = 0; j < kNumMoments; j++)  // lane j writes moment j
        if (lane == j) P.mom[(int64_t)j * P.max_sv + sc] = m[j];
    } else {
    const bool run = CB.done == 0;
    // candidate j on lane j: u = m - c, weight b = ln(w) - ln(A), -nu W/2
    double u[3] = {0, 0, 0}, h[6] = {0, 0, 0, 0, 0, 0}, b = 0.0;
    if (lane < kJ) {
      const double* L = CB.llc[lane];
      for (int e = 0; e < 6; e++) h[e] = L[e];
      b = L[6] - CB.ln_alpha;
      u[0] = L[7] - (double)c0;
      u[1] = L[8] - (double)c1;
      u[2] = L[9] - (double)c2;
    }
    const unsigned fin = __ballot_sync(0xffffffffu, lane < kJ && isfinite(b));
    const unsigned nan_w = __ballot_sync(0xffffffffu, lane < kJ && (isnan(b) || b == (double)kInfF));
    const unsigned w4m = __ballot_sync(0xffffffffu, lane >= kJ || (h[2] == 0.0 && h[4] == 0.0));
    // a NaN weight makes the reference's density NaN for every voxel (skipped); no finite
    // weight means a zero density everywhere: the tiles are consumed unread
    const bool compute = run && fin && !nan_w;
    if (kFp64) {
      LLShared64& Q = sh64[warp];
      if (lane < kJ) {
        for (int d = 0; d < 3; d++) Q.u[lane][d] = u[d];
        for (int e = 0; e < 6; e++) Q.A[lane][e] = (e == 0 || e == 3 || e == 5) ? -2.0 * h[e] : -h[e];
        Q.w[lane] = exp(b);
      }
    } else if (lane < kJ) {
      // the five candidates' FP32 constants in the packed layout (pairs 0-1, 2-3; single 4)
      float* fu = lane < 4 ? &cs->u[lane >> 1][0].x + (lane & 1) : cs->u4;
      float* fa = lane < 4 ? &cs->A[lane >> 1][0].x + (lane & 1) : cs->A4;
      const int st = lane < 4 ? 2 : 1;
      for (int d = 0; d < 3; d++) fu[st * d] = -__double2float_rn(u[d]);
      for (int e = 0; e < 6; e++) fa[st * e] = __double2float_rn(h[e]);
      if (lane < 4)
        (&cs->b[lane >> 1].x)[lane & 1] = __double2float_rn(b);
      else
        cs->b4 = __double2float_rn(b);
    }
    __syncwarp();
    double lt = 0.0, lr = 0.0;
    unsigned fix = 0;  // kept tiles with voxels of zero density
    // a finished frame issues no more tiles; those issued early are consumed unread
    const int ntr = run ? nt : ic;
    // the supervoxel's tiles and, rarely, the kept window's zero-density voxels, with the
    // candidates' constants of one evaluation form held in registers through the loop (the
    // 4-DOF form keeps 40 floats live, the general one 50)
    auto run_tiles = [&](const auto& eval) {
      for (int t = 0; t < ntr; t++) {
        const float* slot = ring_next(ntr);
        if (!slot) {
          failed = true;
          break;
        }
        if (compute) {
          if constexpr (kFp64)
            ll_consume(eval, slot, pk, t, nt, nv, r0, c0, c1, c2, lt, lr, fix);
          else
            ll_consume4(eval, slot, t, nt, nv, r0, lt, lr, fix);
        }
        gc++;
      }
      if (!failed && fix) {
        if constexpr (kFp64)
          lr += ll_fixup(eval, CA.rec, fix, c0, c1, c2);
        else
          lr += ll_fixup4(eval, P.vox4 + CA.ll.v0, nt, r0, fix);
      }
    };
    if constexpr (kFp64) {
      run_tiles(VoxelEval<2>{sh64[warp]});
    } else if (w4m == 0xffffffffu) {
      const CandF cf = load_cand<true>(*cs);
      run_tiles(VoxelEval<0>{cf});
    } else {
      const CandF cf = load_cand<false>(*cs);
      run_tiles(VoxelEval<1>{cf});
    }
    if (failed) break;
    if (run) {
      lt = warp_sum(lt);
      lr = warp_sum(lr);
      if (lane == 0) {
        if (f != acc_f) {
          publish();
          acc_f = f;
          acc_nsv = nsv;
        }
        fixed_acc(acc_i0, acc_r0, lt);
        fixed_acc(acc_i1, acc_r1, lr);
        acc_n++;
      }
    }
    }  // the log-likelihood pass
    __syncwarp();  // the records of this supervoxel are refilled from the next iteration on
    sc = sn;
    sn = s2;
    ic = in;
  }
  if (failed) {
    // a tile was not delivered within the plan's wait limit: before the warp leaves, every
    // copy it issued -- the late one included -- must have landed in its shared memory, so
    // it waits for them with the fixed bound kLLWaitNs, then reports and leaves
    for (unsigned g = gc; g < gi; g++) mbar_wait(bar0 + 8 * (g % kLLStages), (g / kLLStages) & 1, kLLWaitNs);
    if (lane == 0) atomicOr(&S->flags, F_STAGE_TIMEOUT);
  }
  cp_wait_all();
  publish();
  while (knn_more) knn_step();
  if (lane == 0 && atomicAdd(&P.work[1], 1) == (int)(gridDim.x * kLLWarps) - 1) {
    P.work[0] = 0;
    P.work[1] = 0;
    P.work[2] = 0;
  }
}

// ===========================================================================
// assign + export: post-loop supervoxel assignment (rnk > 0.5, at most 16 per Gaussian,
// GMEMupdateCUDA.cu:4310-4350) and SoA -> AoS.
// ===========================================================================
__global__ void __launch_bounds__(kSvPerBlockT) k_assign(DevPlan P) {
  const int s = blockIdx.x * kSvPerBlockT + threadIdx.x;
  if (s >= P.info->total_sv) return;
  const int f = P.sv_frame[s];
  const FrameDesc D = load_desc(P, f);
  const FrameState& S = P.state[f];
  if (S.flags & (F_BAD_CSR | F_FEW_GAUSS)) return;
  const int sl = s - D.sv_base;
  // the last E-step that ran (a kNN/E-step run ahead of a converged frame is ignored); its
  // responsibilities and candidates are the call's outputs
  const int last = S.iter - 1;
  const float* rnk = rnk_buf(P, last);
  const int32_t* cand = cand_buf(P, last);
#pragma unroll
  for (int j = 0; j < kJ; j++) {
    const float r = rnk[(int64_t)s * kJ + j];
    const int k = cand[(int64_t)s * kJ + j];
    if (last >= 1) {
      D.rnk_out[(int64_t)j * D.n_sv + sl] = r;
      D.ind_out[(int64_t)j * D.n_sv + sl] = k - D.g_base;
    }
    if ((double)r > 0.5) {
      const int b = atomicAdd(&P.acnt[k], 1);
      if (b < kBucketCap) P.abucket[(int64_t)k * kBucketCap + b] = j * D.n_sv + sl;
    }
  }
}

__global__ void __launch_bounds__(kGChunk) k_export(DevPlan P) {
  const int c = blockIdx.x;
  if (c >= P.info->n_gchunks) return;
  const GChunk ch = P.gchunks[c];
  const FrameDesc D = load_desc(P, ch.frame);
  const FrameState S = P.state[ch.frame];
  __shared__ int s_ovf[kGChunk];
  __shared__ int s_novf;
  __shared__ int s_first[kGChunk][TGMM_MAX_SV_PER_GAUSSIAN + 1];
  __shared__ int s_list[kGChunk];
  __shared__ int s_cnt[kGChunk / 32 + 1];
  if (threadIdx.x == 0) s_novf = 0;
  __syncthreads();
  const int k = ch.g_begin + threadIdx.x;
  const bool valid = k < ch.g_end;
  const bool ran = !(S.flags & (F_BAD_CSR | F_FEW_GAUSS));
  int n = 0;
  if (valid && ran) {
    n = P.acnt[k];
    P.acnt[k] = 0;
    if (n > kBucketCap) {
      const int o = atomicAdd(&s_novf, 1);
      s_ovf[o] = threadIdx.x;
      atomicOr(&P.state[ch.frame].flags, F_ASSIGN_OVERFLOW);
    } else {
      int* bk = P.abucket + (int64_t)k * kBucketCap;  // this Gaussian's own bucket
      for (int i = 1; i < n; i++) {                   // insertion sort by position
        const int v = bk[i];
        int q = i;
        while (q > 0 && bk[q - 1] > v) {
          bk[q] = bk[q - 1];
          q--;
        }
        bk[q] = v;
      }
    }
  }
  __syncthreads();
  const int novf = s_novf;
  for (int o = 0; o < novf; o++) {
    const int tk = s_ovf[o];
    int taken = 0;
    int* dst = s_first[tk];
    ordered_scan(P, D, S.iter - 1, ch.g_begin + tk, 0.5, s_list, s_cnt, [&](int p) {
      if (taken < TGMM_MAX_SV_PER_GAUSSIAN) dst[taken++] = p;
    });
    if (threadIdx.x == 0) dst[TGMM_MAX_SV_PER_GAUSSIAN] = taken;
    __syncthreads();
  }
  if (!valid) return;
  TgmmGaussian& g = D.gm[k - D.g_base];
  if (ran) {
    g.beta_k = gcomp(P, G_BETA, k);
    g.nu_k = gcomp(P, G_NU, k);
    g.alpha_k = gcomp(P, G_ALPHA, k);
    for (int d = 0; d < 3; d++) g.m_k[d] = gcomp(P, G_M0 + d, k);
    for (int e = 0; e < 6; e++) g.W_k[e] = gcomp(P, G_W0 + e, k);
    const int last = (S.iter - 1) & 1;  // parity of the last iteration that ran
    const double eld = gcomp(P, G_ELD0 + last, k);
    g.expectedLogDetCovarianceCUDA = eld;
    g.expectedLogResponsivityCUDA = (eld == -1e32) ? -1e32 : gcomp(P, G_PSIA0 + last, k) - S.psi_total[last];
    for (int d = 0; d < 3; d++) g.m_o[d] = gcomp(P, G_MO0 + d, k);
    g.W_o[5] = gcomp(P, G_WO5, k);
    if (n > kBucketCap) {
      const int taken = s_first[threadIdx.x][TGMM_MAX_SV_PER_GAUSSIAN];
      for (int i = 0; i < taken; i++) g.supervoxelIdx[i] = s_first[threadIdx.x][i] % D.n_sv;
      g.supervoxelNum = taken;
    } else {
      const int taken = min(n, TGMM_MAX_SV_PER_GAUSSIAN);
      const int* bk = P.abucket + (int64_t)k * kBucketCap;
      for (int i = 0; i < taken; i++) g.supervoxelIdx[i] = bk[i] % D.n_sv;
      g.supervoxelNum = taken;
    }
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline int div_up(int a, int b) { return (a + b - 1) / b; }

void launch_build_maps(const DevPlan& P, cudaStream_t st) {
  k_build_maps<<<dim3(P.max_frames, kMapSlices), kFrameThreads, 0, st>>>(P);
}
// The caller's page-locked records into the plan's device records, 16 bytes a thread, read
// by the SMs over the bus (not a copy engine, so they do not queue behind the caller's own
// uploads), for every frame whose descriptor names a source.
__global__ void __launch_bounds__(256) k_fetch_records(DevPlan P) {
  const int nf = P.info->n_frames;
  for (int f = 0; f < nf; f++) {
    const FrameDesc& D = P.frames[f];
    const uint4* src = reinterpret_cast<const uint4*>(D.gm_src);
    if (!src) continue;
    uint4* dst = reinterpret_cast<uint4*>(D.gm);
    const int64_t n16 = (int64_t)D.n_gauss * (int64_t)sizeof(TgmmGaussian) / 16;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n16; i += (int64_t)gridDim.x * blockDim.x)
      dst[i] = src[i];
  }
}
void launch_fetch_records(const DevPlan& P, cudaStream_t st) {
  k_fetch_records<<<min(P.max_gchunks * (kGChunk * (int)sizeof(TgmmGaussian) / 16 / 256), 148 * 4), 256, 0, st>>>(P);
}
void launch_import(const DevPlan& P, cudaStream_t st) { k_import<<<P.max_gchunks, kGChunk, 0, st>>>(P); }
void launch_order(const DevPlan& P, cudaStream_t st) {
  k_sv_records<<<div_up(P.max_sv, 256), 256, 0, st>>>(P);
  k_order_base<<<P.max_frames, 32, 0, st>>>(P);
  k_order_scatter<<<div_up(P.max_sv, 256), 256, 0, st>>>(P);
}
void launch_moments(const DevPlan& P, cudaStream_t st) {
  k_ll_pass<false, 0, true><<<P.ll_blocks, kLLWarps * 32, kLLSmemBytes, st>>>(P);
}
void launch_knn_estep(const DevPlan& P, cudaStream_t st) {
  const int G = P.knn_group;
  const int grid = div_up(P.max_sv, kKnnWarps * 32 / G);
  if (G == 32)
    k_knn_estep<32><<<grid, kKnnWarps * 32, 0, st>>>(P);
  else if (G == 16)
    k_knn_estep<16><<<grid, kKnnWarps * 32, 0, st>>>(P);
  else if (G == 8)
    k_knn_estep<8><<<grid, kKnnWarps * 32, 0, st>>>(P);
  else
    k_knn_estep<4><<<grid, kKnnWarps * 32, 0, st>>>(P);
}
void launch_mstep_update(const DevPlan& P, cudaStream_t st) {
  k_mstep_update<<<2 * P.max_gchunks, kMChunk, 0, st>>>(P);
}
void launch_kill_prep(const DevPlan& P, cudaStream_t st) {
  k_kill_prep<<<P.max_gchunks, kGChunk, 0, st>>>(P);
}
void launch_ll_pass(const DevPlan& P, int fp64, int knn_group, cudaStream_t st) {
  const int grid = P.ll_blocks;
  const int bs = kLLWarps * 32;
  if (fp64)
    k_ll_pass<true, 0, false><<<P.ll_blocks64, bs, kLLSmemBytes, st>>>(P);
  else if (knn_group == 8)
    k_ll_pass<false, 8, false><<<grid, bs, kLLSmemBytes, st>>>(P);
  else if (knn_group == 16)
    k_ll_pass<false, 16, false><<<grid, bs, kLLSmemBytes, st>>>(P);
  else if (knn_group == 32)
    k_ll_pass<false, 32, false><<<grid, bs, kLLSmemBytes, st>>>(P);
  else
    k_ll_pass<false, 0, false><<<grid, bs, kLLSmemBytes, st>>>(P);
}

// Host tables reach the device as launch parameters of k_stage (24 KB a launch), so staging
// a batch takes no copy engine: a batch is not queued behind large uploads of other frames.
constexpr int kStageChunk16 = 1536;
struct StageArgs {
  uint4* dst;
  int n16;
  int pad;
  uint4 data[kStageChunk16];
};

__global__ void __launch_bounds__(256) k_stage(const __grid_constant__ StageArgs a) {
  for (int i = threadIdx.x; i < a.n16; i += blockDim.x) a.dst[i] = a.data[i];
}

cudaError_t launch_stage_bytes(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  StageArgs a;
  const unsigned char* s = static_cast<const unsigned char*>(src);
  for (size_t off = 0; off < bytes; off += 16 * (size_t)kStageChunk16) {
    const size_t n = std::min(bytes - off, 16 * (size_t)kStageChunk16);
    memset(a.data, 0, 16 * ((n + 15) / 16));
    memcpy(a.data, s + off, n);
    a.dst = reinterpret_cast<uint4*>(static_cast<unsigned char*>(dst) + off);
    a.n16 = (int)((n + 15) / 16);
    a.pad = 0;
    k_stage<<<1, 256, 0, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t configure_kernels(DevPlan& P, int device) {
  // every form of the voxel pass: its dynamic shared memory, and the blocks per SM its
  // persistent grid is sized for -- the fewest of the FP32 forms and the moment pass, and
  // separately the FP64 form, whose per-warp FP64 constants take more shared memory
  const void* forms[6] = {(const void*)k_ll_pass<false, 0, false>, (const void*)k_ll_pass<false, 8, false>,
                          (const void*)k_ll_pass<false, 16, false>, (const void*)k_ll_pass<false, 32, false>,
                          (const void*)k_ll_pass<false, 0, true>, (const void*)k_ll_pass<true, 0, false>};
  int sms = 0, per = 1 << 30, per64 = 1 << 30;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  for (int i = 0; i < 6; i++) {
    int p = 0;
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(forms[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLLSmemBytes);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, forms[i], kLLWarps * 32, kLLSmemBytes);
    int& m = i < 5 ? per : per64;
    m = p < m ? p : m;
  }
  P.ll_blocks = sms * (per > 0 && per < (1 << 30) ? per : 1);
  P.ll_blocks64 = sms * (per64 > 0 && per64 < (1 << 30) ? per64 : 1);
  return e;
}
// The condition of the next iteration's conditional graph node: whether any frame of the
// batch is still running (its done flag is set by the voxel pass's convergence test, or at
// the start for a frame that cannot run).  A batch whose frames have all stopped skips the
// remaining iterations' launches, which would find nothing to do.
__global__ void __launch_bounds__(1024) k_iter_cond(DevPlan P, cudaGraphConditionalHandle h) {
  const int nf = P.info->n_frames;
  int running = 0;
  for (int f = threadIdx.x; f < nf; f += blockDim.x) running |= P.state[f].done == 0;
  running = __syncthreads_or(running);
  if (threadIdx.x == 0) cudaGraphSetConditional(h, running ? 1u : 0u);
}
void launch_iter_cond(const DevPlan& P, cudaGraphConditionalHandle h, cudaStream_t st) {
  k_iter_cond<<<1, 1024, 0, st>>>(P, h);
}

void launch_assign(const DevPlan& P, cudaStream_t st) {
  k_assign<<<div_up(P.max_sv, kSvPerBlockT), kSvPerBlockT, 0, st>>>(P);
}
void launch_export(const DevPlan& P, cudaStream_t st) { k_export<<<P.max_gchunks, kGChunk, 0, st>>>(P); }


// ---------------------------------------------------------------------------
// Standalone exact kNN (tgmm_knn): the same grid search over one point set.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_sa_geometry(const float* q, int64_t nq, float s0, float s1, float s2,
                                                      int nref, int budget, FrameState* S) {
  __shared__ float smin[3][32], smax[3][32];
  const float sc[3] = {s0, s1, s2};
  float lo[3] = {kInfF, kInfF, kInfF}, hi[3] = {-kInfF, -kInfF, -kInfF};
  for (int64_t i = threadIdx.x; i < nq; i += blockDim.x)
    for (int d = 0; d < 3; d++) {
      const float y = q[d * nq + i] * sc[d];
      if (!isfinite(y)) continue;
      lo[d] = fminf(lo[d], y);
      hi[d] = fmaxf(hi[d], y);
    }
  for (int d = 0; d < 3; d++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int d = 0; d < 3; d++) {
      smin[d][w] = lo[d];
      smax[d][w] = hi[d];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int d = 0; d < 3; d++) {
      lo[d] = smin[d][0];
      hi[d] = smax[d][0];
      for (int i = 1; i < (int)(blockDim.x >> 5); i++) {
        lo[d] = fminf(lo[d], smin[d][i]);
        hi[d] = fmaxf(hi[d], smax[d][i]);
      }
      if (!(lo[d] <= hi[d])) lo[d] = hi[d] = 0.0f;
    }
    set_geometry(S, lo, hi, nref, budget);
  }
}

// Reference point k, coordinate d, sits at ref[k * step + d * comp]: AoS xyz (step 3,
// comp 1) or SoA x-block, y-block, z-block (step 1, comp nref).
__global__ void k_sa_count(const float* ref, int nref, int step, int64_t comp, float s0, float s1, float s2,
                           const FrameState* S, int* cnt, int* rcell) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nref) return;
  const float* rk = ref + (int64_t)k * step;
  const float ys[3] = {rk[0] * s0, rk[comp] * s1, rk[2 * comp] * s2};
  int cell = 0;
  for (int d = 0; d < 3; d++)
    if (!isfinite(ys[d]) || fabsf(ys[d]) >= 1e25f) cell = -1;
  if (cell == 0) {
    const int cx = cell_coord(ys[0], S->lo[0], S->inv_h, S->dims[0]);
    const int cy = cell_coord(ys[1], S->lo[1], S->inv_h, S->dims[1]);
    const int cz = cell_coord(ys[2], S->lo[2], S->inv_h, S->dims[2]);
    cell = (cz * S->dims[1] + cy) * S->dims[0] + cx;
    atomicAdd(&cnt[cell], 1);
  }
  rcell[k] = cell;
}

__global__ void __launch_bounds__(1024) k_sa_scan(const FrameState* S, int* cnt, int* start, int* cur) {
  __shared__ int scan[1024];
  const int n = S->n_cells;
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b0 = min(n, (int)threadIdx.x * per), b1 = min(n, b0 + per);
  int local = 0;
  for (int i = b0; i < b1; i++) local += cnt[i];
  scan[threadIdx.x] = local;
  __syncthreads();
  for (int off = 1; off < (int)blockDim.x; off <<= 1) {
    int v = (threadIdx.x >= (unsigned)off) ? scan[threadIdx.x - off] : 0;
    __syncthreads();
    scan[threadIdx.x] += v;
    __syncthreads();
  }
  int run = scan[threadIdx.x] - local;
  for (int i = b0; i < b1; i++) {
    start[i] = run;
    cur[i] = run;
    run += cnt[i];
  }
  if (threadIdx.x == blockDim.x - 1) start[n] = scan[blockDim.x - 1];
}

__global__ void k_sa_fill(const float* ref, int nref, int step, int64_t comp, const int* rcell, int* cur,
                          float4* refs) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nref || rcell[k] < 0) return;
  const int pos = atomicAdd(&cur[rcell[k]], 1);
  const float* rk = ref + (int64_t)k * step;
  refs[pos] = make_float4(rk[0], rk[comp], rk[2 * comp], __int_as_float(k));
}

__global__ void k_sa_query(const float* q, int64_t nq, const float* ref, int nref, float s0, float s1, float s2,
                           const FrameState* S, const int* start, const float4* refs, int32_t* ind) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const float sc[3] = {s0, s1, s2};
  const float q0 = q[i], q1 = q[nq + i], q2 = q[2 * nq + i];
  GridGeom g;
  for (int d = 0; d < 3; d++) {
    g.lo[d] = S->lo[d];
    g.dims[d] = S->dims[d];
  }
  g.h = S->h;
  g.inv_h = S->inv_h;
  Top5 t;
  top5_init(t);
  knn_grid_search<kJ>(q0, q1, q2, sc, g, start, refs, t);
  if (!(t.d[kJ - 1] < kInfF)) {
    top5_init(t);
    for (int k = 0; k < nref; k++) top5_insert(t, knn_dist(q0, q1, q2, ref[3 * k], ref[3 * k + 1], ref[3 * k + 2], sc), k);
  }
  for (int j = 0; j < kJ; j++) ind[(int64_t)j * nq + i] = t.i[j];
}

// The K nearest (K <= kMaxK) of each query with their squared scaled distances, for the
// tracking graph's supervoxel kNN: the same grid search, the same exact fallback scan when
// fewer than K finite distances were found, (distance, index) order; a slot with no
// reference point closer than 1e32 (squared) gets index -1 and distance 1e32.
template <int K>
__global__ void k_sa_query_k(const float* q, int64_t nq, const float* ref, int nref, int step, int64_t comp,
                             float s0, float s1, float s2, const FrameState* S, const int* start, const float4* refs,
                             int32_t* ind, float* dist) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const float sc[3] = {s0, s1, s2};
  const float q0 = q[i], q1 = q[nq + i], q2 = q[2 * nq + i];
  GridGeom g;
  for (int d = 0; d < 3; d++) {
    g.lo[d] = S->lo[d];
    g.dims[d] = S->dims[d];
  }
  g.h = S->h;
  g.inv_h = S->inv_h;
  TopN<K> t;
  topn_init<K>(t);
  knn_grid_search<K>(q0, q1, q2, sc, g, start, refs, t);
  if (!(t.d[K - 1] < kInfF)) {
    topn_init<K>(t);
    for (int k = 0; k < nref; k++) {
      const float* rk = ref + (int64_t)k * step;
      topn_insert<K>(t, knn_dist(q0, q1, q2, rk[0], rk[comp], rk[2 * comp], sc), k);
    }
  }
#pragma unroll
  for (int j = 0; j < K; j++) {
    const bool real = t.i[j] != 0x7fffffff && t.d[j] < 1e32f;
    ind[(int64_t)j * nq + i] = real ? t.i[j] : -1;
    if (dist) dist[(int64_t)j * nq + i] = real ? t.d[j] : 1e32f;
  }
}

cudaError_t knn_grid_standalone(const float* q, int64_t nq, const float* ref, int32_t nref, const float scale[3],
                                int32_t* ind, cudaStream_t st) {
  const int budget = 2 * nref + 2;
  char* buf = nullptr;
  const size_t off_state = 0, off_cnt = 256, off_start = off_cnt + 4 * (size_t)budget,
               off_cur = off_start + 4 * ((size_t)budget + 1), off_rc = off_cur + 4 * (size_t)budget,
               off_refs = (off_rc + 4 * (size_t)nref + 255) / 256 * 256, total = off_refs + 16 * (size_t)nref;
  cudaError_t e = cudaMallocAsync((void**)&buf, total, st);
  if (e != cudaSuccess) return e;
  FrameState* S = (FrameState*)(buf + off_state);
  int* cnt = (int*)(buf + off_cnt);
  int* start = (int*)(buf + off_start);
  int* cur = (int*)(buf + off_cur);
  int* rc = (int*)(buf + off_rc);
  float4* refs = (float4*)(buf + off_refs);
  cudaMemsetAsync(cnt, 0, 4 * (size_t)budget, st);
  k_sa_geometry<<<1, 1024, 0, st>>>(q, nq, scale[0], scale[1], scale[2], nref, budget, S);
  const int gb = (nref + 255) / 256;
  k_sa_count<<<gb, 256, 0, st>>>(ref, nref, 3, 1, scale[0], scale[1], scale[2], S, cnt, rc);
  k_sa_scan<<<1, 1024, 0, st>>>(S, cnt, start, cur);
  k_sa_fill<<<gb, 256, 0, st>>>(ref, nref, 3, 1, rc, cur, refs);
  k_sa_query<<<(unsigned)((nq + 127) / 128), 128, 0, st>>>(q, nq, ref, nref, scale[0], scale[1], scale[2], S, start,
                                                          refs, ind);
  e = cudaGetLastError();
  cudaFreeAsync(buf, st);
  return e;
}

// The K-nearest grid search (1 <= K <= kMaxK) over reference points in AoS or SoA layout
// (see k_sa_count), with distances; scratch from the stream-ordered allocator.
cudaError_t knn_grid_topk(const float* q, int64_t nq, const float* ref, int32_t nref, int soa, int K,
                          const float scale[3], int32_t* ind, float* dist, cudaStream_t st) {
  const int step = soa ? 1 : 3;
  const int64_t comp = soa ? nref : 1;
  const int budget = 2 * nref + 2;
  char* buf = nullptr;
  const size_t off_state = 0, off_cnt = 256, off_start = off_cnt + 4 * (size_t)budget,
               off_cur = off_start + 4 * ((size_t)budget + 1), off_rc = off_cur + 4 * (size_t)budget,
               off_refs = (off_rc + 4 * (size_t)nref + 255) / 256 * 256, total = off_refs + 16 * (size_t)nref;
  cudaError_t e = cudaMallocAsync((void**)&buf, total, st);
  if (e != cudaSuccess) return e;
  FrameState* S = (FrameState*)(buf + off_state);
  int* cnt = (int*)(buf + off_cnt);
  int* start = (int*)(buf + off_start);
  int* cur = (int*)(buf + off_cur);
  int* rc = (int*)(buf + off_rc);
  float4* refs = (float4*)(buf + off_refs);
  cudaMemsetAsync(cnt, 0, 4 * (size_t)budget, st);
  k_sa_geometry<<<1, 1024, 0, st>>>(q, nq, scale[0], scale[1], scale[2], nref, budget, S);
  const int gb = (nref + 255) / 256;
  k_sa_count<<<gb, 256, 0, st>>>(ref, nref, step, comp, scale[0], scale[1], scale[2], S, cnt, rc);
  k_sa_scan<<<1, 1024, 0, st>>>(S, cnt, start, cur);
  k_sa_fill<<<gb, 256, 0, st>>>(ref, nref, step, comp, rc, cur, refs);
  const unsigned grid = (unsigned)((nq + 127) / 128);
  switch (K) {
#define TGMM_TOPK_CASE(KK)                                                                                     \
  case KK:                                                                                                   \
    k_sa_query_k<KK><<<grid, 128, 0, st>>>(q, nq, ref, nref, step, comp, scale[0], scale[1], scale[2], S, start, \
                                           refs, ind, dist);                                                 \
    break;
    TGMM_TOPK_CASE(1) TGMM_TOPK_CASE(2) TGMM_TOPK_CASE(3) TGMM_TOPK_CASE(4) TGMM_TOPK_CASE(5) TGMM_TOPK_CASE(6)
    TGMM_TOPK_CASE(7) TGMM_TOPK_CASE(8) TGMM_TOPK_CASE(9) TGMM_TOPK_CASE(10) TGMM_TOPK_CASE(11)
#undef TGMM_TOPK_CASE
    default:
      break;
  }
  e = cudaGetLastError();
  cudaFreeAsync(buf, st);
  return e;
}

// Bytes of scratch the grid kNN needs for nref reference points.
size_t knn_grid_scratch_bytes(int32_t nref) {
  const size_t budget = 2 * (size_t)nref + 2;
  const size_t refs_off = (256 + 4 * budget + 4 * (budget + 1) + 4 * budget + 4 * (size_t)nref + 255) / 256 * 256;
  return refs_off + 16 * (size_t)nref;
}

// The grid kNN on caller-provided scratch (at least knn_grid_scratch_bytes(nref), 256-byte
// aligned); allocates nothing.
cudaError_t knn_grid_in_scratch(const float* q, int64_t nq, const float* ref, int32_t nref, const float scale[3],
                                int32_t* ind, cudaStream_t st, void* scratch) {
  const int budget = 2 * nref + 2;
  char* buf = (char*)scratch;
  const size_t off_state = 0, off_cnt = 256, off_start = off_cnt + 4 * (size_t)budget,
               off_cur = off_start + 4 * ((size_t)budget + 1), off_rc = off_cur + 4 * (size_t)budget,
               off_refs = (off_rc + 4 * (size_t)nref + 255) / 256 * 256;
  static_assert(sizeof(FrameState) <= 256, "the grid geometry record fits the scratch's 256-byte header");
  FrameState* S = (FrameState*)(buf + off_state);
  int* cnt = (int*)(buf + off_cnt);
  int* start = (int*)(buf + off_start);
  int* cur = (int*)(buf + off_cur);
  int* rc = (int*)(buf + off_rc);
  float4* refs = (float4*)(buf + off_refs);
  cudaError_t e = cudaMemsetAsync(cnt, 0, 4 * (size_t)budget, st);  // counts start at zero every call
  if (e != cudaSuccess) return e;
  k_sa_geometry<<<1, 1024, 0, st>>>(q, nq, scale[0], scale[1], scale[2], nref, budget, S);
  const int gb = (nref + 255) / 256;
  k_sa_count<<<gb, 256, 0, st>>>(ref, nref, 3, 1, scale[0], scale[1], scale[2], S, cnt, rc);
  k_sa_scan<<<1, 1024, 0, st>>>(S, cnt, start, cur);
  k_sa_fill<<<gb, 256, 0, st>>>(ref, nref, 3, 1, rc, cur, refs);
  k_sa_query<<<(unsigned)((nq + 127) / 128), 128, 0, st>>>(q, nq, ref, nref, scale[0], scale[1], scale[2], S, start,
                                                          refs, ind);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Posterior -> prior on the device (GaussianMixtureModel::updatePriors,
// GaussianMixtureModel.cpp:892-910; N_k = nu_k - nu_o as copyFromGMEM_CUDA/updateNk
// derive it; then nu_k *= 2, W_k /= 2 as mainTrackingGaussianMixtureModel.cpp:961-969).
// One block: the optional alpha total is a fixed-order block sum.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_update_priors(TgmmGaussian* gm, int n, double bp, double np, double ap,
                                                        double atot, int compute) {
  __shared__ double sh[32];
  __shared__ double s_tot;
  if (compute && atot < 0.0) {
    double a = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) a += gm[k].alpha_k;
    a = warp_sum(a);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += sh[i];
      s_tot = t;
    }
    __syncthreads();
    atot = s_tot;
  }
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    TgmmGaussian& g = gm[k];
    const double Nk = g.nu_k - g.nu_o;
    for (int d = 0; d < 3; d++) g.m_o[d] = g.m_k[d];
    g.beta_o = fmax(bp * Nk, 1e-5);
    g.nu_o = fmax(np * Nk, 3.0);
    for (int e = 0; e < 6; e++) g.W_o[e] = g.W_k[e] * g.nu_k / g.nu_o;
    if (atot >= 0.0) g.alpha_o = atot * TGMM_MIN_PI_FOR_DEAD * ap;
    g.nu_k *= 2.0;
    for (int e = 0; e < 6; e++) g.W_k[e] /= 2.0;
  }
}

cudaError_t update_priors_device(TgmmGaussian* gm, int32_t n, double bp, double np, double ap, double atot,
                                 int compute, cudaStream_t st) {
  k_update_priors<<<1, 1024, 0, st>>>(gm, n, bp, np, ap, atot, compute);
  return cudaGetLastError();
}

}  // namespace tgmm
