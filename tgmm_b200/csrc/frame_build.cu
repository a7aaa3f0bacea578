// frame_build.cu -- frame preparation on the device: the EM's input arrays (coordinates SoA,
// intensities, CSR, centroids) from the raw 16-bit image and the label volume of the
// segmentation at tau, as the tracking program builds them on the host
// (mainTrackingGaussianMixtureModel.cpp:553-651, 774-870; supervoxel.cpp:1410-1450,
// 1556-1747; hierarchicalSegmentation.cpp:1064-1092; mylib/array.p:2769-2822).
//
//   k_fb_scan    one pass over the label volume (16-byte loads, all-background groups
//                skipped): voxels and bounding box per supervoxel (lanes of a warp with the
//                same label add once);
//   k_fb_ptr     the supervoxels' CSR (one block);
//   k_fb_group   a warp per supervoxel walks its box in raster order and lists its voxels
//                in ascending linear index (ballot + popcount: no sort), with their values;
//   k_fb_trim    a block per supervoxel: the trimming threshold (two order statistics by a
//                two-pass radix select over 256-bin histograms, Otsu's threshold), the
//                flood from the brightest voxel (level-synchronous; candidate and reached
//                bits of the supervoxel's box in shared memory, or one bit per volume voxel
//                in global memory for boxes beyond 65536 voxels), each list entry's verdict,
//                and for kept supervoxels the FP32 centroid in the reference's summation
//                order and the range of the background-subtracted values;
//   k_fb_order   one block: the reference's erase order (a closed form of its
//                swap-to-the-back loop, resolved by pointer jumping), the [0,1] rescale
//                factors;
//   k_fb_csr     one block: the output CSR in that order;
//   k_fb_emit    a warp per output supervoxel writes its kept voxels in ascending order.
// Every rounding step is written with explicit _rn intrinsics so that no multiply-add is
// contracted: the results are the host build's bits.
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "tgmm_internal.cuh"

namespace tgmm {
namespace {

constexpr int kFbMaxOff = 74;
constexpr int kFbTrimThreads = 256;  // also the Otsu histogram's bins: a thread per bin
constexpr int kFbScanDepth = 4;  // 16-byte label groups each lane of the scan has in flight

struct FbBox {
  int32_t lo[3], hi[3];
};

struct FbOffsets {
  int64_t off[kFbMaxOff];    // linear-index offsets, as the reference builds them
  int8_t d[kFbMaxOff][3];    // their (dx, dy, dz)
  int32_t n;
  // unsigned division of a 32-bit linear index by X and by X*Y as a multiply-high and shifts
  // (Granlund and Montgomery's method; exact for every 32-bit numerator)
  uint32_t mx, mxy;
  int32_t lx, lxy;
};

// The magic number m and the shift l of the division by d (1 <= d < 2^32): l = ceil(log2 d),
// m = floor(2^32 (2^l - d) / d) + 1.
void div_magic(uint32_t d, uint32_t* m, int32_t* l) {
  int32_t k = 0;
  while (((uint64_t)1 << k) < d) k++;
  *m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << k) - d)) / d + 1);
  *l = k;
}

__device__ __forceinline__ uint32_t div_by_magic(uint32_t n, uint32_t m, int32_t l) {
  const uint32_t t = __umulhi(n, m);
  return l == 0 ? n : (t + ((n - t) >> 1)) >> (l - 1);
}

// per-call scalars shared by the kernels
struct FbStat {
  uint32_t flags;        // 1: a label above n_labels; 2: every supervoxel erased; 4: lists inconsistent
  uint32_t sub_min;      // range of the background-subtracted values of kept voxels
  uint32_t sub_max;
  uint32_t pad;
  unsigned long long kept_vox;
  int64_t n_vox;         // output sizes
  int32_t n_sv;
  int32_t scaled;        // the rescale applies (the volume is not constant)
  double fct, shift;     // img = (float)(fct * ((double)v + shift))
};

struct FbWork {
  int32_t* cnt;     // [n] voxels per supervoxel (untrimmed)
  FbBox* box;       // [n]
  int64_t* uptr;    // [n+1] CSR of the untrimmed lists
  uint32_t* ulin;   // [nvol] lists: linear indices, ascending within a supervoxel
  uint16_t* uval;   // [nvol] their raw values
  uint32_t* queue;  // [nvol] flood queues (a supervoxel's at its list offset)
  uint32_t* bits;   // [nvol/32] flood: reached voxels (supervoxels whose box exceeds shared memory)
  uint8_t* ukeep;   // [nvol] 1 where a list entry survived trimming
  int32_t* tcnt;    // [n] voxels kept by trimming
  uint32_t* thr;    // [n] trimming thresholds
  float* tcent;     // [3n] centroids (AoS)
  int32_t* rank;    // [n] erased supervoxels before each index
  int32_t* order;   // [n] output supervoxel -> supervoxel
  int32_t* nxt;     // [n] pointer jumping over the tail positions
  FbStat* stat;
};

size_t align_up(size_t x) { return (x + 255) / 256 * 256; }

// Carves the workspace; returns its size (base may be null to measure).  n_list < 0: the
// volume form (lists built here, one entry per volume voxel at most); else the list form (the
// caller's n_list entries, read in place).
size_t carve(char* base, int64_t nvol, int32_t n, FbWork* w, int64_t n_list = -1) {
  size_t at = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + at : nullptr;
    at += align_up(bytes);
    return p;
  };
  const bool lists = n_list >= 0;
  const int64_t ne = lists ? n_list : nvol;
  w->cnt = (int32_t*)take(4 * (size_t)n);
  w->box = (FbBox*)take(sizeof(FbBox) * (size_t)n);
  w->uptr = lists ? nullptr : (int64_t*)take(8 * ((size_t)n + 1));
  w->ulin = lists ? nullptr : (uint32_t*)take(4 * (size_t)nvol);
  w->uval = lists ? nullptr : (uint16_t*)take(2 * (size_t)nvol);
  w->queue = (uint32_t*)take(4 * (size_t)ne);
  w->bits = (uint32_t*)take(4 * (size_t)((nvol + 31) / 32));
  w->ukeep = (uint8_t*)take((size_t)ne);
  w->tcnt = (int32_t*)take(4 * (size_t)n);
  w->thr = (uint32_t*)take(4 * (size_t)n);
  w->tcent = (float*)take(12 * (size_t)n);
  w->rank = (int32_t*)take(4 * (size_t)n);
  w->order = (int32_t*)take(4 * (size_t)n);
  w->nxt = (int32_t*)take(4 * (size_t)n);
  w->stat = (FbStat*)take(sizeof(FbStat));
  return at;
}

__global__ void __launch_bounds__(256) k_fb_init(int32_t n, FbWork w) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    FbStat* st = w.stat;
    st->flags = 0;
    st->sub_min = 0xffffffffu;
    st->sub_max = 0;
    st->kept_vox = 0;
    st->n_vox = 0;
    st->n_sv = 0;
  }
  if (s >= n) return;
  w.cnt[s] = 0;
  for (int d = 0; d < 3; d++) {
    w.box[s].lo[d] = 0x7fffffff;
    w.box[s].hi[d] = -1;
  }
}

// One label of the scan: its lanes (those that matched) add their count and extent once.
__device__ __forceinline__ void scan_label(uint32_t l, uint32_t v, uint32_t X, uint32_t XY, int32_t n, int lane,
                                           FbWork& w) {
  if (l > (uint32_t)n) {
    atomicOr(&w.stat->flags, 1u);
    l = 0;
  }
  const unsigned m = __match_any_sync(0xffffffffu, l);
  const uint32_t z = v / XY, r = v - z * XY, y = r / X, x = r - y * X;
  const int32_t x0 = (int32_t)__reduce_min_sync(m, x), x1 = (int32_t)__reduce_max_sync(m, x);
  const int32_t y0 = (int32_t)__reduce_min_sync(m, y), y1 = (int32_t)__reduce_max_sync(m, y);
  const int32_t z0 = (int32_t)__reduce_min_sync(m, z), z1 = (int32_t)__reduce_max_sync(m, z);
  if (l != 0 && (m & ((1u << lane) - 1u)) == 0) {
    const int s = (int)l - 1;
    FbBox* b = &w.box[s];
    atomicAdd(&w.cnt[s], __popc(m));
    atomicMin(&b->lo[0], x0);
    atomicMax(&b->hi[0], x1);
    atomicMin(&b->lo[1], y0);
    atomicMax(&b->hi[1], y1);
    atomicMin(&b->lo[2], z0);
    atomicMax(&b->hi[2], z1);
  }
}

// The four consecutive voxels v..v+3 of one lane (labels q), one distinct nonzero label at a
// time: the lane's voxels of that label give a count and a coordinate extent, the lanes of the
// warp holding the same label combine theirs (match, reductions) and one of them adds the sums
// into the supervoxel's count and box.  Neighbouring voxels almost always share a label, so a
// warp usually takes one round for its 128 voxels.
__device__ __forceinline__ void scan_group(uint4 q, uint32_t v, uint32_t X, uint32_t XY, int32_t n, int lane,
                                           FbWork& w) {
  uint32_t l[4] = {q.x, q.y, q.z, q.w};
  bool bad = false;
#pragma unroll
  for (int i = 0; i < 4; i++)
    if (l[i] > (uint32_t)n) {
      bad = true;
      l[i] = 0;
    }
  if (bad) atomicOr(&w.stat->flags, 1u);
  const uint32_t z = v / XY, r = v - z * XY, y = r / X, x = r - y * X;
  while (true) {
    const uint32_t cur = l[0] ? l[0] : l[1] ? l[1] : l[2] ? l[2] : l[3];
    if (!__any_sync(0xffffffffu, cur != 0)) break;
    int cnt = 0;
    int32_t x0 = 0x7fffffff, x1 = -1, y0 = 0x7fffffff, y1 = -1, z0 = 0x7fffffff, z1 = -1;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      if (cur != 0 && l[i] == cur) {
        uint32_t xi = x + i, yi = y, zi = z;
        if (xi >= X) {  // the group runs into the next row
          const uint32_t vi = v + i;
          zi = vi / XY;
          const uint32_t ri = vi - zi * XY;
          yi = ri / X;
          xi = ri - yi * X;
        }
        x0 = min(x0, (int32_t)xi);
        x1 = max(x1, (int32_t)xi);
        y0 = min(y0, (int32_t)yi);
        y1 = max(y1, (int32_t)yi);
        z0 = min(z0, (int32_t)zi);
        z1 = max(z1, (int32_t)zi);
        cnt++;
        l[i] = 0;
      }
    }
    const unsigned m = __match_any_sync(0xffffffffu, cur);
    cnt = (int)__reduce_add_sync(m, (unsigned)cnt);
    x0 = __reduce_min_sync(m, x0);
    x1 = __reduce_max_sync(m, x1);
    y0 = __reduce_min_sync(m, y0);
    y1 = __reduce_max_sync(m, y1);
    z0 = __reduce_min_sync(m, z0);
    z1 = __reduce_max_sync(m, z1);
    if (cur != 0 && (m & ((1u << lane) - 1u)) == 0) {
      const int s = (int)cur - 1;
      FbBox* b = &w.box[s];
      atomicAdd(&w.cnt[s], cnt);
      atomicMin(&b->lo[0], x0);
      atomicMax(&b->hi[0], x1);
      atomicMin(&b->lo[1], y0);
      atomicMax(&b->hi[1], y1);
      atomicMin(&b->lo[2], z0);
      atomicMax(&b->hi[2], z1);
    }
  }
}

// One pass over the label volume, four labels per lane (16-byte loads); warps whose 128
// labels are all 0 (most of a volume) do nothing more.  Coordinates in 32-bit arithmetic
// (X*Y*Z < 2^32).
__global__ void __launch_bounds__(256) k_fb_scan(const uint32_t* __restrict__ label, int64_t nvol, int32_t X,
                                                 int32_t Y, int32_t n, FbWork w) {
  const int lane = threadIdx.x & 31;
  const uint32_t XY = (uint32_t)X * (uint32_t)Y;
  const int64_t nq = nvol / 4;  // whole 16-byte groups
  const uint4* l4 = reinterpret_cast<const uint4*>(label);
  const int64_t G = (int64_t)gridDim.x * blockDim.x;
  // kFbScanDepth groups in flight per lane
  for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)); base < nq;
       base += kFbScanDepth * G) {
    uint4 q[kFbScanDepth];
#pragma unroll
    for (int u = 0; u < kFbScanDepth; u++) {
      const int64_t i = base + u * G + lane;
      q[u] = i < nq ? __ldcs(l4 + i) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < kFbScanDepth; u++) {
      if (__ballot_sync(0xffffffffu, (q[u].x | q[u].y | q[u].z | q[u].w) != 0) == 0) continue;
      const uint32_t v = (uint32_t)(4 * (base + u * G + lane));
      scan_group(q[u], v, X, XY, n, lane, w);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x < 32) {  // the last nvol % 4 labels
    const int64_t v = 4 * nq + lane;
    scan_label(v < nvol ? label[v] : 0u, (uint32_t)v, X, XY, n, lane, w);
  }
}

// Exclusive scan of `count(i)` over i < n by one block of 1024 threads (contiguous chunks per
// thread); out[i] = sum of the counts before i, returns the total to every thread.
template <typename T, typename F>
__device__ T block_scan_1024(int32_t n, F count, T* out) {
  __shared__ T part[1024];
  const int t = threadIdx.x;
  const int per = (n + 1023) / 1024;
  const int a = min(n, t * per), b = min(n, a + per);
  T sum = 0;
  for (int i = a; i < b; i++) sum += count(i);
  part[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const T v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  T run = part[t] - sum;
  for (int i = a; i < b; i++) {
    out[i] = run;
    run += count(i);
  }
  const T total = part[1023];
  __syncthreads();
  return total;
}

__global__ void __launch_bounds__(1024) k_fb_ptr(int32_t n, FbWork w) {
  const int64_t total = block_scan_1024<int64_t>(n, [&](int i) { return (int64_t)w.cnt[i]; }, w.uptr);
  if (threadIdx.x == 0) w.uptr[n] = total;
}

__global__ void __launch_bounds__(256) k_fb_group(const uint32_t* __restrict__ label, const uint16_t* __restrict__ raw,
                                                  int32_t X, int32_t Y, int32_t n, FbWork w) {
  const int lane = threadIdx.x & 31;
  const int s = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (s >= n) return;
  const FbBox bx = w.box[s];
  const uint32_t want = (uint32_t)s + 1u;
  int64_t at = w.uptr[s];
  if (at == w.uptr[s + 1]) return;  // no voxels: no box
  const unsigned below = (1u << lane) - 1u;
  if (bx.hi[0] - bx.lo[0] < 32) {  // one chunk per row: four rows' labels in flight
    const int32_t x = bx.lo[0] + lane;
    const bool xin = x <= bx.hi[0];
    for (int32_t z = bx.lo[2]; z <= bx.hi[2]; z++)
      for (int32_t y = bx.lo[1]; y <= bx.hi[1]; y += 4) {
        uint32_t l[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
          l[u] = (xin && y + u <= bx.hi[1]) ? label[((int64_t)z * Y + y + u) * X + x] : 0u;
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const bool in = l[u] == want;
          const unsigned m = __ballot_sync(0xffffffffu, in);
          if (in) {
            const int64_t p = at + __popc(m & below), v = ((int64_t)z * Y + y + u) * X + x;
            w.ulin[p] = (uint32_t)v;
            w.uval[p] = raw[v];
          }
          at += __popc(m);
        }
      }
    if (lane == 0 && at != w.uptr[s + 1]) atomicOr(&w.stat->flags, 4u);  // box and count disagree
    return;
  }
  for (int32_t z = bx.lo[2]; z <= bx.hi[2]; z++)
    for (int32_t y = bx.lo[1]; y <= bx.hi[1]; y++) {
      const int64_t row = ((int64_t)z * Y + y) * X;
      for (int32_t x0 = bx.lo[0]; x0 <= bx.hi[0]; x0 += 32) {
        const int32_t x = x0 + lane;
        const bool in = x <= bx.hi[0] && label[row + x] == want;
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) {
          const int64_t p = at + __popc(m & below);
          w.ulin[p] = (uint32_t)(row + x);
          w.uval[p] = raw[row + x];
        }
        at += __popc(m);
      }
    }
  if (lane == 0 && at != w.uptr[s + 1]) atomicOr(&w.stat->flags, 4u);  // box and count disagree
}

// List form: a warp per supervoxel checks its list (ascending linear indices inside the
// volume; else the lists are flagged inconsistent) and takes its count and box.
__global__ void __launch_bounds__(256) k_fbl_boxes(int32_t X, int32_t Y, int64_t nvol, int64_t n_list, int32_t n,
                                                   FbWork w) {
  const int lane = threadIdx.x & 31;
  const int s = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (s >= n) return;
  const int64_t a = w.uptr[s], b = w.uptr[s + 1];
  if (a < 0 || b < a || b > n_list || b - a > 0x7fffffff) {  // nothing of such a list is read
    if (lane == 0) {
      atomicOr(&w.stat->flags, 4u);
      w.cnt[s] = 0;
    }
    return;
  }
  const uint32_t XY = (uint32_t)X * (uint32_t)Y;
  int32_t lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, hi[3] = {-1, -1, -1};
  bool bad = false;
  for (int64_t i = a + lane; i < b; i += 32) {
    const uint32_t v = w.ulin[i];
    bad |= (int64_t)v >= nvol || (i > a && w.ulin[i - 1] >= v);
    const uint32_t zz = v / XY, r = v - zz * XY, yy = r / (uint32_t)X;
    const int32_t c[3] = {(int32_t)(r - yy * (uint32_t)X), (int32_t)yy, (int32_t)zz};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      lo[d] = min(lo[d], c[d]);
      hi[d] = max(hi[d], c[d]);
    }
  }
  const bool any_bad = __any_sync(0xffffffffu, bad);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
    hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
  }
  if (lane == 0) {
    if (any_bad) atomicOr(&w.stat->flags, 4u);
    w.cnt[s] = (int32_t)(b - a);
    for (int d = 0; d < 3; d++) {
      w.box[s].lo[d] = lo[d];
      w.box[s].hi[d] = hi[d];
    }
  }
}

// The k-th smallest value (0-based) from a 256-bin histogram, by one warp: each lane holds 8
// bins, a scan over the lanes finds the lane holding it.  0 <= k < the histogram's total.
__device__ void warp_hist_select(const int32_t* h, int32_t k, int32_t* bucket, int32_t* rest) {
  const int lane = threadIdx.x & 31;
  int32_t c[8], sum = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    c[i] = h[lane * 8 + i];
    sum += c[i];
  }
  int32_t inc = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  int32_t run = inc - sum;
  if (run <= k && k < inc) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if (run + c[i] > k) {
        *bucket = lane * 8 + i;
        *rest = k - run;
        break;
      }
      run += c[i];
    }
  }
}

constexpr int kFbMaskWords = 2048;  // bounding boxes up to 65536 voxels flood in shared memory

// A linear index's coordinates, with the precomputed divisions of `o`.
__device__ __forceinline__ void decode(uint32_t v, uint32_t X, uint32_t XY, const FbOffsets& o, int32_t* x,
                                       int32_t* y, int32_t* z) {
  const uint32_t zz = div_by_magic(v, o.mxy, o.lxy), r = v - zz * XY, yy = div_by_magic(r, o.mx, o.lx);
  *x = (int32_t)(r - yy * X), *y = (int32_t)yy, *z = (int32_t)zz;
}

template <bool kLists>
__global__ void __launch_bounds__(kFbTrimThreads) k_fb_trim(const uint32_t* __restrict__ label,
                                                            const uint16_t* __restrict__ raw, int64_t nvol,
                                                            int32_t X, int32_t Y, int32_t Z, int32_t n,
                                                            int32_t max_size, float max_pct, int32_t min_size,
                                                            FbOffsets off, FbWork w) {
  __shared__ int32_t h_hi[256], h_lo1[256], h_lo2[256], h_ot[256];
  __shared__ float s_sumb[256];
  __shared__ int32_t s_wb[256];
  __shared__ uint32_t s_min, s_max, s_seed, s_tail;
  __shared__ int32_t s_b1, s_r1, s_b2, s_r2, s_l1, s_l2, s_rr, s_best;
  __shared__ float s_mm;
  __shared__ uint32_t s_cand[kFbMaskWords], s_reach[kFbMaskWords];
  const int s = blockIdx.x, t = threadIdx.x, lane = t & 31;
  if (w.stat->flags) return;
  const int64_t a = w.uptr[s];
  const int32_t N = (int32_t)(w.uptr[s + 1] - a);
  const uint32_t* lin = w.ulin + a;
  const uint16_t* val = w.uval + a;
  uint8_t* keep = w.ukeep + a;
  if (N == 0) {
    if (t == 0) {
      w.tcnt[s] = 0;
      w.thr[s] = 0;
    }
    return;
  }
  const uint32_t uX = (uint32_t)X, XY = (uint32_t)X * (uint32_t)Y;
  h_hi[t] = 0;
  h_lo1[t] = 0;
  h_lo2[t] = 0;
  h_ot[t] = 0;
  if (t == 0) {
    s_min = 0xffffffffu;
    s_max = 0;
    s_seed = 0xffffffffu;
    s_tail = 0;
    s_b1 = s_b2 = 255;
    s_r1 = s_r2 = s_l1 = s_l2 = s_rr = 0;
  }
  __syncthreads();
  // pass 1: range and the high bytes
  uint32_t mn = 0xffffffffu, mx = 0;
  for (int32_t i = t; i < N; i += kFbTrimThreads) {
    const uint32_t v = val[i];
    mn = min(mn, v);
    mx = max(mx, v);
    atomicAdd(&h_hi[v >> 8], 1);
  }
  atomicMin(&s_min, mn);
  atomicMax(&s_max, mx);
  __syncthreads();
  const int32_t k1 = max(0, N - max_size);
  int32_t k2 = __float2int_rz(__fmul_rn(__fsub_rn(1.0f, max_pct), (float)N));
  k2 = min(max(k2, 0), N - 1);  // the reference reads past the end only for max_pct < 1/N
  if (t < 32) {
    warp_hist_select(h_hi, k1, &s_b1, &s_r1);
    warp_hist_select(h_hi, k2, &s_b2, &s_r2);
    if (t == 0) s_mm = __fdiv_rn(255.0f, __fsub_rn((float)s_max, (float)s_min));
  }
  __syncthreads();
  const float fmin = (float)s_min, mm = s_mm;
  const bool otsu = isfinite(mm);
  const int32_t b1 = s_b1, b2 = s_b2;
  // pass 2: low bytes inside the two buckets, Otsu's histogram, the first brightest voxel
  for (int32_t i = t; i < N; i += kFbTrimThreads) {
    const uint32_t v = val[i];
    if ((int32_t)(v >> 8) == b1) atomicAdd(&h_lo1[v & 255], 1);
    if ((int32_t)(v >> 8) == b2) atomicAdd(&h_lo2[v & 255], 1);
    if (otsu) {
      const int b = __float2int_rz(__fmul_rn(__fsub_rn((float)v, fmin), mm));
      atomicAdd(&h_ot[min(b, 255)], 1);
    }
    if (v == s_max) atomicMin(&s_seed, (uint32_t)i);
  }
  __syncthreads();
  // Otsu's running sums over the bins (thread t = bin t): the class weights by a block scan of
  // the counts, the class sums of bin * count in the reference's FP32 order.  When their total
  // is below 2^24 every FP32 partial sum is an exact integer, so the scan's integers are those
  // bits; larger supervoxels sum in order on one thread.
  {
    const int64_t hb = h_ot[t], tb = (int64_t)t * hb;
    int64_t w_inc = hb, s_inc = tb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t yw = __shfl_up_sync(0xffffffffu, w_inc, o), ys = __shfl_up_sync(0xffffffffu, s_inc, o);
      if (lane >= o) {
        w_inc += yw;
        s_inc += ys;
      }
    }
    __shared__ int64_t s_ws[kFbTrimThreads / 32], s_ss[kFbTrimThreads / 32];
    if (lane == 31) {
      s_ws[t >> 5] = w_inc;
      s_ss[t >> 5] = s_inc;
    }
    __syncthreads();
    int64_t w_before = 0, s_before = 0, s_total = 0;
#pragma unroll
    for (int q = 0; q < kFbTrimThreads / 32; q++) {
      if (q < (t >> 5)) {
        w_before += s_ws[q];
        s_before += s_ss[q];
      }
      s_total += s_ss[q];
    }
    s_wb[t] = (int32_t)(w_before + w_inc);
    if (s_total < (1 << 24)) {
      s_sumb[t] = (float)(s_before + s_inc);
    } else if (t == 0) {
      float sum_b = 0.0f;
      for (int bin = 0; bin < 256; bin++) {
        sum_b = __fadd_rn(sum_b, (float)(bin * h_ot[bin]));
        s_sumb[bin] = sum_b;
      }
    }
  }
  __syncthreads();
  if (t < 32) {
    warp_hist_select(h_lo1, s_r1, &s_l1, &s_rr);
    warp_hist_select(h_lo2, s_r2, &s_l2, &s_rr);
    // the bin of the largest between-class variance (the first of equals; 0 if none is > 0)
    float best_v = 0.0f;
    int32_t best_b = 0x7fffffff;
    if (otsu) {
      const float sum = s_sumb[255];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int bin = lane * 8 + i;
        const int32_t wb = s_wb[bin], wf = N - wb;
        if (wb > 0 && wf > 0) {
          const float sb = s_sumb[bin];
          const float m_b = __fdiv_rn(sb, (float)wb), m_f = __fdiv_rn(__fsub_rn(sum, sb), (float)wf);
          const float d = __fsub_rn(m_b, m_f);
          const float var = __fmul_rn(__fmul_rn(__fmul_rn((float)wb, (float)wf), d), d);
          if (var > best_v) {
            best_v = var;
            best_b = bin;
          }
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, best_v, o);
      const int32_t ob = __shfl_xor_sync(0xffffffffu, best_b, o);
      if (ov > best_v || (ov == best_v && ob < best_b)) {
        best_v = ov;
        best_b = ob;
      }
    }
    if (t == 0) {
      float t3 = -FLT_MAX;
      if (otsu) t3 = __fadd_rn(__fdiv_rn((float)(best_v > 0.0f ? best_b : 0), mm), fmin);
      float thr = (float)((b1 << 8) | s_l1);
      const float v2 = (float)((b2 << 8) | s_l2);
      if (v2 > thr) thr = v2;
      if (t3 > thr) thr = t3;
      const uint32_t th = (uint32_t)(uint16_t)__float2uint_rz(thr);
      w.thr[s] = th;
      s_best = (int32_t)th;
    }
  }
  __syncthreads();
  // the flood from the brightest voxel: a voxel joins when it carries this label, is brighter
  // than the threshold and was not reached yet.  Neighbours are the reference's linear-index
  // offsets: inside the volume they are the coordinate steps; across an x or y border they wrap
  // into the next row or slice, and those are decoded from the linear index.
  const uint32_t th = (uint32_t)s_best;
  const FbBox bx = w.box[s];
  const int32_t bw = bx.hi[0] - bx.lo[0] + 1, bh = bx.hi[1] - bx.lo[1] + 1, bd = bx.hi[2] - bx.lo[2] + 1;
  const bool shared_path = (int64_t)bw * bh * bd <= 32 * kFbMaskWords;
  uint32_t* q = w.queue + a;
  if (shared_path) {
    const int32_t words = (bw * bh * bd + 31) / 32;
    for (int i = t; i < words; i += kFbTrimThreads) s_cand[i] = s_reach[i] = 0u;
    __syncthreads();
    for (int32_t i = t; i < N; i += kFbTrimThreads)
      if (val[i] > th) {
        int32_t x, y, z;
        decode(lin[i], uX, XY, off, &x, &y, &z);
        const int32_t li = (x - bx.lo[0]) + bw * ((y - bx.lo[1]) + bh * (z - bx.lo[2]));
        atomicOr(&s_cand[li >> 5], 1u << (li & 31));
      }
    __syncthreads();
    if (t == 0 && val[s_seed] > th) {
      int32_t x, y, z;
      decode(lin[s_seed], uX, XY, off, &x, &y, &z);
      const int32_t li = (x - bx.lo[0]) + bw * ((y - bx.lo[1]) + bh * (z - bx.lo[2]));
      s_reach[li >> 5] |= 1u << (li & 31);
      q[0] = lin[s_seed];
      s_tail = 1;
    }
  } else if (t == 0 && val[s_seed] > th) {
    const uint32_t v = lin[s_seed];
    atomicOr(&w.bits[v >> 5], 1u << (v & 31));
    q[0] = v;
    s_tail = 1;
  }
  __syncthreads();
  const uint32_t want = (uint32_t)s + 1u;
  uint32_t head = 0;
  for (;;) {
    const uint32_t tail = s_tail;
    __syncthreads();
    if (head == tail) break;
    for (uint32_t i = head + t; i < tail; i += kFbTrimThreads) {
      const uint32_t v = q[i];
      if (shared_path) {
        int32_t x, y, z;
        decode(v, uX, XY, off, &x, &y, &z);
        for (int j = 0; j < off.n; j++) {
          int32_t tx = x + off.d[j][0], ty = y + off.d[j][1], tz = z + off.d[j][2];
          if (tx < 0 || tx >= X || ty < 0 || ty >= Y) {  // wraps: where the linear offset lands
            const int64_t nb = (int64_t)v + off.off[j];
            if (nb < 0 || nb >= nvol) continue;
            decode((uint32_t)nb, uX, XY, off, &tx, &ty, &tz);
          } else if (tz < 0 || tz >= Z) {
            continue;
          }
          const int32_t lx = tx - bx.lo[0], ly = ty - bx.lo[1], lz = tz - bx.lo[2];
          if (lx < 0 || lx >= bw || ly < 0 || ly >= bh || lz < 0 || lz >= bd) continue;
          const int32_t li = lx + bw * (ly + bh * lz);
          const uint32_t bit = 1u << (li & 31);
          if (!(s_cand[li >> 5] & bit)) continue;
          if (atomicOr(&s_reach[li >> 5], bit) & bit) continue;
          q[atomicAdd(&s_tail, 1u)] = (uint32_t)tx + uX * (uint32_t)ty + XY * (uint32_t)tz;
        }
      } else {
        for (int j = 0; j < off.n; j++) {
          const int64_t nb = (int64_t)v + off.off[j];
          if (nb < 0 || nb >= nvol) continue;
          if (kLists) {
            // a voxel of this supervoxel (its ascending list, as lower_bound finds it there)
            // brighter than the threshold
            int32_t lo = 0, hi = N;
            while (lo < hi) {
              const int32_t mid = (lo + hi) >> 1;
              if ((int64_t)lin[mid] < nb)
                lo = mid + 1;
              else
                hi = mid;
            }
            if (lo >= N || (int64_t)lin[lo] != nb || val[lo] <= th) continue;
          } else if (label[nb] != want || raw[nb] <= th) {
            continue;
          }
          const uint32_t bit = 1u << (nb & 31);
          if (atomicOr(&w.bits[nb >> 5], bit) & bit) continue;
          q[atomicAdd(&s_tail, 1u)] = (uint32_t)nb;
        }
      }
    }
    head = tail;
    __syncthreads();
  }
  const int32_t kept = (int32_t)s_tail;
  // each list entry's verdict, for the centroid and the emission
  for (int32_t i = t; i < N; i += kFbTrimThreads) {
    const uint32_t v = lin[i];
    bool in;
    if (shared_path) {
      int32_t x, y, z;
      decode(v, uX, XY, off, &x, &y, &z);
      const int32_t li = (x - bx.lo[0]) + bw * ((y - bx.lo[1]) + bh * (z - bx.lo[2]));
      in = (s_reach[li >> 5] >> (li & 31)) & 1u;
    } else {  // the flood's bits were set by atomics at L2: read them there
      in = (__ldcg(&w.bits[v >> 5]) >> (v & 31)) & 1u;
    }
    keep[i] = in ? 1 : 0;
  }
  if (t == 0) w.tcnt[s] = kept;
  if (kept < min_size) return;
  __syncthreads();
  if (t >= 32) return;
  // warp 0: the centroid in list order (FP32, as the reference sums it) and the range of the
  // background-subtracted values.  Each lane forms its voxel's products and stages them (zeros
  // for a voxel not kept: every term is non-negative, so adding +0 leaves a sum's bits as they
  // are); the four running sums then add the group's 32 entries in lane order (list order), from
  // broadcast loads issued ahead of the additions, so the chains hold only the additions.
  __shared__ float4 st4[32];
  float sw = 0.0f, c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
  uint32_t smin = 0xffffffffu, smax = 0;
  for (int32_t i0 = 0; i0 < N; i0 += 32) {
    const int32_t i = i0 + lane;
    bool in = false;
    uint32_t v = 0, r = 0;
    if (i < N) {
      v = lin[i];
      r = val[i];
      in = keep[i] != 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, in);
    float I = 0.0f, px = 0.0f, py = 0.0f, pz = 0.0f;
    if (in) {
      int32_t x, y, z;
      decode(v, uX, XY, off, &x, &y, &z);
      I = (float)r;
      px = __fmul_rn(I, (float)x);
      py = __fmul_rn(I, (float)y);
      pz = __fmul_rn(I, (float)z);
      const uint32_t sub = (uint16_t)(r - th);
      smin = min(smin, sub);
      smax = max(smax, sub);
    }
    st4[lane] = make_float4(I, px, py, pz);
    __syncwarp();
    if (m) {
#pragma unroll
      for (int p = 0; p < 32; p++) {
        const float4 e = st4[p];
        sw = __fadd_rn(sw, e.x);
        c0 = __fadd_rn(c0, e.y);
        c1 = __fadd_rn(c1, e.z);
        c2 = __fadd_rn(c2, e.w);
      }
    }
    __syncwarp();
  }
  for (int o = 16; o > 0; o >>= 1) {
    smin = min(smin, __shfl_xor_sync(0xffffffffu, smin, o));
    smax = max(smax, __shfl_xor_sync(0xffffffffu, smax, o));
  }
  if (lane == 0) {
    const bool zero = (double)sw < 1e-5;
    w.tcent[3 * s] = zero ? 0.0f : __fdiv_rn(c0, sw);
    w.tcent[3 * s + 1] = zero ? 0.0f : __fdiv_rn(c1, sw);
    w.tcent[3 * s + 2] = zero ? 0.0f : __fdiv_rn(c2, sw);
    atomicMin(&w.stat->sub_min, smin);
    atomicMax(&w.stat->sub_max, smax);
    atomicAdd(&w.stat->kept_vox, (unsigned long long)kept);
  }
}

// The reference erases each index of the ascending list E (m of n), from the last, by trading
// places with the current last supervoxel.  Step i (erasing E[i]) swaps with position n-m+i,
// whose content is then: the supervoxel at n-m+i if that index is kept, else -- it was itself
// erased, as E[j] for some j > i, and received position n-m+j's content -- the content of
// n-m+j.  These chains only climb, so output p is p when kept, else the end of the chain from
// n-m+rank(p).
__global__ void __launch_bounds__(1024) k_fb_order(int32_t n, int64_t nvol, int32_t min_size, FbWork w) {
  __shared__ int s_changed;
  const int t = threadIdx.x;
  if (w.stat->flags) return;
  const int32_t m = block_scan_1024<int32_t>(n, [&](int i) { return (int32_t)(w.tcnt[i] < min_size); }, w.rank);
  FbStat* st = w.stat;
  if (m >= n) {
    if (t == 0) {
      st->flags |= 2u;
      st->n_sv = 0;
      st->n_vox = 0;
    }
    return;
  }
  const int32_t S = n - m;
  for (int32_t q = S + t; q < n; q += 1024) w.nxt[q] = w.tcnt[q] < min_size ? S + w.rank[q] : q;
  __syncthreads();
  for (int round = 0; round < 40; round++) {
    if (t == 0) s_changed = 0;
    __syncthreads();
    int changed = 0;
    for (int32_t q = S + t; q < n; q += 1024) {
      const int32_t j = w.nxt[q], k = w.nxt[j];
      if (k != j) {
        w.nxt[q] = k;
        changed = 1;
      }
    }
    if (changed) s_changed = 1;
    __syncthreads();
    if (!s_changed) break;
    __syncthreads();
  }
  for (int32_t p = t; p < S; p += 1024) w.order[p] = w.tcnt[p] < min_size ? w.nxt[S + w.rank[p]] : p;
  if (t == 0) {
    const int64_t N = (int64_t)st->kept_vox;
    double lo = (double)st->sub_min, hi = (double)st->sub_max;
    if (N < nvol) {
      lo = lo < 0.0 ? lo : 0.0;
      hi = hi > 0.0 ? hi : 0.0;
    }
    double f = 1.0;
    f /= hi - lo;
    st->fct = f;
    st->shift = 0.0 / f - lo;
    st->scaled = hi != lo;
    st->n_sv = S;
    st->n_vox = N;
  }
}

// Output CSR (one block) over the output order.
__global__ void __launch_bounds__(1024) k_fb_csr(int64_t max_vox, int32_t max_sv, FbWork w, int64_t* lptr) {
  const FbStat* st = w.stat;
  if (st->flags) return;
  const int32_t S = st->n_sv;
  if (S > max_sv || st->n_vox > max_vox) return;
  const int64_t total = block_scan_1024<int64_t>(S, [&](int p) { return (int64_t)w.tcnt[w.order[p]]; }, lptr);
  if (threadIdx.x == 0) lptr[S] = total;
}

__global__ void __launch_bounds__(256) k_fb_emit(int32_t X, int32_t Y, int64_t max_vox, int32_t max_sv, FbWork w,
                                                 const int64_t* __restrict__ lptr, float* query, float* img,
                                                 float* cent, uint16_t* thr_out) {
  const FbStat* st = w.stat;
  const int lane = threadIdx.x & 31;
  const int p = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (st->flags) return;
  const int32_t S = st->n_sv;
  const int64_t N = st->n_vox;
  if (p >= S || S > max_sv || N > max_vox) return;
  const int s = w.order[p];
  const uint32_t th = w.thr[s];
  const bool scaled = st->scaled;
  const double f = st->fct, sh = st->shift;
  const int64_t a = w.uptr[s];
  const int32_t n = (int32_t)(w.uptr[s + 1] - a);
  int64_t at = lptr[p];
  const unsigned below = (1u << lane) - 1u;
  for (int32_t i0 = 0; i0 < n; i0 += 32) {
    const int32_t i = i0 + lane;
    bool in = false;
    uint32_t v = 0;
    if (i < n) {
      v = w.ulin[a + i];
      in = w.ukeep[a + i] != 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, in);
    if (in) {
      const int64_t o = at + __popc(m & below);
      query[o] = (float)(v % (uint32_t)X);
      query[N + o] = (float)((v / (uint32_t)X) % (uint32_t)Y);
      query[2 * N + o] = (float)(v / ((uint32_t)X * (uint32_t)Y));
      const float sub = (float)(uint16_t)(w.uval[a + i] - th);
      img[o] = scaled ? (float)__dmul_rn(f, __dadd_rn((double)sub, sh)) : sub;
    }
    at += __popc(m);
  }
  if (lane == 0) {
    for (int d = 0; d < 3; d++) cent[(int64_t)d * S + p] = w.tcent[3 * s + d];
    if (thr_out) thr_out[p] = (uint16_t)th;
  }
}

int fb_offsets(int32_t conn, const int32_t dims[3], FbOffsets* o) {
  const int64_t X = dims[0], XY = (int64_t)dims[0] * dims[1];
  int rz, rxy;
  switch (conn) {
    case 4:
    case 8:
      rz = 0, rxy = 1;
      break;
    case 6:
    case 26:
      rz = 1, rxy = 1;
      break;
    case 74:
      rz = 1, rxy = 2;
      break;
    default:
      return 0;
  }
  int n = 0;
  for (int z = -rz; z <= rz; z++)
    for (int y = -rxy; y <= rxy; y++)
      for (int x = -rxy; x <= rxy; x++) {
        if (!(x || y || z)) continue;
        if ((conn == 4 || conn == 6) && (x != 0) + (y != 0) + (z != 0) != 1) continue;  // faces only
        o->off[n] = x + X * y + XY * z;
        o->d[n][0] = (int8_t)x, o->d[n][1] = (int8_t)y, o->d[n][2] = (int8_t)z;
        n++;
      }
  o->n = n;
  div_magic((uint32_t)X, &o->mx, &o->lx);
  div_magic((uint32_t)XY, &o->mxy, &o->lxy);
  return n;
}

}  // namespace
}  // namespace tgmm

using namespace tgmm;

extern "C" void tgmm_frame_build_default_params(TgmmFrameBuildParams* p) {
  if (!p) return;
  p->max_nuclei_size = 3000;
  p->max_percentile = 0.4f;
  p->conn3d = 6;
  p->min_nuclei_size = 50;
}

extern "C" int64_t tgmm_frame_build_bytes(const int32_t dims[3], int32_t n_labels) {
  if (!dims || dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || n_labels < 1) return -1;
  const int64_t nvol = (int64_t)dims[0] * dims[1] * dims[2];
  FbWork w;
  return (int64_t)carve(nullptr, nvol, n_labels, &w);
}

namespace {
// The build; with `ev` (TGMM_FRAME_BUILD_STAGES + 1 events) an event is recorded before the
// first step and after each.
int frame_build(const uint16_t* raw, const uint32_t* label, const int32_t dims[3], int32_t n_labels,
                const TgmmFrameBuildParams* p, void* workspace, int64_t workspace_bytes, float* query, float* img,
                float* cent, int64_t* lptr, uint16_t* thr, int64_t max_vox, int32_t max_sv, int64_t* n_vox_out,
                int32_t* n_sv_out, cudaStream_t st, cudaEvent_t* ev) {
  static const char* kWhat = "tgmm_frame_build";
  if (!raw || !label || !dims || !p || !workspace || !query || !img || !cent || !lptr || !n_vox_out || !n_sv_out ||
      n_labels < 1 || max_vox < 0 || max_sv < 0)
    return report_error(TGMM_ERR_INVALID_ARG, kWhat, cudaSuccess);
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1)
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build: dimensions", cudaSuccess);
  const int64_t nvol = (int64_t)dims[0] * dims[1] * dims[2];
  if (nvol >= ((int64_t)1 << 32) || n_labels > (1 << 24))
    return report_error(TGMM_ERR_BAD_SIZE, "tgmm_frame_build: more than 2^32 voxels or 2^24 labels", cudaSuccess);
  if (p->max_nuclei_size < 0 || !(p->max_percentile >= 0.0f && p->max_percentile <= 1.0f))
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build: trimming parameters", cudaSuccess);
  if (((uintptr_t)label & 15) != 0)
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build: label volume not 16-byte aligned", cudaSuccess);
  FbOffsets off;
  if (!fb_offsets(p->conn3d, dims, &off))
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build: conn3d must be 4, 6, 8, 26 or 74", cudaSuccess);
  FbWork w;
  if ((int64_t)carve(nullptr, nvol, n_labels, &w) > workspace_bytes)
    return report_error(TGMM_ERR_BAD_SIZE, "tgmm_frame_build: workspace smaller than tgmm_frame_build_bytes",
                        cudaSuccess);
  carve((char*)workspace, nvol, n_labels, &w);
  const int32_t X = dims[0], Y = dims[1], n = n_labels;
  int stage = 0;
  auto mark = [&]() {
    if (ev) cudaEventRecord(ev[stage++], st);
  };
  mark();
  cudaError_t e = cudaMemsetAsync(w.bits, 0, 4 * (size_t)((nvol + 31) / 32), st);
  if (e != cudaSuccess) return report_error(TGMM_ERR_CUDA, kWhat, e);
  const unsigned warp_blocks = (unsigned)(((int64_t)n * 32 + 255) / 256);
  k_fb_init<<<(n + 255) / 256, 256, 0, st>>>(n, w);
  mark();
  // the scan: as many blocks as fit on the device at once (it strides over the volume)
  int dev = 0, sms = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fb_scan, 256, 0);
  const int64_t span = (nvol / 4 + 256 * kFbScanDepth - 1) / (256 * kFbScanDepth);
  const int64_t full = (int64_t)sms * (occ > 0 ? occ : 1);
  k_fb_scan<<<(unsigned)(span < 1 ? 1 : span < full ? span : full), 256, 0, st>>>(label, nvol, X, Y, n, w);
  mark();
  k_fb_ptr<<<1, 1024, 0, st>>>(n, w);
  mark();
  k_fb_group<<<warp_blocks, 256, 0, st>>>(label, raw, X, Y, n, w);
  mark();
  k_fb_trim<false><<<n, kFbTrimThreads, 0, st>>>(label, raw, nvol, X, Y, dims[2], n, p->max_nuclei_size,
                                                 p->max_percentile, p->min_nuclei_size, off, w);
  mark();
  k_fb_order<<<1, 1024, 0, st>>>(n, nvol, p->min_nuclei_size, w);
  mark();
  k_fb_csr<<<1, 1024, 0, st>>>(max_vox, max_sv, w, lptr);
  mark();
  k_fb_emit<<<warp_blocks, 256, 0, st>>>(X, Y, max_vox, max_sv, w, lptr, query, img, cent, thr);
  mark();
  FbStat h;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, w.stat, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return report_error(TGMM_ERR_CUDA, kWhat, e);
  if (h.flags & 1u) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build: a label above n_labels", cudaSuccess);
  if (h.flags & 4u)
    return report_error(TGMM_ERR_DEVICE_FLAG, "tgmm_frame_build: supervoxel lists inconsistent", cudaSuccess);
  *n_vox_out = h.n_vox;
  *n_sv_out = h.n_sv;
  if (h.flags & 2u)
    return report_error(TGMM_ERR_NO_SUPERVOXEL, "tgmm_frame_build: every supervoxel was erased", cudaSuccess);
  if (h.n_vox > max_vox || h.n_sv > max_sv)
    return report_error(TGMM_ERR_BAD_SIZE, "tgmm_frame_build: more voxels or supervoxels than the outputs hold",
                        cudaSuccess);
  return TGMM_OK;
}
}  // namespace

namespace {
// The list form: the supervoxels' lists as the segmentation holds them (each supervoxel's
// voxels in ascending linear index with their raw values, CSR over the supervoxels), read in
// place; the steps after the grouping are the volume form's.
int frame_build_lists(const uint32_t* lin, const uint16_t* val, const int64_t* lists_ptr, int64_t n_list,
                      const int32_t dims[3], int32_t n_labels, const TgmmFrameBuildParams* p, void* workspace,
                      int64_t workspace_bytes, float* query, float* img, float* cent, int64_t* lptr, uint16_t* thr,
                      int64_t max_vox, int32_t max_sv, int64_t* n_vox_out, int32_t* n_sv_out, cudaStream_t st,
                      float* stage_ms) {
  static const char* kWhat = "tgmm_frame_build_lists";
  if (!lists_ptr || !dims || !p || !workspace || !query || !img || !cent || !lptr || !n_vox_out || !n_sv_out ||
      n_labels < 1 || n_list < 0 || (n_list > 0 && (!lin || !val)) || max_vox < 0 || max_sv < 0)
    return report_error(TGMM_ERR_INVALID_ARG, kWhat, cudaSuccess);
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1)
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build_lists: dimensions", cudaSuccess);
  const int64_t nvol = (int64_t)dims[0] * dims[1] * dims[2];
  if (nvol >= ((int64_t)1 << 32) || n_labels > (1 << 24) || n_list > nvol)
    return report_error(TGMM_ERR_BAD_SIZE,
                        "tgmm_frame_build_lists: more than 2^32 voxels, 2^24 labels or list entries than voxels",
                        cudaSuccess);
  if (p->max_nuclei_size < 0 || !(p->max_percentile >= 0.0f && p->max_percentile <= 1.0f))
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build_lists: trimming parameters", cudaSuccess);
  FbOffsets off;
  if (!fb_offsets(p->conn3d, dims, &off))
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build_lists: conn3d must be 4, 6, 8, 26 or 74",
                        cudaSuccess);
  FbWork w;
  if ((int64_t)carve(nullptr, nvol, n_labels, &w, n_list) > workspace_bytes)
    return report_error(TGMM_ERR_BAD_SIZE,
                        "tgmm_frame_build_lists: workspace smaller than tgmm_frame_build_lists_bytes", cudaSuccess);
  carve((char*)workspace, nvol, n_labels, &w, n_list);
  w.uptr = const_cast<int64_t*>(lists_ptr);
  w.ulin = const_cast<uint32_t*>(lin);
  w.uval = const_cast<uint16_t*>(val);
  const int32_t X = dims[0], Y = dims[1], n = n_labels;
  // with stage_ms: an event before the first step and after each
  struct Events {
    cudaEvent_t e[TGMM_FRAME_BUILD_STAGES + 1] = {};
    int n = 0;
    ~Events() {
      for (int i = 0; i < n; i++) cudaEventDestroy(e[i]);
    }
  } evs;
  if (stage_ms)
    for (; evs.n <= TGMM_FRAME_BUILD_STAGES; evs.n++)
      if (cudaEventCreate(&evs.e[evs.n]) != cudaSuccess)
        return report_error(TGMM_ERR_CUDA, "tgmm_frame_build_lists: events", cudaGetLastError());
  int stage = 0;
  auto mark = [&]() {
    if (stage_ms) cudaEventRecord(evs.e[stage++], st);
  };
  mark();
  cudaError_t e = cudaMemsetAsync(w.bits, 0, 4 * (size_t)((nvol + 31) / 32), st);
  if (e != cudaSuccess) return report_error(TGMM_ERR_CUDA, kWhat, e);
  const unsigned warp_blocks = (unsigned)(((int64_t)n * 32 + 255) / 256);
  k_fb_init<<<(n + 255) / 256, 256, 0, st>>>(n, w);
  mark();
  k_fbl_boxes<<<warp_blocks, 256, 0, st>>>(X, Y, nvol, n_list, n, w);
  mark();
  mark();  // no CSR to build: the lists come with theirs
  mark();  // no grouping: the lists are grouped
  k_fb_trim<true><<<n, kFbTrimThreads, 0, st>>>(nullptr, nullptr, nvol, X, Y, dims[2], n, p->max_nuclei_size,
                                                p->max_percentile, p->min_nuclei_size, off, w);
  mark();
  k_fb_order<<<1, 1024, 0, st>>>(n, nvol, p->min_nuclei_size, w);
  mark();
  k_fb_csr<<<1, 1024, 0, st>>>(max_vox, max_sv, w, lptr);
  mark();
  k_fb_emit<<<warp_blocks, 256, 0, st>>>(X, Y, max_vox, max_sv, w, lptr, query, img, cent, thr);
  mark();
  FbStat h;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, w.stat, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return report_error(TGMM_ERR_CUDA, kWhat, e);
  if (stage_ms)
    for (int i = 0; i < TGMM_FRAME_BUILD_STAGES; i++) cudaEventElapsedTime(&stage_ms[i], evs.e[i], evs.e[i + 1]);
  if (h.flags & 4u)
    return report_error(TGMM_ERR_DEVICE_FLAG,
                        "tgmm_frame_build_lists: a list is not ascending inside the volume, or the CSR is invalid",
                        cudaSuccess);
  *n_vox_out = h.n_vox;
  *n_sv_out = h.n_sv;
  if (h.flags & 2u)
    return report_error(TGMM_ERR_NO_SUPERVOXEL, "tgmm_frame_build_lists: every supervoxel was erased", cudaSuccess);
  if (h.n_vox > max_vox || h.n_sv > max_sv)
    return report_error(TGMM_ERR_BAD_SIZE,
                        "tgmm_frame_build_lists: more voxels or supervoxels than the outputs hold", cudaSuccess);
  return TGMM_OK;
}
}  // namespace

extern "C" int64_t tgmm_frame_build_lists_bytes(const int32_t dims[3], int32_t n_labels, int64_t n_list) {
  if (!dims || dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || n_labels < 1 || n_list < 0) return -1;
  const int64_t nvol = (int64_t)dims[0] * dims[1] * dims[2];
  FbWork w;
  return (int64_t)carve(nullptr, nvol, n_labels, &w, n_list);
}

extern "C" int tgmm_frame_build_lists(const uint32_t* lin, const uint16_t* val, const int64_t* lists_ptr,
                                      int64_t n_list, const int32_t dims[3], int32_t n_labels,
                                      const TgmmFrameBuildParams* p, void* workspace, int64_t workspace_bytes,
                                      float* query, float* img, float* cent, int64_t* lptr, uint16_t* thr,
                                      int64_t max_vox, int32_t max_sv, int64_t* n_vox_out, int32_t* n_sv_out,
                                      void* stream, float* stage_ms) {
  if (stage_ms)
    for (int i = 0; i < TGMM_FRAME_BUILD_STAGES; i++) stage_ms[i] = 0.0f;
  return frame_build_lists(lin, val, lists_ptr, n_list, dims, n_labels, p, workspace, workspace_bytes, query, img,
                           cent, lptr, thr, max_vox, max_sv, n_vox_out, n_sv_out, (cudaStream_t)stream, stage_ms);
}

extern "C" int tgmm_frame_build(const uint16_t* raw, const uint32_t* label, const int32_t dims[3], int32_t n_labels,
                                const TgmmFrameBuildParams* p, void* workspace, int64_t workspace_bytes, float* query,
                                float* img, float* cent, int64_t* lptr, uint16_t* thr, int64_t max_vox, int32_t max_sv,
                                int64_t* n_vox_out, int32_t* n_sv_out, void* stream) {
  return frame_build(raw, label, dims, n_labels, p, workspace, workspace_bytes, query, img, cent, lptr, thr, max_vox,
                     max_sv, n_vox_out, n_sv_out, (cudaStream_t)stream, nullptr);
}

extern "C" int tgmm_frame_build_timed(const uint16_t* raw, const uint32_t* label, const int32_t dims[3],
                                      int32_t n_labels, const TgmmFrameBuildParams* p, void* workspace,
                                      int64_t workspace_bytes, float* query, float* img, float* cent, int64_t* lptr,
                                      uint16_t* thr, int64_t max_vox, int32_t max_sv, int64_t* n_vox_out,
                                      int32_t* n_sv_out, void* stream, float* stage_ms) {
  if (!stage_ms) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_build_timed", cudaSuccess);
  cudaEvent_t ev[TGMM_FRAME_BUILD_STAGES + 1] = {};
  int created = 0, rc = TGMM_OK;
  for (; created <= TGMM_FRAME_BUILD_STAGES; created++)
    if (cudaEventCreate(&ev[created]) != cudaSuccess) {
      rc = report_error(TGMM_ERR_CUDA, "tgmm_frame_build_timed: events", cudaGetLastError());
      break;
    }
  if (rc == TGMM_OK)
    rc = frame_build(raw, label, dims, n_labels, p, workspace, workspace_bytes, query, img, cent, lptr, thr, max_vox,
                     max_sv, n_vox_out, n_sv_out, (cudaStream_t)stream, ev);
  for (int i = 0; i < TGMM_FRAME_BUILD_STAGES; i++) {
    stage_ms[i] = 0.0f;
    if (rc == TGMM_OK || rc == TGMM_ERR_BAD_SIZE || rc == TGMM_ERR_NO_SUPERVOXEL)
      cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
  }
  for (int i = 0; i < created; i++) cudaEventDestroy(ev[i]);
  return rc;
}
