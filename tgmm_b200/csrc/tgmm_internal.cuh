// tgmm_internal.cuh -- device-side data layout of a plan (all workspace of the EM),
// the per-frame descriptor/state records and the kernel entry points.
//
// Layout in HBM (capacities fixed at plan creation):
//   per Gaussian, SoA doubles  [component][max_gauss]: beta, nu, alpha, m[3], W[6],
//                              beta_o, nu_o, alpha_o, m_o[3], W_o[6], eLD[2], psiA[2]
//   per voxel                  the centred voxel stream [max_vox] float4 (e = x - c, I),
//                              written once per call, read by every log-likelihood pass
//   per supervoxel             moments [19][max_sv] doubles (centred at the supervoxel
//                              centroid: sum e, sum e e', sum I, sum I e, sum I e e'),
//                              cand/rnk [max_sv][5], ll partials [2][max_sv]
//   kNN grid                   per frame a uniform grid over the centroid bounding box
//                              (scaled space); per cell a count and kCellCap float centres
//   M-step buckets             [max_gauss][kBucketCap] (supervoxel, slot) positions
//   chunk tables               frame-aligned chunks of kGChunk Gaussians, so that every
//                              per-frame sum is a fixed-order sum of chunk partials.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tgmm_gmem.h"
#include "tgmm_math.cuh"

namespace tgmm {

constexpr int kJ = TGMM_J;
constexpr int kBucketCap = 32;   // M-step pairs per Gaussian held in the fast bucket
constexpr int kGChunk = 256;     // Gaussians per block in per-Gaussian kernels
constexpr int kMChunk = kGChunk / 2;  // Gaussians per block of the M-step (two per chunk)
constexpr int kSvPerBlockT = 128;  // supervoxels per block, thread-per-supervoxel kernels
constexpr int kWarpsPerBlockV = 8;   // warps per block, warp-per-supervoxel kernels
constexpr int kSvPerWarpV = 2;
constexpr int kSvPerBlockV = kWarpsPerBlockV * kSvPerWarpV;
constexpr int kNumMoments = 19;
constexpr int kFrameThreads = 1024;
constexpr int kMapSlices = 8;  // blocks per frame of the frame-map kernel
constexpr int kCellCap = 32;   // Gaussian centres per kNN grid cell
#ifndef TGMM_NBR
#define TGMM_NBR 8
#endif
#ifndef TGMM_REFS_PER_CELL
#define TGMM_REFS_PER_CELL 3
#endif
constexpr int kNbr = TGMM_NBR;  // Gaussians kept per supervoxel in its kNN neighbour list
constexpr int kRefsPerCell = TGMM_REFS_PER_CELL;  // kNN grid resolution: references per cell
static_assert(kNbr >= TGMM_J && kNbr <= 16, "a list holds the five candidates, at most four members per lane of 4");
constexpr int kEcStride = 12;  // doubles per E-step record

// moment component indices
enum : int {
  M_E0 = 0, M_E1, M_E2,                      // sum e
  M_EE00, M_EE01, M_EE02, M_EE11, M_EE12, M_EE22,  // sum e e'
  M_I,                                        // sum I
  M_IE0, M_IE1, M_IE2,                       // sum I e
  M_IEE00, M_IEE01, M_IEE02, M_IEE11, M_IEE12, M_IEE22  // sum I e e'
};

// device flags (per frame, OR-ed into FrameState::flags)
enum : int {
  F_BAD_CSR = 1,
  F_NAN_INPUT = 2,
  F_FEW_GAUSS = 4,
  F_BUCKET_OVERFLOW = 8,
  F_ASSIGN_OVERFLOW = 16,
  F_CELL_OVERFLOW = 32,
  F_STAGE_TIMEOUT = 64  // a voxel tile copy did not complete within its wait limit
};
static_assert(F_BAD_CSR == TGMM_FLAG_BAD_CSR && F_NAN_INPUT == TGMM_FLAG_NAN_INPUT &&
                  F_FEW_GAUSS == TGMM_FLAG_FEW_GAUSS && F_BUCKET_OVERFLOW == TGMM_FLAG_BUCKET_OVERFLOW &&
                  F_ASSIGN_OVERFLOW == TGMM_FLAG_ASSIGN_OVERFLOW && F_CELL_OVERFLOW == TGMM_FLAG_CELL_OVERFLOW &&
                  F_STAGE_TIMEOUT == TGMM_FLAG_STAGE_TIMEOUT,
              "the device flags are the public TgmmEmStats.device_flags bits");

struct FrameDesc {
  const float* query;
  const float* img;
  const float* cent;
  const int64_t* lptr;
  TgmmGaussian* gm;  // device AoS records of this frame
  // the caller's page-locked host records (their device-mapped address), copied into gm by
  // the call's graph beside the voxel work; nullptr when gm already holds the records
  const TgmmGaussian* gm_src;
  float* rnk_out;    // device, 5*n_sv, slot-major
  int32_t* ind_out;  // device, 5*n_sv, slot-major, frame-local Gaussian ids
  int64_t n_vox;
  int64_t vox_base;  // the frame's first voxel in the plan's centred voxel stream (vox4)
  int32_t n_sv, n_gauss;
  int32_t sv_base, g_base;
  int32_t cell_base, cell_budget;
  int32_t gchunk_base, n_gchunks;
  float scale[3];      // kNN distance scale
  float reg_scale[3];  // regularisation scale
  int32_t w4dof;
  double lambda_min, lambda_max, max_exc, tol;
  int32_t max_iter, ll_mode, ll_prec, frame_id;
};

struct FrameState {
  float lo[3];
  float h;
  float inv_h;
  int32_t dims[3];
  int32_t n_cells;
  int32_t iter;  // numIterEM of the reference: the next iteration to run (starts at 1)
  int32_t done;
  int32_t converged;
  int32_t flags;
  int32_t n_dead;
  double total_alpha;  // post-kill sum of alpha (the value the E-step and the ll use)
  double ln_alpha;     // ln(total_alpha)
  double psi_total[2];
  double ll, ll1, ll2, ll3;
  double ll_true, ll_ref;
  // order-free accumulation of the per-supervoxel log-likelihoods: integer parts and
  // 2^-40 fractions in 64-bit integers (true, as reference)
  long long ll_int[2];
  unsigned long long ll_frac[2];
  int32_t sv_done;   // supervoxels finished in this iteration's voxel pass
  int32_t blk_done;  // Gaussian chunks finished in this iteration's kill step
  // kNN neighbour lists: disp_cum bounds how far any live Gaussian's float centre has moved
  // (scaled units) since the call began, as the sum over iterations of the largest move of
  // one iteration; disp_max is the current iteration's largest move (float bits, rounded up)
  double disp_cum;
  uint32_t disp_max;
  int32_t knn_searches;  // supervoxel grid searches after the first iteration (list misses)
};

// Voxel tiles of the per-iteration voxel pass: kVoxTile voxels of a supervoxel per copy;
// the reference's kept window of a supervoxel's last 1024 voxels is its last kKeptTiles.
#ifndef TGMM_VOX_TILE
#define TGMM_VOX_TILE 256
#endif
constexpr int kVoxTile = TGMM_VOX_TILE;
constexpr int kKeptTiles = 1024 / kVoxTile;
constexpr int kOrderBuckets = 64;  // supervoxel order: tile counts 0..62, and 63 or more
static_assert(kVoxTile >= 32 && kVoxTile % 32 == 0 && 1024 % kVoxTile == 0, "tiles split the kept window evenly");

// Per-supervoxel stream record of the voxel pass, built once per call (k_moments).
// Tiles are aligned to the END of the supervoxel: tile 0 holds its first r0 voxels
// (1 <= r0 <= kVoxTile) and every later tile kVoxTile voxels, so the reference's kept
// window of the last 1024 voxels is exactly the last kKeptTiles tiles.  Component c (x, y, z,
// I) of tile 0 is the 16-byte aligned span [lo0[c], + n0[c]); of tile t >= 1 the span
// [lo1[c] + 4 kVoxTile (t - 1), + (nf[c] & 0xffff)).  The first voxel of tile 0 sits
// (nf[c] >> 16) & 3 floats into its span, that of the later tiles (nf[c] >> 20) & 3.
struct SvRec {
  unsigned long long lo0[4];
  unsigned long long lo1[4];
  unsigned n0[4];
  unsigned nf[4];
  int32_t ntiles, nv;
  int32_t frame, frame_nsv;
  float c0, c1, c2;
  int32_t r0;
};
static_assert(sizeof(SvRec) == 128, "SvRec is eight 16-byte chunks");

// Per-supervoxel record of the log-likelihood pass: where the supervoxel's voxels sit in
// the plan's centred voxel stream vox4 (one float4 per voxel: x - c0, y - c1, z - c2 in FP32
// and I, written once per call by the moment pass), its tiles (end-aligned like SvRec's: tile
// 0 holds r0 voxels, later tiles kVoxTile), its frame and its centroid.
struct SvLL {
  long long v0;
  int32_t nv, ntiles, r0, frame, frame_nsv;
  float c0, c1, c2;
  int32_t pad[2];
};
static_assert(sizeof(SvLL) == 48, "SvLL is three 16-byte chunks");

struct BatchInfo {
  int32_t n_frames;
  int32_t total_sv;
  int32_t total_gauss;
  int32_t n_gchunks;
  int32_t total_cells;
  int32_t pad[3];
};

struct GChunk {
  int32_t frame, g_begin, g_end, pad;
};

// Device pointers of a plan (passed by value to kernels).
struct DevPlan {
  int64_t max_vox;
  int32_t max_sv, max_gauss, max_frames, max_gchunks, max_cells;
  BatchInfo* info;
  FrameDesc* frames;
  FrameState* state;
  GChunk* gchunks;
  // per Gaussian
  int32_t* g_frame;
  double* gd;  // SoA block, see G_* offsets (component * max_gauss)
  uint8_t* fixed;
  float4* cell_refs;  // [max_cells][kCellCap]: float centre + frame-local index
  int32_t* cell_cnt;
  int32_t* bcnt;
  int32_t* bucket;
  int32_t* acnt;
  int32_t* abucket;
  double* alpha_part_e;
  // per M-step block: the smallest alpha of its live, non-fixed Gaussians (+inf if none), and
  // 1 when one of its Gaussians has a NaN in W or in this iteration's E[ln|Lambda|]
  double* alpha_min_e;
  int32_t* nan_e;
  double* alpha_part_f;
  int32_t* dead_part;
  int32_t* work;   // [0] next supervoxel of the voxel pass, [1] warps that left it
  int32_t ll_blocks;    // resident blocks of the voxel pass's FP32 forms (SMs x blocks per SM)
  int32_t ll_blocks64;  // the same for its FP64 form
  int32_t knn_group;  // lanes per supervoxel of the kNN/E-step (8, 16 or 32)
  int32_t iter;       // the EM iteration a launch belongs to (1-based; set per launch)
  unsigned long long stage_wait_ns;  // wait limit of a voxel tile copy (default 1 s)
  float4* kpos;  // per Gaussian: the float centre the kNN sees (x, y, z; w = 1 live, 0 dead)
  double* ec;   // per Gaussian E-step record, kEcStride doubles: nu W [6], m [3], 3/beta, psi(alpha)+eLD/2
  double* llc;  // per Gaussian, 10 doubles: -nu*W/2 (off-diagonals doubled) [6], log weight [1], m [3]
  // per supervoxel
  int32_t* sv_frame;
  int32_t* sv_order;  // the order in which the voxel passes take supervoxels (k_order_*)
  int32_t* ord_hist;  // [max_frames][64]: per frame, supervoxels per tile-count bucket, then bases
  int32_t* ord_cur;   // [max_frames][64]: cursors of the scatter
  SvRec* sv_rec;
  SvLL* sv_ll;
  float4* vox4;  // [max_vox]: the centred voxel stream of the batch (see SvLL)
  double* mom;
  int32_t* cand;  // [2][max_sv][kJ]: candidates of the odd / even iterations' E-steps
  float* rnk;     // [2][max_sv][kJ]: their responsibilities
  int32_t* nbr;    // [max_sv][kNbr]: the supervoxel's kNbr nearest Gaussians when last searched
  double* nbr_b;   // validity bound of that list (see k_knn_estep)
  double* ll_part;  // [2][max_sv]
};

// component offsets inside DevPlan::gd (each component is max_gauss doubles)
enum : int {
  G_BETA = 0, G_NU, G_ALPHA,
  G_M0, G_M1, G_M2,
  G_W0, G_W1, G_W2, G_W3, G_W4, G_W5,
  G_BETAO, G_NUO, G_ALPHAO,
  G_MO0, G_MO1, G_MO2,
  G_WO0, G_WO1, G_WO2, G_WO3, G_WO4, G_WO5,
  G_ELD0, G_ELD1,
  G_PSIA0, G_PSIA1,
  G_NUM
};

__device__ __forceinline__ double& gcomp(const DevPlan& P, int c, int k) {
  return P.gd[(int64_t)c * P.max_gauss + k];
}

// The E-step buffers of iteration `it` (two, by parity: the kNN/E-step of the next
// iteration may run while the voxel pass still reads this one's candidates).
__device__ __forceinline__ int32_t* cand_buf(const DevPlan& P, int it) {
  return P.cand + (int64_t)(it & 1) * P.max_sv * kJ;
}
__device__ __forceinline__ float* rnk_buf(const DevPlan& P, int it) {
  return P.rnk + (int64_t)(it & 1) * P.max_sv * kJ;
}

// ---- kernel launchers (em_kernels.cu) ----
void launch_build_maps(const DevPlan& P, cudaStream_t st);
void launch_fetch_records(const DevPlan& P, cudaStream_t st);
void launch_import(const DevPlan& P, cudaStream_t st);
void launch_order(const DevPlan& P, cudaStream_t st);
void launch_moments(const DevPlan& P, cudaStream_t st);
void launch_knn_estep(const DevPlan& P, cudaStream_t st);
void launch_mstep_update(const DevPlan& P, cudaStream_t st);
void launch_kill_prep(const DevPlan& P, cudaStream_t st);
void launch_ll_pass(const DevPlan& P, int fp64, int knn_group, cudaStream_t st);
void launch_iter_cond(const DevPlan& P, cudaGraphConditionalHandle h, cudaStream_t st);
void launch_assign(const DevPlan& P, cudaStream_t st);
cudaError_t configure_kernels(DevPlan& P, int device);
// bytes from host memory to 16-byte aligned device memory through kernel launch
// parameters (the tail up to the next 16 bytes is written with zeros)
cudaError_t launch_stage_bytes(void* dst, const void* src, size_t bytes, cudaStream_t st);
void launch_export(const DevPlan& P, cudaStream_t st);

// standalone kNN (tgmm_knn): brute force over refs in shared memory tiles
cudaError_t knn_bruteforce(const float* query, int64_t nq, const float* ref_xyz, int32_t nref,
                           const float scale[3], int32_t* ind, cudaStream_t st);
// grid kNN over a single point set, for tgmm_knn with large nref
cudaError_t knn_grid_standalone(const float* query, int64_t nq, const float* ref_xyz,
                                int32_t nref, const float scale[3], int32_t* ind,
                                cudaStream_t st);

// grid kNN on caller-provided scratch (no allocation)
size_t knn_grid_scratch_bytes(int32_t nref);
constexpr int kMaxK = 11;  // neighbours of the tracking graph's supervoxel kNN (maxKNN)
cudaError_t knn_grid_topk(const float* q, int64_t nq, const float* ref, int32_t nref, int soa, int K,
                          const float scale[3], int32_t* ind, float* dist, cudaStream_t st);
cudaError_t knn_grid_in_scratch(const float* query, int64_t nq, const float* ref_xyz, int32_t nref,
                                const float scale[3], int32_t* ind, cudaStream_t st, void* scratch);
// records a failure for tgmm_last_error() and returns code
int report_error(int code, const char* what, cudaError_t e);

// device-side posterior -> prior
cudaError_t update_priors_device(TgmmGaussian* gm, int32_t n, double bp, double np, double ap,
                                 double atot, int compute_total, cudaStream_t st);

}  // namespace tgmm
