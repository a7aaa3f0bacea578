// em_host.cu -- C ABI of the EM engine: plans (all device workspace), batch tables,
// CUDA-graph capture of the whole fixed-length EM, and the reference-shaped entry points.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "tgmm_internal.cuh"

using namespace tgmm;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
  char buf[512];
  if (e != cudaSuccess)
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  else
    snprintf(buf, sizeof(buf), "%s", what);
  g_last_error = buf;
  return code;
}

#define TG_CUDA(call, what)                                   \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return fail(TGMM_ERR_CUDA, what, e_); \
  } while (0)

int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

struct Layout {
  // byte offsets of every device array inside one allocation
  int64_t info, frames, state, gchunks, g_frame, gd, fixed, cell_refs, cell_cnt, bcnt, bucket, acnt, abucket, ape, apf, dead, ec, llc, kpos, work, sv_frame, sv_order, ord_hist, ord_cur, sv_rec, sv_ll, vox4, mom, cand, rnk, nbr, nbr_b, llp, gm_scratch, total;
};

Layout make_layout(const TgmmPlanDesc& d, int32_t max_gchunks, int32_t max_cells) {
  Layout L;
  int64_t o = 0;
  auto take = [&](int64_t bytes) {
    int64_t at = o;
    o = align_up(o + std::max<int64_t>(bytes, 1), 256);
    return at;
  };
  const int64_t G = d.max_gauss, S = d.max_sv, F = d.max_frames;
  L.info = take(sizeof(BatchInfo));
  L.frames = take(sizeof(FrameDesc) * F);
  L.state = take(sizeof(FrameState) * F);
  L.gchunks = take(sizeof(GChunk) * max_gchunks);
  L.g_frame = take(4 * G);
  L.gd = take(8 * G * G_NUM);
  L.fixed = take(G);
  L.cell_refs = take(16 * (int64_t)kCellCap * max_cells);
  L.cell_cnt = take(4 * (int64_t)max_cells);
  L.bcnt = take(4 * G);
  L.bucket = take(4 * G * kBucketCap);
  L.acnt = take(4 * G);
  L.abucket = take(4 * G * kBucketCap);
  L.ape = take(8 * 2 * (int64_t)max_gchunks * 3);  // the M-step's sums, minima and NaN flags
  L.apf = take(8 * (int64_t)max_gchunks);
  L.dead = take(4 * (int64_t)max_gchunks);
  L.ec = take(8 * kEcStride * G);
  L.llc = take(8 * 10 * G);
  L.kpos = take(16 * G);
  L.work = take(64);
  L.sv_frame = take(4 * S);
  L.sv_order = take(4 * S);
  L.ord_hist = take(4 * 64 * (int64_t)d.max_frames);
  L.ord_cur = take(4 * 64 * (int64_t)d.max_frames);
  L.sv_rec = take((int64_t)sizeof(SvRec) * S);
  L.sv_ll = take((int64_t)sizeof(SvLL) * S);
  L.vox4 = take(16 * d.max_vox);
  L.mom = take(8 * S * kNumMoments);
  L.cand = take(2 * 4 * S * kJ);
  L.rnk = take(2 * 4 * S * kJ);
  L.nbr = take(4 * S * kNbr);
  L.nbr_b = take(8 * S);
  L.llp = take(8 * 2 * S);
  L.gm_scratch = take((int64_t)sizeof(TgmmGaussian) * G);
  L.total = o;
  return L;
}

int32_t gchunks_cap(const TgmmPlanDesc& d) { return (d.max_gauss + kGChunk - 1) / kGChunk + d.max_frames; }
int32_t cells_cap(const TgmmPlanDesc& d) { return d.max_gauss / 2 + 8 * d.max_frames; }

}  // namespace

namespace tgmm {
int report_error(int code, const char* what, cudaError_t e) { return fail(code, what, e); }
}  // namespace tgmm

struct TgmmPlan {
  TgmmPlanDesc desc;
  Layout L;
  char* base = nullptr;
  DevPlan dev;
  FrameState* h_state = nullptr;  // pinned: per-frame state read back for stats
  cudaStream_t cap_stream = nullptr;
  cudaEvent_t done_ev = nullptr;       // end of the last call
  cudaStream_t last_stream = nullptr;  // its stream
  bool used = false;
  bool fuse_knn = false;  // the voxel pass runs the next iteration's kNN/E-step (autotuned)
  // (max_iter, ll_prec, conditional iterations) -> exec
  std::map<std::tuple<int, int, int>, cudaGraphExec_t> graphs;
  cudaStream_t body_stream = nullptr;  // captures the bodies of the conditional iterations
  cudaStream_t fork_stream = nullptr;  // the records' branch of a call (fetch, import)
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  // host copy of the tables of the last staged batch
  BatchInfo s_info{};
  std::vector<FrameDesc> s_frames;
  std::vector<GChunk> s_gchunks;
  std::mutex mu;
};

extern "C" {

void tgmm_default_params(TgmmEmParams* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->max_iter_em = 400;
  p->w4dof = 1;
  p->tol_likelihood = 1e-6;
  p->lambda_min = 0.02;
  p->lambda_max = 0.2222;
  p->max_excentricity = 9.0;
  p->scale[0] = p->scale[1] = p->scale[2] = 1.0f;
  p->ll_mode = TGMM_LL_AS_REFERENCE;
  p->ll_precision = TGMM_LLPREC_MIXED;
}

const char* tgmm_last_error(void) { return g_last_error.c_str(); }
const char* tgmm_version(void) { return "tgmm_b200 0.1 (sm_100a)"; }

int64_t tgmm_plan_bytes(const TgmmPlanDesc* d) {
  if (!d || d->max_gauss <= 0 || d->max_sv < 0 || d->max_frames <= 0) return -1;
  return make_layout(*d, gchunks_cap(*d), cells_cap(*d)).total;
}

int tgmm_plan_create(const TgmmPlanDesc* d, TgmmPlan** out) {
  if (!d || !out) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_create: null argument");
  if (d->max_gauss < TGMM_J || d->max_sv < 1 || d->max_frames < 1 || d->max_vox < 0)
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_create: capacities must be positive (max_gauss >= 5)");
  if ((int64_t)d->max_sv * kJ >= (1LL << 31) || (int64_t)d->max_gauss * kBucketCap >= (1LL << 31))
    return fail(TGMM_ERR_BAD_SIZE, "tgmm_plan_create: capacities beyond 32-bit indexing");
  *out = nullptr;
  TG_CUDA(cudaSetDevice(d->device), "cudaSetDevice");
  TgmmPlan* P = new TgmmPlan();
  P->desc = *d;
  const int32_t mgc = gchunks_cap(*d), mcl = cells_cap(*d);
  P->L = make_layout(*d, mgc, mcl);
  cudaError_t e = cudaMalloc(&P->base, P->L.total);
  if (e != cudaSuccess) {
    delete P;
    return fail(TGMM_ERR_OOM, "tgmm_plan_create: cudaMalloc", e);
  }
  e = cudaMemset(P->base, 0, P->L.total);
  if (e == cudaSuccess) e = cudaMallocHost(&P->h_state, sizeof(FrameState) * d->max_frames);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P->body_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P->fork_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->fork_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->join_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->done_ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    tgmm_plan_destroy(P);
    return fail(TGMM_ERR_CUDA, "tgmm_plan_create: setup", e);
  }
  P->s_frames.assign(d->max_frames, FrameDesc{});
  P->s_gchunks.assign(mgc, GChunk{});
  DevPlan& D = P->dev;
  char* b = P->base;
  D.max_vox = d->max_vox;
  D.max_sv = d->max_sv;
  D.max_gauss = d->max_gauss;
  D.max_frames = d->max_frames;
  D.max_gchunks = mgc;
  D.max_cells = mcl;
  D.info = (BatchInfo*)(b + P->L.info);
  D.frames = (FrameDesc*)(b + P->L.frames);
  D.state = (FrameState*)(b + P->L.state);
  D.gchunks = (GChunk*)(b + P->L.gchunks);
  D.g_frame = (int32_t*)(b + P->L.g_frame);
  D.gd = (double*)(b + P->L.gd);
  D.fixed = (uint8_t*)(b + P->L.fixed);
  D.cell_refs = (float4*)(b + P->L.cell_refs);
  D.cell_cnt = (int32_t*)(b + P->L.cell_cnt);
  D.bcnt = (int32_t*)(b + P->L.bcnt);
  D.bucket = (int32_t*)(b + P->L.bucket);
  D.acnt = (int32_t*)(b + P->L.acnt);
  D.abucket = (int32_t*)(b + P->L.abucket);
  D.alpha_part_e = (double*)(b + P->L.ape);
  D.alpha_min_e = D.alpha_part_e + 2 * (int64_t)mgc;
  D.nan_e = (int32_t*)(D.alpha_min_e + 2 * (int64_t)mgc);
  D.alpha_part_f = (double*)(b + P->L.apf);
  D.dead_part = (int32_t*)(b + P->L.dead);
  D.ec = (double*)(b + P->L.ec);
  D.llc = (double*)(b + P->L.llc);
  D.kpos = (float4*)(b + P->L.kpos);
  D.work = (int32_t*)(b + P->L.work);
  D.knn_group = 8;
  D.stage_wait_ns = 1000000000ull;
  e = configure_kernels(D, d->device);
  if (e != cudaSuccess) {
    tgmm_plan_destroy(P);
    return fail(TGMM_ERR_CUDA, "tgmm_plan_create: kernel configuration", e);
  }
  D.sv_frame = (int32_t*)(b + P->L.sv_frame);
  D.sv_order = (int32_t*)(b + P->L.sv_order);
  D.ord_hist = (int32_t*)(b + P->L.ord_hist);
  D.ord_cur = (int32_t*)(b + P->L.ord_cur);
  D.sv_rec = (SvRec*)(b + P->L.sv_rec);
  D.sv_ll = (SvLL*)(b + P->L.sv_ll);
  D.vox4 = (float4*)(b + P->L.vox4);
  D.mom = (double*)(b + P->L.mom);
  D.cand = (int32_t*)(b + P->L.cand);
  D.rnk = (float*)(b + P->L.rnk);
  D.nbr = (int32_t*)(b + P->L.nbr);
  D.nbr_b = (double*)(b + P->L.nbr_b);
  D.ll_part = (double*)(b + P->L.llp);
  *out = P;
  return TGMM_OK;
}

int tgmm_plan_destroy(TgmmPlan* P) {
  if (!P) return TGMM_OK;
  if (P->used) cudaEventSynchronize(P->done_ev);
  for (auto& kv : P->graphs) cudaGraphExecDestroy(kv.second);
  if (P->cap_stream) cudaStreamDestroy(P->cap_stream);
  if (P->body_stream) cudaStreamDestroy(P->body_stream);
  if (P->fork_stream) cudaStreamDestroy(P->fork_stream);
  if (P->fork_ev) cudaEventDestroy(P->fork_ev);
  if (P->join_ev) cudaEventDestroy(P->join_ev);
  if (P->done_ev) cudaEventDestroy(P->done_ev);
  if (P->h_state) cudaFreeHost(P->h_state);
  if (P->base) cudaFree(P->base);
  delete P;
  return TGMM_OK;
}

}  // extern "C"

namespace {

int validate_params(const TgmmEmParams* p) {
  if (!p) return fail(TGMM_ERR_INVALID_ARG, "params is null");
  if (p->max_iter_em < 1) return fail(TGMM_ERR_INVALID_ARG, "max_iter_em must be >= 1");
  if (!(p->lambda_min > 0) || !(p->lambda_max > 0) || !(p->max_excentricity > 0))
    return fail(TGMM_ERR_NOT_SET,
                "regularisation constants not set (lambda_min, lambda_max, max_excentricity must be > 0)");
  for (int d = 0; d < 3; d++)
    if (!(p->scale[d] >= 1e-3f)) return fail(TGMM_ERR_INVALID_ARG, "scale must be >= 1e-3");
  const bool reg_zero = p->reg_scale[0] == 0.0f && p->reg_scale[1] == 0.0f && p->reg_scale[2] == 0.0f;
  for (int d = 0; d < 3 && !reg_zero; d++)
    if (!(p->reg_scale[d] >= 1e-3f)) return fail(TGMM_ERR_INVALID_ARG, "reg_scale must be >= 1e-3 (or all zero)");
  if (p->ll_mode != TGMM_LL_AS_REFERENCE && p->ll_mode != TGMM_LL_TRUE)
    return fail(TGMM_ERR_INVALID_ARG, "unknown ll_mode");
  if (p->ll_precision != TGMM_LLPREC_MIXED && p->ll_precision != TGMM_LLPREC_FP64)
    return fail(TGMM_ERR_INVALID_ARG, "unknown ll_precision");
  return TGMM_OK;
}

// Fill the pinned batch tables.  Returns a status.
int stage_batch(TgmmPlan* P, int32_t n, const TgmmFrame* fr, TgmmGaussian* const* gm, float* const* rnk,
                int32_t* const* ind, const TgmmEmParams* prm) {
  if (n < 1 || n > P->desc.max_frames) return fail(TGMM_ERR_BAD_SIZE, "frame count beyond plan capacity");
  int64_t tv = 0;
  int64_t ts = 0, tg = 0, tc = 0;
  int32_t gc = 0;
  for (int32_t f = 0; f < n; f++) {
    const TgmmFrame& F = fr[f];
    if (!F.query || !F.img || !F.centroids || !F.label_ptr || !gm[f] || !rnk[f] || !ind[f])
      return fail(TGMM_ERR_INVALID_ARG, "null frame pointer");
    if (F.n_vox < 0 || F.n_sv < 1 || F.n_gauss < 1) return fail(TGMM_ERR_INVALID_ARG, "frame sizes must be positive");
    if (F.n_gauss < TGMM_J) return fail(TGMM_ERR_BAD_SIZE, "a frame needs at least 5 Gaussians");
    tv += F.n_vox;
    ts += F.n_sv;
    tg += F.n_gauss;
  }
  if (tv > P->desc.max_vox || ts > P->desc.max_sv || tg > P->desc.max_gauss)
    return fail(TGMM_ERR_BAD_SIZE, "batch exceeds plan capacity");
  ts = tg = 0;
  int64_t vb = 0;
  for (int32_t f = 0; f < n; f++) {
    const TgmmFrame& F = fr[f];
    FrameDesc& D = P->s_frames[f];
    memset(&D, 0, sizeof(D));
    D.vox_base = vb;
    vb += F.n_vox;
    D.query = F.query;
    D.img = F.img;
    D.cent = F.centroids;
    D.lptr = F.label_ptr;
    D.gm = gm[f];
    D.rnk_out = rnk[f];
    D.ind_out = ind[f];
    D.n_vox = F.n_vox;
    D.n_sv = F.n_sv;
    D.n_gauss = F.n_gauss;
    D.sv_base = (int32_t)ts;
    D.g_base = (int32_t)tg;
    D.cell_base = (int32_t)tc;
    D.cell_budget = F.n_gauss / 2 + 8;
    D.gchunk_base = gc;
    D.n_gchunks = (F.n_gauss + kGChunk - 1) / kGChunk;
    const bool reg_zero = prm->reg_scale[0] == 0.0f && prm->reg_scale[1] == 0.0f && prm->reg_scale[2] == 0.0f;
    for (int d = 0; d < 3; d++) {
      D.scale[d] = prm->scale[d];
      D.reg_scale[d] = reg_zero ? prm->scale[d] : prm->reg_scale[d];
    }
    D.w4dof = prm->w4dof ? 1 : 0;
    D.lambda_min = prm->lambda_min;
    D.lambda_max = prm->lambda_max;
    D.max_exc = prm->max_excentricity;
    D.tol = prm->tol_likelihood;
    D.max_iter = prm->max_iter_em;
    D.ll_mode = prm->ll_mode;
    D.ll_prec = prm->ll_precision;
    D.frame_id = f;
    for (int32_t c = 0; c < D.n_gchunks; c++) {
      GChunk& C = P->s_gchunks[gc + c];
      C.frame = f;
      C.g_begin = D.g_base + c * kGChunk;
      C.g_end = std::min(D.g_base + F.n_gauss, C.g_begin + kGChunk);
      C.pad = 0;
    }
    gc += D.n_gchunks;
    ts += F.n_sv;
    tg += F.n_gauss;
    tc += D.cell_budget;
  }
  BatchInfo& I = P->s_info;
  memset(&I, 0, sizeof(I));
  I.n_frames = n;
  I.total_sv = (int32_t)ts;
  I.total_gauss = (int32_t)tg;
  I.n_gchunks = gc;
  I.total_cells = (int32_t)tc;
  return TGMM_OK;
}

// A call on `st` starts after the plan's previous call, even on another stream.
int order_after_previous(TgmmPlan* P, cudaStream_t st) {
  if (P->used && P->last_stream != st) TG_CUDA(cudaStreamWaitEvent(st, P->done_ev, 0), "order after previous call");
  return TGMM_OK;
}

// The staged batch tables to the device (kernel launches, no copy engine).
int stage_tables(TgmmPlan* P, cudaStream_t st) {
  const DevPlan& D = P->dev;
  TG_CUDA(launch_stage_bytes(D.info, &P->s_info, sizeof(BatchInfo), st), "stage info");
  TG_CUDA(launch_stage_bytes(D.frames, P->s_frames.data(), sizeof(FrameDesc) * P->s_info.n_frames, st),
          "stage frames");
  TG_CUDA(launch_stage_bytes(D.gchunks, P->s_gchunks.data(), sizeof(GChunk) * P->s_info.n_gchunks, st),
          "stage chunks");
  return TGMM_OK;
}

// Appends to the graph being captured on `st` one conditional (IF) node whose body is what
// `body` enqueues (captured on the plan's body stream), preceded by k_iter_cond, which sets
// the node's condition on the device: whether any frame of the batch still runs.
template <class F>
int capture_if_running(TgmmPlan* P, const DevPlan& D, cudaStream_t st, F body) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  unsigned long long id = 0;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  TG_CUDA(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd), "capture info");
  if (cs != cudaStreamCaptureStatusActive) return fail(TGMM_ERR_CUDA, "conditional iteration outside a capture");
  cudaGraphConditionalHandle h;
  TG_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault), "conditional handle");
  launch_iter_cond(D, h, st);
  TG_CUDA(cudaGetLastError(), "iteration condition");
  TG_CUDA(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd), "capture info");
  std::vector<cudaGraphNode_t> dv(deps, deps + nd);
  cudaGraphNodeParams prm = {cudaGraphNodeTypeConditional};
  prm.conditional.handle = h;
  prm.conditional.type = cudaGraphCondTypeIf;
  prm.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  TG_CUDA(cudaGraphAddNode(&node, g, dv.data(), dv.size(), &prm), "conditional node");
  TG_CUDA(cudaStreamBeginCaptureToGraph(P->body_stream, prm.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal),
          "begin body capture");
  body(P->body_stream);
  cudaGraph_t bg = nullptr;
  const cudaError_t e = cudaStreamEndCapture(P->body_stream, &bg);
  TG_CUDA(cudaGetLastError(), "iteration body");
  TG_CUDA(e, "end body capture");
  TG_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies),
          "capture dependencies");
  return TGMM_OK;
}

// The whole EM (after the tables are staged) as a stream of async operations on `st`.
// Each launch carries its iteration number.  With fuse_knn the voxel pass of iteration t
// also runs the kNN/E-step of iteration t + 1 (mixed-precision voxel terms only); else that
// kernel follows the pass.  With `cond` (a graph capture with a convergence tolerance) each
// iteration is a conditional graph node that runs only while a frame of the batch is still
// running, so a batch that converged early launches none of the remaining iterations' kernels
// (which would all find their frames done and return).
int enqueue_em(TgmmPlan* P, int max_iter, int ll_prec, bool cond, cudaStream_t st) {
  DevPlan D = P->dev;
  D.iter = 1;
  launch_build_maps(D, st);
  // two branches after the frame maps: the Gaussian records (fetched from the caller's
  // page-locked memory where the descriptor names it, then imported) beside the supervoxel
  // order and the moment pass, which need no Gaussian; joined before the first kNN/E-step
  TG_CUDA(cudaEventRecord(P->fork_ev, st), "fork");
  TG_CUDA(cudaStreamWaitEvent(P->fork_stream, P->fork_ev, 0), "fork");
  launch_fetch_records(D, P->fork_stream);
  launch_import(D, P->fork_stream);
  TG_CUDA(cudaEventRecord(P->join_ev, P->fork_stream), "join");
  launch_order(D, st);
  launch_moments(D, st);
  TG_CUDA(cudaStreamWaitEvent(st, P->join_ev, 0), "join");
  const bool fp64 = ll_prec == TGMM_LLPREC_FP64;
  // (the voxel pass carries the kNN/E-step in groups of 8 lanes or more)
  const bool fuse = P->fuse_knn && !fp64 && D.knn_group >= 8;
  if (max_iter >= 1) launch_knn_estep(D, st);
  for (int it = 1; it <= max_iter; it++) {
    D.iter = it;
    auto body = [&, D, it](cudaStream_t s) {
      launch_mstep_update(D, s);
      launch_kill_prep(D, s);
      const bool more = it < max_iter;
      launch_ll_pass(D, fp64, more && fuse ? D.knn_group : 0, s);
      if (more && !fuse) {
        DevPlan N = D;
        N.iter = it + 1;
        launch_knn_estep(N, s);
      }
    };
    if (cond) {
      const int rc = capture_if_running(P, D, st, body);
      if (rc) return rc;
    } else {
      body(st);
    }
  }
  launch_assign(D, st);
  launch_export(D, st);
  TG_CUDA(cudaGetLastError(), "kernel launch");
  return TGMM_OK;
}

bool use_graphs() {
  const char* e = getenv("TGMM_NO_GRAPH");
  return !(e && e[0] == '1');
}

int run_batch(TgmmPlan* P, int max_iter, int ll_prec, double tol, cudaStream_t st) {
  if (!use_graphs()) return enqueue_em(P, max_iter, ll_prec, false, st);
  // a negative tolerance runs every iteration: no conditional nodes
  const bool cond = tol >= 0.0;
  auto key = std::make_tuple(max_iter, ll_prec, cond ? 1 : 0);
  auto it = P->graphs.find(key);
  if (it == P->graphs.end()) {
    cudaGraph_t g = nullptr;
    TG_CUDA(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int rc = enqueue_em(P, max_iter, ll_prec, cond, P->cap_stream);
    cudaError_t e = cudaStreamEndCapture(P->cap_stream, &g);
    if (rc != TGMM_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(TGMM_ERR_CUDA, "end capture", e);
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(TGMM_ERR_CUDA, "graph instantiate", e);
    it = P->graphs.emplace(key, ex).first;
  }
  TG_CUDA(cudaGraphLaunch(it->second, st), "graph launch");
  return TGMM_OK;
}

int collect_stats(TgmmPlan* P, int32_t n, TgmmEmStats* stats, cudaStream_t st, int* flags_or) {
  TG_CUDA(cudaMemcpyAsync(P->h_state, P->dev.state, sizeof(FrameState) * n, cudaMemcpyDeviceToHost, st),
          "read state");
  TG_CUDA(cudaStreamSynchronize(st), "synchronize");
  int fo = 0;
  for (int32_t f = 0; f < n; f++) {
    const FrameState& S = P->h_state[f];
    fo |= S.flags;
    if (!stats) continue;
    TgmmEmStats& o = stats[f];
    o.iterations = S.iter - 1;
    o.converged = S.converged;
    o.ll = S.ll;
    o.ll_true = S.ll_true;
    o.ll_as_reference = S.ll_ref;
    o.total_alpha = S.total_alpha;
    o.n_dead = S.n_dead;
    o.device_flags = S.flags;
    o.knn_searches = S.knn_searches;
    o.reserved = 0;
  }
  if (flags_or) *flags_or = fo;
  return TGMM_OK;
}

}  // namespace

namespace tgmm {

size_t frame_state_bytes() { return sizeof(FrameState); }

int plan_enqueue_state(TgmmPlan* P, int32_t n, void* dst, cudaStream_t st) {
  if (!P || !dst || n < 1 || n > P->desc.max_frames) return fail(TGMM_ERR_INVALID_ARG, "plan_enqueue_state");
  TG_CUDA(cudaMemcpyAsync(dst, P->dev.state, sizeof(FrameState) * n, cudaMemcpyDeviceToHost, st), "read state");
  return TGMM_OK;
}

int frame_state_to_stats(const void* state, TgmmEmStats* o) {
  const FrameState& S = *static_cast<const FrameState*>(state);
  if (o) {
    o->iterations = S.iter - 1;
    o->converged = S.converged;
    o->ll = S.ll;
    o->ll_true = S.ll_true;
    o->ll_as_reference = S.ll_ref;
    o->total_alpha = S.total_alpha;
    o->n_dead = S.n_dead;
    o->device_flags = S.flags;
    o->knn_searches = S.knn_searches;
    o->reserved = 0;
  }
  int rc = TGMM_OK;
  if (S.flags & F_BAD_CSR)
    rc = TGMM_ERR_BAD_CSR;
  else if (S.flags & F_FEW_GAUSS)
    rc = TGMM_ERR_BAD_SIZE;
  else if (S.flags & F_STAGE_TIMEOUT)
    rc = TGMM_ERR_DEVICE_FLAG;
  else if (S.flags & F_NAN_INPUT)
    rc = TGMM_ERR_NAN_INPUT;
  return rc;
}

}  // namespace tgmm

namespace {

int flags_to_status(int flags) {
  if (flags & F_BAD_CSR) return fail(TGMM_ERR_BAD_CSR, "labelListPtr is not a valid CSR over the voxels");
  if (flags & F_FEW_GAUSS) return fail(TGMM_ERR_BAD_SIZE, "a frame has fewer than 5 Gaussians");
  if (flags & F_STAGE_TIMEOUT)
    return fail(TGMM_ERR_DEVICE_FLAG, "a voxel tile copy did not complete within its wait limit");
  if (flags & F_NAN_INPUT) return fail(TGMM_ERR_NAN_INPUT, "NaN in voxel coordinates, intensities or Gaussians");
  return TGMM_OK;
}

}  // namespace

extern "C" {

namespace {
// tgmm_em_run_batch; gm_src (optional, one per frame) names page-locked host records (their
// device-mapped addresses) that the call's graph copies into gm_dev first.
int em_run_batch(TgmmPlan* P, int32_t n_frames, const TgmmFrame* frames, TgmmGaussian* const* gm_dev,
                 float* const* rnk_dev, int32_t* const* ind_dev, const TgmmEmParams* params, TgmmEmStats* stats,
                 void* stream, const TgmmGaussian* const* gm_src) {
  if (!P || !frames || !gm_dev || !rnk_dev || !ind_dev) return fail(TGMM_ERR_INVALID_ARG, "null argument");
  int rc = validate_params(params);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(P->mu);
  cudaStream_t st = (cudaStream_t)stream;
  TG_CUDA(cudaSetDevice(P->desc.device), "cudaSetDevice");
  rc = stage_batch(P, n_frames, frames, gm_dev, rnk_dev, ind_dev, params);
  if (rc) return rc;
  if (gm_src)
    for (int32_t f = 0; f < n_frames; f++) P->s_frames[f].gm_src = gm_src[f];
  rc = order_after_previous(P, st);
  if (rc) return rc;
  rc = stage_tables(P, st);
  if (rc) return rc;
  rc = run_batch(P, params->max_iter_em, params->ll_precision, params->tol_likelihood, st);
  if (rc) return rc;
  TG_CUDA(cudaEventRecord(P->done_ev, st), "record");
  P->used = true;
  P->last_stream = st;
  if (stats) {
    int fo = 0;
    rc = collect_stats(P, n_frames, stats, st, &fo);
    if (rc) return rc;
    return flags_to_status(fo);
  }
  return TGMM_OK;
}
}  // namespace

int tgmm_em_run_batch(TgmmPlan* P, int32_t n_frames, const TgmmFrame* frames, TgmmGaussian* const* gm_dev,
                      float* const* rnk_dev, int32_t* const* ind_dev, const TgmmEmParams* params,
                      TgmmEmStats* stats, void* stream) {
  return em_run_batch(P, n_frames, frames, gm_dev, rnk_dev, ind_dev, params, stats, stream, nullptr);
}

int tgmm_plan_set_knn_group(TgmmPlan* P, int32_t lanes) {
  if (!P) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_set_knn_group: null plan");
  if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_set_knn_group: lanes per supervoxel must be 4, 8, 16 or 32");
  std::lock_guard<std::mutex> lock(P->mu);
  if (P->dev.knn_group == lanes) return TGMM_OK;
  TG_CUDA(cudaSetDevice(P->desc.device), "cudaSetDevice");
  if (P->used) TG_CUDA(cudaEventSynchronize(P->done_ev), "wait for the previous call on this plan");
  for (auto& kv : P->graphs) cudaGraphExecDestroy(kv.second);  // captured with the old launch shape
  P->graphs.clear();
  P->dev.knn_group = lanes;
  return TGMM_OK;
}

int tgmm_plan_set_knn_fusion(TgmmPlan* P, int32_t on) {
  if (!P) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_set_knn_fusion: null plan");
  if (on != 0 && on != 1) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_set_knn_fusion: on must be 0 or 1");
  std::lock_guard<std::mutex> lock(P->mu);
  if (P->fuse_knn == (on == 1)) return TGMM_OK;
  TG_CUDA(cudaSetDevice(P->desc.device), "cudaSetDevice");
  if (P->used) TG_CUDA(cudaEventSynchronize(P->done_ev), "wait for the previous call on this plan");
  for (auto& kv : P->graphs) cudaGraphExecDestroy(kv.second);  // captured with the other arrangement
  P->graphs.clear();
  P->fuse_knn = on == 1;
  return TGMM_OK;
}

int tgmm_plan_set_stage_wait(TgmmPlan* P, int64_t wait_ns) {
  if (!P) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_set_stage_wait: null plan");
  if (wait_ns < 1 || wait_ns > 60000000000LL)
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_set_stage_wait: the limit must be 1 ns .. 60 s");
  std::lock_guard<std::mutex> lock(P->mu);
  if (P->dev.stage_wait_ns == (unsigned long long)wait_ns) return TGMM_OK;
  TG_CUDA(cudaSetDevice(P->desc.device), "cudaSetDevice");
  if (P->used) TG_CUDA(cudaEventSynchronize(P->done_ev), "wait for the previous call on this plan");
  for (auto& kv : P->graphs) cudaGraphExecDestroy(kv.second);  // captured with the old limit
  P->graphs.clear();
  P->dev.stage_wait_ns = (unsigned long long)wait_ns;
  return TGMM_OK;
}

int tgmm_plan_tuning(TgmmPlan* P, int32_t* lanes, int32_t* fused) {
  if (!P) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_tuning: null plan");
  std::lock_guard<std::mutex> lock(P->mu);
  if (lanes) *lanes = P->dev.knn_group;
  if (fused) *fused = P->fuse_knn && P->dev.knn_group >= 8 ? 1 : 0;
  return TGMM_OK;
}

// The autotuner runs the whole EM call of the batch (its CUDA graph, at most 20
// iterations) for every kNN/E-step width and arrangement and keeps the fastest: the
// kernels' costs interact (the width changes the kNN/E-step's occupancy, running it inside
// the voxel pass changes what hides whose latency), so only the call shows the best pair.
// The runs work on the plan's scratch copy of the Gaussians, refreshed before each run.
int tgmm_plan_autotune(TgmmPlan* P, int32_t n_frames, const TgmmFrame* frames, TgmmGaussian* const* gm_dev,
                       float* const* rnk_dev, int32_t* const* ind_dev, const TgmmEmParams* params, int32_t reps,
                       int32_t* lanes_out, void* stream) {
  if (!P || !frames || !gm_dev || !rnk_dev || !ind_dev || reps < 1 || n_frames < 1)
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_autotune");
  int rc = validate_params(params);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(P->mu);
  cudaStream_t st = (cudaStream_t)stream;
  TG_CUDA(cudaSetDevice(P->desc.device), "cudaSetDevice");
  if (n_frames > P->desc.max_frames) return fail(TGMM_ERR_BAD_SIZE, "frame count beyond plan capacity");
  int64_t tg = 0;
  for (int32_t f = 0; f < n_frames; f++) {
    if (!gm_dev[f] || frames[f].n_gauss < 1) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_autotune: bad frame");
    tg += frames[f].n_gauss;
  }
  if (tg > P->desc.max_gauss) return fail(TGMM_ERR_BAD_SIZE, "batch exceeds plan capacity");
  TgmmGaussian* scratch = (TgmmGaussian*)(P->base + P->L.gm_scratch);
  std::vector<TgmmGaussian*> work(n_frames);
  for (int32_t f = 0, off = 0; f < n_frames; off += frames[f].n_gauss, f++) work[f] = scratch + off;
  TgmmEmParams tp = *params;
  tp.max_iter_em = std::min(tp.max_iter_em, 20);
  rc = stage_batch(P, n_frames, frames, work.data(), rnk_dev, ind_dev, &tp);
  if (rc) return rc;
  rc = order_after_previous(P, st);  // the scratch Gaussians may still be in use
  if (rc) return rc;
  const bool can_fuse = tp.ll_precision != TGMM_LLPREC_FP64 && tp.max_iter_em > 1;
  cudaEvent_t ev[2];
  TG_CUDA(cudaEventCreate(&ev[0]), "event");
  TG_CUDA(cudaEventCreate(&ev[1]), "event");
  const int widths[4] = {4, 8, 16, 32};
  float best_ms = 0.0f;
  int best_w = P->dev.knn_group;
  bool best_f = P->fuse_knn, have = false;
  for (int w : widths) {
    for (int fu = 0; fu < (can_fuse && w >= 8 ? 2 : 1); fu++) {
      for (auto& kv : P->graphs) cudaGraphExecDestroy(kv.second);
      P->graphs.clear();
      P->dev.knn_group = w;
      P->fuse_knn = fu == 1;
      float best_here = 0.0f;
      for (int r = 0; r <= reps && rc == TGMM_OK; r++) {  // run 0 captures the graph and warms up
        for (int32_t f = 0; f < n_frames && rc == TGMM_OK; f++)
          if (cudaMemcpyAsync(work[f], gm_dev[f], sizeof(TgmmGaussian) * (size_t)frames[f].n_gauss,
                              cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            rc = fail(TGMM_ERR_CUDA, "tgmm_plan_autotune: copy Gaussians", cudaGetLastError());
        if (rc == TGMM_OK) rc = stage_tables(P, st);
        if (rc == TGMM_OK && cudaEventRecord(ev[0], st) != cudaSuccess) rc = fail(TGMM_ERR_CUDA, "record");
        if (rc == TGMM_OK) rc = run_batch(P, tp.max_iter_em, tp.ll_precision, tp.tol_likelihood, st);
        if (rc == TGMM_OK && cudaEventRecord(ev[1], st) != cudaSuccess) rc = fail(TGMM_ERR_CUDA, "record");
        if (rc == TGMM_OK && cudaEventSynchronize(ev[1]) != cudaSuccess) rc = fail(TGMM_ERR_CUDA, "synchronize");
        float ms = 0.0f;
        if (rc == TGMM_OK && r > 0) {
          cudaEventElapsedTime(&ms, ev[0], ev[1]);
          if (r == 1 || ms < best_here) best_here = ms;
        }
      }
      if (rc == TGMM_OK && (!have || best_here < best_ms)) {
        have = true;
        best_ms = best_here;
        best_w = w;
        best_f = fu == 1;
      }
    }
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  for (auto& kv : P->graphs) cudaGraphExecDestroy(kv.second);  // recaptured with the chosen tuning
  P->graphs.clear();
  P->dev.knn_group = best_w;
  P->fuse_knn = best_f;
  TG_CUDA(cudaEventRecord(P->done_ev, st), "record");
  P->used = true;
  P->last_stream = st;
  if (rc) return rc;
  if (lanes_out) *lanes_out = best_w;
  return TGMM_OK;
}

int tgmm_plan_time_kernel(TgmmPlan* P, int32_t kernel, int32_t reps, float* ms, void* stream) {
  if (!P || !ms || reps < 1) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_time_kernel");
  if (kernel != TGMM_KERNEL_MOMENTS && kernel != TGMM_KERNEL_LL_PASS && kernel != TGMM_KERNEL_LL_PASS_KNN)
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_time_kernel: only the moment and log-likelihood passes");
  std::lock_guard<std::mutex> lock(P->mu);
  cudaStream_t st = (cudaStream_t)stream;
  TG_CUDA(cudaSetDevice(P->desc.device), "cudaSetDevice");
  if (P->used) TG_CUDA(cudaEventSynchronize(P->done_ev), "wait for the previous call on this plan");
  const int nf = P->s_info.n_frames;
  if (nf < 1) return fail(TGMM_ERR_INVALID_ARG, "tgmm_plan_time_kernel: run a batch first");
  std::vector<FrameState> backup(nf), live(nf);
  TG_CUDA(cudaMemcpy(backup.data(), P->dev.state, sizeof(FrameState) * nf, cudaMemcpyDeviceToHost), "read state");
  live = backup;
  for (auto& s : live)
    if (!(s.flags & (F_BAD_CSR | F_FEW_GAUSS))) s.done = 0;
  TG_CUDA(cudaMemcpy(P->dev.state, live.data(), sizeof(FrameState) * nf, cudaMemcpyHostToDevice), "write state");
  // the voxel pass runs the convergence test; keep every frame running while timing
  std::vector<FrameDesc> frames(P->s_frames.begin(), P->s_frames.begin() + nf);
  for (auto& d : frames) {
    d.max_iter = 0x7fffffff;
    d.tol = -1.0;
  }
  TG_CUDA(cudaMemcpy(P->dev.frames, frames.data(), sizeof(FrameDesc) * nf, cudaMemcpyHostToDevice), "write frames");
  cudaEvent_t a, b;
  TG_CUDA(cudaEventCreate(&a), "event");
  TG_CUDA(cudaEventCreate(&b), "event");
  // as the last iteration of frame 0 ran; the kNN/E-step form writes the buffers of the
  // iteration after it, which the returned results do not use, and M-step bucket counts,
  // cleared below
  DevPlan D = P->dev;
  D.iter = backup[0].iter > 1 ? backup[0].iter - 1 : 1;
  const int fp64 = P->s_frames[0].ll_prec == TGMM_LLPREC_FP64;
  TG_CUDA(cudaEventRecord(a, st), "record");
  for (int r = 0; r < reps; r++) {
    if (kernel == TGMM_KERNEL_MOMENTS) launch_moments(D, st);
    if (kernel == TGMM_KERNEL_LL_PASS) launch_ll_pass(D, fp64, 0, st);
    // (groups of 4 lanes run the kNN/E-step in their own kernel: the pass is timed with 8)
    if (kernel == TGMM_KERNEL_LL_PASS_KNN) launch_ll_pass(D, fp64, fp64 ? 0 : std::max(D.knn_group, 8), st);
  }
  TG_CUDA(cudaEventRecord(b, st), "record");
  if (kernel == TGMM_KERNEL_LL_PASS_KNN)
    TG_CUDA(cudaMemsetAsync(D.bcnt, 0, 4 * (size_t)P->s_info.total_gauss, st), "clear buckets");
  TG_CUDA(cudaEventSynchronize(b), "synchronize");
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t / reps;
  TG_CUDA(cudaMemcpyAsync(P->dev.state, backup.data(), sizeof(FrameState) * nf, cudaMemcpyHostToDevice, st),
          "restore state");
  TG_CUDA(cudaMemcpyAsync(P->dev.frames, P->s_frames.data(), sizeof(FrameDesc) * nf, cudaMemcpyHostToDevice, st),
          "restore frames");
  TG_CUDA(cudaStreamSynchronize(st), "synchronize");
  TG_CUDA(cudaGetLastError(), "kernel launch");
  return TGMM_OK;
}

int tgmm_em_run_device(TgmmPlan* P, const TgmmFrame* frame, TgmmGaussian* gm_dev, float* rnk_dev, int32_t* ind_dev,
                       const TgmmEmParams* params, TgmmEmStats* stats, void* stream) {
  if (!frame) return fail(TGMM_ERR_INVALID_ARG, "null frame");
  return tgmm_em_run_batch(P, 1, frame, &gm_dev, &rnk_dev, &ind_dev, params, stats, stream);
}

int tgmm_em_run(TgmmPlan* P, const TgmmFrame* frame, TgmmGaussian* gm_host, float* rnk_dev, int32_t* ind_dev,
                int32_t* ind_tr_dev, const TgmmEmParams* params, TgmmEmStats* stats, void* stream) {
  if (!P || !frame || !gm_host) return fail(TGMM_ERR_INVALID_ARG, "null argument");
  if (frame->n_gauss > P->desc.max_gauss) return fail(TGMM_ERR_BAD_SIZE, "n_gauss beyond plan capacity");
  cudaStream_t st = (cudaStream_t)stream;
  TG_CUDA(cudaSetDevice(P->desc.device), "cudaSetDevice");
  int orc = order_after_previous(P, st);  // the scratch Gaussians may still be in use
  if (orc) return orc;
  TgmmGaussian* scratch = (TgmmGaussian*)(P->base + P->L.gm_scratch);
  const size_t bytes = sizeof(TgmmGaussian) * (size_t)frame->n_gauss;
  cudaPointerAttributes pa;
  const void* mapped = nullptr;
  if (cudaPointerGetAttributes(&pa, gm_host) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer &&
      ((uintptr_t)pa.devicePointer & 15) == 0)
    mapped = pa.devicePointer;
  cudaGetLastError();  // a pageable pointer may leave an error behind on older drivers
  // page-locked records are read by the call's graph, beside the supervoxel order and the
  // moment pass (and by the SMs, so not behind uploads the caller has in flight on the copy
  // engines); others are copied first
  if (!mapped) TG_CUDA(cudaMemcpyAsync(scratch, gm_host, bytes, cudaMemcpyHostToDevice, st), "upload Gaussians");
  const TgmmGaussian* src = (const TgmmGaussian*)mapped;
  TgmmEmStats local;
  int rc = em_run_batch(P, 1, frame, &scratch, &rnk_dev, &ind_dev, params, stats ? stats : &local, stream,
                        mapped ? &src : nullptr);
  if (rc != TGMM_OK && rc != TGMM_ERR_NAN_INPUT) return rc;
  TG_CUDA(cudaMemcpyAsync(gm_host, scratch, bytes, cudaMemcpyDeviceToHost, st), "download Gaussians");
  if (ind_tr_dev) {
    // reference-compatible Gaussian-sorted copy of the candidate ids (indCUDAtr)
    const size_t n = (size_t)TGMM_J * frame->n_sv;
    std::vector<int32_t> h(n);
    TG_CUDA(cudaMemcpyAsync(h.data(), ind_dev, n * 4, cudaMemcpyDeviceToHost, st), "read ind");
    TG_CUDA(cudaStreamSynchronize(st), "synchronize");
    std::stable_sort(h.begin(), h.end());
    TG_CUDA(cudaMemcpyAsync(ind_tr_dev, h.data(), n * 4, cudaMemcpyHostToDevice, st), "write ind_tr");
  }
  TG_CUDA(cudaStreamSynchronize(st), "synchronize");
  return rc;
}

int tgmm_frame_upload(const float* q, const float* img, const float* cent, const int64_t* lptr, int64_t n_vox,
                      int32_t n_sv, TgmmFrame* out) {
  if (!q || !img || !cent || !lptr || !out || n_vox < 0 || n_sv < 1) return fail(TGMM_ERR_INVALID_ARG, "bad frame");
  memset(out, 0, sizeof(*out));
  float *dq = nullptr, *di = nullptr, *dc = nullptr;
  int64_t* dl = nullptr;
  cudaError_t e = cudaMalloc(&dq, sizeof(float) * 3 * std::max<int64_t>(n_vox, 1));
  if (e == cudaSuccess) e = cudaMalloc(&di, sizeof(float) * std::max<int64_t>(n_vox, 1));
  if (e == cudaSuccess) e = cudaMalloc(&dc, sizeof(float) * 3 * n_sv);
  if (e == cudaSuccess) e = cudaMalloc(&dl, sizeof(int64_t) * (n_sv + 1));
  if (e != cudaSuccess) {
    cudaFree(dq);
    cudaFree(di);
    cudaFree(dc);
    cudaFree(dl);
    return fail(TGMM_ERR_OOM, "tgmm_frame_upload", e);
  }
  e = cudaMemcpy(dq, q, sizeof(float) * 3 * n_vox, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(di, img, sizeof(float) * n_vox, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dc, cent, sizeof(float) * 3 * n_sv, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dl, lptr, sizeof(int64_t) * (n_sv + 1), cudaMemcpyHostToDevice);
  out->query = dq;
  out->img = di;
  out->centroids = dc;
  out->label_ptr = dl;
  out->n_vox = n_vox;
  out->n_sv = n_sv;
  if (e != cudaSuccess) {
    tgmm_frame_release(out);
    return fail(TGMM_ERR_CUDA, "tgmm_frame_upload copy", e);
  }
  return TGMM_OK;
}

int tgmm_frame_release(TgmmFrame* f) {
  if (!f) return TGMM_OK;
  cudaFree((void*)f->query);
  cudaFree((void*)f->img);
  cudaFree((void*)f->centroids);
  cudaFree((void*)f->label_ptr);
  memset(f, 0, sizeof(*f));
  return TGMM_OK;
}

int tgmm_assign_supervoxels(const float* rnk, const int32_t* ind, int32_t n_sv, TgmmGaussian* gm, int32_t n_gauss) {
  if (!rnk || !ind || !gm || n_sv < 0) return fail(TGMM_ERR_INVALID_ARG, "tgmm_assign_supervoxels");
  for (int32_t k = 0; k < n_gauss; k++) gm[k].supervoxelNum = 0;
  int64_t p = 0;
  for (int j = 0; j < TGMM_J; j++)
    for (int32_t s = 0; s < n_sv; s++, p++) {
      if ((double)rnk[p] > 0.5) {
        const int32_t k = ind[p];
        if (k < 0 || k >= n_gauss) return fail(TGMM_ERR_INVALID_ARG, "ind out of range");
        TgmmGaussian& g = gm[k];
        if (g.supervoxelNum < TGMM_MAX_SV_PER_GAUSSIAN) g.supervoxelIdx[g.supervoxelNum++] = s;
      }
    }
  return TGMM_OK;
}

int tgmm_write_rnk_file(const char* path, const float* rnk, const int32_t* ind, int32_t n_sv) {
  if (!path || !rnk || !ind || n_sv < 0) return fail(TGMM_ERR_INVALID_ARG, "tgmm_write_rnk_file");
  FILE* fp = fopen(path, "wb");
  if (!fp) return fail(TGMM_ERR_INVALID_ARG, "cannot open rnk file");
  const int32_t hdr[2] = {n_sv, TGMM_J};
  size_t ok = fwrite(hdr, sizeof(int32_t), 2, fp);
  ok += fwrite(rnk, sizeof(float), (size_t)TGMM_J * n_sv, fp);
  ok += fwrite(ind, sizeof(int32_t), (size_t)TGMM_J * n_sv, fp);
  fclose(fp);
  if (ok != 2 + 2 * (size_t)TGMM_J * n_sv) return fail(TGMM_ERR_INVALID_ARG, "short write of rnk file");
  return TGMM_OK;
}

int tgmm_knn(const float* query, int64_t nq, const float* ref, int32_t nref, const float scale[3], int32_t* ind,
             void* stream) {
  if (!query || !ref || !scale || !ind || nq < 0) return fail(TGMM_ERR_INVALID_ARG, "tgmm_knn");
  if (nref < TGMM_J) return fail(TGMM_ERR_BAD_SIZE, "tgmm_knn needs at least 5 reference points");
  if (nq == 0) return TGMM_OK;
  cudaError_t e = knn_grid_standalone(query, nq, ref, nref, scale, ind, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(TGMM_ERR_CUDA, "tgmm_knn", e);
  return TGMM_OK;
}

int tgmm_knn_k(const float* query, int64_t nq, const float* ref, int32_t nref, int32_t k, const float scale[3],
               int32_t* ind, float* dist, void* stream) {
  if (!query || !ref || !scale || !ind || nq < 0 || nref < 0) return fail(TGMM_ERR_INVALID_ARG, "tgmm_knn_k");
  if (k < 1 || k > kMaxK) return fail(TGMM_ERR_BAD_SIZE, "tgmm_knn_k: k must be 1..11");
  if (nq == 0) return TGMM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (nref == 0) {  // nothing to assign: every slot empty
    TG_CUDA(cudaMemsetAsync(ind, 0xff, sizeof(int32_t) * (size_t)k * nq, st), "tgmm_knn_k");
    if (dist) {
      std::vector<float> big((size_t)k * nq, 1e32f);
      TG_CUDA(cudaMemcpyAsync(dist, big.data(), big.size() * 4, cudaMemcpyHostToDevice, st), "tgmm_knn_k");
      TG_CUDA(cudaStreamSynchronize(st), "tgmm_knn_k");
    }
    return TGMM_OK;
  }
  cudaError_t e = knn_grid_topk(query, nq, ref, nref, 1, k, scale, ind, dist, st);
  if (e != cudaSuccess) return fail(TGMM_ERR_CUDA, "tgmm_knn_k", e);
  return TGMM_OK;
}

int tgmm_update_priors(TgmmGaussian* gm, int32_t n, double bp, double np, double ap, double atot, int32_t compute,
                       void* stream) {
  if (!gm || n < 0) return fail(TGMM_ERR_INVALID_ARG, "tgmm_update_priors");
  if (n == 0) return TGMM_OK;
  cudaError_t e = update_priors_device(gm, n, bp, np, ap, atot, compute, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(TGMM_ERR_CUDA, "tgmm_update_priors", e);
  return TGMM_OK;
}

}  // extern "C"
