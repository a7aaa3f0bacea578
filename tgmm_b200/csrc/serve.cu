// serve.cu -- the served form of the EM (tgmm_serve.h): lineages resident on the device,
// a worker thread that admits submitted frames against an HBM budget, packs ready frames
// of different lineages into batches and runs each batch through tgmm_em_run_batch on one
// of several lanes (stream + plan), then turns each lineage's posterior into the prior of
// its next frame on the device.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/tgmm_serve.h"
#include "em_plan.h"

namespace {

constexpr int64_t kGranule = 256;
int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// First-fit allocator over byte offsets of one device allocation; neighbouring free
// ranges are merged on release.
class Arena {
 public:
  explicit Arena(int64_t capacity) : cap_(capacity) {
    if (cap_ > 0) free_[0] = cap_;
  }
  int64_t alloc(int64_t n) {
    n = round_up(std::max<int64_t>(n, 1), kGranule);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const int64_t off = it->first, rest = it->second - n;
      free_.erase(it);
      if (rest) free_[off + n] = rest;
      used_ += n;
      peak_ = std::max(peak_, used_);
      return off;
    }
    return -1;
  }
  void release(int64_t off, int64_t n) {
    n = round_up(std::max<int64_t>(n, 1), kGranule);
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  int64_t capacity() const { return cap_; }
  int64_t used() const { return used_; }
  int64_t peak() const { return peak_; }
  size_t fragments() const { return free_.size(); }

 private:
  int64_t cap_, used_ = 0, peak_ = 0;
  std::map<int64_t, int64_t> free_;
};

// How a request's voxels cross to the device: the float arrays, the 6-byte codes, or runs.
enum class Form { kFloat, kCompact, kRuns };

Form form_of(const TgmmServeRequest& r) {
  if (!r.query && !r.img && !r.lin && r.raw && r.run_ptr && r.run_start && r.run_len) return Form::kRuns;
  if (!r.query && !r.img && r.lin && r.raw) return Form::kCompact;
  return Form::kFloat;
}

// Device bytes of one frame: inputs, outputs and (compact and run forms) the uploaded voxel
// codes, each 256-byte aligned.
struct FrameLayout {
  int64_t query, img, cent, lptr, rnk, ind, lin = -1, raw = -1, rptr = -1, rstart = -1, rlen = -1, total;
  FrameLayout(const TgmmServeRequest& r) : FrameLayout(r.n_vox, r.n_sv, form_of(r), r.n_runs) {}
  FrameLayout(int64_t n_vox, int32_t n_sv, Form form, int64_t n_runs) {
    int64_t o = 0;
    auto take = [&](int64_t b) {
      const int64_t at = o;
      o += round_up(std::max<int64_t>(b, 1), kGranule);
      return at;
    };
    query = take(12 * n_vox);
    img = take(4 * n_vox);
    cent = take(12 * (int64_t)n_sv);
    lptr = take(8 * ((int64_t)n_sv + 1));
    rnk = take(4 * (int64_t)TGMM_J * n_sv);
    ind = take(4 * (int64_t)TGMM_J * n_sv);
    if (form == Form::kCompact) lin = take(4 * n_vox);
    if (form != Form::kFloat) raw = take(2 * n_vox);
    if (form == Form::kRuns) {
      rptr = take(4 * ((int64_t)n_sv + 1));
      rstart = take(4 * n_runs);
      rlen = take(2 * n_runs);
    }
    total = o;
  }
};

// Host memory the device can copy into directly (page-locked or registered).
bool page_locked(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Compact voxels -> the float frame (x, y, z blocks and intensities), exactly as the host
// builds them.
__global__ void k_expand_frame(const uint32_t* __restrict__ lin, const uint16_t* __restrict__ raw, int64_t n,
                               uint32_t X, uint32_t Y, double off, double den, float* __restrict__ query,
                               float* __restrict__ img) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = lin[i];
    const uint32_t q = v / X;
    query[i] = (float)(v - q * X);
    query[n + i] = (float)(q % Y);
    query[2 * n + i] = (float)(q / Y);
    img[i] = (float)(((double)raw[i] - off) / den);
  }
}

// Runs -> the float frame.  A warp per supervoxel s walks its runs rp[s] .. rp[s+1] in groups
// of 32 (a run per lane): a warp scan of the lengths places each run inside the supervoxel's
// voxel range lptr[s] .. lptr[s+1], then the lanes write the group's voxels together (voxel j
// of the group belongs to the run whose scanned end is the first above j), so that the stores
// are coalesced.  Nothing is written outside the supervoxel's range, whatever the run table
// says.  Coordinates and intensities as k_expand_frame.
__global__ void __launch_bounds__(256) k_expand_runs(const int32_t* __restrict__ rp, const uint32_t* __restrict__ rs,
                                                     const uint16_t* __restrict__ rl, const uint16_t* __restrict__ raw,
                                                     const int64_t* __restrict__ lptr, int32_t n_sv, int64_t n_runs,
                                                     int64_t n, uint32_t X, uint32_t Y, double off, double den,
                                                     float* __restrict__ query, float* __restrict__ img) {
  const int lane = threadIdx.x & 31;
  const int warps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int s = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); s < n_sv; s += warps) {
    const int64_t v0 = lptr[s], v1 = lptr[s + 1];
    if (v0 < 0 || v1 < v0 || v1 > n) continue;  // an invalid CSR, which the EM reports
    // runs outside 0 .. n_runs are never read
    const int64_t r0 = max((int64_t)rp[s], (int64_t)0), r1 = min((int64_t)rp[s + 1], n_runs);
    int64_t base = v0;
    for (int64_t r = r0; r < r1 && base < v1; r += 32) {
      const bool has = r + lane < r1;
      const int len = has ? (int)rl[r + lane] : 0;
      const uint32_t st = has ? rs[r + lane] : 0u;
      int inc = len;  // inclusive scan of the lengths
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      const int total = __shfl_sync(0xffffffffu, inc, 31);
      for (int j0 = 0; j0 < total; j0 += 32) {
        const int j = j0 + lane;
        int m = 0;  // lanes whose run ends at or before voxel j
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int t = __shfl_sync(0xffffffffu, inc, m + step - 1);
          if (t <= j) m += step;
        }
        const int end = __shfl_sync(0xffffffffu, inc, m);
        const int lm = __shfl_sync(0xffffffffu, len, m);
        const uint32_t sm = __shfl_sync(0xffffffffu, st, m);
        const int64_t i = base + j;
        if (j < total && i < v1) {
          const uint32_t v = sm + (uint32_t)(j - (end - lm));
          const uint32_t q = v / X;
          query[i] = (float)(v - q * X);
          query[n + i] = (float)(q % Y);
          query[2 * n + i] = (float)(q / Y);
          img[i] = (float)(((double)raw[i] - off) / den);
        }
      }
      base += total;
    }
  }
}

int expand_runs(const int32_t* rp, const uint32_t* rs, const uint16_t* rl, const uint16_t* raw, const int64_t* lptr,
                int32_t n_sv, int64_t n_runs, int64_t n_vox, const int32_t* dims, double off, double den, float* query,
                float* img, cudaStream_t st) {
  if (n_sv == 0 || n_vox == 0) return TGMM_OK;
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t blocks = std::min<int64_t>(((int64_t)n_sv + 7) / 8, (int64_t)sms * 8);
  k_expand_runs<<<(int)blocks, 256, 0, st>>>(rp, rs, rl, raw, lptr, n_sv, n_runs, n_vox, (uint32_t)dims[0],
                                             (uint32_t)dims[1], off, den, query, img);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return tgmm::report_error(TGMM_ERR_CUDA, "tgmm_frame_expand_runs", e);
  return TGMM_OK;
}

}  // namespace

extern "C" int tgmm_frame_expand_runs(const int32_t* run_ptr_dev, const uint32_t* run_start_dev,
                                      const uint16_t* run_len_dev, const uint16_t* raw_dev,
                                      const int64_t* label_ptr_dev, int32_t n_sv, int64_t n_runs, int64_t n_vox,
                                      const int32_t dims[3], double raw_offset, double raw_denom, float* query_dev,
                                      float* img_dev, void* stream) {
  if (!dims || n_vox < 0 || n_sv < 0 || n_runs < 0 ||
      (n_vox > 0 && n_sv > 0 &&
       (!run_ptr_dev || !run_start_dev || !run_len_dev || !raw_dev || !label_ptr_dev || !query_dev || !img_dev)))
    return tgmm::report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_expand_runs: null argument or negative size",
                              cudaSuccess);
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || (int64_t)dims[0] * dims[1] * dims[2] > 0xffffffffLL)
    return tgmm::report_error(TGMM_ERR_BAD_SIZE, "tgmm_frame_expand_runs: the volume must have 1 .. 2^32 voxels",
                              cudaSuccess);
  if (!(raw_denom != 0.0))
    return tgmm::report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_expand_runs: raw_denom is 0", cudaSuccess);
  return expand_runs(run_ptr_dev, run_start_dev, run_len_dev, raw_dev, label_ptr_dev, n_sv, n_runs, n_vox, dims,
                     raw_offset,
                     raw_denom, query_dev, img_dev, (cudaStream_t)stream);
}

extern "C" int tgmm_frame_expand(const uint32_t* lin_dev, const uint16_t* raw_dev, int64_t n_vox,
                                 const int32_t dims[3], double raw_offset, double raw_denom, float* query_dev,
                                 float* img_dev, void* stream) {
  if (!dims || n_vox < 0 || (n_vox > 0 && (!lin_dev || !raw_dev || !query_dev || !img_dev)))
    return tgmm::report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_expand: null argument or negative size", cudaSuccess);
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || (int64_t)dims[0] * dims[1] * dims[2] > 0xffffffffLL)
    return tgmm::report_error(TGMM_ERR_BAD_SIZE, "tgmm_frame_expand: the volume must have 1 .. 2^32 voxels", cudaSuccess);
  if (!(raw_denom != 0.0)) return tgmm::report_error(TGMM_ERR_INVALID_ARG, "tgmm_frame_expand: raw_denom is 0", cudaSuccess);
  if (n_vox == 0) return TGMM_OK;
  const int threads = 256;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t blocks = std::min<int64_t>((n_vox + threads - 1) / threads, (int64_t)sms * 16);
  k_expand_frame<<<(int)blocks, threads, 0, (cudaStream_t)stream>>>(lin_dev, raw_dev, n_vox, (uint32_t)dims[0],
                                                                     (uint32_t)dims[1], raw_offset, raw_denom,
                                                                     query_dev, img_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return tgmm::report_error(TGMM_ERR_CUDA, "tgmm_frame_expand", e);
  return TGMM_OK;
}

namespace {

struct Request {
  TgmmServeRequest r;
  bool direct[3] = {false, false, false};  // rnk, ind, gm outputs downloaded in place
  uint64_t seq = 0;
  double t_submit = 0.0, t_start = 0.0;
  int64_t off = -1, bytes = 0;  // arena range once admitted
  cudaEvent_t ready = nullptr;  // its upload (and expansion) done
};

struct Lineage {
  int32_t n_gauss = 0;
  int64_t off = -1, bytes = 0;
  TgmmGaussian* gm_dev = nullptr;
  std::deque<Request*> queue;  // the front one is in flight when in_flight
  bool in_flight = false;
};

struct Lane {
  TgmmPlan* plan = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  bool busy = false;
  bool tuned = false;  // the plan's kNN/E-step width and arrangement set (see launch)
  int launch_rc = TGMM_OK;
  int32_t batch_id = 0;
  std::vector<Request*> reqs;
  std::vector<int32_t> lineage_ids;
  std::vector<TgmmGaussian*> gm_dev;  // the batch's lineages, captured when it is formed
  std::vector<int32_t> n_gauss;
  // pinned staging of the batch outputs
  float* h_rnk = nullptr;
  int32_t* h_ind = nullptr;
  TgmmGaussian* h_gm = nullptr;
  unsigned char* h_state = nullptr;
  std::vector<int64_t> sv_off, g_off;
};

}  // namespace

struct TgmmServer {
  TgmmServerDesc desc{};
  char* dev = nullptr;
  Arena* arena = nullptr;
  std::vector<Lane> lanes;
  std::map<int32_t, Lineage> lineages;
  int32_t next_lineage = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> inbox;
  std::deque<TgmmServeResult> results;
  std::thread worker;
  bool stop = false;
  cudaStream_t copy = nullptr;         // uploads of admitted frames
  std::vector<cudaEvent_t> free_events;
  int64_t h2d_bytes = 0;
  uint64_t seq = 0;
  int64_t submitted = 0, completed = 0, rejected = 0, batches = 0, frames_in_batches = 0;
  int32_t queued = 0, in_flight = 0;  // in the inbox; in lineage queues (waiting or running)
  int64_t lineage_bytes = 0;          // arena bytes held by resident lineages
  std::chrono::steady_clock::time_point t0;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  void run();
  void admit();
  int upload(Request* q);
  void finish(Request* q, int status, const TgmmEmStats* st, int32_t batch_id, int32_t batch_frames);
  bool form_batch(Lane& L, std::vector<Request*>& batch);
  void launch(Lane& L);
  void complete(Lane& L);
};

namespace {

int fail(int code, const char* what, cudaError_t e = cudaSuccess) { return tgmm::report_error(code, what, e); }

#define SV_CUDA(call, what)                                     \
  do {                                                          \
    cudaError_t e_ = (call);                                    \
    if (e_ != cudaSuccess) return fail(TGMM_ERR_CUDA, what, e_); \
  } while (0)

}  // namespace

// Result of one request (lock held).  The request leaves its lineage's queue.
void TgmmServer::finish(Request* q, int status, const TgmmEmStats* st, int32_t batch_id, int32_t batch_frames) {
  TgmmServeResult res;
  memset(&res, 0, sizeof(res));
  res.tag = q->r.tag;
  res.lineage = q->r.lineage;
  res.status = status;
  if (st) res.stats = *st;
  res.submit_ms = q->t_submit;
  res.start_ms = q->t_start;
  res.done_ms = now_ms();
  res.batch_id = batch_id;
  res.batch_frames = batch_frames;
  results.push_back(res);
  if (q->off >= 0) arena->release(q->off, q->bytes);
  if (q->ready) free_events.push_back(q->ready);
  completed++;
  if (status == TGMM_ERR_ADMISSION || status == TGMM_ERR_BAD_SIZE || status == TGMM_ERR_INVALID_ARG) rejected++;
  delete q;
  cv_done.notify_all();
}

// Frames for lane L: the oldest ready frame of each lineage with nothing in flight, in
// submission order, while the batch capacity and the HBM budget allow (lock held).
bool TgmmServer::form_batch(Lane& L, std::vector<Request*>& batch) {
  std::vector<std::pair<uint64_t, int32_t>> ready;
  for (auto& kv : lineages)
    if (!kv.second.in_flight && !kv.second.queue.empty() && kv.second.queue.front()->off >= 0)
      ready.push_back({kv.second.queue.front()->seq, kv.first});
  std::sort(ready.begin(), ready.end());
  int64_t vox = 0, sv = 0, gauss = 0;
  for (auto& rd : ready) {
    if ((int32_t)batch.size() >= desc.max_batch_frames) break;
    Lineage& G = lineages[rd.second];
    Request* q = G.queue.front();
    if (vox + q->r.n_vox > desc.max_batch_vox || sv + q->r.n_sv > desc.max_batch_sv ||
        gauss + G.n_gauss > desc.max_batch_gauss)
      continue;
    G.in_flight = true;
    batch.push_back(q);
    L.lineage_ids.push_back(rd.second);
    L.gm_dev.push_back(G.gm_dev);
    L.n_gauss.push_back(G.n_gauss);
    vox += q->r.n_vox;
    sv += q->r.n_sv;
    gauss += G.n_gauss;
  }
  return !batch.empty();
}

// Enqueue the batch on the lane (lock not held; only the lane and its requests are used).
void TgmmServer::launch(Lane& L) {
  const int n = (int)L.reqs.size();
  std::vector<TgmmFrame> fr(n);
  std::vector<TgmmGaussian*> gm(n);
  std::vector<float*> rnk(n);
  std::vector<int32_t*> ind(n);
  L.sv_off.assign(n, 0);
  L.g_off.assign(n, 0);
  int rc = TGMM_OK;
  int64_t so = 0, go = 0;
  for (int i = 0; i < n && rc == TGMM_OK; i++) {
    Request* q = L.reqs[i];
    const FrameLayout lay(q->r);
    char* base = dev + q->off;
    const int64_t N = q->r.n_vox, S = q->r.n_sv;
    const cudaError_t e = cudaStreamWaitEvent(L.st, q->ready, 0);  // its upload
    if (e != cudaSuccess) rc = fail(TGMM_ERR_CUDA, "serve: wait for upload", e);
    fr[i].query = (const float*)(base + lay.query);
    fr[i].img = (const float*)(base + lay.img);
    fr[i].centroids = (const float*)(base + lay.cent);
    fr[i].label_ptr = (const int64_t*)(base + lay.lptr);
    fr[i].n_vox = N;
    fr[i].n_sv = (int32_t)S;
    fr[i].n_gauss = L.n_gauss[i];
    gm[i] = L.gm_dev[i];
    rnk[i] = (float*)(base + lay.rnk);
    ind[i] = (int32_t*)(base + lay.ind);
    L.sv_off[i] = so;
    L.g_off[i] = go;
    so += TGMM_J * S;
    go += L.n_gauss[i];
  }
  if (rc == TGMM_OK && !L.tuned) {
    // the server's first batch tunes its lane's plan; every other lane takes the same
    // setting, so no later batch (and no lane first used late in a stream) pays for tuning
    int32_t width = 0, fused = 0;
    rc = tgmm_plan_autotune(L.plan, n, fr.data(), gm.data(), rnk.data(), ind.data(), &desc.params, 2, &width, L.st);
    if (rc == TGMM_OK) rc = tgmm_plan_tuning(L.plan, &width, &fused);
    for (Lane& O : lanes)
      if (rc == TGMM_OK && &O != &L) {
        rc = tgmm_plan_set_knn_group(O.plan, width);
        if (rc == TGMM_OK) rc = tgmm_plan_set_knn_fusion(O.plan, fused);
      }
    for (Lane& O : lanes) O.tuned = true;
  }
  if (rc == TGMM_OK)
    rc = tgmm_em_run_batch(L.plan, n, fr.data(), gm.data(), rnk.data(), ind.data(), &desc.params, nullptr, L.st);
  if (rc == TGMM_OK) rc = tgmm::plan_enqueue_state(L.plan, n, L.h_state, L.st);
  for (int i = 0; i < n && rc == TGMM_OK; i++) {
    Request* q = L.reqs[i];
    const int64_t S = q->r.n_sv;
    const int32_t K = fr[i].n_gauss;
    cudaError_t e = cudaSuccess;
    // outputs in page-locked memory are written in place, the others through the lane's
    // staging and a host copy when the batch is done
    q->direct[0] = page_locked(q->r.rnk_out);
    q->direct[1] = page_locked(q->r.ind_out);
    q->direct[2] = page_locked(q->r.gm_out);
    if (q->r.rnk_out)
      e = cudaMemcpyAsync(q->direct[0] ? q->r.rnk_out : L.h_rnk + L.sv_off[i], rnk[i], 4 * TGMM_J * S,
                          cudaMemcpyDeviceToHost, L.st);
    if (e == cudaSuccess && q->r.ind_out)
      e = cudaMemcpyAsync(q->direct[1] ? q->r.ind_out : L.h_ind + L.sv_off[i], ind[i], 4 * TGMM_J * S,
                          cudaMemcpyDeviceToHost, L.st);
    if (e == cudaSuccess && q->r.gm_out)
      e = cudaMemcpyAsync(q->direct[2] ? q->r.gm_out : L.h_gm + L.g_off[i], gm[i], sizeof(TgmmGaussian) * K,
                          cudaMemcpyDeviceToHost, L.st);
    if (e != cudaSuccess) rc = fail(TGMM_ERR_CUDA, "serve: download", e);
    // posterior -> prior of the lineage's next frame
    if (rc == TGMM_OK)
      rc = tgmm_update_priors(gm[i], K, desc.beta_pct, desc.nu_pct, desc.alpha_pct, -1.0, 1, L.st);
  }
  if (rc == TGMM_OK) {
    cudaError_t e = cudaEventRecord(L.ev, L.st);
    if (e != cudaSuccess) rc = fail(TGMM_ERR_CUDA, "serve: record", e);
  }
  L.launch_rc = rc;
}

// The lane's batch has finished on the device (lock held).
void TgmmServer::complete(Lane& L) {
  const int n = (int)L.reqs.size();
  const size_t sb = tgmm::frame_state_bytes();
  for (int i = 0; i < n; i++) {
    Request* q = L.reqs[i];
    Lineage& G = lineages.at(L.lineage_ids[i]);
    TgmmEmStats st;
    memset(&st, 0, sizeof(st));
    int status = L.launch_rc;
    if (status == TGMM_OK) {
      status = tgmm::frame_state_to_stats(L.h_state + sb * i, &st);
      const int64_t S = q->r.n_sv;
      if (q->r.rnk_out && !q->direct[0]) memcpy(q->r.rnk_out, L.h_rnk + L.sv_off[i], 4 * TGMM_J * S);
      if (q->r.ind_out && !q->direct[1]) memcpy(q->r.ind_out, L.h_ind + L.sv_off[i], 4 * TGMM_J * S);
      if (q->r.gm_out && !q->direct[2]) memcpy(q->r.gm_out, L.h_gm + L.g_off[i], sizeof(TgmmGaussian) * G.n_gauss);
    }
    G.in_flight = false;
    G.queue.pop_front();
    in_flight--;
    finish(q, status, status == TGMM_OK || status == TGMM_ERR_NAN_INPUT ? &st : nullptr, L.batch_id, n);
  }
  L.reqs.clear();
  L.lineage_ids.clear();
  L.gm_dev.clear();
  L.n_gauss.clear();
  L.busy = false;
}

// Upload of an admitted frame on the copy stream (lock held; the copies are asynchronous
// from page-locked memory).
int TgmmServer::upload(Request* q) {
  const Form form = form_of(q->r);
  const FrameLayout lay(q->r);
  char* base = dev + q->off;
  const int64_t N = q->r.n_vox, S = q->r.n_sv;
  cudaError_t e = cudaSuccess;
  if (form == Form::kRuns) {
    // the label_ptr the expansion reads goes up first
    const int64_t R = q->r.n_runs;
    e = cudaMemcpyAsync(base + lay.lptr, q->r.label_ptr, 8 * (S + 1), cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + lay.rptr, q->r.run_ptr, 4 * (S + 1), cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + lay.rstart, q->r.run_start, 4 * R, cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + lay.rlen, q->r.run_len, 2 * R, cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + lay.raw, q->r.raw, 2 * N, cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess &&
        expand_runs((const int32_t*)(base + lay.rptr), (const uint32_t*)(base + lay.rstart),
                    (const uint16_t*)(base + lay.rlen), (const uint16_t*)(base + lay.raw),
                    (const int64_t*)(base + lay.lptr), (int32_t)S, R, N, q->r.dims, q->r.raw_offset, q->r.raw_denom,
                    (float*)(base + lay.query), (float*)(base + lay.img), copy) != TGMM_OK)
      e = cudaErrorLaunchFailure;
    h2d_bytes += 2 * N + 6 * R + 4 * (S + 1);
  } else if (form == Form::kCompact) {
    e = cudaMemcpyAsync(base + lay.lin, q->r.lin, 4 * N, cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + lay.raw, q->r.raw, 2 * N, cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess && N > 0) {
      const int threads = 256;
      const int64_t blocks = std::min<int64_t>((N + threads - 1) / threads, 148 * 16);
      k_expand_frame<<<(int)blocks, threads, 0, copy>>>(
          (const uint32_t*)(base + lay.lin), (const uint16_t*)(base + lay.raw), N, (uint32_t)q->r.dims[0],
          (uint32_t)q->r.dims[1], q->r.raw_offset, q->r.raw_denom, (float*)(base + lay.query),
          (float*)(base + lay.img));
      e = cudaGetLastError();
    }
    h2d_bytes += 6 * N;
  } else {
    e = cudaMemcpyAsync(base + lay.query, q->r.query, 12 * N, cudaMemcpyHostToDevice, copy);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + lay.img, q->r.img, 4 * N, cudaMemcpyHostToDevice, copy);
    h2d_bytes += 16 * N;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + lay.cent, q->r.centroids, 12 * S, cudaMemcpyHostToDevice, copy);
  if (e == cudaSuccess && form != Form::kRuns)
    e = cudaMemcpyAsync(base + lay.lptr, q->r.label_ptr, 8 * (S + 1), cudaMemcpyHostToDevice, copy);
  h2d_bytes += 12 * S + 8 * (S + 1);
  if (e == cudaSuccess) {
    if (free_events.empty()) {
      cudaEvent_t ev;
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e == cudaSuccess) free_events.push_back(ev);
    }
    if (e == cudaSuccess) {
      q->ready = free_events.back();
      free_events.pop_back();
      e = cudaEventRecord(q->ready, copy);
    }
  }
  return e == cudaSuccess ? TGMM_OK : fail(TGMM_ERR_CUDA, "serve: upload", e);
}

// Admission in arrival order: every queued frame that fits the HBM budget gets its buffers
// and its upload, whether or not its lineage is ready (lock held).
void TgmmServer::admit() {
  std::vector<Request*> waiting;
  for (auto& kv : lineages)
    for (Request* q : kv.second.queue)
      if (q->off < 0) waiting.push_back(q);
  std::sort(waiting.begin(), waiting.end(), [](const Request* a, const Request* b) { return a->seq < b->seq; });
  for (Request* q : waiting) {
    const FrameLayout lay(q->r);
    const int64_t off = arena->alloc(lay.total);
    if (off < 0) break;  // later frames wait behind this one: admission keeps arrival order
    q->off = off;
    q->bytes = lay.total;
    if (upload(q) != TGMM_OK) {
      q->ready = nullptr;
      // leaves the frame admitted; its batch reports the failure through the lane
    }
  }
}

void TgmmServer::run() {
  cudaSetDevice(desc.device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    // intake: frames join their lineage's queue; frames that can never run are answered
    while (!inbox.empty()) {
      Request* q = inbox.front();
      inbox.pop_front();
      queued--;
      auto it = lineages.find(q->r.lineage);
      if (it == lineages.end()) {
        finish(q, TGMM_ERR_INVALID_ARG, nullptr, -1, 0);
        continue;
      }
      const FrameLayout lay(q->r);
      if (q->r.n_vox > desc.max_batch_vox || q->r.n_sv > desc.max_batch_sv ||
          it->second.n_gauss > desc.max_batch_gauss) {
        finish(q, TGMM_ERR_BAD_SIZE, nullptr, -1, 0);
        continue;
      }
      if (lay.total > arena->capacity() - lineage_bytes) {  // could never be admitted
        finish(q, TGMM_ERR_ADMISSION, nullptr, -1, 0);
        continue;
      }
      it->second.queue.push_back(q);
      in_flight++;
    }
    admit();
    bool progressed = false;
    for (Lane& L : lanes) {
      if (!L.busy) continue;
      const cudaError_t e = L.launch_rc == TGMM_OK ? cudaEventQuery(L.ev) : cudaSuccess;
      if (e == cudaErrorNotReady) continue;
      if (e != cudaSuccess && L.launch_rc == TGMM_OK) L.launch_rc = fail(TGMM_ERR_CUDA, "serve: batch", e);
      complete(L);
      progressed = true;
    }
    for (Lane& L : lanes) {
      if (L.busy) continue;
      std::vector<Request*> batch;
      if (!form_batch(L, batch)) break;
      L.reqs = batch;
      L.busy = true;
      L.batch_id = (int32_t)batches++;
      frames_in_batches += (int64_t)batch.size();
      const double t = now_ms();
      for (Request* q : batch) q->t_start = t;
      lk.unlock();
      launch(L);
      lk.lock();
      if (L.launch_rc != TGMM_OK) {  // nothing to wait for: answer the batch now
        cudaStreamSynchronize(L.st);
        complete(L);
      }
      progressed = true;
    }
    bool any_busy = false, any_queued = false;
    for (Lane& L : lanes) any_busy |= L.busy;
    for (auto& kv : lineages) any_queued |= !kv.second.queue.empty();
    if (stop && !any_busy && !any_queued && inbox.empty()) break;
    if (progressed) continue;
    if (any_busy)
      cv_work.wait_for(lk, std::chrono::microseconds(20));
    else
      cv_work.wait(lk, [&] { return !inbox.empty() || stop; });
  }
}

extern "C" {

void tgmm_server_default_desc(TgmmServerDesc* d) {
  if (!d) return;
  memset(d, 0, sizeof(*d));
  d->device = 0;
  d->hbm_budget = 0;
  d->lanes = 2;
  d->max_batch_frames = 64;
  d->max_batch_vox = (int64_t)1 << 25;
  d->max_batch_sv = 1 << 17;
  d->max_batch_gauss = 1 << 17;
  tgmm_default_params(&d->params);
  d->beta_pct = 0.01;
  d->nu_pct = 1.0;
  d->alpha_pct = 0.8;
}

int tgmm_server_create(const TgmmServerDesc* d, TgmmServer** out) {
  if (!d || !out) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_create: null argument");
  *out = nullptr;
  if (d->lanes < 1 || d->max_batch_frames < 1 || d->max_batch_vox < 1 || d->max_batch_sv < 1 ||
      d->max_batch_gauss < TGMM_J || d->hbm_budget < 0)
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_create: capacities must be positive");
  SV_CUDA(cudaSetDevice(d->device), "cudaSetDevice");
  TgmmServer* S = new TgmmServer();
  S->desc = *d;
  S->t0 = std::chrono::steady_clock::now();
  auto bail = [&](int rc) {
    tgmm_server_destroy(S);
    return rc;
  };
  TgmmPlanDesc pd;
  pd.max_vox = d->max_batch_vox;
  pd.max_sv = d->max_batch_sv;
  pd.max_gauss = d->max_batch_gauss;
  pd.max_frames = d->max_batch_frames;
  pd.device = d->device;
  S->lanes.resize(d->lanes);
  const size_t sb = tgmm::frame_state_bytes();
  for (Lane& L : S->lanes) {
    int rc = tgmm_plan_create(&pd, &L.plan);
    if (rc) return bail(rc);
    cudaError_t e = cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L.ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(&L.h_rnk, 4 * (size_t)TGMM_J * d->max_batch_sv);
    if (e == cudaSuccess) e = cudaMallocHost(&L.h_ind, 4 * (size_t)TGMM_J * d->max_batch_sv);
    if (e == cudaSuccess) e = cudaMallocHost(&L.h_gm, sizeof(TgmmGaussian) * (size_t)d->max_batch_gauss);
    if (e == cudaSuccess) e = cudaMallocHost(&L.h_state, sb * (size_t)d->max_batch_frames);
    if (e != cudaSuccess) return bail(fail(TGMM_ERR_CUDA, "tgmm_server_create: lane", e));
  }
  int64_t budget = d->hbm_budget;
  if (budget == 0) {
    size_t fr = 0, tot = 0;
    cudaError_t e = cudaMemGetInfo(&fr, &tot);
    if (e != cudaSuccess) return bail(fail(TGMM_ERR_CUDA, "tgmm_server_create: cudaMemGetInfo", e));
    budget = (int64_t)(0.8 * (double)fr);
  }
  budget = round_up(budget, kGranule);
  cudaError_t e = cudaMalloc(&S->dev, budget);
  if (e != cudaSuccess) return bail(fail(TGMM_ERR_OOM, "tgmm_server_create: HBM budget", e));
  S->desc.hbm_budget = budget;
  S->arena = new Arena(budget);
  e = cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(fail(TGMM_ERR_CUDA, "tgmm_server_create: copy stream", e));
  S->worker = std::thread([S] { S->run(); });
  *out = S;
  return TGMM_OK;
}

int tgmm_server_destroy(TgmmServer* S) {
  if (!S) return TGMM_OK;
  if (S->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->stop = true;
    }
    S->cv_work.notify_all();
    S->worker.join();
  }
  cudaSetDevice(S->desc.device);
  for (Lane& L : S->lanes) {
    if (L.st) cudaStreamSynchronize(L.st);
    if (L.plan) tgmm_plan_destroy(L.plan);
    if (L.ev) cudaEventDestroy(L.ev);
    if (L.st) cudaStreamDestroy(L.st);
    if (L.h_rnk) cudaFreeHost(L.h_rnk);
    if (L.h_ind) cudaFreeHost(L.h_ind);
    if (L.h_gm) cudaFreeHost(L.h_gm);
    if (L.h_state) cudaFreeHost(L.h_state);
  }
  if (S->copy) cudaStreamSynchronize(S->copy);
  for (Request* q : S->inbox) delete q;
  for (auto& kv : S->lineages)
    for (Request* q : kv.second.queue) {
      if (q->ready) cudaEventDestroy(q->ready);
      delete q;
    }
  for (cudaEvent_t ev : S->free_events) cudaEventDestroy(ev);
  if (S->copy) cudaStreamDestroy(S->copy);
  if (S->dev) cudaFree(S->dev);
  delete S->arena;
  delete S;
  return TGMM_OK;
}

int tgmm_server_open_lineage(TgmmServer* S, const TgmmGaussian* gm, int32_t n_gauss, int32_t* id) {
  if (!S || !gm || !id) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_open_lineage: null argument");
  if (n_gauss < TGMM_J) return fail(TGMM_ERR_BAD_SIZE, "tgmm_server_open_lineage: a lineage needs 5 Gaussians");
  if (n_gauss > S->desc.max_batch_gauss) return fail(TGMM_ERR_BAD_SIZE, "tgmm_server_open_lineage: beyond batch capacity");
  std::lock_guard<std::mutex> lk(S->mu);
  const int64_t bytes = (int64_t)sizeof(TgmmGaussian) * n_gauss;
  const int64_t off = S->arena->alloc(bytes);
  if (off < 0) return fail(TGMM_ERR_ADMISSION, "tgmm_server_open_lineage: HBM budget exhausted");
  SV_CUDA(cudaSetDevice(S->desc.device), "cudaSetDevice");
  cudaError_t e = cudaMemcpy(S->dev + off, gm, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    S->arena->release(off, bytes);
    return fail(TGMM_ERR_CUDA, "tgmm_server_open_lineage: upload", e);
  }
  Lineage G;
  G.n_gauss = n_gauss;
  G.off = off;
  G.bytes = bytes;
  G.gm_dev = (TgmmGaussian*)(S->dev + off);
  S->lineage_bytes += round_up(bytes, kGranule);
  *id = S->next_lineage++;
  S->lineages.emplace(*id, std::move(G));
  return TGMM_OK;
}

int tgmm_server_close_lineage(TgmmServer* S, int32_t id) {
  if (!S) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_close_lineage: null server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->lineages.find(id);
  if (it == S->lineages.end()) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_close_lineage: unknown lineage");
  for (Request* q : S->inbox)
    if (q->r.lineage == id) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_close_lineage: frames pending");
  if (!it->second.queue.empty()) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_close_lineage: frames pending");
  S->arena->release(it->second.off, it->second.bytes);
  S->lineage_bytes -= round_up(it->second.bytes, kGranule);
  S->lineages.erase(it);
  return TGMM_OK;
}

int tgmm_server_read_lineage(TgmmServer* S, int32_t id, TgmmGaussian* gm) {
  if (!S || !gm) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_read_lineage: null argument");
  std::unique_lock<std::mutex> lk(S->mu);
  auto pending = [&] {
    auto it = S->lineages.find(id);
    if (it == S->lineages.end()) return false;
    if (!it->second.queue.empty()) return true;
    for (Request* q : S->inbox)
      if (q->r.lineage == id) return true;
    return false;
  };
  S->cv_done.wait(lk, [&] { return !pending(); });
  auto it = S->lineages.find(id);
  if (it == S->lineages.end()) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_read_lineage: unknown lineage");
  SV_CUDA(cudaSetDevice(S->desc.device), "cudaSetDevice");
  SV_CUDA(cudaMemcpy(gm, it->second.gm_dev, sizeof(TgmmGaussian) * it->second.n_gauss, cudaMemcpyDeviceToHost),
          "tgmm_server_read_lineage: download");
  return TGMM_OK;
}

int tgmm_server_submit(TgmmServer* S, const TgmmServeRequest* r) {
  if (!S || !r) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_submit: null argument");
  const Form form = form_of(*r);
  if ((form == Form::kFloat && (!r->query || !r->img)) || !r->centroids || !r->label_ptr || r->n_vox < 0 ||
      r->n_sv < 1)
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_submit: bad frame");
  if (form != Form::kFloat &&
      (r->dims[0] < 1 || r->dims[1] < 1 || r->dims[2] < 1 || (int64_t)r->dims[0] * r->dims[1] * r->dims[2] > 0xffffffffLL ||
       !(r->raw_denom != 0.0)))
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_submit: bad compact or run frame");
  if (form == Form::kRuns && (r->n_runs < 0 || r->n_runs > r->n_vox))
    return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_submit: bad run count");
  Request* q = new Request();
  q->r = *r;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) {
      delete q;
      return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_submit: server stopping");
    }
    q->seq = S->seq++;
    q->t_submit = S->now_ms();
    S->inbox.push_back(q);
    S->queued++;
    S->submitted++;
  }
  S->cv_work.notify_one();
  return TGMM_OK;
}

int tgmm_server_poll(TgmmServer* S, TgmmServeResult* out, int32_t max, int32_t wait_ms, int32_t* n_out) {
  if (!S || !out || max < 1 || !n_out) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_poll: bad argument");
  std::unique_lock<std::mutex> lk(S->mu);
  auto ready = [&] { return !S->results.empty() || (S->queued == 0 && S->in_flight == 0); };
  if (wait_ms < 0)
    S->cv_done.wait(lk, ready);
  else if (wait_ms > 0)
    S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  int32_t n = 0;
  while (n < max && !S->results.empty()) {
    out[n++] = S->results.front();
    S->results.pop_front();
  }
  *n_out = n;
  return TGMM_OK;
}

int tgmm_server_stats(TgmmServer* S, TgmmServerStats* o) {
  if (!S || !o) return fail(TGMM_ERR_INVALID_ARG, "tgmm_server_stats: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  o->submitted = S->submitted;
  o->completed = S->completed;
  o->rejected = S->rejected;
  o->batches = S->batches;
  o->frames_in_batches = S->frames_in_batches;
  o->hbm_budget = S->arena->capacity();
  o->hbm_in_use = S->arena->used();
  o->hbm_peak = S->arena->peak();
  o->h2d_bytes = S->h2d_bytes;
  o->queued = S->queued;
  o->in_flight = S->in_flight;
  return TGMM_OK;
}

int tgmm_server_selftest(void) {
  int bad = 0;
  auto check = [&](bool c) { bad += c ? 0 : 1; };
  Arena a(10 * kGranule);
  const int64_t x = a.alloc(1), y = a.alloc(kGranule + 1), z = a.alloc(3 * kGranule);
  check(x == 0 && y == kGranule && z == 3 * kGranule);
  check(a.used() == 6 * kGranule);
  check(a.alloc(5 * kGranule) == -1);  // 4 granules left
  a.release(y, kGranule + 1);
  check(a.alloc(3 * kGranule) == 6 * kGranule);  // first fit skips the 2-granule hole
  check(a.alloc(2 * kGranule) == kGranule);      // and fills it next
  a.release(x, 1);
  a.release(kGranule, 2 * kGranule);
  a.release(z, 3 * kGranule);
  a.release(6 * kGranule, 3 * kGranule);
  check(a.used() == 0 && a.fragments() == 1);  // fully coalesced
  check(a.alloc(10 * kGranule) == 0);
  check(a.peak() == 10 * kGranule);
  const FrameLayout lay(1000, 10, Form::kFloat, 0);
  check(lay.total % kGranule == 0 && lay.img >= 12 * 1000 && lay.ind + 4 * 5 * 10 <= lay.total && lay.lin < 0 &&
        lay.raw < 0 && lay.rptr < 0);
  const FrameLayout cl(1000, 10, Form::kCompact, 0);
  check(cl.lin > cl.ind && cl.raw >= cl.lin + 4000 && cl.raw + 2000 <= cl.total && cl.rptr < 0);
  const FrameLayout rl(1000, 10, Form::kRuns, 300);
  check(rl.lin < 0 && rl.raw > rl.ind && rl.rptr >= rl.raw + 2000 && rl.rstart >= rl.rptr + 44 &&
        rl.rlen >= rl.rstart + 1200 && rl.rlen + 600 <= rl.total);
  return bad;
}

}  // extern "C"
