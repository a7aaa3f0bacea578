// split_round.cu -- the split round of one time point (mainTrackingGaussianMixtureModel.cpp:
// 1233-1507), with the candidates chosen by the caller instead of the reference's 3D Haar
// feature classifier, and the accept/reject decision left to the caller (the reference calls
// likelihoodRatioTestSplitMerge there, which its sources do not define).
//
//   1. the local log-likelihood around each candidate before the split: its supervoxels
//      (supervoxelIdx of the first EM), the first EM's mixture and candidates (main:1303-1331);
//   2. each candidate splits along its principal axis (GaussianMixtureModel::splitGaussian(GM,
//      id), GaussianMixtureModel.cpp:514-557) into itself and a new Gaussian appended after the
//      mixture, both with the split proposal's priors (updatePriorsAfterSplitProposal, :912-922);
//      every other Gaussian is fixed (main:1263);
//   3. the EM on the split mixture (main:1339-1346);
//   4. the local log-likelihood of the same supervoxels after it (main:1353-1358).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "tgmm_internal.cuh"

namespace {

// The principal-axis split of one record: S = nu W / (s_i s_j) (float products of the
// scale), lmin, v = its smallest eigenvalue and eigenvector, lmax its largest; sigma =
// 1/sqrt(max(lmin, 1e-3)); both halves take W = (lmax / nu) I with W_ii *= s_i s_i and
// N_k / 2 (N_k = nu_k - nu_o, as copyFromGMEM_CUDA derives it); a = m + sigma v,
// b = a - 2 sigma v; then the split proposal's priors: m_o = m_k, beta_o = max(N_k/2, 1e-5),
// nu_o = max(N_k/2, 3), W_o = W_k nu_k / nu_o.  v's sign makes its largest-magnitude
// component positive.
void split_proposal(const TgmmGaussian& g, const float s[3], TgmmGaussian* a, TgmmGaussian* b) {
  static const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  double w[6], d[3], v[9];
  for (int e = 0; e < 6; e++) w[e] = (g.W_k[e] * g.nu_k) / (double)(s[ij[e][0]] * s[ij[e][1]]);
  tgmm::eig3(w, d, v);
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
  const double sm2 = 1.0 / sqrt(d[imin] < 1e-3 ? 1e-3 : d[imin]);
  const double nk = 0.5 * (g.nu_k - g.nu_o);
  *a = g;
  for (int e = 0; e < 6; e++) a->W_k[e] = 0.0;
  a->W_k[0] = d[imax] / g.nu_k * (double)(s[0] * s[0]);
  a->W_k[3] = d[imax] / g.nu_k * (double)(s[1] * s[1]);
  a->W_k[5] = d[imax] / g.nu_k * (double)(s[2] * s[2]);
  for (int i = 0; i < 3; i++) a->m_k[i] = g.m_k[i] + sm2 * u[i];
  *b = *a;
  for (int i = 0; i < 3; i++) b->m_k[i] = a->m_k[i] - 2.0 * sm2 * u[i];
  TgmmGaussian* h[2] = {a, b};
  for (TgmmGaussian* x : h) {
    for (int i = 0; i < 3; i++) x->m_o[i] = x->m_k[i];
    x->beta_o = 0.5 * nk > 1e-5 ? 0.5 * nk : 1e-5;
    x->nu_o = 0.5 * nk > 3.0 ? 0.5 * nk : 3.0;
    for (int e = 0; e < 6; e++) x->W_o[e] = x->W_k[e] * x->nu_k / x->nu_o;
  }
}

}  // namespace

extern "C" int tgmm_split_proposal(const TgmmGaussian* g, const float scale[3], TgmmGaussian* a, TgmmGaussian* b) {
  if (!g || !scale || !a || !b) return tgmm::report_error(TGMM_ERR_INVALID_ARG, "tgmm_split_proposal: null argument", cudaSuccess);
  TgmmGaussian ga, gb;
  split_proposal(*g, scale, &ga, &gb);
  *a = ga;
  *b = gb;
  return TGMM_OK;
}

extern "C" int tgmm_split_round(TgmmPlan* plan, const TgmmFrame* frame, TgmmGaussian* gm_host, int32_t n_gauss,
                                const int32_t* ind_dev, const int32_t* cand, int32_t n_split, float* rnk_dev,
                                int32_t* ind_out_dev, const TgmmEmParams* params, double* ll_before, double* ll_after,
                                TgmmEmStats* stats, void* stream) {
  using tgmm::report_error;
  if (!plan || !frame || !gm_host || !ind_dev || !rnk_dev || !ind_out_dev || !params || n_split < 0 ||
      n_gauss < TGMM_J || (n_split > 0 && (!cand || !ll_before || !ll_after)))
    return report_error(TGMM_ERR_INVALID_ARG, "tgmm_split_round: null argument or bad size", cudaSuccess);
  std::vector<char> seen(n_gauss, 0);
  for (int32_t i = 0; i < n_split; i++) {
    const int32_t k = cand[i];
    if (k < 0 || k >= n_gauss) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_split_round: candidate out of range", cudaSuccess);
    if (seen[k]) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_split_round: a candidate is listed twice", cudaSuccess);
    if (gm_host[k].m_o[0] < -1e31) return report_error(TGMM_ERR_INVALID_ARG, "tgmm_split_round: a candidate is dead", cudaSuccess);
    if (gm_host[k].supervoxelNum < 0 || gm_host[k].supervoxelNum > TGMM_MAX_SV_PER_GAUSSIAN)
      return report_error(TGMM_ERR_INVALID_ARG, "tgmm_split_round: bad supervoxelNum", cudaSuccess);
    seen[k] = 1;
  }
  const int32_t n_total = n_gauss + n_split;
  cudaStream_t st = (cudaStream_t)stream;
  // the supervoxels around each candidate, from the first EM's assignment
  std::vector<int32_t> ptr(n_split + 1, 0), idx;
  for (int32_t i = 0; i < n_split; i++) {
    const TgmmGaussian& g = gm_host[cand[i]];
    idx.insert(idx.end(), g.supervoxelIdx, g.supervoxelIdx + g.supervoxelNum);
    ptr[i + 1] = (int32_t)idx.size();
  }
  if (idx.empty()) idx.push_back(0);
  TgmmGaussian* gd = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&gd, sizeof(TgmmGaussian) * (size_t)n_total, st);
  if (e != cudaSuccess) return report_error(TGMM_ERR_OOM, "tgmm_split_round: scratch", e);
  auto done = [&](int rc) {
    cudaFreeAsync(gd, st);
    cudaStreamSynchronize(st);
    return rc;
  };
  // 1. before the split
  if (n_split > 0) {
    e = cudaMemcpyAsync(gd, gm_host, sizeof(TgmmGaussian) * (size_t)n_gauss, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return done(report_error(TGMM_ERR_CUDA, "tgmm_split_round: upload", e));
    const int rc = tgmm_local_likelihood(frame, ind_dev, gd, n_gauss, ptr.data(), idx.data(), n_split, ll_before, stream);
    if (rc != TGMM_OK) return done(rc);
  }
  // 2. the split mixture
  float s[3];
  const bool reg_zero = params->reg_scale[0] == 0.0f && params->reg_scale[1] == 0.0f && params->reg_scale[2] == 0.0f;
  for (int d = 0; d < 3; d++) s[d] = reg_zero ? params->scale[d] : params->reg_scale[d];
  for (int32_t k = 0; k < n_gauss; k++)
    if (!seen[k]) gm_host[k].fixed = 1;
  for (int32_t i = 0; i < n_split; i++) {
    TgmmGaussian a, b;
    split_proposal(gm_host[cand[i]], s, &a, &b);
    gm_host[cand[i]] = a;
    gm_host[n_gauss + i] = b;
  }
  // 3. the EM on it
  TgmmFrame f = *frame;
  f.n_gauss = n_total;
  TgmmEmStats local;
  int rc = tgmm_em_run(plan, &f, gm_host, rnk_dev, ind_out_dev, nullptr, params, stats ? stats : &local, stream);
  if (rc != TGMM_OK && rc != TGMM_ERR_NAN_INPUT) return done(rc);
  // 4. after it
  if (n_split > 0) {
    e = cudaMemcpyAsync(gd, gm_host, sizeof(TgmmGaussian) * (size_t)n_total, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return done(report_error(TGMM_ERR_CUDA, "tgmm_split_round: upload", e));
    const int rc2 = tgmm_local_likelihood(frame, ind_out_dev, gd, n_total, ptr.data(), idx.data(), n_split, ll_after, stream);
    if (rc2 != TGMM_OK) return done(rc2);
  }
  return done(rc);
}
