// ref_split_harness.cpp -- TEST INFRASTRUCTURE ONLY.  A C entry point over the reference's own
// split proposal: GaussianMixtureModel::splitGaussian(GM, id) (GaussianMixtureModel.cpp:514-557,
// the principal-axis split) followed by updatePriorsAfterSplitProposal (:912-922) on both
// halves, as mainTrackingGaussianMixtureModel.cpp:1255-1261 applies them, compiled from the
// reference sources by oracle/build_ref.sh into oracle/_ref/libtgmm_ref_gmm.so (host code).
// The 288-byte records are moved in and out of the class as the reference's
// copyFromGMEM_CUDA / copy2GMEM_CUDA do (variationalInference.cpp:951-1016).
#include "GaussianMixtureModel.h"

namespace {

struct Rec {
  double beta_k, nu_k, alpha_k, m_k[3], W_k[6], eLD, eLR, splitScore, beta_o, nu_o, alpha_o, m_o[3], W_o[6];
  unsigned char fixed;
  int supervoxelIdx[16];
  int supervoxelNum;
};
static_assert(sizeof(Rec) == 288, "the 288-byte GaussianMixtureModelCUDA layout");

void from_rec(const Rec& r, GaussianMixtureModel* g) {
  g->beta_k = r.beta_k;
  g->nu_k = r.nu_k;
  g->alpha_k = r.alpha_k;
  int e = 0;
  for (int i = 0; i < 3; i++) {
    g->m_k(i) = r.m_k[i];
    g->m_o(i) = r.m_o[i];
    for (int j = i; j < 3; j++, e++) {
      g->W_k(i, j) = g->W_k(j, i) = r.W_k[e];
      g->W_o(i, j) = g->W_o(j, i) = r.W_o[e];
    }
  }
  g->beta_o = r.beta_o;
  g->nu_o = r.nu_o;
  g->alpha_o = r.alpha_o;
  g->fixed = r.fixed != 0;
  g->splitScore = r.splitScore;
  g->updateNk();
  g->supervoxelIdx.assign(r.supervoxelIdx, r.supervoxelIdx + r.supervoxelNum);
}

void to_rec(const GaussianMixtureModel* g, Rec* r) {
  r->beta_k = g->beta_k;
  r->nu_k = g->nu_k;
  r->alpha_k = g->alpha_k;
  int e = 0;
  for (int i = 0; i < 3; i++) {
    r->m_k[i] = g->m_k(i);
    r->m_o[i] = g->m_o(i);
    for (int j = i; j < 3; j++, e++) {
      r->W_k[e] = g->W_k(i, j);
      r->W_o[e] = g->W_o(i, j);
    }
  }
  r->beta_o = g->beta_o;
  r->nu_o = g->nu_o;
  r->alpha_o = g->alpha_o;
  r->fixed = g->fixed ? 1 : 0;
  r->splitScore = g->splitScore;
  r->supervoxelNum = (int)g->supervoxelIdx.size();
  for (int i = 0; i < r->supervoxelNum && i < 16; i++) r->supervoxelIdx[i] = g->supervoxelIdx[i];
}

}  // namespace

// in: one record; out_a: the split Gaussian itself, out_b: the new one (both with the
// priors of the split proposal).
extern "C" int ref_split_gaussian(const void* in, const float* scale, void* out_a, void* out_b) {
  GaussianMixtureModel::setScale(scale);
  GaussianMixtureModel* a = new GaussianMixtureModel(0);
  GaussianMixtureModel* b = new GaussianMixtureModel(1);
  from_rec(*static_cast<const Rec*>(in), a);
  a->splitGaussian(b, 1);
  b->updatePriorsAfterSplitProposal();
  a->updatePriorsAfterSplitProposal();
  *static_cast<Rec*>(out_a) = *static_cast<const Rec*>(in);
  *static_cast<Rec*>(out_b) = *static_cast<const Rec*>(in);
  to_rec(a, static_cast<Rec*>(out_a));
  to_rec(b, static_cast<Rec*>(out_b));
  delete a;
  delete b;
  return 0;
}
