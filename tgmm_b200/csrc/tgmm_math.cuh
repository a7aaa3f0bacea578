// tgmm_math.cuh -- per-Gaussian FP64 algebra shared by the device kernels and the
// host-side frame initialisation: digamma, 3x3 symmetric determinant / inverse,
// closed-form symmetric eigen-decomposition, precision-matrix regularisation and the
// Dirichlet / Normal-Wishart update.  Symmetric 3x3 matrices are stored as the upper
// triangle, row major: 00,01,02,11,12,22 (GaussianMixtureModelCUDA::W_k layout).
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define TG_HD __host__ __device__ __forceinline__
#else
#define TG_HD static inline
#endif

// Device code scales by one reciprocal per shared denominator instead of dividing each
// term (about 1 ulp apart, shorter FP64 chains); host code keeps the plain divisions with
// which the synthetic generator's seeded workloads were pinned.
#if defined(__CUDA_ARCH__)
#define TG_RCP 1
#else
#define TG_RCP 0
#endif

namespace tgmm {

constexpr double kLn2 = 0.69314718055994530942;
constexpr double kPi = 3.14159265358979323846;
constexpr double kLnTwoPi = 1.83787706640934548356;  // ln(2*pi)

TG_HD bool is_dead_prior(double m_o0) { return m_o0 < -1e31; }

// psi(x) for x > 0: Bernardo's AS 103 as modified by Minka -- a small-argument
// expansion below 1e-6, upward recurrence psi(x) = psi(x+1) - 1/x to x >= 12, then
// the asymptotic series ln x - 1/(2x) - sum B_2n / (2n x^2n) with five terms.
// (Reference: UtilsCUDA/GMEMupdateCUDA.cu:494-525.)  The recurrence's terms are summed
// as one fraction num/den (1/x + num/den = (num x + den) / (den x)), so the chain holds
// one division instead of one per step; den stays below 12^12.
TG_HD double digamma_pos(double x) {
  if (x <= 1e-6) return -0.57721566490153286 - 1.0 / x + 1.6449340668482264365 * x;
  double num = 0.0, den = 1.0;
  while (x < 12.0) {
    num = num * x + den;
    den *= x;
    x += 1.0;
  }
  const double inv = 1.0 / x;
  const double t = inv * inv;
  double acc = log(x) - 0.5 * inv - num / den;
  acc -= t * (1.0 / 12 - t * (1.0 / 120 - t * (1.0 / 252 - t * (1.0 / 240 - t * (1.0 / 132)))));
  return acc;
}

// psi over the reals: -1e300 at the poles, reflection for negative arguments.
TG_HD double digamma(double x) {
  if (x <= 0 && floor(x) == x) return -1e300;
  if (x < 0) return digamma_pos(1.0 - x) + kPi / tan(-kPi * x);
  return digamma_pos(x);
}

TG_HD double det3(const double* w) {
  return w[0] * (w[3] * w[5] - w[4] * w[4]) - w[1] * (w[1] * w[5] - w[2] * w[4]) +
         w[2] * (w[1] * w[4] - w[2] * w[3]);
}

// Adjugate inverse; |det| < 1e-16 is treated as singular and yields 1e300 entries
// (GMEMupdateCUDA.cu:170-192).  The cofactors are scaled by one reciprocal of det.
TG_HD void inv3(const double* w, double* o) {
  const double det = det3(w);
  if (fabs(det) < 1e-16) {
    for (int i = 0; i < 6; i++) o[i] = 1e300;
    return;
  }
  const double r = 1.0 / det;
  const double c00 = w[3] * w[5] - w[4] * w[4];
  const double c01 = w[4] * w[2] - w[1] * w[5];
  const double c02 = w[1] * w[4] - w[3] * w[2];
  const double c11 = w[0] * w[5] - w[2] * w[2];
  const double c12 = w[1] * w[2] - w[0] * w[4];
  const double c22 = w[0] * w[3] - w[1] * w[1];
  o[0] = c00 * r;
  o[1] = c01 * r;
  o[2] = c02 * r;
  o[3] = c11 * r;
  o[4] = c12 * r;
  o[5] = c22 * r;
}

TG_HD bool unit3(double* a) {
  const double n = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  if (n > 1e-12) {
    if (TG_RCP) {
      const double r = 1.0 / n;
      a[0] *= r;
      a[1] *= r;
      a[2] *= r;
    } else {
      a[0] /= n;
      a[1] /= n;
      a[2] /= n;
    }
    return true;
  }
  return false;
}

// Closed-form eigen-decomposition of a symmetric 3x3 matrix: eigenvalues from the
// trigonometric solution of the characteristic cubic (near-singular matrices, |det| <
// 1e-24, take one zero eigenvalue and solve the remaining quadratic); eigenvectors from
// the cross product of two rows of (W - d I), rows 0x1 first, rows 0x2 as fallback.
// Degenerate eigenvector sets are completed with the same conventions as the
// reference (GMEMupdateCUDA.cu:198-422), including its sign pattern, so that the
// regularised matrix is the same.  Eigenvalue order: d0 largest, d1 smallest, d2 middle.
TG_HD void eig3(const double* w, double* d, double* v) {
  if (fabs(det3(w)) < 1e-24) {
    const double b = -w[0] - w[3] - w[5];
    const double c = w[0] * w[3] + w[0] * w[5] + w[3] * w[5] - w[1] * w[1] - w[2] * w[2] - w[4] * w[4];
    double disc = b * b - 4.0 * c;
    disc = disc < 0 ? 0.0 : sqrt(disc);
    d[0] = 0.0;
    d[1] = 0.5 * (-b + disc);
    d[2] = 0.5 * (-b - disc);
  } else {
    const double mean = (w[0] + w[3] + w[5]) / 3.0;
    const double a0 = w[0] - mean, a3 = w[3] - mean, a5 = w[5] - mean;
    const double q = 0.5 * (a0 * (a3 * a5 - w[4] * w[4]) - w[1] * (w[1] * a5 - w[2] * w[4]) +
                            w[2] * (w[1] * w[4] - w[2] * a3));
    const double p = (2.0 * (w[1] * w[1] + w[2] * w[2] + w[4] * w[4]) + a0 * a0 + a3 * a3 + a5 * a5) / 6.0;
    const double r = sqrt(p);
    const double ratio = TG_RCP ? q / (p * r) : q / pow(p, 1.5);
    double phi;
    if (ratio <= -1)
      phi = 3.14159265358979311600 / 3.0;
    else if (ratio >= 1)
      phi = 0;
    else
      phi = acos(ratio) / 3.0;
    double s, c;
    if (TG_RCP) {
      sincos(phi, &s, &c);
    } else {
      c = cos(phi);
      s = sin(phi);
    }
    const double root3 = 1.73205080756887719318;
    d[0] = mean + 2.0 * r * c;
    d[1] = mean - r * (c + root3 * s);
    d[2] = mean - r * (c - root3 * s);
  }
  int missing = 0;
  for (int i = 0; i < 3; i++) {
    const double di = d[i];
    double* e = v + 3 * i;
    e[0] = w[1] * w[4] - w[2] * (w[3] - di);
    e[1] = w[2] * w[1] - w[4] * (w[0] - di);
    e[2] = (w[0] - di) * (w[3] - di) - w[1] * w[1];
    if (!unit3(e)) {
      e[0] = w[1] * (w[5] - di) - w[2] * w[4];
      e[1] = w[2] * w[2] - (w[5] - di) * (w[0] - di);
      e[2] = (w[0] - di) * w[4] - w[1] * w[2];
      if (!unit3(e)) missing |= 1 << i;
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
        v[3] = 1.0; v[4] = 0.0; v[5] = 0.0;
      } else {
        v[3] = -v[7] / n; v[4] = v[6] / n; v[5] = 0.0;
      }
      v[0] = v[4] * v[8] - v[5] * v[7];
      v[1] = v[5] * v[6] - v[3] * v[8];
      v[2] = v[3] * v[7] - v[4] * v[6];
      break;
    case 6:
      n = sqrt(v[1] * v[1] + v[0] * v[0]);
      if (n < 1e-12) {
        v[6] = 1.0; v[7] = 0.0; v[8] = 0.0;
      } else {
        v[6] = -v[1] / n; v[7] = v[0] / n; v[8] = 0.0;
      }
      v[3] = v[1] * v[8] - v[2] * v[7];
      v[4] = v[2] * v[6] - v[0] * v[8];
      v[5] = v[0] * v[7] - v[1] * v[6];
      break;
    case 5:
      n = sqrt(v[4] * v[4] + v[5] * v[5]);
      if (n < 1e-12) {
        v[0] = 1.0; v[1] = 0.0; v[2] = 0.0;
      } else {
        v[0] = -v[4] / n; v[1] = v[5] / n; v[2] = 0.0;
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
  const double handed = v[0] * (v[4] * v[8] - v[5] * v[7]) - v[1] * (v[3] * v[8] - v[5] * v[6]) +
                        v[2] * (v[3] * v[7] - v[4] * v[6]);
  if (handed < 0) {
    v[0] = -v[0];
    v[1] = -v[1];
    v[2] = -v[2];
  }
}

struct RegConst {
  float scale[3];
  int w4dof;
  double lambda_min, lambda_max, max_exc;
};

// Precision-matrix regularisation (GMEMregularizeWkKernel, GMEMupdateCUDA.cu:1693-1809):
// undo the anisotropy (divide by s_i s_j, float products), optionally force the 4-DOF
// shape (W02 = W12 = 0), clamp eigenvalues to [lambda_min/nu, lambda_max/nu], cap the
// pairwise eigenvalue ratio at max_exc in the order (0,1), (0,2), (1,2), rebuild and
// re-apply the anisotropy.
TG_HD void regularize_W(double* Wk, double nu, const RegConst& rc) {
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
  const double inu = 1.0 / nu;
  const double hi = TG_RCP ? rc.lambda_max * inu : rc.lambda_max / nu;
  const double lo = TG_RCP ? rc.lambda_min * inu : rc.lambda_min / nu;
  double W[6];
  for (int e = 0; e < 6; e++) {
    const double s2 = (double)(rc.scale[ia[e]] * rc.scale[ib[e]]);
    W[e] = TG_RCP ? Wk[e] * (1.0 / s2) : Wk[e] / s2;
  }
  if (rc.w4dof) {
    W[2] = 0.0;
    W[4] = 0.0;
  }
  double d[3], v[9];
  eig3(W, d, v);
  for (int i = 0; i < 3; i++) d[i] = d[i] > hi ? hi : d[i];
  for (int i = 0; i < 3; i++) d[i] = d[i] < lo ? lo : d[i];
  const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
  for (int q = 0; q < 3; q++) {
    const double r = d[pa[q]] / d[pb[q]];
    if (r > rc.max_exc)
      d[pa[q]] = rc.max_exc * d[pb[q]];
    else if (1. / r > rc.max_exc)
      d[pb[q]] = rc.max_exc * d[pa[q]];
  }
  W[0] = d[0] * v[0] * v[0] + d[1] * v[3] * v[3] + d[2] * v[6] * v[6];
  W[3] = d[0] * v[1] * v[1] + d[1] * v[4] * v[4] + d[2] * v[7] * v[7];
  W[5] = d[0] * v[2] * v[2] + d[1] * v[5] * v[5] + d[2] * v[8] * v[8];
  W[1] = d[0] * v[0] * v[1] + d[1] * v[3] * v[4] + d[2] * v[6] * v[7];
  if (!rc.w4dof) {
    W[2] = d[0] * v[0] * v[2] + d[1] * v[3] * v[5] + d[2] * v[6] * v[8];
    W[4] = d[0] * v[1] * v[2] + d[1] * v[4] * v[5] + d[2] * v[7] * v[8];
  }
  for (int e = 0; e < 6; e++) Wk[e] = W[e] * (double)(rc.scale[ia[e]] * rc.scale[ib[e]]);
}

// E[ln |Lambda|] = 3 ln 2 + ln det W + sum_{i=0..2} psi((nu + 1 - i)/2)
// (GMEMupdateCUDA.cu:553-576; the index starts at 0 as in the reference).
TG_HD double expected_log_det(const double* W, double nu) {
  double out = 3.0 * kLn2 + log(det3(W));
  for (int i = 0; i < 3; i++) out += digamma(0.5 * (nu + 1.0 - i));
  return out;
}

}  // namespace tgmm
