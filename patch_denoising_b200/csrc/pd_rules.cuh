// Decision rules shared by the eigensolvers.
#pragma once

namespace pd {

// MP-PCA (space_time/lowrank.py:42-63) and hybrid (lowrank.py:104-119) on the
// top ne (<= 10) eigenvalues lam[0..ne) of the scaled Gram, ascending; the
// true covariance eigenvalues are lam * tscale / (M - 1), zero-padded to 10 as
// the reference's subset. Returns the rank and the noise variance estimate.
__device__ inline void mp_hybrid_rule(bool mppca, double threshold_scale, double varest, const float* lam, int ne,
                                      double tscale, double M, double pt, int* rank_out, double* var_out) {
  double l[10];
  for (int i = 0; i < 10; ++i) l[i] = 0.0;
  for (int i = 0; i < ne; ++i) l[10 - ne + i] = (double)lam[i] * tscale / (M - 1.0);
  int k = 0;
  double var;
  if (mppca) {
    double s = 0.0;
    for (int i = 0; i < 10; ++i) s += l[i];
    double crit = (s / 10.0) * (4.0 * sqrt((10.0 - 0 + 1.0) / M));
    while (k < 10 && crit < l[9 - k] - l[0]) {
      ++k;
      if (k < 10) {
        double t = 0.0;
        for (int i = 0; i < 10 - k; ++i) t += l[i];
        crit = (t / (10 - k)) * (4.0 * sqrt((pt - k + 1.0) / M));
      } else {
        crit = nan("");
      }
    }
    if (k < 10) {
      double t = 0.0;
      for (int i = 0; i < 10 - k; ++i) t += l[i];
      var = t / (10 - k);
    } else {
      var = nan("");
    }
    const double cut = var * threshold_scale * threshold_scale;
    int r = 0;
    for (int i = 0; i < 10; ++i) r += (l[i] > cut) ? 1 : 0;
    k = r;
  } else {
    double s = 0.0;
    for (int i = 0; i < 10; ++i) s += l[i];
    var = s / 10.0;
    while (var > varest && k < 10 - 2) {
      ++k;
      double t = 0.0;
      for (int i = 0; i < 10 - k; ++i) t += l[i];
      var = t / (10 - k);
    }
  }
  *rank_out = k;
  *var_out = var;
}

}  // namespace pd
