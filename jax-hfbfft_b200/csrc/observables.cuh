// Scalar part of the nuclear observables (calculate_complete_observables,
// output.py:177-340): everything that follows from the per-isospin grid
// sums of the density, in FP64.  Host- and device-callable; the sums come
// from obs_moments_kernel (observables.cu).
#pragma once
#include <math.h>
#include "../../include/hfb.h"

namespace hfb {

// Per-isospin grid sums (without the volume element) of one density:
//   [0] sum rho, [1..3] sum x_d rho, [4..6] sum of the current components,
//   [7..12] sum (x - cm)_i (x - cm)_j rho for ij = xx, yy, zz, xy, xz, yz
//   about the isospin's own centre of mass.
constexpr int kObsSums = 13;

// Eigenvalues of a real symmetric 3x3 matrix, ascending: cyclic Jacobi
// rotations (Jacobi 1846; the rotation of Numerical Recipes 11.1), at most
// 50 sweeps, stopping once the off-diagonal part is below 1e-32 of the
// matrix's squared Frobenius norm.
__host__ __device__ inline void sym3_eigvals(const double m[3][3], double ev[3]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = 0.5 * (m[i][j] + m[j][i]);
  const int pp[3] = {0, 0, 1}, qq[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 50; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off == 0.0 || off <= 1e-32 * (dia + 2.0 * off)) break;
    for (int r = 0; r < 3; ++r) {
      const int p = pp[r], q = qq[r];
      if (a[p][q] == 0.0) continue;
      const double th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
      const double t = fabs(th) > 1e150 ? 0.5 / th : (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
      for (int k = 0; k < 3; ++k) {   // columns p, q
        const double akp = a[k][p], akq = a[k][q];
        a[k][p] = c * akp - s * akq;
        a[k][q] = s * akp + c * akq;
      }
      for (int k = 0; k < 3; ++k) {   // rows p, q
        const double apk = a[p][k], aqk = a[q][k];
        a[p][k] = c * apk - s * aqk;
        a[q][k] = s * apk + c * aqk;
      }
    }
  }
  double d[3] = {a[0][0], a[1][1], a[2][2]};
  for (int i = 0; i < 2; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (d[j] < d[i]) {
        const double x = d[i];
        d[i] = d[j];
        d[j] = x;
      }
  ev[0] = d[0];
  ev[1] = d[1];
  ev[2] = d[2];
}

// out[HFB_NOBS] from the sums of both isospins (laid out as in hfb.h).
__host__ __device__ inline void obs_finalize(const double* sums, double wxyz, double nneut, double nprot,
                                             double* out) {
  const double kPi_ = 3.141592653589793238462643383279502884;
  const double c20 = sqrt(5.0 / (16.0 * kPi_)), c22 = sqrt(5.0 / (96.0 * kPi_));
  double pnr[2], rms[2], x2m[3][2], cm[3][2], q[3][3][2];
  for (int iq = 0; iq < 2; ++iq) {
    const double* s = sums + iq * kObsSums;
    pnr[iq] = s[0] * wxyz;
    for (int d = 0; d < 3; ++d) {
      cm[d][iq] = s[1 + d] * wxyz / pnr[iq];
      out[HFB_OBS_PCM + 2 * d + iq] = s[4 + d] * wxyz;
      x2m[d][iq] = s[7 + d] * wxyz / pnr[iq];
    }
    const double r2 = s[7] + s[8] + s[9];
    rms[iq] = sqrt(r2 * wxyz / pnr[iq]);
    for (int d = 0; d < 3; ++d) q[d][d][iq] = (3.0 * s[7 + d] - r2) * wxyz;
    q[0][1][iq] = q[1][0][iq] = 3.0 * s[10] * wxyz;
    q[0][2][iq] = q[2][0][iq] = 3.0 * s[11] * wxyz;
    q[1][2][iq] = q[2][1][iq] = 3.0 * s[12] * wxyz;
    double m[3][3], ev[3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[i][j] = q[i][j][iq];
    sym3_eigvals(m, ev);
    out[HFB_OBS_PNR + iq] = pnr[iq];
    out[HFB_OBS_RMS + iq] = rms[iq];
    out[HFB_OBS_Q20 + iq] = c20 * ev[2];
    out[HFB_OBS_Q22 + iq] = c22 * (ev[1] - ev[0]);
    for (int d = 0; d < 3; ++d) {
      out[HFB_OBS_CM + 2 * d + iq] = cm[d][iq];
      out[HFB_OBS_X2M + 2 * d + iq] = x2m[d][iq];
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[HFB_OBS_QMAT + 6 * i + 2 * j + iq] = q[i][j][iq];
  }
  const double pt = pnr[0] + pnr[1];
  out[HFB_OBS_PNRTOT] = pt;
  for (int d = 0; d < 3; ++d) {
    out[HFB_OBS_CMTOT + d] = (pnr[0] * cm[d][0] + pnr[1] * cm[d][1]) / pt;
    out[HFB_OBS_X2MTOT + d] = (pnr[0] * x2m[d][0] + pnr[1] * x2m[d][1]) / pt;
    out[HFB_OBS_DIPOLE + d] = cm[d][0] - cm[d][1];   // sum x (rho_n / N - rho_p / Z) dV
  }
  const double rmstot = sqrt((pnr[0] * rms[0] * rms[0] + pnr[1] * rms[1] * rms[1]) / pt);
  out[HFB_OBS_RMSTOT] = rmstot;
  double m[3][3], ev[3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m[i][j] = q[i][j][0] + q[i][j][1];
  sym3_eigvals(m, ev);
  const double q20t = c20 * ev[2], q22t = c22 * (ev[1] - ev[0]);
  out[HFB_OBS_Q20TOT] = q20t;
  out[HFB_OBS_Q22TOT] = q22t;
  out[HFB_OBS_Q20T1] = -out[HFB_OBS_Q20] / nneut + out[HFB_OBS_Q20 + 1] / nprot;
  const double scale = 4.0 * kPi_ / (5.0 * rmstot * rmstot * pt);
  const double b20 = q20t * scale, b22 = q22t * scale;
  out[HFB_OBS_BETA20] = b20;
  out[HFB_OBS_BETA22] = b22;
  out[HFB_OBS_BETA] = sqrt(b20 * b20 + 2.0 * b22 * b22);
  double g = fabs(atan2(sqrt(2.0) * b22, b20)) * 180.0 / kPi_;
  if (g > 120.0) g -= 120.0;
  if (g <= 120.0 && g > 60.0) g = 120.0 - g;
  out[HFB_OBS_GAMMA] = g;
}

}  // namespace hfb
