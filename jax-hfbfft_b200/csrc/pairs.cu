// BCS pairing on the device (pair / _pairdn / _bcs_occupation / _soft_cutoff
// of pairs.py:25-220).  One warp per isospin; the particle-number sum over
// states is a fixed-order warp reduction, so results are deterministic.
//
// The Fermi level is the root of  sum_k w_k clip(v2_k, 1e-10, 1-1e-10) - N
// on [-100, 100] found with Brent's method (Brent 1973, "Algorithms for
// Minimization without Derivatives", ch. 4: bisection safeguarded inverse
// quadratic / secant steps), stopping when the bracket is below
// xtol + rtol |x| with xtol = 1e-14 and rtol = 4 eps, the tolerances the
// reference passes to scipy.optimize.brentq (pairs.py:59).
#include <float.h>
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {

__device__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sum over the isospin's states of wstates * clip(v2) (pairs.py:25-45)
__device__ double bcs_number(double ef, int n, const double* e, const double* d, const double* ws) {
  double s = 0.0;
  for (int k = threadIdx.x % 32; k < n; k += 32) {
    const double ed = e[k] - ef;
    const double eq = fmax(sqrt(ed * ed + d[k] * d[k]), 1.0e-20);
    double v2 = 0.5 * (1.0 - ed / eq);
    v2 = fmin(fmax(v2, 1.0e-10), 1.0 - 1.0e-10);
    s += v2 * ws[k];
  }
  return warp_sum(s);
}

__global__ void pair_kernel(hfb_pair_args a, int* status) {
  const int iq = threadIdx.x / 32;
  if (iq > 1) return;
  const int n = a.npsi[iq], o = iq == 0 ? 0 : a.npsi[0];
  const double npart = iq == 0 ? (double)a.nneut : (double)a.nprot;
  const double* e = a.sp_energy + o;
  double* dl = a.deltaf + o;
  const int lane = threadIdx.x % 32;
  // _pairgap (pairs.py:133-141): constant gap for the first iterations
  if (a.use_const_gap)
    for (int k = lane; k < n; k += 32) dl[k] = a.const_gap;
  __syncwarp();
  const double* ws = a.wstates + o;
  auto f = [&](double x) { return bcs_number(x, n, e, dl, ws) - npart; };
  // ---- Brent's method
  double xa = -100.0, xb = 100.0;
  double fa = f(xa), fb = f(xb);
  double ef = 0.0;
  int err = 0;
  if (fa * fb > 0.0) {
    err = HFB_ERR_NOT_BRACKETED;
  } else if (fa == 0.0) {
    ef = xa;
  } else if (fb == 0.0) {
    ef = xb;
  } else {
    const double xtol = 1e-14, rtol = 4.0 * DBL_EPSILON;
    double xc = xa, fc = fa, dstep = xb - xa, estep = dstep;
    int it = 0;
    for (; it < 100; ++it) {
      if (fb * fc > 0.0) { xc = xa; fc = fa; dstep = estep = xb - xa; }
      if (fabs(fc) < fabs(fb)) {  // keep b the best estimate
        xa = xb; xb = xc; xc = xa;
        fa = fb; fb = fc; fc = fa;
      }
      const double tol = 0.5 * (xtol + rtol * fabs(xb));
      const double mid = 0.5 * (xc - xb);
      if (fabs(mid) <= tol || fb == 0.0) break;
      if (fabs(estep) >= tol && fabs(fa) > fabs(fb)) {
        const double s = fb / fa;
        double p, q;
        if (xa == xc) {           // secant
          p = 2.0 * mid * s;
          q = 1.0 - s;
        } else {                  // inverse quadratic interpolation
          const double qq = fa / fc, r = fb / fc;
          p = s * (2.0 * mid * qq * (qq - r) - (xb - xa) * (r - 1.0));
          q = (qq - 1.0) * (r - 1.0) * (s - 1.0);
        }
        if (p > 0.0) q = -q;
        else p = -p;
        if (2.0 * p < fmin(3.0 * mid * q - fabs(tol * q), fabs(estep * q))) {
          estep = dstep;
          dstep = p / q;
        } else {
          dstep = mid;
          estep = mid;
        }
      } else {
        dstep = mid;
        estep = mid;
      }
      xa = xb;
      fa = fb;
      xb += fabs(dstep) > tol ? dstep : (mid > 0.0 ? tol : -tol);
      fb = f(xb);
    }
    if (it >= 100) err = HFB_ERR_NO_CONVERGENCE;
    ef = xb;
  }
  if (err) {
    if (lane == 0) latch_error(status, err);
    return;
  }
  // soft cutoffs (pairs.py:88-99)
  double* pw = a.pairwg + o;
  double* wst = a.wstates + o;
  const double pc = a.pair_cutoff[iq], sc = a.state_cutoff[iq];
  for (int k = lane; k < n; k += 32) {
    if (pc > 0.0) pw[k] = 1.0 / (1.0 + exp((e[k] - (ef + pc)) / (a.softcut_range * pc)));
    if (sc > 0.0) wst[k] = 1.0 / (1.0 + exp((e[k] - (ef + sc)) / (a.softcut_range * sc)));
  }
  __syncwarp();
  // occupations and sums (pairs.py:102-129)
  double sumuv = 0, sumduv = 0, sumv2 = 0, sumdv2 = 0;
  for (int k = lane; k < n; k += 32) {
    const double ed = e[k] - ef;
    const double eq = fmax(sqrt(ed * ed + dl[k] * dl[k]), 1.0e-20);
    const double v2 = 0.5 * (1.0 - ed / eq);
    const double uv = sqrt(fmax(v2 - v2 * v2, 1.0e-6));
    const double wo = fmin(fmax(v2, 1e-10), 1.0 - 1e-10);
    a.wocc[o + k] = wo;
    a.wguv[o + k] = uv;
    const double vol = 0.5 * uv * wst[k];
    sumuv += vol;
    sumduv += vol * dl[k];
    sumv2 += wo * wst[k];
    sumdv2 += dl[k] * wo * wst[k];
  }
  sumuv = warp_sum(sumuv);
  sumduv = warp_sum(sumduv);
  sumv2 = warp_sum(sumv2);
  sumdv2 = warp_sum(sumdv2);
  if (lane == 0) {
    const double su = fmax(sumuv, 1.0e-20), sv = fmax(sumv2, 1.0e-20);
    a.out[0 * 2 + iq] = ef;
    a.out[1 * 2 + iq] = sumduv;
    a.out[2 * 2 + iq] = sumduv / su;
    a.out[3 * 2 + iq] = sumdv2 / sv;
    a.out[4 * 2 + iq] = sumduv / (su * su);
  }
}

}  // namespace hfb

extern "C" int hfb_pair(hfb_ctx_t ctx, const hfb_pair_args* a, void* stream) {
  if (!ctx || !a || !a->sp_energy || !a->deltaf || !a->wocc || !a->wguv || !a->pairwg || !a->wstates || !a->out)
    return HFB_ERR_ARG;
  hfb::pair_kernel<<<1, 64, 0, hfb::as_stream(stream)>>>(*a, ctx->dev_status);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
