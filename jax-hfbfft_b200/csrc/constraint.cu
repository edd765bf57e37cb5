// Quadrupole / principal-axis constraints (constraint.py:47-342 of the
// reference, wired into the iteration by hfb.constraint): the masked
// constraint fields, their expectation values and variances in the
// densities, the constraint potential upot -= sum lambda_i Q_i, and the
// state correction psi_s *= exp(wstates_s wocc_s (-sum qcorr_i Q_i)).
// The fields act on both isospins alike and are stored once, [nc][n^3].
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {

namespace {

struct ConCoef {
  double c[HFB_CON_MAX];
};

__global__ void con_fields_kernel(int n, int kinds, double dx, double dy, double dz, double norm, double damprad,
                                  double dampgamma, double* fields) {
  const size_t n3 = (size_t)n * n * n;
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= n3) return;
  const int ix = (int)(g / ((size_t)n * n)), iy = (int)((g / n) % n), iz = (int)(g % n);
  const double h = (n - 1) / 2.0;
  const double x = (ix - h) * dx, y = (iy - h) * dy, z = (iz - h) * dz;
  const double r = sqrt(x * x + y * y + z * z);
  const double mask = 1.0 / (1.0 + exp((r - damprad) / dampgamma));
  const double pi = 3.141592653589793238462643383279502884;
  int k = 0;
  if (kinds & HFB_CON_Q20) fields[(size_t)k++ * n3 + g] = sqrt(pi / 5.0) / norm * (2.0 * z * z - x * x - y * y) * mask;
  if (kinds & HFB_CON_Q22) fields[(size_t)k++ * n3 + g] = sqrt(1.2 * pi) / norm * (x * x - y * y) * mask;
  if (kinds & HFB_CON_PRINCIPAL) {
    const double f = 0.5 * sqrt(pi / 5.0) / norm * mask;
    fields[(size_t)k++ * n3 + g] = f * x * y;
    fields[(size_t)k++ * n3 + g] = f * x * z;
    fields[(size_t)k++ * n3 + g] = f * y * z;
    fields[(size_t)k++ * n3 + g] = f * x;
    fields[(size_t)k++ * n3 + g] = f * y;
    fields[(size_t)k++ * n3 + g] = f * z;
  }
}

// block c < nc: sum Q_c rho and sum Q_c^2 rho; block nc: sum rho
__global__ void con_moments_kernel(size_t n3, int nc, const double* __restrict__ fields,
                                   const double* __restrict__ rho, double* part) {
  __shared__ double red[2][32];
  const int c = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (size_t g = threadIdx.x; g < n3; g += blockDim.x) {
    const double r = rho[g] + rho[n3 + g];
    if (c < nc) {
      const double f = fields[(size_t)c * n3 + g];
      a += f * r;
      b += f * f * r;
    } else {
      a += r;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = a;
    red[1][threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, t = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
      s += red[0][w];
      t += red[1][w];
    }
    part[2 * c] = s;
    part[2 * c + 1] = t;
  }
}

// out[c] = <Q_c>, out[nc + c] = |<Q_c^2> - <Q_c>^2 / N|, out[2 nc] = N
__global__ void con_moments_final_kernel(int nc, const double* part, double wxyz, double* out) {
  const double npart = wxyz * part[2 * nc];
  for (int c = 0; c < nc; ++c) {
    const double ex = wxyz * part[2 * c], m2 = wxyz * part[2 * c + 1];
    out[c] = ex;
    out[nc + c] = fabs(m2 - ex * ex / npart);
  }
  out[2 * nc] = npart;
}

template <class R>
__global__ void con_potential_kernel(size_t n3, int nc, const double* __restrict__ fields, ConCoef lam, double* upot,
                                     R* pot) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= n3) return;
  double v = 0.0;
  for (int c = 0; c < nc; ++c) v += lam.c[c] * fields[(size_t)c * n3 + g];
  for (int iq = 0; iq < 2; ++iq) {
    if (upot) upot[(size_t)iq * n3 + g] -= v;
    if (pot) pot[(size_t)iq * 12 * n3 + g] -= (R)v;   // field 0 of the packed hpsi potentials
  }
}

template <class R>
__global__ void con_correct_kernel(size_t n3, int nc, const double* __restrict__ fields, ConCoef q,
                                   const double* __restrict__ wocc, const double* __restrict__ wstates,
                                   cplx<R>* psi) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (g >= n3) return;
  double corr = 0.0;
  for (int c = 0; c < nc; ++c) corr -= q.c[c] * fields[(size_t)c * n3 + g];
  const R e = (R)exp(wstates[s] * wocc[s] * corr);
  cplx<R>* p = psi + (size_t)s * 2 * n3;
  p[g] = e * p[g];
  p[n3 + g] = e * p[n3 + g];
}

}  // namespace

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_constraint_fields(hfb_ctx_t ctx, int kinds, double mass_number, double r0rms, double damprad,
                                     double dampgamma, double* fields, void* stream) {
  if (!ctx || !fields || kinds <= 0 || kinds > 7 || !(mass_number > 0.0) || !(dampgamma > 0.0)) return HFB_ERR_ARG;
  const int n = ctx->n;
  const size_t n3 = (size_t)n * n * n;
  const double norm = r0rms * r0rms * pow(mass_number, 5.0 / 3.0);
  con_fields_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, as_stream(stream)>>>(
      n, kinds, ctx->d[0], ctx->d[1], ctx->d[2], norm, damprad, dampgamma, fields);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_constraint_moments(hfb_ctx_t ctx, int nc, const double* fields, const double* rho, double* out,
                                      void* stream) {
  if (!ctx || !fields || !rho || !out || nc <= 0 || nc > HFB_CON_MAX) return HFB_ERR_ARG;
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  cudaStream_t st = as_stream(stream);
  double* part = (double*)scratch(ctx, hfb_ctx_s::S_PART2, sizeof(double) * 2 * (HFB_CON_MAX + 1));
  if (!part) return HFB_ERR_ALLOC;
  con_moments_kernel<<<nc + 1, 1024, 0, st>>>(n3, nc, fields, rho, part);
  HFB_CHECK_LAUNCH();
  con_moments_final_kernel<<<1, 1, 0, st>>>(nc, part, ctx->wxyz, out);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_constraint_potential(hfb_ctx_t ctx, int prec, int nc, const double* fields, const double* lambda,
                                        double* upot, void* pot, void* stream) {
  if (!ctx || !fields || !lambda || nc <= 0 || nc > HFB_CON_MAX || (!upot && !pot)) return HFB_ERR_ARG;
  if (prec != HFB_F64 && prec != HFB_F32) return HFB_ERR_ARG;
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  ConCoef lam = {};
  for (int c = 0; c < nc; ++c) lam.c[c] = lambda[c];
  const unsigned nb = (unsigned)((n3 + 255) / 256);
  if (prec == HFB_F64)
    con_potential_kernel<double><<<nb, 256, 0, as_stream(stream)>>>(n3, nc, fields, lam, upot, (double*)pot);
  else
    con_potential_kernel<float><<<nb, 256, 0, as_stream(stream)>>>(n3, nc, fields, lam, upot, (float*)pot);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_constraint_correct(hfb_ctx_t ctx, int prec, int nst, int nc, const double* fields,
                                      const double* qcorr, const double* wocc, const double* wstates, void* psi,
                                      void* stream) {
  if (!ctx || !fields || !qcorr || !wocc || !wstates || !psi || nst <= 0 || nc <= 0 || nc > HFB_CON_MAX)
    return HFB_ERR_ARG;
  if (prec != HFB_F64 && prec != HFB_F32) return HFB_ERR_ARG;
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  ConCoef q = {};
  for (int c = 0; c < nc; ++c) q.c[c] = qcorr[c];
  dim3 grid((unsigned)((n3 + 255) / 256), nst);
  if (prec == HFB_F64)
    con_correct_kernel<double><<<grid, 256, 0, as_stream(stream)>>>(n3, nc, fields, q, wocc, wstates, (double2*)psi);
  else
    con_correct_kernel<float><<<grid, 256, 0, as_stream(stream)>>>(n3, nc, fields, q, wocc, wstates, (float2*)psi);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
