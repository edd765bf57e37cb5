// Energies (integ_energy / sum_energy, energies.py:90-372), point rms radii
// (output.py:187-226, 246) and the harmonic-oscillator initial states
// (harmosc, static.py:580-738).  FP64, deterministic two-stage reductions.
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {

int density_derivatives(hfb_ctx_s* c, const double* rho, const double* cur, const double* sd, const double* so,
                        bool need_grad_curls, double** dv_out, cudaStream_t st);
constexpr int kNDerivE = 11;   // layout of density_derivatives (skyrme.cu)

enum { I_EHF0 = 0, I_CRHO0, I_CRHO1, I_EHF3, I_EHF2, I_CDRHO0, I_CDRHO1, I_CTAU0, I_CTAU1, I_EHF1, I_LSEVEN, I_CDJ0,
       I_CDJ1, I_LSODD, I_EHFC, I_ECORC, I_EHFT, I_NSUM };

constexpr int kEnBlocks = 296;

__global__ void __launch_bounds__(256)
energy_points_kernel(hfb_force f, int tcoul, size_t n3, const double* rho, const double* tau, const double* sd,
                     const double* wcoul, const double* dv, double* part) {
  double acc[I_NSUM];
#pragma unroll
  for (int k = 0; k < I_NSUM; ++k) acc[k] = 0.0;
  const double* d0 = dv;
  const double* d1 = dv + (size_t)kNDerivE * n3;
  const double sc = (f.ex != 0) ? -3.0 / 4.0 * f.slate : 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    const double rn = rho[i], rp = rho[n3 + i];
    const double rt = rn + rp, r1 = -rn + rp;
    const double ln = d0[n3 + i], lp = d1[n3 + i];
    const double d2 = ln + lp, d21 = -ln + lp;
    const double tn = tau[i], tp = tau[n3 + i];
    const double t0 = tn + tp, t1 = -tn + tp;
    const double rtp = pow(rt, f.power);
    acc[I_EHF0] += (f.b0 * rt * rt - f.b0p * (rp * rp + rn * rn)) / 2.0;
    acc[I_CRHO0] += (f.Crho0 + f.Crho0D * rtp) * rt * rt;
    acc[I_CRHO1] += (f.Crho1 + f.Crho1D * rtp) * r1 * r1;
    acc[I_EHF3] += rtp * (f.b3 * rt * rt - f.b3p * (rp * rp + rn * rn)) / 3.0;
    acc[I_EHF2] += (-f.b2 * rt * d2 + f.b2p * (rp * lp + rn * ln)) / 2.0;
    acc[I_CDRHO0] += f.Cdrho0 * rt * d2;
    acc[I_CDRHO1] += f.Cdrho1 * r1 * d21;
    acc[I_CTAU0] += f.Ctau0 * t0 * rt;
    acc[I_CTAU1] += f.Ctau1 * t1 * r1;
    acc[I_EHF1] += f.b1 * (rt * t0) - f.b1p * (rn * tn + rp * tp);
    const double jn = d0[i], jp = d1[i];   // div J
    acc[I_LSEVEN] += -f.b4 * rt * (jn + jp) - f.b4p * (rp * jp + rn * jn);
    acc[I_CDJ0] += f.CdJ0 * rt * (jn + jp);
    acc[I_CDJ1] += f.CdJ1 * r1 * (-jn + jp);
    double odd_b4 = 0.0, odd_b4p = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double cn = d0[(8 + k) * n3 + i], cp = d1[(8 + k) * n3 + i];   // curl j
      const double sn = sd[(size_t)k * n3 + i], sp = sd[(size_t)(3 + k) * n3 + i];
      odd_b4 += (sn + sp) * (cn + cp);
      odd_b4p += sn * cn + sp * cp;
    }
    acc[I_LSODD] += -f.b4 * odd_b4 - f.b4p * odd_b4p;
    if (tcoul) {
      const double r43 = pow(rp, 4.0 / 3.0);
      acc[I_EHFC] += 0.5 * rp * wcoul[i] + sc * r43;
      acc[I_ECORC] += sc / 3.0 * r43;
    }
    acc[I_EHFT] += f.h2m[0] * tn + f.h2m[1] * tp;
  }
  __shared__ double red[I_NSUM][8];
#pragma unroll
  for (int k = 0; k < I_NSUM; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x % 32 == 0) red[k][threadIdx.x / 32] = v;
  }
  __syncthreads();
  if (threadIdx.x < I_NSUM) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += red[threadIdx.x][w];
    part[(size_t)blockIdx.x * I_NSUM + threadIdx.x] = v;
  }
}

__global__ void energy_final_kernel(hfb_force f, int tcoul, double A, double wxyz, int n, int nblk, const double* part,
                                    const double* cur, const double* epair, double* out, int* status) {
  __shared__ double s[I_NSUM];
  if (threadIdx.x < I_NSUM) {
    double v = 0.0;
    for (int b = 0; b < nblk; ++b) v += part[(size_t)b * I_NSUM + threadIdx.x];
    s[threadIdx.x] = wxyz * v;
  }
  __syncthreads();
  // energies.py:157-167 (diagnostic; indexes current[iq, comp, x, c, s] with
  // y = c, z = s): the 2 x 3 x n x 3 terms spread over the warp
  const size_t n3 = (size_t)n * n * n;
  double cj0 = 0.0, cj1 = 0.0;
  for (int e = threadIdx.x; e < 2 * 3 * n * 3; e += blockDim.x) {
    const int c = e % 3, x = (e / 3) % n, comp = (e / (3 * n)) % 3, iq = e / (9 * n);
    const double* base = cur + ((size_t)iq * 3 + comp) * n3 + (size_t)x * n * n + (size_t)c * n;
    const double a0 = base[0], a1 = base[1];
    cj0 += (a0 + a1) * (a0 + a1);
    cj1 += (-a0 + a1) * (-a0 + a1);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cj0 += __shfl_xor_sync(0xffffffffu, cj0, o);
    cj1 += __shfl_xor_sync(0xffffffffu, cj1, o);
  }
  if (threadIdx.x != 0) return;
  const double ep = epair[0] + epair[1];
  const double ehf3 = s[I_EHF3];
  const double e3corr = -f.power * ehf3 / 2.0;
  const double ehfls = s[I_LSEVEN] + s[I_LSODD];
  const double ezpe = f.zpe == 1 ? 17.3 / pow(A, 0.2) : 0.0;
  const double ehfc = tcoul ? s[I_EHFC] : 0.0, ecorc = tcoul ? s[I_ECORC] : 0.0;
  const double ehfint = s[I_EHFT] + s[I_EHF0] + s[I_EHF1] + s[I_EHF2] + ehf3 + ehfls + ehfc - ep - ezpe;
  out[HFB_E_EHFT] = s[I_EHFT];
  out[HFB_E_EHF0] = s[I_EHF0];
  out[HFB_E_EHF1] = s[I_EHF1];
  out[HFB_E_EHF2] = s[I_EHF2];
  out[HFB_E_EHF3] = ehf3;
  out[HFB_E_EHFLS] = ehfls;
  out[HFB_E_EHFLSODD] = s[I_LSODD];
  out[HFB_E_EHFC] = ehfc;
  out[HFB_E_ECORC] = ecorc;
  out[HFB_E_EHFINT] = ehfint;
  out[HFB_E_E3CORR] = e3corr;
  out[HFB_E_EZPE] = ezpe;
  out[HFB_E_CRHO0] = s[I_CRHO0];
  out[HFB_E_CRHO1] = s[I_CRHO1];
  out[HFB_E_CDRHO0] = s[I_CDRHO0];
  out[HFB_E_CDRHO1] = s[I_CDRHO1];
  out[HFB_E_CTAU0] = s[I_CTAU0];
  out[HFB_E_CTAU1] = s[I_CTAU1];
  out[HFB_E_CDJ0] = s[I_CDJ0];
  out[HFB_E_CDJ1] = s[I_CDJ1];
  out[HFB_E_CJ0] = -wxyz * f.Ctau0 * cj0;
  out[HFB_E_CJ1] = -wxyz * f.Ctau1 * cj1;
  if (!isfinite(ehfint)) latch_error(status, HFB_ERR_NONFINITE);
}

// sum_energy (energies.py:309-318): one warp, fixed-order sums.
__global__ void sum_energy_kernel(int nst, const double* wocc, const double* wstates, const double* kin,
                                  const double* spe, const double* epair, const double* ecorrp, double* out,
                                  int* status) {
  double sk = 0.0, tk = 0.0;
  for (int k = threadIdx.x; k < nst; k += 32) {
    const double ww = wocc[k] * wstates[k];
    sk += ww * (kin[k] + spe[k]);
    tk += ww * kin[k];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sk += __shfl_xor_sync(0xffffffffu, sk, o);
    tk += __shfl_xor_sync(0xffffffffu, tk, o);
  }
  if (threadIdx.x == 0) {
    const double ehf = sk / 2.0 + out[HFB_E_E3CORR] + ecorrp[0] + out[HFB_E_ECORC] - (epair[0] + epair[1]) -
                       out[HFB_E_EZPE];
    out[HFB_E_EHF] = ehf;
    out[HFB_E_TKE] = tk;
    if (!isfinite(ehf)) latch_error(status, HFB_ERR_NONFINITE);
  }
}

// rms radii: one CTA per isospin, two passes (c.m., then <r^2> about it)
__global__ void rms_kernel(int n, const double* rho, double dx, double dy, double dz, double wxyz, double* part) {
  const int iq = blockIdx.x;
  const size_t n3 = (size_t)n * n * n;
  const double* r = rho + (size_t)iq * n3;
  __shared__ double red[4][32];
  __shared__ double mom[4];
  double s[4] = {0, 0, 0, 0};
  for (size_t i = threadIdx.x; i < n3; i += blockDim.x) {
    const int x = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), z = (int)(i % n);
    const double cx = (x - (n - 1) / 2.0) * dx, cy = (y - (n - 1) / 2.0) * dy, cz = (z - (n - 1) / 2.0) * dz;
    s[0] += r[i];
    s[1] += cx * r[i];
    s[2] += cy * r[i];
    s[3] += cz * r[i];
  }
  for (int k = 0; k < 4; ++k) {
    double v = s[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x % 32 == 0) red[k][threadIdx.x / 32] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += red[threadIdx.x][w];
    mom[threadIdx.x] = v;
  }
  __syncthreads();
  const double pnr = mom[0] * wxyz;
  const double cmx = mom[1] * wxyz / pnr, cmy = mom[2] * wxyz / pnr, cmz = mom[3] * wxyz / pnr;
  double q = 0.0;
  for (size_t i = threadIdx.x; i < n3; i += blockDim.x) {
    const int x = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), z = (int)(i % n);
    const double cx = (x - (n - 1) / 2.0) * dx - cmx, cy = (y - (n - 1) / 2.0) * dy - cmy,
                 cz = (z - (n - 1) / 2.0) * dz - cmz;
    q += (cx * cx + cy * cy + cz * cz) * r[i];
  }
  for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
  __syncthreads();
  if (threadIdx.x % 32 == 0) red[0][threadIdx.x / 32] = q;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += red[0][w];
    part[iq * 2 + 0] = pnr;
    part[iq * 2 + 1] = sqrt(v * wxyz / pnr);
  }
}

__global__ void rms_final_kernel(const double* part, double* out) {
  const double p0 = part[0], r0 = part[1], p1 = part[2], r1 = part[3];
  out[0] = p0;
  out[1] = p1;
  out[2] = r0;
  out[3] = r1;
  out[4] = sqrt((p0 * r0 * r0 + p1 * r1 * r1) / (p0 + p1));
}

// ---------------------------------------------------------------- harmosc --
__device__ __forceinline__ double ipow(double x, int k) {
  double r = 1.0;
  for (int j = 0; j < k; ++j) r *= x;
  return r;
}

template <class R>
__global__ void ho_fill_kernel(int n, int nst, const int* qn, double rx, double ry, double rz, double dx, double dy,
                               double dz, cplx<R>* psi) {
  const size_t n3 = (size_t)n * n * n;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= n3) return;
  const int x = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), z = (int)(i % n);
  const double cx = (x - (n - 1) / 2.0) * dx, cy = (y - (n - 1) / 2.0) * dy, cz = (z - (n - 1) / 2.0) * dz;
  const double g = exp(-((cx / rx) * (cx / rx) + (cy / ry) * (cy / ry) + (cz / rz) * (cz / rz)));
  const int qi = qn[4 * s], qj = qn[4 * s + 1], qk = qn[4 * s + 2], c = qn[4 * s + 3];
  const double v = g * ipow(cx, qi) * ipow(cy, qj) * ipow(cz, qk);
  cplx<R>* p = psi + (size_t)s * 2 * n3;
  p[(size_t)c * n3 + i] = mk<R>((R)v, R(0));
  p[(size_t)(1 - c) * n3 + i] = mk<R>(R(0), R(0));
}

// norm[s] = wxyz sum |psi_s|^2 and the Gaussian's own norm (static.py:608-610).
template <class R>
__global__ void ho_norm_kernel(int n, const cplx<R>* psi, double rx, double ry, double rz, double dx, double dy,
                               double dz, double wxyz, double* norms, double* gnorm) {
  const size_t n3 = (size_t)n * n * n;
  const int s = blockIdx.x;
  __shared__ double red[2][32];
  double a = 0.0, g2 = 0.0;
  const cplx<R>* p = psi + (size_t)s * 2 * n3;
  for (size_t i = threadIdx.x; i < 2 * n3; i += blockDim.x) {
    const double re = p[i].x, im = p[i].y;
    a += re * re + im * im;
    if (s == 0 && i < n3) {
      const int x = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), z = (int)(i % n);
      const double cx = (x - (n - 1) / 2.0) * dx, cy = (y - (n - 1) / 2.0) * dy, cz = (z - (n - 1) / 2.0) * dz;
      const double g = exp(-((cx / rx) * (cx / rx) + (cy / ry) * (cy / ry) + (cz / rz) * (cz / rz)));
      g2 += g * g;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    g2 += __shfl_xor_sync(0xffffffffu, g2, o);
  }
  if (threadIdx.x % 32 == 0) { red[0][threadIdx.x / 32] = a; red[1][threadIdx.x / 32] = g2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0, v = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) { u += red[0][w]; v += red[1][w]; }
    norms[s] = wxyz * u;
    if (s == 0) gnorm[0] = wxyz * v;
  }
}

// Normalise: the reference divides by sqrt(anorm) with anorm measured on
// the Gaussian-normalised product, and skips states with anorm <= 1e-12
// (static.py:727-729); the first state of each isospin is always scaled.
template <class R>
__global__ void ho_scale_kernel(int n, const int* qn, const double* norms, const double* gnorm, cplx<R>* psi) {
  const size_t n3 = (size_t)n * n * n;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= 2 * n3) return;
  const double an = norms[s] / gnorm[0];
  const bool first = qn[4 * s] == 0 && qn[4 * s + 1] == 0 && qn[4 * s + 2] == 0 && qn[4 * s + 3] == 0;
  if (!first && !(an > 1e-12)) {
    // leave the state Gaussian-normalised only
    const double sc = 1.0 / sqrt(gnorm[0]);
    cplx<R>* p = psi + (size_t)s * 2 * n3;
    p[i] = mk<R>((R)(p[i].x * sc), (R)(p[i].y * sc));
    return;
  }
  const double sc = 1.0 / sqrt(norms[s]);
  cplx<R>* p = psi + (size_t)s * 2 * n3;
  p[i] = mk<R>((R)(p[i].x * sc), (R)(p[i].y * sc));
}

// ---------------------------------------------------------------------------
// Explicit derivatives of the integrated Skyrme functional (energies.py:
// 117-258, the terms of ehfint) with respect to its coefficients b0 .. b4p
// and the density-dependence power alpha, at fixed densities.  Each term of
// ehfint is linear in one b coefficient, so dE/db is the integral that
// multiplies it; dE/dalpha = int rho^alpha ln(rho) (b3 rho^2 - b3p sum_q
// rho_q^2) / 3 (points with rho = 0 contribute nothing).
enum { G_B0 = 0, G_B0P, G_B1, G_B1P, G_B2, G_B2P, G_B3, G_B3P, G_B4, G_B4P, G_POWER, G_NSUM };
static_assert(G_NSUM == HFB_NG, "gradient slots");

__global__ void __launch_bounds__(256)
energy_grad_points_kernel(hfb_force f, size_t n3, const double* rho, const double* tau, const double* sd,
                          const double* dv, double* part) {
  double acc[G_NSUM];
#pragma unroll
  for (int k = 0; k < G_NSUM; ++k) acc[k] = 0.0;
  const double* d0 = dv;
  const double* d1 = dv + (size_t)kNDerivE * n3;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    const double rn = rho[i], rp = rho[n3 + i];
    const double rt = rn + rp, rq2 = rn * rn + rp * rp;
    const double ln = d0[n3 + i], lp = d1[n3 + i];   // Laplacians
    const double tn = tau[i], tp = tau[n3 + i];
    const double jn = d0[i], jp = d1[i];             // div J
    const double rtp = pow(rt, f.power);
    acc[G_B0] += rt * rt / 2.0;
    acc[G_B0P] += -rq2 / 2.0;
    acc[G_B1] += rt * (tn + tp);
    acc[G_B1P] += -(rn * tn + rp * tp);
    acc[G_B2] += -rt * (ln + lp) / 2.0;
    acc[G_B2P] += (rp * lp + rn * ln) / 2.0;
    acc[G_B3] += rtp * rt * rt / 3.0;
    acc[G_B3P] += -rtp * rq2 / 3.0;
    double odd_b4 = 0.0, odd_b4p = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double cn = d0[(8 + k) * n3 + i], cp = d1[(8 + k) * n3 + i];   // curl j
      const double sn = sd[(size_t)k * n3 + i], sp = sd[(size_t)(3 + k) * n3 + i];
      odd_b4 += (sn + sp) * (cn + cp);
      odd_b4p += sn * cn + sp * cp;
    }
    acc[G_B4] += -rt * (jn + jp) - odd_b4;
    acc[G_B4P] += -(rp * jp + rn * jn) - odd_b4p;
    if (rt > 0.0) acc[G_POWER] += rtp * log(rt) * (f.b3 * rt * rt - f.b3p * rq2) / 3.0;
  }
  __shared__ double red[G_NSUM][8];
#pragma unroll
  for (int k = 0; k < G_NSUM; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x % 32 == 0) red[k][threadIdx.x / 32] = v;
  }
  __syncthreads();
  if (threadIdx.x < G_NSUM) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) v += red[threadIdx.x][w];
    part[(size_t)blockIdx.x * G_NSUM + threadIdx.x] = v;
  }
}

__global__ void energy_grad_final_kernel(double wxyz, int nblk, const double* part, double* out) {
  if (threadIdx.x >= G_NSUM) return;
  double v = 0.0;
  for (int b = 0; b < nblk; ++b) v += part[(size_t)b * G_NSUM + threadIdx.x];
  out[threadIdx.x] = wxyz * v;
}

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_energies(hfb_ctx_t ctx, const hfb_force* f, int tcoul, double mass_number, const double* rho,
                            const double* tau, const double* current, const double* sdens, const double* sodens,
                            const double* wcoul, const double* epair, double* out, void* stream) {
  if (!ctx || !f || !rho || !tau || !current || !sdens || !sodens || !epair || !out) return HFB_ERR_ARG;
  if (tcoul && !wcoul) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  double* dv = nullptr;
  int r = density_derivatives(ctx, rho, current, sdens, sodens, false, &dv, st);
  if (r) return r;
  double* part = (double*)scratch(ctx, hfb_ctx_s::S_PART2, sizeof(double) * (size_t)kEnBlocks * I_NSUM);
  if (!part) return HFB_ERR_ALLOC;
  energy_points_kernel<<<kEnBlocks, 256, 0, st>>>(*f, tcoul, n3, rho, tau, sdens, wcoul, dv, part);
  HFB_CHECK_LAUNCH();
  energy_final_kernel<<<1, 32, 0, st>>>(*f, tcoul, mass_number, ctx->wxyz, ctx->n, kEnBlocks, part, current, epair,
                                        out, ctx->dev_status);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_sum_energy(hfb_ctx_t ctx, int nst, const double* wocc, const double* wstates,
                              const double* sp_kinetic, const double* sp_energy, const double* epair,
                              const double* ecorrp, double* out, void* stream) {
  if (!ctx || !wocc || !wstates || !sp_kinetic || !sp_energy || !epair || !ecorrp || !out || nst <= 0)
    return HFB_ERR_ARG;
  sum_energy_kernel<<<1, 32, 0, as_stream(stream)>>>(nst, wocc, wstates, sp_kinetic, sp_energy, epair, ecorrp, out,
                                                      ctx->dev_status);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_rms(hfb_ctx_t ctx, const double* rho, double* out, void* stream) {
  if (!ctx || !rho || !out) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  double* part = (double*)scratch(ctx, hfb_ctx_s::S_PART2, sizeof(double) * 8);
  if (!part) return HFB_ERR_ALLOC;
  rms_kernel<<<2, 1024, 0, st>>>(ctx->n, rho, ctx->d[0], ctx->d[1], ctx->d[2], ctx->wxyz, part);
  HFB_CHECK_LAUNCH();
  rms_final_kernel<<<1, 1, 0, st>>>(part, out);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_harmosc(hfb_ctx_t ctx, int prec, int nst, const int* qn, double radinx, double radiny,
                           double radinz, void* psi, void* stream) {
  if (!ctx || !qn || !psi || nst <= 0) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const int n = ctx->n;
  const size_t n3 = (size_t)n * n * n;
  double* nrm = (double*)scratch(ctx, hfb_ctx_s::S_PART2, sizeof(double) * ((size_t)nst + 2));
  if (!nrm) return HFB_ERR_ALLOC;
  dim3 g1((unsigned)((n3 + 255) / 256), nst), g2((unsigned)((2 * n3 + 255) / 256), nst);
  const double* d = ctx->d;
  if (prec == HFB_F64) {
    ho_fill_kernel<double><<<g1, 256, 0, st>>>(n, nst, qn, radinx, radiny, radinz, d[0], d[1], d[2], (double2*)psi);
    HFB_CHECK_LAUNCH();
    ho_norm_kernel<double><<<nst, 256, 0, st>>>(n, (const double2*)psi, radinx, radiny, radinz, d[0], d[1], d[2],
                                                ctx->wxyz, nrm, nrm + nst);
    HFB_CHECK_LAUNCH();
    ho_scale_kernel<double><<<g2, 256, 0, st>>>(n, qn, nrm, nrm + nst, (double2*)psi);
  } else {
    ho_fill_kernel<float><<<g1, 256, 0, st>>>(n, nst, qn, radinx, radiny, radinz, d[0], d[1], d[2], (float2*)psi);
    HFB_CHECK_LAUNCH();
    ho_norm_kernel<float><<<nst, 256, 0, st>>>(n, (const float2*)psi, radinx, radiny, radinz, d[0], d[1], d[2],
                                               ctx->wxyz, nrm, nrm + nst);
    HFB_CHECK_LAUNCH();
    ho_scale_kernel<float><<<g2, 256, 0, st>>>(n, qn, nrm, nrm + nst, (float2*)psi);
  }
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_energy_grad(hfb_ctx_t ctx, const hfb_force* f, const double* rho, const double* tau,
                               const double* current, const double* sdens, const double* sodens, double* out,
                               void* stream) {
  if (!ctx || !f || !rho || !tau || !current || !sdens || !sodens || !out) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  double* dv = nullptr;
  int r = density_derivatives(ctx, rho, current, sdens, sodens, false, &dv, st);
  if (r) return r;
  double* part = (double*)scratch(ctx, hfb_ctx_s::S_PART2, sizeof(double) * (size_t)kEnBlocks * G_NSUM);
  if (!part) return HFB_ERR_ALLOC;
  energy_grad_points_kernel<<<kEnBlocks, 256, 0, st>>>(*f, n3, rho, tau, sdens, dv, part);
  HFB_CHECK_LAUNCH();
  energy_grad_final_kernel<<<1, 32, 0, st>>>(ctx->wxyz, kEnBlocks, part, out);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
