// Nyquist-line terms for the vector-Jacobian products of hpsi and of the
// densities.
//
// The second derivative of cderv02 (levels.py:284-395) replaces the Nyquist
// bin of each line along the derivative axis by -(pi/d)^2 mean(B) x_N / n,
// x_N = sum_j (-1)^j x_j.  As an operator on x this is c mean(B) e e^T with
// e_j = (-1)^j and c = -(pi/d)^2 / n: Hermitian in x and linear in B.  The
// rest of hpsi's bilinear form <a|h[P]|b> is the integral of each field
// times the pair density of (a, b) that the density kernel computes, so
// these two kernels are all the VJPs add to the library's hpsi and density
// kernels:
//   hfb_nyquist_pair   the bmass cotangent from this term,
//   hfb_nyquist_apply  the term itself, with B a density cotangent (the
//                      density tau has no Nyquist term, so the density VJP,
//                      formed with hpsi, takes it back out).
// Lines along axis ax are numbered by the two other coordinates (u, v) in
// increasing order; every sum runs in a fixed order.
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {
namespace {

constexpr int kVjThreads = 128;

struct LineGeo {
  size_t off, stride;
};

__device__ __forceinline__ LineGeo line_geo(int n, int ax, int line) {
  const int u = line / n, v = line % n;
  const size_t n2 = (size_t)n * n;
  if (ax == 0) return {(size_t)u * n + v, n2};
  if (ax == 1) return {(size_t)u * n2 + v, (size_t)n};
  return {(size_t)u * n2 + (size_t)v * n, 1};
}

// m[iq][ax][line] = sum_{s in iq} w_s sum_c Re(conj(a_N) b_N)
template <class Z>
__global__ void nyq_pair_lines_kernel(int n, int nst, int nneut, const Z* __restrict__ a, const Z* __restrict__ b,
                                      const double* __restrict__ w, double* __restrict__ m) {
  const int line = blockIdx.x * kVjThreads + threadIdx.x, ax = blockIdx.y, iq = blockIdx.z;
  if (line >= n * n) return;
  const LineGeo g = line_geo(n, ax, line);
  const size_t n3 = (size_t)n * n * n;
  const int s0 = iq == 0 ? 0 : nneut, s1 = iq == 0 ? nneut : nst;
  double acc = 0.0;
  for (int s = s0; s < s1; ++s) {
    double t = 0.0;
    for (int c = 0; c < 2; ++c) {
      const Z* pa = a + ((size_t)s * 2 + c) * n3 + g.off;
      const Z* pb = b + ((size_t)s * 2 + c) * n3 + g.off;
      double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
      for (int j = 0; j < n; ++j) {
        const double sg = (j & 1) ? -1.0 : 1.0;
        const Z x = pa[(size_t)j * g.stride], y = pb[(size_t)j * g.stride];
        ar += sg * (double)x.x;
        ai += sg * (double)x.y;
        br += sg * (double)y.x;
        bi += sg * (double)y.y;
      }
      t += ar * br + ai * bi;
    }
    acc += w[s] * t;
  }
  m[((size_t)iq * 3 + ax) * n * n + line] = acc;
}

// field[iq][x][y][z] += sum_ax (pi/d_ax)^2 / n^2 m[iq][ax][line_ax(x, y, z)]
__global__ void nyq_pair_field_kernel(int n, double k0, double k1, double k2, const double* __restrict__ m,
                                      double* __restrict__ field) {
  const size_t n3 = (size_t)n * n * n, n2 = (size_t)n * n;
  const size_t i = blockIdx.x * (size_t)kVjThreads + threadIdx.x;
  if (i >= 2 * n3) return;
  const int iq = (int)(i / n3);
  const size_t r = i % n3;
  const int x = (int)(r / n2), y = (int)((r / n) % n), z = (int)(r % n);
  const double* mq = m + (size_t)iq * 3 * n2;
  field[i] += k0 * mq[(size_t)y * n + z] + k1 * mq[n2 + (size_t)x * n + z] + k2 * mq[2 * n2 + (size_t)x * n + y];
}

// y_s += scale_s c mean_line(field[iq(s)]) (-1)^j x_N for the lines along ax
template <class Z>
__global__ void nyq_apply_kernel(int n, int nst, int nneut, int ax, double c, const double* __restrict__ field,
                                 const double* __restrict__ scale, const Z* __restrict__ x, Z* __restrict__ y) {
  const int line = blockIdx.x * kVjThreads + threadIdx.x;
  const int sc = blockIdx.y, s = sc / 2, comp = sc % 2;
  if (line >= n * n || s >= nst) return;
  const LineGeo g = line_geo(n, ax, line);
  const size_t n3 = (size_t)n * n * n;
  const double* f = field + (size_t)(s < nneut ? 0 : 1) * n3 + g.off;
  double fm = 0.0;
  for (int j = 0; j < n; ++j) fm += f[(size_t)j * g.stride];
  fm /= n;
  const Z* px = x + ((size_t)s * 2 + comp) * n3 + g.off;
  double xr = 0.0, xi = 0.0;
  for (int j = 0; j < n; ++j) {
    const double sg = (j & 1) ? -1.0 : 1.0;
    const Z v = px[(size_t)j * g.stride];
    xr += sg * (double)v.x;
    xi += sg * (double)v.y;
  }
  const double k = scale[s] * c * fm;
  Z* py = y + ((size_t)s * 2 + comp) * n3 + g.off;
  for (int j = 0; j < n; ++j) {
    const double sg = (j & 1) ? -k : k;
    Z v = py[(size_t)j * g.stride];
    v.x += sg * xr;
    v.y += sg * xi;
    py[(size_t)j * g.stride] = v;
  }
}

}  // namespace
}  // namespace hfb

using namespace hfb;

extern "C" int hfb_nyquist_pair(hfb_ctx_t ctx, int prec, int nst, int nneut, const void* a, const void* b,
                                const double* w, double* field, void* stream) {
  if (!ctx || !a || !b || !w || !field || nst <= 0 || nneut < 0 || nneut > nst) return HFB_ERR_ARG;
  const int n = ctx->n;
  double* m = (double*)scratch(ctx, hfb_ctx_s::S_VJP, sizeof(double) * 6 * (size_t)n * n);
  if (!m) return HFB_ERR_ALLOC;
  cudaStream_t st = as_stream(stream);
  const dim3 grid((n * n + kVjThreads - 1) / kVjThreads, 3, 2);
  if (prec == HFB_F64)
    nyq_pair_lines_kernel<double2><<<grid, kVjThreads, 0, st>>>(n, nst, nneut, (const double2*)a, (const double2*)b,
                                                                w, m);
  else
    nyq_pair_lines_kernel<float2><<<grid, kVjThreads, 0, st>>>(n, nst, nneut, (const float2*)a, (const float2*)b, w,
                                                               m);
  HFB_CHECK_LAUNCH();
  double k[3];
  for (int ax = 0; ax < 3; ++ax) k[ax] = (M_PI / ctx->d[ax]) * (M_PI / ctx->d[ax]) / ((double)n * n);
  const size_t tot = 2 * (size_t)n * n * n;
  nyq_pair_field_kernel<<<(unsigned)((tot + kVjThreads - 1) / kVjThreads), kVjThreads, 0, st>>>(n, k[0], k[1], k[2],
                                                                                               m, field);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_nyquist_apply(hfb_ctx_t ctx, int prec, int nst, int nneut, const double* field,
                                 const double* scale, const void* x, void* y, void* stream) {
  if (!ctx || !field || !scale || !x || !y || nst <= 0 || nneut < 0 || nneut > nst || x == y) return HFB_ERR_ARG;
  const int n = ctx->n;
  cudaStream_t st = as_stream(stream);
  const dim3 grid((n * n + kVjThreads - 1) / kVjThreads, 2 * nst);
  for (int ax = 0; ax < 3; ++ax) {
    const double c = -(M_PI / ctx->d[ax]) * (M_PI / ctx->d[ax]) / n;
    if (prec == HFB_F64)
      nyq_apply_kernel<double2><<<grid, kVjThreads, 0, st>>>(n, nst, nneut, ax, c, field, scale, (const double2*)x,
                                                             (double2*)y);
    else
      nyq_apply_kernel<float2><<<grid, kVjThreads, 0, st>>>(n, nst, nneut, ax, c, field, scale, (const float2*)x,
                                                            (float2*)y);
    HFB_CHECK_LAUNCH();
  }
  return HFB_OK;
}
