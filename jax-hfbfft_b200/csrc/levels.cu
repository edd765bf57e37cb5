// Spectral derivatives along one axis: cderv{x,y,z}{00,01,02} of
// levels.py:132-395, on nsp spinors (2 components each).
//   kind 0: d1 = F^-1[i k kfac/n F psi], bins 0 and n/2 zeroed
//   kind 1: d1 and d2 = F^-1[-(|k| kfac)^2/n F psi] (Nyquist kept)
//   kind 2: d1 and d(B d1): F^-1[i k kfac/n F(B d1)] with bin 0 zeroed and
//           bin n/2 = -(pi/h)^2 mean_axis(B) (F psi)(n/2) / n
// (F unnormalised forward, F^-1 unnormalised inverse: the reference's
// fft(norm="backward") / ifft(norm="forward") pair.)
#include "hfb_ctx.cuh"

namespace hfb {

template <class R, int N, int AXIS, int KIND>
__global__ void __launch_bounds__(256)
cderv_kernel(int nfield, const cplx<R>* __restrict__ in, const double* __restrict__ bf, double kscale, double k2scale,
             double nyq_scale, cplx<R>* d1, cplx<R>* d2) {
  constexpr int P = PencilSplit<R, N>::P;
  constexpr int M = N / P, T = (M + P - 1) / P, L = 256 / P, NB = N + 4;
  using PC = Pencil<R, N, P>;
  using Z = cplx<R>;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  __shared__ __align__(16) Z xball[L * NB];
  __shared__ Z tw[N];
  fill_twiddles<R>(tw, N);
  __syncthreads();
  const int lg = threadIdx.x / P, p = threadIdx.x % P;
  const long line_raw = (long)blockIdx.x * L + lg;
  const bool active = line_raw < (long)nfield * N * N;
  const long line = active ? line_raw : 0;
  const int fld = (int)(line / (N * N));
  const int rem = (int)(line % (N * N));
  const int u = rem / N, v = rem % N;
  size_t base, stride;
  if (AXIS == 2) { base = (size_t)u * N2 + (size_t)v * N; stride = 1; }
  else if (AXIS == 1) { base = (size_t)u * N2 + v; stride = N; }
  else { base = (size_t)u * N + v; stride = N2; }
  const size_t fb = (size_t)fld * N3;
  Z* xb = xball + lg * NB;
  Z x[M];
  Z f[T][P];
#pragma unroll
  for (int m = 0; m < M; ++m) x[m] = in[fb + base + (size_t)(p + P * m) * stride];
  PC::forward(x, f, xb, tw, p, 0xffffffffu);
  const Z nyq = f[0][P / 2];
  Z g[T][P];
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      const int k = PC::freq(p, t, k1);
      const R s = (k == 0 || 2 * k == N) ? R(0) : (R)(signed_k(k, N) * kscale);
      g[t][k1] = mk<R>(-s * f[t][k1].y, s * f[t][k1].x);
    }
  Z o1[M];
  PC::inverse(g, o1, xb, tw, p, 0xffffffffu);
  if (active) {
#pragma unroll
    for (int m = 0; m < M; ++m) d1[fb + base + (size_t)(p + P * m) * stride] = o1[m];
  }
  if (KIND == 1) {
#pragma unroll
    for (int t = 0; t < T; ++t)
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) {
        const int k = PC::freq(p, t, k1);
        const int ka = k <= N / 2 ? k : N - k;
        const R s = (R)(-(double)ka * ka * k2scale);
        f[t][k1] = s * f[t][k1];
      }
    Z o2[M];
    PC::inverse(f, o2, xb, tw, p, 0xffffffffu);
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) d2[fb + base + (size_t)(p + P * m) * stride] = o2[m];
    }
  } else if (KIND == 2) {
    R bsum = 0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const R b = (R)bf[base + (size_t)(p + P * m) * stride];
      bsum += b;
      o1[m] = b * o1[m];
    }
#pragma unroll
    for (int o = 1; o < P; o <<= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
    const R bbar = bsum / R(N);
    PC::forward(o1, f, xb, tw, p, 0xffffffffu);
#pragma unroll
    for (int t = 0; t < T; ++t)
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) {
        const int k = PC::freq(p, t, k1);
        if (2 * k == N) {
          f[t][k1] = (-(R)nyq_scale * bbar) * nyq;
        } else {
          const R s = (k == 0) ? R(0) : (R)(signed_k(k, N) * kscale);
          f[t][k1] = mk<R>(-s * f[t][k1].y, s * f[t][k1].x);
        }
      }
    Z o2[M];
    PC::inverse(f, o2, xb, tw, p, 0xffffffffu);
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) d2[fb + base + (size_t)(p + P * m) * stride] = o2[m];
    }
  }
}

template <class R, int N, int AXIS>
static int cderv_axis(int kind, int nsp, const void* in, const double* bf, double h, void* d1, void* d2,
                      cudaStream_t st) {
  using Z = cplx<R>;
  constexpr int P = PencilSplit<R, N>::P;
  constexpr int L = 256 / P;
  const int nfield = 2 * nsp;
  const long lines = (long)nfield * N * N;
  const unsigned grid = (unsigned)((lines + L - 1) / L);
  const double kfac = 2.0 * kPi / (h * N);
  const double ks = kfac / N, k2s = kfac * kfac / N, nq = (kPi / h) * (kPi / h) / N;
  if (kind == 0)
    cderv_kernel<R, N, AXIS, 0><<<grid, 256, 0, st>>>(nfield, (const Z*)in, bf, ks, k2s, nq, (Z*)d1, (Z*)d2);
  else if (kind == 1)
    cderv_kernel<R, N, AXIS, 1><<<grid, 256, 0, st>>>(nfield, (const Z*)in, bf, ks, k2s, nq, (Z*)d1, (Z*)d2);
  else
    cderv_kernel<R, N, AXIS, 2><<<grid, 256, 0, st>>>(nfield, (const Z*)in, bf, ks, k2s, nq, (Z*)d1, (Z*)d2);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

template <class R, int N>
static int cderv_t(hfb_ctx_s* c, int kind, int axis, int nsp, const void* in, const double* bf, void* d1, void* d2,
                   cudaStream_t st) {
  const double h = c->d[axis];
  if (axis == 0) return cderv_axis<R, N, 0>(kind, nsp, in, bf, h, d1, d2, st);
  if (axis == 1) return cderv_axis<R, N, 1>(kind, nsp, in, bf, h, d1, d2, st);
  return cderv_axis<R, N, 2>(kind, nsp, in, bf, h, d1, d2, st);
}

}  // namespace hfb

extern "C" int hfb_cderv(hfb_ctx_t ctx, int prec, int kind, int axis, int nsp, const void* psin, const double* bfield,
                         void* d1, void* d2, void* stream) {
  if (!ctx || !psin || !d1 || nsp <= 0 || kind < 0 || kind > 2 || axis < 0 || axis > 2) return HFB_ERR_ARG;
  if (kind > 0 && !d2) return HFB_ERR_ARG;
  if (kind == 2 && !bfield) return HFB_ERR_ARG;
  cudaStream_t st = hfb::as_stream(stream);
  return hfb::dispatch_n(ctx->n, [&](auto nn) -> int {
    constexpr int N = decltype(nn)::value;
    if (prec == HFB_F64) return hfb::cderv_t<double, N>(ctx, kind, axis, nsp, psin, bfield, d1, d2, st);
    return hfb::cderv_t<float, N>(ctx, kind, axis, nsp, psin, bfield, d1, d2, st);
  });
}
