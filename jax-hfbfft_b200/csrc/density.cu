// Occupation-weighted densities (add_density, densities.py:177-330) and the
// single-particle kinetic energy of sp_properties (inout.py:64-150).
//
// Every density term is local or bilinear in psi and ONE first derivative
// d_d psi (cderv d00), so the work splits into three line kernels, one per
// axis d.  A CTA owns a tile of lines along d and loops over a chunk of
// states of one isospin: per state it FFTs each line, forms d_d psi, and
// accumulates its fields in FP64 registers (lane-owned points, no atomics).
// Per-chunk partial fields are summed in a fixed order by a combine kernel,
// which also applies the density mixing of static.py:1820-1823.
//
// Kinetic energy: with the unnormalised FFT and Parseval,
//   sum_k k_d^2 |psi_k|^2 / Ntot = sum_r |D_d psi|^2
//                                 + (pi/h_d)^2 / n * sum_lines |psi_hat_d(n/2)|^2
// where D_d is the Nyquist-zeroed derivative and psi_hat_d(n/2) the 1-D FFT
// of the line at the Nyquist bin; sp_kinetic = wxyz h2m_q sum_d (...).
#include "hfb_ctx.cuh"

namespace hfb {

template <class R, int N>
struct DensGeo {
  static constexpr int P = (N >= 32) ? 8 : (N >= 16 ? 4 : 2);
  static constexpr int M = N / P;
  static constexpr int T = (M + P - 1) / P;
  static constexpr int L = 256 / P;          // lines per CTA
  static constexpr int THREADS = L * P;
  static constexpr int NB = N + 4;
  static constexpr int NTILE = (N * N + L - 1) / L;
  static constexpr int WARPS = THREADS / 32;
};

// number of accumulated fields per axis kernel
template <int AXIS> struct DensFields { static constexpr int value = AXIS == 2 ? 9 : 4; };

template <class R, int N, int AXIS>
__global__ void __launch_bounds__(DensGeo<R, N>::THREADS)
density_axis_kernel(const cplx<R>* __restrict__ psi, int nst, int nneut, int nchunk, const double* __restrict__ wocc,
                    const double* __restrict__ wguv, const double* __restrict__ pairwg,
                    const double* __restrict__ wstates, double kscale, double nyq_fac, int want_fields, double* part,
                    double* kin_part) {
  using G = DensGeo<R, N>;
  using PC = Pencil<R, N, G::P>;
  using Z = cplx<R>;
  constexpr int P = G::P, M = G::M, T = G::T;
  constexpr int NF = DensFields<AXIS>::value;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  __shared__ __align__(16) cplx<R> xball[G::L * G::NB];
  __shared__ cplx<R> tw[N];
  fill_twiddles<R>(tw, N);
  __syncthreads();
  const int tile = blockIdx.x;
  const int iq = blockIdx.y / nchunk, chunk = blockIdx.y % nchunk;
  const int q0 = iq == 0 ? 0 : nneut, q1 = iq == 0 ? nneut : nst;
  const int cnt = q1 - q0;
  const int sa = q0 + (int)(((long)cnt * chunk) / nchunk), sb = q0 + (int)(((long)cnt * (chunk + 1)) / nchunk);
  const int lg = threadIdx.x / P, p = threadIdx.x % P;
  const int line_raw = tile * G::L + lg;
  const bool active = line_raw < N * N;
  const int line = active ? line_raw : 0;
  // line -> (u, v) transverse coordinates with the contiguous one fastest
  const int u = line / N, v = line % N;
  size_t base, stride;
  if (AXIS == 2) { base = (size_t)u * N2 + (size_t)v * N; stride = 1; }        // (x, y) fixed
  else if (AXIS == 1) { base = (size_t)u * N2 + v; stride = N; }               // (x, z) fixed
  else { base = (size_t)u * N + v; stride = N2; }                             // (y, z) fixed
  Z* xb = xball + lg * G::NB;
  double acc[NF][M];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int m = 0; m < M; ++m) acc[f][m] = 0.0;

  // the line values of the next state are loaded while this one is
  // transformed and accumulated
  Z an[M], bn[M];
  if (sa < sb) {
    const Z* ps = psi + (size_t)sa * 2 * N3 + base;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      an[m] = ps[(size_t)(p + P * m) * stride];
      bn[m] = ps[N3 + (size_t)(p + P * m) * stride];
    }
  }
  for (int s = sa; s < sb; ++s) {
    const double w = want_fields ? wocc[s] * wstates[s] : 0.0;
    const double wu = want_fields ? wguv[s] * pairwg[s] * wstates[s] : 0.0;
    Z a[M], b[M], da[M], db[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      a[m] = an[m];
      b[m] = bn[m];
    }
    if (s + 1 < sb) {
      const Z* ps = psi + (size_t)(s + 1) * 2 * N3 + base;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        an[m] = ps[(size_t)(p + P * m) * stride];
        bn[m] = ps[N3 + (size_t)(p + P * m) * stride];
      }
    }
    double knyq = 0.0;
    // D_d psi for both components (cderv d00: k = 0 and Nyquist zeroed)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      Z vv[M];
      Z f[T][P];
#pragma unroll
      for (int m = 0; m < M; ++m) vv[m] = c == 0 ? a[m] : b[m];
      PC::forward(vv, f, xb, tw, p, 0xffffffffu);
      if (p == 0) knyq += (double)f[0][P / 2].x * f[0][P / 2].x + (double)f[0][P / 2].y * f[0][P / 2].y;
#pragma unroll
      for (int t = 0; t < T; ++t) {
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) {
          int k = PC::freq(p, t, k1);
          R sc = (k == 0 || 2 * k == N) ? R(0) : (R)(signed_k(k, N) * kscale);
          Z z = f[t][k1];
          f[t][k1] = mk<R>(-sc * z.y, sc * z.x);
        }
      }
      if (c == 0) PC::inverse(f, da, xb, tw, p, 0xffffffffu);
      else PC::inverse(f, db, xb, tw, p, 0xffffffffu);
    }
    double kin = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const double ar = a[m].x, ai = a[m].y, br = b[m].x, bi = b[m].y;
      const double d0r = da[m].x, d0i = da[m].y, d1r = db[m].x, d1i = db[m].y;
      const double dd = d0r * d0r + d0i * d0i + d1r * d1r + d1i * d1i;
      kin += dd;
      if (want_fields) {
        // Im(d0 conj(a) + d1 conj(b)), Im(d0 conj(a) - d1 conj(b)), ...
        const double im_d0a = d0i * ar - d0r * ai, im_d1b = d1i * br - d1r * bi;
        const double im_d1a = d1i * ar - d1r * ai, im_d0b = d0i * br - d0r * bi;
        const double re_d1a = d1r * ar + d1i * ai, re_d0b = d0r * br + d0i * bi;
        if (AXIS == 2) {
          const double aa = ar * ar + ai * ai, bb = br * br + bi * bi;
          acc[0][m] += w * (aa + bb);
          acc[1][m] += 0.5 * wu * (aa + bb);
          acc[2][m] += 2.0 * w * (ar * br + ai * bi);     // Re(conj(a) b)
          acc[3][m] += 2.0 * w * (ar * bi - ai * br);     // Im(conj(a) b)
          acc[4][m] += w * (aa - bb);
          acc[5][m] += w * dd;
          acc[6][m] += w * (im_d0a + im_d1b);
          acc[7][m] += w * (re_d1a - re_d0b);             // J_x, z part (densities.py:308-311)
          acc[8][m] += w * (im_d1a + im_d0b);             // J_y, z part (312-315)
        } else if (AXIS == 1) {
          acc[0][m] += w * dd;
          acc[1][m] += w * (im_d0a + im_d1b);
          acc[2][m] += w * (im_d0a - im_d1b);             // J_x, y part (289-292)
          acc[3][m] += -w * (im_d1a + im_d0b);            // J_z, y part (293-296)
        } else {
          // Re(a conj(d1) - b conj(d0)) = Re(d1 conj(a)) - Re(d0 conj(b))
          acc[0][m] += w * dd;
          acc[1][m] += w * (im_d0a + im_d1b);
          acc[2][m] += -w * (im_d0a - im_d1b);            // J_y, x part (270-273)
          acc[3][m] += -w * (re_d1a - re_d0b);            // J_z, x part (274-277)
        }
      }
    }
    kin += nyq_fac * knyq;
    if (!active) kin = 0.0;
    if (kin_part) {
      // per-warp partials, summed in a fixed order by kinetic_reduce_kernel
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) kin += __shfl_xor_sync(0xffffffffu, kin, o);
      if ((threadIdx.x & 31) == 0)
        kin_part[((size_t)s * G::NTILE + tile) * G::WARPS + threadIdx.x / 32] = kin;
    }
  }
  if (want_fields && active) {
    double* dst = part + (size_t)blockIdx.y * NF * N3;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int m = 0; m < M; ++m) dst[(size_t)f * N3 + base + (size_t)(p + P * m) * stride] = acc[f][m];
  }
}

// Sum the per-chunk partials of the three axis kernels into the reference's
// density arrays; rho, tau, chi are mixed as mix*new + (1-mix)*old.
__global__ void density_combine_kernel(size_t n3, int nchunk, const double* pz, const double* py, const double* px,
                                       double mix, double* rho, double* chi, double* tau, double* cur, double* sd,
                                       double* so) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int iq = blockIdx.y;
  if (i >= n3) return;
  double f9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double fy[4] = {0, 0, 0, 0}, fx[4] = {0, 0, 0, 0};
  for (int c = 0; c < nchunk; ++c) {
    const size_t b = (size_t)(iq * nchunk + c);
    for (int f = 0; f < 9; ++f) f9[f] += pz[(b * 9 + f) * n3 + i];
    for (int f = 0; f < 4; ++f) {
      fy[f] += py[(b * 4 + f) * n3 + i];
      fx[f] += px[(b * 4 + f) * n3 + i];
    }
  }
  const double tnew = f9[5] + fy[0] + fx[0];
  const size_t o = (size_t)iq * n3 + i;
  if (mix < 1.0) {
    rho[o] = mix * f9[0] + (1.0 - mix) * rho[o];
    chi[o] = mix * f9[1] + (1.0 - mix) * chi[o];
    tau[o] = mix * tnew + (1.0 - mix) * tau[o];
  } else {
    rho[o] = f9[0];
    chi[o] = f9[1];
    tau[o] = tnew;
  }
  const size_t v = (size_t)iq * 3 * n3 + i;
  sd[v] = f9[2];
  sd[v + n3] = f9[3];
  sd[v + 2 * n3] = f9[4];
  cur[v] = fx[1];
  cur[v + n3] = fy[1];
  cur[v + 2 * n3] = f9[6];
  so[v] = fy[2] + f9[7];
  so[v + n3] = fx[2] + f9[8];
  so[v + 2 * n3] = fx[3] + fy[3];
}

// sp_kinetic[s] = wxyz h2m_q sum over axes, tiles and warps (``np`` partials
// per state and axis); one warp per state, lanes over strided partials, then
// a fixed shuffle tree.
__global__ void kinetic_reduce_kernel(int nst, int nneut, int np, const double* kz, const double* ky,
                                      const double* kx, double wxyz, double h2m_n, double h2m_p, double* out) {
  const int s = blockIdx.x, lane = threadIdx.x;
  if (s >= nst) return;
  double t = 0;
  for (int j = lane; j < np; j += 32)
    t += kx[(size_t)s * np + j] + ky[(size_t)s * np + j] + kz[(size_t)s * np + j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) out[s] = wxyz * (s >= nneut ? h2m_p : h2m_n) * t;
}

template <class R, int N>
int density_launch_t(hfb_ctx_s* c, int nst, int nneut, const void* psi, const double* wocc, const double* wguv,
                     const double* pairwg, const double* wstates, double mix, double* rho, double* chi, double* tau,
                     double* cur, double* sd, double* so, const double* h2m, double* sp_kinetic, cudaStream_t st) {
  using G = DensGeo<R, N>;
  using Z = cplx<R>;
  constexpr size_t N3 = (size_t)N * N * N;
  const bool fields = rho != nullptr;
  const int nq = 2;
  int nchunk = (2 * 148 + 2 * G::NTILE - 1) / (2 * G::NTILE);
  if (nchunk < 1) nchunk = 1;
  if (nchunk > 8) nchunk = 8;
  const int nb = nq * nchunk;
  double* part = nullptr;
  if (fields) {
    part = (double*)scratch(c, hfb_ctx_s::S_DENS, sizeof(double) * (size_t)nb * 17 * N3);
    if (!part) return HFB_ERR_ALLOC;
  }
  double* kin = nullptr;
  if (sp_kinetic) {
    kin = (double*)scratch(c, hfb_ctx_s::S_RED, sizeof(double) * (size_t)3 * nst * G::NTILE * G::WARPS);
    if (!kin) return HFB_ERR_ALLOC;
  }
  double* pz = part;
  double* py = part ? part + (size_t)nb * 9 * N3 : nullptr;
  double* px = part ? py + (size_t)nb * 4 * N3 : nullptr;
  double* kz = kin;
  double* ky = kin ? kin + (size_t)nst * G::NTILE * G::WARPS : nullptr;
  double* kx = kin ? kin + (size_t)2 * nst * G::NTILE * G::WARPS : nullptr;
  dim3 grid(G::NTILE, nb);
  const double ks[3] = {2.0 * kPi / (c->d[0] * N) / N, 2.0 * kPi / (c->d[1] * N) / N, 2.0 * kPi / (c->d[2] * N) / N};
  double nf[3];
  for (int a = 0; a < 3; ++a) nf[a] = (kPi / c->d[a]) * (kPi / c->d[a]) / N;
  density_axis_kernel<R, N, 2><<<grid, G::THREADS, 0, st>>>((const Z*)psi, nst, nneut, nchunk, wocc, wguv, pairwg,
                                                            wstates, ks[2], nf[2], fields, pz, kz);
  HFB_CHECK_LAUNCH();
  density_axis_kernel<R, N, 1><<<grid, G::THREADS, 0, st>>>((const Z*)psi, nst, nneut, nchunk, wocc, wguv, pairwg,
                                                            wstates, ks[1], nf[1], fields, py, ky);
  HFB_CHECK_LAUNCH();
  density_axis_kernel<R, N, 0><<<grid, G::THREADS, 0, st>>>((const Z*)psi, nst, nneut, nchunk, wocc, wguv, pairwg,
                                                            wstates, ks[0], nf[0], fields, px, kx);
  HFB_CHECK_LAUNCH();
  if (fields) {
    dim3 g2((unsigned)((N3 + 255) / 256), 2);
    density_combine_kernel<<<g2, 256, 0, st>>>(N3, nchunk, pz, py, px, mix, rho, chi, tau, cur, sd, so);
    HFB_CHECK_LAUNCH();
  }
  if (sp_kinetic) {
    kinetic_reduce_kernel<<<nst, 32, 0, st>>>(nst, nneut, G::NTILE * G::WARPS, kz, ky, kx, c->wxyz, h2m[0], h2m[1],
                                              sp_kinetic);
    HFB_CHECK_LAUNCH();
  }
  return HFB_OK;
}

int density_launch(hfb_ctx_s* c, int prec, int nst, int nneut, const void* psi, const double* wocc,
                   const double* wguv, const double* pairwg, const double* wstates, double mix, double* rho,
                   double* chi, double* tau, double* cur, double* sd, double* so, const double* h2m,
                   double* sp_kinetic, cudaStream_t st) {
  return dispatch_n(c->n, [&](auto nn) -> int {
    constexpr int N = decltype(nn)::value;
    if (prec == HFB_F64)
      return density_launch_t<double, N>(c, nst, nneut, psi, wocc, wguv, pairwg, wstates, mix, rho, chi, tau, cur, sd,
                                         so, h2m, sp_kinetic, st);
    return density_launch_t<float, N>(c, nst, nneut, psi, wocc, wguv, pairwg, wstates, mix, rho, chi, tau, cur, sd, so,
                                      h2m, sp_kinetic, st);
  });
}

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_add_density(hfb_ctx_t ctx, int prec, int nst, int nneut, const void* psi, const double* wocc,
                               const double* wguv, const double* pairwg, const double* wstates, double mix,
                               double* rho, double* chi, double* tau, double* current, double* sdens, double* sodens,
                               const double* h2m, double* sp_kinetic, void* stream) {
  if (!ctx || !psi || !wocc || !wguv || !pairwg || !wstates || !rho || !chi || !tau || !current || !sdens || !sodens)
    return HFB_ERR_ARG;
  if (sp_kinetic && !h2m) return HFB_ERR_ARG;
  if (nst <= 0) return HFB_ERR_ARG;
  return density_launch(ctx, prec, nst, nneut, psi, wocc, wguv, pairwg, wstates, mix, rho, chi, tau, current, sdens,
                        sodens, h2m, sp_kinetic, as_stream(stream));
}

extern "C" int hfb_sp_kinetic(hfb_ctx_t ctx, int prec, int nst, int nneut, const void* psi, const double* h2m,
                              double* sp_kinetic, void* stream) {
  if (!ctx || !psi || !h2m || !sp_kinetic || nst <= 0) return HFB_ERR_ARG;
  // weights are not read when no fields are accumulated
  return density_launch(ctx, prec, nst, nneut, psi, nullptr, nullptr, nullptr, nullptr, 1.0, nullptr, nullptr, nullptr,
                        nullptr, nullptr, nullptr, h2m, sp_kinetic, as_stream(stream));
}
