// Single-particle Hamiltonian h_q on 2-spinors: hpsi01 of meanfield.py:41-159.
//
// Per state the work splits into three independent line passes (x, y, z):
// along axis d the reference computes
//     cderv d02(psi, B) -> (d1, d(B d1))          (4 1-D FFT passes)
//     pout += coef(aq, wl) * d1 - d(B d1)
//     pout += cderv d00(pswk2(aq, wl, psi))       (2 passes)
// and every term only involves lines along d.  By linearity
//     -d(B d1) + d00(pswk2) = D_d(pswk2 - B d1)
// where D_d multiplies bin k by i k kfac / n and puts the cderv02 Nyquist
// value (pi/d)^2 * mean_d(B) * psi_hat(n/2) / n into bin n/2 (levels.py:314-315
// with the sign of the subtraction).  So one axis costs 2 forward + 2 inverse
// line FFTs (12 per spinor component instead of 18).
//
// Kernel A (one CTA per (state, x-plane)): stages psi(x0, :, :) for both
// spinor components in shared memory, runs the z lines (plus the local
// upot / spin-current terms) and then the y lines, accumulating pout_mf in
// global memory (L2-resident between the passes).
// Kernel B (one CTA per (state, y-plane)): x lines, then the final weights
// pout = weight * h psi - weightuv * v_pair psi, pout_del = v_pair psi, and
// optional per-plane overlaps <psi|h psi>, <psi|pout> for the gradient step.
#include "hfb_ctx.cuh"
#include "hpsi.cuh"

namespace hfb {

template <class R, int N>
struct HpsiGeo {
  static constexpr int P = PencilSplit<R, N>::P;
  static constexpr int M = N / P;
  static constexpr int T = (M + P - 1) / P;
  static constexpr int LD = N + 4;                   // shared row stride (elements)
  static constexpr int NB = N + 4;                   // exchange buffer per line
  static constexpr int THREADS = ((N * P + 31) / 32) * 32;
  static constexpr int LINES = THREADS / P;          // >= N (extra lines are idle)
  static constexpr size_t SMEM = sizeof(cplx<R>) * (size_t)(2 * N * LD + LINES * NB + N);
};

// One axis pass over one line of a staged plane.  ``plane`` is [2][N][LD]
// (component, a, b); row lines run along b, column lines along a.  Returns
// the contribution to pout (both components) at the lane's M points
// (positions j = p + P m along the line).
template <class R, int N, int AXIS, bool ROW, bool LOCAL>
__device__ __forceinline__ void hpsi_line(const cplx<R>* plane, cplx<R>* xb, const cplx<R>* tw, int line, int p,
                                          const R* pot, size_t base, size_t sa, size_t sb, double kscale,
                                          double nyq_scale, cplx<R> (&out0)[HpsiGeo<R, N>::M],
                                          cplx<R> (&out1)[HpsiGeo<R, N>::M]) {
  using G = HpsiGeo<R, N>;
  using PC = Pencil<R, N, G::P>;
  using Z = cplx<R>;
  constexpr int M = G::M, T = G::T, P = G::P;
  constexpr size_t N3 = (size_t)N * N * N;
  const unsigned mask = 0xffffffffu;
  auto sidx = [&](int c, int j) -> int {
    return ROW ? (c * N + line) * G::LD + j : (c * N + j) * G::LD + line;
  };
  auto gidx = [&](int j) -> size_t { return ROW ? base + (size_t)line * sa + (size_t)j * sb : base + (size_t)j * sa + (size_t)line * sb; };

  Z d1[2][M];
  Z nyq[2];
  // ---- d1 = D psi (first derivative, k = 0 and Nyquist zeroed)
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    Z v[M];
    Z f[T][P];
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = plane[sidx(c, p + P * m)];
    PC::forward(v, f, xb, tw, p, mask);
    nyq[c] = f[0][P / 2];
#pragma unroll
    for (int t = 0; t < T; ++t) {
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) {
        int k = PC::freq(p, t, k1);
        int kk = signed_k(k, N);
        R s = (k == 0 || 2 * k == N) ? R(0) : (R)(kk * kscale);
        Z z = f[t][k1];
        f[t][k1] = mk<R>(-s * z.y, s * z.x);
      }
    }
    PC::inverse(f, d1[c], xb, tw, p, mask);
  }
  // ---- pointwise terms; d1 is replaced by w = pswk2 - B d1
  R bsum = 0;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int j = p + P * m;
    const size_t g = gidx(j);
    const Z a0 = plane[sidx(0, j)], a1 = plane[sidx(1, j)];
    const R bm = pot[1 * N3 + g];
    const R aqd = pot[(3 + AXIS) * N3 + g];
    const R w0 = pot[9 * N3 + g], w1 = pot[10 * N3 + g], w2 = pot[11 * N3 + g];
    const R h = R(0.5);
    Z o0, o1;
    if (LOCAL) {
      const R up = pot[g], s0 = pot[6 * N3 + g], s1 = pot[7 * N3 + g], s2 = pot[8 * N3 + g];
      // upot psi + sigma.spot psi (meanfield.py:47-58)
      o0 = (up + s2) * a0 + cmulri(s0, -s1, a1);
      o1 = (up - s2) * a1 + cmulri(s0, s1, a0);
    } else {
      o0 = czero<Z>();
      o1 = czero<Z>();
    }
    Z e0 = d1[0][m], e1 = d1[1][m];
    Z n0, n1;
    if (AXIS == 0) {
      // meanfield.py:63-83
      o0 = o0 + cmulri(R(0), -(h * aqd - h * w1), e0) - (h * w2) * e1;
      o1 = o1 + cmulri(R(0), -(h * aqd + h * w1), e1) + (h * w2) * e0;
      n0 = cmulri(R(0), -h * (aqd - w1), a0) - (h * w2) * a1;
      n1 = cmulri(R(0), -h * (aqd + w1), a1) + (h * w2) * a0;
    } else if (AXIS == 1) {
      // meanfield.py:92-112
      o0 = o0 + cmulri(R(0), -(h * aqd + h * w0), e0) + cmulri(R(0), h * w2, e1);
      o1 = o1 + cmulri(R(0), -(h * aqd - h * w0), e1) + cmulri(R(0), h * w2, e0);
      n0 = cmulri(R(0), -h * (aqd + w0), a0) + cmulri(R(0), h * w2, a1);
      n1 = cmulri(R(0), -h * (aqd - w0), a1) + cmulri(R(0), h * w2, a0);
    } else {
      // meanfield.py:121-141
      o0 = o0 + cmulri(R(0), -(h * aqd), e0) + cmulri(h * w0, -(h * w1), e1);
      o1 = o1 + cmulri(R(0), -(h * aqd), e1) + cmulri(-(h * w0), -(h * w1), e0);
      n0 = cmulri(R(0), -h * aqd, a0) + cmulri(h * w0, -(h * w1), a1);
      n1 = cmulri(R(0), -h * aqd, a1) + cmulri(-(h * w0), -(h * w1), a0);
    }
    out0[m] = o0;
    out1[m] = o1;
    d1[0][m] = n0 - bm * e0;
    d1[1][m] = n1 - bm * e1;
    bsum += bm;
  }
#pragma unroll
  for (int o = 1; o < P; o <<= 1) bsum += __shfl_xor_sync(mask, bsum, o);
  const R bbar = bsum / R(N);
  // ---- D_d (pswk2 - B d1) with the cderv02 Nyquist term
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    Z f[T][P];
    Z r[M];
    PC::forward(d1[c], f, xb, tw, p, mask);
#pragma unroll
    for (int t = 0; t < T; ++t) {
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) {
        int k = PC::freq(p, t, k1);
        int kk = signed_k(k, N);
        Z z = f[t][k1];
        if (2 * k == N) {
          R s = (R)nyq_scale * bbar;
          f[t][k1] = s * nyq[c];
        } else {
          R s = (k == 0) ? R(0) : (R)(kk * kscale);
          f[t][k1] = mk<R>(-s * z.y, s * z.x);
        }
      }
    }
    PC::inverse(f, r, xb, tw, p, mask);
    if (c == 0) {
#pragma unroll
      for (int m = 0; m < M; ++m) out0[m] = out0[m] + r[m];
    } else {
#pragma unroll
      for (int m = 0; m < M; ++m) out1[m] = out1[m] + r[m];
    }
  }
}

template <class R, int N>
__global__ void __launch_bounds__(HpsiGeo<R, N>::THREADS)
hpsi_xplane_kernel(const R* __restrict__ pot, const cplx<R>* __restrict__ psi, cplx<R>* acc, int s0, int nneut,
                   double ks_y, double ks_z, double ny_y, double ny_z) {
  using G = HpsiGeo<R, N>;
  using Z = cplx<R>;
  constexpr int P = G::P, M = G::M;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Z* plane = reinterpret_cast<Z*>(smem_raw);
  Z* xball = plane + 2 * N * G::LD;
  Z* tw = xball + G::LINES * G::NB;
  const int x0 = blockIdx.x;
  const int s = s0 + blockIdx.y;
  const int iq = s >= nneut ? 1 : 0;
  const R* potq = pot + (size_t)iq * 12 * N3;
  fill_twiddles<R>(tw, N);
  const Z* src = psi + (size_t)s * 2 * N3 + (size_t)x0 * N2;
  for (int e = threadIdx.x; e < 2 * N * N; e += blockDim.x) {
    int c = e / (N * N), r = e - c * N * N;
    plane[(c * N + r / N) * G::LD + r % N] = src[(size_t)c * N3 + r];
  }
  __syncthreads();
  const int line_raw = threadIdx.x / P, p = threadIdx.x % P;
  const bool active = line_raw < N;
  const int line = active ? line_raw : 0;
  Z* xb = xball + line_raw * G::NB;
  Z* dst = acc + (size_t)s * 2 * N3;
  const size_t base = (size_t)x0 * N2;
  {
    Z o0[M], o1[M];
    hpsi_line<R, N, 2, true, true>(plane, xb, tw, line, p, potq, base, N, 1, ks_z, ny_z, o0, o1);
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) {
        size_t g = base + (size_t)line * N + p + P * m;
        dst[g] = o0[m];
        dst[N3 + g] = o1[m];
      }
    }
  }
  __syncthreads();
  {
    Z o0[M], o1[M];
    hpsi_line<R, N, 1, false, false>(plane, xb, tw, line, p, potq, base, N, 1, ks_y, ny_y, o0, o1);
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) {
        size_t g = base + (size_t)(p + P * m) * N + line;
        dst[g] = dst[g] + o0[m];
        dst[N3 + g] = dst[N3 + g] + o1[m];
      }
    }
  }
}

template <class R, int N>
__global__ void __launch_bounds__(HpsiGeo<R, N>::THREADS)
hpsi_yplane_kernel(const R* __restrict__ pot, const cplx<R>* __restrict__ psi, cplx<R>* acc, int s0, int nneut,
                   double ks_x, double ny_x, const double* __restrict__ weight, const double* __restrict__ weightuv,
                   cplx<R>* pout, cplx<R>* pout_mf, cplx<R>* pout_del, double* ovl) {
  using G = HpsiGeo<R, N>;
  using Z = cplx<R>;
  constexpr int P = G::P, M = G::M;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Z* plane = reinterpret_cast<Z*>(smem_raw);
  Z* xball = plane + 2 * N * G::LD;
  Z* tw = xball + G::LINES * G::NB;
  __shared__ double red[2][32];
  const int y0 = blockIdx.x;
  const int s = s0 + blockIdx.y;
  const int iq = s >= nneut ? 1 : 0;
  const R* potq = pot + (size_t)iq * 12 * N3;
  fill_twiddles<R>(tw, N);
  const Z* src = psi + (size_t)s * 2 * N3 + (size_t)y0 * N;
  // plane (a = x, b = z) at fixed y0
  for (int e = threadIdx.x; e < 2 * N * N; e += blockDim.x) {
    int c = e / (N * N), r = e - c * N * N;
    int a = r / N, b = r % N;
    plane[(c * N + a) * G::LD + b] = src[(size_t)c * N3 + (size_t)a * N2 + b];
  }
  __syncthreads();
  const int line_raw = threadIdx.x / P, p = threadIdx.x % P;
  const bool active = line_raw < N;
  const int line = active ? line_raw : 0;
  Z* xb = xball + line_raw * G::NB;
  const size_t base = (size_t)y0 * N;
  Z o0[M], o1[M];
  hpsi_line<R, N, 0, false, false>(plane, xb, tw, line, p, potq, base, N2, 1, ks_x, ny_x, o0, o1);
  const double wt = weight ? weight[s] : 1.0;
  const double wu = weightuv ? weightuv[s] : 0.0;
  Z* a_s = acc + (size_t)s * 2 * N3;
  double ov_mf = 0.0, ov_po = 0.0;
  if (active) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int a = p + P * m;
      const size_t g = base + (size_t)a * N2 + line;
      const R vp = potq[2 * N3 + g];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const size_t gi = (size_t)c * N3 + g;
        Z mf = a_s[gi] + (c == 0 ? o0[m] : o1[m]);
        Z ps = plane[(c * N + a) * G::LD + line];
        Z dl = vp * ps;
        Z po = (R)wt * mf - (R)wu * dl;
        if (pout_mf) pout_mf[(size_t)s * 2 * N3 + gi] = mf;
        if (pout) pout[(size_t)s * 2 * N3 + gi] = po;
        if (pout_del) pout_del[(size_t)s * 2 * N3 + gi] = dl;
        if (ovl) {
          ov_mf += (double)ps.x * (double)mf.x + (double)ps.y * (double)mf.y;
          ov_po += (double)ps.x * (double)po.x + (double)ps.y * (double)po.y;
        }
      }
    }
  }
  if (ovl) {
    // deterministic block reduction: warp shuffles, then warp 0
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ov_mf += __shfl_xor_sync(0xffffffffu, ov_mf, o);
      ov_po += __shfl_xor_sync(0xffffffffu, ov_po, o);
    }
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) { red[0][w] = ov_mf; red[1][w] = ov_po; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0, b = 0;
      for (int i = 0; i < (int)(blockDim.x / 32); ++i) { a += red[0][i]; b += red[1][i]; }
      ovl[((size_t)blockIdx.y * N + y0) * 2 + 0] = a;
      ovl[((size_t)blockIdx.y * N + y0) * 2 + 1] = b;
    }
  }
}

template <class R, int N>
int hpsi_launch_t(hfb_ctx_s* c, const void* pot, int s0, int ns, int nneut, const void* psi, const double* weight,
                  const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del, double* ovl,
                  cudaStream_t st) {
  using G = HpsiGeo<R, N>;
  using Z = cplx<R>;
  if (ns <= 0) return HFB_OK;
  const double kf[3] = {2.0 * kPi / (c->d[0] * N), 2.0 * kPi / (c->d[1] * N), 2.0 * kPi / (c->d[2] * N)};
  double ks[3], nq[3];
  for (int a = 0; a < 3; ++a) {
    ks[a] = kf[a] / N;
    nq[a] = (kPi / c->d[a]) * (kPi / c->d[a]) / N;
  }
  allow_max_dynamic_smem(hpsi_xplane_kernel<R, N>);
  allow_max_dynamic_smem(hpsi_yplane_kernel<R, N>);
  dim3 grid(N, ns);
  hpsi_xplane_kernel<R, N><<<grid, G::THREADS, G::SMEM, st>>>((const R*)pot, (const Z*)psi, (Z*)acc, s0, nneut, ks[1],
                                                             ks[2], nq[1], nq[2]);
  HFB_CHECK_LAUNCH();
  hpsi_yplane_kernel<R, N><<<grid, G::THREADS, G::SMEM, st>>>((const R*)pot, (const Z*)psi, (Z*)acc, s0, nneut, ks[0],
                                                             nq[0], weight, weightuv, (Z*)pout, (Z*)pout_mf,
                                                             (Z*)pout_del, ovl);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

int hpsi_ovl_parts(hfb_ctx_s* c, int prec) {
  if (hpsi_bf3_available(c, prec)) return hpsi_bf3_parts(c);
  return hpsi_tc_available(c, prec) ? hpsi_tc_parts(c) : c->n;
}

int hpsi_launch(hfb_ctx_s* c, int prec, const void* pot, int s0, int ns, int nneut, const void* psi,
                const double* weight, const double* weightuv, void* acc, void* pout, void* pout_mf, void* pout_del,
                double* ovl, cudaStream_t st) {
  if (hpsi_bf3_available(c, prec))
    return hpsi_bf3_launch(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
  if (hpsi_tc_available(c, prec))
    return hpsi_tc_launch(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
  if (hpsi_dmma_available(c, prec))
    return hpsi_dmma_launch(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
  return dispatch_n(c->n, [&](auto nn) -> int {
    constexpr int N = decltype(nn)::value;
    if (prec == HFB_F64)
      return hpsi_launch_t<double, N>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl,
                                      st);
    return hpsi_launch_t<float, N>(c, pot, s0, ns, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, ovl, st);
  });
}

}  // namespace hfb

extern "C" int hfb_hpsi(hfb_ctx_t ctx, int prec, const void* pot, int nst, int nneut, const void* psi,
                        const double* weight, const double* weightuv, void* pout, void* pout_mf, void* pout_del,
                        void* stream) {
  if (!ctx || !pot || !psi || nst < 0 || (!pout && !pout_mf)) return HFB_ERR_ARG;
  if (prec != HFB_F64 && prec != HFB_F32) return HFB_ERR_ARG;
  // pout_mf doubles as the accumulator; without it the pout buffer is used.
  void* acc = pout_mf ? pout_mf : pout;
  return hfb::hpsi_launch(ctx, prec, pot, 0, nst, nneut, psi, weight, weightuv, acc, pout, pout_mf, pout_del, nullptr,
                          hfb::as_stream(stream));
}
