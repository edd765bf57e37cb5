// Damped-gradient step: grstep / grstep_helper / e0dmp_gt_zero of
// static.py:93-259, and the k-space preconditioner laplace of
// levels.py:398-437.
//
// The preconditioner is a 3-D FFT, a division by
//   (max(wg,.1) (E0 + h2ma k^2) + 0.5 max(wguv,.1) vmax) * Ntot
// and an inverse 3-D FFT.  It runs as three plane kernels:
//   A (x-plane):  v = ps1 - lagrange (or - <h> psi), norms for efluct, z and y
//                 forward line FFTs;
//   B (y-plane):  x forward FFT, divide, x inverse FFT (stays in registers);
//   C (x-plane):  y and z inverse line FFTs, psi -= x0 * result.
#include "hfb_ctx.cuh"
#include "hpsi.cuh"

namespace hfb {

template <class R, int N>
struct PlaneGeo {
  static constexpr int P = PencilSplit<R, N>::P;
  static constexpr int M = N / P;
  static constexpr int T = (M + P - 1) / P;
  static constexpr int LD = N + 4;
  static constexpr int NB = N + 4;
  static constexpr int THREADS = ((N * P + 31) / 32) * 32;
  static constexpr int LINES = THREADS / P;
  static constexpr size_t SMEM = sizeof(cplx<R>) * (size_t)(2 * N * LD + LINES * NB + N);
};

// Forward (DIR = -1) or inverse (+1) transform of every line of one staged
// component ``pl`` ([N][LD]); data stays in natural order in the plane.
template <class R, int N, bool ROW, int DIR>
__device__ __forceinline__ void plane_lines(cplx<R>* pl, cplx<R>* xb, const cplx<R>* tw, int line, int p,
                                            bool active) {
  using G = PlaneGeo<R, N>;
  using PC = Pencil<R, N, G::P>;
  using Z = cplx<R>;
  constexpr int M = G::M, T = G::T, P = G::P;
  auto at = [&](int j) -> Z& { return ROW ? pl[line * G::LD + j] : pl[j * G::LD + line]; };
  Z v[M];
  Z f[T][P];
  if (DIR < 0) {
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = at(p + P * m);
    PC::forward(v, f, xb, tw, p, 0xffffffffu);
    if (active) {
#pragma unroll
      for (int t = 0; t < T; ++t)
        if (PC::valid(p, t)) {
#pragma unroll
          for (int k1 = 0; k1 < P; ++k1) at(PC::freq(p, t, k1)) = f[t][k1];
        }
    }
  } else {
#pragma unroll
    for (int t = 0; t < T; ++t) {
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) f[t][k1] = PC::valid(p, t) ? at(PC::freq(p, t, k1)) : czero<Z>();
    }
    PC::inverse(f, v, xb, tw, p, 0xffffffffu);
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) at(p + P * m) = v[m];
    }
  }
}

template <class R>
__device__ __forceinline__ void block_sum2(double& a, double& b, double (*red)[32]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) { red[0][w] = a; red[1][w] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0, y = 0;
    for (int i = 0; i < (int)(blockDim.x / 32); ++i) { x += red[0][i]; y += red[1][i]; }
    a = x;
    b = y;
  }
}

// A: x-plane, build v and transform along z and y.
template <class R, int N>
__global__ void __launch_bounds__(PlaneGeo<R, N>::THREADS)
precond_a_kernel(const cplx<R>* __restrict__ src, const cplx<R>* __restrict__ lag, int use_lag,
                 const cplx<R>* __restrict__ psi, const double* __restrict__ coef, cplx<R>* tmp, double* fluct) {
  using G = PlaneGeo<R, N>;
  using Z = cplx<R>;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[2][32];
  Z* plane = reinterpret_cast<Z*>(smem_raw);
  Z* xball = plane + 2 * N * G::LD;
  Z* tw = xball + G::LINES * G::NB;
  const int x0 = blockIdx.x, s = blockIdx.y;
  fill_twiddles<R>(tw, N);
  const size_t off = (size_t)s * 2 * N3 + (size_t)x0 * N2;
  const R cf = coef ? (R)coef[s] : R(0);
  double n1 = 0, n2 = 0;
  for (int e = threadIdx.x; e < 2 * N * N; e += G::THREADS) {
    int c = e / (N * N), r = e - c * N * N;
    size_t g = off + (size_t)c * N3 + r;
    Z v = src[g];
    if (psi) {
      Z ps = psi[g];
      Z lg = lag ? lag[g] : czero<Z>();
      Z hp = cf * ps;
      v = use_lag ? v - lg : v - hp;
      if (fluct) {
        Z e2 = lg - hp;
        n1 += (double)v.x * v.x + (double)v.y * v.y;
        n2 += (double)e2.x * e2.x + (double)e2.y * e2.y;
      }
    }
    plane[(c * N + r / N) * G::LD + r % N] = v;
  }
  if (fluct) {
    block_sum2<R>(n1, n2, red);
    if (threadIdx.x == 0) {
      fluct[((size_t)s * N + x0) * 2 + 0] = n1;
      fluct[((size_t)s * N + x0) * 2 + 1] = n2;
    }
  }
  __syncthreads();
  const int line_raw = threadIdx.x / G::P, p = threadIdx.x % G::P;
  const bool active = line_raw < N;
  const int line = active ? line_raw : 0;
  Z* xb = xball + line_raw * G::NB;
  for (int c = 0; c < 2; ++c) plane_lines<R, N, true, -1>(plane + c * N * G::LD, xb, tw, line, p, active);
  __syncthreads();
  for (int c = 0; c < 2; ++c) plane_lines<R, N, false, -1>(plane + c * N * G::LD, xb, tw, line, p, active);
  __syncthreads();
  for (int e = threadIdx.x; e < 2 * N * N; e += G::THREADS) {
    int c = e / (N * N), r = e - c * N * N;
    tmp[off + (size_t)c * N3 + r] = plane[(c * N + r / N) * G::LD + r % N];
  }
}

// B: y-plane (fixed ky), transform along x, divide, transform back.
template <class R, int N>
__global__ void __launch_bounds__(PlaneGeo<R, N>::THREADS)
precond_b_kernel(cplx<R>* tmp, int nneut, const double* __restrict__ wg, const double* __restrict__ wu,
                 const double* __restrict__ vmax_dev, double vmax_host, double e0, double h2ma, double kfx, double kfy,
                 double kfz) {
  using G = PlaneGeo<R, N>;
  using PC = Pencil<R, N, G::P>;
  using Z = cplx<R>;
  constexpr int M = G::M, T = G::T, P = G::P;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Z* plane = reinterpret_cast<Z*>(smem_raw);
  Z* xball = plane + 2 * N * G::LD;
  Z* tw = xball + G::LINES * G::NB;
  const int y0 = blockIdx.x, s = blockIdx.y;
  const int iq = s >= nneut ? 1 : 0;
  fill_twiddles<R>(tw, N);
  const size_t off = (size_t)s * 2 * N3 + (size_t)y0 * N;
  // compile-time trip count, unrolled: several loads in flight per thread
#pragma unroll 8
  for (int e = threadIdx.x; e < 2 * N * N; e += G::THREADS) {
    int c = e / (N * N), r = e - c * N * N;
    int a = r / N, b = r % N;
    plane[(c * N + a) * G::LD + b] = tmp[off + (size_t)c * N3 + (size_t)a * N2 + b];
  }
  __syncthreads();
  const int line_raw = threadIdx.x / P, p = threadIdx.x % P;
  const bool active = line_raw < N;
  const int line = active ? line_raw : 0;  // line = kz
  Z* xb = xball + line_raw * G::NB;
  const double wgm = fmax(wg ? wg[s] : 1.0, 0.1);
  const double wum = fmax(wu ? wu[s] : 0.0, 0.1);
  const double vm = vmax_dev ? vmax_dev[iq] : vmax_host;
  const int kyi = signed_k(y0, N), kzi = signed_k(line, N);
  const double kyz2 = (kyi * kfy) * (kyi * kfy) + (kzi * kfz) * (kzi * kfz);
  const double shift = wgm * e0 + 0.5 * wum * vm;
  for (int c = 0; c < 2; ++c) {
    Z* pl = plane + c * N * G::LD;
    Z v[M];
    Z f[T][P];
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = pl[(p + P * m) * G::LD + line];
    PC::forward(v, f, xb, tw, p, 0xffffffffu);
#pragma unroll
    for (int t = 0; t < T; ++t) {
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) {
        int kxi = signed_k(PC::freq(p, t, k1), N);
        double k2 = (kxi * kfx) * (kxi * kfx) + kyz2;
        double den = (shift + wgm * h2ma * k2) * (double)N3;
        f[t][k1] = (R)(1.0 / den) * f[t][k1];
      }
    }
    PC::inverse(f, v, xb, tw, p, 0xffffffffu);
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) pl[(p + P * m) * G::LD + line] = v[m];
    }
  }
  __syncthreads();
  // compile-time trip count, unrolled: several loads in flight per thread
#pragma unroll 8
  for (int e = threadIdx.x; e < 2 * N * N; e += G::THREADS) {
    int c = e / (N * N), r = e - c * N * N;
    int a = r / N, b = r % N;
    tmp[off + (size_t)c * N3 + (size_t)a * N2 + b] = plane[(c * N + a) * G::LD + b];
  }
}

// C: x-plane, inverse along y and z, then write or update.
template <class R, int N>
__global__ void __launch_bounds__(PlaneGeo<R, N>::THREADS)
precond_c_kernel(const cplx<R>* tmp, int mode, double x0, const double* x0_dev, cplx<R>* dst) {
  using G = PlaneGeo<R, N>;
  using Z = cplx<R>;
  constexpr size_t N2 = (size_t)N * N, N3 = N2 * N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Z* plane = reinterpret_cast<Z*>(smem_raw);
  Z* xball = plane + 2 * N * G::LD;
  Z* tw = xball + G::LINES * G::NB;
  const int xp = blockIdx.x, s = blockIdx.y;
  fill_twiddles<R>(tw, N);
  const size_t off = (size_t)s * 2 * N3 + (size_t)xp * N2;
  // compile-time trip count, unrolled: several loads in flight per thread
#pragma unroll 8
  for (int e = threadIdx.x; e < 2 * N * N; e += G::THREADS) {
    int c = e / (N * N), r = e - c * N * N;
    plane[(c * N + r / N) * G::LD + r % N] = tmp[off + (size_t)c * N3 + r];
  }
  __syncthreads();
  const int line_raw = threadIdx.x / G::P, p = threadIdx.x % G::P;
  const bool active = line_raw < N;
  const int line = active ? line_raw : 0;
  Z* xb = xball + line_raw * G::NB;
  for (int c = 0; c < 2; ++c) plane_lines<R, N, false, +1>(plane + c * N * G::LD, xb, tw, line, p, active);
  __syncthreads();
  for (int c = 0; c < 2; ++c) plane_lines<R, N, true, +1>(plane + c * N * G::LD, xb, tw, line, p, active);
  __syncthreads();
  const R xr = (R)(x0_dev ? *x0_dev : x0);
  // compile-time trip count, unrolled: several loads in flight per thread
#pragma unroll 8
  for (int e = threadIdx.x; e < 2 * N * N; e += G::THREADS) {
    int c = e / (N * N), r = e - c * N * N;
    size_t g = off + (size_t)c * N3 + r;
    Z v = plane[(c * N + r / N) * G::LD + r % N];
    if (mode == 0) dst[g] = v;
    else dst[g] = dst[g] - xr * v;
  }
}

template <class R, int N>
int precond_launch_t(hfb_ctx_s* c, int ns, int nneut, const void* src, const void* lag, int use_lag, const void* psi,
                     const double* coef, const double* wg, const double* wu, const double* vmax_dev, double vmax_host,
                     double e0, double h2ma, int mode, double x0, void* tmp, void* dst, double* fluct,
                     cudaStream_t st, const double* x0_dev) {
  using G = PlaneGeo<R, N>;
  using Z = cplx<R>;
  if (ns <= 0) return HFB_OK;
  allow_max_dynamic_smem(precond_a_kernel<R, N>);
  allow_max_dynamic_smem(precond_b_kernel<R, N>);
  allow_max_dynamic_smem(precond_c_kernel<R, N>);
  dim3 grid(N, ns);
  precond_a_kernel<R, N><<<grid, G::THREADS, G::SMEM, st>>>((const Z*)src, (const Z*)lag, use_lag, (const Z*)psi,
                                                            coef, (Z*)tmp, fluct);
  HFB_CHECK_LAUNCH();
  const double kf[3] = {2.0 * kPi / (c->d[0] * N), 2.0 * kPi / (c->d[1] * N), 2.0 * kPi / (c->d[2] * N)};
  precond_b_kernel<R, N><<<grid, G::THREADS, G::SMEM, st>>>((Z*)tmp, nneut, wg, wu, vmax_dev, vmax_host, e0, h2ma,
                                                            kf[0], kf[1], kf[2]);
  HFB_CHECK_LAUNCH();
  precond_c_kernel<R, N><<<grid, G::THREADS, G::SMEM, st>>>((const Z*)tmp, mode, x0, x0_dev, (Z*)dst);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

int precond_launch(hfb_ctx_s* c, int prec, int ns, int nneut, const void* src, const void* lag, int use_lag,
                   const void* psi, const double* coef, const double* wg, const double* wu, const double* vmax_dev,
                   double vmax_host, double e0, double h2ma, int mode, double x0, void* tmp, void* dst,
                   double* fluct, cudaStream_t st, const double* x0_dev) {
  return dispatch_n(c->n, [&](auto nn) -> int {
    constexpr int N = decltype(nn)::value;
    if (prec == HFB_F64)
      return precond_launch_t<double, N>(c, ns, nneut, src, lag, use_lag, psi, coef, wg, wu, vmax_dev, vmax_host, e0,
                                         h2ma, mode, x0, tmp, dst, fluct, st, x0_dev);
    return precond_launch_t<float, N>(c, ns, nneut, src, lag, use_lag, psi, coef, wg, wu, vmax_dev, vmax_host, e0,
                                      h2ma, mode, x0, tmp, dst, fluct, st, x0_dev);
  });
}

// ------------------------------------------------------ gradient-step glue --
// Per-state weights (static.py:152-170, 125-136): hpsi weights and the
// preconditioner weights.
__global__ void grstep_weights_kernel(int ns, int tbcs, const double* wocc, const double* wguv, const double* pairwg,
                                      const double* wstates, double* wt, double* wu, double* lw, double* lu) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  if (tbcs) {
    wt[s] = 1.0; wu[s] = 0.0; lw[s] = 1.0; lu[s] = 0.0;
  } else {
    wt[s] = wstates[s] * wocc[s];
    wu[s] = wstates[s] * wguv[s] * pairwg[s];
    lw[s] = wocc[s];
    lu[s] = wguv[s] * pairwg[s];
  }
}

// max(v_pair[iq]) over the grid, one block per isospin (order-independent).
__global__ void vpair_max_kernel(const double* v_pair, size_t n3, int zero, double* vmax) {
  __shared__ double red[32];
  const int iq = blockIdx.x;
  double m = -1.0e300;
  if (!zero)
    for (size_t i = threadIdx.x; i < n3; i += blockDim.x) m = fmax(m, v_pair[iq * n3 + i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int i = 1; i < (int)(blockDim.x / 32); ++i) r = fmax(r, red[i]);
    vmax[iq] = zero ? 0.0 : r;
  }
}

// Per-state sums of plane partials: out[s] = scale * sum_j part[s][j][k].
__global__ void state_reduce_kernel(int ns, int nplanes, const double* part, int k, double scale, double* out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  double a = 0;
  for (int j = 0; j < nplanes; ++j) a += part[((size_t)s * nplanes + j) * 2 + k];
  out[s] = scale * a;
}

// Simple damped step when e0dmp <= 0 (static.py:181-185).
template <class R>
__global__ void simple_step_kernel(int ns, size_t n3, const double* spe_new, const double* spe_old, double x0h,
                                   const double* x0_dev, const cplx<R>* ps1, cplx<R>* psi) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t tot = (size_t)ns * 2 * n3;
  if (i >= tot) return;
  const double x0 = x0_dev ? *x0_dev : x0h;
  int s = (int)(i / (2 * n3));
  R a = (R)(1.0 + x0 * (spe_new[s] - spe_old[s]));
  psi[i] = a * psi[i] - (R)x0 * ps1[i];
}

// Finalise efluct, denerg and the running sums (static.py:110-111, 211, 251-257).
// One block; deterministic sequential sums.
__global__ void grstep_finish_kernel(int ns, int do_fluct, int nplanes, const double* fl, double wxyz,
                                     const double* spe_new, const double* wocc, const double* wstates,
                                     double* sp_energy, double* ef1, double* ef2, double* sums) {
  for (int s = threadIdx.x; s < ns; s += blockDim.x) {
    if (do_fluct) {
      double a = 0, b = 0;
      for (int j = 0; j < nplanes; ++j) {
        a += fl[((size_t)s * nplanes + j) * 2 + 0];
        b += fl[((size_t)s * nplanes + j) * 2 + 1];
      }
      ef1[s] = sqrt(wxyz * a);
      ef2[s] = sqrt(wxyz * b);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sf = 0, sd = 0;
    for (int s = 0; s < ns; ++s) {
      double den = (sp_energy[s] - spe_new[s]) / fabs(spe_new[s]);
      sf += ef1[s];
      sd += wocc[s] * wstates[s] * den;
    }
    sums[0] = sf;
    sums[1] = sd;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < ns; s += blockDim.x) sp_energy[s] = spe_new[s];
}

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_laplace(hfb_ctx_t ctx, int prec, int nsp, const void* psin, const double* wg, const double* wguv,
                           double v_pairmax, double e0inv, double h2ma, void* psout, void* stream) {
  if (!ctx || !psin || !psout || nsp < 0) return HFB_ERR_ARG;
  return precond_launch(ctx, prec, nsp, 1 << 30, psin, nullptr, 0, nullptr, nullptr, wg, wguv, nullptr, v_pairmax,
                        e0inv, h2ma, 0, 0.0, psout, psout, nullptr, as_stream(stream));
}

extern "C" int hfb_grstep(hfb_ctx_t ctx, int prec, const hfb_grstep_args* a, void* stream) {
  if (!ctx || !a || !a->psi || !a->hampsi || !a->hmfpsi || !a->pot || !a->sp_energy) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const int ns = a->nst, n = ctx->n;
  if (ns <= 0) return HFB_OK;
  const size_t n3 = (size_t)n * n * n;
  const int nov = hpsi_ovl_parts(ctx, prec);
  double* part = (double*)scratch(ctx, hfb_ctx_s::S_PART, sizeof(double) * (size_t)ns * (nov + n) * 2);
  double* vec = (double*)scratch(ctx, hfb_ctx_s::S_SMALL, sizeof(double) * ((size_t)ns * 6 + 8));
  if (!part || !vec) return HFB_ERR_ALLOC;
  double* ovl = part;
  double* fl = part + (size_t)ns * nov * 2;
  double *wt = vec, *wu = vec + ns, *lw = vec + 2 * ns, *lu = vec + 3 * ns, *spe_new = vec + 4 * ns,
         *hexp = vec + 5 * ns, *vmax = vec + 6 * ns;
  grstep_weights_kernel<<<(ns + 127) / 128, 128, 0, st>>>(ns, a->tbcs, a->wocc, a->wguv, a->pairwg, a->wstates, wt,
                                                           wu, lw, lu);
  HFB_CHECK_LAUNCH();
  vpair_max_kernel<<<2, 256, 0, st>>>(a->v_pair, n3, a->tbcs || !a->v_pair, vmax);
  HFB_CHECK_LAUNCH();
  // 1) h psi_old: ps1 (weighted) into hmfpsi (scratch), h psi into hampsi
  int r = hpsi_launch(ctx, prec, a->pot, 0, ns, a->nneut, a->psi, wt, wu, a->hampsi, a->hmfpsi, a->hampsi, nullptr,
                      ovl, st);
  if (r) return r;
  state_reduce_kernel<<<(ns + 127) / 128, 128, 0, st>>>(ns, nov, ovl, 0, a->wxyz, spe_new);
  HFB_CHECK_LAUNCH();
  state_reduce_kernel<<<(ns + 127) / 128, 128, 0, st>>>(ns, nov, ovl, 1, a->wxyz, hexp);
  HFB_CHECK_LAUNCH();
  // 2) damped step
  if (a->e0dmp > 0.0) {
    r = precond_launch(ctx, prec, ns, a->nneut, a->hmfpsi, a->lagrange, a->use_lagrange, a->psi, hexp, lw, lu, vmax,
                       0.0, a->e0dmp, a->h2ma, 1, a->x0dmp, a->hmfpsi, a->psi, a->do_fluct ? fl : nullptr, st,
                       a->x0dmp_dev);
    if (r) return r;
  } else {
    size_t tot = (size_t)ns * 2 * n3;
    if (prec == HFB_F64)
      simple_step_kernel<double><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(
          ns, n3, spe_new, a->sp_energy, a->x0dmp, a->x0dmp_dev, (const double2*)a->hmfpsi, (double2*)a->psi);
    else
      simple_step_kernel<float><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(
          ns, n3, spe_new, a->sp_energy, a->x0dmp, a->x0dmp_dev, (const float2*)a->hmfpsi, (float2*)a->psi);
    HFB_CHECK_LAUNCH();
  }
  grstep_finish_kernel<<<1, 256, 0, st>>>(ns, a->do_fluct && a->e0dmp > 0.0, n, fl, a->wxyz, spe_new, a->wocc,
                                          a->wstates, a->sp_energy, a->sp_efluct1, a->sp_efluct2, a->sums);
  HFB_CHECK_LAUNCH();
  // 3) h psi_new into hmfpsi (and v_pair psi_new into delpsi when requested)
  return hpsi_launch(ctx, prec, a->pot, 0, ns, a->nneut, a->psi, wt, wu, a->hmfpsi, nullptr, a->hmfpsi, a->delpsi,
                     nullptr, st);
}
