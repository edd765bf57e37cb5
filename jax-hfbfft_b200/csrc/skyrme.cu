// Mean fields from densities (skyrme, meanfield.py:164-391) and the Coulomb
// potential by FFT on the doubled grid (coulomb.py:14-75).  All FP64.
//
// Derivatives of densities use the dense spectral matrices der1/der2 along
// each axis exactly as the reference's einsums do (an O(n^4) matrix apply;
// small next to the per-state work).  A "job" writes
//     out = sum_t coef_t * D_t applied along axis_t to in_t      (t < 3)
// so divergences, curls and Laplacians are single jobs and one launch runs
// many jobs without write conflicts.
#include <mutex>
#include "hfb_ctx.cuh"

namespace hfb {

struct DerivJob {
  const double* in[3];
  double coef[3];
  int axis[3];
  int der[3];   // 1 or 2
  int nterm;
  double* out;
};
constexpr int kMaxJobs = 24;
struct DerivJobs {
  DerivJob j[kMaxJobs];
};

// Term t of every job as dense line transforms on shared-memory tiles: a
// block stages one plane of the input (the x-plane for y and z lines, the
// y-plane for x lines: n lines of n points) and the n x n derivative matrix,
// and each thread forms 4 x 4 outputs (4 lines x 4 derivative points).
// Term 0 writes coef * D f, later terms add to it (fixed order).
constexpr int kDerivMaxN = 48;

__global__ void __launch_bounds__(144)
deriv_pass_kernel(DerivJobs jobs, int t, int n, const double* d1x, const double* d1y, const double* d1z,
                  const double* d2x, const double* d2y, const double* d2z) {
  __shared__ double F[kDerivMaxN][kDerivMaxN + 1];   // [line][point along the axis]
  __shared__ double Dm[kDerivMaxN][kDerivMaxN + 1];  // [output point][input point]
  const DerivJob& jb = jobs.j[blockIdx.y];
  if (t >= jb.nterm) return;
  const int ax = jb.axis[t];
  const double* D = jb.der[t] == 1 ? (ax == 0 ? d1x : ax == 1 ? d1y : d1z) : (ax == 0 ? d2x : ax == 1 ? d2y : d2z);
  const double* f = jb.in[t];
  const double coef = jb.coef[t];
  const size_t n2 = (size_t)n * n;
  const int tile = blockIdx.x;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, q = e % n;   // q runs over the contiguous index
    Dm[r][q] = D[e];
    if (ax == 2) F[r][q] = f[tile * n2 + (size_t)r * n + q];          // line y = r, point z = q
    else if (ax == 1) F[q][r] = f[tile * n2 + (size_t)r * n + q];     // line z = q, point y = r
    else F[q][r] = f[(size_t)r * n2 + (size_t)tile * n + q];          // line z = q, point x = r
  }
  __syncthreads();
  const int g = n / 4, nthr = g * g;
  if ((int)threadIdx.x >= nthr) return;
  // consecutive threads run along the output's contiguous index
  const int tfast = threadIdx.x % g, tslow = threadIdx.x / g;
  const int tl = ax == 2 ? tslow : tfast, tk = ax == 2 ? tfast : tslow;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int l = 0; l < n; ++l) {
    double fv[4], dv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) fv[i] = F[tl + g * i][l];
#pragma unroll
    for (int j = 0; j < 4; ++j) dv[j] = Dm[tk + g * j][l];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] += dv[j] * fv[i];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int line = tl + g * i, k = tk + g * j;
      size_t o;
      if (ax == 2) o = tile * n2 + (size_t)line * n + k;
      else if (ax == 1) o = tile * n2 + (size_t)k * n + line;
      else o = (size_t)k * n2 + (size_t)tile * n + line;
      const double v = coef * acc[i][j];
      jb.out[o] = t == 0 ? v : jb.out[o] + v;
    }
}

static int run_jobs(hfb_ctx_s* c, DerivJobs& jobs, int nj, cudaStream_t st) {
  if (nj <= 0) return HFB_OK;
  if (c->n > kDerivMaxN || c->n % 4 != 0) return HFB_ERR_UNSUPPORTED_GRID;
  int tmax = 0;
  for (int q = 0; q < nj; ++q) tmax = jobs.j[q].nterm > tmax ? jobs.j[q].nterm : tmax;
  dim3 grid((unsigned)c->n, nj);
  for (int t = 0; t < tmax; ++t) {
    deriv_pass_kernel<<<grid, 144, 0, st>>>(jobs, t, c->n, c->der1[0], c->der1[1], c->der1[2], c->der2[0],
                                            c->der2[1], c->der2[2]);
    HFB_CHECK_LAUNCH();
  }
  return HFB_OK;
}

static DerivJob job1(const double* in, int axis, int der, double* out) {
  DerivJob j{};
  j.in[0] = in; j.coef[0] = 1.0; j.axis[0] = axis; j.der[0] = der; j.nterm = 1; j.out = out;
  return j;
}
static DerivJob jobdiv(const double* vx, const double* vy, const double* vz, double* out) {
  DerivJob j{};
  const double* v[3] = {vx, vy, vz};
  for (int t = 0; t < 3; ++t) { j.in[t] = v[t]; j.coef[t] = 1.0; j.axis[t] = t; j.der[t] = 1; }
  j.nterm = 3; j.out = out;
  return j;
}
static DerivJob joblap(const double* f, double* out) {
  DerivJob j{};
  for (int t = 0; t < 3; ++t) { j.in[t] = f; j.coef[t] = 1.0; j.axis[t] = t; j.der[t] = 2; }
  j.nterm = 3; j.out = out;
  return j;
}
// component k of curl v: d_a v_b - d_b v_a with (a, b) = (y, z), (z, x), (x, y)
static DerivJob jobcurl(const double* v /*[3][n3]*/, size_t n3, int k, double* out) {
  static const int A[3] = {1, 2, 0}, B[3] = {2, 0, 1};
  DerivJob j{};
  j.in[0] = v + (size_t)B[k] * n3; j.coef[0] = 1.0; j.axis[0] = A[k]; j.der[0] = 1;
  j.in[1] = v + (size_t)A[k] * n3; j.coef[1] = -1.0; j.axis[1] = B[k]; j.der[1] = 1;
  j.nterm = 2; j.out = out;
  return j;
}

// Derivative fields of the densities kept in scratch S_DERIV, per isospin:
//   [0] div J   [1] lap rho   [2..4] grad rho   [5..7] curl s   [8..10] curl j
constexpr int kNDeriv = 11;

int density_derivatives(hfb_ctx_s* c, const double* rho, const double* cur, const double* sd, const double* so,
                        bool need_grad_curls, double** dv_out, cudaStream_t st) {
  const size_t n3 = (size_t)c->n * c->n * c->n;
  double* dv = (double*)scratch(c, hfb_ctx_s::S_DERIV, sizeof(double) * (size_t)2 * kNDeriv * n3);
  if (!dv) return HFB_ERR_ALLOC;
  *dv_out = dv;
  DerivJobs jobs;
  int nj = 0;
  for (int iq = 0; iq < 2; ++iq) {
    double* o = dv + (size_t)iq * kNDeriv * n3;
    const double* s3 = so + (size_t)iq * 3 * n3;
    const double* r = rho + (size_t)iq * n3;
    jobs.j[nj++] = jobdiv(s3, s3 + n3, s3 + 2 * n3, o);
    jobs.j[nj++] = joblap(r, o + n3);
    for (int k = 0; k < 3; ++k) {
      if (need_grad_curls) {
        jobs.j[nj++] = job1(r, k, 1, o + (2 + k) * n3);
        jobs.j[nj++] = jobcurl(sd + (size_t)iq * 3 * n3, n3, k, o + (5 + k) * n3);
      }
      jobs.j[nj++] = jobcurl(cur + (size_t)iq * 3 * n3, n3, k, o + (8 + k) * n3);
    }
  }
  return run_jobs(c, jobs, nj, st);
}

// ------------------------------------------------------ doubled-grid FFT --
// In-place line FFT along one axis of a complex n2^3 array, for lines whose
// two transverse indices lie below (lim_u, lim_v) (the zero-padded Poisson
// solve only needs part of the lines).  Lines are ordered with the
// contiguous transverse index fastest.
template <int N2> struct CoulGeo { static constexpr int THREADS = N2 >= 80 ? 128 : 256; };

template <int N2, int AXIS, int DIR>
__global__ void __launch_bounds__(CoulGeo<N2>::THREADS) coul_fft_kernel(double2* a, int lim_u, int lim_v) {
  constexpr int P = PencilSplit<double, N2>::P;
  constexpr int M = N2 / P, T = (M + P - 1) / P, L = CoulGeo<N2>::THREADS / P, NB = N2 + 4;
  using PC = Pencil<double, N2, P>;
  __shared__ __align__(16) double2 xball[L * NB];
  __shared__ double2 tw[N2];
  fill_twiddles<double>(tw, N2);
  __syncthreads();
  const int lg = threadIdx.x / P, p = threadIdx.x % P;
  const long line_raw = (long)blockIdx.x * L + lg;
  const bool active = line_raw < (long)lim_u * lim_v;
  const long line = active ? line_raw : 0;
  const int u = (int)(line / lim_v), v = (int)(line % lim_v);
  constexpr size_t S2 = (size_t)N2 * N2;
  size_t base, stride;
  if (AXIS == 2) { base = (size_t)u * S2 + (size_t)v * N2; stride = 1; }
  else if (AXIS == 1) { base = (size_t)u * S2 + v; stride = N2; }
  else { base = (size_t)u * N2 + v; stride = S2; }
  double2* xb = xball + lg * NB;
  double2 vv[M];
  double2 f[T][P];
  if (DIR < 0) {
#pragma unroll
    for (int m = 0; m < M; ++m) vv[m] = a[base + (size_t)(p + P * m) * stride];
    PC::forward(vv, f, xb, tw, p, 0xffffffffu);
    if (active) {
#pragma unroll
      for (int t = 0; t < T; ++t)
        if (PC::valid(p, t)) {
#pragma unroll
          for (int k1 = 0; k1 < P; ++k1) a[base + (size_t)PC::freq(p, t, k1) * stride] = f[t][k1];
        }
    }
  } else {
#pragma unroll
    for (int t = 0; t < T; ++t)
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1)
        f[t][k1] = PC::valid(p, t) ? a[base + (size_t)PC::freq(p, t, k1) * stride] : make_double2(0.0, 0.0);
    PC::inverse(f, vv, xb, tw, p, 0xffffffffu);
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) a[base + (size_t)(p + P * m) * stride] = vv[m];
    }
  }
}

template <int N2, int AXIS, int DIR>
static int coul_pass(double2* a, int lim_u, int lim_v, cudaStream_t st) {
  constexpr int P = PencilSplit<double, N2>::P;
  constexpr int L = CoulGeo<N2>::THREADS / P;
  long lines = (long)lim_u * lim_v;
  coul_fft_kernel<N2, AXIS, DIR><<<(unsigned)((lines + L - 1) / L), CoulGeo<N2>::THREADS, 0, st>>>(a, lim_u, lim_v);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

template <int N2, int DIR>
static int coul_fft3(double2* a, int n, bool pruned, cudaStream_t st) {
  // forward: z lines for x,y < n; y lines for x < n; x lines everywhere.
  // inverse: x lines everywhere; y lines for x < n; z lines for x,y < n.
  const int lim = pruned ? n : N2;
  int r;
  if (DIR < 0) {
    if ((r = coul_pass<N2, 2, -1>(a, lim, lim, st))) return r;
    if ((r = coul_pass<N2, 1, -1>(a, lim, N2, st))) return r;
    if ((r = coul_pass<N2, 0, -1>(a, N2, N2, st))) return r;
  } else {
    if ((r = coul_pass<N2, 0, +1>(a, N2, N2, st))) return r;
    if ((r = coul_pass<N2, 1, +1>(a, lim, N2, st))) return r;
    if ((r = coul_pass<N2, 2, +1>(a, lim, lim, st))) return r;
  }
  return HFB_OK;
}

template <class F>
static int dispatch_n2(int n2, F&& fn) {
  switch (n2) {
    case 8: return fn(std::integral_constant<int, 8>{});
    case 16: return fn(std::integral_constant<int, 16>{});
    case 24: return fn(std::integral_constant<int, 24>{});
    case 32: return fn(std::integral_constant<int, 32>{});
    case 40: return fn(std::integral_constant<int, 40>{});
    case 48: return fn(std::integral_constant<int, 48>{});
    case 64: return fn(std::integral_constant<int, 64>{});
    case 80: return fn(std::integral_constant<int, 80>{});
    case 96: return fn(std::integral_constant<int, 96>{});
    default: return HFB_ERR_UNSUPPORTED_GRID;
  }
}

// q(r) on the doubled grid (coulomb.py:31-47): 1/|r| with wrapped indices,
// the r = 0 cell 2.84 / dV^(1/3); periodic: 1/k^2 with q(0) = 0.
__global__ void coul_green_kernel(double2* q, int n2, double dx, double dy, double dz, int periodic) {
  const size_t tot = (size_t)n2 * n2 * n2;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= tot) return;
  int ix = (int)(i / ((size_t)n2 * n2)), iy = (int)((i / n2) % n2), iz = (int)(i % n2);
  ix = ix <= n2 / 2 ? ix : ix - n2;
  iy = iy <= n2 / 2 ? iy : iy - n2;
  iz = iz <= n2 / 2 ? iz : iz - n2;
  double v;
  if (periodic) {
    const double kx = 2.0 * kPi * ix / (n2 * dx), ky = 2.0 * kPi * iy / (n2 * dy), kz = 2.0 * kPi * iz / (n2 * dz);
    const double s = kx * kx + ky * ky + kz * kz;
    v = (i == 0) ? 0.0 : 1.0 / s;
  } else {
    const double s = (dx * ix) * (dx * ix) + (dy * iy) * (dy * iy) + (dz * iz) * (dz * iz);
    v = (i == 0) ? 2.84 / cbrt(dx * dy * dz) : 1.0 / sqrt(s);
  }
  q[i] = make_double2(v, 0.0);
}

int coulomb_init(hfb_ctx_s* c) {
  const size_t tot = (size_t)c->n2 * c->n2 * c->n2;
  coul_green_kernel<<<(unsigned)((tot + 255) / 256), 256>>>(c->coul_q, c->n2, c->d[0], c->d[1], c->d[2], c->periodic);
  HFB_CHECK_LAUNCH();
  if (c->periodic) return HFB_OK;
  return dispatch_n2(c->n2, [&](auto nn) -> int {
    constexpr int N2 = decltype(nn)::value;
    return coul_fft3<N2, -1>(c->coul_q, c->n, false, 0);
  });
}

__global__ void pois_load_kernel(double2* a, int n, int n2, const double* rho_p) {
  const size_t tot = (size_t)n2 * n2 * n2;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= tot) return;
  int x = (int)(i / ((size_t)n2 * n2)), y = (int)((i / n2) % n2), z = (int)(i % n2);
  double v = 0.0;
  if (x < n && y < n && z < n) v = rho_p[((size_t)x * n + y) * n + z];
  a[i] = make_double2(v, 0.0);
}

__global__ void pois_mul_kernel(double2* a, const double2* q, size_t tot, double fac, int periodic) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= tot) return;
  double2 v = a[i], g = q[i];
  if (periodic) a[i] = make_double2(fac * g.x * v.x, fac * g.x * v.y);
  else a[i] = make_double2(fac * (g.x * v.x - g.y * v.y), fac * (g.x * v.y + g.y * v.x));
}

__global__ void pois_store_kernel(const double2* a, int n, int n2, double scale, double* w) {
  const size_t tot = (size_t)n * n * n;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= tot) return;
  int x = (int)(i / ((size_t)n * n)), y = (int)((i / n) % n), z = (int)(i % n);
  w[i] = scale * a[((size_t)x * n2 + y) * n2 + z].x;
}

// The doubled-grid solve on the work buffer ``a`` (n2^3 complex doubles;
// every element is rewritten, so it may hold anything on entry).
static int poisson_solve(const hfb_ctx_s* c, const double* rho_p, double* wcoul, double2* a, cudaStream_t st) {
  const int n = c->n, n2 = c->n2;
  const size_t tot = (size_t)n2 * n2 * n2;
  pois_load_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(a, n, n2, rho_p);
  HFB_CHECK_LAUNCH();
  const bool pruned = !c->periodic;
  int r = dispatch_n2(n2, [&](auto nn) -> int {
    constexpr int N2 = decltype(nn)::value;
    return coul_fft3<N2, -1>(a, n, pruned, st);
  });
  if (r) return r;
  // coulomb.py:68-71: periodic 4 pi e2 Re(q); else e2 wxyz q
  const double e2 = 1.4399784085965135;
  const double fac = c->periodic ? 4.0 * kPi * e2 : e2 * c->wxyz;
  pois_mul_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(a, c->coul_q, tot, fac, c->periodic);
  HFB_CHECK_LAUNCH();
  r = dispatch_n2(n2, [&](auto nn) -> int {
    constexpr int N2 = decltype(nn)::value;
    return coul_fft3<N2, +1>(a, n, pruned, st);
  });
  if (r) return r;
  const size_t t3 = (size_t)n * n * n;
  pois_store_kernel<<<(unsigned)((t3 + 255) / 256), 256, 0, st>>>(a, n, n2, 1.0 / (double)tot, wcoul);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

int poisson_launch(hfb_ctx_s* c, const double* rho_p, double* wcoul, cudaStream_t st) {
  const size_t tot = (size_t)c->n2 * c->n2 * c->n2;
  double2* a = (double2*)scratch(c, hfb_ctx_s::S_POIS, tot * sizeof(double2));
  if (!a) return HFB_ERR_ALLOC;
  return poisson_solve(c, rho_p, wcoul, a, st);
}

// ----------------------------------------------------- potential assembly --
// Steps 1-10 and 13 of skyrme (meanfield.py:176-385) at one grid point.
__global__ void skyrme_assemble_kernel(hfb_force f, int tcoul, size_t n3, const double* rho, const double* tau,
                                       const double* chi, const double* cur, const double* dv, const double* wcoul,
                                       double* upot, double* bmass, double* v_pair, double* aq, double* spot,
                                       double* wlspot, double* rearr_out) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n3) return;
  const double r0 = rho[i], r1 = rho[n3 + i];
  const double rt = r0 + r1;
  const double rtp = pow(rt, f.power);
  const double* d0 = dv;
  const double* d1 = dv + (size_t)kNDeriv * n3;
  double rearr = 0.0;
  if (f.ipair == 6)
    rearr = (f.v0neut / f.rho0pr) * chi[i] * chi[i] + (f.v0prot / f.rho0pr) * chi[n3 + i] * chi[n3 + i];
  for (int iq = 0; iq < 2; ++iq) {
    const int ic = 1 - iq;
    const double* dq = iq == 0 ? d0 : d1;
    const double* dc = iq == 0 ? d1 : d0;
    const double rq = rho[iq * n3 + i], rc = rho[ic * n3 + i];
    double u = rtp * ((f.b3 * (f.power + 2.0) / 3.0 - 2.0 * f.b3p / 3.0) * rq + f.b3 * (f.power + 2.0) / 3.0 * rc -
                      (f.b3p * f.power / 3.0) * (r0 * r0 + r1 * r1) / (rt + 1.0e-25));
    u += -(f.b4 + f.b4p) * dq[i] - f.b4 * dc[i];
    if (tcoul && iq == 1) {
      u += wcoul[i];
      if (f.ex != 0) u += -f.slate * cbrt(r1);
    }
    u += (f.b0 - f.b0p) * rq + f.b0 * rc + (f.b1 - f.b1p) * tau[iq * n3 + i] + f.b1 * tau[ic * n3 + i] -
         (f.b2 - f.b2p) * dq[n3 + i] - f.b2 * dc[n3 + i];
    u += rearr;
    upot[iq * n3 + i] = u;
    bmass[iq * n3 + i] = f.h2m[iq] + (f.b1 - f.b1p) * rq + f.b1 * rc;
    for (int k = 0; k < 3; ++k) {
      const size_t o = ((size_t)iq * 3 + k) * n3 + i;
      wlspot[o] = (f.b4 + f.b4p) * dq[(2 + k) * n3 + i] + f.b4 * dc[(2 + k) * n3 + i];
      aq[o] = -2.0 * (f.b1 - f.b1p) * cur[((size_t)iq * 3 + k) * n3 + i] -
              2.0 * f.b1 * cur[((size_t)ic * 3 + k) * n3 + i] - (f.b4 + f.b4p) * dq[(5 + k) * n3 + i] -
              f.b4 * dc[(5 + k) * n3 + i];
      spot[o] = -(f.b4 + f.b4p) * dq[(8 + k) * n3 + i] - f.b4 * dc[(8 + k) * n3 + i];
    }
    const double v0 = iq == 1 ? f.v0prot : f.v0neut;
    v_pair[iq * n3 + i] = f.ipair == 6 ? v0 * chi[iq * n3 + i] * (1.0 - rt / f.rho0pr) : v0 * chi[iq * n3 + i];
  }
  if (rearr_out) rearr_out[i] = rt * rearr;
}

// ecorrp = -sum(rho_tot * rearr) * wxyz / 2 (meanfield.py:364), one block.
__global__ void ecorrp_kernel(size_t n3, const double* t, double wxyz, int ipair, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  if (ipair == 6)
    for (size_t i = threadIdx.x; i < n3; i += blockDim.x) s += t[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) a += red[k];
    out[0] = ipair == 6 ? -a * wxyz / 2.0 : 0.0;
  }
}

// pot[iq][field][i] in precision R: upot, bmass, v_pair, aq, spot, wlspot.
template <class R>
__global__ void pack_pot_kernel(size_t n3, const double* upot, const double* bmass, const double* v_pair,
                                const double* aq, const double* spot, const double* wlspot, R* pot) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n3) return;
  for (int iq = 0; iq < 2; ++iq) {
    R* o = pot + (size_t)iq * 12 * n3;
    o[i] = (R)upot[iq * n3 + i];
    o[n3 + i] = (R)bmass[iq * n3 + i];
    o[2 * n3 + i] = (R)v_pair[iq * n3 + i];
    for (int k = 0; k < 3; ++k) {
      o[(3 + k) * n3 + i] = (R)aq[((size_t)iq * 3 + k) * n3 + i];
      o[(6 + k) * n3 + i] = (R)spot[((size_t)iq * 3 + k) * n3 + i];
      o[(9 + k) * n3 + i] = (R)wlspot[((size_t)iq * 3 + k) * n3 + i];
    }
  }
}

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_poisson(hfb_ctx_t ctx, const double* rho_p, double* wcoul, void* stream) {
  if (!ctx || !rho_p || !wcoul) return HFB_ERR_ARG;
  return poisson_launch(ctx, rho_p, wcoul, as_stream(stream));
}

extern "C" int hfb_skyrme(hfb_ctx_t ctx, const hfb_force* f, int tcoul, const double* rho, const double* tau,
                          const double* chi, const double* current, const double* sdens, const double* sodens,
                          double* upot, double* bmass, double* divaq, double* v_pair, double* aq, double* spot,
                          double* wlspot, double* dbmass, double* wcoul, double* ecorrp, int prec, void* pot,
                          void* stream) {
  if (!ctx || !f || !rho || !tau || !chi || !current || !sdens || !sodens || !upot || !bmass || !divaq || !v_pair ||
      !aq || !spot || !wlspot || !dbmass || !ecorrp)
    return HFB_ERR_ARG;
  if (tcoul && !wcoul) return HFB_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  double* dv = nullptr;
  // the Coulomb solve needs rho_p only: on the side stream, beside the
  // derivatives of the densities
  const bool fork = tcoul && ctx->side;
  int r;
  if (fork) {
    cudaEventRecord(ctx->ev_fork, st);
    cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0);
    r = poisson_launch(ctx, rho + n3, wcoul, ctx->side);
    if (r) return r;
    cudaEventRecord(ctx->ev_join, ctx->side);
  }
  r = density_derivatives(ctx, rho, current, sdens, sodens, true, &dv, st);
  if (r) return r;
  if (fork) {
    cudaStreamWaitEvent(st, ctx->ev_join, 0);
  } else if (tcoul) {
    r = poisson_launch(ctx, rho + n3, wcoul, st);
    if (r) return r;
  }
  double* tmp = (double*)scratch(ctx, hfb_ctx_s::S_MAT, sizeof(double) * n3);
  if (!tmp) return HFB_ERR_ALLOC;
  skyrme_assemble_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(*f, tcoul, n3, rho, tau, chi, current, dv,
                                                                      wcoul, upot, bmass, v_pair, aq, spot, wlspot,
                                                                      tmp);
  HFB_CHECK_LAUNCH();
  ecorrp_kernel<<<1, 1024, 0, st>>>(n3, tmp, ctx->wxyz, f->ipair, ecorrp);
  HFB_CHECK_LAUNCH();
  // steps 11-12: div aq and grad bmass
  DerivJobs jobs;
  int nj = 0;
  for (int iq = 0; iq < 2; ++iq) {
    const double* a = aq + (size_t)iq * 3 * n3;
    jobs.j[nj++] = jobdiv(a, a + n3, a + 2 * n3, divaq + (size_t)iq * n3);
    for (int k = 0; k < 3; ++k) jobs.j[nj++] = job1(bmass + (size_t)iq * n3, k, 1, dbmass + ((size_t)iq * 3 + k) * n3);
  }
  r = run_jobs(ctx, jobs, nj, st);
  if (r) return r;
  if (pot) {
    if (prec == HFB_F64)
      pack_pot_kernel<double><<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(n3, upot, bmass, v_pair, aq, spot, wlspot,
                                                                           (double*)pot);
    else
      pack_pot_kernel<float><<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(n3, upot, bmass, v_pair, aq, spot, wlspot,
                                                                          (float*)pot);
    HFB_CHECK_LAUNCH();
  }
  return HFB_OK;
}

// --------------------------------------------- Poisson without allocation --
// A second entry point for the Coulomb solve, for callers that cannot let
// the library allocate device memory when they call it: applications whose
// device memory is entirely owned by their own pool allocator (a cudaMalloc
// behind its back can fail or fragment the pool), and latency-critical loops
// where an allocation, with the synchronisation it implies, would stall.
// Its work buffer is a fixed array in the library's device image instead of
// the context's growable scratch arena.
namespace hfb {

// Doubled-grid work buffer: 64^3 complex doubles (4 MiB).  The Coulomb grid
// n2 (2n non-periodic, n periodic) must be at most 64: n <= 32 for a
// non-periodic grid; every periodic grid a context accepts (n <= 48) fits.
// Every GPU that loads the library holds it until the process exits.
constexpr int kNoAllocN2 = 64;
static __device__ __align__(256) double2 g_poisson_noalloc[(size_t)kNoAllocN2 * kNoAllocN2 * kNoAllocN2];

// Device address of g_poisson_noalloc per device ordinal, looked up on the
// first call made on that device (the array's host-side name is only a
// stand-in and must never be passed to a kernel).
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[64] = {nullptr};

static int noalloc_buffer(int dev, double2** out) {
  if (dev < 0 || dev >= 64) return HFB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_poisson_noalloc) != cudaSuccess || !p) {
      cudaGetLastError();
      return HFB_ERR_CUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = (double2*)g_noalloc_addr[dev];
  return HFB_OK;
}

}  // namespace hfb

extern "C" int hfb_poisson_noalloc(hfb_ctx_t ctx, const double* rho_p, double* wcoul, void* stream) {
  using namespace hfb;
  if (!ctx || !rho_p || !wcoul) return HFB_ERR_ARG;
  if (ctx->n2 > kNoAllocN2) return HFB_ERR_UNSUPPORTED_GRID;   // work buffer too small for this grid
  // the buffer is looked up on the current device; the context's Green's
  // function lives on the device it was created on: they must be the same
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return HFB_ERR_CUDA;
  }
  if (dev != ctx->device) return HFB_ERR_ARG;
  double2* a = nullptr;
  const int r = noalloc_buffer(dev, &a);
  if (r) return r;
  // the solve rewrites every element of the n2^3 region, padding zeros
  // included, so nothing left by an earlier call leaks into this one
  return poisson_solve(ctx, rho_p, wcoul, a, as_stream(stream));
}
