// Configuration-space sub-iterations: hfb_natural (static.py:920-1070).
//
// For one isospin block of nst states, with h = hmatrix[iq], gap =
// gapmatrix[iq] as they were at entry, the sub-iterations update a unitary
// nst x nst transformation cm (start I):
//   cm[j][:] -= damp_j symcond[j][:]                  (static.py:952-957)
//   cm <- Q of the QR factorisation of cm             (959-960)
//   htran = cm^H h cm, gaptran = cm^H gap cm, hcm = h cm, gcm = gap cm
//   sp_energy <- Re diag(htran), deltaf <- Re diag(gaptran) pairwg (with
//     pairing, else on the last sub-iteration only)  (972-992)
//   [the host runs the BCS solver here when pairing is on]
//   symcond[:, j] <- wt_j hcm[:, j] - wu_j gcm[:, j] - (cm lambda)[:, j]
//     with lambda = (lt + lt^H)/2, lt[:, j] = wt_j htran[:, j] - wu_j
//     gaptran[:, j] (1030-1046), between sub-iterations (994-1015)
// and at the end rotate the states, psi <- psi cm, set the Lagrange fields
// to psi cm htran (the reference passes htran there, 1018), hmatrix <-
// htran, gapmatrix <- gaptran, lambda_save <- lambda (1021-1026).
// damp_j = delstepbas / (e_j - e_first + e0bas), or delstepbas / (max e -
// min e) for all j when e0bas = 0 (932-943).
//
// The QR factorisation follows LAPACK's Householder conventions (zgeqr2:
// beta = -sign(Re alpha) |(alpha, x)|, tau = (beta - alpha) / beta, v = x /
// (alpha - beta); zung2r forms Q = H_1 H_2 ... H_n), which numpy's and
// JAX's CPU qr use, so Q carries the same column phases.  It runs in one
// CTA (nst <= 256) on the matrix in global memory, one warp per column of
// the trailing update; the products are the library's small complex GEMMs.
// The work matrices stay in the context between the calls of one sequence
// (begin, step / symcond per sub-iteration, end); sequences on one context
// must not interleave.
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {

int zgemm_small_one(int n, int ld, int ta, int tb, const double2* A, const double2* B, double2* C,
                    cudaStream_t st);   // diag.cu
int rotate_launch(hfb_ctx_s* c, int prec, int s0, int ns, const void* psi, const double2* U, const double2* L, int ld,
                  void* out1, void* out2, cudaStream_t st, int pre);   // diag.cu

namespace {

constexpr int kNatMax = 256;
constexpr int kQrThreads = 256;

// Work matrices [nst][nst]: cm, h0, g0, htran, gaptran, hcm, gcm, lam, cml;
// vectors: damp [nst], tau [nst] complex
struct NatWork {
  double2 *cm, *h0, *g0, *ht, *gt, *hcm, *gcm, *lam, *cml, *tau;
  double* damp;
};

NatWork nat_work(hfb_ctx_s* c, int nst) {
  const size_t m = (size_t)nst * nst;
  NatWork w{};
  char* p = (char*)scratch(c, hfb_ctx_s::S_NAT, sizeof(double2) * (9 * m + nst) + sizeof(double) * nst);
  if (!p) return w;
  double2* z = (double2*)p;
  w.cm = z;
  w.h0 = z + m;
  w.g0 = z + 2 * m;
  w.ht = z + 3 * m;
  w.gt = z + 4 * m;
  w.hcm = z + 5 * m;
  w.gcm = z + 6 * m;
  w.lam = z + 7 * m;
  w.cml = z + 8 * m;
  w.tau = z + 9 * m;
  w.damp = (double*)(z + 9 * m + nst);
  return w;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {   // conj(a) b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {    // a / b, Smith's method
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const double r = b.x / b.y, d = b.y + b.x * r;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

// cm = I, h0 / g0 = the block's h and gap matrices, damping per state
__global__ void nat_begin_kernel(int nst, int ld, const double2* __restrict__ h, const double2* __restrict__ g,
                                 const double* __restrict__ spe, double delstepbas, double e0bas, NatWork w) {
  __shared__ double red[2][kQrThreads];
  const int t = threadIdx.x;
  for (int e = t; e < nst * nst; e += blockDim.x) {
    const int i = e / nst, j = e % nst;
    w.cm[e] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    w.h0[e] = h[(size_t)i * ld + j];
    w.g0[e] = g[(size_t)i * ld + j];
  }
  double mx = -INFINITY, mn = INFINITY;
  for (int j = t; j < nst; j += blockDim.x) {
    mx = fmax(mx, spe[j]);
    mn = fmin(mn, spe[j]);
  }
  red[0][t] = mx;
  red[1][t] = mn;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) {
      red[0][t] = fmax(red[0][t], red[0][t + s]);
      red[1][t] = fmin(red[1][t], red[1][t + s]);
    }
    __syncthreads();
  }
  for (int j = t; j < nst; j += blockDim.x)
    w.damp[j] = e0bas == 0.0 ? delstepbas / (red[0][0] - red[1][0]) : delstepbas / (spe[j] - spe[0] + e0bas);
}

// cm[j][:] -= damp_j symcond[j][:]
__global__ void nat_gradient_kernel(int nst, int ld, const double2* __restrict__ sym, NatWork w) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nst * nst) return;
  const int i = e / nst, j = e % nst;
  const double2 s = sym[(size_t)i * ld + j];
  const double d = w.damp[i];
  w.cm[e] = make_double2(w.cm[e].x - d * s.x, w.cm[e].y - d * s.y);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// A (n x n, row-major, leading dimension n) <- Q of its QR factorisation
__global__ void __launch_bounds__(kQrThreads) nat_qr_kernel(int n, double2* A, double2* tau) {
  __shared__ double red[kQrThreads / 32];
  __shared__ double2 scal;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31, nw = kQrThreads / 32;
  // zgeqr2
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int r = i + 1 + t; r < n; r += kQrThreads) {
      const double2 x = A[(size_t)r * n + i];
      s += x.x * x.x + x.y * x.y;
    }
    s = warp_sum(s);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (t == 0) {
      double xn2 = 0.0;
      for (int q = 0; q < nw; ++q) xn2 += red[q];
      const double2 alpha = A[(size_t)i * n + i];
      if (xn2 == 0.0 && alpha.y == 0.0) {
        tau[i] = make_double2(0.0, 0.0);
        scal = make_double2(1.0, 0.0);
      } else {
        const double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
        tau[i] = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
        scal = cdiv(make_double2(1.0, 0.0), make_double2(alpha.x - beta, alpha.y));
        A[(size_t)i * n + i] = make_double2(beta, 0.0);
      }
    }
    __syncthreads();
    const double2 sc = scal;
    for (int r = i + 1 + t; r < n; r += kQrThreads) A[(size_t)r * n + i] = cmul(A[(size_t)r * n + i], sc);
    __syncthreads();
    // A[i:, j] -= conj(tau) v (v^H A[i:, j]), j > i, v = (1, A[i+1:, i])
    const double2 tc = make_double2(tau[i].x, -tau[i].y);
    for (int j = i + 1 + warp; j < n; j += nw) {
      double2 d = make_double2(0.0, 0.0);
      for (int r = i + lane; r < n; r += 32) {
        const double2 v = r == i ? make_double2(1.0, 0.0) : A[(size_t)r * n + i];
        const double2 p = cmulc(v, A[(size_t)r * n + j]);
        d.x += p.x;
        d.y += p.y;
      }
      d.x = warp_sum(d.x);
      d.y = warp_sum(d.y);
      const double2 f = cmul(tc, d);
      for (int r = i + lane; r < n; r += 32) {
        const double2 v = r == i ? make_double2(1.0, 0.0) : A[(size_t)r * n + i];
        const double2 p = cmul(f, v);
        A[(size_t)r * n + j].x -= p.x;
        A[(size_t)r * n + j].y -= p.y;
      }
    }
    __syncthreads();
  }
  // zung2r: Q = H_1 ... H_n, built from the last reflector backwards
  for (int i = n - 1; i >= 0; --i) {
    const double2 ti = tau[i];
    if (i < n - 1) {
      // A[i:, j] -= tau v (v^H A[i:, j]) for j > i, with A[i][i] taken as 1
      for (int j = i + 1 + warp; j < n; j += nw) {
        double2 d = make_double2(0.0, 0.0);
        for (int r = i + lane; r < n; r += 32) {
          const double2 v = r == i ? make_double2(1.0, 0.0) : A[(size_t)r * n + i];
          const double2 p = cmulc(v, A[(size_t)r * n + j]);
          d.x += p.x;
          d.y += p.y;
        }
        d.x = warp_sum(d.x);
        d.y = warp_sum(d.y);
        const double2 f = cmul(ti, d);
        for (int r = i + lane; r < n; r += 32) {
          const double2 v = r == i ? make_double2(1.0, 0.0) : A[(size_t)r * n + i];
          const double2 p = cmul(f, v);
          A[(size_t)r * n + j].x -= p.x;
          A[(size_t)r * n + j].y -= p.y;
        }
      }
      __syncthreads();
      const double2 mt = make_double2(-ti.x, -ti.y);
      for (int r = i + 1 + t; r < n; r += kQrThreads) A[(size_t)r * n + i] = cmul(mt, A[(size_t)r * n + i]);
    }
    __syncthreads();
    if (t == 0) A[(size_t)i * n + i] = make_double2(1.0 - ti.x, -ti.y);
    for (int r = t; r < i; r += kQrThreads) A[(size_t)r * n + i] = make_double2(0.0, 0.0);
    __syncthreads();
  }
}

// sp_energy <- Re diag(htran); with pairing deltaf <- Re diag(gaptran) pairwg
__global__ void nat_diag_kernel(int nst, int ipair, NatWork w, const double* __restrict__ pairwg, double* spe,
                                double* deltaf) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nst) return;
  spe[j] = w.ht[(size_t)j * nst + j].x;
  if (ipair) deltaf[j] = w.gt[(size_t)j * nst + j].x * pairwg[j];
}

// lambda = (lt + lt^H) / 2, lt[:, j] = wt_j htran[:, j] - wu_j gaptran[:, j]
__global__ void nat_lambda_kernel(int nst, NatWork w, const double* __restrict__ wocc, const double* __restrict__ wguv,
                                  const double* __restrict__ pairwg, const double* __restrict__ wstates,
                                  double2* out, int ldo) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nst * nst) return;
  const int i = e / nst, j = e % nst;
  const double wtj = wocc[j] * wstates[j], wuj = wguv[j] * pairwg[j] * wstates[j];
  const double wti = wocc[i] * wstates[i], wui = wguv[i] * pairwg[i] * wstates[i];
  const double2 hij = w.ht[(size_t)i * nst + j], gij = w.gt[(size_t)i * nst + j];
  const double2 hji = w.ht[(size_t)j * nst + i], gji = w.gt[(size_t)j * nst + i];
  const double2 a = make_double2(wtj * hij.x - wuj * gij.x, wtj * hij.y - wuj * gij.y);   // lt[i][j]
  const double2 b = make_double2(wti * hji.x - wui * gji.x, wti * hji.y - wui * gji.y);   // lt[j][i]
  out[(size_t)i * ldo + j] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
}

// symcond[:, j] = wt_j hcm[:, j] - wu_j gcm[:, j] - cml[:, j]
__global__ void nat_symcond_kernel(int nst, int ld, NatWork w, const double* __restrict__ wocc,
                                   const double* __restrict__ wguv, const double* __restrict__ pairwg,
                                   const double* __restrict__ wstates, double2* sym) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nst * nst) return;
  const int i = e / nst, j = e % nst;
  const double wt = wocc[j] * wstates[j], wu = wguv[j] * pairwg[j] * wstates[j];
  const double2 a = w.hcm[e], b = w.gcm[e], c = w.cml[e];
  sym[(size_t)i * ld + j] = make_double2(wt * a.x - wu * b.x - c.x, wt * a.y - wu * b.y - c.y);
}

__global__ void nat_store_kernel(int nst, int ld, const double2* __restrict__ src, double2* dst) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nst * nst) return;
  dst[(size_t)(e / nst) * ld + (e % nst)] = src[e];
}

int nat_check(const hfb_natural_args* a) {
  if (!a || a->nst <= 0 || a->nst > kNatMax || a->ld < a->nst || a->iq < 0 || a->iq > 1 || a->start < 0)
    return HFB_ERR_ARG;
  if (!a->hmatrix || !a->gapmatrix || !a->symcond || !a->lambda_save || !a->sp_energy || !a->wocc || !a->wguv ||
      !a->pairwg || !a->wstates)
    return HFB_ERR_ARG;
  if (a->ipair && !a->deltaf) return HFB_ERR_ARG;
  return HFB_OK;
}

inline const double2* mat(const double* m, const hfb_natural_args* a) {
  return (const double2*)m + (size_t)a->iq * a->ld * a->ld;
}
inline double2* matw(double* m, const hfb_natural_args* a) { return (double2*)m + (size_t)a->iq * a->ld * a->ld; }

}  // namespace
}  // namespace hfb

using namespace hfb;

extern "C" int hfb_natural_begin(hfb_ctx_t ctx, const hfb_natural_args* a, void* stream) {
  if (!ctx) return HFB_ERR_ARG;
  int r = nat_check(a);
  if (r) return r;
  NatWork w = nat_work(ctx, a->nst);
  if (!w.cm) return HFB_ERR_ALLOC;
  nat_begin_kernel<<<1, kQrThreads, 0, as_stream(stream)>>>(a->nst, a->ld, mat(a->hmatrix, a), mat(a->gapmatrix, a),
                                                            a->sp_energy + a->start, a->delstepbas, a->e0bas, w);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_natural_step(hfb_ctx_t ctx, const hfb_natural_args* a, int last, void* stream) {
  if (!ctx) return HFB_ERR_ARG;
  int r = nat_check(a);
  if (r) return r;
  NatWork w = nat_work(ctx, a->nst);
  if (!w.cm) return HFB_ERR_ALLOC;
  cudaStream_t st = as_stream(stream);
  const int n = a->nst, nn = n * n;
  nat_gradient_kernel<<<(nn + 255) / 256, 256, 0, st>>>(n, a->ld, mat(a->symcond, a), w);
  HFB_CHECK_LAUNCH();
  nat_qr_kernel<<<1, kQrThreads, 0, st>>>(n, w.cm, w.tau);
  HFB_CHECK_LAUNCH();
  if ((r = zgemm_small_one(n, n, 0, 0, w.h0, w.cm, w.hcm, st))) return r;     // h cm
  if ((r = zgemm_small_one(n, n, 1, 0, w.cm, w.hcm, w.ht, st))) return r;     // cm^H h cm
  if ((r = zgemm_small_one(n, n, 0, 0, w.g0, w.cm, w.gcm, st))) return r;     // gap cm
  if ((r = zgemm_small_one(n, n, 1, 0, w.cm, w.gcm, w.gt, st))) return r;     // cm^H gap cm
  if (a->ipair || last) {
    nat_diag_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, a->ipair, w, a->pairwg + a->start, a->sp_energy + a->start,
                                                     a->deltaf ? a->deltaf + a->start : nullptr);
    HFB_CHECK_LAUNCH();
  }
  return HFB_OK;
}

extern "C" int hfb_natural_symcond(hfb_ctx_t ctx, const hfb_natural_args* a, void* stream) {
  if (!ctx) return HFB_ERR_ARG;
  int r = nat_check(a);
  if (r) return r;
  NatWork w = nat_work(ctx, a->nst);
  if (!w.cm) return HFB_ERR_ALLOC;
  cudaStream_t st = as_stream(stream);
  const int n = a->nst, nn = n * n, s = a->start;
  nat_lambda_kernel<<<(nn + 255) / 256, 256, 0, st>>>(n, w, a->wocc + s, a->wguv + s, a->pairwg + s, a->wstates + s,
                                                      w.lam, n);
  HFB_CHECK_LAUNCH();
  if ((r = zgemm_small_one(n, n, 0, 0, w.cm, w.lam, w.cml, st))) return r;    // cm lambda
  nat_symcond_kernel<<<(nn + 255) / 256, 256, 0, st>>>(n, a->ld, w, a->wocc + s, a->wguv + s, a->pairwg + s,
                                                       a->wstates + s, matw(a->symcond, a));
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_natural_end(hfb_ctx_t ctx, int prec, const hfb_natural_args* a, const void* psi, void* psi_out,
                               void* lagrange, void* stream) {
  if (!ctx || !psi || !psi_out || !lagrange || psi_out == psi || lagrange == psi) return HFB_ERR_ARG;
  int r = nat_check(a);
  if (r) return r;
  NatWork w = nat_work(ctx, a->nst);
  if (!w.cm) return HFB_ERR_ALLOC;
  cudaStream_t st = as_stream(stream);
  const int n = a->nst, nn = n * n, s = a->start;
  // [psi cm | psi (cm htran)] for the block's states
  if ((r = zgemm_small_one(n, n, 0, 0, w.cm, w.ht, w.cml, st))) return r;
  if ((r = rotate_launch(ctx, prec, s, n, psi, w.cm, w.cml, n, psi_out, lagrange, st, -1))) return r;
  nat_store_kernel<<<(nn + 255) / 256, 256, 0, st>>>(n, a->ld, w.ht, matw(a->hmatrix, a));
  HFB_CHECK_LAUNCH();
  nat_store_kernel<<<(nn + 255) / 256, 256, 0, st>>>(n, a->ld, w.gt, matw(a->gapmatrix, a));
  HFB_CHECK_LAUNCH();
  nat_lambda_kernel<<<(nn + 255) / 256, 256, 0, st>>>(n, w, a->wocc + s, a->wguv + s, a->pairwg + s, a->wstates + s,
                                                      matw(a->lambda_save, a), a->ld);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
