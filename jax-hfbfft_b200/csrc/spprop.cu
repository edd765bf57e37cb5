// Single-particle orbital angular momentum, spin and parity (sp_properties,
// inout.py:64-150), FP64 accumulation for FP64 or FP32 states.
//
// With x relative to the centre of mass cm and the spectral first
// derivative D_d (cderv01, Nyquist zeroed; the dense matrix der1[d]):
//   L_x = dV sum Im(psi^* (y d_z - z d_y) psi), and cyclic,
//   S   = dV/2 sum psi^+ sigma psi,
//   P   = dV sum Re(psi^*(r) psi(-r)).
// Orbital: one block per (plane, axis d, state) holds der1[d] and a plane of
// lines along d of both components in shared memory, forms the derivative
// at every point of the plane and accumulates S_d[c] = sum c Im(psi^* d_d
// psi) for the two coordinates c other than d; a final kernel combines
// L_x = S_z[y] - S_y[z], L_y = S_x[z] - S_z[x], L_z = S_y[x] - S_x[y].
// Spin and parity are pointwise sums over chunks of the grid.  All block
// and final sums run in a fixed order.
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {

namespace {

constexpr int kSpThreads = 256;
constexpr int kSpChunk = kSpThreads * 16;   // grid points per spin / parity block

__device__ double sp_block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kSpThreads / 32; ++w) t += red[w];
  return t;
}

template <class R>
__device__ __forceinline__ double2 ld_d2(const cplx<R>* p, size_t i) {
  const cplx<R> v = p[i];
  return make_double2((double)v.x, (double)v.y);
}

// Plane p of lines along axis d (d = 0: y = p, lines z; d = 1: x = p,
// lines z; d = 2: x = p, lines y); point j along the line.
__device__ __forceinline__ size_t sp_point(int n, int d, int p, int line, int j) {
  const size_t nn = (size_t)n;
  if (d == 0) return (size_t)j * nn * nn + (size_t)p * nn + line;
  if (d == 1) return (size_t)p * nn * nn + (size_t)j * nn + line;
  return (size_t)p * nn * nn + (size_t)line * nn + j;
}

template <class R>
__global__ void __launch_bounds__(kSpThreads) sp_orbital_kernel(int n, const cplx<R>* __restrict__ psi,
                                                                const double* __restrict__ d0,
                                                                const double* __restrict__ d1,
                                                                const double* __restrict__ d2, double h0, double h1,
                                                                double h2, double cm0, double cm1, double cm2,
                                                                double* part) {
  extern __shared__ __align__(16) unsigned char sp_smem[];
  __shared__ double red[kSpThreads / 32];
  const int p = blockIdx.x, d = blockIdx.y, s = blockIdx.z;
  const size_t n3 = (size_t)n * n * n;
  double* D = reinterpret_cast<double*>(sp_smem);
  double2* pl = reinterpret_cast<double2*>(D + (size_t)n * n);   // [c][line][j]
  const double* Dg = d == 0 ? d0 : (d == 1 ? d1 : d2);
  for (int e = threadIdx.x; e < n * n; e += kSpThreads) D[e] = Dg[e];
  const cplx<R>* ps = psi + (size_t)s * 2 * n3;
  for (int e = threadIdx.x; e < 2 * n * n; e += kSpThreads) {
    const int c = e / (n * n), r = e - c * n * n, line = r / n, j = r - line * n;
    pl[e] = ld_d2<R>(ps + (size_t)c * n3, sp_point(n, d, p, line, j));
  }
  __syncthreads();
  const double h[3] = {h0, h1, h2}, cm[3] = {cm0, cm1, cm2};
  // the two coordinates other than d, in increasing axis order
  const int ca = d == 0 ? 1 : 0, cb = d == 2 ? 1 : 2;
  double sa = 0.0, sb = 0.0;
  for (int e = threadIdx.x; e < 2 * n * n; e += kSpThreads) {
    const int c = e / (n * n), r = e - c * n * n, line = r / n, j = r - line * n;
    const double2* row = pl + (size_t)(c * n + line) * n;
    const double* Dj = D + (size_t)j * n;
    double dr = 0.0, di = 0.0;
    for (int l = 0; l < n; ++l) {
      dr += Dj[l] * row[l].x;
      di += Dj[l] * row[l].y;
    }
    const double2 v = row[j];
    const double im = v.x * di - v.y * dr;   // Im(psi^* d psi)
    int idx[3];
    idx[d] = j;
    if (d == 0) { idx[1] = p; idx[2] = line; }
    else if (d == 1) { idx[0] = p; idx[2] = line; }
    else { idx[0] = p; idx[1] = line; }
    const double xa = (idx[ca] - (n - 1) / 2.0) * h[ca] - cm[ca];
    const double xb = (idx[cb] - (n - 1) / 2.0) * h[cb] - cm[cb];
    sa += xa * im;
    sb += xb * im;
  }
  sa = sp_block_sum(sa, red);
  sb = sp_block_sum(sb, red);
  if (threadIdx.x == 0) {
    double* o = part + (((size_t)s * 3 + d) * n + p) * 2;
    o[0] = sa;
    o[1] = sb;
  }
}

template <class R>
__global__ void __launch_bounds__(kSpThreads) sp_spin_kernel(size_t n3, const cplx<R>* __restrict__ psi,
                                                             double* part) {
  __shared__ double red[kSpThreads / 32];
  const int s = blockIdx.y;
  const cplx<R>* a = psi + (size_t)s * 2 * n3;
  const cplx<R>* b = a + n3;
  double sx = 0, sy = 0, sz = 0, pr = 0;
  const size_t g0 = (size_t)blockIdx.x * kSpChunk;
  for (size_t g = g0 + threadIdx.x; g < g0 + kSpChunk && g < n3; g += kSpThreads) {
    const double2 u = ld_d2<R>(a, g), v = ld_d2<R>(b, g);
    const double2 uf = ld_d2<R>(a, n3 - 1 - g), vf = ld_d2<R>(b, n3 - 1 - g);
    sx += u.x * v.x + u.y * v.y;               // Re(a^* b)
    sy += u.x * v.y - u.y * v.x;               // Im(a^* b)
    sz += 0.5 * ((u.x * u.x + u.y * u.y) - (v.x * v.x + v.y * v.y));
    pr += u.x * uf.x + u.y * uf.y + v.x * vf.x + v.y * vf.y;
  }
  sx = sp_block_sum(sx, red);
  sy = sp_block_sum(sy, red);
  sz = sp_block_sum(sz, red);
  pr = sp_block_sum(pr, red);
  if (threadIdx.x == 0) {
    double* o = part + ((size_t)s * gridDim.x + blockIdx.x) * 4;
    o[0] = sx;
    o[1] = sy;
    o[2] = sz;
    o[3] = pr;
  }
}

__global__ void sp_final_kernel(int nst, int n, int nchunk, const double* porb, const double* pspin, double wxyz,
                                double* orbital, double* spin, double* parity) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nst) return;
  // S_d[k]: k = 0 the lower, k = 1 the higher of the two other axes
  double S[3][2];
  for (int d = 0; d < 3; ++d) {
    double a = 0.0, b = 0.0;
    for (int p = 0; p < n; ++p) {
      a += porb[(((size_t)s * 3 + d) * n + p) * 2 + 0];
      b += porb[(((size_t)s * 3 + d) * n + p) * 2 + 1];
    }
    S[d][0] = a;
    S[d][1] = b;
  }
  // S_x[y] = S[0][0], S_x[z] = S[0][1]; S_y[x] = S[1][0], S_y[z] = S[1][1];
  // S_z[x] = S[2][0], S_z[y] = S[2][1]
  if (orbital) {
    orbital[(size_t)s * 3 + 0] = wxyz * (S[2][1] - S[1][1]);
    orbital[(size_t)s * 3 + 1] = wxyz * (S[0][1] - S[2][0]);
    orbital[(size_t)s * 3 + 2] = wxyz * (S[1][0] - S[0][0]);
  }
  double t[4] = {0, 0, 0, 0};
  for (int c = 0; c < nchunk; ++c)
    for (int k = 0; k < 4; ++k) t[k] += pspin[((size_t)s * nchunk + c) * 4 + k];
  if (spin) {
    spin[(size_t)s * 3 + 0] = wxyz * t[0];
    spin[(size_t)s * 3 + 1] = wxyz * t[1];
    spin[(size_t)s * 3 + 2] = wxyz * t[2];
  }
  if (parity) parity[s] = wxyz * t[3];
}

template <class R>
int sp_launch(hfb_ctx_s* c, int nst, const void* psi, const double* cm, double* orbital, double* spin,
              double* parity, cudaStream_t st) {
  const int n = c->n;
  const size_t n3 = (size_t)n * n * n;
  const int nchunk = (int)((n3 + kSpChunk - 1) / kSpChunk);
  const size_t norb = (size_t)nst * 3 * n * 2, nsp = (size_t)nst * nchunk * 4;
  double* part = (double*)scratch(c, hfb_ctx_s::S_PART, sizeof(double) * (norb + nsp));
  if (!part) return HFB_ERR_ALLOC;
  const double cmv[3] = {cm ? cm[0] : 0.0, cm ? cm[1] : 0.0, cm ? cm[2] : 0.0};
  const size_t smem = sizeof(double) * (size_t)n * n + sizeof(double2) * 2 * (size_t)n * n;
  allow_max_dynamic_smem(sp_orbital_kernel<R>);
  sp_orbital_kernel<R><<<dim3(n, 3, nst), kSpThreads, smem, st>>>(n, (const cplx<R>*)psi, c->der1[0], c->der1[1],
                                                                   c->der1[2], c->d[0], c->d[1], c->d[2], cmv[0],
                                                                   cmv[1], cmv[2], part);
  HFB_CHECK_LAUNCH();
  sp_spin_kernel<R><<<dim3(nchunk, nst), kSpThreads, 0, st>>>(n3, (const cplx<R>*)psi, part + norb);
  HFB_CHECK_LAUNCH();
  sp_final_kernel<<<(nst + 127) / 128, 128, 0, st>>>(nst, n, nchunk, part, part + norb, c->wxyz, orbital, spin,
                                                      parity);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

}  // namespace

}  // namespace hfb

using namespace hfb;

extern "C" int hfb_sp_properties(hfb_ctx_t ctx, int prec, int nst, const void* psi, const double* cm,
                                 double* orbital, double* spin, double* parity, void* stream) {
  if (!ctx || !psi || nst <= 0 || (!orbital && !spin && !parity)) return HFB_ERR_ARG;
  if (prec != HFB_F64 && prec != HFB_F32) return HFB_ERR_ARG;
  if (ctx->n > 64) return HFB_ERR_UNSUPPORTED_GRID;
  cudaStream_t st = as_stream(stream);
  return prec == HFB_F64 ? sp_launch<double>(ctx, nst, psi, cm, orbital, spin, parity, st)
                         : sp_launch<float>(ctx, nst, psi, cm, orbital, spin, parity, st);
}
