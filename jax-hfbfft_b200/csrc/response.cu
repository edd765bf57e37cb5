// State-vector algebra for the linear-response (implicit adjoint) solver:
// sets of nsp two-spinors laid out like psi ([nsp][2][n^3] complex), FP64 or
// FP32.  Reductions are FP64 with a fixed order (per-block partial sums,
// then one block adds them in block order), so results do not depend on
// scheduling.
#include <math.h>
#include "hfb_ctx.cuh"

namespace hfb {
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsBlocks = 592;   // 4 x 148 SMs

template <class Z>
__global__ void rs_dot_kernel(size_t tot, const Z* __restrict__ a, const Z* __restrict__ b, double* part) {
  __shared__ double red[kRsThreads / 32];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)kRsThreads + threadIdx.x; i < tot; i += (size_t)gridDim.x * kRsThreads) {
    const Z x = a[i], y = b[i];
    s += (double)x.x * (double)y.x + (double)x.y * (double)y.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kRsThreads / 32; ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

__global__ void rs_sum_kernel(int n, const double* __restrict__ part, double scale, double* out) {
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < n; ++i) t += part[i];
    *out = scale * t;
  }
}

template <class Z>
__global__ void rs_axpby_kernel(size_t tot, double a, const Z* __restrict__ x, double b, Z* y) {
  for (size_t i = blockIdx.x * (size_t)kRsThreads + threadIdx.x; i < tot; i += (size_t)gridDim.x * kRsThreads) {
    const Z u = x[i], v = y[i];
    Z r;
    r.x = a * u.x + b * v.x;
    r.y = a * u.y + b * v.y;
    y[i] = r;
  }
}

template <class Z>
__global__ void rs_field_kernel(size_t tot, size_t n3, const double* __restrict__ f, const Z* __restrict__ x, Z* y) {
  for (size_t i = blockIdx.x * (size_t)kRsThreads + threadIdx.x; i < tot; i += (size_t)gridDim.x * kRsThreads) {
    const double w = f[i % n3];
    const Z u = x[i];
    Z r;
    r.x = w * u.x;
    r.y = w * u.y;
    y[i] = r;
  }
}

// v[j] -= sum_i psi[i] C[i][j] over the K = 2 n^3 complex points (C complex
// [np][nv], FP64)
template <class Z>
__global__ void rs_project_kernel(size_t K, int np, int nv, const Z* __restrict__ psi, const double2* __restrict__ C,
                                  Z* v) {
  extern __shared__ double2 cs[];
  for (int e = threadIdx.x; e < np * nv; e += blockDim.x) cs[e] = C[e];
  __syncthreads();
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < K; k += (size_t)gridDim.x * blockDim.x) {
    for (int j = 0; j < nv; ++j) {
      double re = 0.0, im = 0.0;
      for (int i = 0; i < np; ++i) {
        const Z p = psi[(size_t)i * K + k];
        const double2 c = cs[i * nv + j];
        re += (double)p.x * c.x - (double)p.y * c.y;
        im += (double)p.x * c.y + (double)p.y * c.x;
      }
      Z r = v[(size_t)j * K + k];
      r.x -= re;
      r.y -= im;
      v[(size_t)j * K + k] = r;
    }
  }
}

// C[i][j] = wxyz <psi_i | v_j>, one block per (i, j), fixed-order sums
template <class Z>
__global__ void rs_overlap_kernel(size_t K, int nv, const Z* __restrict__ psi, const Z* __restrict__ v, double wxyz,
                                  double2* C) {
  __shared__ double red[2][kRsThreads / 32];
  const int i = blockIdx.y, j = blockIdx.x;
  const Z* a = psi + (size_t)i * K;
  const Z* b = v + (size_t)j * K;
  double re = 0.0, im = 0.0;
  for (size_t k = threadIdx.x; k < K; k += kRsThreads) {
    const Z x = a[k], y = b[k];
    re += (double)x.x * (double)y.x + (double)x.y * (double)y.y;
    im += (double)x.x * (double)y.y - (double)x.y * (double)y.x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = re;
    red[1][threadIdx.x >> 5] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    for (int w = 0; w < kRsThreads / 32; ++w) {
      x += red[0][w];
      y += red[1][w];
    }
    C[(size_t)i * nv + j] = make_double2(wxyz * x, wxyz * y);
  }
}

template <class Z>
__global__ void rs_axpby_diag_kernel(size_t tot, size_t per, const double* __restrict__ a, const Z* __restrict__ x,
                                     double b, Z* y) {
  for (size_t i = blockIdx.x * (size_t)kRsThreads + threadIdx.x; i < tot; i += (size_t)gridDim.x * kRsThreads) {
    const double w = a[i / per];
    const Z u = x[i], v = y[i];
    Z r;
    r.x = w * u.x + b * v.x;
    r.y = w * u.y + b * v.y;
    y[i] = r;
  }
}

// field = scale (|r - c|^2 - r0^2) on the centred grid x_i = (i - (n-1)/2) d
__global__ void rs_rms_field_kernel(int n, double dx, double dy, double dz, double cx, double cy, double cz, double r0,
                                    double scale, double* f) {
  const size_t n3 = (size_t)n * n * n;
  for (size_t g = blockIdx.x * (size_t)kRsThreads + threadIdx.x; g < n3; g += (size_t)gridDim.x * kRsThreads) {
    const int ix = (int)(g / ((size_t)n * n)), iy = (int)((g / n) % n), iz = (int)(g % n);
    const double x = (ix - 0.5 * (n - 1)) * dx - cx, y = (iy - 0.5 * (n - 1)) * dy - cy,
                 z = (iz - 0.5 * (n - 1)) * dz - cz;
    f[g] = scale * (x * x + y * y + z * z - r0 * r0);
  }
}

unsigned rs_grid(size_t tot) {
  const size_t b = (tot + kRsThreads - 1) / kRsThreads;
  return (unsigned)(b < (size_t)kRsBlocks ? (b > 0 ? b : 1) : kRsBlocks);
}

}  // namespace
}  // namespace hfb

using namespace hfb;

extern "C" int hfb_state_dot(hfb_ctx_t ctx, int prec, int nsp, const void* a, const void* b, double* out,
                             void* stream) {
  if (!ctx || !a || !b || !out || nsp < 0) return HFB_ERR_ARG;
  const size_t tot = (size_t)nsp * 2 * ctx->n * ctx->n * ctx->n;
  const unsigned g = rs_grid(tot);
  double* part = (double*)scratch(ctx, hfb_ctx_s::S_RESP, sizeof(double) * kRsBlocks);
  if (!part) return HFB_ERR_ALLOC;
  cudaStream_t st = as_stream(stream);
  if (prec == HFB_F64)
    rs_dot_kernel<double2><<<g, kRsThreads, 0, st>>>(tot, (const double2*)a, (const double2*)b, part);
  else
    rs_dot_kernel<float2><<<g, kRsThreads, 0, st>>>(tot, (const float2*)a, (const float2*)b, part);
  HFB_CHECK_LAUNCH();
  rs_sum_kernel<<<1, 32, 0, st>>>((int)g, part, ctx->wxyz, out);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_state_axpby(hfb_ctx_t ctx, int prec, int nsp, double a, const void* x, double b, void* y,
                               void* stream) {
  if (!ctx || !x || !y || nsp < 0) return HFB_ERR_ARG;
  const size_t tot = (size_t)nsp * 2 * ctx->n * ctx->n * ctx->n;
  cudaStream_t st = as_stream(stream);
  if (prec == HFB_F64)
    rs_axpby_kernel<double2><<<rs_grid(tot), kRsThreads, 0, st>>>(tot, a, (const double2*)x, b, (double2*)y);
  else
    rs_axpby_kernel<float2><<<rs_grid(tot), kRsThreads, 0, st>>>(tot, a, (const float2*)x, b, (float2*)y);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_state_mul_field(hfb_ctx_t ctx, int prec, int nsp, const double* field, const void* x, void* y,
                                   void* stream) {
  if (!ctx || !field || !x || !y || nsp < 0) return HFB_ERR_ARG;
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n, tot = (size_t)nsp * 2 * n3;
  cudaStream_t st = as_stream(stream);
  if (prec == HFB_F64)
    rs_field_kernel<double2><<<rs_grid(tot), kRsThreads, 0, st>>>(tot, n3, field, (const double2*)x, (double2*)y);
  else
    rs_field_kernel<float2><<<rs_grid(tot), kRsThreads, 0, st>>>(tot, n3, field, (const float2*)x, (float2*)y);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_state_project(hfb_ctx_t ctx, int prec, int np, const void* psi, int nv, void* v, void* stream) {
  if (!ctx || !psi || !v || np <= 0 || nv <= 0 || (size_t)np * nv * sizeof(double2) > 160 * 1024) return HFB_ERR_ARG;
  const size_t K = (size_t)2 * ctx->n * ctx->n * ctx->n;
  double2* C = (double2*)scratch(ctx, hfb_ctx_s::S_RESP2, sizeof(double2) * (size_t)np * nv);
  if (!C) return HFB_ERR_ALLOC;
  cudaStream_t st = as_stream(stream);
  const size_t smem = sizeof(double2) * (size_t)np * nv;
  const unsigned g = (unsigned)((K + 255) / 256);
  if (prec == HFB_F64) {
    rs_overlap_kernel<double2><<<dim3(nv, np), kRsThreads, 0, st>>>(K, nv, (const double2*)psi, (const double2*)v,
                                                                    ctx->wxyz, C);
    HFB_CHECK_LAUNCH();
    allow_max_dynamic_smem(rs_project_kernel<double2>);
    rs_project_kernel<double2><<<g, 256, smem, st>>>(K, np, nv, (const double2*)psi, C, (double2*)v);
  } else {
    rs_overlap_kernel<float2><<<dim3(nv, np), kRsThreads, 0, st>>>(K, nv, (const float2*)psi, (const float2*)v,
                                                                   ctx->wxyz, C);
    HFB_CHECK_LAUNCH();
    allow_max_dynamic_smem(rs_project_kernel<float2>);
    rs_project_kernel<float2><<<g, 256, smem, st>>>(K, np, nv, (const float2*)psi, C, (float2*)v);
  }
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_state_axpby_diag(hfb_ctx_t ctx, int prec, int nsp, const double* a, const void* x, double b,
                                    void* y, void* stream) {
  if (!ctx || !a || !x || !y || nsp < 0) return HFB_ERR_ARG;
  const size_t per = (size_t)2 * ctx->n * ctx->n * ctx->n, tot = (size_t)nsp * per;
  cudaStream_t st = as_stream(stream);
  if (prec == HFB_F64)
    rs_axpby_diag_kernel<double2><<<rs_grid(tot), kRsThreads, 0, st>>>(tot, per, a, (const double2*)x, b,
                                                                       (double2*)y);
  else
    rs_axpby_diag_kernel<float2><<<rs_grid(tot), kRsThreads, 0, st>>>(tot, per, a, (const float2*)x, b, (float2*)y);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}

extern "C" int hfb_rms_field(hfb_ctx_t ctx, const double* cm, double r0, double scale, double* field, void* stream) {
  if (!ctx || !cm || !field) return HFB_ERR_ARG;
  const size_t n3 = (size_t)ctx->n * ctx->n * ctx->n;
  rs_rms_field_kernel<<<rs_grid(n3), kRsThreads, 0, as_stream(stream)>>>(ctx->n, ctx->d[0], ctx->d[1], ctx->d[2],
                                                                         cm[0], cm[1], cm[2], r0, scale, field);
  HFB_CHECK_LAUNCH();
  return HFB_OK;
}
